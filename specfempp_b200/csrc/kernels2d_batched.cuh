// Batched-shot kernels of the 2D elastic time step (FP32).
//
// S independent shots (different sources, same mesh and model) advance in one
// launch per colour.  Fields are [point][component][shot], so the 32 lanes of
// a warp are 32 shots of one GLL point: the index, Jacobian and material
// loads of a point are warp-uniform (one transaction serves all shots) and
// the field loads are 128-byte coalesced.  A block is one element: 25 warps,
// one per GLL point, over a tile of up to 32 shots.  The Lagrange
// coefficients a warp needs are warp-uniform too and come from constant
// memory.
//
// Per shot the arithmetic is the single-shot element kernel's, operation for
// operation (same explicit FMAs in the contractions, everything else rounded
// separately), so a batched run gives the same bits as S separate runs.
// Reference: as kernels2d.cuh (compute_stiffness_interaction.tpp:140-247,
// stacey.tpp:50-80, compute_source_interaction.tpp:17-104, newmark.tpp:10-128,
// compute_seismogram.tpp:19-171).
#pragma once

#include "kernels2d.cuh"

namespace sfg {
namespace dev {

__constant__ float c_hp[NP];    // hp[i*5+j] = l'_j(xi_i)
__constant__ float c_hpw[NP];   // hp[l*5+i] * w[l]
__constant__ float c_w[NG];

struct BatchArgs {
  const int *__restrict__ ibool;
  const float *__restrict__ xix, *__restrict__ xiz, *__restrict__ gax, *__restrict__ gaz,
      *__restrict__ jac, *__restrict__ prop0, *__restrict__ prop1;
  const int *__restrict__ bc_slot;
  const float *__restrict__ bc_w, *__restrict__ bc_nx, *__restrict__ bc_nz, *__restrict__ bc_j1,
      *__restrict__ bc_imp0, *__restrict__ bc_imp1;
  const int *__restrict__ src_head, *__restrict__ src_next, *__restrict__ src_shot;
  const float *__restrict__ src_arr;   // [nsrc][2][25]
  const float *__restrict__ stf;       // [nstep][nsrc]
  int nsrc, nstep;
  const int *__restrict__ step;
  const float *__restrict__ u, *__restrict__ v;   // [nglob][NC][S]
  float *__restrict__ accum;
  float *__restrict__ r;               // owner-computes: [slot[element*25 + point]][NC][S]
  const int *__restrict__ slot;
  int e0;                              // first element of the colour
  int S;                               // shots
  int nspec_b;                         // elements (persistent kernel)
};

// grid: (elements of the colour, shot tiles of 32); block: 25 warps x 32 lanes.
// LOCAL: write the element's contribution to its own slot of A.r instead of
// adding it into the accumulator (then e0 = 0 and the grid covers all elements).
template <int NC, bool LOCAL>
__global__ void __launch_bounds__(NP * 32) k_stiffness_batched(BatchArgs A) {
  __shared__ float su[NC][NP][32];
  __shared__ float sF[NC][2][NP][32];
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int shot = blockIdx.y * 32 + lane;
  const bool act = shot < A.S;
  const int e = A.e0 + blockIdx.x;
  const size_t p = size_t(e) * NP + q;
  const int iz = q / NG, ix = q - iz * NG;
  const int g = __ldg(A.ibool + p);
  const float xix = __ldg(A.xix + p), xiz = __ldg(A.xiz + p), gax = __ldg(A.gax + p),
              gaz = __ldg(A.gaz + p), jac = __ldg(A.jac + p);
  const float c0 = __ldg(A.prop0 + p), mu = __ldg(A.prop1 + p);
  float uu[NC], acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const size_t k = (size_t(g) * NC + c) * A.S + shot;
    uu[c] = act ? A.u[k] : 0.f;
    acc[c] = (act && !LOCAL) ? A.accum[k] : 0.f;
    su[c][q][lane] = uu[c];
  }
  const int bs = __ldg(A.bc_slot + e);
  const int src = __ldg(A.src_head + e);
  __syncthreads();
  float dxi[NC], dga[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    dxi[c] = 0.f;
    dga[c] = 0.f;
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      dxi[c] = fmaf(c_hp[ix * NG + l], su[c][iz * NG + l][lane], dxi[c]);
      dga[c] = fmaf(c_hp[iz * NG + l], su[c][l * NG + ix][lane], dga[c]);
    }
  }
  float Sx[NC], Sz[NC];
  if (NC == 2) {
    const float du00 = xix * dxi[0] + gax * dga[0], du01 = xiz * dxi[0] + gaz * dga[0];
    const float du10 = xix * dxi[NC - 1] + gax * dga[NC - 1];
    const float du11 = xiz * dxi[NC - 1] + gaz * dga[NC - 1];
    const float lam = c0 - 2.f * mu;
    const float sxx = c0 * du00 + lam * du11;
    const float szz = c0 * du11 + lam * du00;
    const float sxz = mu * (du01 + du10);
    Sx[0] = sxx; Sz[0] = sxz; Sx[NC - 1] = sxz; Sz[NC - 1] = szz;
  } else {
    Sx[0] = mu * (xix * dxi[0] + gax * dga[0]);
    Sz[0] = mu * (xiz * dxi[0] + gaz * dga[0]);
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    sF[c][0][q][lane] = jac * (Sx[c] * xix + Sz[c] * xiz);
    sF[c][1][q][lane] = jac * (Sx[c] * gax + Sz[c] * gaz);
  }
  __syncthreads();
  if (!act) return;
  float a[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    float t1 = 0.f, t2 = 0.f;
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      t1 = fmaf(sF[c][0][iz * NG + l][lane], c_hpw[l * NG + ix], t1);
      t2 = fmaf(sF[c][1][l * NG + ix][lane], c_hpw[l * NG + iz], t2);
    }
    a[c] = -(c_w[iz] * t1 + c_w[ix] * t2);
  }
  if (bs >= 0) {
    const size_t k = size_t(bs) * NP + q;
    const float wq = A.bc_w[k];
    if (wq != 0.f) {
      const float nx = A.bc_nx[k], nz = A.bc_nz[k], j1 = A.bc_j1[k];
      if (NC == 2) {
        const float vx = A.v[(size_t(g) * NC) * A.S + shot];
        const float vz = A.v[(size_t(g) * NC + NC - 1) * A.S + shot];
        const float rvp = A.bc_imp0[k], rvs = A.bc_imp1[k];
        const float vn = vx * nx + vz * nz;
        const float fx = ((vn * nx / (j1 * j1)) * (rvp - rvs)) + vx * rvs;
        const float fz = ((vn * nz / (j1 * j1)) * (rvp - rvs)) + vz * rvs;
        a[0] += -1.f * fx * j1 * wq;
        a[NC - 1] += -1.f * fz * j1 * wq;
      } else {
        a[0] += -1.f * (wq * j1) * A.bc_imp1[k] * A.v[size_t(g) * A.S + shot];
      }
    }
  }
  if (src >= 0) {
    const int step = *A.step;
    for (int s = src; s >= 0; s = A.src_next[s]) {
      if (A.src_shot[s] != shot) continue;
      const float f = step < A.nstep ? A.stf[size_t(step) * A.nsrc + s] : 0.f;
#pragma unroll
      for (int c = 0; c < NC; ++c) a[c] += f * A.src_arr[(size_t(s) * 2 + c) * NP + q];
    }
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (LOCAL) A.r[(size_t(__ldg(A.slot + p)) * NC + c) * A.S + shot] = a[c];
    else A.accum[(size_t(g) * NC + c) * A.S + shot] = acc[c] + a[c];
  }
}

// Owner-computes update for [point][NC][S] fields: each (point, comp, shot)
// gathers its element contributions in colour order (bitwise the colour
// passes' sum), then M^-1, corrector and optional predictor.
__global__ void __launch_bounds__(256) k_update_batched_gather(UpdateArgs A, int S, int NC) {
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += stride) {
    const int s = i % S;
    const int gc = i / S;
    const int g = gc / NC, c = gc - g * NC;
    float acc = 0.f;
    const int k1 = A.inv_start[g + 1];
    for (int k = A.inv_start[g]; k < k1; ++k)
      acc = acc + A.r[(size_t(k) * NC + c) * S + s];
    const float a = __fmul_rn(acc, A.minv[gc]);
    float vv = newmark_correct(A.v[i], a, A.dt2);
    float uu = A.u[i];
    if (A.predict) newmark_predict(uu, vv, a, A.dt, A.dt2, A.dtsq2);
    A.u[i] = uu;
    A.v[i] = vv;
    if (A.a_store) A.a_store[i] = a;
    bad |= !isfinite(uu);
  }
  if (bad) *A.flag = 1;
  if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) *A.step += 1;
}

// ---------------------------------------------------------------------------
// Quad-shot form (S a multiple of 4): each thread carries 4 consecutive shots
// of one GLL point as a float4, so it has four times the field bytes in
// flight of the one-shot-per-lane kernel.  Block: one element, 25 points x T
// threads (T = shots in the tile / 4, at most 8); grid: (elements, shot tiles).
// Per shot the operations are those of k_stiffness_batched.
template <int NC, bool LOCAL>
__global__ void __launch_bounds__(NP * 8) k_stiffness_batched4(BatchArgs A, int T) {
  __shared__ float4 su[NC][NP][8];
  __shared__ float4 sF[NC][2][NP][8];
  const int q = threadIdx.x / T, j = threadIdx.x - q * T;
  const int shot0 = (blockIdx.y * T + j) * 4;
  const bool act = shot0 < A.S;
  const int e = A.e0 + blockIdx.x;
  const size_t p = size_t(e) * NP + q;
  const int iz = q / NG, ix = q - iz * NG;
  const int g = __ldg(A.ibool + p);
  const float xix = __ldg(A.xix + p), xiz = __ldg(A.xiz + p), gax = __ldg(A.gax + p),
              gaz = __ldg(A.gaz + p), jac = __ldg(A.jac + p);
  const float c0 = __ldg(A.prop0 + p), mu = __ldg(A.prop1 + p);
  float4 acc4[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const size_t k = (size_t(g) * NC + c) * A.S + shot0;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    su[c][q][j] = act ? *reinterpret_cast<const float4 *>(A.u + k) : z;
    acc4[c] = (act && !LOCAL) ? *reinterpret_cast<const float4 *>(A.accum + k) : z;
  }
  const int bs = __ldg(A.bc_slot + e);
  const int src = __ldg(A.src_head + e);
  __syncthreads();
  float a[NC][4];
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    float dxi[NC], dga[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      dxi[c] = 0.f;
      dga[c] = 0.f;
#pragma unroll
      for (int l = 0; l < NG; ++l) {
        dxi[c] = fmaf(c_hp[ix * NG + l], (&su[c][iz * NG + l][j].x)[w], dxi[c]);
        dga[c] = fmaf(c_hp[iz * NG + l], (&su[c][l * NG + ix][j].x)[w], dga[c]);
      }
    }
    float Sx[NC], Sz[NC];
    if (NC == 2) {
      const float du00 = xix * dxi[0] + gax * dga[0], du01 = xiz * dxi[0] + gaz * dga[0];
      const float du10 = xix * dxi[NC - 1] + gax * dga[NC - 1];
      const float du11 = xiz * dxi[NC - 1] + gaz * dga[NC - 1];
      const float lam = c0 - 2.f * mu;
      const float sxx = c0 * du00 + lam * du11;
      const float szz = c0 * du11 + lam * du00;
      const float sxz = mu * (du01 + du10);
      Sx[0] = sxx; Sz[0] = sxz; Sx[NC - 1] = sxz; Sz[NC - 1] = szz;
    } else {
      Sx[0] = mu * (xix * dxi[0] + gax * dga[0]);
      Sz[0] = mu * (xiz * dxi[0] + gaz * dga[0]);
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      a[c][w] = jac * (Sx[c] * xix + Sz[c] * xiz);       // F0 for now
      (&sF[c][1][q][j].x)[w] = jac * (Sx[c] * gax + Sz[c] * gaz);
    }
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) sF[c][0][q][j] = make_float4(a[c][0], a[c][1], a[c][2], a[c][3]);
  __syncthreads();
  if (!act) return;
#pragma unroll
  for (int w = 0; w < 4; ++w) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      float t1 = 0.f, t2 = 0.f;
#pragma unroll
      for (int l = 0; l < NG; ++l) {
        t1 = fmaf((&sF[c][0][iz * NG + l][j].x)[w], c_hpw[l * NG + ix], t1);
        t2 = fmaf((&sF[c][1][l * NG + ix][j].x)[w], c_hpw[l * NG + iz], t2);
      }
      a[c][w] = -(c_w[iz] * t1 + c_w[ix] * t2);
    }
  }
  if (bs >= 0) {
    const size_t k = size_t(bs) * NP + q;
    const float wq = A.bc_w[k];
    if (wq != 0.f) {
      const float nx = A.bc_nx[k], nz = A.bc_nz[k], j1 = A.bc_j1[k];
      if (NC == 2) {
        const float4 vx4 = *reinterpret_cast<const float4 *>(A.v + (size_t(g) * NC) * A.S + shot0);
        const float4 vz4 = *reinterpret_cast<const float4 *>(A.v + (size_t(g) * NC + NC - 1) * A.S + shot0);
        const float rvp = A.bc_imp0[k], rvs = A.bc_imp1[k];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const float vx = (&vx4.x)[w], vz = (&vz4.x)[w];
          const float vn = vx * nx + vz * nz;
          const float fx = ((vn * nx / (j1 * j1)) * (rvp - rvs)) + vx * rvs;
          const float fz = ((vn * nz / (j1 * j1)) * (rvp - rvs)) + vz * rvs;
          a[0][w] += -1.f * fx * j1 * wq;
          a[NC - 1][w] += -1.f * fz * j1 * wq;
        }
      } else {
        const float4 v4 = *reinterpret_cast<const float4 *>(A.v + size_t(g) * A.S + shot0);
#pragma unroll
        for (int w = 0; w < 4; ++w) a[0][w] += -1.f * (wq * j1) * A.bc_imp1[k] * (&v4.x)[w];
      }
    }
  }
  if (src >= 0) {
    const int step = *A.step;
    for (int s = src; s >= 0; s = A.src_next[s]) {
      const int w = A.src_shot[s] - shot0;
      if (w < 0 || w > 3) continue;
      const float f = step < A.nstep ? A.stf[size_t(step) * A.nsrc + s] : 0.f;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float add = f * A.src_arr[(size_t(s) * 2 + c) * NP + q];
        // the one-shot kernel adds sources in chain order; so does this loop
        if (w == 0) a[c][0] += add;
        else if (w == 1) a[c][1] += add;
        else if (w == 2) a[c][2] += add;
        else a[c][3] += add;
      }
    }
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (LOCAL) {
      *reinterpret_cast<float4 *>(A.r + (size_t(__ldg(A.slot + p)) * NC + c) * A.S + shot0) =
          make_float4(a[c][0], a[c][1], a[c][2], a[c][3]);
    } else {
      *reinterpret_cast<float4 *>(A.accum + (size_t(g) * NC + c) * A.S + shot0) =
          make_float4(acc4[c].x + a[c][0], acc4[c].y + a[c][1], acc4[c].z + a[c][2], acc4[c].w + a[c][3]);
    }
  }
}

// Row form of k_stiffness_batched4 (owner-computes): one thread per element
// row (five points, iz fixed) and quad of shots; EB elements x 5 rows x T
// quads per block.  The xi-direction contractions of the gradient and of the
// divergence run on the row held in registers (warp-uniform coefficients);
// the gamma-direction ones read columns of the element's displacement and F1
// in shared memory.  Per shot the operations and their order are those of
// k_stiffness_batched4 (same bits).  Dynamic shared memory: EB x NC x 2 x 25
// x T float4.
template <int NC, int EB>
__global__ void __launch_bounds__(EB * NG * 8, EB <= 4 ? 3 : 2) k_stiffness_batched4r(BatchArgs A, int T) {
  extern __shared__ __align__(16) float4 dynb[];
  // the block's Jacobian and material words [EB][7][25], loaded once by all threads
  __shared__ float sgeo[EB * 7 * NP];
  const int rowq = threadIdx.x / T, j = threadIdx.x - rowq * T;
  const int le = rowq / NG, iz = rowq - le * NG;
  const int shot0 = (blockIdx.y * T + j) * 4;
  const int e = blockIdx.x * EB + le;
  const bool act = shot0 < A.S && e < A.nspec_b;
  float4 *su = dynb + size_t(le) * NC * 2 * NP * T;   // [c][25][T]
  float4 *sF1 = su + NC * NP * T;                     // [c][25][T]
  for (int i = threadIdx.x; i < EB * NP; i += blockDim.x) {
    const int ee = i / NP, q = i - ee * NP;
    const int eg = blockIdx.x * EB + ee;
    const size_t pg = size_t(eg < A.nspec_b ? eg : 0) * NP + q;
    float *d = sgeo + ee * 7 * NP + q;
    d[0] = __ldg(A.xix + pg); d[NP] = __ldg(A.xiz + pg); d[2 * NP] = __ldg(A.gax + pg);
    d[3 * NP] = __ldg(A.gaz + pg); d[4 * NP] = __ldg(A.jac + pg);
    d[5 * NP] = __ldg(A.prop0 + pg); d[6 * NP] = __ldg(A.prop1 + pg);
  }
  const size_t pe = size_t(act ? e : 0) * NP + iz * NG;
  int g[NG];
  float4 ur[NC][NG];
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) g[ix] = act ? __ldg(A.ibool + pe + ix) : 0;
#pragma unroll
  for (int ix = 0; ix < NG; ++ix)
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      ur[c][ix] = act ? *reinterpret_cast<const float4 *>(A.u + (size_t(g[ix]) * NC + c) * A.S + shot0)
                      : make_float4(0.f, 0.f, 0.f, 0.f);
      su[(c * NP + iz * NG + ix) * T + j] = ur[c][ix];
    }
  float hz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) hz[l] = c_hp[iz * NG + l];
  __syncthreads();
  // xi-direction derivatives of the row's five points, in place of the row
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    float4 dx[NG];
#pragma unroll
    for (int ix = 0; ix < NG; ++ix) {
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        float d = 0.f;
#pragma unroll
        for (int l = 0; l < NG; ++l) d = fmaf(c_hp[ix * NG + l], (&ur[c][l].x)[w], d);
        (&dx[ix].x)[w] = d;
      }
    }
#pragma unroll
    for (int ix = 0; ix < NG; ++ix) ur[c][ix] = dx[ix];
  }
  // per point: gamma-direction derivatives from the columns, stress, F; F0
  // replaces the xi derivatives in registers, F1 goes to shared memory
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    const float *gw = sgeo + le * 7 * NP + iz * NG + ix;
    const float xix = gw[0], xiz = gw[NP], gax = gw[2 * NP], gaz = gw[3 * NP], jac = gw[4 * NP];
    const float c0 = gw[5 * NP], mu = gw[6 * NP];
    float4 dg[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        float d = 0.f;
#pragma unroll
        for (int l = 0; l < NG; ++l) d = fmaf(hz[l], (&su[(c * NP + l * NG + ix) * T + j].x)[w], d);
        (&dg[c].x)[w] = d;
      }
    }
    float4 f0[NC], f1[NC];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      float dxi[NC], dga[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        dxi[c] = (&ur[c][ix].x)[w];
        dga[c] = (&dg[c].x)[w];
      }
      float Sx[NC], Sz[NC];
      if (NC == 2) {
        const float du00 = xix * dxi[0] + gax * dga[0], du01 = xiz * dxi[0] + gaz * dga[0];
        const float du10 = xix * dxi[NC - 1] + gax * dga[NC - 1];
        const float du11 = xiz * dxi[NC - 1] + gaz * dga[NC - 1];
        const float lam = c0 - 2.f * mu;
        const float sxx = c0 * du00 + lam * du11;
        const float szz = c0 * du11 + lam * du00;
        const float sxz = mu * (du01 + du10);
        Sx[0] = sxx; Sz[0] = sxz; Sx[NC - 1] = sxz; Sz[NC - 1] = szz;
      } else {
        Sx[0] = mu * (xix * dxi[0] + gax * dga[0]);
        Sz[0] = mu * (xiz * dxi[0] + gaz * dga[0]);
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        (&f0[c].x)[w] = jac * (Sx[c] * xix + Sz[c] * xiz);
        (&f1[c].x)[w] = jac * (Sx[c] * gax + Sz[c] * gaz);
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      ur[c][ix] = f0[c];
      sF1[(c * NP + iz * NG + ix) * T + j] = f1[c];
    }
  }
  const int bs = act ? __ldg(A.bc_slot + e) : -1;
  const int src = act ? __ldg(A.src_head + e) : -1;
  float wz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) wz[l] = c_hpw[l * NG + iz];
  const float wiz = c_w[iz];
  __syncthreads();
  if (!act) return;
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    const int q = iz * NG + ix;
    float a[NC][4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        float t1 = 0.f, t2 = 0.f;
#pragma unroll
        for (int l = 0; l < NG; ++l) {
          t1 = fmaf((&ur[c][l].x)[w], c_hpw[l * NG + ix], t1);
          t2 = fmaf((&sF1[(c * NP + l * NG + ix) * T + j].x)[w], wz[l], t2);
        }
        a[c][w] = -(wiz * t1 + c_w[ix] * t2);
      }
    }
    if (bs >= 0) {
      const size_t k = size_t(bs) * NP + q;
      const float wq = A.bc_w[k];
      if (wq != 0.f) {
        const float nx = A.bc_nx[k], nz = A.bc_nz[k], j1 = A.bc_j1[k];
        if (NC == 2) {
          const float4 vx4 = *reinterpret_cast<const float4 *>(A.v + (size_t(g[ix]) * NC) * A.S + shot0);
          const float4 vz4 = *reinterpret_cast<const float4 *>(A.v + (size_t(g[ix]) * NC + NC - 1) * A.S + shot0);
          const float rvp = A.bc_imp0[k], rvs = A.bc_imp1[k];
#pragma unroll
          for (int w = 0; w < 4; ++w) {
            const float vx = (&vx4.x)[w], vz = (&vz4.x)[w];
            const float vn = vx * nx + vz * nz;
            const float fx = ((vn * nx / (j1 * j1)) * (rvp - rvs)) + vx * rvs;
            const float fz = ((vn * nz / (j1 * j1)) * (rvp - rvs)) + vz * rvs;
            a[0][w] += -1.f * fx * j1 * wq;
            a[NC - 1][w] += -1.f * fz * j1 * wq;
          }
        } else {
          const float4 v4 = *reinterpret_cast<const float4 *>(A.v + size_t(g[ix]) * A.S + shot0);
#pragma unroll
          for (int w = 0; w < 4; ++w) a[0][w] += -1.f * (wq * j1) * A.bc_imp1[k] * (&v4.x)[w];
        }
      }
    }
    if (src >= 0) {
      const int step = *A.step;
      for (int s = src; s >= 0; s = A.src_next[s]) {
        const int ws = A.src_shot[s] - shot0;
        if (ws < 0 || ws > 3) continue;
        const float f = step < A.nstep ? A.stf[size_t(step) * A.nsrc + s] : 0.f;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const float add = f * A.src_arr[(size_t(s) * 2 + c) * NP + q];
          // sources in chain order, as the one-shot kernel adds them
          if (ws == 0) a[c][0] += add;
          else if (ws == 1) a[c][1] += add;
          else if (ws == 2) a[c][2] += add;
          else a[c][3] += add;
        }
      }
    }
    const int sl = __ldg(A.slot + pe + ix);
#pragma unroll
    for (int c = 0; c < NC; ++c)
      *reinterpret_cast<float4 *>(A.r + (size_t(sl) * NC + c) * A.S + shot0) =
          make_float4(a[c][0], a[c][1], a[c][2], a[c][3]);
  }
}

// Quad-shot updates (S a multiple of 4): flat float4 index over [nglob][NC][S].
__global__ void __launch_bounds__(256) k_update_batched4(UpdateArgs A, int S) {
  const int n4 = A.n >> 2;
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    const float mi = A.minv[(4 * i) / S];
    float4 ac = reinterpret_cast<const float4 *>(A.accum)[i];
    float4 uu = reinterpret_cast<float4 *>(A.u)[i];
    float4 vv = reinterpret_cast<float4 *>(A.v)[i];
    float *pa = &ac.x, *pu = &uu.x, *pv = &vv.x;
    float a[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      a[w] = __fmul_rn(pa[w], mi);
      pv[w] = newmark_correct(pv[w], a[w], A.dt2);
      if (A.predict) newmark_predict(pu[w], pv[w], a[w], A.dt, A.dt2, A.dtsq2);
      bad |= !isfinite(pu[w]);
    }
    if (A.predict) reinterpret_cast<float4 *>(A.u)[i] = uu;
    reinterpret_cast<float4 *>(A.v)[i] = vv;
    reinterpret_cast<float4 *>(A.accum)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (A.a_store) reinterpret_cast<float4 *>(A.a_store)[i] = make_float4(a[0], a[1], a[2], a[3]);
  }
  if (bad) *A.flag = 1;
  if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) *A.step += 1;
}

__global__ void __launch_bounds__(256) k_update_batched4_gather(UpdateArgs A, int S, int NC) {
  const int n4 = A.n >> 2;
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    const int s = (4 * i) % S;
    const int gc = (4 * i) / S;
    const int g = gc / NC, c = gc - g * NC;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const int k1 = A.inv_start[g + 1];
    for (int k = A.inv_start[g]; k < k1; ++k) {
      const float4 t = *reinterpret_cast<const float4 *>(A.r + (size_t(k) * NC + c) * S + s);
      acc.x = acc.x + t.x; acc.y = acc.y + t.y; acc.z = acc.z + t.z; acc.w = acc.w + t.w;
    }
    const float mi = A.minv[gc];
    float4 uu = reinterpret_cast<float4 *>(A.u)[i];
    float4 vv = reinterpret_cast<float4 *>(A.v)[i];
    float *pc = &acc.x, *pu = &uu.x, *pv = &vv.x;
    float a[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      a[w] = __fmul_rn(pc[w], mi);
      pv[w] = newmark_correct(pv[w], a[w], A.dt2);
      if (A.predict) newmark_predict(pu[w], pv[w], a[w], A.dt, A.dt2, A.dtsq2);
      bad |= !isfinite(pu[w]);
    }
    if (A.predict) reinterpret_cast<float4 *>(A.u)[i] = uu;
    reinterpret_cast<float4 *>(A.v)[i] = vv;
    if (A.a_store) reinterpret_cast<float4 *>(A.a_store)[i] = make_float4(a[0], a[1], a[2], a[3]);
  }
  if (bad) *A.flag = 1;
  if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) *A.step += 1;
}

// a = accum * M^-1 (M^-1 shared by the shots); corrector; optional fused
// predictor; accumulator clear.  Flat index i over [nglob][NC][S].
__global__ void __launch_bounds__(256) k_update_batched(UpdateArgs A, int S) {
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += stride) {
    const float a = __fmul_rn(A.accum[i], A.minv[i / S]);
    float vv = newmark_correct(A.v[i], a, A.dt2);
    float uu = A.u[i];
    if (A.predict) newmark_predict(uu, vv, a, A.dt, A.dt2, A.dtsq2);
    A.u[i] = uu;
    A.v[i] = vv;
    A.accum[i] = 0.f;
    if (A.a_store) A.a_store[i] = a;
    bad |= !isfinite(uu);
  }
  if (bad) *A.flag = 1;
  if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) *A.step += 1;
}

// One block per receiver, lanes over shots (tiles of 32): displacement,
// velocity (corrected) or acceleration interpolated with the receiver's
// Lagrange weights.  seis is [S][nsig][ntypes][nrec][2].
__global__ void __launch_bounds__(32) k_receivers_batched(RecArgs A, int S) {
  const int step = *A.step;
  if (step % A.nsb != 0) return;
  const int isig = step / A.nsb;
  if (isig >= A.nsig) return;
  const int r = A.rec_list[blockIdx.x];
  const int ce = A.rec_elem[r];
  const int NC = A.ncomp;
  for (int s0 = 0; s0 < S; s0 += 32) {
    const int shot = s0 + threadIdx.x;
    if (shot >= S) continue;
    for (int t = 0; t < A.ntypes; ++t) {
      float tr[2] = {0.f, 0.f};
      for (int c = 0; c < NC; ++c) {
        // the 25 weighted values, summed in the order of the single-shot
        // kernel's xor butterfly (lane i + lane i^o), so traces match it bitwise
        float x[32];
#pragma unroll
        for (int q = 0; q < 32; ++q) x[q] = 0.f;
        for (int q = 0; q < NP; ++q) {
          const int g = A.ibool[size_t(ce) * NP + q];
          const size_t k = (size_t(g) * NC + c) * S + shot;
          float sum = 0.f;
          if (A.cpl.inv_start) {
            for (int j = A.cpl.inv_start[g]; j < A.cpl.inv_start[g + 1]; ++j)
              sum = sum + A.cpl.r[(size_t(j) * NC + c) * S + shot];
          } else {
            sum = A.accum[k];
          }
          const float acc = __fmul_rn(sum, A.minv[size_t(g) * NC + c]);
          float val;
          switch (A.types[t]) {
            case 0: val = A.u[k]; break;
            case 1: val = newmark_correct(A.v[k], acc, A.dt2); break;
            default: val = acc; break;
          }
          x[q] = A.rec_h[size_t(r) * NP + q] * val;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
          for (int i = 0; i < o; ++i) x[i] = x[i] + x[i + o];
        tr[c] = x[0];
      }
      float *dst = A.seis + (((size_t(shot) * A.nsig + isig) * A.ntypes + t) * A.nrec_total + r) * 2;
      dst[0] = tr[0];
      dst[1] = NC > 1 ? tr[1] : 0.f;
    }
  }
}

}  // namespace dev
}  // namespace sfg
