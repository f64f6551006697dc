// Batched tile kernel in row form (S shots, S a multiple of 4; one isotropic
// elastic medium, P-SV or SH).
//
// A block is a tile of up to four elements (a 2 x 2 patch: consecutive
// groups of four in the Morton order of the element centroids), sorted by
// colour, and all the shots of a shot tile: one thread per element row (five
// points) and quad of shots, the shots of a point across the lanes of a warp
// as in k_stiffness_batched4r, whose element arithmetic this kernel repeats
// operation for operation.  The element results of the block are staged in
// shared memory; a point that only the tile's elements touch (interior) is
// then assembled in the block, its contributions summed in the tile's element
// order (the colour order: elements of one colour share no point), and
// finished there: M^-1, corrector and the next predictor.  The contributions
// at points that other tiles touch go to their owner-computes slots, and
// k_update_batched4_list finishes those points after the launch.  The sum
// order per point is that of the colour passes and of owner-computes, so the
// results are the same bits.
// Reference: include/kokkos_kernels/impl/compute_stiffness_interaction.tpp:140-247,
// include/algorithms/gradient.hpp:40-82, divergence.hpp:41-74,
// include/boundary_conditions/stacey/stacey.tpp:50-80,
// include/kokkos_kernels/impl/compute_source_interaction.tpp:17-104,
// core/specfem/timescheme/newmark.tpp:10-128.
#pragma once

#include "kernels2d_batched.cuh"

namespace sfg {
namespace dev {

constexpr int BT_E = 4;          // elements of a tile
constexpr int BT_MAXP = 81;      // points of a tile at most (9 x 9)

struct BTileArgs {
  BatchArgs B;                   // element arrays, fields, sources, slots (B.r, B.slot)
  const int *__restrict__ tel;   // [ntiles][4] compute element ids in colour order (-1: none)
  const int *__restrict__ tloc;  // [nspec][25] tile-interior index of the element point, -1 at shared points
  const int *__restrict__ tpt;   // [ntiles][81] global id of tile-interior point k (-1: none)
  const int *__restrict__ tctr;  // [ntiles][81][4] contributions of point k: le * 25 + q, colour order (-1: none)
  const float *__restrict__ minv;
  float *__restrict__ v_out;     // velocity (written), = B.v
  float *__restrict__ u_out;     // displacement (written), = B.u
  float *__restrict__ a_store;   // new acceleration (optional)
  float dt, dt2, dtsq2;
  int predict;
  int *flag;
  int ntiles;
};

template <int NC>
__global__ void __launch_bounds__(BT_E * NG * 8, 3) k_btile_row(BTileArgs P, int T) {
  extern __shared__ __align__(16) float4 dynb[];
  __shared__ float sgeo[BT_E * 7 * NP];
  const BatchArgs &A = P.B;
  const int rowq = threadIdx.x / T, j = threadIdx.x - rowq * T;
  const int le = rowq / NG, iz = rowq - le * NG;
  const int shot0 = (blockIdx.y * T + j) * 4;
  const int t = blockIdx.x;
  const int e = __ldg(P.tel + t * BT_E + le);
  const bool act = shot0 < A.S && e >= 0;
  float4 *su = dynb + size_t(le) * NC * 2 * NP * T;   // [c][25][T]; later the element results
  float4 *sF1 = su + NC * NP * T;                     // [c][25][T]
  for (int i = threadIdx.x; i < BT_E * NP; i += blockDim.x) {
    const int ee = i / NP, q = i - ee * NP;
    const int eg = __ldg(P.tel + t * BT_E + ee);
    const size_t pg = size_t(eg >= 0 ? eg : 0) * NP + q;
    float *d = sgeo + ee * 7 * NP + q;
    d[0] = __ldg(A.xix + pg); d[NP] = __ldg(A.xiz + pg); d[2 * NP] = __ldg(A.gax + pg);
    d[3 * NP] = __ldg(A.gaz + pg); d[4 * NP] = __ldg(A.jac + pg);
    d[5 * NP] = __ldg(A.prop0 + pg); d[6 * NP] = __ldg(A.prop1 + pg);
  }
  const size_t pe = size_t(e >= 0 ? e : 0) * NP + iz * NG;
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
  // divergence and epilogue; the results go to the staging (the element's
  // displacement rows are no longer read) and, at shared points, to the slots
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
    if (act && bs >= 0) {
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
    if (act && src >= 0) {
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
    if (act) {
      if (__ldg(P.tloc + pe + ix) >= 0) {
#pragma unroll
        for (int c = 0; c < NC; ++c) su[(c * NP + q) * T + j] = make_float4(a[c][0], a[c][1], a[c][2], a[c][3]);
      } else {
        const int sl = __ldg(A.slot + pe + ix);
#pragma unroll
        for (int c = 0; c < NC; ++c)
          *reinterpret_cast<float4 *>(A.r + (size_t(sl) * NC + c) * A.S + shot0) =
              make_float4(a[c][0], a[c][1], a[c][2], a[c][3]);
      }
    }
  }
  __syncthreads();
  // the tile's interior points, one thread per point and quad of shots
  const int S = A.S;
  const int nq = BT_MAXP * T;
  bool bad = false;
  for (int i = threadIdx.x; i < nq; i += blockDim.x) {
    const int k = i / T, jj = i - k * T;
    const int s0 = (blockIdx.y * T + jj) * 4;
    const int gp = __ldg(P.tpt + t * BT_MAXP + k);
    if (gp < 0 || s0 >= S) continue;
    const int4 ct = __ldg(reinterpret_cast<const int4 *>(P.tctr) + t * BT_MAXP + k);
    const int cs[4] = {ct.x, ct.y, ct.z, ct.w};
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        if (cs[m] < 0) continue;
        const int el = cs[m] / NP, qq = cs[m] - el * NP;
        const float4 x = dynb[size_t(el) * NC * 2 * NP * T + (c * NP + qq) * T + jj];
        sum = make_float4(sum.x + x.x, sum.y + x.y, sum.z + x.z, sum.w + x.w);
      }
      const size_t o = (size_t(gp) * NC + c) * S + s0;
      const float mi = P.minv[size_t(gp) * NC + c];
      float4 uu = *reinterpret_cast<const float4 *>(P.u_out + o);
      float4 vv = *reinterpret_cast<const float4 *>(P.v_out + o);
      float4 ac;
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        (&ac.x)[w] = __fmul_rn((&sum.x)[w], mi);
        (&vv.x)[w] = newmark_correct((&vv.x)[w], (&ac.x)[w], P.dt2);
        if (P.predict) newmark_predict((&uu.x)[w], (&vv.x)[w], (&ac.x)[w], P.dt, P.dt2, P.dtsq2);
        bad |= !isfinite((&uu.x)[w]);
      }
      if (P.predict) *reinterpret_cast<float4 *>(P.u_out + o) = uu;
      *reinterpret_cast<float4 *>(P.v_out + o) = vv;
      if (P.a_store) *reinterpret_cast<float4 *>(P.a_store + o) = ac;
    }
  }
  if (bad) *P.flag = 1;
}

// The points tiles share: k_update_batched4_gather over a list of points.
__global__ void __launch_bounds__(256) k_update_batched4_list(UpdateArgs A, int S, int NC, const int *pts, int npts) {
  const int per = NC * S / 4;   // quads per point
  const int n4 = npts * per;
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    const int b = i / per, rem = i - b * per;
    const int c = (4 * rem) / S, s = (4 * rem) % S;
    const int g = pts[b];
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const int k1 = A.inv_start[g + 1];
    for (int k = A.inv_start[g]; k < k1; ++k) {
      const float4 t = *reinterpret_cast<const float4 *>(A.r + (size_t(k) * NC + c) * S + s);
      acc.x = acc.x + t.x; acc.y = acc.y + t.y; acc.z = acc.z + t.z; acc.w = acc.w + t.w;
    }
    const size_t o = (size_t(g) * NC + c) * S + s;
    const float mi = A.minv[size_t(g) * NC + c];
    float4 uu = *reinterpret_cast<float4 *>(A.u + o);
    float4 vv = *reinterpret_cast<float4 *>(A.v + o);
    float *pc = &acc.x, *pu = &uu.x, *pv = &vv.x;
    float a[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      a[w] = __fmul_rn(pc[w], mi);
      pv[w] = newmark_correct(pv[w], a[w], A.dt2);
      if (A.predict) newmark_predict(pu[w], pv[w], a[w], A.dt, A.dt2, A.dtsq2);
      bad |= !isfinite(pu[w]);
    }
    if (A.predict) *reinterpret_cast<float4 *>(A.u + o) = uu;
    *reinterpret_cast<float4 *>(A.v + o) = vv;
    if (A.a_store) *reinterpret_cast<float4 *>(A.a_store + o) = make_float4(a[0], a[1], a[2], a[3]);
  }
  if (bad) *A.flag = 1;
  if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) *A.step += 1;
}

}  // namespace dev
}  // namespace sfg
