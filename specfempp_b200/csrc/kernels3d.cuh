// sm_100a kernels of the 3D elastic spectral-element time step (FP32).
//
// One step: [element kernel] -> [receivers] -> [point update].
// * Element kernel: one thread per element GLL point (125 per element), E
//   elements per block.  The displacement gathered at the 125 points goes to
//   shared memory; the three 5-term Lagrange-derivative contractions per
//   component (include/algorithms/gradient.hpp:103-156), the map to physical
//   derivatives, the isotropic stress (include/medium/dim3/elastic/isotropic/
//   stress.hpp:46-99) and F = |J| sigma . grad(xi_k) (core/specfem/point/
//   stress.hpp:217-240) run in registers; F goes through shared memory for the
//   divergence with its pairwise weight products (include/algorithms/
//   divergence.hpp:90-137).  The epilogue applies the absorbing-face traction
//   -C v (C: per element point, the symmetric 3x3 sum over the element's
//   absorbing faces at that point, precomputed) and point sources, and stores
//   the element point's contribution at its point-major slot (owner-computes
//   assembly: the update sums each point's contributions in element order).
// * Point update: a = (sum of contributions) M^-1, Newmark corrector, and the
//   next step's predictor fused in (newmark.tpp:10-128); the last step of a
//   run stops after the corrector.
// * Receivers: one block per receiver, Lagrange interpolation of the chosen
//   field with a fixed-order tree sum.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sfg3 {
namespace dev {

constexpr int NG = 5;
constexpr int NQ = 125;

__constant__ float c3_hp[NG * NG];    // hp[i*5+j] = l'_j(xi_i)
__constant__ float c3_hpw[NG * NG];   // hp[l*5+i] * w[l]
__constant__ float c3_w[NG];

struct Elem3Args {
  const int *__restrict__ ibool;      // [nspec][125] lattice point
  const float *__restrict__ g9;       // [9][nspec*125] d xi_k / d x_j, k-major
  const float *__restrict__ jac;      // [nspec*125]
  const float *__restrict__ c0, *__restrict__ mu;   // lambda + 2 mu, mu
  const int *__restrict__ slot;       // point-major position of each element point
  const int *__restrict__ bc_slot;    // [nspec]: absorbing data slot or -1
  const float *__restrict__ bc_c;     // [slot][6][125]: C xx yy zz xy xz yz
  const int *__restrict__ src_head, *__restrict__ src_next;
  const float *__restrict__ src_arr;  // [nsrc][3][125]
  const float *__restrict__ stf;      // [nstep][nsrc]
  int nsrc, nstep;
  const int *__restrict__ step;
  const float *__restrict__ u, *__restrict__ v;   // [nglob][3]
  float *__restrict__ r;              // [slot][3]
  int nspec;
  size_t nloc;
};

// Point algebra shared by both element-kernel forms, written as explicit FMA
// chains (the build turns off contraction, so these are the only FMAs and
// every form rounds alike): the map to physical derivatives, the isotropic
// stress and F = |J| sigma . grad(xi_k).
__device__ __forceinline__ float dot3(float a0, float b0, float a1, float b1, float a2, float b2) {
  return fmaf(a2, b2, fmaf(a1, b1, a0 * b0));
}

__device__ __forceinline__ void stress3(const float du[3][3], float c0, float mu, float sig[3][3]) {
  const float lam = c0 - 2.f * mu;
  sig[0][0] = fmaf(c0, du[0][0], lam * (du[1][1] + du[2][2]));
  sig[1][1] = fmaf(c0, du[1][1], lam * (du[0][0] + du[2][2]));
  sig[2][2] = fmaf(c0, du[2][2], lam * (du[0][0] + du[1][1]));
  sig[0][1] = sig[1][0] = mu * (du[0][1] + du[1][0]);
  sig[0][2] = sig[2][0] = mu * (du[0][2] + du[2][0]);
  sig[1][2] = sig[2][1] = mu * (du[1][2] + du[2][1]);
}

template <int E>
__global__ void __launch_bounds__(NQ * E) k_stiffness3d(Elem3Args A) {
  __shared__ float su[E][3][NQ];
  __shared__ float sF[E][3][3][NQ];
  const int tid = threadIdx.x;
  const int le = tid / NQ, q = tid - le * NQ;
  const int e = blockIdx.x * E + le;
  const bool act = e < A.nspec;
  const size_t p = size_t(act ? e : 0) * NQ + q;
  const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
  const int g = act ? __ldg(A.ibool + p) : 0;
  float gi[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) gi[k] = __ldg(A.g9 + size_t(k) * A.nloc + p);
  const float jac = __ldg(A.jac + p), c0 = __ldg(A.c0 + p), mu = __ldg(A.mu + p);
  const int bs = act ? __ldg(A.bc_slot + e) : -1;
  const int src = act ? __ldg(A.src_head + e) : -1;
#pragma unroll
  for (int c = 0; c < 3; ++c) su[le][c][q] = act ? A.u[size_t(g) * 3 + c] : 0.f;
  // this point's Lagrange coefficients in registers: the points of a warp
  // differ, so indexed constant-bank loads would serialize
  float hx[NG], hy[NG], hz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    hx[l] = c3_hp[ix * NG + l];
    hy[l] = c3_hp[iy * NG + l];
    hz[l] = c3_hp[iz * NG + l];
  }
  __syncthreads();
  float du[3][3];  // du[c][j] = d u_c / d x_j
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float d0 = 0.f, d1 = 0.f, d2 = 0.f;
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      d0 = fmaf(hx[l], su[le][c][(iz * NG + iy) * NG + l], d0);
      d1 = fmaf(hy[l], su[le][c][(iz * NG + l) * NG + ix], d1);
      d2 = fmaf(hz[l], su[le][c][(l * NG + iy) * NG + ix], d2);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) du[c][j] = dot3(d0, gi[0 * 3 + j], d1, gi[1 * 3 + j], d2, gi[2 * 3 + j]);
  }
  float sig[3][3];
  stress3(du, c0, mu, sig);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      sF[le][c][k][q] = jac * dot3(sig[c][0], gi[k * 3 + 0], sig[c][1], gi[k * 3 + 1], sig[c][2], gi[k * 3 + 2]);
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    hx[l] = c3_hpw[l * NG + ix];
    hy[l] = c3_hpw[l * NG + iy];
    hz[l] = c3_hpw[l * NG + iz];
  }
  const float wx = c3_w[ix], wy = c3_w[iy], wz = c3_w[iz];
  const float wzy = wz * wy, wzx = wz * wx, wyx = wy * wx;
  __syncthreads();
  if (!act) return;
  float a[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float t1 = 0.f, t2 = 0.f, t3 = 0.f;
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      t1 = fmaf(sF[le][c][0][(iz * NG + iy) * NG + l], hx[l], t1);
      t2 = fmaf(sF[le][c][1][(iz * NG + l) * NG + ix], hy[l], t2);
      t3 = fmaf(sF[le][c][2][(l * NG + iy) * NG + ix], hz[l], t3);
    }
    a[c] = -dot3(wzy, t1, wzx, t2, wyx, t3);
  }
  if (bs >= 0) {
    const float *C = A.bc_c + size_t(bs) * 6 * NQ + q;
    const float cxx = C[0], cyy = C[NQ], czz = C[2 * NQ], cxy = C[3 * NQ], cxz = C[4 * NQ], cyz = C[5 * NQ];
    if (cxx != 0.f || cyy != 0.f || czz != 0.f) {
      const float vx = A.v[size_t(g) * 3], vy = A.v[size_t(g) * 3 + 1], vz = A.v[size_t(g) * 3 + 2];
      a[0] -= cxx * vx + cxy * vy + cxz * vz;
      a[1] -= cxy * vx + cyy * vy + cyz * vz;
      a[2] -= cxz * vx + cyz * vy + czz * vz;
    }
  }
  if (src >= 0) {
    const int step = *A.step;
    for (int s = src; s >= 0; s = A.src_next[s]) {
      const float f = step < A.nstep ? A.stf[size_t(step) * A.nsrc + s] : 0.f;
#pragma unroll
      for (int c = 0; c < 3; ++c) a[c] += f * A.src_arr[(size_t(s) * 3 + c) * NQ + q];
    }
  }
  const size_t sl = size_t(__ldg(A.slot + p)) * 3;
  A.r[sl] = a[0];
  A.r[sl + 1] = a[1];
  A.r[sl + 2] = a[2];
}

// Column form of the element kernel: one thread per (x, y) column of GLL
// points of an element, the column's five points (z = 0..4) in registers, E
// elements per block (25 E threads).  The z-direction contractions of the
// gradient and of the divergence run on the column's registers with
// warp-uniform coefficients; the x- and y-direction ones read the element's
// displacement and F arrays in shared memory, whose x rows are padded to 8
// floats so that a row is one float4 load plus one float load.  Per point the
// operations and their order are those of k_stiffness3d, so both kernels give
// the same bits.  Dynamic shared memory: E x (3 + 6) x 25 x 8 floats.  With 8
// elements per block the registers are capped for three blocks per SM; with
// 6 the compiler may keep the five points' index, Jacobian and material
// loads of a column in flight together.
constexpr int RP3 = 8;
template <int E>
__global__ void __launch_bounds__(NG * NG * E, E == 8 ? 3 : 1) k_stiffness3d_col(Elem3Args A) {
  extern __shared__ __align__(16) float dyn3[];
  const int tid = threadIdx.x;
  const int le = tid / (NG * NG), cq = tid - le * (NG * NG);
  const int iy = cq / NG, ix = cq - iy * NG;
  const int e = blockIdx.x * E + le;
  const bool act = e < A.nspec;
  const size_t pe = size_t(act ? e : 0) * NQ;
  float *su = dyn3 + size_t(le) * 9 * NG * NG * RP3;   // [c][z*5 + y][x]
  float *sF = su + 3 * NG * NG * RP3;                  // [c][k = 0, 1][z*5 + y][x]
  float uz[3][NG];
  int g[NG];
#pragma unroll
  for (int iz = 0; iz < NG; ++iz) g[iz] = act ? __ldg(A.ibool + pe + (iz * NG + iy) * NG + ix) : 0;
#pragma unroll
  for (int iz = 0; iz < NG; ++iz)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      uz[c][iz] = act ? A.u[size_t(g[iz]) * 3 + c] : 0.f;
      su[(c * NG * NG + iz * NG + iy) * RP3 + ix] = uz[c][iz];
    }
  float hx[NG], hy[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    hx[l] = c3_hp[ix * NG + l];
    hy[l] = c3_hp[iy * NG + l];
  }
  __syncthreads();
  float fz[3][NG];   // F[c][2] of the column's points
#pragma unroll
  for (int iz = 0; iz < NG; ++iz) {
    const size_t p = pe + (iz * NG + iy) * NG + ix;
    float gi[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) gi[k] = __ldg(A.g9 + size_t(k) * A.nloc + p);
    const float jac = __ldg(A.jac + p), c0 = __ldg(A.c0 + p), mu = __ldg(A.mu + p);
    float du[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float *row = su + (c * NG * NG + iz * NG + iy) * RP3;
      const float4 r4 = *reinterpret_cast<const float4 *>(row);
      const float rv[NG] = {r4.x, r4.y, r4.z, r4.w, row[4]};
      float d0 = 0.f, d1 = 0.f, d2 = 0.f;
#pragma unroll
      for (int l = 0; l < NG; ++l) {
        d0 = fmaf(hx[l], rv[l], d0);
        d1 = fmaf(hy[l], su[(c * NG * NG + iz * NG + l) * RP3 + ix], d1);
        d2 = fmaf(c3_hp[iz * NG + l], uz[c][l], d2);
      }
#pragma unroll
      for (int j = 0; j < 3; ++j) du[c][j] = dot3(d0, gi[0 * 3 + j], d1, gi[1 * 3 + j], d2, gi[2 * 3 + j]);
    }
    float sig[3][3];
    stress3(du, c0, mu, sig);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int k = 0; k < 2; ++k)
        sF[((c * 2 + k) * NG * NG + iz * NG + iy) * RP3 + ix] =
            jac * dot3(sig[c][0], gi[k * 3 + 0], sig[c][1], gi[k * 3 + 1], sig[c][2], gi[k * 3 + 2]);
      fz[c][iz] = jac * dot3(sig[c][0], gi[6], sig[c][1], gi[7], sig[c][2], gi[8]);
    }
  }
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    hx[l] = c3_hpw[l * NG + ix];
    hy[l] = c3_hpw[l * NG + iy];
  }
  const float wx = c3_w[ix], wy = c3_w[iy];
  const int bs = act ? __ldg(A.bc_slot + e) : -1;
  const int src = act ? __ldg(A.src_head + e) : -1;
  __syncthreads();
  if (!act) return;
#pragma unroll
  for (int iz = 0; iz < NG; ++iz) {
    const int q = (iz * NG + iy) * NG + ix;
    const float wz = c3_w[iz];
    const float wzy = wz * wy, wzx = wz * wx, wyx = wy * wx;
    float a[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float *row = sF + ((c * 2 + 0) * NG * NG + iz * NG + iy) * RP3;
      const float4 r4 = *reinterpret_cast<const float4 *>(row);
      const float rv[NG] = {r4.x, r4.y, r4.z, r4.w, row[4]};
      float t1 = 0.f, t2 = 0.f, t3 = 0.f;
#pragma unroll
      for (int l = 0; l < NG; ++l) {
        t1 = fmaf(rv[l], hx[l], t1);
        t2 = fmaf(sF[((c * 2 + 1) * NG * NG + iz * NG + l) * RP3 + ix], hy[l], t2);
        t3 = fmaf(fz[c][l], c3_hpw[l * NG + iz], t3);
      }
      a[c] = -dot3(wzy, t1, wzx, t2, wyx, t3);
    }
    if (bs >= 0) {
      const float *C = A.bc_c + size_t(bs) * 6 * NQ + q;
      const float cxx = C[0], cyy = C[NQ], czz = C[2 * NQ], cxy = C[3 * NQ], cxz = C[4 * NQ], cyz = C[5 * NQ];
      if (cxx != 0.f || cyy != 0.f || czz != 0.f) {
        const size_t gv = size_t(g[iz]) * 3;
        const float vx = A.v[gv], vy = A.v[gv + 1], vz = A.v[gv + 2];
        a[0] -= cxx * vx + cxy * vy + cxz * vz;
        a[1] -= cxy * vx + cyy * vy + cyz * vz;
        a[2] -= cxz * vx + cyz * vy + czz * vz;
      }
    }
    if (src >= 0) {
      const int step = *A.step;
      for (int s = src; s >= 0; s = A.src_next[s]) {
        const float f = step < A.nstep ? A.stf[size_t(step) * A.nsrc + s] : 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) a[c] += f * A.src_arr[(size_t(s) * 3 + c) * NQ + q];
      }
    }
    const size_t sl = size_t(__ldg(A.slot + pe + q)) * 3;
    A.r[sl] = a[0];
    A.r[sl + 1] = a[1];
    A.r[sl + 2] = a[2];
  }
}

struct Update3Args {
  float *__restrict__ u, *__restrict__ v, *__restrict__ a_store;
  const float *__restrict__ minv;
  const int *__restrict__ inv_start;
  const float *__restrict__ r;
  int npts;
  float dt, dt2, dtsq2;
  int predict;
  int *flag;
  int *step;
  int advance;
};

__device__ __forceinline__ void nm_predict(float &u, float &v, float a, float dt, float dt2, float dtsq2) {
  u = __fadd_rn(u, __fadd_rn(__fmul_rn(dt, v), __fmul_rn(dtsq2, a)));
  v = __fadd_rn(v, __fmul_rn(dt2, a));
}

__global__ void __launch_bounds__(256) k_update3d(Update3Args A) {
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < A.npts; g += stride) {
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    const int k1 = A.inv_start[g + 1];
    for (int k = A.inv_start[g]; k < k1; ++k) {
      s0 = s0 + A.r[size_t(k) * 3];
      s1 = s1 + A.r[size_t(k) * 3 + 1];
      s2 = s2 + A.r[size_t(k) * 3 + 2];
    }
    const float acc[3] = {s0, s1, s2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t i = size_t(g) * 3 + c;
      const float a = __fmul_rn(acc[c], A.minv[i]);
      float vv = __fadd_rn(A.v[i], __fmul_rn(A.dt2, a));
      float uu = A.u[i];
      if (A.predict) nm_predict(uu, vv, a, A.dt, A.dt2, A.dtsq2);
      if (A.predict) A.u[i] = uu;
      A.v[i] = vv;
      if (A.a_store) A.a_store[i] = a;
      bad |= !isfinite(uu);
    }
  }
  if (bad) *A.flag = 1;
  if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) *A.step += 1;
}

__global__ void __launch_bounds__(256) k_predict3d(float *__restrict__ u, float *__restrict__ v,
                                                   const float *__restrict__ a, size_t n, float dt, float dt2,
                                                   float dtsq2) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    float uu = u[i], vv = v[i];
    nm_predict(uu, vv, a[i], dt, dt2, dtsq2);
    u[i] = uu;
    v[i] = vv;
  }
}

struct Rec3Args {
  const int *__restrict__ ibool;
  const int *__restrict__ rec_elem;
  const float *__restrict__ rec_h;    // [nrec][125]
  const int *__restrict__ types;      // per type: 0 displacement, 1 velocity, 2 acceleration
  int ntypes, nrec, nsig;
  const float *__restrict__ u, *__restrict__ v;
  // acceleration of the step: the update's input (sum of contributions x M^-1)
  const float *__restrict__ minv, *__restrict__ r;
  const int *__restrict__ inv_start;
  float dt2;
  const int *__restrict__ step;
  float *__restrict__ seis;           // [nsig][ntypes][nrec][3]
};

// One block of 128 threads per receiver; run before the update of the step
// (velocity and acceleration are formed from the step's contributions the
// same way the update forms them).
__global__ void __launch_bounds__(128) k_receivers3d(Rec3Args A) {
  __shared__ float red[3][128];
  const int rr = blockIdx.x, q = threadIdx.x;
  const int step = *A.step;
  if (step >= A.nsig) return;
  const int e = A.rec_elem[rr];
  for (int t = 0; t < A.ntypes; ++t) {
    float val[3] = {0.f, 0.f, 0.f};
    if (q < NQ) {
      const int g = A.ibool[size_t(e) * NQ + q];
      const float h = A.rec_h[size_t(rr) * NQ + q];
      float f[3];
      if (A.types[t] == 0) {
        for (int c = 0; c < 3; ++c) f[c] = A.u[size_t(g) * 3 + c];
      } else {
        float s[3] = {0.f, 0.f, 0.f};
        for (int k = A.inv_start[g]; k < A.inv_start[g + 1]; ++k)
          for (int c = 0; c < 3; ++c) s[c] = s[c] + A.r[size_t(k) * 3 + c];
        for (int c = 0; c < 3; ++c) {
          const float acc = __fmul_rn(s[c], A.minv[size_t(g) * 3 + c]);
          f[c] = A.types[t] == 2 ? acc : __fadd_rn(A.v[size_t(g) * 3 + c], __fmul_rn(A.dt2, acc));
        }
      }
      for (int c = 0; c < 3; ++c) val[c] = h * f[c];
    }
    for (int c = 0; c < 3; ++c) red[c][q] = val[c];
    __syncthreads();
    for (int o = 64; o > 0; o >>= 1) {
      if (q < o)
        for (int c = 0; c < 3; ++c) red[c][q] = red[c][q] + red[c][q + o];
      __syncthreads();
    }
    if (q < 3) A.seis[((size_t(step) * A.ntypes + t) * A.nrec + rr) * 3 + q] = red[q][0];
    __syncthreads();
  }
}

}  // namespace dev
}  // namespace sfg3
