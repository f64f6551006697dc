// Row form of the owner-computes element kernel (single shot; isotropic P-SV
// and acoustic media, one launch for both).
//
// One thread per element row (the five points of a row iz), E elements per
// block (5 E threads).  The row's displacement is gathered into registers,
// and its Jacobian, material words and slot indices are requested at the
// same time (their latency overlaps the gather's);
// the xi-direction contractions of the gradient and of the divergence run
// on the row in registers with warp-uniform coefficients (constant bank),
// the gamma-direction ones read columns of the element's displacement and
// F1 in shared memory, so a point needs a fifth of the shared-memory and
// coefficient loads of the point-per-thread kernel.  Per point the
// operations and their order are those of elastic_block<E, 0, true> and
// acoustic_block<E, true> (the P-SV components paired in FFMA2, the acoustic
// directions paired; FFMA2 rounds each lane as fmaf), so the results are the
// same bits.
// Reference: include/kokkos_kernels/impl/compute_stiffness_interaction.tpp:140-247,
// include/algorithms/gradient.hpp:40-82, divergence.hpp:41-74,
// include/boundary_conditions/stacey/stacey.tpp:50-80, 291-326,
// include/kokkos_kernels/impl/compute_source_interaction.tpp:17-104.
#pragma once

#include "kernels2d_batched.cuh"

namespace sfg {
namespace dev {

template <int E>
__device__ __forceinline__ void elastic_rows(const StiffArgs &S, const MedArgs &A, int ebase, float2 *smem) {
  const int tid = threadIdx.x;
  const int le = tid / NG, iz = tid - le * NG;
  const int e = ebase + le;
  const bool act = e < A.e1;
  float2 *su = smem + le * NP;              // [25] (u_x, u_z)
  float2 *sF1 = smem + (E + le) * NP;       // [25] F1 of both components
  const size_t pe = size_t(act ? e : A.e0) * NP + iz * NG;
  int g[NG], sl[NG];
  float2 ur[NG];
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) g[ix] = act ? __ldg(A.ibool + pe + ix) : 0;
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) sl[ix] = __ldg(A.slot + pe + ix);
  // the row's Jacobian and material words, requested with the gather
  float gxix[NG], gxiz[NG], ggax[NG], ggaz[NG], gjac[NG], gc0[NG], gmu[NG];
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    gxix[ix] = __ldg(A.xix + pe + ix); gxiz[ix] = __ldg(A.xiz + pe + ix);
    ggax[ix] = __ldg(A.gax + pe + ix); ggaz[ix] = __ldg(A.gaz + pe + ix);
    gjac[ix] = __ldg(A.jac + pe + ix); gc0[ix] = __ldg(A.prop0 + pe + ix); gmu[ix] = __ldg(A.prop1 + pe + ix);
  }
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    ur[ix] = act ? reinterpret_cast<const float2 *>(A.u)[g[ix]] : make_float2(0.f, 0.f);
    su[iz * NG + ix] = ur[ix];
  }
  float hz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) hz[l] = c_hp[iz * NG + l];
  __syncthreads();
  // xi derivatives of the row's points (both components paired), in place
  {
    float2 dx[NG];
#pragma unroll
    for (int ix = 0; ix < NG; ++ix) {
      float2 px = make_float2(0.f, 0.f);
#pragma unroll
      for (int l = 0; l < NG; ++l) px = fma2(f2(c_hp[ix * NG + l]), ur[l], px);
      dx[ix] = px;
    }
#pragma unroll
    for (int ix = 0; ix < NG; ++ix) ur[ix] = dx[ix];
  }
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    const float xix = gxix[ix], xiz = gxiz[ix], gax = ggax[ix], gaz = ggaz[ix], jac = gjac[ix];
    const float c0 = gc0[ix], mu = gmu[ix];
    float2 pg = make_float2(0.f, 0.f);
#pragma unroll
    for (int l = 0; l < NG; ++l) pg = fma2(f2(hz[l]), su[l * NG + ix], pg);
    const float dxi0 = ur[ix].x, dxi1 = ur[ix].y, dga0 = pg.x, dga1 = pg.y;
    const float du00 = xix * dxi0 + gax * dga0, du01 = xiz * dxi0 + gaz * dga0;
    const float du10 = xix * dxi1 + gax * dga1;
    const float du11 = xiz * dxi1 + gaz * dga1;
    const float lam = c0 - 2.f * mu;
    const float sxx = c0 * du00 + lam * du11;
    const float szz = c0 * du11 + lam * du00;
    const float sxz = mu * (du01 + du10);
    // Sx = (sxx, sxz), Sz = (sxz, szz) for components (x, z)
    ur[ix] = make_float2(jac * (sxx * xix + sxz * xiz), jac * (sxz * xix + szz * xiz));   // F0
    sF1[iz * NG + ix] = make_float2(jac * (sxx * gax + sxz * gaz), jac * (sxz * gax + szz * gaz));
  }
  float wz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) wz[l] = c_hpw[l * NG + iz];
  const float wiz = c_w[iz];
  const int bs = act ? __ldg(A.bc_slot + e) : -1;
  const int src = act ? __ldg(A.src_head + e) : -1;
  __syncthreads();
  if (!act) return;
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    const int q = iz * NG + ix;
    float2 t1 = make_float2(0.f, 0.f), t2 = make_float2(0.f, 0.f);
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      t1 = fma2(ur[l], f2(c_hpw[l * NG + ix]), t1);
      t2 = fma2(sF1[l * NG + ix], f2(wz[l]), t2);
    }
    float a0 = -(wiz * t1.x + c_w[ix] * t2.x);
    float a1 = -(wiz * t1.y + c_w[ix] * t2.y);
    if (bs >= 0) {
      const size_t k = size_t(bs) * NP + q;
      const float wq = A.bc_w[k];
      if (wq != 0.f) {
        const float nx = A.bc_nx[k], nz = A.bc_nz[k], j1 = A.bc_j1[k];
        const float2 vv = reinterpret_cast<const float2 *>(A.v)[g[ix]];
        const float rvp = A.bc_imp0[k], rvs = A.bc_imp1[k];
        const float vn = vv.x * nx + vv.y * nz;
        const float fx = ((vn * nx / (j1 * j1)) * (rvp - rvs)) + vv.x * rvs;
        const float fz = ((vn * nz / (j1 * j1)) * (rvp - rvs)) + vv.y * rvs;
        a0 += -1.f * fx * j1 * wq;
        a1 += -1.f * fz * j1 * wq;
      }
    }
    if (src >= 0) {
      const int step = *S.step;
      for (int s = src; s >= 0; s = S.src_next[s]) {
        const float f = step < S.nstep ? S.stf[size_t(step) * S.nsrc + s] : 0.f;
        a0 += f * S.src_arr[(size_t(s) * 2 + 0) * NP + q];
        a1 += f * S.src_arr[(size_t(s) * 2 + 1) * NP + q];
      }
    }
    reinterpret_cast<float2 *>(A.r)[sl[ix]] = make_float2(a0, a1);
  }
}

template <int E>
__device__ __forceinline__ void acoustic_rows(const StiffArgs &S, const MedArgs &A, int ebase, float *smem) {
  const int tid = threadIdx.x;
  const int le = tid / NG, iz = tid - le * NG;
  const int e = ebase + le;
  const bool act = e < A.e1;
  float *su = smem + le * NP;               // [25] chi
  float *sF1 = smem + (E + le) * NP;        // [25] F1
  const size_t pe = size_t(act ? e : A.e0) * NP + iz * NG;
  int g[NG], sl[NG];
  float ur[NG];
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) g[ix] = act ? __ldg(A.ibool + pe + ix) : 0;
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) sl[ix] = __ldg(A.slot + pe + ix);
  // the row's Jacobian and material words, requested with the gather
  float gxix[NG], gxiz[NG], ggax[NG], ggaz[NG], gjac[NG], grho[NG];
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    gxix[ix] = __ldg(A.xix + pe + ix); gxiz[ix] = __ldg(A.xiz + pe + ix);
    ggax[ix] = __ldg(A.gax + pe + ix); ggaz[ix] = __ldg(A.gaz + pe + ix);
    gjac[ix] = __ldg(A.jac + pe + ix); grho[ix] = __ldg(A.prop0 + pe + ix);
  }
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    ur[ix] = act ? A.u[g[ix]] : 0.f;
    su[iz * NG + ix] = ur[ix];
  }
  float hz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) hz[l] = c_hp[iz * NG + l];
  __syncthreads();
  float f0[NG];
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    const float xix = gxix[ix], xiz = gxiz[ix], gax = ggax[ix], gaz = ggaz[ix], jac = gjac[ix];
    const float rhoinv = grho[ix];
    // the two derivative directions paired (FFMA2, rounding as fmaf)
    float2 d = make_float2(0.f, 0.f);
#pragma unroll
    for (int l = 0; l < NG; ++l) d = fma2(make_float2(c_hp[ix * NG + l], hz[l]), make_float2(ur[l], su[l * NG + ix]), d);
    const float dxi = d.x, dga = d.y;
    const float s0 = rhoinv * (xix * dxi + gax * dga);
    const float s1 = rhoinv * (xiz * dxi + gaz * dga);
    f0[ix] = jac * (s0 * xix + s1 * xiz);
    sF1[iz * NG + ix] = jac * (s0 * gax + s1 * gaz);
  }
  float wz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) wz[l] = c_hpw[l * NG + iz];
  const float wiz = c_w[iz];
  const int bs = act ? __ldg(A.bc_slot + e) : -1;
  const int src = act ? __ldg(A.src_head + e) : -1;
  __syncthreads();
  if (!act) return;
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    const int q = iz * NG + ix;
    float2 t = make_float2(0.f, 0.f);
#pragma unroll
    for (int l = 0; l < NG; ++l)
      t = fma2(make_float2(f0[l], sF1[l * NG + ix]), make_float2(c_hpw[l * NG + ix], wz[l]), t);
    float a = -(wiz * t.x + c_w[ix] * t.y);
    if (bs >= 0) {
      const size_t k = size_t(bs) * NP + q;
      const float wq = A.bc_w[k];
      if (wq != 0.f) a += -1.f * (wq * A.bc_j1[k]) * A.bc_imp0[k] * A.v[g[ix]];
      a *= A.bc_keep[k];   // acoustic free surface (Dirichlet) zeroes the element term
    }
    if (src >= 0) {
      const int step = *S.step;
      for (int s = src; s >= 0; s = S.src_next[s]) {
        const float f = step < S.nstep ? S.stf[size_t(step) * S.nsrc + s] : 0.f;
        a += f * S.src_arr[(size_t(s) * 2) * NP + q];
      }
    }
    A.r[sl[ix]] = a;
  }
}

// Blocks [0, el.nblocks) run elastic P-SV elements, the others acoustic ones.
template <int E>
__global__ void __launch_bounds__(NG * E, E == 16 ? 8 : (E == 32 ? 4 : 1)) k_stiffness_row(StiffArgs S) {
  __shared__ __align__(16) float2 smem[2 * E * NP];
  if (int(blockIdx.x) < S.el.nblocks)
    elastic_rows<E>(S, S.el, S.el.e0 + blockIdx.x * E, smem);
  else
    acoustic_rows<E>(S, S.ac, S.ac.e0 + (blockIdx.x - S.el.nblocks) * E, reinterpret_cast<float *>(smem));
}

}  // namespace dev
}  // namespace sfg
