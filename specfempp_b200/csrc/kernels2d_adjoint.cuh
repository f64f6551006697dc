// Discrete adjoint of the 2D elastic P-SV time step (FP32), for rho / kappa /
// mu gradients of a seismogram misfit.
//
// Forward step k (the library's arithmetic, end-of-step state u, v, a):
//   predictor   u~ = u + dt v + dt^2/2 a,   v~ = v + dt/2 a
//   forces      a' = B (f_k - K u~ - C v~)            (B = M_eff^-1, diagonal)
//   corrector   v' = v~ + dt/2 a',  u' = u~;  seismogram d_k = R u'
// Reverse sweep of step k, for adjoint state (lu, lv) of (u', v') with
// mu_k = B (la + dt/2 lv) already formed and g_k = dL/dd_k:
//   lv~ = lv - C mu_k                                   k_adj_stacey (start of the step)
//   lu~ = lu + R^T g_k - K mu_k                         k_adj_elem (-K mu, R^T g_k per element point)
//                                                       + k_adj_post (per-point sum)
//   lu <- lu~,  lv <- dt lu~ + lv~,  la = dt^2/2 lu~ + dt/2 lv~,
//   mu_(k-1) = B (la + dt/2 lv)                         k_adj_post
// and the model gradient of the step, per element GLL point p with
// W_p = w_x w_z |J|:
//   dL/dkappa_p += -W_p (div mu)(div u~)
//   dL/dmu_p    += -W_p [4/3 (mxx uxx + mzz uzz) - 2/3 (mxx uzz + mzz uxx)
//                        + (mxz + mzx)(uxz + uzx)]
//   dL/drho_p   += -W_p G(g_p),  G(g) += mu_k(g) . a'_k(g)   (mass part of B,
//                                                              summed per global point)
// plus, on the absorbing edges, the dependence of the Stacey impedances
// rho vp and rho vs on (rho, kappa, mu) (adj_stacey_grad).
// kappa is the bulk modulus the reference stores (lambda + 2mu = kappa +
// 4/3 mu, include/medium/dim2/elastic/isotropic/properties.hpp:71-91).  The
// per-step terms are summed in FP32 over a checkpoint segment and folded into
// a compensated (Kahan) total once per segment.  These are the exact
// derivatives of the discrete forward model; the reference's continuous
// kernels (include/medium/dim2/elastic/isotropic/frechet_derivative.hpp:55-181)
// carry the same strain products (its mu bracket is half of the one above and
// its kappa prefactor is lambda + mu), integrated in time with -dt.
//
// SH (one component u_y, sigma = mu grad u_y, Stacey traction -rho vs v):
// the same sweep with scalar fields; dL/dmu_p += -W_p grad(mu) . grad(u~),
// kappa does not enter, and of the Stacey sums only A2 and A4 exist (the SH
// reference kernels: frechet_derivative.hpp:219-278).  Kernels that differ
// per wave type take NC, the number of components.
//
// Acoustic (potential chi, sigma = rho^-1 grad chi, M = W / kappa, Stacey
// traction -w |n| chi_dot / (rho vp), free-surface points masked by keep):
// the scalar sweep with the mask applied to the gathered adjoint field;
// dL/d(rho^-1)_p += -W_p grad(keep mu) . grad(chi~), the mass term gives
// kappa, and pressure seismograms d_k = -R chi_dd'_k enter as -R^T g_k on
// the adjoint acceleration (k_adj_psrc), not on lu (the reference's acoustic
// kernels: include/medium/dim2/acoustic/isotropic/frechet_derivative.hpp:61-93).
//
// Coupled acoustic-elastic step (conforming interface): both media's sweeps
// in one reverse step, joined by the transposed coupling of AdjCoupling
// (the reference's combined run over both media:
// include/kokkos_kernels/frechet_kernels.hpp:37-49, compute_coupling.tpp:21-115).
#pragma once

#include "kernels2d_batched.cuh"

namespace sfg {
namespace dev {

struct AdjArgs {
  const int *__restrict__ ibool;
  const float *__restrict__ xix, *__restrict__ xiz, *__restrict__ gax, *__restrict__ gaz,
      *__restrict__ jac, *__restrict__ prop0, *__restrict__ prop1;
  const float *__restrict__ mu;      // adjoint field mu_k [nglob][2]
  const float *__restrict__ uf;      // forward u~ of the step [nglob][2]
  float *__restrict__ r;             // element-point results [pslot[p]][2] (point-major)
  const int *__restrict__ pslot;
  float *__restrict__ seg;           // segment sums [nspec*25][kappa, mu]
  const int *__restrict__ ad_head, *__restrict__ ad_next;  // receivers per element
  const float *__restrict__ ad_h;    // receiver Lagrange weights [nrec][25]
  const float *__restrict__ gtab;    // dL/d seismogram [nstep][nrec][2]
  const int *__restrict__ seg_k0;    // first step of the segment (device)
  const int *__restrict__ bc_slot;   // acoustic: free-surface mask (bc_keep) per boundary element
  const float *__restrict__ bc_keep;
  int slot;                          // step of the segment: k = *seg_k0 + slot
  int nrec;
  int nspec;
  Quad quad;
};

template <int E>
__global__ void __launch_bounds__(NP * E) k_adj_elem(AdjArgs A) {
  __shared__ float sm_[2][E][NP], su_[2][E][NP];
  __shared__ float sF[2][2][E][NP];
  __shared__ float shp[NP], shpw[NP], sw[NG];
  const int tid = threadIdx.x;
  load_quad(A.quad, shp, shpw, sw, tid);
  const int le = tid / NP, q = tid - le * NP;
  const int e = blockIdx.x * E + le;
  const bool act = e < A.nspec;
  const size_t p = size_t(act ? e : 0) * NP + q;
  const int g = act ? __ldg(A.ibool + p) : 0;
  const float xix = __ldg(A.xix + p), xiz = __ldg(A.xiz + p), gax = __ldg(A.gax + p),
              gaz = __ldg(A.gaz + p), jac = __ldg(A.jac + p);
  const float c0 = __ldg(A.prop0 + p), mu = __ldg(A.prop1 + p);
  const float2 m2 = act ? reinterpret_cast<const float2 *>(A.mu)[g] : make_float2(0.f, 0.f);
  const float2 u2 = act ? reinterpret_cast<const float2 *>(A.uf)[g] : make_float2(0.f, 0.f);
  const int rh = act ? __ldg(A.ad_head + e) : -1;
  sm_[0][le][q] = m2.x; sm_[1][le][q] = m2.y;
  su_[0][le][q] = u2.x; su_[1][le][q] = u2.y;
  __syncthreads();
  const int iz = q / NG, ix = q - iz * NG;
  float dm[2][2], du[2][2];  // [comp][xi/gamma]
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    dm[c][0] = dm[c][1] = du[c][0] = du[c][1] = 0.f;
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      dm[c][0] = fmaf(shp[ix * NG + l], sm_[c][le][iz * NG + l], dm[c][0]);
      dm[c][1] = fmaf(shp[iz * NG + l], sm_[c][le][l * NG + ix], dm[c][1]);
      du[c][0] = fmaf(shp[ix * NG + l], su_[c][le][iz * NG + l], du[c][0]);
      du[c][1] = fmaf(shp[iz * NG + l], su_[c][le][l * NG + ix], du[c][1]);
    }
  }
  // physical derivatives: mxz = d(mu_x)/dz, mzx = d(mu_z)/dx
  const float mxx = xix * dm[0][0] + gax * dm[0][1], mxz = xiz * dm[0][0] + gaz * dm[0][1];
  const float mzx = xix * dm[1][0] + gax * dm[1][1], mzz = xiz * dm[1][0] + gaz * dm[1][1];
  const float uxx = xix * du[0][0] + gax * du[0][1], uxz = xiz * du[0][0] + gaz * du[0][1];
  const float uzx = xix * du[1][0] + gax * du[1][1], uzz = xiz * du[1][0] + gaz * du[1][1];
  // stress of the adjoint field, as in the forward element kernel
  const float lam = c0 - 2.f * mu;
  const float sxx = c0 * mxx + lam * mzz;
  const float szz = c0 * mzz + lam * mxx;
  const float sxz = mu * (mxz + mzx);
  sF[0][0][le][q] = jac * (sxx * xix + sxz * xiz);
  sF[0][1][le][q] = jac * (sxx * gax + sxz * gaz);
  sF[1][0][le][q] = jac * (sxz * xix + szz * xiz);
  sF[1][1][le][q] = jac * (sxz * gax + szz * gaz);
  __syncthreads();
  if (!act) return;
  float r[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    float t1 = 0.f, t2 = 0.f;
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      t1 = fmaf(sF[c][0][le][iz * NG + l], shpw[l * NG + ix], t1);
      t2 = fmaf(sF[c][1][le][l * NG + ix], shpw[l * NG + iz], t2);
    }
    r[c] = -(sw[iz] * t1 + sw[ix] * t2);
  }
  // receivers of this element inject R^T g (the adjoint sources)
  if (rh >= 0) {
    const float *g_k = A.gtab + size_t(*A.seg_k0 + A.slot) * A.nrec * 2;
    for (int k = rh; k >= 0; k = A.ad_next[k]) {
      const float h = A.ad_h[size_t(k) * NP + q];
      r[0] += g_k[2 * k] * h;
      r[1] += g_k[2 * k + 1] * h;
    }
  }
  reinterpret_cast<float2 *>(A.r)[__ldg(A.pslot + p)] = make_float2(r[0], r[1]);
  // gradient terms of this step, summed over the segment
  const float W = sw[ix] * sw[iz] * jac;
  const float divm = mxx + mzz, divu = uxx + uzz;
  const float tk = -W * (divm * divu);
  const float tm = -W * ((4.f / 3.f) * (mxx * uxx + mzz * uzz) - (2.f / 3.f) * (mxx * uzz + mzz * uxx) +
                         (mxz + mzx) * (uxz + uzx));
  float2 sg = reinterpret_cast<float2 *>(A.seg)[p];
  sg.x += tk;
  sg.y += tm;
  reinterpret_cast<float2 *>(A.seg)[p] = sg;
}

// Row form of k_adj_elem: one thread per element row (five points) of E
// elements; the xi-direction contractions of both fields and of the
// divergence on the row in registers (warp-uniform coefficients, the two
// components paired in FFMA2, which rounds each lane as fmaf), the
// gamma-direction ones from shared-memory columns.  Per point the
// operations and their order are those of k_adj_elem (same bits).
template <int E>
__global__ void __launch_bounds__(NG * E, 4) k_adj_elem_row(AdjArgs A) {
  __shared__ float2 sm2[E][NP], su2[E][NP], sF1[E][NP];
  const int tid = threadIdx.x;
  const int le = tid / NG, iz = tid - le * NG;
  const int e = blockIdx.x * E + le;
  const bool act = e < A.nspec;
  const size_t pe = size_t(act ? e : 0) * NP + iz * NG;
  int g[NG], sl[NG];
  float2 mr[NG], ur[NG];
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) g[ix] = act ? __ldg(A.ibool + pe + ix) : 0;
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) sl[ix] = __ldg(A.pslot + pe + ix);
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    mr[ix] = act ? reinterpret_cast<const float2 *>(A.mu)[g[ix]] : make_float2(0.f, 0.f);
    ur[ix] = act ? reinterpret_cast<const float2 *>(A.uf)[g[ix]] : make_float2(0.f, 0.f);
    sm2[le][iz * NG + ix] = mr[ix];
    su2[le][iz * NG + ix] = ur[ix];
  }
  const int rh = act ? __ldg(A.ad_head + e) : -1;
  // the row's Jacobian and material words, requested with the gathers
  float gxix[NG], gxiz[NG], ggax[NG], ggaz[NG], gjac[NG], gc0[NG], gmu[NG];
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    gxix[ix] = __ldg(A.xix + pe + ix); gxiz[ix] = __ldg(A.xiz + pe + ix);
    ggax[ix] = __ldg(A.gax + pe + ix); ggaz[ix] = __ldg(A.gaz + pe + ix);
    gjac[ix] = __ldg(A.jac + pe + ix); gc0[ix] = __ldg(A.prop0 + pe + ix); gmu[ix] = __ldg(A.prop1 + pe + ix);
  }
  float hz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) hz[l] = c_hp[iz * NG + l];
  __syncthreads();
  // xi derivatives of both fields, both components paired, in place
  {
    float2 dm[NG], du[NG];
#pragma unroll
    for (int ix = 0; ix < NG; ++ix) {
      float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
#pragma unroll
      for (int l = 0; l < NG; ++l) {
        a = fma2(f2(c_hp[ix * NG + l]), mr[l], a);
        b = fma2(f2(c_hp[ix * NG + l]), ur[l], b);
      }
      dm[ix] = a;
      du[ix] = b;
    }
#pragma unroll
    for (int ix = 0; ix < NG; ++ix) { mr[ix] = dm[ix]; ur[ix] = du[ix]; }
  }
  const float wiz = c_w[iz];
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    const size_t p = pe + ix;
    const float xix = gxix[ix], xiz = gxiz[ix], gax = ggax[ix], gaz = ggaz[ix], jac = gjac[ix];
    const float c0 = gc0[ix], mu = gmu[ix];
    float2 gm = make_float2(0.f, 0.f), gu = make_float2(0.f, 0.f);
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      gm = fma2(f2(hz[l]), sm2[le][l * NG + ix], gm);
      gu = fma2(f2(hz[l]), su2[le][l * NG + ix], gu);
    }
    // dm[c][0] = mr[ix].c (xi), dm[c][1] = gm.c (gamma)
    const float mxx = xix * mr[ix].x + gax * gm.x, mxz = xiz * mr[ix].x + gaz * gm.x;
    const float mzx = xix * mr[ix].y + gax * gm.y, mzz = xiz * mr[ix].y + gaz * gm.y;
    const float uxx = xix * ur[ix].x + gax * gu.x, uxz = xiz * ur[ix].x + gaz * gu.x;
    const float uzx = xix * ur[ix].y + gax * gu.y, uzz = xiz * ur[ix].y + gaz * gu.y;
    const float lam = c0 - 2.f * mu;
    const float sxx = c0 * mxx + lam * mzz;
    const float szz = c0 * mzz + lam * mxx;
    const float sxz = mu * (mxz + mzx);
    mr[ix] = make_float2(jac * (sxx * xix + sxz * xiz), jac * (sxz * xix + szz * xiz));   // F0
    sF1[le][iz * NG + ix] = make_float2(jac * (sxx * gax + sxz * gaz), jac * (sxz * gax + szz * gaz));
    if (act) {
      // gradient terms of this step, summed over the segment
      const float W = c_w[ix] * wiz * jac;
      const float divm = mxx + mzz, divu = uxx + uzz;
      const float tk = -W * (divm * divu);
      const float tm = -W * ((4.f / 3.f) * (mxx * uxx + mzz * uzz) - (2.f / 3.f) * (mxx * uzz + mzz * uxx) +
                             (mxz + mzx) * (uxz + uzx));
      float2 sg = reinterpret_cast<float2 *>(A.seg)[p];
      sg.x += tk;
      sg.y += tm;
      reinterpret_cast<float2 *>(A.seg)[p] = sg;
    }
  }
  float wz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) wz[l] = c_hpw[l * NG + iz];
  __syncthreads();
  if (!act) return;
#pragma unroll
  for (int ix = 0; ix < NG; ++ix) {
    const int q = iz * NG + ix;
    float2 t1 = make_float2(0.f, 0.f), t2 = make_float2(0.f, 0.f);
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      t1 = fma2(mr[l], f2(c_hpw[l * NG + ix]), t1);
      t2 = fma2(sF1[le][l * NG + ix], f2(wz[l]), t2);
    }
    float r0 = -(wiz * t1.x + c_w[ix] * t2.x);
    float r1 = -(wiz * t1.y + c_w[ix] * t2.y);
    // receivers of this element inject R^T g (the adjoint sources)
    if (rh >= 0) {
      const float *g_k = A.gtab + size_t(*A.seg_k0 + A.slot) * A.nrec * 2;
      for (int k = rh; k >= 0; k = A.ad_next[k]) {
        const float h = A.ad_h[size_t(k) * NP + q];
        r0 += g_k[2 * k] * h;
        r1 += g_k[2 * k + 1] * h;
      }
    }
    reinterpret_cast<float2 *>(A.r)[sl[ix]] = make_float2(r0, r1);
  }
}

// SH reverse element step (one component): -K mu with sigma = mu grad,
// adjoint sources R^T g (first seismogram component, BXY), and the mu term.
template <int E>
__global__ void __launch_bounds__(NP * E) k_adj_elem_sh(AdjArgs A) {
  __shared__ float sm_[E][NP], su_[E][NP];
  __shared__ float sF[2][E][NP];
  __shared__ float shp[NP], shpw[NP], sw[NG];
  const int tid = threadIdx.x;
  load_quad(A.quad, shp, shpw, sw, tid);
  const int le = tid / NP, q = tid - le * NP;
  const int e = blockIdx.x * E + le;
  const bool act = e < A.nspec;
  const size_t p = size_t(act ? e : 0) * NP + q;
  const int g = act ? __ldg(A.ibool + p) : 0;
  const float xix = __ldg(A.xix + p), xiz = __ldg(A.xiz + p), gax = __ldg(A.gax + p),
              gaz = __ldg(A.gaz + p), jac = __ldg(A.jac + p);
  const float mu = __ldg(A.prop1 + p);
  sm_[le][q] = act ? A.mu[g] : 0.f;
  su_[le][q] = act ? A.uf[g] : 0.f;
  const int rh = act ? __ldg(A.ad_head + e) : -1;
  __syncthreads();
  const int iz = q / NG, ix = q - iz * NG;
  float dm0 = 0.f, dm1 = 0.f, du0 = 0.f, du1 = 0.f;
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    dm0 = fmaf(shp[ix * NG + l], sm_[le][iz * NG + l], dm0);
    dm1 = fmaf(shp[iz * NG + l], sm_[le][l * NG + ix], dm1);
    du0 = fmaf(shp[ix * NG + l], su_[le][iz * NG + l], du0);
    du1 = fmaf(shp[iz * NG + l], su_[le][l * NG + ix], du1);
  }
  const float mx = xix * dm0 + gax * dm1, mz = xiz * dm0 + gaz * dm1;
  const float ux = xix * du0 + gax * du1, uz = xiz * du0 + gaz * du1;
  const float sx = mu * mx, sz = mu * mz;
  sF[0][le][q] = jac * (sx * xix + sz * xiz);
  sF[1][le][q] = jac * (sx * gax + sz * gaz);
  __syncthreads();
  if (!act) return;
  float t1 = 0.f, t2 = 0.f;
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    t1 = fmaf(sF[0][le][iz * NG + l], shpw[l * NG + ix], t1);
    t2 = fmaf(sF[1][le][l * NG + ix], shpw[l * NG + iz], t2);
  }
  float r = -(sw[iz] * t1 + sw[ix] * t2);
  if (rh >= 0) {
    const float *g_k = A.gtab + size_t(*A.seg_k0 + A.slot) * A.nrec * 2;
    for (int k = rh; k >= 0; k = A.ad_next[k]) r += g_k[2 * k] * A.ad_h[size_t(k) * NP + q];
  }
  A.r[__ldg(A.pslot + p)] = r;
  const float W = sw[ix] * sw[iz] * jac;
  A.seg[2 * p + 1] += -W * (mx * ux + mz * uz);
}

// Acoustic reverse element step: -K (keep mu) with sigma = rho^-1 grad and
// the rho^-1 term (no receiver term here: pressure seismograms act on the
// adjoint acceleration, k_adj_psrc).
template <int E>
__global__ void __launch_bounds__(NP * E) k_adj_elem_ac(AdjArgs A) {
  __shared__ float sm_[E][NP], su_[E][NP];
  __shared__ float sF[2][E][NP];
  __shared__ float shp[NP], shpw[NP], sw[NG];
  const int tid = threadIdx.x;
  load_quad(A.quad, shp, shpw, sw, tid);
  const int le = tid / NP, q = tid - le * NP;
  const int e = blockIdx.x * E + le;
  const bool act = e < A.nspec;
  const size_t p = size_t(act ? e : 0) * NP + q;
  const int g = act ? __ldg(A.ibool + p) : 0;
  const float xix = __ldg(A.xix + p), xiz = __ldg(A.xiz + p), gax = __ldg(A.gax + p),
              gaz = __ldg(A.gaz + p), jac = __ldg(A.jac + p);
  const float rhoinv = __ldg(A.prop0 + p);
  float m = act ? A.mu[g] : 0.f;
  const int bs = act ? __ldg(A.bc_slot + e) : -1;
  if (bs >= 0) m *= A.bc_keep[size_t(bs) * NP + q];
  sm_[le][q] = m;
  su_[le][q] = act ? A.uf[g] : 0.f;
  __syncthreads();
  const int iz = q / NG, ix = q - iz * NG;
  float dm0 = 0.f, dm1 = 0.f, du0 = 0.f, du1 = 0.f;
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    dm0 = fmaf(shp[ix * NG + l], sm_[le][iz * NG + l], dm0);
    dm1 = fmaf(shp[iz * NG + l], sm_[le][l * NG + ix], dm1);
    du0 = fmaf(shp[ix * NG + l], su_[le][iz * NG + l], du0);
    du1 = fmaf(shp[iz * NG + l], su_[le][l * NG + ix], du1);
  }
  const float mx = xix * dm0 + gax * dm1, mz = xiz * dm0 + gaz * dm1;
  const float ux = xix * du0 + gax * du1, uz = xiz * du0 + gaz * du1;
  const float sx = rhoinv * mx, sz = rhoinv * mz;
  sF[0][le][q] = jac * (sx * xix + sz * xiz);
  sF[1][le][q] = jac * (sx * gax + sz * gaz);
  __syncthreads();
  if (!act) return;
  float t1 = 0.f, t2 = 0.f;
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    t1 = fmaf(sF[0][le][iz * NG + l], shpw[l * NG + ix], t1);
    t2 = fmaf(sF[1][le][l * NG + ix], shpw[l * NG + iz], t2);
  }
  A.r[__ldg(A.pslot + p)] = -(sw[iz] * t1 + sw[ix] * t2);
  const float W = sw[ix] * sw[iz] * jac;
  A.seg[2 * p + 1] += -W * (mx * ux + mz * uz);
}

// Pressure seismograms as adjoint sources: for step k = *seg_k0 + slot (if
// k >= 0), mu(g) += M^-1(g) (-sum over the receivers around g of h g_k), over
// the n points that receivers touch (CSR: start, receiver, weight; fixed
// order).
__global__ void __launch_bounds__(128) k_adj_psrc(float *__restrict__ mu, const float *__restrict__ minv,
                                                  const int *__restrict__ pts, const int *__restrict__ start,
                                                  const int *__restrict__ rec, const float *__restrict__ hw,
                                                  const float *__restrict__ gtab, const int *__restrict__ seg_k0,
                                                  int slot, int nrec, int n) {
  const int k = *seg_k0 + slot;
  if (k < 0) return;
  const float *g_k = gtab + size_t(k) * nrec * 2;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int i = start[j]; i < start[j + 1]; ++i) s = s + hw[i] * g_k[2 * rec[i]];
    const int g = pts[j];
    mu[g] += minv[g] * (-1.f * s);
  }
}

// Acoustic pressure sources carry the source array l / kappa: per source
// element point (t = s * 25 + q) sum mu_k(g) f_k over the steps (the kappa
// derivative of the source term is -that * l / kappa^2), for step k =
// *seg_k0 + slot.
// src_id (null: s itself) is the source's column in the STF table [nstep][stf_cols]
// when only some of the model's sources lie in the acoustic medium.
__global__ void __launch_bounds__(128) k_adj_srcterm(float *__restrict__ acc, const float *__restrict__ mu,
                                                     const int *__restrict__ ibool, const int *__restrict__ src_ce,
                                                     const float *__restrict__ stf, const int *__restrict__ seg_k0,
                                                     int slot, int nsrc, int nstep, const int *__restrict__ src_id,
                                                     int stf_cols) {
  const int k = *seg_k0 + slot;
  if (k >= nstep) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nsrc * NP; t += gridDim.x * blockDim.x) {
    const int s = t / NP, q = t - s * NP;
    const int g = ibool[size_t(src_ce[s]) * NP + q];
    acc[t] += mu[g] * stf[size_t(k) * stf_cols + (src_id ? src_id[s] : s)];
  }
}

// Transposed acoustic-elastic coupling of a conforming interface (one
// partner per interface point), for the coupled sweep.  Forward, the
// acoustic force at interface point p takes n_p . u~_el(q_p) and the elastic
// force at q takes n'_q chi_dd'(p_q) (k_update / coupling_entry).  So
//   elastic lu~(q) += n_p mu_ac(p)        (p = other[q], n = the acoustic normal at p)
//   acoustic adjoint of chi_dd'(p) += n'_q . mu_el(q)   (q = other[p], n' = the elastic normal at q)
// other, nx, nz are indexed by this medium's interface point (< niface);
// omu is the other medium's mu.
struct AdjCoupling {
  const int *__restrict__ other;
  const float *__restrict__ nx, *__restrict__ nz;
  const float *__restrict__ omu;
  int niface;
};

// Per point: lu~ = lu + sum of the element-point results (colour order);
// G += mu_k . a'_k; then the transposed predictor and mu_(k-1).  lv holds
// lv~ (Stacey already applied).  One thread per point.  CPL (coupled sweep):
// the elastic post (NC 2) adds the acoustic mu_k to lu~ at interface points,
// the acoustic post (NC 1, after the elastic one) adds the elastic mu_(k-1)
// to the adjoint acceleration before B.
template <int NC, bool CPL = false>
__global__ void __launch_bounds__(256) k_adj_post(float *__restrict__ lu, float *__restrict__ lv,
                                                  float *__restrict__ mu, float *__restrict__ grho,
                                                  const float *__restrict__ af,
                                                  const float *__restrict__ minv,
                                                  const float *__restrict__ r,
                                                  const int *__restrict__ inv_start, int npts, float dt,
                                                  float dt2, float dtsq2, AdjCoupling cp = AdjCoupling{}) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < npts; g += gridDim.x * blockDim.x) {
    float s[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) s[c] = 0.f;
    for (int k = inv_start[g]; k < inv_start[g + 1]; ++k) {
#pragma unroll
      for (int c = 0; c < NC; ++c) s[c] = s[c] + r[size_t(k) * NC + c];
    }
    float cpa = 0.f;
    if (CPL && g < cp.niface) {
      const int o2 = cp.other[g];
      if (NC == 2) {
        const float m = cp.omu[o2];
        s[0] = s[0] + cp.nx[g] * m;
        s[NC - 1] = s[NC - 1] + cp.nz[g] * m;
      } else {
        cpa = cp.nx[g] * cp.omu[2 * size_t(o2)] + cp.nz[g] * cp.omu[2 * size_t(o2) + 1];
      }
    }
    const size_t o = size_t(g) * NC;
    float ma = mu[o] * af[o];
    if (NC == 2) ma = ma + mu[o + NC - 1] * af[o + NC - 1];
    grho[g] += ma;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const float l = lu[o + c] + s[c];
      const float v = lv[o + c];
      const float nv = dt * l + v;
      float la = dtsq2 * l + dt2 * v;
      if (CPL && NC == 1) la = la + cpa;
      lu[o + c] = l;
      lv[o + c] = nv;
      mu[o + c] = __fmul_rn(minv[o + c], __fadd_rn(la, __fmul_rn(dt2, nv)));
    }
  }
}

// Start of a recording step (one block): store the predicted velocity v~ of
// the step at the Stacey points (the step's element kernels read v~ next),
// then set the step counter to the segment's next step.
template <int NC>
__global__ void __launch_bounds__(512) k_record_begin(SegRecord *__restrict__ rec,
                                                      const float *__restrict__ v, int *step) {
  const int i = rec->i, n = rec->nst;
  float *dst = rec->vst + size_t(i) * rec->vstride;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
#pragma unroll
    for (int c = 0; c < NC; ++c) dst[size_t(j) * NC + c] = v[size_t(rec->st_pt[j]) * NC + c];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *step = rec->k0 + i;
    rec->i = i + 1;
  }
}

// Model dependence of the Stacey terms, per element-local boundary point i
// (global point g, Stacey slot j, unnormalised normal n, |n| = j1, edge
// weight wq).  The traction is -C v~ with C = wq j1 [(rvp - rvs) n n^T / j1^2
// + rvs I] and the implicit mass term adds dt/2 wq j1 [(nx + nz) n_c (rvp -
// rvs) / j1^2 + rvs] to M_c, so per step
//   dL/drvp = -wq j1 (A1 + dt/2 A3),  dL/drvs = -wq j1 (A2 - A1 + dt/2 (A4 - A3))
// with A1 = (mu.n)(n.v~)/j1^2, A2 = mu.v~, A3 = (nx + nz)/j1^2 sum_c mu_c n_c a'_c,
// A4 = mu.a'.  The four sums are accumulated per point (acc[4 i + 0..3]).
template <int NC>
__device__ __forceinline__ void adj_stacey_grad(const int *__restrict__ lb_g, const int *__restrict__ lb_j,
                                                const float4 *__restrict__ geo, const float *__restrict__ mu,
                                                const float *__restrict__ vst, const float *__restrict__ af,
                                                float *__restrict__ acc, int n, int first, int stride) {
  if constexpr (NC == 1) {
    // SH: C = wq j1 rvs, only A2 = mu v~ and A4 = mu a'
    for (int i = first; i < n; i += stride) {
      const int g = lb_g[i];
      const float m = mu[g];
      float4 t = reinterpret_cast<float4 *>(acc)[i];
      t.y += geo[i].x * (m * vst[lb_j[i]]);     // x: 1, or the acoustic free-surface mask
      t.w += m * af[g];
      reinterpret_cast<float4 *>(acc)[i] = t;
    }
  } else {
    for (int i = first; i < n; i += stride) {
      const int g = lb_g[i];
      const float4 q = geo[i];
      const float2 m = reinterpret_cast<const float2 *>(mu)[g];
      const float2 v = reinterpret_cast<const float2 *>(vst)[lb_j[i]];
      const float2 a = reinterpret_cast<const float2 *>(af)[g];
      const float inv = 1.0f / (q.z * q.z);
      const float mn = m.x * q.x + m.y * q.y, vn = v.x * q.x + v.y * q.y;
      float4 t = reinterpret_cast<float4 *>(acc)[i];
      t.x += mn * vn * inv;
      t.y += m.x * v.x + m.y * v.y;
      t.z += (q.x + q.y) * inv * (m.x * q.x * a.x + m.y * q.y * a.y);
      t.w += m.x * a.x + m.y * a.y;
      reinterpret_cast<float4 *>(acc)[i] = t;
    }
  }
}

// Stacey part of the transposed step at the start of a reverse step, one
// launch: blocks [0, nb_grad) accumulate the impedance terms per
// element-local boundary point, the others apply lv -= C mu per Stacey point
// (C symmetric 2x2 per point: xx, xz, zz; SH: the scalar in the xx slot).
struct AdjStaceyArgs {
  const int *lb_g, *lb_j;
  const float4 *geo;
  const float *mu, *vst, *af;
  float *acc;
  int nlb;
  float *lv;
  const int *pt;
  const float *cm;
  int nst;
  int nb_grad;
};

template <int NC>
__global__ void __launch_bounds__(256) k_adj_stacey(AdjStaceyArgs S) {
  if (int(blockIdx.x) < S.nb_grad) {
    adj_stacey_grad<NC>(S.lb_g, S.lb_j, S.geo, S.mu, S.vst, S.af, S.acc, S.nlb,
                    blockIdx.x * blockDim.x + threadIdx.x, S.nb_grad * blockDim.x);
    return;
  }
  const int stride = (gridDim.x - S.nb_grad) * blockDim.x;
  for (int j = (blockIdx.x - S.nb_grad) * blockDim.x + threadIdx.x; j < S.nst; j += stride) {
    const int g = S.pt[j];
    if (NC == 1) {
      S.lv[g] -= S.cm[3 * j] * S.mu[g];    // SH: C scalar in the xx slot
      continue;
    }
    const float mx = S.mu[2 * g], mz = S.mu[2 * g + 1];
    S.lv[2 * g] -= S.cm[3 * j] * mx + S.cm[3 * j + 1] * mz;
    S.lv[2 * g + 1] -= S.cm[3 * j + 1] * mx + S.cm[3 * j + 2] * mz;
  }
}

// Point the recording at one segment buffer and set the step counter to the
// segment's first step.
__global__ void k_set_segment(SegRecord *rec, int *step, float *u, float *a, float *vst, int k0) {
  rec->u = u;
  rec->a = a;
  rec->vst = vst;
  rec->k0 = k0;
  rec->i = 0;
  *step = k0;
}

// Step counter after a recorded segment.
__global__ void k_set_step(int *step, int k) { *step = k; }

// total += segment sum with Kahan compensation; segment sum cleared.
__global__ void __launch_bounds__(256) k_kahan_fold(float *__restrict__ total, float *__restrict__ comp,
                                                    float *__restrict__ seg, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float y = __fsub_rn(seg[i], comp[i]);
    const float t = __fadd_rn(total[i], y);
    comp[i] = __fsub_rn(__fsub_rn(t, total[i]), y);
    total[i] = t;
    seg[i] = 0.f;
  }
}

}  // namespace dev
}  // namespace sfg
