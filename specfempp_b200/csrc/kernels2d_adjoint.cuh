// Discrete adjoint of the 2D elastic P-SV time step (FP32), for rho / kappa /
// mu gradients of a seismogram misfit.
//
// Forward step k (the library's arithmetic, end-of-step state u, v, a):
//   predictor   u~ = u + dt v + dt^2/2 a,   v~ = v + dt/2 a
//   forces      a' = B (f_k - K u~ - C v~)            (B = M_eff^-1, diagonal)
//   corrector   v' = v~ + dt/2 a',  u' = u~;  seismogram d_k = R u'
// Reverse sweep of step k, for adjoint state (lu, lv, la) of (u', v', a')
// and g_k = dL/dd_k:
//   mu  = B (la + dt/2 lv)                              k_adj_pre
//   lu~ = lu + R^T g_k - K mu                           k_adj_elem (-K mu, R^T g_k per element point)
//                                                       + k_adj_post (per-point sum)
//   lv~ = lv - C mu                                     k_adj_stacey
//   (lu, lv, la) <- (lu~, dt lu~ + lv~, dt^2/2 lu~ + dt/2 lv~)
// and the model gradient of the step, per element GLL point p with
// W_p = w_x w_z |J|:
//   dL/dkappa_p += -W_p (div mu)(div u~)
//   dL/dmu_p    += -W_p [4/3 (mxx uxx + mzz uzz) - 2/3 (mxx uzz + mzz uxx)
//                        + (mxz + mzx)(uxz + uzx)]
//   dL/drho_p   += -W_p mu . a'        (mass part of B)
// kappa is the bulk modulus the reference stores (lambda + 2mu = kappa +
// 4/3 mu, include/medium/dim2/elastic/isotropic/properties.hpp:71-91).  The
// per-step terms are summed in FP32 over a checkpoint segment and folded into
// a compensated (Kahan) total once per segment.  These are the exact
// derivatives of the discrete forward model; the reference's continuous
// kernels (include/medium/dim2/elastic/isotropic/frechet_derivative.hpp:55-181)
// carry the same strain products (its mu bracket is half of the one above and
// its kappa prefactor is lambda + mu), integrated in time with -dt.
#pragma once

#include "kernels2d.cuh"

namespace sfg {
namespace dev {

struct AdjArgs {
  const int *__restrict__ ibool;
  const float *__restrict__ xix, *__restrict__ xiz, *__restrict__ gax, *__restrict__ gaz,
      *__restrict__ jac, *__restrict__ prop0, *__restrict__ prop1;
  const float *__restrict__ mu;      // adjoint field B (la + dt/2 lv) [nglob][2]
  const float *__restrict__ uf;      // forward u~ of the step [nglob][2]
  const float *__restrict__ af;      // forward a' of the step [nglob][2]
  float *__restrict__ r;             // element-point results [nspec*25][2]
  float *__restrict__ seg_k, *__restrict__ seg_m, *__restrict__ seg_r;  // segment sums [nspec*25]
  const int *__restrict__ ad_head, *__restrict__ ad_next;  // receivers per element
  const float *__restrict__ ad_h;    // receiver Lagrange weights [nrec][25]
  const float *__restrict__ ad_g;    // dL/d seismogram of this step [nrec][2]
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
  const float2 a2 = act ? reinterpret_cast<const float2 *>(A.af)[g] : make_float2(0.f, 0.f);
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
  for (int k = rh; k >= 0; k = A.ad_next[k]) {
    const float h = A.ad_h[size_t(k) * NP + q];
    r[0] += A.ad_g[2 * k] * h;
    r[1] += A.ad_g[2 * k + 1] * h;
  }
  reinterpret_cast<float2 *>(A.r)[p] = make_float2(r[0], r[1]);
  // gradient terms of this step, summed over the segment
  const float W = sw[ix] * sw[iz] * jac;
  const float divm = mxx + mzz, divu = uxx + uzz;
  const float tk = -W * (divm * divu);
  const float tm = -W * ((4.f / 3.f) * (mxx * uxx + mzz * uzz) - (2.f / 3.f) * (mxx * uzz + mzz * uxx) +
                         (mxz + mzx) * (uxz + uzx));
  const float tr = -W * (m2.x * a2.x + m2.y * a2.y);
  A.seg_k[p] += tk;
  A.seg_m[p] += tm;
  A.seg_r[p] += tr;
}

// mu = B (la + dt/2 lv)
__global__ void __launch_bounds__(256) k_adj_pre(const float *__restrict__ la, const float *__restrict__ lv,
                                                 const float *__restrict__ minv, float *__restrict__ mu,
                                                 int n, float dt2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    mu[i] = __fmul_rn(minv[i], __fadd_rn(la[i], __fmul_rn(dt2, lv[i])));
}

// lu~ = lu + sum of the element-point results (colour order); then the
// transposed predictor.  One thread per point.
__global__ void __launch_bounds__(256) k_adj_post(float *__restrict__ lu, float *__restrict__ lv,
                                                  float *__restrict__ la, const float *__restrict__ r,
                                                  const int *__restrict__ inv_start,
                                                  const int *__restrict__ inv_idx, int npts, float dt,
                                                  float dt2, float dtsq2) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < npts; g += gridDim.x * blockDim.x) {
    float s0 = 0.f, s1 = 0.f;
    for (int k = inv_start[g]; k < inv_start[g + 1]; ++k) {
      const float2 t = reinterpret_cast<const float2 *>(r)[inv_idx[k]];
      s0 = s0 + t.x;
      s1 = s1 + t.y;
    }
    const float2 u = reinterpret_cast<const float2 *>(lu)[g];
    const float2 v = reinterpret_cast<const float2 *>(lv)[g];
    const float lux = u.x + s0, luz = u.y + s1;
    reinterpret_cast<float2 *>(lu)[g] = make_float2(lux, luz);
    reinterpret_cast<float2 *>(lv)[g] = make_float2(dt * lux + v.x, dt * luz + v.y);
    reinterpret_cast<float2 *>(la)[g] = make_float2(dtsq2 * lux + dt2 * v.x, dtsq2 * luz + dt2 * v.y);
  }
}

// Stacey part of the transposed step on the absorbing points:
// lv -= C mu, la -= dt/2 C mu (C symmetric 2x2 per point: xx, xz, zz).
__global__ void __launch_bounds__(256) k_adj_stacey(float *__restrict__ lv, float *__restrict__ la,
                                                    const float *__restrict__ mu,
                                                    const int *__restrict__ pt,
                                                    const float *__restrict__ cm, int n, float dt2) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int g = pt[j];
    const float mx = mu[2 * g], mz = mu[2 * g + 1];
    const float cx = cm[3 * j] * mx + cm[3 * j + 1] * mz;
    const float cz = cm[3 * j + 1] * mx + cm[3 * j + 2] * mz;
    lv[2 * g] -= cx;
    lv[2 * g + 1] -= cz;
    la[2 * g] -= dt2 * cx;
    la[2 * g + 1] -= dt2 * cz;
  }
}

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
