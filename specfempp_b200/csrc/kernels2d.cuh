// sm_100a kernels of the 2D spectral-element time step (FP32).
//
// One time step of one medium is: [colour passes of the element kernel]
// -> [receiver kernel] -> [point update kernel].
//
// * Element kernel (stiffness): one thread per element GLL point, E elements
//   per block (25*E threads, element-local arrays [element][25] so a block
//   reads one contiguous run of each geometry array).  The displacement is
//   gathered through ibool into shared memory, the 5-term Lagrange-derivative
//   contractions and the stress run in registers, the stress integrand F goes
//   back to shared memory for the divergence, and the epilogue adds Stacey
//   traction, the acoustic/elastic coupling term and point sources before a
//   plain (non-atomic) += into the accumulator.  Elements of one launch share
//   no global point (mesh colouring), so the assembly is race-free and its
//   summation order is fixed: results are deterministic.
//   Reference: include/kokkos_kernels/impl/compute_stiffness_interaction.tpp:140-247,
//   include/algorithms/gradient.hpp:40-82, divergence.hpp:41-74,
//   include/medium/dim2/*/isotropic/stress.hpp, core/specfem/point/stress.hpp:166-183,
//   include/boundary_conditions/stacey/stacey.tpp:50-80,130-146,296-326,
//   include/boundary_conditions/dirichlet/dirichlet.hpp:38-62,
//   include/kokkos_kernels/impl/compute_coupling.tpp:21-115,
//   include/kokkos_kernels/impl/compute_source_interaction.tpp:17-104.
// * Point update: a = accum * M^-1, the Newmark corrector of this step and
//   the predictor of the next step in one streaming pass; the accumulator is
//   cleared for the next step (divide_mass_matrix.tpp:10-65, newmark.tpp:10-128).
// * Receiver kernel: one warp per receiver, Lagrange interpolation of the
//   corrected fields (compute_seismogram.tpp:19-171).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sfg {
namespace dev {

constexpr int NG = 5;
constexpr int NP = 25;

struct Quad {
  float hp[NP];    // hp[i*5+j] = l'_j(xi_i)
  float hpw[NP];   // hp[l*5+i] * w[l]
  float w[NG];
};

struct ElemArgs {
  const int *__restrict__ ibool;
  const float *__restrict__ xix, *__restrict__ xiz, *__restrict__ gax, *__restrict__ gaz,
      *__restrict__ jac, *__restrict__ prop0, *__restrict__ prop1;
  const int *__restrict__ bc_slot;
  const float *__restrict__ bc_w, *__restrict__ bc_nx, *__restrict__ bc_nz, *__restrict__ bc_j1,
      *__restrict__ bc_imp0, *__restrict__ bc_imp1, *__restrict__ bc_keep;
  const int *__restrict__ cp_slot;
  const float *__restrict__ cp_nx, *__restrict__ cp_nz;
  const int *__restrict__ cp_other;
  const float *__restrict__ other;     // elastic: acoustic chi_dd; acoustic: elastic u (float2)
  const int *__restrict__ src_head, *__restrict__ src_next;
  const float *__restrict__ src_arr;   // [nsrc][2][25]
  const float *__restrict__ stf;       // [nstep][nsrc]
  int nsrc, nstep;
  const int *__restrict__ step;        // device step counter
  const float *__restrict__ u, *__restrict__ v;
  float *__restrict__ accum;
  int e0, e1;
  Quad quad;
};

// 2D elastic P-SV, two components.
template <int E>
__global__ void __launch_bounds__(NP * E) k_stiffness_psv(ElemArgs A) {
  __shared__ float2 su[NP * E];
  __shared__ float4 sF[NP * E];
  __shared__ float shp[NP], shpw[NP], sw[NG];
  const int tid = threadIdx.x;
  if (tid < NP) { shp[tid] = A.quad.hp[tid]; shpw[tid] = A.quad.hpw[tid]; }
  if (tid < NG) sw[tid] = A.quad.w[tid];
  const int le = tid / NP, q = tid - le * NP;
  const int e = A.e0 + blockIdx.x * E + le;
  const bool act = e < A.e1;
  const size_t p = size_t(e) * NP + q;
  const float2 *u2 = reinterpret_cast<const float2 *>(A.u);
  int g = 0;
  float2 uu = make_float2(0.f, 0.f);
  if (act) {
    g = __ldg(A.ibool + p);
    uu = u2[g];
  }
  su[tid] = uu;
  __syncthreads();
  const int iz = q / NG, ix = q - iz * NG;
  const int rb = le * NP + iz * NG, cb = le * NP + ix;
  float dxi0 = 0.f, dxi1 = 0.f, dga0 = 0.f, dga1 = 0.f;
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    const float hx = shp[ix * NG + l], hz = shp[iz * NG + l];
    const float2 ur = su[rb + l], uc = su[cb + l * NG];
    dxi0 = fmaf(hx, ur.x, dxi0);
    dxi1 = fmaf(hx, ur.y, dxi1);
    dga0 = fmaf(hz, uc.x, dga0);
    dga1 = fmaf(hz, uc.y, dga1);
  }
  float4 F = make_float4(0.f, 0.f, 0.f, 0.f);
  if (act) {
    const float xix = __ldg(A.xix + p), xiz = __ldg(A.xiz + p), gax = __ldg(A.gax + p),
                gaz = __ldg(A.gaz + p), jac = __ldg(A.jac + p);
    const float l2m = __ldg(A.prop0 + p), mu = __ldg(A.prop1 + p);
    const float du00 = xix * dxi0 + gax * dga0, du01 = xiz * dxi0 + gaz * dga0;
    const float du10 = xix * dxi1 + gax * dga1, du11 = xiz * dxi1 + gaz * dga1;
    const float lam = l2m - 2.f * mu;
    const float sxx = l2m * du00 + lam * du11;
    const float szz = l2m * du11 + lam * du00;
    const float sxz = mu * (du01 + du10);
    F.x = jac * (sxx * xix + sxz * xiz);
    F.y = jac * (sxx * gax + sxz * gaz);
    F.z = jac * (sxz * xix + szz * xiz);
    F.w = jac * (sxz * gax + szz * gaz);
  }
  sF[tid] = F;
  __syncthreads();
  if (!act) return;
  float t1x = 0.f, t1z = 0.f, t2x = 0.f, t2z = 0.f;
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    const float4 fr = sF[rb + l], fc = sF[cb + l * NG];
    const float h1 = shpw[l * NG + ix], h2 = shpw[l * NG + iz];
    t1x = fmaf(fr.x, h1, t1x);
    t1z = fmaf(fr.z, h1, t1z);
    t2x = fmaf(fc.y, h2, t2x);
    t2z = fmaf(fc.w, h2, t2z);
  }
  float ax = -(sw[iz] * t1x + sw[ix] * t2x);
  float az = -(sw[iz] * t1z + sw[ix] * t2z);
  const int bs = __ldg(A.bc_slot + e);
  if (bs >= 0) {
    const size_t k = size_t(bs) * NP + q;
    const float wq = A.bc_w[k];
    if (wq != 0.f) {
      const float2 vv = reinterpret_cast<const float2 *>(A.v)[g];
      const float nx = A.bc_nx[k], nz = A.bc_nz[k], j1 = A.bc_j1[k];
      const float rvp = A.bc_imp0[k], rvs = A.bc_imp1[k];
      const float vn = vv.x * nx + vv.y * nz;
      const float fx = ((vn * nx / (j1 * j1)) * (rvp - rvs)) + vv.x * rvs;
      const float fz = ((vn * nz / (j1 * j1)) * (rvp - rvs)) + vv.y * rvs;
      ax += -1.f * fx * j1 * wq;
      az += -1.f * fz * j1 * wq;
    }
  }
  const int cs = __ldg(A.cp_slot + e);
  if (cs >= 0) {
    const size_t k = size_t(cs) * NP + q;
    const int o = A.cp_other[k];
    if (o >= 0) {
      const float chi_dd = A.other[o];
      ax += A.cp_nx[k] * chi_dd;
      az += A.cp_nz[k] * chi_dd;
    }
  }
  int s = __ldg(A.src_head + e);
  if (s >= 0) {
    const int step = *A.step;
    while (s >= 0) {
      const float f = step < A.nstep ? A.stf[size_t(step) * A.nsrc + s] : 0.f;
      ax += f * A.src_arr[(size_t(s) * 2) * NP + q];
      az += f * A.src_arr[(size_t(s) * 2 + 1) * NP + q];
      s = A.src_next[s];
    }
  }
  float2 *acc2 = reinterpret_cast<float2 *>(A.accum);
  float2 acc = acc2[g];
  acc.x += ax;
  acc.y += az;
  acc2[g] = acc;
}

// One-component media: KIND 0 acoustic (potential chi), KIND 1 elastic SH.
template <int E, int KIND>
__global__ void __launch_bounds__(NP * E) k_stiffness_1c(ElemArgs A) {
  __shared__ float su[NP * E];
  __shared__ float2 sF[NP * E];
  __shared__ float shp[NP], shpw[NP], sw[NG];
  const int tid = threadIdx.x;
  if (tid < NP) { shp[tid] = A.quad.hp[tid]; shpw[tid] = A.quad.hpw[tid]; }
  if (tid < NG) sw[tid] = A.quad.w[tid];
  const int le = tid / NP, q = tid - le * NP;
  const int e = A.e0 + blockIdx.x * E + le;
  const bool act = e < A.e1;
  const size_t p = size_t(e) * NP + q;
  int g = 0;
  float uu = 0.f;
  if (act) {
    g = __ldg(A.ibool + p);
    uu = A.u[g];
  }
  su[tid] = uu;
  __syncthreads();
  const int iz = q / NG, ix = q - iz * NG;
  const int rb = le * NP + iz * NG, cb = le * NP + ix;
  float dxi = 0.f, dga = 0.f;
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    dxi = fmaf(shp[ix * NG + l], su[rb + l], dxi);
    dga = fmaf(shp[iz * NG + l], su[cb + l * NG], dga);
  }
  float2 F = make_float2(0.f, 0.f);
  if (act) {
    const float xix = __ldg(A.xix + p), xiz = __ldg(A.xiz + p), gax = __ldg(A.gax + p),
                gaz = __ldg(A.gaz + p), jac = __ldg(A.jac + p);
    // acoustic: sigma = rho^-1 grad chi; SH: sigma = mu grad u_y
    const float c = KIND == 0 ? __ldg(A.prop0 + p) : __ldg(A.prop1 + p);
    const float s0 = c * (xix * dxi + gax * dga);
    const float s1 = c * (xiz * dxi + gaz * dga);
    F.x = jac * (s0 * xix + s1 * xiz);
    F.y = jac * (s0 * gax + s1 * gaz);
  }
  sF[tid] = F;
  __syncthreads();
  if (!act) return;
  float t1 = 0.f, t2 = 0.f;
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    t1 = fmaf(sF[rb + l].x, shpw[l * NG + ix], t1);
    t2 = fmaf(sF[cb + l * NG].y, shpw[l * NG + iz], t2);
  }
  float a = -(sw[iz] * t1 + sw[ix] * t2);
  const int bs = __ldg(A.bc_slot + e);
  if (bs >= 0) {
    const size_t k = size_t(bs) * NP + q;
    const float wq = A.bc_w[k];
    if (wq != 0.f) {
      const float imp = KIND == 0 ? A.bc_imp0[k] : A.bc_imp1[k];
      a += -1.f * (wq * A.bc_j1[k]) * imp * A.v[g];
    }
    a *= A.bc_keep[k];   // acoustic free surface (Dirichlet) zeroes the element term
  }
  if (KIND == 0) {
    const int cs = __ldg(A.cp_slot + e);
    if (cs >= 0) {
      const size_t k = size_t(cs) * NP + q;
      const int o = A.cp_other[k];
      if (o >= 0) {
        const float2 ue = reinterpret_cast<const float2 *>(A.other)[o];
        a += A.cp_nx[k] * ue.x + A.cp_nz[k] * ue.y;
      }
    }
  }
  int s = __ldg(A.src_head + e);
  if (s >= 0) {
    const int step = *A.step;
    while (s >= 0) {
      const float f = step < A.nstep ? A.stf[size_t(step) * A.nsrc + s] : 0.f;
      a += f * A.src_arr[(size_t(s) * 2) * NP + q];
      s = A.src_next[s];
    }
  }
  A.accum[g] += a;
}

struct UpdateArgs {
  float *__restrict__ u, *__restrict__ v, *__restrict__ accum;
  const float *__restrict__ minv;
  float *__restrict__ a_store;   // optional copy of the new acceleration
  int n;                         // nglob * ncomp
  float dt, dt2, dtsq2;
  int *flag;                     // set to 1 on a non-finite displacement
  int *step;
  int advance;                   // increment the step counter (last update of a step)
};

// a = accum * M^-1; v += dt/2 a (corrector); u += dt v + dt^2/2 a; v += dt/2 a
// (predictor of the next step); accum = 0.  Streams float4.
__global__ void __launch_bounds__(256) k_update(UpdateArgs A) {
  const int n4 = A.n >> 2;
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    float4 ac = reinterpret_cast<float4 *>(A.accum)[i];
    const float4 mi = reinterpret_cast<const float4 *>(A.minv)[i];
    float4 uu = reinterpret_cast<float4 *>(A.u)[i];
    float4 vv = reinterpret_cast<float4 *>(A.v)[i];
    float a[4] = {ac.x * mi.x, ac.y * mi.y, ac.z * mi.z, ac.w * mi.w};
    float *pu = &uu.x, *pv = &vv.x;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      pv[c] = pv[c] + A.dt2 * a[c];
      pu[c] = pu[c] + (A.dt * pv[c] + A.dtsq2 * a[c]);
      pv[c] = pv[c] + A.dt2 * a[c];
      bad |= !isfinite(pu[c]);
    }
    reinterpret_cast<float4 *>(A.u)[i] = uu;
    reinterpret_cast<float4 *>(A.v)[i] = vv;
    reinterpret_cast<float4 *>(A.accum)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (A.a_store) reinterpret_cast<float4 *>(A.a_store)[i] = make_float4(a[0], a[1], a[2], a[3]);
  }
  for (int i = (n4 << 2) + blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += stride) {
    const float a = A.accum[i] * A.minv[i];
    float vv = A.v[i] + A.dt2 * a;
    const float uu = A.u[i] + (A.dt * vv + A.dtsq2 * a);
    vv = vv + A.dt2 * a;
    A.u[i] = uu;
    A.v[i] = vv;
    A.accum[i] = 0.f;
    if (A.a_store) A.a_store[i] = a;
    bad |= !isfinite(uu);
  }
  if (bad) *A.flag = 1;
  if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) *A.step += 1;
}

struct RecArgs {
  int nrec;
  const int *__restrict__ rec_list;    // receivers of this medium
  const int *__restrict__ rec_elem;    // compute element in the medium
  const float *__restrict__ rec_h;     // [nrec][25]
  const int *__restrict__ ibool;
  const float *__restrict__ xix, *__restrict__ xiz, *__restrict__ gax, *__restrict__ gaz,
      *__restrict__ prop0, *__restrict__ prop1;
  const float *__restrict__ u, *__restrict__ v, *__restrict__ accum, *__restrict__ minv;
  int ncomp, acoustic;
  int ntypes;
  int types[4];
  int nsb, nsig, nrec_total;
  float dt2;
  const int *__restrict__ step;
  float *__restrict__ seis;            // [nsig][ntypes][nrec_total][2]
  Quad quad;
};

__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// One warp per receiver of one medium; runs before that medium's update, so
// it reconstructs the corrected velocity and the new acceleration from the
// accumulator.
__global__ void __launch_bounds__(32) k_receivers(RecArgs A) {
  __shared__ float sf[3][NP];
  const int step = *A.step;
  if (step % A.nsb != 0) return;
  const int isig = step / A.nsb;
  if (isig >= A.nsig) return;
  const int r = A.rec_list[blockIdx.x];
  const int ce = A.rec_elem[r];
  const int lane = threadIdx.x;
  const bool on = lane < NP;
  const int q = on ? lane : 0;
  const size_t p = size_t(ce) * NP + q;
  const int g = A.ibool[p];
  const float h = on ? A.rec_h[size_t(r) * NP + q] : 0.f;
  if (!A.acoustic) {
    for (int t = 0; t < A.ntypes; ++t) {
      float o[2] = {0.f, 0.f};
      if (A.types[t] == 3) {
        // pressure -(lambda + 2/3 mu) div u from the displacement gradient
        // (include/medium/dim2/elastic/isotropic/wavefield.hpp:57-89)
        float pr = 0.f;
        if (A.ncomp == 2) {
          const int iz = q / NG, ix = q - iz * NG;
          float dxi0 = 0.f, dxi1 = 0.f, dga0 = 0.f, dga1 = 0.f;
          for (int l = 0; l < NG; ++l) {
            const int gr = A.ibool[size_t(ce) * NP + iz * NG + l];
            const int gc = A.ibool[size_t(ce) * NP + l * NG + ix];
            const float hx = A.quad.hp[ix * NG + l], hz = A.quad.hp[iz * NG + l];
            dxi0 += hx * A.u[size_t(gr) * 2];
            dxi1 += hx * A.u[size_t(gr) * 2 + 1];
            dga0 += hz * A.u[size_t(gc) * 2];
            dga1 += hz * A.u[size_t(gc) * 2 + 1];
          }
          if (on) {
            const float dux = A.xix[p] * dxi0 + A.gax[p] * dga0;
            const float duz = A.xiz[p] * dxi1 + A.gaz[p] * dga1;
            const float l2m = A.prop0[p], mu = A.prop1[p];
            pr = -1.f * ((l2m - 2.f * mu + (2.f / 3.f) * mu) * (dux + duz));
          }
        }
        o[0] = warp_sum(h * pr);
        if (lane == 0) {
          float *dst = A.seis + ((size_t(isig) * A.ntypes + t) * A.nrec_total + r) * 2;
          dst[0] = o[0];
          dst[1] = 0.f;
        }
        continue;
      }
      for (int c = 0; c < A.ncomp; ++c) {
        const size_t k = size_t(g) * A.ncomp + c;
        const float a = A.accum[k] * A.minv[k];
        float val = 0.f;
        switch (A.types[t]) {
          case 0: val = A.u[k]; break;
          case 1: val = A.v[k] + A.dt2 * a; break;
          case 2: val = a; break;
          default: val = 0.f; break;
        }
        o[c] = warp_sum(h * val);
      }
      if (lane == 0) {
        float *dst = A.seis + ((size_t(isig) * A.ntypes + t) * A.nrec_total + r) * 2;
        dst[0] = o[0];
        dst[1] = A.ncomp > 1 ? o[1] : 0.f;
      }
    }
    return;
  }
  // acoustic: displacement-like outputs are rho^-1 grad(field); pressure = -chi_dd
  const float a = A.accum[g] * A.minv[g];
  if (on) {
    sf[0][q] = A.u[g];
    sf[1][q] = A.v[g] + A.dt2 * a;
    sf[2][q] = a;
  }
  __syncwarp();
  const int iz = q / NG, ix = q - iz * NG;
  for (int t = 0; t < A.ntypes; ++t) {
    const int ty = A.types[t];
    float ox = 0.f, oz = 0.f;
    if (ty == 3) {
      ox = warp_sum(on ? h * (-1.f * sf[2][q]) : 0.f);
    } else {
      const int f = ty < 3 ? ty : 0;
      float dxi = 0.f, dga = 0.f;
      for (int l = 0; l < NG; ++l) {
        dxi += A.quad.hp[ix * NG + l] * sf[f][iz * NG + l];
        dga += A.quad.hp[iz * NG + l] * sf[f][l * NG + ix];
      }
      float gx = 0.f, gz = 0.f;
      if (on) {
        const float ri = A.prop0[p];
        gx = ri * (A.xix[p] * dxi + A.gax[p] * dga);
        gz = ri * (A.xiz[p] * dxi + A.gaz[p] * dga);
      }
      ox = warp_sum(h * gx);
      oz = warp_sum(h * gz);
    }
    if (lane == 0) {
      float *dst = A.seis + ((size_t(isig) * A.ntypes + t) * A.nrec_total + r) * 2;
      dst[0] = ox;
      dst[1] = oz;
    }
  }
}

}  // namespace dev
}  // namespace sfg
