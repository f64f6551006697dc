// sm_100a kernels of the 2D spectral-element time step (FP32).
//
// One time step is: [one element-kernel launch per mesh colour, covering the
// elements of that colour in both media] -> [acoustic receivers] ->
// [acoustic point update] -> [elastic receivers] -> [elastic point update].
//
// * Element kernel (stiffness): one thread per element GLL point, E elements
//   per block (25*E threads; element-local arrays are [element][25] so a block
//   reads one contiguous run of each geometry array).  Every load that does not
//   depend on shared memory (index, Jacobian, material, the gathered
//   displacement and the accumulator value) is issued before the first
//   barrier.  The 5-term Lagrange-derivative contractions and the stress run
//   in registers, the stress integrand F goes through shared memory for the
//   divergence, and the epilogue adds Stacey traction, the acoustic free
//   surface and point sources before a plain (non-atomic) += into the
//   accumulator.  Elements of one launch share no global point (mesh
//   colouring), so assembly is race-free with a fixed summation order: results
//   are deterministic and independent of the launch shape.
//   Reference: include/kokkos_kernels/impl/compute_stiffness_interaction.tpp:140-247,
//   include/algorithms/gradient.hpp:40-82, divergence.hpp:41-74,
//   include/medium/dim2/*/isotropic/stress.hpp, core/specfem/point/stress.hpp:166-183,
//   include/boundary_conditions/stacey/stacey.tpp:50-80,130-146,296-326,
//   include/boundary_conditions/dirichlet/dirichlet.hpp:38-62,
//   include/kokkos_kernels/impl/compute_source_interaction.tpp:17-104.
// * Point update: a = (accum + coupling) * M^-1 and the Newmark corrector of
//   this step; inside a run the predictor of the next step is fused into the
//   same float4 streaming pass, the last step of a run stops after the
//   corrector (so the fields read back are the reference's end-of-step state)
//   and k_predict applies the pending predictor when the next run starts
//   (divide_mass_matrix.tpp:10-65, newmark.tpp:10-128).  The acoustic/elastic
//   coupling term (compute_coupling.tpp:21-115) is linear in the other
//   medium's field at the same point; the interface points are numbered first
//   in each medium, so the update adds it for indices below niface only.
// * Receiver kernel: one warp per receiver, Lagrange interpolation of the
//   corrected fields (compute_seismogram.tpp:19-171).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sfg {
namespace dev {

constexpr int NG = 5;
constexpr int NP = 25;

// Paired FP32 fused multiply-add (sm_100 FFMA2): each lane rounds exactly as
// the scalar fmaf, so 5-term contractions (explicit fmaf in every kernel)
// can run two at a time with unchanged results.  Products and sums stay
// scalar: paired multiplies feeding paired adds are fused into FFMA2 by the
// code generator even with explicit rounding, which would change rounding.
__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

struct Quad {
  float hp[NP];    // hp[i*5+j] = l'_j(xi_i)
  float hpw[NP];   // hp[l*5+i] * w[l]
  float w[NG];
};

// Element arrays of one medium.
struct MedArgs {
  const int *__restrict__ ibool;
  const float *__restrict__ xix, *__restrict__ xiz, *__restrict__ gax, *__restrict__ gaz,
      *__restrict__ jac, *__restrict__ prop0, *__restrict__ prop1;
  const float *__restrict__ prop2, *__restrict__ prop3, *__restrict__ prop4, *__restrict__ prop5;  // anisotropic
  const float *__restrict__ prop6, *__restrict__ prop7, *__restrict__ prop8;  // poroelastic damping
  const int *__restrict__ bc_slot;
  const float *__restrict__ bc_w, *__restrict__ bc_nx, *__restrict__ bc_nz, *__restrict__ bc_j1,
      *__restrict__ bc_imp0, *__restrict__ bc_imp1, *__restrict__ bc_keep;
  const float *__restrict__ bc_imp2;   // Cosserat rotational impedance
  const int *__restrict__ src_head;
  const float *__restrict__ u, *__restrict__ v;
  float *__restrict__ accum;
  // owner-computes: element results in point-major order, the contribution
  // of element point p at r[slot[p]] (each point's contributions adjacent,
  // in increasing element order)
  float *__restrict__ r;
  const int *__restrict__ slot;
  int e0, e1;      // element range of the colour
  int nblocks;     // blocks of this medium in the launch
};

struct StiffArgs {
  MedArgs el, ac;
  const int *__restrict__ src_next;
  const float *__restrict__ src_arr;   // [nsrc][2][25]
  const float *__restrict__ src_arr2;  // poroelastic fluid rows [nsrc][2][25] (else null)
  const float *__restrict__ stf;       // [nstep][nsrc]
  int nsrc, nstep;
  const int *__restrict__ step;        // device step counter
  Quad quad;
};

__device__ __forceinline__ void load_quad(const Quad &Q, float *shp, float *shpw, float *sw,
                                          int tid) {
  if (tid < NP) { shp[tid] = Q.hp[tid]; shpw[tid] = Q.hpw[tid]; }
  if (tid < NG) sw[tid] = Q.w[tid];
}

// Elastic element block; EK 0 = P-SV (two components), 1 = SH (one component),
// 2 = anisotropic P-SV (prop0..prop5 = c11, c13, c15, c33, c35, c55;
// include/medium/dim2/elastic/anisotropic/stress.hpp), 3 = isotropic Cosserat
// P-SV-T (u_x, u_z, rotation phi; prop0..prop3 = lambda, mu, nu, mu_c + nu_c;
// isotropic_cosserat/stress.hpp, cosserat_stress.hpp: the rows of u_x and u_z
// carry (sxx, szx) and (sxz, szz) with sxz += 2 nu phi, szx -= 2 nu phi, the
// rotation row (mu_c + nu_c) grad(phi); after the divergence the rotation
// gets -W (sxz - szx), W = w_x w_z |J| (compute_stiffness_interaction.tpp:
// 216-229, cosserat_couple_stress.hpp), then Stacey with the rotational
// impedance on phi (stacey.tpp:183-230)), 4 = isotropic poroelastic (solid
// u_x, u_z, fluid w_x, w_z; prop0..prop8 = H_Biot, mu_G, C_Biot, M_Biot,
// phi / tort, rho_f / rho_bar, eta_f k^-1 (xx, xz, zz);
// poroelastic/isotropic/stress.hpp: lambda_G = H - 2 mu_G, solid rows sigma -
// phi/tort sigma_p, fluid rows sigma_p - rho_f/rho_bar sigma; after the
// divergence the viscous damping of the fluid velocity, w_x w_z |J| eta_f k^-1
// v_f, added to the solid rows times phi/tort and taken from the fluid rows
// (damping.hpp, compute_stiffness_interaction.tpp:216-223)).
// LOCAL: write the element's contribution to its own slot of A.r (summed per
// point later by the update) instead of adding it into the accumulator.
template <int E, int EK, bool LOCAL>
__device__ __forceinline__ void elastic_block(const StiffArgs &S, const MedArgs &A, int ebase,
                                              unsigned char *smem, float *shp, float *shpw,
                                              float *sw) {
  constexpr int NC = EK == 1 ? 1 : (EK == 3 ? 3 : (EK == 4 ? 4 : 2));
  float *su = reinterpret_cast<float *>(smem);                                // [E][NC][25]
  float *sF = reinterpret_cast<float *>(smem + sizeof(float) * NP * E * NC);  // [E][NC][2][25]
  const int tid = threadIdx.x;
  const int le = tid / NP, q = tid - le * NP;
  const int e = ebase + le;
  const bool act = e < A.e1;
  const size_t p = size_t(act ? e : A.e0) * NP + q;
  // early loads: everything that does not need shared memory
  const int g = act ? __ldg(A.ibool + p) : 0;
  const float xix = __ldg(A.xix + p), xiz = __ldg(A.xiz + p), gax = __ldg(A.gax + p),
              gaz = __ldg(A.gaz + p), jac = __ldg(A.jac + p);
  const float c0 = __ldg(A.prop0 + p), mu = __ldg(A.prop1 + p);
  float uu[NC], acc[NC];
  if (NC == 4) {
    const float4 t = act ? reinterpret_cast<const float4 *>(A.u)[g] : make_float4(0.f, 0.f, 0.f, 0.f);
    uu[0] = t.x; uu[1 % NC] = t.y; uu[2 % NC] = t.z; uu[3 % NC] = t.w;
    if (!LOCAL) {
      const float4 r = act ? reinterpret_cast<const float4 *>(A.accum)[g] : make_float4(0.f, 0.f, 0.f, 0.f);
      acc[0] = r.x; acc[1 % NC] = r.y; acc[2 % NC] = r.z; acc[3 % NC] = r.w;
    }
  } else if (NC == 3) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      uu[c] = act ? A.u[size_t(g) * 3 + c] : 0.f;
      if (!LOCAL) acc[c] = act ? A.accum[size_t(g) * 3 + c] : 0.f;
    }
  } else if (NC == 2) {
    const float2 t = act ? reinterpret_cast<const float2 *>(A.u)[g] : make_float2(0.f, 0.f);
    uu[0] = t.x; uu[NC - 1] = t.y;
    if (!LOCAL) {
      const float2 r = act ? reinterpret_cast<const float2 *>(A.accum)[g] : make_float2(0.f, 0.f);
      acc[0] = r.x; acc[NC - 1] = r.y;
    }
  } else {
    uu[0] = act ? A.u[g] : 0.f;
    if (!LOCAL) acc[0] = act ? A.accum[g] : 0.f;
  }
  const int bs = act ? __ldg(A.bc_slot + e) : -1;
  const int src = act ? __ldg(A.src_head + e) : -1;
  const int iz = q / NG, ix = q - iz * NG;
  float dxi[NC], dga[NC];
  if (EK == 0) {
    // P-SV: the two components' contractions paired (FFMA2, rounding as fmaf)
    float2 *su2 = reinterpret_cast<float2 *>(smem);   // [E][25] (u_x, u_z)
    su2[le * NP + q] = make_float2(uu[0], uu[NC - 1]);
    __syncthreads();
    const float2 *fu = su2 + le * NP;
    float2 px = make_float2(0.f, 0.f), pg = make_float2(0.f, 0.f);
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      px = fma2(f2(shp[ix * NG + l]), fu[iz * NG + l], px);
      pg = fma2(f2(shp[iz * NG + l]), fu[l * NG + ix], pg);
    }
    dxi[0] = px.x; dxi[NC - 1] = px.y; dga[0] = pg.x; dga[NC - 1] = pg.y;
  } else {
#pragma unroll
  for (int c = 0; c < NC; ++c) su[(le * NC + c) * NP + q] = uu[c];
  __syncthreads();
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    dxi[c] = 0.f;
    dga[c] = 0.f;
    const float *fu = su + (le * NC + c) * NP;
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      dxi[c] = fmaf(shp[ix * NG + l], fu[iz * NG + l], dxi[c]);
      dga[c] = fmaf(shp[iz * NG + l], fu[l * NG + ix], dga[c]);
    }
  }
  }
  // stress (P-SV: isotropic Hooke with lambda+2mu = c0; SH: sigma = mu grad u_y)
  float Sx[NC], Sz[NC];
  float csxz = 0.f, cszx = 0.f;   // Cosserat sigma_xz, sigma_zx
  if (EK == 4) {
    const float du00 = xix * dxi[0] + gax * dga[0], du01 = xiz * dxi[0] + gaz * dga[0];
    const float du10 = xix * dxi[1 % NC] + gax * dga[1 % NC], du11 = xiz * dxi[1 % NC] + gaz * dga[1 % NC];
    const float du20 = xix * dxi[2 % NC] + gax * dga[2 % NC];
    const float du31 = xiz * dxi[3 % NC] + gaz * dga[3 % NC];
    const float C = __ldg(A.prop2 + p), M = __ldg(A.prop3 + p);
    const float pt = __ldg(A.prop4 + p), rr = __ldg(A.prop5 + p);
    const float lam = c0 - 2.0f * mu, l2m = lam + 2.0f * mu;   // c0 = H_Biot, mu = mu_G
    const float dw = du20 + du31;
    const float sxx = l2m * du00 + lam * du11 + C * dw;
    const float szz = l2m * du11 + lam * du00 + C * dw;
    const float sxz = mu * (du01 + du10);
    const float sp = C * (du00 + du11) + M * dw;
    Sx[0] = sxx - pt * sp; Sz[0] = sxz;
    Sx[1 % NC] = sxz; Sz[1 % NC] = szz - pt * sp;
    Sx[2 % NC] = sp - rr * sxx; Sz[2 % NC] = -1.0f * rr * sxz;
    Sx[3 % NC] = -1.0f * rr * sxz; Sz[3 % NC] = sp - rr * szz;
  } else if (EK == 3) {
    const float du00 = xix * dxi[0] + gax * dga[0], du01 = xiz * dxi[0] + gaz * dga[0];
    const float du10 = xix * dxi[1] + gax * dga[1], du11 = xiz * dxi[1] + gaz * dga[1];
    const float du20 = xix * dxi[NC - 1] + gax * dga[NC - 1], du21 = xiz * dxi[NC - 1] + gaz * dga[NC - 1];
    const float nu = __ldg(A.prop2 + p), mcn = __ldg(A.prop3 + p);
    const float lam = c0, dv = du00 + du11;        // c0 = lambda here
    const float sxx = lam * dv + 2.f * mu * du00;
    const float szz = lam * dv + 2.f * mu * du11;
    float sxz = mu * (du10 + du01) + nu * (du10 - du01);
    float szx = mu * (du01 + du10) + nu * (du01 - du10);
    szx -= 2.f * nu * uu[NC - 1];
    sxz += 2.f * nu * uu[NC - 1];
    csxz = sxz; cszx = szx;
    Sx[0] = sxx; Sz[0] = szx; Sx[1] = sxz; Sz[1] = szz;
    Sx[NC - 1] = mcn * du20; Sz[NC - 1] = mcn * du21;
  } else if (EK == 2) {
    const float du00 = xix * dxi[0] + gax * dga[0], du01 = xiz * dxi[0] + gaz * dga[0];
    const float du10 = xix * dxi[NC - 1] + gax * dga[NC - 1];
    const float du11 = xiz * dxi[NC - 1] + gaz * dga[NC - 1];
    const float c15 = __ldg(A.prop2 + p), c33 = __ldg(A.prop3 + p), c35 = __ldg(A.prop4 + p),
                c55 = __ldg(A.prop5 + p);
    const float sh = du10 + du01;
    const float sxx = c0 * du00 + mu * du11 + c15 * sh;     // c0 = c11, mu = c13 here
    const float szz = mu * du00 + c33 * du11 + c35 * sh;
    const float sxz = c15 * du00 + c35 * du11 + c55 * sh;
    Sx[0] = sxx; Sz[0] = sxz; Sx[NC - 1] = sxz; Sz[NC - 1] = szz;
  } else if (EK == 0) {
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
  float a[NC];
  if (EK == 0) {
    float2 *sF2 = reinterpret_cast<float2 *>(smem + sizeof(float) * NP * E * NC);   // [E][2][25]
    sF2[(le * 2 + 0) * NP + q] = make_float2(jac * (Sx[0] * xix + Sz[0] * xiz), jac * (Sx[NC - 1] * xix + Sz[NC - 1] * xiz));
    sF2[(le * 2 + 1) * NP + q] = make_float2(jac * (Sx[0] * gax + Sz[0] * gaz), jac * (Sx[NC - 1] * gax + Sz[NC - 1] * gaz));
    __syncthreads();
    if (!act) return;
    const float2 *g0 = sF2 + (le * 2 + 0) * NP, *g1 = sF2 + (le * 2 + 1) * NP;
    float2 t1 = make_float2(0.f, 0.f), t2 = make_float2(0.f, 0.f);
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      t1 = fma2(g0[iz * NG + l], f2(shpw[l * NG + ix]), t1);
      t2 = fma2(g1[l * NG + ix], f2(shpw[l * NG + iz]), t2);
    }
    a[0] = -(sw[iz] * t1.x + sw[ix] * t2.x);
    a[NC - 1] = -(sw[iz] * t1.y + sw[ix] * t2.y);
  } else {
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    sF[((le * NC + c) * 2 + 0) * NP + q] = jac * (Sx[c] * xix + Sz[c] * xiz);
    sF[((le * NC + c) * 2 + 1) * NP + q] = jac * (Sx[c] * gax + Sz[c] * gaz);
  }
  __syncthreads();
  if (!act) return;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const float *f0 = sF + ((le * NC + c) * 2 + 0) * NP;
    const float *f1 = sF + ((le * NC + c) * 2 + 1) * NP;
    float t1 = 0.f, t2 = 0.f;
#pragma unroll
    for (int l = 0; l < NG; ++l) {
      t1 = fmaf(f0[iz * NG + l], shpw[l * NG + ix], t1);
      t2 = fmaf(f1[l * NG + ix], shpw[l * NG + iz], t2);
    }
    a[c] = -(sw[iz] * t1 + sw[ix] * t2);
  }
  }
  if (EK == 3) a[NC - 1] -= (csxz - cszx) * (sw[ix] * sw[iz] * jac);   // couple stress
  if (EK == 4) {
    // viscous damping of the fluid motion; factor w_x w_z |J|
    const float4 vv = reinterpret_cast<const float4 *>(A.v)[g];
    const float fac = sw[ix] * sw[iz] * jac;
    const float exx = __ldg(A.prop6 + p), exz = __ldg(A.prop7 + p), ezz = __ldg(A.prop8 + p);
    const float viscx = fac * ((exx * vv.z) + (exz * vv.w));
    const float viscz = fac * ((exz * vv.z) + (ezz * vv.w));
    const float pt = __ldg(A.prop4 + p);
    a[0] += pt * viscx;
    a[1 % NC] += pt * viscz;
    a[2 % NC] -= viscx;
    a[3 % NC] -= viscz;
  }
  if (bs >= 0) {
    const size_t k = size_t(bs) * NP + q;
    const float wq = A.bc_w[k];
    if (wq != 0.f) {
      const float nx = A.bc_nx[k], nz = A.bc_nz[k], j1 = A.bc_j1[k];
      if (EK == 3) {
        const float vx = A.v[size_t(g) * 3], vz = A.v[size_t(g) * 3 + 1], vr = A.v[size_t(g) * 3 + 2];
        const float rvp = A.bc_imp0[k], rvs = A.bc_imp1[k];
        const float vn = vx * nx + vz * nz;
        const float fx = ((vn * nx / (j1 * j1)) * (rvp - rvs)) + vx * rvs;
        const float fz = ((vn * nz / (j1 * j1)) * (rvp - rvs)) + vz * rvs;
        a[0] += -1.f * fx * j1 * wq;
        a[1] += -1.f * fz * j1 * wq;
        a[NC - 1] += -1.f * A.bc_imp2[k] * vr * j1 * wq;
      } else if (EK != 1) {
        const float2 vv = reinterpret_cast<const float2 *>(A.v)[g];
        const float rvp = A.bc_imp0[k], rvs = A.bc_imp1[k];
        const float vn = vv.x * nx + vv.y * nz;
        const float fx = ((vn * nx / (j1 * j1)) * (rvp - rvs)) + vv.x * rvs;
        const float fz = ((vn * nz / (j1 * j1)) * (rvp - rvs)) + vv.y * rvs;
        a[0] += -1.f * fx * j1 * wq;
        a[NC - 1] += -1.f * fz * j1 * wq;
      } else {
        a[0] += -1.f * (wq * j1) * A.bc_imp1[k] * A.v[g];
      }
    }
  }
  if (src >= 0) {
    const int step = *S.step;
    for (int s = src; s >= 0; s = S.src_next[s]) {
      const float f = step < S.nstep ? S.stf[size_t(step) * S.nsrc + s] : 0.f;
#pragma unroll
      for (int c = 0; c < (NC < 2 ? NC : 2); ++c) a[c] += f * S.src_arr[(size_t(s) * 2 + c) * NP + q];
      if (EK == 4) {
        a[2 % NC] += f * S.src_arr2[(size_t(s) * 2) * NP + q];
        a[3 % NC] += f * S.src_arr2[(size_t(s) * 2 + 1) * NP + q];
      }
    }
  }
  if (LOCAL) {
    const int sl = __ldg(A.slot + p);
    if (NC == 4) {
      reinterpret_cast<float4 *>(A.r)[sl] = make_float4(a[0], a[1 % NC], a[2 % NC], a[3 % NC]);
    } else if (NC == 3) {
#pragma unroll
      for (int c = 0; c < NC; ++c) A.r[size_t(sl) * 3 + c] = a[c];
    } else if (NC == 2) reinterpret_cast<float2 *>(A.r)[sl] = make_float2(a[0], a[NC - 1]);
    else A.r[sl] = a[0];
  } else if (NC == 4) {
    reinterpret_cast<float4 *>(A.accum)[g] = make_float4(acc[0] + a[0], acc[1 % NC] + a[1 % NC],
                                                         acc[2 % NC] + a[2 % NC], acc[3 % NC] + a[3 % NC]);
  } else if (NC == 3) {
#pragma unroll
    for (int c = 0; c < NC; ++c) A.accum[size_t(g) * 3 + c] = acc[c] + a[c];
  } else if (NC == 2) {
    reinterpret_cast<float2 *>(A.accum)[g] = make_float2(acc[0] + a[0], acc[NC - 1] + a[NC - 1]);
  } else {
    A.accum[g] = acc[0] + a[0];
  }
}

// Acoustic element block (potential chi; sigma = rho^-1 grad chi).
template <int E, bool LOCAL>
__device__ __forceinline__ void acoustic_block(const StiffArgs &S, const MedArgs &A, int ebase,
                                               unsigned char *smem, float *shp, float *shpw,
                                               float *sw) {
  float *su = reinterpret_cast<float *>(smem);
  float *sF = reinterpret_cast<float *>(smem + sizeof(float) * NP * E * 2);
  const int tid = threadIdx.x;
  const int le = tid / NP, q = tid - le * NP;
  const int e = ebase + le;
  const bool act = e < A.e1;
  const size_t p = size_t(act ? e : A.e0) * NP + q;
  const int g = act ? __ldg(A.ibool + p) : 0;
  const float xix = __ldg(A.xix + p), xiz = __ldg(A.xiz + p), gax = __ldg(A.gax + p),
              gaz = __ldg(A.gaz + p), jac = __ldg(A.jac + p);
  const float rhoinv = __ldg(A.prop0 + p);
  const float chi = act ? A.u[g] : 0.f;
  const float acc = (act && !LOCAL) ? A.accum[g] : 0.f;
  const int bs = act ? __ldg(A.bc_slot + e) : -1;
  const int src = act ? __ldg(A.src_head + e) : -1;
  su[le * NP + q] = chi;
  __syncthreads();
  const int iz = q / NG, ix = q - iz * NG;
  // the two derivative directions paired (FFMA2, rounding as fmaf)
  float2 d = make_float2(0.f, 0.f);
#pragma unroll
  for (int l = 0; l < NG; ++l)
    d = fma2(make_float2(shp[ix * NG + l], shp[iz * NG + l]),
             make_float2(su[le * NP + iz * NG + l], su[le * NP + l * NG + ix]), d);
  const float dxi = d.x, dga = d.y;
  const float s0 = rhoinv * (xix * dxi + gax * dga);
  const float s1 = rhoinv * (xiz * dxi + gaz * dga);
  sF[(le * 2 + 0) * NP + q] = jac * (s0 * xix + s1 * xiz);
  sF[(le * 2 + 1) * NP + q] = jac * (s0 * gax + s1 * gaz);
  __syncthreads();
  if (!act) return;
  float2 t = make_float2(0.f, 0.f);
#pragma unroll
  for (int l = 0; l < NG; ++l)
    t = fma2(make_float2(sF[(le * 2 + 0) * NP + iz * NG + l], sF[(le * 2 + 1) * NP + l * NG + ix]),
             make_float2(shpw[l * NG + ix], shpw[l * NG + iz]), t);
  float a = -(sw[iz] * t.x + sw[ix] * t.y);
  if (bs >= 0) {
    const size_t k = size_t(bs) * NP + q;
    const float wq = A.bc_w[k];
    if (wq != 0.f) a += -1.f * (wq * A.bc_j1[k]) * A.bc_imp0[k] * A.v[g];
    a *= A.bc_keep[k];   // acoustic free surface (Dirichlet) zeroes the element term
  }
  if (src >= 0) {
    const int step = *S.step;
    for (int s = src; s >= 0; s = S.src_next[s]) {
      const float f = step < S.nstep ? S.stf[size_t(step) * S.nsrc + s] : 0.f;
      a += f * S.src_arr[(size_t(s) * 2) * NP + q];
    }
  }
  if (LOCAL) A.r[__ldg(A.slot + p)] = a;
  else A.accum[g] = acc + a;
}

// One launch per colour: blocks [0, el.nblocks) run elastic elements of the
// colour, the following ac.nblocks blocks acoustic ones.
// occupancy held at the warp limit of an SM (64 warps): the kernel is bound
// by memory latency, so registers may not grow past what that allows
template <int E, int EK, bool LOCAL>
__global__ void __launch_bounds__(NP * E, 64 / ((NP * E + 31) / 32)) k_stiffness(StiffArgs S) {
  __shared__ __align__(16) unsigned char smem[sizeof(float) * NP * E * (EK == 4 ? 12 : EK == 3 ? 9 : 6)];
  __shared__ float shp[NP], shpw[NP], sw[NG];
  load_quad(S.quad, shp, shpw, sw, threadIdx.x);
  if (int(blockIdx.x) < S.el.nblocks)
    elastic_block<E, EK, LOCAL>(S, S.el, S.el.e0 + blockIdx.x * E, smem, shp, shpw, sw);
  else
    acoustic_block<E, LOCAL>(S, S.ac, S.ac.e0 + (blockIdx.x - S.el.nblocks) * E, smem, shp, shpw, sw);
}

// ---------------------------------------------------------------------------
// Persistent variant of the element kernel.  A colour launch holds exactly as
// many blocks as fit on the GPU at once; blocks [0, el.nblocks) loop over the
// elastic element chunks of the colour, the others over the acoustic ones
// (chunk = E consecutive elements).  While a chunk is computed, the next
// chunk's index and geometry are already in flight, and its displacement and
// accumulator values are requested once its indices have arrived, so the
// memory latency of one chunk hides behind the arithmetic of the previous.
// Shared memory keeps every field both as rows and as transposed rows
// (padded to 8), so each 5-term contraction reads two vectors; the Lagrange
// coefficients a thread needs stay in registers for the whole loop.
// Elements of one colour share no global point, so the order in which the
// chunks run does not change any sum: results equal the one-pass kernel's.

template <int NC>
struct ChunkRegs {
  int g;
  float xix, xiz, gax, gaz, jac, c0, c1;
  float u[NC], acc[NC];
  int bs, src;
  bool act;
};

template <int NC>
__device__ __forceinline__ void chunk_fetch_static(const MedArgs &A, int e, int q, ChunkRegs<NC> &R) {
  R.act = e < A.e1;
  const size_t p = size_t(R.act ? e : A.e0) * NP + q;
  R.g = R.act ? __ldg(A.ibool + p) : 0;
  R.xix = __ldg(A.xix + p); R.xiz = __ldg(A.xiz + p);
  R.gax = __ldg(A.gax + p); R.gaz = __ldg(A.gaz + p); R.jac = __ldg(A.jac + p);
  R.c0 = __ldg(A.prop0 + p); R.c1 = __ldg(A.prop1 + p);
  R.bs = R.act ? __ldg(A.bc_slot + e) : -1;
  R.src = R.act ? __ldg(A.src_head + e) : -1;
}

template <int NC>
__device__ __forceinline__ void chunk_fetch_fields(const MedArgs &A, ChunkRegs<NC> &R) {
  if (NC == 2) {
    const float2 t = R.act ? reinterpret_cast<const float2 *>(A.u)[R.g] : make_float2(0.f, 0.f);
    const float2 r = R.act ? reinterpret_cast<const float2 *>(A.accum)[R.g] : make_float2(0.f, 0.f);
    R.u[0] = t.x; R.u[NC - 1] = t.y; R.acc[0] = r.x; R.acc[NC - 1] = r.y;
  } else {
    R.u[0] = R.act ? A.u[R.g] : 0.f;
    R.acc[0] = R.act ? A.accum[R.g] : 0.f;
  }
}

__device__ __forceinline__ float dot5(const float *row, const float (&c)[NG]) {
  const float4 a = *reinterpret_cast<const float4 *>(row);
  float s = c[0] * a.x;
  s = fmaf(c[1], a.y, s);
  s = fmaf(c[2], a.z, s);
  s = fmaf(c[3], a.w, s);
  return fmaf(c[4], row[4], s);
}

// KIND 0 acoustic, 1 elastic SH, 2 elastic P-SV.
template <int E, int KIND>
__device__ __forceinline__ void stiffness_loop(const StiffArgs &S, const MedArgs &A, int chunk0,
                                               int stride, float *sm, const float *shp,
                                               const float *shpw, const float *sw) {
  constexpr int NC = KIND == 2 ? 2 : 1;
  constexpr int RS = 8;                     // padded row stride
  constexpr int ARR = NG * RS;              // one 5x5 array, rows padded
  const int nchunks = (A.e1 - A.e0 + E - 1) / E;
  if (chunk0 >= nchunks) return;
  const int tid = threadIdx.x;
  const int le = tid / NP, q = tid - le * NP;
  const int iz = q / NG, ix = q - iz * NG;
  // per element: NC x {U, UT, F0, F1T}
  float *base = sm + le * (NC * 4 * ARR);
  float hx[NG], hz[NG], wx[NG], wz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    hx[l] = shp[ix * NG + l];
    hz[l] = shp[iz * NG + l];
    wx[l] = shpw[l * NG + ix];
    wz[l] = shpw[l * NG + iz];
  }
  const float wiz = sw[iz], wix = sw[ix];
  ChunkRegs<NC> cur, nxt;
  nxt.act = false;
  chunk_fetch_static<NC>(A, A.e0 + chunk0 * E + le, q, cur);
  chunk_fetch_fields<NC>(A, cur);
  for (int chunk = chunk0; chunk < nchunks; chunk += stride) {
    const int e = A.e0 + chunk * E + le;
    const bool more = chunk + stride < nchunks;
    if (more) chunk_fetch_static<NC>(A, A.e0 + (chunk + stride) * E + le, q, nxt);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      base[(c * 4 + 0) * ARR + iz * RS + ix] = cur.u[c];
      base[(c * 4 + 1) * ARR + ix * RS + iz] = cur.u[c];
    }
    __syncthreads();
    float Sx[NC], Sz[NC];
    {
      float dxi[NC], dga[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        dxi[c] = dot5(base + (c * 4 + 0) * ARR + iz * RS, hx);
        dga[c] = dot5(base + (c * 4 + 1) * ARR + ix * RS, hz);
      }
      if (KIND == 2) {
        const float du00 = cur.xix * dxi[0] + cur.gax * dga[0];
        const float du01 = cur.xiz * dxi[0] + cur.gaz * dga[0];
        const float du10 = cur.xix * dxi[NC - 1] + cur.gax * dga[NC - 1];
        const float du11 = cur.xiz * dxi[NC - 1] + cur.gaz * dga[NC - 1];
        const float lam = cur.c0 - 2.f * cur.c1;
        const float sxx = cur.c0 * du00 + lam * du11;
        const float szz = cur.c0 * du11 + lam * du00;
        const float sxz = cur.c1 * (du01 + du10);
        Sx[0] = sxx; Sz[0] = sxz; Sx[NC - 1] = sxz; Sz[NC - 1] = szz;
      } else {
        // acoustic: rho^-1 grad chi (c0 = 1/rho); SH: mu grad u_y (c1 = mu)
        const float k = KIND == 0 ? cur.c0 : cur.c1;
        Sx[0] = k * (cur.xix * dxi[0] + cur.gax * dga[0]);
        Sz[0] = k * (cur.xiz * dxi[0] + cur.gaz * dga[0]);
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      base[(c * 4 + 2) * ARR + iz * RS + ix] = cur.jac * (Sx[c] * cur.xix + Sz[c] * cur.xiz);
      base[(c * 4 + 3) * ARR + ix * RS + iz] = cur.jac * (Sx[c] * cur.gax + Sz[c] * cur.gaz);
    }
    if (more) chunk_fetch_fields<NC>(A, nxt);
    __syncthreads();
    if (cur.act) {
      float a[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float t1 = dot5(base + (c * 4 + 2) * ARR + iz * RS, wx);
        const float t2 = dot5(base + (c * 4 + 3) * ARR + ix * RS, wz);
        a[c] = -(wiz * t1 + wix * t2);
      }
      if (cur.bs >= 0) {
        const size_t k = size_t(cur.bs) * NP + q;
        const float wq = A.bc_w[k];
        if (KIND == 2) {
          if (wq != 0.f) {
            const float nx = A.bc_nx[k], nz = A.bc_nz[k], j1 = A.bc_j1[k];
            const float2 vv = reinterpret_cast<const float2 *>(A.v)[cur.g];
            const float rvp = A.bc_imp0[k], rvs = A.bc_imp1[k];
            const float vn = vv.x * nx + vv.y * nz;
            const float fx = ((vn * nx / (j1 * j1)) * (rvp - rvs)) + vv.x * rvs;
            const float fz = ((vn * nz / (j1 * j1)) * (rvp - rvs)) + vv.y * rvs;
            a[0] += -1.f * fx * j1 * wq;
            a[NC - 1] += -1.f * fz * j1 * wq;
          }
        } else {
          if (wq != 0.f) {
            const float imp = KIND == 0 ? A.bc_imp0[k] : A.bc_imp1[k];
            a[0] += -1.f * (wq * A.bc_j1[k]) * imp * A.v[cur.g];
          }
          if (KIND == 0) a[0] *= A.bc_keep[k];
        }
      }
      if (cur.src >= 0) {
        const int step = *S.step;
        for (int s = cur.src; s >= 0; s = S.src_next[s]) {
          const float f = step < S.nstep ? S.stf[size_t(step) * S.nsrc + s] : 0.f;
#pragma unroll
          for (int c = 0; c < NC; ++c) a[c] += f * S.src_arr[(size_t(s) * 2 + c) * NP + q];
        }
      }
      if (NC == 2) {
        reinterpret_cast<float2 *>(A.accum)[cur.g] =
            make_float2(cur.acc[0] + a[0], cur.acc[NC - 1] + a[NC - 1]);
      } else {
        A.accum[cur.g] = cur.acc[0] + a[0];
      }
    }
    (void)e;
    cur = nxt;
  }
}

template <int E, int EK>
__global__ void __launch_bounds__(NP * E) k_stiffness_persistent(StiffArgs S) {
  // largest need: P-SV, 2 components x 4 padded arrays of 40 floats per element
  __shared__ __align__(16) float sm[E * 2 * 4 * NG * 8];
  __shared__ float shp[NP], shpw[NP], sw[NG];
  load_quad(S.quad, shp, shpw, sw, threadIdx.x);
  __syncthreads();
  if (int(blockIdx.x) < S.el.nblocks) {
    if (EK == 0) stiffness_loop<E, 2>(S, S.el, blockIdx.x, S.el.nblocks, sm, shp, shpw, sw);
    else stiffness_loop<E, 1>(S, S.el, blockIdx.x, S.el.nblocks, sm, shp, shpw, sw);
  } else {
    stiffness_loop<E, 0>(S, S.ac, blockIdx.x - S.el.nblocks, S.ac.nblocks, sm, shp, shpw, sw);
  }
}

// Recording of a recomputed forward segment (adjoint runs): the update of
// step k writes the step's displacement u~ and new acceleration a' to slot
// k - k0 of the segment buffers.
struct SegRecord {
  float *u, *a;
  size_t stride;  // floats per slot (a multiple of 4)
  int k0;
  // predicted velocity v~ of the step at the nst Stacey points st_pt
  float *vst;
  size_t vstride;
  const int *st_pt;
  int nst;
  int i;          // next step of the segment (k0 + i)
};

struct UpdateArgs {
  float *__restrict__ u, *__restrict__ v, *__restrict__ accum;
  const float *__restrict__ minv;
  float *__restrict__ a_store;   // copy of the new acceleration (optional when predicting)
  int n;                         // nglob * ncomp
  int ncomp;
  // coupling: the first niface points take cp_n . other[cp_other] (acoustic
  // self: other = elastic displacement, float2) or cp_n * other (elastic self:
  // other = acoustic chi_dd); with nonconforming interfaces a sum of such
  // terms over the entries cp_start[pt] .. cp_start[pt + 1] (cp_start null:
  // entry pt alone)
  int niface;
  const float *__restrict__ cp_nx, *__restrict__ cp_nz;
  const int *__restrict__ cp_other;
  const int *__restrict__ cp_start;
  const float *__restrict__ other;
  // owner-computes assembly: accum of point g = sum of r[inv_start[g] .. inv_start[g+1])
  const int *__restrict__ inv_start;
  const float *__restrict__ r;
  float dt, dt2, dtsq2;
  int predict;                   // fuse the next step's predictor
  int *flag;                     // set to 1 on a non-finite displacement
  int *step;
  int advance;                   // increment the step counter (last update of a step)
  const SegRecord *rec;          // optional segment recording (then advance = 0)
};

__device__ __forceinline__ float coupling_entry(const UpdateArgs &A, int k, int comp) {
  const int o = A.cp_other[k];
  if (A.ncomp == 1) {  // acoustic self: n . u_elastic
    const float2 ue = reinterpret_cast<const float2 *>(A.other)[o];
    return A.cp_nx[k] * ue.x + A.cp_nz[k] * ue.y;
  }
  const float chi_dd = A.other[o];  // elastic self: n * chi_dd
  return (comp == 0 ? A.cp_nx[k] : A.cp_nz[k]) * chi_dd;
}

__device__ __forceinline__ float coupling_term(const UpdateArgs &A, int pt, int comp) {
  if (!A.cp_start) return coupling_entry(A, pt, comp);
  const int k1 = A.cp_start[pt + 1];
  float t = 0.f;
  for (int k = A.cp_start[pt]; k < k1; ++k) t += coupling_entry(A, k, comp);
  return t;
}

// Newmark predictor u += dt v + dt^2/2 a; v += dt/2 a (newmark.tpp:64-128),
// with every product and sum rounded separately (no contraction into FMA), so
// the fused update and k_predict give equal bits, as does a CPU build with
// contraction off.
__device__ __forceinline__ void newmark_predict(float &u, float &v, float a, float dt, float dt2,
                                                float dtsq2) {
  u = __fadd_rn(u, __fadd_rn(__fmul_rn(dt, v), __fmul_rn(dtsq2, a)));
  v = __fadd_rn(v, __fmul_rn(dt2, a));
}

// Newmark corrector v += dt/2 a (newmark.tpp:10-62).
__device__ __forceinline__ float newmark_correct(float v, float a, float dt2) {
  return __fadd_rn(v, __fmul_rn(dt2, a));
}

// a = (accum [+ coupling]) * M^-1; v += dt/2 a (corrector); optionally the
// predictor of the next step; accum = 0.
__global__ void __launch_bounds__(256) k_update(UpdateArgs A) {
  const int n4 = A.n >> 2;
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  const int nc_iface = A.niface * A.ncomp;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    float4 ac = reinterpret_cast<float4 *>(A.accum)[i];
    const float4 mi = reinterpret_cast<const float4 *>(A.minv)[i];
    float4 uu = reinterpret_cast<float4 *>(A.u)[i];
    float4 vv = reinterpret_cast<float4 *>(A.v)[i];
    float *pa = &ac.x, *pu = &uu.x, *pv = &vv.x;
    const float *pm = &mi.x;
    if (4 * i < nc_iface) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int k = 4 * i + c;
        if (k < nc_iface) pa[c] += coupling_term(A, k / A.ncomp, k % A.ncomp);
      }
    }
    float a[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) a[c] = __fmul_rn(pa[c], pm[c]);
    if (A.rec) {
      const size_t off = size_t(*A.step - A.rec->k0) * A.rec->stride;
      reinterpret_cast<float4 *>(A.rec->u + off)[i] = uu;
      reinterpret_cast<float4 *>(A.rec->a + off)[i] = make_float4(a[0], a[1], a[2], a[3]);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      pv[c] = newmark_correct(pv[c], a[c], A.dt2);
      if (A.predict) newmark_predict(pu[c], pv[c], a[c], A.dt, A.dt2, A.dtsq2);
      bad |= !isfinite(pu[c]);
    }
    if (A.predict) reinterpret_cast<float4 *>(A.u)[i] = uu;
    reinterpret_cast<float4 *>(A.v)[i] = vv;
    reinterpret_cast<float4 *>(A.accum)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (A.a_store) reinterpret_cast<float4 *>(A.a_store)[i] = make_float4(a[0], a[1], a[2], a[3]);
  }
  for (int i = (n4 << 2) + blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += stride) {
    float acc = A.accum[i];
    if (i < nc_iface) acc += coupling_term(A, i / A.ncomp, i % A.ncomp);
    const float a = __fmul_rn(acc, A.minv[i]);
    float vv = newmark_correct(A.v[i], a, A.dt2);
    float uu = A.u[i];
    if (A.rec) {
      const size_t off = size_t(*A.step - A.rec->k0) * A.rec->stride;
      A.rec->u[off + i] = uu;
      A.rec->a[off + i] = a;
    }
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

// Owner-computes form of k_update: one thread per point gathers the
// element-local contributions in increasing compute order (colour order), so
// the sum is the colour passes' sum bit for bit; then coupling, M^-1,
// corrector and optional predictor as k_update.  No accumulator to clear.
template <int NC>
__device__ __forceinline__ bool update_gather_point(const UpdateArgs &A, int g) {
  float acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.f;
  const int k1 = A.inv_start[g + 1];
  for (int k = A.inv_start[g]; k < k1; ++k) {
    if (NC == 2) {
      const float2 t = reinterpret_cast<const float2 *>(A.r)[k];
      acc[0] = acc[0] + t.x;
      acc[NC - 1] = acc[NC - 1] + t.y;
    } else {
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[c] = acc[c] + A.r[size_t(k) * NC + c];
    }
  }
  if (g < A.niface) {
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] += coupling_term(A, g, c);
  }
  float uu[NC], vv[NC], mi[NC];
  if (NC == 2) {
    const float2 u2 = reinterpret_cast<const float2 *>(A.u)[g];
    const float2 v2 = reinterpret_cast<const float2 *>(A.v)[g];
    const float2 m2 = reinterpret_cast<const float2 *>(A.minv)[g];
    uu[0] = u2.x; uu[NC - 1] = u2.y; vv[0] = v2.x; vv[NC - 1] = v2.y; mi[0] = m2.x; mi[NC - 1] = m2.y;
  } else {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const size_t i = size_t(g) * NC + c;
      uu[c] = A.u[i]; vv[c] = A.v[i]; mi[c] = A.minv[i];
    }
  }
  float a[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) a[c] = __fmul_rn(acc[c], mi[c]);
  if (A.rec) {
    const size_t off = size_t(*A.step - A.rec->k0) * A.rec->stride;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      A.rec->u[off + size_t(g) * NC + c] = uu[c];
      A.rec->a[off + size_t(g) * NC + c] = a[c];
    }
  }
  bool bad = false;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    vv[c] = newmark_correct(vv[c], a[c], A.dt2);
    if (A.predict) newmark_predict(uu[c], vv[c], a[c], A.dt, A.dt2, A.dtsq2);
    bad |= !isfinite(uu[c]);
  }
  if (NC == 2) {
    if (A.predict) reinterpret_cast<float2 *>(A.u)[g] = make_float2(uu[0], uu[NC - 1]);
    reinterpret_cast<float2 *>(A.v)[g] = make_float2(vv[0], vv[NC - 1]);
    if (A.a_store) reinterpret_cast<float2 *>(A.a_store)[g] = make_float2(a[0], a[NC - 1]);
  } else {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const size_t i = size_t(g) * NC + c;
      if (A.predict) A.u[i] = uu[c];
      A.v[i] = vv[c];
      if (A.a_store) A.a_store[i] = a[c];
    }
  }
  return bad;
}

template <int NC>
__global__ void __launch_bounds__(256) k_update_gather(UpdateArgs A) {
  const int npts = A.n / NC;
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < npts; g += stride)
    bad |= update_gather_point<NC>(A, g);
  if (bad) *A.flag = 1;
  if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) *A.step += 1;
}

// Both media's owner-computes point updates in one launch (coupled P-SV
// model, one shot).  Threads [0, n_el) take the elastic points, the others
// the acoustic points past the interface.  The acoustic update of an
// interface point reads the elastic predicted displacement there, and the
// elastic update reads the acoustic chi_dd: the interface points pair one to
// one (elastic i <-> acoustic El.cp_other[i]), so the thread of elastic
// interface point i first updates its acoustic partner (as the acoustic
// launch would, before this thread overwrites the displacement) and then
// itself (reading the chi_dd it has just stored).  Same arithmetic as the two
// launches: equal bits.
__global__ void __launch_bounds__(256) k_update_coupled(UpdateArgs El, UpdateArgs Ac) {
  const int nel = El.n / 2, nac = Ac.n;
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nel + nac - Ac.niface; t += stride) {
    if (t < nel) {
      if (t < El.niface) bad |= update_gather_point<1>(Ac, El.cp_other[t]);
      bad |= update_gather_point<2>(El, t);
    } else {
      bad |= update_gather_point<1>(Ac, Ac.niface + (t - nel));
    }
  }
  if (bad) *El.flag = 1;
  if (El.advance && blockIdx.x == 0 && threadIdx.x == 0) *El.step += 1;
}

// Step-wise interface (the reference's update_wavefields / corrector phases):
// a = (sum of the element contributions in colour order + coupling) * M^-1,
// stored; divide_mass_matrix.tpp:10-65 after compute_coupling.
template <int NC>
__global__ void __launch_bounds__(256) k_accel_gather(UpdateArgs A) {
  const int npts = A.n / NC;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < npts; g += gridDim.x * blockDim.x) {
    float acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = 0.f;
    const int k1 = A.inv_start[g + 1];
    for (int k = A.inv_start[g]; k < k1; ++k)
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[c] = acc[c] + A.r[size_t(k) * NC + c];
    if (g < A.niface) {
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[c] += coupling_term(A, g, c);
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const size_t i = size_t(g) * NC + c;
      A.a_store[i] = __fmul_rn(acc[c], A.minv[i]);
    }
  }
}

// Newmark corrector phase v += dt/2 a (newmark.tpp:10-62).
__global__ void __launch_bounds__(256) k_correct(float *__restrict__ v, const float *__restrict__ a, int n, float dt2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i] = newmark_correct(v[i], a[i], dt2);
}

// Pending predictor of a run that ended on a corrector-only update.
__global__ void __launch_bounds__(256) k_predict(float *__restrict__ u, float *__restrict__ v,
                                                 const float *__restrict__ a, int n, float dt,
                                                 float dt2, float dtsq2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float uu = u[i], vv = v[i];
    newmark_predict(uu, vv, a[i], dt, dt2, dtsq2);
    u[i] = uu;
    v[i] = vv;
  }
}

struct RecArgs {
  int nrec;
  const int *__restrict__ rec_list;    // receivers of this medium
  const int *__restrict__ rec_elem;    // compute element in the medium
  const float *__restrict__ rec_h;     // [nrec][25]
  const int *__restrict__ ibool;
  const float *__restrict__ xix, *__restrict__ xiz, *__restrict__ gax, *__restrict__ gaz,
      *__restrict__ prop0, *__restrict__ prop1;
  const float *__restrict__ prop2, *__restrict__ prop3;   // poroelastic C_Biot, M_Biot
  const float *__restrict__ u, *__restrict__ v, *__restrict__ accum, *__restrict__ minv;
  UpdateArgs cpl;                      // coupling data of the medium (niface, cp_*, other)
  int ncomp, acoustic;
  int ntypes;
  int types[8];
  int nsb, nsig, nrec_total;
  float dt2;
  const int *__restrict__ step;
  float *__restrict__ seis;            // [nsig][ntypes][nrec_total][2]
  Quad quad;
  // the end-of-step fields are final (corrected v, stored a: the step-wise
  // interface): read them instead of reconstructing from the accumulator
  const float *__restrict__ a;
  int final_fields;
  int isig_fixed;                      // sample index given by the caller (-1: from the step counter)
};

__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__device__ __forceinline__ float rec_accel(const RecArgs &A, int g, int c) {
  const size_t k = size_t(g) * A.ncomp + c;
  float acc;
  if (A.cpl.inv_start) {   // owner-computes: gather in colour order
    acc = 0.f;
    for (int j = A.cpl.inv_start[g]; j < A.cpl.inv_start[g + 1]; ++j)
      acc = acc + A.cpl.r[size_t(j) * A.ncomp + c];
  } else {
    acc = A.accum[k];
  }
  if (g < A.cpl.niface) acc += coupling_term(A.cpl, g, c);
  return __fmul_rn(acc, A.minv[k]);
}

// One warp per receiver of one medium; runs before that medium's update, so
// it reconstructs the corrected velocity and the new acceleration from the
// accumulator (plus the coupling term on interface points).
__global__ void __launch_bounds__(32) k_receivers(RecArgs A) {
  __shared__ float sf[3][NP];
  int isig = A.isig_fixed;
  if (isig < 0) {
    const int step = *A.step;
    if (step % A.nsb != 0) return;
    isig = step / A.nsb;
  }
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
    const int nc = A.ncomp;
    for (int t = 0; t < A.ntypes; ++t) {
      float o[2] = {0.f, 0.f};
      const int ty = A.types[t];
      if (ty == 3 || ty == 5 || ty == 6) {
        // from the displacement gradient at the element point: pressure
        // -(lambda + 2/3 mu) div u (include/medium/dim2/elastic/isotropic/
        // wavefield.hpp:57-89; Cosserat: prop0 = lambda); Cosserat curl
        // du_x/dz - du_z/dx and intrinsic rotation phi - curl / 2
        // (isotropic_cosserat/wavefield.hpp)
        float pr = 0.f;
        if (nc >= 2) {
          const int iz = q / NG, ix = q - iz * NG;
          float dxi0 = 0.f, dxi1 = 0.f, dga0 = 0.f, dga1 = 0.f;
          for (int l = 0; l < NG; ++l) {
            const int gr = A.ibool[size_t(ce) * NP + iz * NG + l];
            const int gc = A.ibool[size_t(ce) * NP + l * NG + ix];
            const float hx = A.quad.hp[ix * NG + l], hz = A.quad.hp[iz * NG + l];
            dxi0 += hx * A.u[size_t(gr) * nc];
            dxi1 += hx * A.u[size_t(gr) * nc + 1];
            dga0 += hz * A.u[size_t(gc) * nc];
            dga1 += hz * A.u[size_t(gc) * nc + 1];
          }
          if (on && ty == 3 && nc == 4) {
            // pore pressure -(C div u_s + M div w) (poroelastic/isotropic/wavefield.hpp)
            float dxi2 = 0.f, dxi3 = 0.f, dga2 = 0.f, dga3 = 0.f;
            for (int l = 0; l < NG; ++l) {
              const int gr = A.ibool[size_t(ce) * NP + iz * NG + l];
              const int gc = A.ibool[size_t(ce) * NP + l * NG + ix];
              const float hx = A.quad.hp[ix * NG + l], hz = A.quad.hp[iz * NG + l];
              dxi2 += hx * A.u[size_t(gr) * 4 + 2];
              dxi3 += hx * A.u[size_t(gr) * 4 + 3];
              dga2 += hz * A.u[size_t(gc) * 4 + 2];
              dga3 += hz * A.u[size_t(gc) * 4 + 3];
            }
            const float dux = A.xix[p] * dxi0 + A.gax[p] * dga0;
            const float duz = A.xiz[p] * dxi1 + A.gaz[p] * dga1;
            const float dwx = A.xix[p] * dxi2 + A.gax[p] * dga2;
            const float dwz = A.xiz[p] * dxi3 + A.gaz[p] * dga3;
            pr = -1.f * (A.prop2[p] * (dux + duz) + A.prop3[p] * (dwx + dwz));
          } else if (on && ty == 3) {
            const float dux = A.xix[p] * dxi0 + A.gax[p] * dga0;
            const float duz = A.xiz[p] * dxi1 + A.gaz[p] * dga1;
            const float l2m = A.prop0[p], mu = A.prop1[p];
            pr = nc == 3 ? -1.f * ((l2m + (2.f / 3.f) * mu) * (dux + duz))
                         : -1.f * ((l2m - 2.f * mu + (2.f / 3.f) * mu) * (dux + duz));
          } else if (on && nc == 3) {
            const float duxz = A.xiz[p] * dxi0 + A.gaz[p] * dga0;
            const float duzx = A.xix[p] * dxi1 + A.gax[p] * dga1;
            const float curl = duxz - duzx;
            pr = ty == 6 ? curl : A.u[size_t(g) * 3 + 2] - 0.5f * curl;
          }
        }
        o[0] = warp_sum(h * pr);
      } else if (ty == 4) {                    // Cosserat rotation
        o[0] = warp_sum(nc == 3 ? h * A.u[size_t(g) * 3 + 2] : 0.f);
      } else {
        for (int c = 0; c < (nc < 2 ? nc : 2); ++c) {
          const size_t k = size_t(g) * A.ncomp + c;
          float val = 0.f;
          switch (A.types[t]) {
            case 0: val = A.u[k]; break;
            case 1: val = A.final_fields ? A.v[k] : newmark_correct(A.v[k], rec_accel(A, g, c), A.dt2); break;
            default: val = A.final_fields ? A.a[k] : rec_accel(A, g, c); break;
          }
          o[c] = warp_sum(h * val);
        }
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
  const float a = A.final_fields ? A.a[g] : rec_accel(A, g, 0);
  if (on) {
    sf[0][q] = A.u[g];
    sf[1][q] = A.final_fields ? A.v[g] : newmark_correct(A.v[g], a, A.dt2);
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
