// Element kernel with bulk-copy (TMA engine) staging of the element arrays.
//
// A persistent block walks the tiles b, b + G, b + 2G, ... (G = grid size;
// a tile is E consecutive elements of one medium).  The eight element arrays
// of a tile (global index, xi_x, xi_z, gamma_x, gamma_z, |J| and the two
// material words), E*25 words each, stream from HBM into a ring of S
// shared-memory stages with cp.async.bulk, completing on one mbarrier per
// stage; the copy of tile j+S is issued as soon as every thread has read
// tile j's stage, so S-1 tiles of element data are always in flight while a
// tile is computed.  Per tile: gather of the field at the 25 global points,
// the 5-term Lagrange-derivative contractions on rows padded to 8 words
// (float4 reads; each field is held as rows and as transposed rows), the
// stress, the integrand F, the divergence, then the Stacey / free-surface /
// source epilogue and the element-local store (owner-computes assembly, the
// point update sums each point's element contributions in a fixed order).
// The arithmetic, operand order included, is that of k_stiffness<..., true>,
// so the results are bit-identical to it.
//
// Every wait on an mbarrier has an iteration limit; a wait that gives up sets
// *err (the host reports it) and the block drains the copies it issued
// before returning.
#pragma once

#include "kernels2d.cuh"

namespace sfg {
namespace dev {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false after about 2^22 polls (each poll may suspend briefly).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (int i = 0; i < (1 << 22); ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// One bulk copy global -> shared (16-byte aligned addresses, size a multiple
// of 16), completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

constexpr int TMA_ARRAYS = 8;  // ibool, xix, xiz, gax, gaz, jac, c0, c1
// Shared words per element: NC x {U, UT, F0, F1T} as 5 rows of 8, plus 4 so
// that consecutive elements start 4 banks apart (fewer bank conflicts).
constexpr int ELEM_WORK = 2 * 4 * NG * 8 + 4;

template <int E>
struct TmaLayout {
  static constexpr int TW = E * NP;                                   // words per array per tile
  static constexpr int STAGE_BYTES = TMA_ARRAYS * TW * 4;
  static constexpr int WORK_FLOATS = E * ELEM_WORK;
  static constexpr int bytes(int S) { return 64 + S * STAGE_BYTES + WORK_FLOATS * 4; }
};

template <int E, int S>
__device__ __forceinline__ void tma_issue(const StiffArgs &A, int nt_el, int tile, unsigned char *stage,
                                          uint64_t *bar) {
  constexpr int TW = TmaLayout<E>::TW;
  const MedArgs &M = tile < nt_el ? A.el : A.ac;
  const size_t off = size_t(tile < nt_el ? tile : tile - nt_el) * TW;
  const void *src[TMA_ARRAYS] = {M.ibool + off, M.xix + off, M.xiz + off, M.gax + off,
                                 M.gaz + off,   M.jac + off, M.prop0 + off, M.prop1 + off};
  mbar_expect_tx(bar, TmaLayout<E>::STAGE_BYTES);
#pragma unroll
  for (int k = 0; k < TMA_ARRAYS; ++k) bulk_g2s(stage + k * TW * 4, src[k], TW * 4, bar);
}

// Per-element-point geometry and material words.
struct PointGeom {
  int g;
  float xix, xiz, gax, gaz, jac, c0, c1;
};

// One tile of one medium (KIND 0 acoustic, 1 elastic SH, 2 elastic P-SV),
// given this thread's point geometry and field value.  Returns after the
// tile's second barrier; `refill` runs right after it.
template <int E, int KIND, typename Refill>
__device__ __forceinline__ void tile_compute(const StiffArgs &S, const MedArgs &A, int e, int q, int iz, int ix,
                                             const PointGeom &P, float *base, const float (&hx)[NG],
                                             const float (&hz)[NG], const float (&wx)[NG], const float (&wz)[NG],
                                             float wix, float wiz, float2 u_in, Refill refill) {
  constexpr int NC = KIND == 2 ? 2 : 1;
  constexpr int RS = 8;
  constexpr int ARR = NG * RS;
  const bool act = e < A.e1;
  const int g = P.g;
  const float xix = P.xix, xiz = P.xiz, gax = P.gax, gaz = P.gaz, jac = P.jac, c0 = P.c0, c1 = P.c1;
  const int bs = act ? __ldg(A.bc_slot + e) : -1;
  const int src = act ? __ldg(A.src_head + e) : -1;
  float uu[NC];
  uu[0] = u_in.x;
  if (NC == 2) uu[NC - 1] = u_in.y;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    base[(c * 4 + 0) * ARR + iz * RS + ix] = uu[c];
    base[(c * 4 + 1) * ARR + ix * RS + iz] = uu[c];
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
      const float du00 = xix * dxi[0] + gax * dga[0], du01 = xiz * dxi[0] + gaz * dga[0];
      const float du10 = xix * dxi[NC - 1] + gax * dga[NC - 1];
      const float du11 = xiz * dxi[NC - 1] + gaz * dga[NC - 1];
      const float lam = c0 - 2.f * c1;
      const float sxx = c0 * du00 + lam * du11;
      const float szz = c0 * du11 + lam * du00;
      const float sxz = c1 * (du01 + du10);
      Sx[0] = sxx; Sz[0] = sxz; Sx[NC - 1] = sxz; Sz[NC - 1] = szz;
    } else {
      // acoustic: rho^-1 grad chi (c0 = 1/rho); SH: mu grad u_y (c1 = mu)
      const float k = KIND == 0 ? c0 : c1;
      Sx[0] = k * (xix * dxi[0] + gax * dga[0]);
      Sz[0] = k * (xiz * dxi[0] + gaz * dga[0]);
    }
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    base[(c * 4 + 2) * ARR + iz * RS + ix] = jac * (Sx[c] * xix + Sz[c] * xiz);
    base[(c * 4 + 3) * ARR + ix * RS + iz] = jac * (Sx[c] * gax + Sz[c] * gaz);
  }
  __syncthreads();
  refill();
  if (!act) return;
  float a[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const float t1 = dot5(base + (c * 4 + 2) * ARR + iz * RS, wx);
    const float t2 = dot5(base + (c * 4 + 3) * ARR + ix * RS, wz);
    a[c] = -(wiz * t1 + wix * t2);
  }
  const size_t p = size_t(e) * NP + q;
  if (bs >= 0) {
    const size_t k = size_t(bs) * NP + q;
    const float wq = A.bc_w[k];
    if (KIND == 2) {
      if (wq != 0.f) {
        const float nx = A.bc_nx[k], nz = A.bc_nz[k], j1 = A.bc_j1[k];
        const float2 vv = reinterpret_cast<const float2 *>(A.v)[g];
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
        a[0] += -1.f * (wq * A.bc_j1[k]) * imp * A.v[g];
      }
      if (KIND == 0) a[0] *= A.bc_keep[k];
    }
  }
  if (src >= 0) {
    const int step = *S.step;
    for (int s = src; s >= 0; s = S.src_next[s]) {
      const float f = step < S.nstep ? S.stf[size_t(step) * S.nsrc + s] : 0.f;
#pragma unroll
      for (int c = 0; c < NC; ++c) a[c] += f * S.src_arr[(size_t(s) * 2 + c) * NP + q];
    }
  }
  const int sl = __ldg(A.slot + p);
  if (NC == 2) reinterpret_cast<float2 *>(A.r)[sl] = make_float2(a[0], a[NC - 1]);
  else A.r[sl] = a[0];
}

template <int E, int KIND, typename Refill>
__device__ __forceinline__ void tma_tile(const StiffArgs &S, const MedArgs &A, int e, int le, int q, int iz,
                                         int ix, const unsigned char *stage, float *base, const float (&hx)[NG],
                                         const float (&hz)[NG], const float (&wx)[NG], const float (&wz)[NG],
                                         float wix, float wiz, float2 u_in, Refill refill) {
  constexpr int TW = TmaLayout<E>::TW;
  const int t = le * NP + q;
  const float *sg = reinterpret_cast<const float *>(stage);
  PointGeom P;
  P.g = e < A.e1 ? reinterpret_cast<const int *>(stage)[t] : 0;
  P.xix = sg[1 * TW + t]; P.xiz = sg[2 * TW + t]; P.gax = sg[3 * TW + t]; P.gaz = sg[4 * TW + t];
  P.jac = sg[5 * TW + t]; P.c0 = sg[6 * TW + t]; P.c1 = sg[7 * TW + t];
  tile_compute<E, KIND>(S, A, e, q, iz, ix, P, base, hx, hz, wx, wz, wix, wiz, u_in, refill);
}

// The field at this thread's point of a tile (read from the tile's staged
// global indices): issued one tile ahead, so its latency hides behind the
// arithmetic of the current tile.
template <int E, int EK>
__device__ __forceinline__ float2 tma_gather(const StiffArgs &A, int nt_el, int tile, const unsigned char *stage,
                                             int le, int q) {
  const bool el = tile < nt_el;
  const MedArgs &M = el ? A.el : A.ac;
  const int e = (el ? tile : tile - nt_el) * E + le;
  if (e >= M.e1) return make_float2(0.f, 0.f);
  const int g = reinterpret_cast<const int *>(stage)[le * NP + q];
  if (el && EK == 0) return reinterpret_cast<const float2 *>(M.u)[g];
  return make_float2(M.u[g], 0.f);
}

// Persistent element kernel over nt_el elastic tiles then nt_ac acoustic
// tiles.  The element arrays must hold whole tiles (padded to a multiple of E
// elements); dynamic shared memory TmaLayout<E>::bytes(S).
template <int E, int EK, int S>
__global__ void __launch_bounds__(NP * E) k_stiffness_tma(StiffArgs A, int nt_el, int nt_ac, int *err) {
  extern __shared__ __align__(128) unsigned char dyn[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(dyn);
  unsigned char *stages = dyn + 64;
  float *work = reinterpret_cast<float *>(stages + S * TmaLayout<E>::STAGE_BYTES);
  __shared__ float shp[NP], shpw[NP], sw[NG];
  const int tid = threadIdx.x;
  const int G = gridDim.x, b = blockIdx.x;
  const int ntiles = nt_el + nt_ac;
  const int nmine = b < ntiles ? (ntiles - 1 - b) / G + 1 : 0;
  load_quad(A.quad, shp, shpw, sw, tid);
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) mbar_init(bar + s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    for (int j = 0; j < S && j < nmine; ++j)
      tma_issue<E, S>(A, nt_el, b + j * G, stages + j * TmaLayout<E>::STAGE_BYTES, bar + j);
  }
  const int le = tid / NP, q = tid - le * NP;
  const int iz = q / NG, ix = q - iz * NG;
  float hx[NG], hz[NG], wx[NG], wz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    hx[l] = shp[ix * NG + l];
    hz[l] = shp[iz * NG + l];
    wx[l] = shpw[l * NG + ix];
    wz[l] = shpw[l * NG + iz];
  }
  const float wiz = sw[iz], wix = sw[ix];
  float *base = work + le * ELEM_WORK;
  int j = 0;
  float2 u_cur = make_float2(0.f, 0.f);
  if (nmine > 0) {
    const bool ok = mbar_wait(bar, 0u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicExch(err, 2);
      for (int k = 0; tid == 0 && k < nmine && k < S; ++k) mbar_wait(bar + k, 0u);
      return;
    }
    u_cur = tma_gather<E, EK>(A, nt_el, b, stages, le, q);
  }
  for (; j < nmine; ++j) {
    const int st = j % S;
    const unsigned char *stage = stages + st * TmaLayout<E>::STAGE_BYTES;
    // stage j landed (waited one iteration earlier); wait for stage j+1 and
    // request the next tile's field values
    float2 u_next = make_float2(0.f, 0.f);
    if (j + 1 < nmine) {
      const int sn = (j + 1) % S;
      const bool ok = mbar_wait(bar + sn, uint32_t(((j + 1) / S) & 1));
      if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicExch(err, 2);
        break;
      }
      u_next = tma_gather<E, EK>(A, nt_el, b + (j + 1) * G, stages + sn * TmaLayout<E>::STAGE_BYTES, le, q);
    }
    const int tile = b + j * G;
    auto refill = [&]() {
      if (tid == 0 && j + S < nmine) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tma_issue<E, S>(A, nt_el, b + (j + S) * G, stages + st * TmaLayout<E>::STAGE_BYTES, bar + st);
      }
    };
    if (tile < nt_el) {
      const int e = tile * E + le;
      if (EK == 0)
        tma_tile<E, 2>(A, A.el, e, le, q, iz, ix, stage, base, hx, hz, wx, wz, wix, wiz, u_cur, refill);
      else
        tma_tile<E, 1>(A, A.el, e, le, q, iz, ix, stage, base, hx, hz, wx, wz, wix, wiz, u_cur, refill);
    } else {
      const int e = (tile - nt_el) * E + le;
      tma_tile<E, 0>(A, A.ac, e, le, q, iz, ix, stage, base, hx, hz, wx, wz, wix, wiz, u_cur, refill);
    }
    u_cur = u_next;
  }
  if (j < nmine && tid == 0) {
    // gave up waiting: let the copies already issued land before leaving
    for (int k = j + 1; k < nmine && k < j + S; ++k) mbar_wait(bar + (k % S), uint32_t((k / S) & 1));
  }
}

}  // namespace dev
}  // namespace sfg
