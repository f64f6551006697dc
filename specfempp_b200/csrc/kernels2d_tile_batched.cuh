// Fused tile kernel of the batched 2D time step: S shots on one mesh (S a
// multiple of 4; one isotropic elastic medium, P-SV or SH), fields
// [point][component][shot].
//
// The tiles, the point numbering (each tile's interior points contiguous) and
// the tile records are those of the single-shot tile kernel.  A work item is
// one tile and one quad of shots (4 consecutive shots); every thread is one
// element GLL point of the tile and carries its four shots as a float4.  Per
// item a 3-stage ring of shared-memory buffers receives the tile record and
// its shared-point ids by cp.async.bulk (one mbarrier per stage, bounded
// waits); the displacement quads are loaded one item ahead into registers.
// The element arithmetic is k_stiffness_batched4's, operation for operation
// (the 5-term contractions as explicit FMAs, two shots per FFMA2; FFMA2 rounds
// each lane as fmaf), so every shot gives the bits of a single-shot run.
// Assembly as in k_tile: contributions at tile-interior points go to one
// shared-memory slot per colour, summed per point in increasing colour order
// (the order of the colour passes and of owner-computes), followed in the
// same kernel by M^-1, the corrector and the next predictor; contributions at
// boundary points go to per-colour slots in HBM that k_tile_boundary_b sums
// in the same order.  The interior points never make the round trip through
// an assembly buffer in HBM.
// Reference: include/kokkos_kernels/impl/compute_stiffness_interaction.tpp:140-247,
// include/algorithms/gradient.hpp:40-82, divergence.hpp:41-74,
// include/boundary_conditions/stacey/stacey.tpp:50-80,
// include/kokkos_kernels/impl/compute_source_interaction.tpp:17-104,
// core/specfem/timescheme/newmark.tpp:10-128,
// include/kokkos_kernels/impl/compute_seismogram.tpp:19-171.
#pragma once

#include "kernels2d_tile.cuh"

namespace sfg {
namespace dev {

constexpr int TILEB_STAGES = 3;
constexpr int SIDEB_W = 6;   // side words per point and shot: u(2) v(2) a(2)

struct TileBArgs {
  TileMed el;                  // u, v, a, r: [..][NC][S]; minv: [point][NC]
  MedArgs bel;                 // Stacey arrays
  const int *src_next, *src_shot;
  const float *src_arr;        // [nsrc][2][25]
  const float *stf;            // [nstep][nsrc]
  int nsrc, nstep;
  const int *step;
  float dt, dt2, dtsq2;
  int predict;
  int *flag;
  float *side;                 // [slot][6][S]
  int S;
  // dynamic shared memory (bytes): 64 bytes of barriers, the stages (record,
  // shared-point ids), the element work arrays, the accumulators
  int stage_bytes, off_sh, work_off, acc_off, kcap;
  Quad quad;
};

__device__ __forceinline__ void tileb_issue(const TileMed &M, int t, int4 h, unsigned char *stage, int off_sh,
                                            uint64_t *bar) {
  const uint32_t shbytes = uint32_t((h.z + 3) & ~3) * 4u;
  mbar_expect_tx(bar, uint32_t(M.rec_bytes) + shbytes);
  bulk_g2s(stage, M.rec + size_t(t) * M.rec_bytes, uint32_t(M.rec_bytes), bar);
  if (shbytes) bulk_g2s(stage + off_sh, M.sh + h.w, shbytes, bar);
}

// The four shots from s0 of this thread's element point, tile in a landed stage.
template <int NC>
__device__ __forceinline__ void tileb_fetch_u(const TileMed &M, const unsigned char *stage, int off_sh, int tid,
                                              int S, int s0, float4 (&u)[NC]) {
  const int *hd = reinterpret_cast<const int *>(stage);
  const int ibeg = hd[0], nint = hd[1];
  const int k = reinterpret_cast<const uint16_t *>(stage + TREC_LIDX)[tid];
  const int g = k < nint ? ibeg + k : reinterpret_cast<const int *>(stage + off_sh)[k - nint];
#pragma unroll
  for (int c = 0; c < NC; ++c) u[c] = *reinterpret_cast<const float4 *>(M.u + (size_t(g) * NC + c) * S + s0);
}

__device__ __forceinline__ float4 add4(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

template <int NC>
__global__ void __launch_bounds__(TILE_P, 2) k_tile_b(TileBArgs A) {
  extern __shared__ __align__(128) unsigned char dyn[];
  constexpr int ST = TILEB_STAGES;
  const TileMed &M = A.el;
  const MedArgs &B = A.bel;
  const int S = A.S, NQ = S >> 2;
  const int tid = threadIdx.x;
  const int le = tid / NP, q = tid - le * NP;
  const int iz = q / NG, ix = q - iz * NG;
  const int b = blockIdx.x, G = gridDim.x;
  const int nitems = M.ntiles * NQ;
  const int nmine = b < nitems ? (nitems - 1 - b) / G + 1 : 0;
  if (nmine == 0) return;
  uint64_t *bar = reinterpret_cast<uint64_t *>(dyn);
  unsigned char *stages = dyn + 64;
  // per element: su[c][25], F0[c][25], F1[c][25] as float4 (four shots)
  float4 *su = reinterpret_cast<float4 *>(dyn + A.work_off) + le * (3 * NC * NP);
  float4 *sF = su + NC * NP;
  float4 *acc = reinterpret_cast<float4 *>(dyn + A.acc_off);
  const int kcap = A.kcap;
  const int ncol = M.ncol;
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < ST; ++s) mbar_init(bar + s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int4 hpend = make_int4(0, 0, 0, 0);
  if (tid == 0) {
    for (int j = 0; j < ST && j < nmine; ++j) {
      const int t = (b + j * G) / NQ;
      tileb_issue(M, t, __ldg(M.hdr + t), stages + j * A.stage_bytes, A.off_sh, bar + j);
    }
    if (ST < nmine) hpend = __ldg(M.hdr + (b + ST * G) / NQ);
  }
  float hx[NG], hz[NG], wx[NG], wz[NG];
#pragma unroll
  for (int l = 0; l < NG; ++l) {
    hx[l] = A.quad.hp[ix * NG + l];
    hz[l] = A.quad.hp[iz * NG + l];
    wx[l] = A.quad.hpw[l * NG + ix];
    wz[l] = A.quad.hpw[l * NG + iz];
  }
  const float wiz = A.quad.w[iz], wix = A.quad.w[ix];
  bool bad = false;
  float4 u_cur[NC];
  {
    const bool ok = mbar_wait(bar, 0u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(A.flag, 2);
        for (int k = 1; k < ST && k < nmine; ++k) mbar_wait(bar + k, 0u);
      }
      return;
    }
    tileb_fetch_u<NC>(M, stages, A.off_sh, tid, S, 4 * (b % NQ), u_cur);
  }
  for (int j = 0; j < nmine; ++j) {
    unsigned char *stage = stages + (j % ST) * A.stage_bytes;
    const int s0 = 4 * ((b + j * G) % NQ);
    float4 u_next[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) u_next[c] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (j + 1 < nmine) {
      const int sn = (j + 1) % ST;
      const bool ok = mbar_wait(bar + sn, uint32_t(((j + 1) / ST) & 1));
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicExch(A.flag, 2);
          // copies issued and not yet waited for: items j + 2 up to the last
          // issued, ST - 1 before the first refill (iteration 1), j + ST - 2 after
          const int issued = j == 0 ? ST : j + ST - 1;
          for (int k = j + 2; k < nmine && k < issued; ++k) mbar_wait(bar + (k % ST), uint32_t((k / ST) & 1));
        }
        return;
      }
      tileb_fetch_u<NC>(M, stages + sn * A.stage_bytes, A.off_sh, tid, S, 4 * ((b + (j + 1) * G) % NQ), u_next);
    }
    const int *hd = reinterpret_cast<const int *>(stage);
    const int ibeg = hd[0], nint = hd[1], nel = hd[3], rp_off = hd[4], rp_cnt = hd[5];
    const int k = reinterpret_cast<const uint16_t *>(stage + TREC_LIDX)[tid];
    const bool act = le < nel;
    const float *F = reinterpret_cast<const float *>(stage + TREC_F);
    const float xix = F[tid], xiz = F[TILE_P + tid], gax = F[2 * TILE_P + tid], gaz = F[3 * TILE_P + tid],
                jac = F[4 * TILE_P + tid], c0 = F[5 * TILE_P + tid], mu = F[6 * TILE_P + tid];
    const int bs = act ? reinterpret_cast<const int *>(stage + TREC_BC)[le] : -1;
    const int src = act ? reinterpret_cast<const int *>(stage + TREC_SRC)[le] : -1;
    const int col = act ? reinterpret_cast<const int *>(stage + TREC_COL)[le] : -1;
#pragma unroll
    for (int c = 0; c < NC; ++c) su[c * NP + q] = u_cur[c];
    __syncthreads();
    // every thread has finished item j - 1: its stage takes item j - 1 + ST
    if (tid == 0 && j >= 1 && j - 1 + ST < nmine) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tileb_issue(M, (b + (j - 1 + ST) * G) / NQ, hpend, stages + ((j - 1) % ST) * A.stage_bytes, A.off_sh,
                  bar + ((j - 1) % ST));
      if (j + ST < nmine) hpend = __ldg(M.hdr + (b + (j + ST) * G) / NQ);
    }
    // gradient of the four shots, two per FFMA2: g?[c][0] = shots (0, 1), [1] = (2, 3)
    float2 gx[NC][2], gg[NC][2];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      gx[c][0] = gx[c][1] = gg[c][0] = gg[c][1] = make_float2(0.f, 0.f);
#pragma unroll
      for (int l = 0; l < NG; ++l) {
        const float4 r4 = su[c * NP + iz * NG + l], c4 = su[c * NP + l * NG + ix];
        gx[c][0] = fma2(f2(hx[l]), make_float2(r4.x, r4.y), gx[c][0]);
        gx[c][1] = fma2(f2(hx[l]), make_float2(r4.z, r4.w), gx[c][1]);
        gg[c][0] = fma2(f2(hz[l]), make_float2(c4.x, c4.y), gg[c][0]);
        gg[c][1] = fma2(f2(hz[l]), make_float2(c4.z, c4.w), gg[c][1]);
      }
    }
    float f0[NC][4], f1[NC][4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      float dxi[NC], dga[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float2 px = gx[c][w >> 1], pg = gg[c][w >> 1];
        dxi[c] = (w & 1) ? px.y : px.x;
        dga[c] = (w & 1) ? pg.y : pg.x;
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
        f0[c][w] = jac * (Sx[c] * xix + Sz[c] * xiz);
        f1[c][w] = jac * (Sx[c] * gax + Sz[c] * gaz);
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      sF[(2 * c) * NP + q] = make_float4(f0[c][0], f0[c][1], f0[c][2], f0[c][3]);
      sF[(2 * c + 1) * NP + q] = make_float4(f1[c][0], f1[c][1], f1[c][2], f1[c][3]);
    }
    __syncthreads();
    float a[NC][4];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      float2 t1[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
      float2 t2[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
      for (int l = 0; l < NG; ++l) {
        const float4 p0 = sF[(2 * c) * NP + iz * NG + l], p1 = sF[(2 * c + 1) * NP + l * NG + ix];
        t1[0] = fma2(make_float2(p0.x, p0.y), f2(wx[l]), t1[0]);
        t1[1] = fma2(make_float2(p0.z, p0.w), f2(wx[l]), t1[1]);
        t2[0] = fma2(make_float2(p1.x, p1.y), f2(wz[l]), t2[0]);
        t2[1] = fma2(make_float2(p1.z, p1.w), f2(wz[l]), t2[1]);
      }
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        const float x1 = (w & 1) ? t1[w >> 1].y : t1[w >> 1].x;
        const float x2 = (w & 1) ? t2[w >> 1].y : t2[w >> 1].x;
        a[c][w] = -(wiz * x1 + wix * x2);
      }
    }
    const bool interior = k < nint;
    if (act) {
      const int g = interior ? ibeg + k : reinterpret_cast<const int *>(stage + A.off_sh)[k - nint];
      if (bs >= 0) {
        const size_t kb = size_t(bs) * NP + q;
        const float wq = B.bc_w[kb];
        if (wq != 0.f) {
          const float j1 = B.bc_j1[kb];
          if (NC == 2) {
            const float nx = B.bc_nx[kb], nz = B.bc_nz[kb];
            const float4 vx4 = *reinterpret_cast<const float4 *>(M.v + (size_t(g) * NC) * S + s0);
            const float4 vz4 = *reinterpret_cast<const float4 *>(M.v + (size_t(g) * NC + NC - 1) * S + s0);
            const float rvp = B.bc_imp0[kb], rvs = B.bc_imp1[kb];
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
            const float4 v4 = *reinterpret_cast<const float4 *>(M.v + size_t(g) * S + s0);
            const float imp = B.bc_imp1[kb];
#pragma unroll
            for (int w = 0; w < 4; ++w) a[0][w] += -1.f * (wq * j1) * imp * (&v4.x)[w];
          }
        }
      }
      if (src >= 0) {
        const int step = *A.step;
        for (int s = src; s >= 0; s = A.src_next[s]) {
          const int w = A.src_shot[s] - s0;
          if (w < 0 || w > 3) continue;
          const float f = step < A.nstep ? A.stf[size_t(step) * A.nsrc + s] : 0.f;
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            const float add = f * A.src_arr[(size_t(s) * 2 + c) * NP + q];
            // sources in chain order, as the one-shot kernel adds them
            if (w == 0) a[c][0] += add;
            else if (w == 1) a[c][1] += add;
            else if (w == 2) a[c][2] += add;
            else a[c][3] += add;
          }
        }
      }
      if (interior) {
        // the point's slot of this element's colour (one element per colour)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[(col * NC + c) * kcap + k] = make_float4(a[c][0], a[c][1], a[c][2], a[c][3]);
      } else {
        const size_t bi = g < M.niface ? size_t(g) : size_t(M.niface) + (g - M.sh0);
#pragma unroll
        for (int c = 0; c < NC; ++c)
          *reinterpret_cast<float4 *>(M.r + ((bi * ncol + col) * NC + c) * S + s0) =
              make_float4(a[c][0], a[c][1], a[c][2], a[c][3]);
      }
    }
    __syncthreads();
    // the tile-interior points, one thread each: the slots of the colours
    // present in increasing colour order, then M^-1, corrector, predictor
    for (int kk = tid; kk < nint; kk += blockDim.x) {
      const int mk = stage[TREC_MASK + kk];
      float4 sum[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) sum[c] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int cl = 0; cl < TILE_MAX_COLORS; ++cl)
        if (mk >> cl & 1) {
#pragma unroll
          for (int c = 0; c < NC; ++c) sum[c] = add4(sum[c], acc[(cl * NC + c) * kcap + kk]);
        }
      const size_t gi = size_t(ibeg + kk);
      float4 uu[NC], vv[NC], ac[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const size_t o = (gi * NC + c) * S + s0;
        const float mi = M.minv[gi * NC + c];
        uu[c] = *reinterpret_cast<const float4 *>(M.u + o);
        vv[c] = *reinterpret_cast<const float4 *>(M.v + o);
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          (&ac[c].x)[w] = __fmul_rn((&sum[c].x)[w], mi);
          (&vv[c].x)[w] = newmark_correct((&vv[c].x)[w], (&ac[c].x)[w], A.dt2);
        }
      }
      if (rp_cnt > 0) {
        // receiver points of the tile (sorted by local index): u of the
        // step, corrected v, new a for the side buffer
        for (int i = 0; i < rp_cnt; ++i) {
          const int2 e = __ldg(M.rp + rp_off + i);
          if (e.x > kk) break;
          if (e.x == kk) {
            float *dst = A.side + size_t(e.y) * SIDEB_W * S + s0;
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              *reinterpret_cast<float4 *>(dst + size_t(c) * S) = uu[c];
              *reinterpret_cast<float4 *>(dst + size_t(2 + c) * S) = vv[c];
              *reinterpret_cast<float4 *>(dst + size_t(4 + c) * S) = ac[c];
            }
          }
        }
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          if (A.predict) newmark_predict((&uu[c].x)[w], (&vv[c].x)[w], (&ac[c].x)[w], A.dt, A.dt2, A.dtsq2);
          bad |= !isfinite((&uu[c].x)[w]);
        }
        const size_t o = (gi * NC + c) * S + s0;
        if (A.predict) *reinterpret_cast<float4 *>(M.u + o) = uu[c];
        *reinterpret_cast<float4 *>(M.v + o) = vv[c];
        if (M.store_a) *reinterpret_cast<float4 *>(M.a + o) = ac[c];
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) u_cur[c] = u_next[c];
  }
  if (bad) *A.flag = 1;
}

// Boundary points, one thread per point and quad of shots: the per-colour
// contributions in colour order (absent colours hold zero), M^-1, corrector,
// predictor.  Advances the step counter.
template <int NC>
__global__ void __launch_bounds__(256) k_tile_boundary_b(UpdateArgs A, BndMed Bm, float *side, int S) {
  const int NQ = S >> 2;
  const int n = Bm.nb * NQ;
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int bi = i / NQ, s0 = 4 * (i - bi * NQ);
    const int g = bnd_point_id(Bm, bi);
    // the slots of the colours that touch the point (the others hold zero):
    // all loads first, then the sum in increasing colour order
    const int mk = Bm.b_mask[bi];
    float4 cv[TILE_MAX_COLORS][NC];
#pragma unroll
    for (int cl = 0; cl < TILE_MAX_COLORS; ++cl)
      if (mk >> cl & 1) {
#pragma unroll
        for (int c = 0; c < NC; ++c)
          cv[cl][c] = *reinterpret_cast<const float4 *>(Bm.r + ((size_t(bi) * Bm.ncol + cl) * NC + c) * S + s0);
      }
    float4 acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int cl = 0; cl < TILE_MAX_COLORS; ++cl)
      if (mk >> cl & 1) {
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = add4(acc[c], cv[cl][c]);
      }
    float4 uu[NC], vv[NC], ac[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const size_t o = (size_t(g) * NC + c) * S + s0;
      const float mi = A.minv[size_t(g) * NC + c];
      uu[c] = *reinterpret_cast<const float4 *>(A.u + o);
      vv[c] = *reinterpret_cast<const float4 *>(A.v + o);
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        (&ac[c].x)[w] = __fmul_rn((&acc[c].x)[w], mi);
        (&vv[c].x)[w] = newmark_correct((&vv[c].x)[w], (&ac[c].x)[w], A.dt2);
      }
    }
    if (Bm.b_side) {
      const int sl = Bm.b_side[bi];
      if (sl >= 0) {
        float *dst = side + size_t(sl) * SIDEB_W * S + s0;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          *reinterpret_cast<float4 *>(dst + size_t(c) * S) = uu[c];
          *reinterpret_cast<float4 *>(dst + size_t(2 + c) * S) = vv[c];
          *reinterpret_cast<float4 *>(dst + size_t(4 + c) * S) = ac[c];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        if (A.predict) newmark_predict((&uu[c].x)[w], (&vv[c].x)[w], (&ac[c].x)[w], A.dt, A.dt2, A.dtsq2);
        bad |= !isfinite((&uu[c].x)[w]);
      }
      const size_t o = (size_t(g) * NC + c) * S + s0;
      if (A.predict) *reinterpret_cast<float4 *>(A.u + o) = uu[c];
      *reinterpret_cast<float4 *>(A.v + o) = vv[c];
      if (A.a_store) *reinterpret_cast<float4 *>(A.a_store + o) = ac[c];
    }
  }
  if (bad) *A.flag = 1;
  if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) *A.step += 1;
}

// Receivers after the boundary kernel (the step counter already advanced):
// one block per receiver, lanes over shots; the 25 weighted values summed in
// the order of k_receivers_batched (and of the single-shot xor butterfly).
__global__ void __launch_bounds__(32) k_receivers_side_b(RecArgs A, const int *__restrict__ rslot,
                                                         const float *__restrict__ side, int S) {
  const int step = *A.step - 1;
  if (step < 0 || step % A.nsb != 0) return;
  const int isig = step / A.nsb;
  if (isig >= A.nsig) return;
  const int r = A.rec_list[blockIdx.x];
  const int NC = A.ncomp;
  for (int s0 = 0; s0 < S; s0 += 32) {
    const int shot = s0 + threadIdx.x;
    if (shot >= S) continue;
    for (int t = 0; t < A.ntypes; ++t) {
      const int f = A.types[t] < 2 ? A.types[t] : 2;
      float tr[2] = {0.f, 0.f};
      for (int c = 0; c < NC; ++c) {
        float x[32];
#pragma unroll
        for (int q = 0; q < 32; ++q) x[q] = 0.f;
        for (int q = 0; q < NP; ++q) {
          const float val = side[(size_t(rslot[size_t(r) * NP + q]) * SIDEB_W + 2 * f + c) * S + shot];
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
