// Fused tile kernel of the 2D time step: element forces, assembly and the
// Newmark point update in one launch (single shot; isotropic P-SV, SH and
// acoustic media, coupled media whose interface points pair one to one).
//
// Tiles.  The elements of each medium are grouped into tiles of TILE_E = 16
// elements that lie close together (a 4 x 4 block on structured meshes).  A
// point only one tile touches, and that lies on no coupled edge, is interior
// to the tile, and the point numbering gives a tile's interior points one
// contiguous range.  Every other point (shared by tiles, or on a coupled
// edge) is a boundary point.
//
// k_tile (persistent, one CTA per 16-element tile at a time, 400 threads =
// one per element GLL point).  Per tile a 4-stage ring of shared-memory
// buffers receives, by cp.async.bulk copies completing on one mbarrier per
// stage, the tile record (local point indices, Stacey slot / source head /
// colour per element, the Jacobian and material arrays) and the tile's
// shared-point ids, and the displacement, velocity and M^-1 of its interior
// range; copies run three tiles ahead of the arithmetic.  Each thread's
// displacement is taken one tile ahead (interior: from the staged range;
// shared: a load from HBM, issued before the current tile's arithmetic).
// Then the element arithmetic of k_stiffness (gradient by the 5-term
// Lagrange contractions, stress, F = J sigma grad(xi), divergence, Stacey /
// free-surface / source epilogue), operand for operand.  Assembly: within a
// mesh colour no two elements share a point, so every interior point has one
// shared-memory slot per colour; each element point writes its contribution
// to its point's slot of its element's colour, and after one barrier one
// thread per tile-interior point sums the slots of the colours that touch it
// (a mask per point in the tile record) in increasing colour order, as the
// colour-pass and owner-computes kernels sum: the results are bit-identical
// to theirs.  Contributions at boundary points go to per-colour slots in HBM
// (slots of colours that do not touch a point hold zero; adding zero
// changes no value).  Finally the interior points get
// a = sum * M^-1, the corrector and (inside a run) the next predictor, and
// are written back.
// Reference: include/kokkos_kernels/impl/compute_stiffness_interaction.tpp:140-247,
// include/algorithms/gradient.hpp:40-82, divergence.hpp:41-74,
// include/kokkos_kernels/impl/divide_mass_matrix.tpp:10-65,
// core/specfem/timescheme/newmark.tpp:10-128.
//
// k_tile_boundary: the boundary points, one thread each: the contributions
// in colour order (one slot per colour), coupling, M^-1, corrector,
// predictor; on a coupled
// interface the acoustic partner first, as k_update_coupled.  It advances
// the step counter.
//
// k_receivers_side: receivers read the end-of-step values (u of the step,
// corrected v, new a) of their element's points from a side buffer that the
// two kernels above fill for the points receivers use; same arithmetic as
// k_receivers (compute_seismogram.tpp:19-171).
//
// Every mbarrier wait has an iteration limit; a wait that gives up sets the
// device flag to 2 and the block drains its own copies before it returns.
#pragma once

#include "kernels2d.cuh"
#include "kernels2d_tma.cuh"

namespace sfg {
namespace dev {

constexpr int TILE_E = 16;
constexpr int TILE_P = TILE_E * NP;  // element points of a tile = threads of a block
constexpr int TILE_STAGES = 4;
// tile record (bytes): header {ibeg, nint, nsh, nel, rp_off, rp_cnt, 0, 0},
// lidx u16[400], mask u8[400] (tile-interior point k: the colours of the
// tile's elements that touch it),
// bc_slot / src_head / colour int[16] each, then nf float arrays [400]:
// xi_x, xi_z, gamma_x, gamma_z, |J|, material words
constexpr int TREC_LIDX = 32, TREC_MASK = 832, TREC_BC = 1232, TREC_SRC = 1296, TREC_COL = 1360,
              TREC_F = 1424;
constexpr int TILE_MAX_COLORS = 7;
__host__ __device__ constexpr int tile_rec_bytes(int nf) { return TREC_F + nf * TILE_P * 4; }
constexpr int TILE_WORK = 2 * 4 * NG * 8 + 4;  // per element: NC x {U, UT, F0, F1T} rows of 8, +4
constexpr int SIDE_W = 8;                      // side buffer words per point: u(2) v(2) a(2) - -

struct TileMed {
  const int4 *hdr;             // [ntiles] {ibeg, nint, nsh, sh_off}
  const unsigned char *rec;    // [ntiles][rec_bytes]
  const int *sh;               // shared-point ids, each tile's list 16-byte aligned
  const int2 *rp;              // receiver points of the tiles (local index, side slot)
  float *u, *v, *a;
  const float *minv;           // padded by 4 floats
  // contributions at boundary points, one slot per colour:
  // r[(b * ncol + colour) * NC + c], b the boundary index of the point
  // (point for points below niface, niface + point - sh0 for the others);
  // slots of colours that do not touch a point stay zero
  float *r;
  int rec_bytes, ntiles, nblocks, ncol, niface, sh0;
  int store_a;                 // write the new acceleration of interior points
};

struct TileArgs {
  TileMed el, ac;
  MedArgs bel, bac;            // Stacey / free-surface arrays of each medium
  const int *src_next;
  const float *src_arr;        // [nsrc][2][25]
  const float *stf;            // [nstep][nsrc]
  int nsrc, nstep;
  const int *step;
  float dt, dt2, dtsq2;
  int predict;
  int *flag;
  float *side;
  // dynamic shared memory layout (bytes): 64 bytes of barriers, the stages,
  // the element work arrays, the accumulators
  int stage_bytes, off_sh, off_u, off_v, off_m, work_off, acc_off, acc_words;
  Quad quad;
};

// Issue the bulk copies of tile t (header h) into one stage (one thread).
template <int NC>
__device__ __forceinline__ void tile_issue(const TileArgs &A, const TileMed &M, int t, int4 h, unsigned char *stage,
                                           uint64_t *bar) {
  const int ibeg = h.x, nint = h.y, nsh = h.z, shoff = h.w;
  const int v0 = (ibeg * NC) & ~3, v1 = ((ibeg + nint) * NC + 3) & ~3;
  const uint32_t fbytes = uint32_t(v1 - v0) * 4u;
  const uint32_t shbytes = uint32_t((nsh + 3) & ~3) * 4u;
  mbar_expect_tx(bar, uint32_t(M.rec_bytes) + shbytes + 3u * fbytes);
  bulk_g2s(stage, M.rec + size_t(t) * M.rec_bytes, uint32_t(M.rec_bytes), bar);
  if (shbytes) bulk_g2s(stage + A.off_sh, M.sh + shoff, shbytes, bar);
  if (fbytes) {
    bulk_g2s(stage + A.off_u, M.u + v0, fbytes, bar);
    bulk_g2s(stage + A.off_v, M.v + v0, fbytes, bar);
    bulk_g2s(stage + A.off_m, M.minv + v0, fbytes, bar);
  }
}

// This thread's displacement in a landed stage.
template <int NC>
__device__ __forceinline__ float2 tile_fetch_u(const TileArgs &A, const TileMed &M, const unsigned char *stage,
                                               int tid) {
  const int *hd = reinterpret_cast<const int *>(stage);
  const int ibeg = hd[0], nint = hd[1];
  const int k = reinterpret_cast<const uint16_t *>(stage + TREC_LIDX)[tid];
  if (k < nint) {
    const float *uin = reinterpret_cast<const float *>(stage + A.off_u);
    const int o = (ibeg + k) * NC - ((ibeg * NC) & ~3);
    return make_float2(uin[o], NC == 2 ? uin[o + 1] : 0.f);
  }
  const int g = reinterpret_cast<const int *>(stage + A.off_sh)[k - nint];
  if (NC == 2) return reinterpret_cast<const float2 *>(M.u)[g];
  return make_float2(M.u[g], 0.f);
}

// Finish tile-interior point k from the sum of its contributions: M^-1,
// corrector and (inside a run) the next predictor, written to HBM.  With
// receiver points in the tile the corrected velocity and the acceleration
// are kept in shared memory (staged v, colour-0 slot) for the side buffer.
template <int NC>
__device__ __forceinline__ bool tile_finish(const TileArgs &A, const TileMed &M, int ibeg, int v0, int k, int kcap,
                                            const float (&sum)[NC], const float *uin, float *vin,
                                            const float *min, float *acc, bool keep) {
  const int o = (ibeg + k) * NC - v0;
  float au[NC], vv[NC], ac[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    ac[c] = __fmul_rn(sum[c], min[o + c]);
    au[c] = uin[o + c];
    vv[c] = newmark_correct(vin[o + c], ac[c], A.dt2);
  }
  if (keep) {
#pragma unroll
    for (int c = 0; c < NC; ++c) { vin[o + c] = vv[c]; acc[c * kcap + k] = ac[c]; }
  }
  bool bad = false;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (A.predict) newmark_predict(au[c], vv[c], ac[c], A.dt, A.dt2, A.dtsq2);
    bad |= !isfinite(au[c]);
  }
  const size_t gi = size_t(ibeg + k);
  if (NC == 2) {
    if (A.predict) reinterpret_cast<float2 *>(M.u)[gi] = make_float2(au[0], au[NC - 1]);
    reinterpret_cast<float2 *>(M.v)[gi] = make_float2(vv[0], vv[NC - 1]);
    if (M.store_a) reinterpret_cast<float2 *>(M.a)[gi] = make_float2(ac[0], ac[NC - 1]);
  } else {
    if (A.predict) M.u[gi] = au[0];
    M.v[gi] = vv[0];
    if (M.store_a) M.a[gi] = ac[0];
  }
  return bad;
}

// Tiles b, b + G, ... of one medium (KIND 0 acoustic, 1 elastic SH, 2 P-SV).
template <int KIND>
__device__ __forceinline__ void tile_loop(const TileArgs &A, const TileMed &M, const MedArgs &B, int b, int G,
                                          unsigned char *dyn) {
  constexpr int NC = KIND == 2 ? 2 : 1;
  constexpr int S = TILE_STAGES;
  constexpr int RS = 8, ARR = NG * RS;
  const int tid = threadIdx.x;
  const int le = tid / NP, q = tid - le * NP;
  const int iz = q / NG, ix = q - iz * NG;
  uint64_t *bar = reinterpret_cast<uint64_t *>(dyn);
  unsigned char *stages = dyn + 64;
  float *base = reinterpret_cast<float *>(dyn + A.work_off) + le * TILE_WORK;
  float *acc = reinterpret_cast<float *>(dyn + A.acc_off);
  const int nmine = b < M.ntiles ? (M.ntiles - 1 - b) / G + 1 : 0;
  if (nmine == 0) return;
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) mbar_init(bar + s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < A.acc_words; i += blockDim.x) acc[i] = 0.f;
  __syncthreads();
  // the header of the next tile to issue is loaded one tile ahead (by the
  // issuing thread), so the issue itself waits for no load
  int4 hpend = make_int4(0, 0, 0, 0);
  if (tid == 0) {
    for (int j = 0; j < S && j < nmine; ++j)
      tile_issue<NC>(A, M, b + j * G, __ldg(M.hdr + b + j * G), stages + j * A.stage_bytes, bar + j);
    if (S < nmine) hpend = __ldg(M.hdr + b + S * G);
  }
  const int ncol = M.ncol;
  const int kcap = A.acc_words / (ncol * NC > 0 ? ncol * NC : 1);   // slots [colour][c][point]
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
  float2 u_cur = make_float2(0.f, 0.f);
  int j = 0;
  {
    const bool ok = mbar_wait(bar, 0u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(A.flag, 2);
        for (int k = 1; k < S && k < nmine; ++k) mbar_wait(bar + k, 0u);
      }
      return;
    }
    u_cur = tile_fetch_u<NC>(A, M, stages, tid);
  }
  for (; j < nmine; ++j) {
    const int st = j % S;
    unsigned char *stage = stages + st * A.stage_bytes;
    float2 u_next = make_float2(0.f, 0.f);
    if (j + 1 < nmine) {
      const int sn = (j + 1) % S;
      const bool ok = mbar_wait(bar + sn, uint32_t(((j + 1) / S) & 1));
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicExch(A.flag, 2);
          // copies issued and not yet waited for: tiles j + 2 up to the last
          // issued, S - 1 before the first refill (iteration 1), j + S - 2 after
          const int issued = j == 0 ? S : j + S - 1;
          for (int k = j + 2; k < nmine && k < issued; ++k) mbar_wait(bar + (k % S), uint32_t((k / S) & 1));
        }
        return;
      }
      u_next = tile_fetch_u<NC>(A, M, stages + sn * A.stage_bytes, tid);
    }
    const int *hd = reinterpret_cast<const int *>(stage);
    const int ibeg = hd[0], nint = hd[1], nel = hd[3], rp_off = hd[4], rp_cnt = hd[5];
    const int k = reinterpret_cast<const uint16_t *>(stage + TREC_LIDX)[tid];
    const bool act = le < nel;
    const float *F = reinterpret_cast<const float *>(stage + TREC_F);
    const float xix = F[tid], xiz = F[TILE_P + tid], gax = F[2 * TILE_P + tid], gaz = F[3 * TILE_P + tid],
                jac = F[4 * TILE_P + tid], c0 = F[5 * TILE_P + tid];
    const float c1 = KIND == 0 ? 0.f : F[6 * TILE_P + tid];
    const int bs = act ? reinterpret_cast<const int *>(stage + TREC_BC)[le] : -1;
    const int src = act ? reinterpret_cast<const int *>(stage + TREC_SRC)[le] : -1;
    const int col = act ? reinterpret_cast<const int *>(stage + TREC_COL)[le] : -1;
    float uu[NC];
    uu[0] = u_cur.x;
    if (NC == 2) uu[NC - 1] = u_cur.y;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      base[(c * 4 + 0) * ARR + iz * RS + ix] = uu[c];
      base[(c * 4 + 1) * ARR + ix * RS + iz] = uu[c];
    }
    __syncthreads();
    // every thread has finished tile j - 1: its stage takes tile j - 1 + S
    if (tid == 0 && j >= 1 && j - 1 + S < nmine) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tile_issue<NC>(A, M, b + (j - 1 + S) * G, hpend, stages + ((j - 1) % S) * A.stage_bytes, bar + ((j - 1) % S));
      if (j + S < nmine) hpend = __ldg(M.hdr + b + (j + S) * G);
    }
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
        const float kk = KIND == 0 ? c0 : c1;
        Sx[0] = kk * (xix * dxi[0] + gax * dga[0]);
        Sz[0] = kk * (xiz * dxi[0] + gaz * dga[0]);
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      base[(c * 4 + 2) * ARR + iz * RS + ix] = jac * (Sx[c] * xix + Sz[c] * xiz);
      base[(c * 4 + 3) * ARR + ix * RS + iz] = jac * (Sx[c] * gax + Sz[c] * gaz);
    }
    __syncthreads();
    float a[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const float t1 = dot5(base + (c * 4 + 2) * ARR + iz * RS, wx);
      const float t2 = dot5(base + (c * 4 + 3) * ARR + ix * RS, wz);
      a[c] = -(wiz * t1 + wix * t2);
    }
    const bool interior = k < nint;
    const int v0 = (ibeg * NC) & ~3;
    float *uin = reinterpret_cast<float *>(stage + A.off_u);
    float *vin = reinterpret_cast<float *>(stage + A.off_v);
    const float *min = reinterpret_cast<const float *>(stage + A.off_m);
    if (act) {
      if (bs >= 0) {
        const int g = interior ? ibeg + k : reinterpret_cast<const int *>(stage + A.off_sh)[k - nint];
        const size_t kb = size_t(bs) * NP + q;
        const float wq = B.bc_w[kb];
        if (KIND == 2) {
          if (wq != 0.f) {
            const float nx = B.bc_nx[kb], nz = B.bc_nz[kb], j1 = B.bc_j1[kb];
            const float2 vv = reinterpret_cast<const float2 *>(M.v)[g];
            const float rvp = B.bc_imp0[kb], rvs = B.bc_imp1[kb];
            const float vn = vv.x * nx + vv.y * nz;
            const float fx = ((vn * nx / (j1 * j1)) * (rvp - rvs)) + vv.x * rvs;
            const float fz = ((vn * nz / (j1 * j1)) * (rvp - rvs)) + vv.y * rvs;
            a[0] += -1.f * fx * j1 * wq;
            a[NC - 1] += -1.f * fz * j1 * wq;
          }
        } else {
          if (wq != 0.f) {
            const float imp = KIND == 0 ? B.bc_imp0[kb] : B.bc_imp1[kb];
            a[0] += -1.f * (wq * B.bc_j1[kb]) * imp * M.v[g];
          }
          if (KIND == 0) a[0] *= B.bc_keep[kb];
        }
      }
      if (src >= 0) {
        const int step = *A.step;
        for (int s = src; s >= 0; s = A.src_next[s]) {
          const float f = step < A.nstep ? A.stf[size_t(step) * A.nsrc + s] : 0.f;
#pragma unroll
          for (int c = 0; c < NC; ++c) a[c] += f * A.src_arr[(size_t(s) * 2 + c) * NP + q];
        }
      }
      if (interior) {
        // the point's slot of this element's colour (one element per colour)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[(col * NC + c) * kcap + k] = a[c];
      } else {
        const int g = reinterpret_cast<const int *>(stage + A.off_sh)[k - nint];
        const size_t bi = g < M.niface ? size_t(g) : size_t(M.niface) + (g - M.sh0);
        const size_t pr = bi * ncol + col;
        if (NC == 2) reinterpret_cast<float2 *>(M.r)[pr] = make_float2(a[0], a[NC - 1]);
        else M.r[pr] = a[0];
      }
    }
    __syncthreads();
    // the tile-interior points, one thread each: the slots of the colours
    // present, in increasing colour order, then M^-1, corrector, predictor
    for (int kk = tid; kk < nint; kk += blockDim.x) {
      const int mk = stage[TREC_MASK + kk];
      float sum[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) sum[c] = 0.f;
#pragma unroll
      for (int cl = 0; cl < TILE_MAX_COLORS; ++cl)
        if (mk >> cl & 1) {
#pragma unroll
          for (int c = 0; c < NC; ++c) sum[c] = sum[c] + acc[(cl * NC + c) * kcap + kk];
        }
      bad |= tile_finish<NC>(A, M, ibeg, v0, kk, kcap, sum, uin, vin, min, acc, rp_cnt > 0);
    }
    if (rp_cnt > 0) {
      // receiver points of the tile: u of the step, corrected v, new a
      __syncthreads();
      for (int i = tid; i < rp_cnt; i += blockDim.x) {
        const int2 e = __ldg(M.rp + rp_off + i);
        const int o = (ibeg + e.x) * NC - v0;
        float *dst = A.side + size_t(e.y) * SIDE_W;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          dst[c] = uin[o + c];
          dst[2 + c] = vin[o + c];
          dst[4 + c] = acc[c * kcap + e.x];
        }
      }
    }
    u_cur = u_next;
  }
  if (bad) *A.flag = 1;
}

// One launch for both media: blocks [0, el.nblocks) walk the elastic tiles,
// the others the acoustic ones.  EK 0 P-SV, 1 SH.
template <int EK>
__global__ void __launch_bounds__(TILE_P, 2) k_tile(TileArgs A) {
  extern __shared__ __align__(128) unsigned char dyn[];
  const int b = blockIdx.x;
  if (b < A.el.nblocks)
    tile_loop<EK == 0 ? 2 : 1>(A, A.el, A.bel, b, A.el.nblocks, dyn);
  else
    tile_loop<0>(A, A.ac, A.bac, b - A.el.nblocks, A.ac.nblocks, dyn);
}

// ---------------------------------------------------------------------------
// Boundary points.

struct BndMed {
  const float *r;              // TileMed::r: one slot per colour and boundary point
  const int *b_side;           // side slot of a boundary point (-1: none), or null
  const unsigned char *b_mask; // colours of the elements touching a boundary point
  int nb, niface, sh0, ncol;
};

template <int NC>
__device__ __forceinline__ bool bnd_point(const UpdateArgs &A, const BndMed &B, int bi, int g, float *side) {
  float acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.f;
  // the contributions in colour order (absent colours hold zero)
  const float *sl = B.r + size_t(bi) * B.ncol * NC;
  float cv[TILE_MAX_COLORS][NC];
#pragma unroll
  for (int cl = 0; cl < TILE_MAX_COLORS; ++cl) {   // all loads first, then the sum in order
    if (cl < B.ncol) {
      if (NC == 2) {
        const float2 t = reinterpret_cast<const float2 *>(sl)[cl];
        cv[cl][0] = t.x;
        cv[cl][NC - 1] = t.y;
      } else {
        cv[cl][0] = sl[cl];
      }
    }
  }
#pragma unroll
  for (int cl = 0; cl < TILE_MAX_COLORS; ++cl)
    if (cl < B.ncol) {
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[c] = acc[c] + cv[cl][c];
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
    uu[0] = A.u[g]; vv[0] = A.v[g]; mi[0] = A.minv[g];
  }
  float a[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) a[c] = __fmul_rn(acc[c], mi[c]);
  bool bad = false;
#pragma unroll
  for (int c = 0; c < NC; ++c) vv[c] = newmark_correct(vv[c], a[c], A.dt2);
  if (B.b_side) {
    const int sl = B.b_side[bi];
    if (sl >= 0) {
      float *dst = side + size_t(sl) * SIDE_W;
#pragma unroll
      for (int c = 0; c < NC; ++c) { dst[c] = uu[c]; dst[2 + c] = vv[c]; dst[4 + c] = a[c]; }
    }
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (A.predict) newmark_predict(uu[c], vv[c], a[c], A.dt, A.dt2, A.dtsq2);
    bad |= !isfinite(uu[c]);
  }
  if (NC == 2) {
    if (A.predict) reinterpret_cast<float2 *>(A.u)[g] = make_float2(uu[0], uu[NC - 1]);
    reinterpret_cast<float2 *>(A.v)[g] = make_float2(vv[0], vv[NC - 1]);
    if (A.a_store) reinterpret_cast<float2 *>(A.a_store)[g] = make_float2(a[0], a[NC - 1]);
  } else {
    if (A.predict) A.u[g] = uu[0];
    A.v[g] = vv[0];
    if (A.a_store) A.a_store[g] = a[0];
  }
  return bad;
}

__device__ __forceinline__ int bnd_point_id(const BndMed &B, int bi) {
  return bi < B.niface ? bi : B.sh0 + (bi - B.niface);
}

// Boundary points of the first medium (NCF components), then, when COUPLED,
// the acoustic boundary points past the interface; an interface point of the
// first medium updates its acoustic partner first.
template <int NCF, bool COUPLED>
__global__ void __launch_bounds__(256) k_tile_boundary(UpdateArgs F, BndMed BF, UpdateArgs Ac, BndMed BA,
                                                       float *side) {
  const int nf = BF.nb, na = COUPLED ? BA.nb - BA.niface : 0;
  const int stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nf + na; t += stride) {
    if (t < nf) {
      const int g = bnd_point_id(BF, t);
      if (COUPLED && g < F.niface) {
        const int ga = F.cp_other[g];
        bad |= bnd_point<1>(Ac, BA, ga, ga, side);
      }
      bad |= bnd_point<NCF>(F, BF, t, g, side);
    } else {
      const int bi = BA.niface + (t - nf);
      bad |= bnd_point<1>(Ac, BA, bi, bnd_point_id(BA, bi), side);
    }
  }
  if (bad) *F.flag = 1;
  if (F.advance && blockIdx.x == 0 && threadIdx.x == 0) *F.step += 1;
}

// ---------------------------------------------------------------------------
// Receivers after the boundary kernel (the step counter already advanced).
__global__ void __launch_bounds__(32) k_receivers_side(RecArgs A, const int *__restrict__ rslot,
                                                       const float *__restrict__ side) {
  __shared__ float sf[3][NP];
  const int step = *A.step - 1;
  if (step < 0 || step % A.nsb != 0) return;
  const int isig = step / A.nsb;
  if (isig >= A.nsig) return;
  const int r = A.rec_list[blockIdx.x];
  const int ce = A.rec_elem[r];
  const int lane = threadIdx.x;
  const bool on = lane < NP;
  const int q = on ? lane : 0;
  const size_t p = size_t(ce) * NP + q;
  const float h = on ? A.rec_h[size_t(r) * NP + q] : 0.f;
  const float *sv = side + size_t(rslot[size_t(r) * NP + q]) * SIDE_W;
  if (!A.acoustic) {
    const int nc = A.ncomp;
    for (int t = 0; t < A.ntypes; ++t) {
      float o[2] = {0.f, 0.f};
      const int ty = A.types[t];
      if (ty == 3) {
        // pressure -(lambda + 2/3 mu) div u from the displacement gradient
        // (include/medium/dim2/elastic/isotropic/wavefield.hpp:57-89)
        float pr = 0.f;
        if (nc >= 2) {
          const int iz = q / NG, ix = q - iz * NG;
          float dxi0 = 0.f, dxi1 = 0.f, dga0 = 0.f, dga1 = 0.f;
          for (int l = 0; l < NG; ++l) {
            const float *sr = side + size_t(rslot[size_t(r) * NP + iz * NG + l]) * SIDE_W;
            const float *sc = side + size_t(rslot[size_t(r) * NP + l * NG + ix]) * SIDE_W;
            const float hx = A.quad.hp[ix * NG + l], hz = A.quad.hp[iz * NG + l];
            dxi0 += hx * sr[0];
            dxi1 += hx * sr[1];
            dga0 += hz * sc[0];
            dga1 += hz * sc[1];
          }
          if (on) {
            const float dux = A.xix[p] * dxi0 + A.gax[p] * dga0;
            const float duz = A.xiz[p] * dxi1 + A.gaz[p] * dga1;
            const float l2m = A.prop0[p], mu = A.prop1[p];
            pr = -1.f * ((l2m - 2.f * mu + (2.f / 3.f) * mu) * (dux + duz));
          }
        }
        o[0] = warp_sum(h * pr);
      } else {
        for (int c = 0; c < (nc < 2 ? nc : 2); ++c) {
          const float val = ty == 0 ? sv[c] : (ty == 1 ? sv[2 + c] : sv[4 + c]);
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
  if (on) {
    sf[0][q] = sv[0];
    sf[1][q] = sv[2];
    sf[2][q] = sv[4];
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
