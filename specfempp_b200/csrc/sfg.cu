// libsfg: handle management, device upload, step scheduling (CUDA graphs) and
// the extern "C" entry points declared in include/sfg.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/sfg.h"
#include "host2d.hpp"
#include "kernels2d.cuh"
#include "kernels2d_batched.cuh"
#include "kernels2d_adjoint.cuh"
#include "kernels2d_tma.cuh"
#include "kernels2d_tile.cuh"
#include "kernels2d_tile_batched.cuh"
#include "kernels2d_row.cuh"
#include "kernels2d_btile.cuh"

namespace {

thread_local std::string g_create_error;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define SFG_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t _e = (call);                                                             \
    if (_e != cudaSuccess)                                                               \
      throw CudaError(std::string(#call) + ": " + cudaGetErrorString(_e));               \
  } while (0)

// Device buffer list owned by a handle.
struct DevMem {
  std::vector<void *> ptrs;
  size_t bytes = 0;
  template <typename T>
  T *upload(const std::vector<T> &h) {
    if (h.empty()) return nullptr;
    T *d = nullptr;
    SFG_CUDA(cudaMalloc(&d, h.size() * sizeof(T)));
    ptrs.push_back(d);
    bytes += h.size() * sizeof(T);
    SFG_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
  }
  template <typename T>
  T *zeros(size_t n) {
    if (n == 0) return nullptr;
    T *d = nullptr;
    SFG_CUDA(cudaMalloc(&d, n * sizeof(T)));
    ptrs.push_back(d);
    bytes += n * sizeof(T);
    SFG_CUDA(cudaMemset(d, 0, n * sizeof(T)));
    return d;
  }
  void free_all() {
    for (void *p : ptrs) cudaFree(p);
    ptrs.clear();
    bytes = 0;
  }
};

struct DevMedium {
  int nspec = 0, nglob = 0, ncomp = 0;
  int S = 1;                       // shots sharing the mesh: fields are [point][comp][shot]
  size_t values() const { return size_t(nglob) * ncomp * S; }
  std::vector<int> color_start;
  int *ibool = nullptr;
  float *xix = nullptr, *xiz = nullptr, *gax = nullptr, *gaz = nullptr, *jac = nullptr,
        *prop0 = nullptr, *prop1 = nullptr;
  float *prop2 = nullptr, *prop3 = nullptr, *prop4 = nullptr, *prop5 = nullptr;  // anisotropic / Cosserat
  float *prop6 = nullptr, *prop7 = nullptr, *prop8 = nullptr;                      // poroelastic damping
  bool aniso = false, poro = false;
  int *bc_slot = nullptr;
  float *bc_w = nullptr, *bc_nx = nullptr, *bc_nz = nullptr, *bc_j1 = nullptr,
        *bc_imp0 = nullptr, *bc_imp1 = nullptr, *bc_keep = nullptr, *bc_imp2 = nullptr;
  int niface = 0;
  float *cp_nx = nullptr, *cp_nz = nullptr;
  int *cp_other = nullptr;
  int *cp_start = nullptr;         // nonconforming interfaces: entry ranges per point
  int *src_head = nullptr;
  float *minv = nullptr;
  float *u = nullptr, *v = nullptr, *accum = nullptr, *a = nullptr;
  float *r = nullptr;              // element-local contributions (owner-computes assembly)
  int *inv_start = nullptr;
  int *slot = nullptr;  // CSR position of each element point's contribution
  int *rec_list = nullptr;
  int nrec = 0;
  // fused tile kernel: tile headers and records, shared-point lists,
  // receiver points of the tiles, per-colour contributions at boundary
  // points and the boundary points' side slots
  int ntiles = 0, sh0 = 0, nb = 0, rec_bytes = 0, max_nint = 0, max_nsh = 0;
  int4 *t_hdr = nullptr;
  unsigned char *t_rec = nullptr;
  int *t_sh = nullptr;
  int2 *t_rp = nullptr;
  float *t_r = nullptr;
  int *b_side = nullptr;
  unsigned char *b_mask = nullptr;  // per boundary point: the colours of the elements touching it
  std::vector<int> rp_off, rp_cnt;  // per tile (host)
  // batched tiles of four elements (variant 7): elements in colour order,
  // tile-interior index of each element point, interior points and their
  // contributions, the points tiles share
  int nbt = 0, nbp = 0;
  int *bt_tel = nullptr, *bt_loc = nullptr, *bt_pt = nullptr, *bt_ctr = nullptr, *bt_bpts = nullptr;
};

}  // namespace

// Device state of the adjoint (allocated on first use).
struct AdjointState {
  int nstep = 0, interval = 0, ncheck = 0;
  size_t nvals = 0, nloc = 0, stride = 0, nglob = 0;
  float *ckpt = nullptr;                        // [ncheck][u, v, a][nvals + 4]
  // nbuf >= 2 segment buffers (as many as the memory budget holds, at most
  // one per segment): the checkpointed forward run records its last nbuf
  // segments on the way, so that only the earlier ones are recomputed, each
  // while the reverse sweep of a later one runs (streams: the handle's and
  // rstream)
  int nbuf = 0;
  size_t budget = 0;                            // bytes for segment buffers; 0: the default
  float *seg_u = nullptr, *seg_a = nullptr;     // [nbuf][interval][stride]
  float *seg_v = nullptr;                       // [nbuf][interval][vstride]: v~ at the Stacey points
  cudaStream_t rstream = nullptr;
  std::vector<cudaEvent_t> ev_rec, ev_rev;      // per buffer
  int rec_from = -1;                            // segments rec_from.. are held from the forward run (-1: none)
  size_t vstride = 0;
  float *lu = nullptr, *lv = nullptr, *mu = nullptr;
  float *r = nullptr;                           // [nloc][2]
  // gradient sums: [nloc][kappa, mu], [nglob] rho-term per global point,
  // then (from a 16-byte boundary) [nlb][4] Stacey impedance terms
  float *sum = nullptr, *comp = nullptr, *seg = nullptr;
  size_t off_lb = 0;
  int nlb = 0;                                  // element-local Stacey points
  int *lb_g = nullptr, *lb_j = nullptr;
  float *lb_geo = nullptr;                      // [nlb][nx, nz, j1, wq]
  std::vector<size_t> lb_k;                     // index into the boundary arrays
  std::vector<size_t> lb_pm;                    // mesh-order element point
  float *gtab = nullptr;                        // [nstep][nrec][2] (the reverse graphs hold this pointer)
  size_t gtab_cap = 0;
  float *h_stage = nullptr;                     // pinned host staging: gtab rows, then the sums
  size_t h_stage_cap = 0;
  int *ad_head = nullptr, *ad_next = nullptr;
  int *st_pt = nullptr;
  float *st_c = nullptr;
  int nst = 0;
  sfg::dev::SegRecord *d_rec = nullptr;
  cudaGraphExec_t graph_r1 = nullptr, graph_re = nullptr;  // recording steps
  cudaGraphExec_t graph_rseg = nullptr;         // interval - 1 recording steps
  std::vector<cudaGraphExec_t> graph_rev;       // reverse sweep of a full segment, per buffer
  int *d_k0 = nullptr;                          // first step of the segment in reverse
  bool forward_done = false;
  int epb = 0;                                  // elements per block of k_adj_elem (timed once)
  // acoustic: per source element point, sum of mu f over the steps
  int nsrc_t = 0;
  int *src_ce = nullptr;
  size_t off_src() const { return off_lb + 4 * size_t(nlb); }
  size_t nsum() const { return off_src() + size_t(sfg::NPTS) * nsrc_t; }
  // acoustic pressure seismograms as adjoint sources: CSR over the points the
  // receivers touch (point, then receiver and Lagrange weight per entry)
  bool pressure = false;
  int nps = 0;
  int *ps_pt = nullptr, *ps_start = nullptr, *ps_rec = nullptr;
  float *ps_h = nullptr;
  // coupled sweep: acoustic sources' STF columns; transposed coupling of this
  // medium's interface points (partner, partner-side normal)
  int *src_id = nullptr;
  std::vector<int> src_list, src_ce_h;
  int *cp_other = nullptr;
  float *cp_nx = nullptr, *cp_nz = nullptr;
};

struct sfg_handle {
  // adjoint: adj holds the sweep's control and the (first) medium's state;
  // adj2 the acoustic medium's state in a coupled model (adj_coupled)
  AdjointState adj, adj2;
  bool adj_coupled = false;
  // update_args: record u~ and a' of each step (adjoint); 2 = recompute
  // (seismograms are those of the forward run and are not computed again)
  int recording = 0;
  // coupled P-SV model whose interface points pair one to one: the two
  // owner-computes point updates can run as one launch
  bool fuse_ok = false;
  sfg::Mesh2D mesh;
  sfg::Assembly2D asmb;
  sfg_options opt{};
  std::vector<sfg::Source2D> sources;
  std::vector<double> rec_x, rec_z;
  bool have_sources = false, have_receivers = false, initialized = false;
  std::vector<float> ext_stf;  // optional external STF table
  int ext_stf_nsrc = 0;
  DevMem mem;
  DevMedium el, ac;
  int *d_src_next = nullptr, *d_src_shot = nullptr;
  float *d_src_arr = nullptr, *d_stf = nullptr;
  float *d_src_arr2 = nullptr;     // poroelastic fluid rows of the source arrays
  int *d_rec_elem = nullptr;
  float *d_rec_h = nullptr, *d_seis = nullptr;
  int *d_step = nullptr, *d_flag = nullptr;
  int host_step = 0;
  int epb = 16;
  // 1 colour passes, 2 persistent colour passes, 3 owner-computes,
  // 4 owner-computes with bulk-copy staged element arrays
  int variant = 1;
  int sm_count = 148;
  int resident[2][3] = {{0}};  // persistent: resident blocks per SM [EK][E index]
  int resident_tma[2][3] = {{0}};  // bulk-copy element kernel: resident blocks per SM
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // receivers that overlap the element kernel
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaGraphExec_t graph_k = nullptr, graph_1 = nullptr, graph_e = nullptr;
  int graph_steps = 0;
  // true when u, v hold the end-of-step state of the reference (after the
  // corrector); false inside a run, where the next predictor is already applied
  bool state_final = true;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // fused tile kernel (variant 5): eligible model, side buffer of the
  // receiver points, receiver -> side slot [nrec][25], shared-memory layout
  bool tile_ok = false;
  float *d_side = nullptr;
  int *d_rslot = nullptr;
  sfg::dev::TileArgs tile_layout{};
  sfg::dev::TileBArgs tileb_layout{};   // batched shots
  int tile_smem = 0, tile_blocks_per_sm = 0;
  bool b4r_attr = false;                 // shared-memory attribute of the row-form batched kernel set
  bool btile_ok = false;                 // batched tiles of four elements (variant 7) built
  void *flush_buf = nullptr;
  size_t flush_bytes = 0;
  // sfg_step_io: one graph per step that reads the source row from and
  // writes the seismogram row to mapped pinned host memory
  // ([flag, pad x3][source row][seismogram rows of the shots])
  void *io_host = nullptr;
  void *io_dev = nullptr;
  cudaGraphExec_t graph_io = nullptr;
  std::string err;
  sfg::dev::Quad quad{};

  ~sfg_handle() {
    for (const AdjointState *A : {&adj, &adj2})
      for (void *p : {(void *)A->ckpt, (void *)A->seg_u, (void *)A->seg_a, (void *)A->lu, (void *)A->lv,
                      (void *)A->mu, (void *)A->r, (void *)A->sum, (void *)A->comp, (void *)A->seg,
                      (void *)A->ad_head, (void *)A->ad_next, (void *)A->st_pt, (void *)A->st_c,
                      (void *)A->d_rec, (void *)A->seg_v, (void *)A->lb_g, (void *)A->lb_j, (void *)A->lb_geo,
                      (void *)A->src_ce, (void *)A->ps_pt, (void *)A->ps_start, (void *)A->ps_rec,
                      (void *)A->ps_h, (void *)A->src_id, (void *)A->cp_other, (void *)A->cp_nx,
                      (void *)A->cp_nz})
        if (p) cudaFree(p);
    if (adj.gtab) cudaFree(adj.gtab);
    if (adj.h_stage) cudaFreeHost(adj.h_stage);
    if (io_host) cudaFreeHost(io_host);
    if (graph_io) cudaGraphExecDestroy(graph_io);
    if (adj.graph_r1) cudaGraphExecDestroy(adj.graph_r1);
    if (adj.graph_rseg) cudaGraphExecDestroy(adj.graph_rseg);
    for (auto &g : adj.graph_rev)
      if (g) cudaGraphExecDestroy(g);
    if (adj.d_k0) cudaFree(adj.d_k0);
    for (auto *ev : {&adj.ev_rec, &adj.ev_rev})
      for (cudaEvent_t e : *ev)
        if (e) cudaEventDestroy(e);
    if (adj.rstream) cudaStreamDestroy(adj.rstream);
    if (adj.graph_re) cudaGraphExecDestroy(adj.graph_re);
    if (graph_k) cudaGraphExecDestroy(graph_k);
    if (graph_1) cudaGraphExecDestroy(graph_1);
    if (graph_e) cudaGraphExecDestroy(graph_e);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
    if (flush_buf) cudaFree(flush_buf);
    mem.free_all();
  }
};

namespace {

template <typename F>
int guarded(sfg_handle *h, F &&fn) {
  if (!h) return SFG_ERR_ARG;
  try {
    return fn();
  } catch (const CudaError &ex) {
    h->err = ex.what();
    return SFG_ERR_CUDA;
  } catch (const std::exception &ex) {
    h->err = ex.what();
    return SFG_ERR_ARG;
  }
}

void upload_medium(sfg_handle *h, const sfg::MediumData &M, DevMedium &D) {
  DevMem &m = h->mem;
  D.nspec = M.nspec;
  D.nglob = M.nglob;
  D.ncomp = M.ncomp;
  D.color_start = M.color_start;
  if (M.nspec == 0) return;
  // element arrays padded with zeros to whole tiles of 32 elements (the
  // bulk-copy element kernel always moves whole tiles)
  const size_t npad = size_t((M.nspec + 31) / 32 * 32) * sfg::NPTS;
  auto padded = [&](const auto &v) {
    auto w = v;
    w.resize(std::max(npad, v.size()), 0);
    return m.upload(w);
  };
  D.ibool = padded(M.ibool);
  D.xix = padded(M.xix); D.xiz = padded(M.xiz); D.gax = padded(M.gax);
  D.gaz = padded(M.gaz); D.jac = padded(M.jac);
  D.prop0 = padded(M.prop0); D.prop1 = padded(M.prop1);
  D.aniso = M.aniso;
  if (M.aniso) {
    D.prop2 = padded(M.prop2); D.prop3 = padded(M.prop3);
    D.prop4 = padded(M.prop4); D.prop5 = padded(M.prop5);
  }
  if (M.cosserat) {            // nu and mu_c + nu_c
    if (M.prop2.size() != M.prop0.size() || M.prop3.size() != M.prop0.size())
      throw std::runtime_error("Cosserat medium without its nu / mu_c + nu_c words");
    D.prop2 = padded(M.prop2); D.prop3 = padded(M.prop3);
  }
  D.poro = M.poro;
  if (M.poro) {                // C, M, phi / tort, rho_f / rho_bar, damping words
    for (const auto *v : {&M.prop2, &M.prop3, &M.prop4, &M.prop5, &M.prop6, &M.prop7, &M.prop8})
      if (v->size() != M.prop0.size()) throw std::runtime_error("poroelastic medium without its material words");
    D.prop2 = padded(M.prop2); D.prop3 = padded(M.prop3); D.prop4 = padded(M.prop4);
    D.prop5 = padded(M.prop5); D.prop6 = padded(M.prop6); D.prop7 = padded(M.prop7);
    D.prop8 = padded(M.prop8);
  }
  D.bc_slot = m.upload(M.bc_slot);
  D.bc_w = m.upload(M.bc_w); D.bc_nx = m.upload(M.bc_nx); D.bc_nz = m.upload(M.bc_nz);
  D.bc_j1 = m.upload(M.bc_j1); D.bc_imp0 = m.upload(M.bc_imp0); D.bc_imp1 = m.upload(M.bc_imp1);
  D.bc_keep = m.upload(M.bc_keep);
  D.bc_imp2 = m.upload(M.bc_imp2);
  D.niface = M.niface;
  D.cp_nx = m.upload(M.cp_nx); D.cp_nz = m.upload(M.cp_nz); D.cp_other = m.upload(M.cp_other);
  D.cp_start = M.cp_start.empty() ? nullptr : m.upload(M.cp_start);
  {
    // padded: the tile kernel's bulk copies round ranges up to 16 bytes
    std::vector<float> mp(M.minv);
    if (!mp.empty()) mp.resize(mp.size() + 4, 0.f);
    D.minv = m.upload(mp);
  }
  D.S = h->asmb.nshots;
  const size_t n = D.values();
  // pad by 4 floats so float4 streaming never runs past an allocation
  D.u = m.zeros<float>(n + 4);
  D.v = m.zeros<float>(n + 4);
  D.accum = m.zeros<float>(n + 4);
  D.a = m.zeros<float>(n + 4);
  D.inv_start = m.upload(M.inv_start);
  {
    std::vector<int> slot(M.inv_idx.size());
    for (size_t k = 0; k < M.inv_idx.size(); ++k) slot[size_t(M.inv_idx[k])] = int(k);
    D.slot = m.upload(slot);
  }
  D.r = m.zeros<float>(size_t(M.nspec) * sfg::NPTS * M.ncomp * D.S + 4);
}

sfg::dev::MedArgs med_args(const DevMedium &D) {
  sfg::dev::MedArgs A{};
  A.ibool = D.ibool;
  A.xix = D.xix; A.xiz = D.xiz; A.gax = D.gax; A.gaz = D.gaz; A.jac = D.jac;
  A.prop0 = D.prop0; A.prop1 = D.prop1;
  A.prop2 = D.prop2; A.prop3 = D.prop3; A.prop4 = D.prop4; A.prop5 = D.prop5;
  A.prop6 = D.prop6; A.prop7 = D.prop7; A.prop8 = D.prop8;
  A.bc_slot = D.bc_slot; A.bc_w = D.bc_w; A.bc_nx = D.bc_nx; A.bc_nz = D.bc_nz;
  A.bc_j1 = D.bc_j1; A.bc_imp0 = D.bc_imp0; A.bc_imp1 = D.bc_imp1; A.bc_keep = D.bc_keep;
  A.bc_imp2 = D.bc_imp2;
  A.src_head = D.src_head;
  A.u = D.u; A.v = D.v; A.accum = D.accum; A.r = D.r; A.slot = D.slot;
  return A;
}

int ncolors(const DevMedium &D) { return D.nspec ? int(D.color_start.size()) - 1 : 0; }

template <int E, int EK>
void launch_stiffness_E(sfg_handle *h, const DevMedium &el, const DevMedium &ac, const int *step,
                        cudaStream_t s, int variant) {
  // the anisotropic and Cosserat stresses exist in the colour-pass and
  // owner-computes kernels
  if (EK >= 2 && (variant == 2 || variant == 4)) variant = variant == 2 ? 1 : 3;
  if ((EK == 2 || EK == 3 || EK == 4) && (!el.prop2 || !el.prop3))
    throw std::runtime_error("element kernel: material words of the medium missing on the device");
  if (EK == 4 && (!el.prop4 || !el.prop5 || !el.prop6 || !el.prop7 || !el.prop8 || !h->d_src_arr2))
    throw std::runtime_error("element kernel: poroelastic words or source rows missing on the device");
  sfg::dev::StiffArgs S{};
  S.el = med_args(el);
  S.ac = med_args(ac);
  S.src_next = h->d_src_next;
  S.src_arr = h->d_src_arr;
  S.src_arr2 = h->d_src_arr2;
  S.stf = h->d_stf;
  S.nsrc = h->asmb.nsrc;
  S.nstep = h->asmb.nstep;
  S.step = step;
  S.quad = h->quad;
  if (variant == 3) {
    // owner-computes: one launch over every element of both media
    S.el.e0 = 0; S.el.e1 = el.nspec; S.el.nblocks = (el.nspec + E - 1) / E;
    S.ac.e0 = 0; S.ac.e1 = ac.nspec; S.ac.nblocks = (ac.nspec + E - 1) / E;
    const int grid = S.el.nblocks + S.ac.nblocks;
    if (grid > 0) sfg::dev::k_stiffness<E, EK, true><<<grid, sfg::dev::NP * E, 0, s>>>(S);
    return;
  }
  if (variant == 4) {
    // owner-computes, persistent, element arrays staged by bulk copies
    constexpr int ST = 3;
    const int smem = sfg::dev::TmaLayout<E>::bytes(ST);
    auto kern = sfg::dev::k_stiffness_tma<E, EK, ST>;
    const int ei = E == 8 ? 0 : (E == 16 ? 1 : 2);
    int &nb = h->resident_tma[EK][ei];
    if (nb == 0) {
      SFG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      SFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, sfg::dev::NP * E, smem));
      nb = std::max(nb, 1);
    }
    S.el.e0 = 0; S.el.e1 = el.nspec;
    S.ac.e0 = 0; S.ac.e1 = ac.nspec;
    const int nt_el = (el.nspec + E - 1) / E, nt_ac = (ac.nspec + E - 1) / E;
    const int grid = std::min(nt_el + nt_ac, nb * h->sm_count);
    if (grid > 0) kern<<<grid, sfg::dev::NP * E, smem, s>>>(S, nt_el, nt_ac, h->d_flag);
    return;
  }
  const bool persistent = variant == 2;
  int capacity = 0;
  if (persistent) {
    const int ei = E == 8 ? 0 : (E == 16 ? 1 : 2);
    int &nb = h->resident[EK][ei];
    if (nb == 0) {
      SFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &nb, sfg::dev::k_stiffness_persistent<E, EK>, sfg::dev::NP * E, 0));
      nb = std::max(nb, 1);
    }
    capacity = nb * h->sm_count;
  }
  const int nc = std::max(ncolors(el), ncolors(ac));
  for (int c = 0; c < nc; ++c) {
    int chunks[2] = {0, 0};
    sfg::dev::MedArgs *M[2] = {&S.el, &S.ac};
    const DevMedium *D[2] = {&el, &ac};
    for (int k = 0; k < 2; ++k) {
      M[k]->e0 = M[k]->e1 = 0;
      if (c < ncolors(*D[k])) {
        M[k]->e0 = D[k]->color_start[c];
        M[k]->e1 = D[k]->color_start[c + 1];
        chunks[k] = (M[k]->e1 - M[k]->e0 + E - 1) / E;
      }
      M[k]->nblocks = chunks[k];
    }
    if (chunks[0] + chunks[1] == 0) continue;
    if (persistent && chunks[0] + chunks[1] > capacity) {
      // split the resident blocks between the media in proportion to their work
      int bel = chunks[0] == 0 ? 0
                : std::max(1, int(double(capacity) * chunks[0] / (chunks[0] + chunks[1]) + 0.5));
      if (chunks[1] > 0) bel = std::min(bel, capacity - 1);
      S.el.nblocks = std::min(bel, chunks[0]);
      S.ac.nblocks = std::min(capacity - S.el.nblocks, chunks[1]);
    }
    const int grid = S.el.nblocks + S.ac.nblocks;
    if (persistent)
      sfg::dev::k_stiffness_persistent<E, EK><<<grid, sfg::dev::NP * E, 0, s>>>(S);
    else
      sfg::dev::k_stiffness<E, EK, false><<<grid, sfg::dev::NP * E, 0, s>>>(S);
  }
}

template <int E>
void launch_stiffness_W(sfg_handle *h, const DevMedium &el, const DevMedium &ac, const int *step,
                        cudaStream_t s, int variant) {
  if (el.ncomp == 1) launch_stiffness_E<E, 1>(h, el, ac, step, s, variant);
  else if (el.aniso) launch_stiffness_E<E, 2>(h, el, ac, step, s, variant);
  else if (el.ncomp == 3) launch_stiffness_E<E, 3>(h, el, ac, step, s, variant);
  else if (el.ncomp == 4) launch_stiffness_E<E, 4>(h, el, ac, step, s, variant);
  else launch_stiffness_E<E, 0>(h, el, ac, step, s, variant);
}

sfg::dev::BatchArgs batch_args(sfg_handle *h, const DevMedium &el, const int *step) {
  sfg::dev::BatchArgs B{};
  B.ibool = el.ibool;
  B.xix = el.xix; B.xiz = el.xiz; B.gax = el.gax; B.gaz = el.gaz; B.jac = el.jac;
  B.prop0 = el.prop0; B.prop1 = el.prop1;
  B.bc_slot = el.bc_slot; B.bc_w = el.bc_w; B.bc_nx = el.bc_nx; B.bc_nz = el.bc_nz;
  B.bc_j1 = el.bc_j1; B.bc_imp0 = el.bc_imp0; B.bc_imp1 = el.bc_imp1;
  B.src_head = el.src_head; B.src_next = h->d_src_next; B.src_shot = h->d_src_shot;
  B.src_arr = h->d_src_arr; B.stf = h->d_stf;
  B.nsrc = h->asmb.nsrc; B.nstep = h->asmb.nstep;
  B.step = step;
  B.u = el.u; B.v = el.v; B.accum = el.accum; B.r = el.r; B.slot = el.slot;
  B.S = el.S;
  B.nspec_b = el.nspec;
  return B;
}

void launch_stiffness_batched(sfg_handle *h, const DevMedium &el, const int *step, cudaStream_t s,
                              int variant) {
  sfg::dev::BatchArgs B{};
  B.ibool = el.ibool;
  B.xix = el.xix; B.xiz = el.xiz; B.gax = el.gax; B.gaz = el.gaz; B.jac = el.jac;
  B.prop0 = el.prop0; B.prop1 = el.prop1;
  B.bc_slot = el.bc_slot; B.bc_w = el.bc_w; B.bc_nx = el.bc_nx; B.bc_nz = el.bc_nz;
  B.bc_j1 = el.bc_j1; B.bc_imp0 = el.bc_imp0; B.bc_imp1 = el.bc_imp1;
  B.src_head = el.src_head; B.src_next = h->d_src_next; B.src_shot = h->d_src_shot;
  B.src_arr = h->d_src_arr; B.stf = h->d_stf;
  B.nsrc = h->asmb.nsrc; B.nstep = h->asmb.nstep;
  B.step = step;
  B.u = el.u; B.v = el.v; B.accum = el.accum; B.r = el.r; B.slot = el.slot;
  B.S = el.S;
  // quad-shot kernels when the shots come in fours
  const bool quad = el.S % 4 == 0;
  const int T = std::min(8, el.S / 4);
  const int tiles = quad ? (el.S + 4 * T - 1) / (4 * T) : (el.S + 31) / 32;
  const int threads = quad ? sfg::dev::NP * T : sfg::dev::NP * 32;
  auto launch = [&](int e0, int n, bool local) {
    B.e0 = e0;
    const dim3 grid(n, tiles);
    if (quad) {
      if (el.ncomp == 2) {
        if (local) sfg::dev::k_stiffness_batched4<2, true><<<grid, threads, 0, s>>>(B, T);
        else sfg::dev::k_stiffness_batched4<2, false><<<grid, threads, 0, s>>>(B, T);
      } else {
        if (local) sfg::dev::k_stiffness_batched4<1, true><<<grid, threads, 0, s>>>(B, T);
        else sfg::dev::k_stiffness_batched4<1, false><<<grid, threads, 0, s>>>(B, T);
      }
    } else if (el.ncomp == 2) {
      if (local) sfg::dev::k_stiffness_batched<2, true><<<grid, threads, 0, s>>>(B);
      else sfg::dev::k_stiffness_batched<2, false><<<grid, threads, 0, s>>>(B);
    } else {
      if (local) sfg::dev::k_stiffness_batched<1, true><<<grid, threads, 0, s>>>(B);
      else sfg::dev::k_stiffness_batched<1, false><<<grid, threads, 0, s>>>(B);
    }
  };
  if (variant == 4 && quad) {
    // owner-computes with the row-form element kernel (4 elements per block)
    constexpr int EB = 4;
    B.nspec_b = el.nspec;
    const int smem = EB * el.ncomp * 2 * sfg::dev::NP * T * int(sizeof(float4));
    if (!h->b4r_attr) {
      SFG_CUDA(cudaFuncSetAttribute(sfg::dev::k_stiffness_batched4r<2, EB>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, EB * 2 * 2 * 25 * 8 * 16));
      SFG_CUDA(cudaFuncSetAttribute(sfg::dev::k_stiffness_batched4r<1, EB>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, EB * 1 * 2 * 25 * 8 * 16));
      h->b4r_attr = true;
    }
    const dim3 grid((el.nspec + EB - 1) / EB, tiles);
    if (el.ncomp == 2) sfg::dev::k_stiffness_batched4r<2, EB><<<grid, EB * sfg::dev::NG * T, smem, s>>>(B, T);
    else sfg::dev::k_stiffness_batched4r<1, EB><<<grid, EB * sfg::dev::NG * T, smem, s>>>(B, T);
    return;
  }
  if (variant >= 3) {
    launch(0, el.nspec, true);
    return;
  }
  for (int c = 0; c < ncolors(el); ++c) {
    const int n = el.color_start[c + 1] - el.color_start[c];
    if (n > 0) launch(el.color_start[c], n, false);
  }
}

// The row-form kernel covers isotropic P-SV and acoustic media.
bool row_ok(const DevMedium &el) { return el.nspec == 0 || (el.ncomp == 2 && !el.aniso); }

template <int E>
void launch_stiffness_row(sfg_handle *h, const DevMedium &el, const DevMedium &ac, const int *step,
                          cudaStream_t s) {
  sfg::dev::StiffArgs S{};
  S.el = med_args(el);
  S.ac = med_args(ac);
  S.src_next = h->d_src_next;
  S.src_arr = h->d_src_arr;
  S.src_arr2 = h->d_src_arr2;
  S.stf = h->d_stf;
  S.nsrc = h->asmb.nsrc;
  S.nstep = h->asmb.nstep;
  S.step = step;
  S.quad = h->quad;
  S.el.e0 = 0; S.el.e1 = el.nspec; S.el.nblocks = (el.nspec + E - 1) / E;
  S.ac.e0 = 0; S.ac.e1 = ac.nspec; S.ac.nblocks = (ac.nspec + E - 1) / E;
  const int grid = S.el.nblocks + S.ac.nblocks;
  if (grid > 0) sfg::dev::k_stiffness_row<E><<<grid, sfg::dev::NG * E, 0, s>>>(S);
}

void launch_stiffness(sfg_handle *h, const DevMedium &el, const DevMedium &ac, const int *step,
                      cudaStream_t s, int variant) {
  if (el.S > 1) {
    launch_stiffness_batched(h, el, step, s, variant);
    return;
  }
  if (variant == 6) {
    // owner-computes with the row-form element kernel (16 or 32 elements per block)
    if (row_ok(el)) {
      if (h->epb == 16) launch_stiffness_row<16>(h, el, ac, step, s);
      else launch_stiffness_row<32>(h, el, ac, step, s);
      return;
    }
    variant = 3;
  }
  switch (h->epb) {
    case 8: launch_stiffness_W<8>(h, el, ac, step, s, variant); break;
    case 32: launch_stiffness_W<32>(h, el, ac, step, s, variant); break;
    default: launch_stiffness_W<16>(h, el, ac, step, s, variant); break;
  }
}

void launch_stiffness(sfg_handle *h, cudaStream_t s) {
  // the fused tile variant falls back to owner-computes for recorded steps
  launch_stiffness(h, h->el, h->ac, h->d_step, s, h->variant == 5 ? 3 : h->variant);
}

sfg::dev::UpdateArgs update_args(sfg_handle *h, const DevMedium &D, const DevMedium &O, int medium,
                                 bool predict, bool advance) {
  sfg::dev::UpdateArgs U{};
  U.u = D.u; U.v = D.v; U.accum = D.accum; U.minv = D.minv;
  // acoustic chi_dd feeds the elastic coupling term; the last step of a run
  // keeps the acceleration for the predictor that resumes the next run
  U.a_store = (medium == SFG_MEDIUM_ACOUSTIC || !predict || h->opt.store_acceleration) ? D.a : nullptr;
  U.n = int(D.values());
  U.ncomp = D.ncomp;
  U.niface = D.niface;
  U.cp_nx = D.cp_nx; U.cp_nz = D.cp_nz; U.cp_other = D.cp_other; U.cp_start = D.cp_start;
  U.other = medium == SFG_MEDIUM_ELASTIC ? O.a : O.u;
  const float dt = float(h->asmb.dt);
  U.dt = dt;
  U.dt2 = dt / 2.0f;
  U.dtsq2 = dt * dt / 2.0f;
  U.predict = predict ? 1 : 0;
  if (h->variant >= 3) {
    U.inv_start = D.inv_start;
    U.r = D.r;
  }
  U.flag = h->d_flag;
  U.step = h->d_step;
  U.advance = advance && !h->recording ? 1 : 0;
  if (h->recording) U.rec = (h->adj_coupled && medium == SFG_MEDIUM_ACOUSTIC) ? h->adj2.d_rec : h->adj.d_rec;
  return U;
}

int grid_for(int n) {
  const int threads = 256;
  int blocks = (n + threads - 1) / threads;
  return std::max(1, std::min(blocks, 148 * 8));
}

// Reads a buffer (float4 by float4) so that the L2 afterwards holds its clean
// lines; the sink is written only on a value the zero-filled buffer never has.
__global__ void __launch_bounds__(256) k_read_flush(const float4 *__restrict__ b, size_t n4, float *sink) {
  float acc = 0.f;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n4; i += size_t(gridDim.x) * blockDim.x) {
    const float4 v = b[i];
    acc += v.x + v.y + v.z + v.w;
  }
  if (acc == 1234.5f) *sink = acc;
}

// sfg_step_io: the step's source row from mapped host memory into the table
// (when the host set the flag), and after the step its seismogram rows back.
__global__ void k_io_in(const int *__restrict__ io, float *stf, const int *step, int nsrc, int nstep) {
  const int st = *step;
  if (io[0] == 0 || st >= nstep) return;
  const float *row = reinterpret_cast<const float *>(io + 4);
  for (int s = threadIdx.x; s < nsrc; s += blockDim.x) stf[size_t(st) * nsrc + s] = row[s];
}
__global__ void k_io_out(const float *__restrict__ seis, float *out, const int *step, int nsb, int nsig, int nshots,
                         int rowlen) {
  const int st = *step - 1;    // the step just taken
  if (st < 0 || st % nsb != 0 || st / nsb >= nsig) return;
  const int isig = st / nsb;
  const int n = nshots * rowlen;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int sh = i / rowlen, k = i - sh * rowlen;
    out[i] = seis[(size_t(sh) * nsig + isig) * rowlen + k];
  }
}

// L2 flush before a timed launch or step: a device write of `bytes`, then a
// read of a second buffer of `bytes`, so the cache holds neither the model's
// data nor dirty lines whose write-back the timed work would pay for.
void flush_l2(sfg_handle *h, size_t bytes, int pattern) {
  if (bytes > h->flush_bytes) {
    if (h->flush_buf) cudaFree(h->flush_buf);
    h->flush_buf = nullptr;
    h->flush_bytes = 0;
    SFG_CUDA(cudaMalloc(&h->flush_buf, 2 * bytes + 16));
    SFG_CUDA(cudaMemset(h->flush_buf, 0, 2 * bytes + 16));
    h->flush_bytes = bytes;
  }
  char *base = static_cast<char *>(h->flush_buf);
  SFG_CUDA(cudaMemsetAsync(base, pattern & 0xff, bytes, h->stream));
  k_read_flush<<<148 * 8, 256, 0, h->stream>>>(reinterpret_cast<const float4 *>(base + h->flush_bytes),
                                                bytes / 16, reinterpret_cast<float *>(base + 2 * h->flush_bytes));
}

sfg::dev::RecArgs rec_args(sfg_handle *h, int medium) {
  DevMedium &D = medium == SFG_MEDIUM_ELASTIC ? h->el : h->ac;
  sfg::dev::RecArgs R{};
  R.nrec = D.nrec;
  R.rec_list = D.rec_list;
  R.rec_elem = h->d_rec_elem;
  R.rec_h = h->d_rec_h;
  R.ibool = D.ibool;
  R.xix = D.xix; R.xiz = D.xiz; R.gax = D.gax; R.gaz = D.gaz; R.prop0 = D.prop0;
  R.prop1 = D.prop1;
  R.prop2 = D.prop2; R.prop3 = D.prop3;
  R.u = D.u; R.v = D.v; R.accum = D.accum; R.minv = D.minv;
  R.cpl = update_args(h, D, medium == SFG_MEDIUM_ELASTIC ? h->ac : h->el, medium, true, false);
  R.ncomp = D.ncomp;
  R.acoustic = medium == SFG_MEDIUM_ACOUSTIC;
  R.ntypes = h->asmb.ntypes;
  for (int t = 0; t < R.ntypes && t < 8; ++t) R.types[t] = h->asmb.types[t];
  R.nsb = h->asmb.nsb;
  R.nsig = h->asmb.nsig;
  R.nrec_total = h->asmb.nrec;
  R.dt2 = float(h->asmb.dt) / 2.0f;
  R.step = h->d_step;
  R.seis = h->d_seis;
  R.quad = h->quad;
  R.a = D.a;
  R.final_fields = 0;
  R.isig_fixed = -1;
  return R;
}

void launch_receivers(sfg_handle *h, int medium, cudaStream_t s) {
  DevMedium &D = medium == SFG_MEDIUM_ELASTIC ? h->el : h->ac;
  if (D.nrec == 0) return;
  const sfg::dev::RecArgs R = rec_args(h, medium);
  if (D.S > 1) sfg::dev::k_receivers_batched<<<D.nrec, 32, 0, s>>>(R, D.S);
  else sfg::dev::k_receivers<<<D.nrec, 32, 0, s>>>(R);
}

void launch_update(sfg_handle *h, int medium, bool predict, bool advance, cudaStream_t s) {
  const DevMedium &D = medium == SFG_MEDIUM_ELASTIC ? h->el : h->ac;
  const DevMedium &O = medium == SFG_MEDIUM_ELASTIC ? h->ac : h->el;
  sfg::dev::UpdateArgs U = update_args(h, D, O, medium, predict, advance);
  if (h->variant >= 3) {
    if (D.S > 1 && D.S % 4 == 0)
      sfg::dev::k_update_batched4_gather<<<grid_for(U.n / 4), 256, 0, s>>>(U, D.S, D.ncomp);
    else if (D.S > 1) sfg::dev::k_update_batched_gather<<<grid_for(U.n), 256, 0, s>>>(U, D.S, D.ncomp);
    else if (D.ncomp == 2) sfg::dev::k_update_gather<2><<<grid_for(U.n / 2), 256, 0, s>>>(U);
    else if (D.ncomp == 3) sfg::dev::k_update_gather<3><<<grid_for(U.n / 3), 256, 0, s>>>(U);
    else if (D.ncomp == 4) sfg::dev::k_update_gather<4><<<grid_for(U.n / 4), 256, 0, s>>>(U);
    else sfg::dev::k_update_gather<1><<<grid_for(U.n), 256, 0, s>>>(U);
    return;
  }
  if (D.S > 1 && D.S % 4 == 0) sfg::dev::k_update_batched4<<<grid_for(U.n / 4), 256, 0, s>>>(U, D.S);
  else if (D.S > 1) sfg::dev::k_update_batched<<<grid_for(U.n), 256, 0, s>>>(U, D.S);
  else sfg::dev::k_update<<<grid_for(U.n / 4), 256, 0, s>>>(U);
}

// Both media's point updates in one launch (owner-computes, interface points
// paired one to one).
void launch_update_coupled(sfg_handle *h, bool predict, cudaStream_t s) {
  sfg::dev::UpdateArgs E = update_args(h, h->el, h->ac, SFG_MEDIUM_ELASTIC, predict, true);
  sfg::dev::UpdateArgs A = update_args(h, h->ac, h->el, SFG_MEDIUM_ACOUSTIC, predict, false);
  const int n = E.n / 2 + A.n - A.niface;
  sfg::dev::k_update_coupled<<<grid_for(n), 256, 0, s>>>(E, A);
}

// Whether this step may use launch_update_coupled: owner-computes, one shot,
// and no elastic receiver that reads this step's acoustic acceleration (the
// elastic receivers then run before the update).
bool fused_update(const sfg_handle *h);

void launch_predict_medium(sfg_handle *h, const DevMedium &D, cudaStream_t s) {
  if (!D.nspec) return;
  const float dt = float(h->asmb.dt);
  const int n = int(D.values());
  sfg::dev::k_predict<<<grid_for(n), 256, 0, s>>>(D.u, D.v, D.a, n, dt, dt / 2.0f, dt * dt / 2.0f);
}

void launch_predict(sfg_handle *h, cudaStream_t s) {
  launch_predict_medium(h, h->ac, s);
  launch_predict_medium(h, h->el, s);
}

// One time step in the reference's medium order (time_marching.tpp:33-83):
// the element launches of both media, then the acoustic update (its coupling
// reads the predicted elastic displacement), then the elastic update (its
// coupling reads the new acoustic chi_dd).  predict = fuse the next step's
// predictor into the updates.
// Seismograms of a medium that read only the step's displacement (elastic
// displacement and pressure, acoustic displacement) can be taken while the
// element kernel runs.
bool receivers_early(const sfg_handle *h, int medium) {
  for (int t = 0; t < h->asmb.ntypes; ++t) {
    const int k = h->asmb.types[t];
    // types that read the displacement only (Cosserat rotation, intrinsic
    // rotation and curl too) may run before the update
    const bool disp = k == SFG_SEIS_DISPLACEMENT || k == SFG_SEIS_ROTATION ||
                      k == SFG_SEIS_INTRINSIC_ROTATION || k == SFG_SEIS_CURL;
    if (!(disp || (k == SFG_SEIS_PRESSURE && medium == SFG_MEDIUM_ELASTIC))) return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Fused tile kernel (variant 5).

// Whether the model can run the fused tile kernel: one shot, isotropic P-SV,
// SH or acoustic media, conforming coupling whose interface points pair one
// to one (P-SV), seismograms of displacement, velocity, acceleration or
// pressure; or S shots (S a multiple of 4) on one isotropic elastic medium
// with displacement, velocity or acceleration seismograms.
static_assert(sfg::TILE_E == sfg::dev::TILE_E, "host and device tile sizes differ");

bool compute_tile_ok(const sfg_handle *h) {
  const sfg::Assembly2D &a = h->asmb;
  const sfg::MediumData &E = a.el, &C = a.ac;
  if (a.nshots != 1) {
    if (a.nshots % 4 != 0 || C.nspec || !E.nspec) return false;
    for (int t : a.types)
      if (t > SFG_SEIS_ACCELERATION) return false;
  }
  if (E.nspec && (E.aniso || E.cosserat || E.poro || E.ncomp > 2)) return false;
  if (!E.cp_start.empty() || !C.cp_start.empty()) return false;
  if (E.nspec && C.nspec && !(h->fuse_ok && E.ncomp == 2)) return false;
  for (int t : a.types)
    if (t > SFG_SEIS_PRESSURE) return false;
  for (const sfg::MediumData *M : {&E, &C})
    if (M->nspec && int(M->color_start.size()) - 1 > sfg::dev::TILE_MAX_COLORS) return false;
  return E.ntiles + C.ntiles > 0;
}

int tile_nf(const sfg::MediumData &M, int medium) { return medium == SFG_MEDIUM_ACOUSTIC || M.ncomp == 0 ? 6 : 7; }

// Records of the fused tile kernel: header {ibeg, nint, nsh, nel, rp_off,
// rp_cnt}, tile-local point indices, per tile-interior point the colours of
// the tile's elements that touch it, the Stacey slot / source head / colour
// of every element, and the Jacobian and material arrays of the element
// points.  Rebuilt when the sources or the
// model change.
std::vector<unsigned char> tile_records(const sfg::MediumData &M, const std::vector<int> &src_head,
                                        const DevMedium &D, int nf) {
  namespace dv = sfg::dev;
  const int rb = dv::tile_rec_bytes(nf);
  std::vector<unsigned char> out(size_t(M.ntiles) * rb, 0);
  const std::vector<float> *arr[7] = {&M.xix, &M.xiz, &M.gax, &M.gaz, &M.jac, &M.prop0, &M.prop1};
  for (int t = 0; t < M.ntiles; ++t) {
    unsigned char *r = out.data() + size_t(t) * rb;
    int *hd = reinterpret_cast<int *>(r);
    int nel = 0;
    for (int e = 0; e < dv::TILE_E; ++e) nel += M.tile_elem[size_t(t) * dv::TILE_E + e] >= 0;
    hd[0] = M.tile_ibeg[t]; hd[1] = M.tile_nint[t]; hd[2] = M.tile_nsh[t]; hd[3] = nel;
    hd[4] = D.rp_off.empty() ? 0 : D.rp_off[t];
    hd[5] = D.rp_cnt.empty() ? 0 : D.rp_cnt[t];
    std::memcpy(r + dv::TREC_LIDX, &M.tile_lidx[size_t(t) * dv::TILE_P], dv::TILE_P * sizeof(uint16_t));
    {
      // colour masks of the tile-interior points
      unsigned char *mask = r + dv::TREC_MASK;
      for (int e = 0; e < dv::TILE_E; ++e) {
        const int ce = M.tile_elem[size_t(t) * dv::TILE_E + e];
        if (ce < 0) continue;
        for (int q = 0; q < sfg::NPTS; ++q) {
          const int k = M.tile_lidx[size_t(t) * dv::TILE_P + e * sfg::NPTS + q];
          if (k < M.tile_nint[t]) mask[k] = static_cast<unsigned char>(mask[k] | (1 << M.elem_color[ce]));
        }
      }
    }
    int *bc = reinterpret_cast<int *>(r + dv::TREC_BC);
    int *sr = reinterpret_cast<int *>(r + dv::TREC_SRC);
    int *co = reinterpret_cast<int *>(r + dv::TREC_COL);
    float *f = reinterpret_cast<float *>(r + dv::TREC_F);
    for (int e = 0; e < dv::TILE_E; ++e) {
      const int ce = M.tile_elem[size_t(t) * dv::TILE_E + e];
      bc[e] = ce >= 0 ? M.bc_slot[ce] : -1;
      sr[e] = ce >= 0 && !src_head.empty() ? src_head[ce] : -1;
      co[e] = ce >= 0 ? M.elem_color[ce] : -1;
      for (int k = 0; k < nf; ++k)
        for (int q = 0; q < sfg::NPTS; ++q)
          f[size_t(k) * dv::TILE_P + e * sfg::NPTS + q] = ce >= 0 ? (*arr[k])[size_t(ce) * sfg::NPTS + q] : 0.f;
    }
  }
  return out;
}

void refresh_tile_records(sfg_handle *h) {
  if (!h->tile_ok) return;
  for (int med = 0; med < 2; ++med) {
    DevMedium &D = med == 1 ? h->el : h->ac;
    const sfg::MediumData &M = med == 1 ? h->asmb.el : h->asmb.ac;
    if (!D.t_rec) continue;
    const auto rec = tile_records(M, med == 1 ? h->asmb.el_src_head : h->asmb.ac_src_head, D,
                                  tile_nf(M, med == 1 ? SFG_MEDIUM_ELASTIC : SFG_MEDIUM_ACOUSTIC));
    SFG_CUDA(cudaMemcpy(D.t_rec, rec.data(), rec.size(), cudaMemcpyHostToDevice));
  }
}

// Device data of the fused tile kernel (after the receivers are known) and
// its shared-memory layout.  Clears h->tile_ok when the layout does not fit.
void upload_tiles(sfg_handle *h) {
  namespace dv = sfg::dev;
  const sfg::Assembly2D &a = h->asmb;
  // side slots: every point a receiver's element touches, per medium
  std::vector<std::unordered_map<int, int>> slot_of(2);
  std::vector<std::vector<std::pair<int, int>>> pts(2);   // (point, slot) in first-use order
  std::vector<int> rslot(size_t(std::max(a.nrec, 1)) * sfg::NPTS, 0);
  int nslot = 0;
  for (int r = 0; r < a.nrec; ++r) {
    const int med = a.rec_medium[r] == 1 ? 1 : 0;
    const sfg::MediumData &M = med == 1 ? a.el : a.ac;
    for (int q = 0; q < sfg::NPTS; ++q) {
      const int pt = M.ibool[size_t(a.rec_elem[r]) * sfg::NPTS + q];
      auto it = slot_of[med].find(pt);
      if (it == slot_of[med].end()) {
        it = slot_of[med].emplace(pt, nslot++).first;
        pts[med].push_back({pt, it->second});
      }
      rslot[size_t(r) * sfg::NPTS + q] = it->second;
    }
  }
  DevMem &m = h->mem;
  const int S = a.nshots;
  h->d_side = m.zeros<float>(size_t(std::max(nslot, 1)) * dv::SIDE_W * S);
  h->d_rslot = m.upload(rslot);
  for (int med = 0; med < 2; ++med) {
    DevMedium &D = med == 1 ? h->el : h->ac;
    const sfg::MediumData &M = med == 1 ? a.el : a.ac;
    D.ntiles = M.ntiles;
    if (M.nspec == 0 || M.ntiles == 0) continue;
    D.sh0 = M.sh0;
    D.nb = M.niface + (M.nglob - M.sh0);
    std::vector<std::vector<int2>> lists(M.ntiles);
    std::vector<int> bside(std::max(D.nb, 1), -1);
    for (const auto &ps : pts[med]) {
      const int pt = ps.first;
      if (pt < M.niface) { bside[pt] = ps.second; continue; }
      if (pt >= M.sh0) { bside[M.niface + pt - M.sh0] = ps.second; continue; }
      const int t = int(std::upper_bound(M.tile_ibeg.begin(), M.tile_ibeg.end(), pt) - M.tile_ibeg.begin()) - 1;
      if (t < 0 || pt >= M.tile_ibeg[t] + M.tile_nint[t]) throw std::runtime_error("tile of a receiver point not found");
      lists[t].push_back(make_int2(pt - M.tile_ibeg[t], ps.second));
    }
    D.rp_off.assign(M.ntiles, 0);
    D.rp_cnt.assign(M.ntiles, 0);
    std::vector<int2> rp;
    for (int t = 0; t < M.ntiles; ++t) {
      std::sort(lists[t].begin(), lists[t].end(), [](const int2 &x, const int2 &y) { return x.x < y.x; });
      D.rp_off[t] = int(rp.size());
      D.rp_cnt[t] = int(lists[t].size());
      rp.insert(rp.end(), lists[t].begin(), lists[t].end());
    }
    std::vector<int4> hdr(M.ntiles);
    D.max_nint = D.max_nsh = 0;
    for (int t = 0; t < M.ntiles; ++t) {
      hdr[t] = make_int4(M.tile_ibeg[t], M.tile_nint[t], M.tile_nsh[t], M.tile_sh_off[t]);
      D.max_nint = std::max(D.max_nint, M.tile_nint[t]);
      D.max_nsh = std::max(D.max_nsh, M.tile_nsh[t]);
    }
    const int nf = tile_nf(M, med == 1 ? SFG_MEDIUM_ELASTIC : SFG_MEDIUM_ACOUSTIC);
    D.rec_bytes = dv::tile_rec_bytes(nf);
    D.t_hdr = m.upload(hdr);
    D.t_rec = m.upload(tile_records(M, med == 1 ? a.el_src_head : a.ac_src_head, D, nf));
    {
      std::vector<int> sh(M.tile_sh);
      sh.resize(sh.size() + 4, 0);
      D.t_sh = m.upload(sh);
    }
    D.t_rp = m.upload(rp);
    D.t_r = m.zeros<float>(size_t(std::max(D.nb, 1)) * ncolors(D) * M.ncomp * S + 4);
    D.b_side = m.upload(bside);
    {
      std::vector<unsigned char> bm(std::max(D.nb, 1), 0);
      for (int ce = 0; ce < M.nspec; ++ce)
        for (int q = 0; q < sfg::NPTS; ++q) {
          const int g = M.ibool[size_t(ce) * sfg::NPTS + q];
          if (g < M.niface) bm[g] |= static_cast<unsigned char>(1 << M.elem_color[ce]);
          else if (g >= M.sh0) bm[M.niface + g - M.sh0] |= static_cast<unsigned char>(1 << M.elem_color[ce]);
        }
      D.b_mask = m.upload(bm);
    }
  }
  auto al4 = [](int x) { return (x + 3) & ~3; };
  if (S > 1) {
    // batched: stages of record + shared-point ids, float4 work arrays and
    // per-colour float4 accumulators
    const DevMedium &D = h->el;
    dv::TileBArgs &L = h->tileb_layout;
    L.off_sh = D.rec_bytes;
    L.stage_bytes = (L.off_sh + 4 * al4(std::max(D.max_nsh, 4)) + 15) & ~15;
    L.work_off = 64 + dv::TILEB_STAGES * L.stage_bytes;
    L.acc_off = L.work_off + 16 * dv::TILE_E * 3 * D.ncomp * sfg::NPTS;
    L.kcap = al4(std::max(D.max_nint, 4));
    h->tile_smem = L.acc_off + 16 * ncolors(D) * D.ncomp * L.kcap;
    if (h->tile_smem > 227 * 1024) { h->tile_ok = false; return; }
    auto kern = D.ncomp == 1 ? dv::k_tile_b<1> : dv::k_tile_b<2>;
    SFG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, h->tile_smem));
    int nb = 0;
    SFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, dv::TILE_P, h->tile_smem));
    h->tile_blocks_per_sm = std::max(nb, 1);
    return;
  }
  // shared-memory layout (uniform over the blocks of both media)
  int rec = 0, fcap = 4, shcap = 4, accw = 4;
  for (const DevMedium *D : {&h->el, &h->ac}) {
    if (!D->t_rec) continue;
    rec = std::max(rec, D->rec_bytes);
    fcap = std::max(fcap, al4(D->max_nint * D->ncomp + 6));
    shcap = std::max(shcap, al4(D->max_nsh));
    accw = std::max(accw, al4(D->max_nint) * ncolors(*D) * D->ncomp);
  }
  dv::TileArgs &L = h->tile_layout;
  L.off_sh = rec;
  L.off_u = L.off_sh + 4 * shcap;
  L.off_v = L.off_u + 4 * fcap;
  L.off_m = L.off_v + 4 * fcap;
  L.stage_bytes = L.off_m + 4 * fcap;
  L.work_off = 64 + dv::TILE_STAGES * L.stage_bytes;
  L.acc_off = L.work_off + 4 * dv::TILE_E * dv::TILE_WORK;
  L.acc_words = accw;
  h->tile_smem = L.acc_off + 4 * accw;
  if (h->tile_smem > 227 * 1024) { h->tile_ok = false; return; }
  auto kern = h->el.ncomp == 1 ? dv::k_tile<1> : dv::k_tile<0>;
  SFG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, h->tile_smem));
  int nb = 0;
  SFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, dv::TILE_P, h->tile_smem));
  h->tile_blocks_per_sm = std::max(nb, 1);
}

// Batched tiles of four elements (variant 7): consecutive groups of four of
// the Morton-ordered 16-element tiles (2 x 2 patches on structured meshes),
// each sorted by colour; a point is interior to a tile when only that tile's
// elements touch it.  Needs S shots in fours, one elastic medium, and
// receivers that record displacement only (they run before the step's
// kernels).
bool compute_btile_ok(const sfg_handle *h) {
  const sfg::Assembly2D &a = h->asmb;
  if (a.nshots <= 1 || a.nshots % 4 != 0 || a.ac.nspec || !a.el.nspec || a.el.ntiles == 0) return false;
  if (a.el.aniso || a.el.cosserat || a.el.poro || a.el.ncomp > 2) return false;
  for (int t : a.types)
    if (t != SFG_SEIS_DISPLACEMENT) return false;
  return true;
}

void upload_btiles(sfg_handle *h) {
  namespace dv = sfg::dev;
  const sfg::MediumData &M = h->asmb.el;
  DevMedium &D = h->el;
  const int n = M.nspec;
  std::vector<int> cnt(size_t(M.nglob), 0);
  for (size_t i = 0; i < size_t(n) * sfg::NPTS; ++i) ++cnt[M.ibool[i]];
  std::vector<int> tel, loc(size_t(n) * sfg::NPTS, -1), tpt, tctr;
  std::vector<char> interior(size_t(M.nglob), 0);
  std::unordered_map<int, int> lcnt, kidx;
  const int ngroups = M.ntiles * (sfg::TILE_E / dv::BT_E);
  for (int gi = 0; gi < ngroups; ++gi) {
    std::vector<int> els;
    for (int i = 0; i < dv::BT_E; ++i) {
      const int ce = M.tile_elem[size_t(gi) * dv::BT_E + i];
      if (ce >= 0) els.push_back(ce);
    }
    if (els.empty()) continue;
    std::stable_sort(els.begin(), els.end(), [&](int x, int y) { return M.elem_color[x] < M.elem_color[y]; });
    const int t = int(tel.size() / dv::BT_E);
    for (int i = 0; i < dv::BT_E; ++i) tel.push_back(i < int(els.size()) ? els[i] : -1);
    lcnt.clear();
    kidx.clear();
    for (int ce : els)
      for (int q = 0; q < sfg::NPTS; ++q) ++lcnt[M.ibool[size_t(ce) * sfg::NPTS + q]];
    tpt.resize(size_t(t + 1) * dv::BT_MAXP, -1);
    tctr.resize(size_t(t + 1) * dv::BT_MAXP * 4, -1);
    for (int le = 0; le < int(els.size()); ++le)
      for (int q = 0; q < sfg::NPTS; ++q) {
        const int g = M.ibool[size_t(els[le]) * sfg::NPTS + q];
        if (lcnt[g] != cnt[g]) continue;        // another tile touches it
        auto it = kidx.find(g);
        if (it == kidx.end()) {
          const int k = int(kidx.size());
          if (k >= dv::BT_MAXP) throw std::runtime_error("batched tile with too many interior points");
          it = kidx.emplace(g, k).first;
          tpt[size_t(t) * dv::BT_MAXP + k] = g;
          interior[g] = 1;
        }
        const int k = it->second;
        int *c = &tctr[(size_t(t) * dv::BT_MAXP + k) * 4];
        int m = 0;
        while (m < 4 && c[m] >= 0) ++m;
        if (m == 4) throw std::runtime_error("batched tile point with more than four contributions");
        c[m] = le * sfg::NPTS + q;
        loc[size_t(els[le]) * sfg::NPTS + q] = k;
      }
  }
  std::vector<int> bpts;
  for (int g = 0; g < M.nglob; ++g)
    if (!interior[g]) bpts.push_back(g);
  DevMem &m = h->mem;
  D.nbt = int(tel.size() / dv::BT_E);
  D.nbp = int(bpts.size());
  D.bt_tel = m.upload(tel);
  D.bt_loc = m.upload(loc);
  D.bt_pt = m.upload(tpt);
  D.bt_ctr = m.upload(tctr);
  if (bpts.empty()) bpts.push_back(0);
  D.bt_bpts = m.upload(bpts);
  const int smem_max = dv::BT_E * 2 * 2 * sfg::NPTS * 8 * int(sizeof(float4));
  SFG_CUDA(cudaFuncSetAttribute(dv::k_btile_row<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max));
  SFG_CUDA(cudaFuncSetAttribute(dv::k_btile_row<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max / 2));
}

sfg::dev::TileMed tile_med(const DevMedium &D, int ncol, bool store_a) {
  sfg::dev::TileMed M{};
  M.hdr = D.t_hdr; M.rec = D.t_rec; M.sh = D.t_sh; M.rp = D.t_rp;
  M.u = D.u; M.v = D.v; M.a = D.a; M.minv = D.minv; M.r = D.t_r;
  M.rec_bytes = D.rec_bytes; M.ntiles = D.t_rec ? D.ntiles : 0; M.ncol = ncol;
  M.niface = D.niface; M.sh0 = D.sh0;
  M.store_a = store_a ? 1 : 0;
  return M;
}

sfg::dev::BndMed bnd_med(const DevMedium &D, const sfg::MediumData &M) {
  sfg::dev::BndMed B{};
  B.r = D.t_r; B.b_side = D.b_side; B.b_mask = D.b_mask;
  B.nb = D.t_rec ? D.nb : 0; B.niface = M.niface; B.sh0 = M.sh0; B.ncol = ncolors(D);
  return B;
}

// Batched tiles of four elements (variant 7): the tile kernel, then the
// points tiles share.
void launch_btile(sfg_handle *h, bool predict, cudaStream_t s) {
  namespace dv = sfg::dev;
  const DevMedium &el = h->el;
  dv::BTileArgs P{};
  P.B = batch_args(h, el, h->d_step);
  P.tel = el.bt_tel; P.tloc = el.bt_loc; P.tpt = el.bt_pt; P.tctr = el.bt_ctr;
  P.minv = el.minv; P.v_out = el.v; P.u_out = el.u;
  P.a_store = (!predict || h->opt.store_acceleration) ? el.a : nullptr;
  const float dt = float(h->asmb.dt);
  P.dt = dt; P.dt2 = dt / 2.0f; P.dtsq2 = dt * dt / 2.0f;
  P.predict = predict ? 1 : 0;
  P.flag = h->d_flag;
  P.ntiles = el.nbt;
  const int T = std::min(8, el.S / 4);
  const int tiles = (el.S + 4 * T - 1) / (4 * T);
  const int smem = dv::BT_E * el.ncomp * 2 * sfg::NPTS * T * int(sizeof(float4));
  const dim3 grid(el.nbt, tiles);
  if (el.nbt == 0) return;
  if (el.ncomp == 2) dv::k_btile_row<2><<<grid, dv::BT_E * dv::NG * T, smem, s>>>(P, T);
  else dv::k_btile_row<1><<<grid, dv::BT_E * dv::NG * T, smem, s>>>(P, T);
}

void launch_btile_shared(sfg_handle *h, bool predict, cudaStream_t s) {
  const DevMedium &el = h->el;
  sfg::dev::UpdateArgs U = update_args(h, el, h->ac, SFG_MEDIUM_ELASTIC, predict, true);
  const int n4 = el.nbp * el.ncomp * el.S / 4;
  sfg::dev::k_update_batched4_list<<<grid_for(std::max(n4, 1)), 256, 0, s>>>(U, el.S, el.ncomp, el.bt_bpts, el.nbp);
}

// The batched fused tile kernel (one elastic medium, S shots): work items
// are (tile, quad of shots), the quads of a tile adjacent in item order so
// that they run at about the same time and share the record through L2.
void launch_tile_kernel_b(sfg_handle *h, bool predict, cudaStream_t s) {
  namespace dv = sfg::dev;
  const sfg::Assembly2D &a = h->asmb;
  dv::TileBArgs A = h->tileb_layout;
  A.el = tile_med(h->el, ncolors(h->el), !predict || h->opt.store_acceleration);
  A.bel = med_args(h->el);
  A.src_next = h->d_src_next; A.src_shot = h->d_src_shot; A.src_arr = h->d_src_arr; A.stf = h->d_stf;
  A.nsrc = a.nsrc; A.nstep = a.nstep; A.step = h->d_step;
  const float dt = float(a.dt);
  A.dt = dt; A.dt2 = dt / 2.0f; A.dtsq2 = dt * dt / 2.0f;
  A.predict = predict ? 1 : 0;
  A.flag = h->d_flag;
  A.side = h->d_side;
  A.S = h->el.S;
  A.quad = h->quad;
  const int items = A.el.ntiles * (A.S / 4);
  const int grid = std::min(h->tile_blocks_per_sm * h->sm_count, items);
  if (grid <= 0) return;
  if (h->el.ncomp == 1) dv::k_tile_b<1><<<grid, dv::TILE_P, h->tile_smem, s>>>(A);
  else dv::k_tile_b<2><<<grid, dv::TILE_P, h->tile_smem, s>>>(A);
}

// The fused tile kernel of both media.
void launch_tile_kernel(sfg_handle *h, bool predict, cudaStream_t s) {
  namespace dv = sfg::dev;
  if (h->asmb.nshots > 1) {
    launch_tile_kernel_b(h, predict, s);
    return;
  }
  const sfg::Assembly2D &a = h->asmb;
  dv::TileArgs A = h->tile_layout;
  A.el = tile_med(h->el, ncolors(h->el), !predict || h->opt.store_acceleration);
  A.ac = tile_med(h->ac, ncolors(h->ac), !predict);
  A.bel = med_args(h->el);
  A.bac = med_args(h->ac);
  A.src_next = h->d_src_next; A.src_arr = h->d_src_arr; A.stf = h->d_stf;
  A.nsrc = a.nsrc; A.nstep = a.nstep; A.step = h->d_step;
  const float dt = float(a.dt);
  A.dt = dt; A.dt2 = dt / 2.0f; A.dtsq2 = dt * dt / 2.0f;
  A.predict = predict ? 1 : 0;
  A.flag = h->d_flag;
  A.side = h->d_side;
  A.quad = h->quad;
  const int cap = h->tile_blocks_per_sm * h->sm_count;
  const int te = A.el.ntiles, ta = A.ac.ntiles;
  int be = te == 0 ? 0 : std::max(1, int(double(cap) * te / (te + ta) + 0.5));
  if (ta > 0) be = std::min(be, cap - 1);
  be = std::min(be, te);
  const int ba = std::min(std::max(cap - be, ta > 0 ? 1 : 0), ta);
  A.el.nblocks = be;
  A.ac.nblocks = ba;
  if (be + ba == 0) return;
  if (h->el.ncomp == 1) dv::k_tile<1><<<be + ba, dv::TILE_P, h->tile_smem, s>>>(A);
  else dv::k_tile<0><<<be + ba, dv::TILE_P, h->tile_smem, s>>>(A);
}

// Boundary points of both media (advances the step counter).
void launch_tile_boundary(sfg_handle *h, bool predict, cudaStream_t s) {
  namespace dv = sfg::dev;
  if (h->asmb.nshots > 1) {
    dv::UpdateArgs U = update_args(h, h->el, h->ac, SFG_MEDIUM_ELASTIC, predict, true);
    const dv::BndMed b = bnd_med(h->el, h->asmb.el);
    const int n = b.nb * (h->el.S / 4);
    if (h->el.ncomp == 1) dv::k_tile_boundary_b<1><<<grid_for(n), 256, 0, s>>>(U, b, h->d_side, h->el.S);
    else dv::k_tile_boundary_b<2><<<grid_for(n), 256, 0, s>>>(U, b, h->d_side, h->el.S);
    return;
  }
  const bool has_el = h->el.nspec > 0, has_ac = h->ac.nspec > 0;
  if (has_el && has_ac) {
    dv::UpdateArgs E = update_args(h, h->el, h->ac, SFG_MEDIUM_ELASTIC, predict, true);
    dv::UpdateArgs C = update_args(h, h->ac, h->el, SFG_MEDIUM_ACOUSTIC, predict, false);
    const dv::BndMed be = bnd_med(h->el, h->asmb.el), ba = bnd_med(h->ac, h->asmb.ac);
    const int n = be.nb + ba.nb - ba.niface;
    dv::k_tile_boundary<2, true><<<grid_for(n), 256, 0, s>>>(E, be, C, ba, h->d_side);
    return;
  }
  const int med = has_el ? SFG_MEDIUM_ELASTIC : SFG_MEDIUM_ACOUSTIC;
  const DevMedium &D = has_el ? h->el : h->ac;
  const DevMedium &O = has_el ? h->ac : h->el;
  dv::UpdateArgs U = update_args(h, D, O, med, predict, true);
  const dv::BndMed b = bnd_med(D, has_el ? h->asmb.el : h->asmb.ac);
  if (D.ncomp == 2)
    dv::k_tile_boundary<2, false><<<grid_for(b.nb), 256, 0, s>>>(U, b, U, b, h->d_side);
  else
    dv::k_tile_boundary<1, false><<<grid_for(b.nb), 256, 0, s>>>(U, b, U, b, h->d_side);
}

void launch_tile_receivers(sfg_handle *h, cudaStream_t s) {
  for (int med : {SFG_MEDIUM_ACOUSTIC, SFG_MEDIUM_ELASTIC}) {
    const DevMedium &D = med == SFG_MEDIUM_ELASTIC ? h->el : h->ac;
    if (D.nspec == 0 || D.nrec == 0) continue;
    if (D.S > 1)
      sfg::dev::k_receivers_side_b<<<D.nrec, 32, 0, s>>>(rec_args(h, med), h->d_rslot, h->d_side, D.S);
    else
      sfg::dev::k_receivers_side<<<D.nrec, 32, 0, s>>>(rec_args(h, med), h->d_rslot, h->d_side);
  }
}

void enqueue_tile_step(sfg_handle *h, cudaStream_t s, bool predict) {
  launch_tile_kernel(h, predict, s);
  launch_tile_boundary(h, predict, s);
  launch_tile_receivers(h, s);
}

void enqueue_step(sfg_handle *h, cudaStream_t s, bool predict) {
  if (h->variant == 5 && !h->recording) {
    enqueue_tile_step(h, s, predict);
    return;
  }
  if (h->variant == 7) {
    // batched tiles: the receivers (displacement only) read the step's
    // displacement first; the tile kernel finishes the tile-interior points,
    // the list update the shared ones (and advances the step counter)
    if (h->el.nrec > 0) launch_receivers(h, SFG_MEDIUM_ELASTIC, s);
    launch_btile(h, predict, s);
    launch_btile_shared(h, predict, s);
    return;
  }
  const bool has_el = h->el.nspec > 0, has_ac = h->ac.nspec > 0;
  if (h->recording) {
    const DevMedium &R = h->el.nspec ? h->el : h->ac;
    if (R.ncomp == 1) sfg::dev::k_record_begin<1><<<1, 512, 0, s>>>(h->adj.d_rec, R.v, h->d_step);
    else sfg::dev::k_record_begin<2><<<1, 512, 0, s>>>(h->adj.d_rec, R.v, h->d_step);
    if (h->adj_coupled) sfg::dev::k_record_begin<1><<<1, 512, 0, s>>>(h->adj2.d_rec, h->ac.v, h->d_step);
  }
  // a recorded (recomputed) step's seismograms are those of the forward run
  const bool rec_ac = has_ac && h->ac.nrec > 0 && h->recording != 2;
  const bool rec_el = has_el && h->el.nrec > 0 && h->recording != 2;
  const bool early_ac = rec_ac && receivers_early(h, SFG_MEDIUM_ACOUSTIC);
  const bool early_el = rec_el && receivers_early(h, SFG_MEDIUM_ELASTIC);
  const bool fork = (early_ac || early_el) && h->side;
  if (fork) {
    // receivers on the side stream, concurrent with the element kernel; they
    // join before the first update changes the displacement
    SFG_CUDA(cudaEventRecord(h->ev_fork, s));
    SFG_CUDA(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
    if (early_ac) launch_receivers(h, SFG_MEDIUM_ACOUSTIC, h->side);
    if (early_el) launch_receivers(h, SFG_MEDIUM_ELASTIC, h->side);
    SFG_CUDA(cudaEventRecord(h->ev_join, h->side));
  }
  launch_stiffness(h, s);
  if (fork) SFG_CUDA(cudaStreamWaitEvent(s, h->ev_join, 0));
  if (fused_update(h)) {
    if (rec_ac && !(fork && early_ac)) launch_receivers(h, SFG_MEDIUM_ACOUSTIC, s);
    if (rec_el && !(fork && early_el)) launch_receivers(h, SFG_MEDIUM_ELASTIC, s);
    launch_update_coupled(h, predict, s);
    return;
  }
  if (has_ac) {
    if (rec_ac && !(fork && early_ac)) launch_receivers(h, SFG_MEDIUM_ACOUSTIC, s);
    launch_update(h, SFG_MEDIUM_ACOUSTIC, predict, !has_el, s);
  }
  if (has_el) {
    if (rec_el && !(fork && early_el)) launch_receivers(h, SFG_MEDIUM_ELASTIC, s);
    launch_update(h, SFG_MEDIUM_ELASTIC, predict, true, s);
  }
}

int kernels_per_step(const sfg_handle *h) {
  if (h->variant == 5) return 2 + (h->el.nspec && h->el.nrec > 0) + (h->ac.nspec && h->ac.nrec > 0);
  if (h->variant == 7) return 2 + (h->el.nrec > 0);
  int n = h->variant >= 3 ? 1 : std::max(ncolors(h->el), ncolors(h->ac));
  for (const DevMedium *D : {&h->ac, &h->el}) {
    if (D->nspec == 0) continue;
    n += (D->nrec > 0 ? 1 : 0) + 1;
  }
  return fused_update(h) ? n - 1 : n;
}

bool fused_update(const sfg_handle *h) {
  if (!h->fuse_ok || h->variant < 3 || h->recording) return false;
  const sfg::Assembly2D &a = h->asmb;
  if (h->el.nrec == 0) return true;
  for (int t : a.types)
    if (t != SFG_SEIS_DISPLACEMENT && t != SFG_SEIS_PRESSURE) return false;
  return true;
}

cudaGraphExec_t capture(sfg_handle *h, int nsteps, bool last_predicts) {
  cudaGraph_t g = nullptr;
  SFG_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < nsteps; ++i) enqueue_step(h, h->stream, i + 1 < nsteps || last_predicts);
  SFG_CUDA(cudaStreamEndCapture(h->stream, &g));
  cudaGraphExec_t ex = nullptr;
  SFG_CUDA(cudaGraphInstantiate(&ex, g, 0));
  cudaGraphDestroy(g);
  return ex;
}

void resume(sfg_handle *h) {
  if (h->state_final) {
    launch_predict(h, h->stream);
    h->state_final = false;
  }
}

// nsteps steps; the run ends on a corrector-only update so that the fields
// are the reference's end-of-step state.
void run_steps(sfg_handle *h, int nsteps) {
  if (nsteps <= 0) return;
  resume(h);
  int fused = nsteps - 1;
  while (fused >= h->graph_steps && h->graph_k) {
    SFG_CUDA(cudaGraphLaunch(h->graph_k, h->stream));
    fused -= h->graph_steps;
  }
  while (fused > 0) {
    SFG_CUDA(cudaGraphLaunch(h->graph_1, h->stream));
    --fused;
  }
  SFG_CUDA(cudaGraphLaunch(h->graph_e, h->stream));
  h->state_final = true;
  SFG_CUDA(cudaGetLastError());
  h->host_step += nsteps;
}

// Launch-shape autotuner: every candidate (colour passes, persistent colour
// passes or owner-computes assembly; 8, 16 or 32 elements per block) gives
// bit-identical results, so the one with the fastest whole step measured on
// this mesh is kept.  Runs at sfg_initialize, before the step graphs are
// captured; the fields and counters it touches are cleared afterwards.
void autotune(sfg_handle *h) {
  const bool fix_e = h->opt.elements_per_block == 8 || h->opt.elements_per_block == 16 ||
                     h->opt.elements_per_block == 32;
  const bool fix_v = h->opt.kernel_variant >= 1 && h->opt.kernel_variant <= 7;
  if (fix_e) h->epb = h->opt.elements_per_block;
  if (fix_v) h->variant = h->opt.kernel_variant;
  if (h->variant == 5 && !h->tile_ok) h->variant = 3;   // the model cannot use the tile kernel
  if (h->variant == 5) h->epb = 16;
  // the row form: isotropic P-SV / acoustic, one shot, 16 or 32 elements per block
  if (h->variant == 6 && (h->asmb.nshots > 1 || !row_ok(h->el))) h->variant = 3;
  if (h->variant == 6 && h->epb != 16) h->epb = 32;
  if (h->variant == 7 && !h->btile_ok) h->variant = 3;   // batched tiles of four elements
  if (h->asmb.nshots > 1 && h->variant == 2) h->variant = 1;  // no persistent batched kernel
  // batched: variant 4 is owner-computes with the row-form element kernel (shots in fours)
  if (h->asmb.nshots > 1 && h->variant == 4 && h->asmb.nshots % 4 != 0) h->variant = 3;
  const bool special = h->el.aniso || h->el.ncomp >= 3;   // anisotropic, Cosserat or poroelastic
  if (special && h->variant == 2) h->variant = 1;
  if (special && h->variant == 4) h->variant = 3;
  std::vector<std::pair<int, int>> cand;
  if (h->asmb.nshots > 1) {
    for (int v : {1, 3, 4})
      if ((!fix_v || v == h->variant) && (v != 4 || h->asmb.nshots % 4 == 0)) cand.push_back({v, 16});
    if (h->tile_ok && (!fix_v || h->variant == 5)) cand.push_back({5, 16});
    if (h->btile_ok && (!fix_v || h->variant == 7)) cand.push_back({7, 16});
  } else {
    for (int v : {1, 2, 3, 4}) {
      // an anisotropic medium has the colour-pass and owner-computes kernels only
      if (special && (v == 2 || v == 4)) continue;
      for (int e : {8, 16, 32})
        if ((!fix_v || v == h->variant) && (!fix_e || e == h->epb)) cand.push_back({v, e});
    }
    // fused tile kernel: tiles of 16 elements
    if (h->tile_ok && (!fix_v || h->variant == 5) && (!fix_e || h->epb == 16)) cand.push_back({5, 16});
    // row-form element kernel
    if (row_ok(h->el) && (!fix_v || h->variant == 6))
      for (int e : {16, 32})
        if (!fix_e || e == h->epb) cand.push_back({6, e});
  }
  if (cand.empty()) cand.push_back({h->variant, h->epb});
  if (cand.size() > 1) {
    float best = 1e30f;
    std::pair<int, int> pick = cand.front();
    const int reps = 5;
    for (auto [v, e] : cand) {
      h->variant = v;
      h->epb = e;
      for (int i = 0; i < 2; ++i) enqueue_step(h, h->stream, true);
      SFG_CUDA(cudaEventRecord(h->ev0, h->stream));
      for (int i = 0; i < reps; ++i) enqueue_step(h, h->stream, true);
      SFG_CUDA(cudaEventRecord(h->ev1, h->stream));
      SFG_CUDA(cudaEventSynchronize(h->ev1));
      SFG_CUDA(cudaGetLastError());
      float t = 0;
      SFG_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
      if (t < best) { best = t; pick = {v, e}; }
    }
    h->variant = pick.first;
    h->epb = pick.second;
  } else {
    h->variant = cand[0].first;
    h->epb = cand[0].second;
  }
  // the tuning steps ran on the (zero) fields: clear every state word again
  for (DevMedium *D : {&h->el, &h->ac}) {
    if (!D->nspec) continue;
    const size_t n = (D->values() + 4) * sizeof(float);
    SFG_CUDA(cudaMemsetAsync(D->u, 0, n, h->stream));
    SFG_CUDA(cudaMemsetAsync(D->v, 0, n, h->stream));
    SFG_CUDA(cudaMemsetAsync(D->accum, 0, n, h->stream));
    SFG_CUDA(cudaMemsetAsync(D->a, 0, n, h->stream));
  }
  const sfg::Assembly2D &a = h->asmb;
  SFG_CUDA(cudaMemsetAsync(h->d_seis, 0,
                           size_t(a.nshots) * a.nsig * a.ntypes * std::max(a.nrec, 1) * 2 * sizeof(float),
                           h->stream));
  SFG_CUDA(cudaMemsetAsync(h->d_step, 0, sizeof(int), h->stream));
  SFG_CUDA(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  SFG_CUDA(cudaStreamSynchronize(h->stream));
}

sfg_handle *make_handle(const sfg_options *opt) {
  if (!opt) throw std::runtime_error("options are required");
  if (!(opt->dt > 0) || opt->nstep <= 0) throw std::runtime_error("dt and nstep must be positive");
  auto *h = new sfg_handle();
  h->opt = *opt;
  if (h->opt.nshots <= 0) h->opt.nshots = 1;
  if (h->opt.nstep_between_samples <= 0) h->opt.nstep_between_samples = 1;
  if (h->opt.steps_per_graph <= 0) h->opt.steps_per_graph = 20;
  h->epb = 16;
  return h;
}

void finish_create(sfg_handle *h) {
  h->mesh.elastic_wave = h->mesh.elastic_wave ? 1 : 0;
  h->asmb.nshots = h->opt.nshots;
  h->asmb.user_t0 = h->opt.has_start_time != 0;
  h->asmb.user_t0_value = h->opt.start_time;
  h->asmb.nstep = h->opt.nstep;
  h->asmb.nsb = h->opt.nstep_between_samples;
  sfg::assemble2d(h->mesh, h->opt.dt, h->asmb);
  if (h->asmb.nshots > 1 &&
      (h->asmb.ac.nspec > 0 || h->asmb.el.nspec == 0 || h->asmb.el.aniso || h->asmb.el.ncomp >= 3))
    throw std::runtime_error("batched shots (nshots > 1) need a single isotropic elastic medium");
}

// ---------------------------------------------------------------------------
// Scratch of sfg_step_noalloc.  The element kernel adds every element's
// contribution into an accumulator that is neither an input nor an output of
// a time step; the handle-based path allocates it with cudaMalloc at
// sfg_initialize.  sfg_step_noalloc uses this fixed array instead, so that it
// allocates nothing.  It is sized for NOALLOC_MAX_VALUES floats (one per point
// component: 2,097,152 two-component points) plus the 4-float tail the float4
// update reads, and every GPU that loads the library holds it (16 MiB) until
// the process exits.  Every call shares it: the accumulator is cleared at the
// start of each call, and calls that overlap on the GPU race on it.
constexpr size_t NOALLOC_MAX_VALUES = size_t(1) << 22;
static __device__ __align__(256) float g_noalloc_accum[NOALLOC_MAX_VALUES + 4];
static __device__ __align__(256) int g_noalloc_words[4];  // [0] step index, [1] non-finite flag

struct NoallocDevice {
  float *accum = nullptr;
  int *words = nullptr;
};

// Device addresses of the scratch, looked up once per device with that device
// current (a __device__ symbol's host-side name is not a device address).
int noalloc_device(NoallocDevice &out, std::string &err) {
  static std::mutex mu;
  static std::vector<NoallocDevice> table;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { err = cudaGetErrorString(e); return SFG_ERR_CUDA; }
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= int(table.size())) table.resize(dev + 1);
  NoallocDevice &d = table[dev];
  if (!d.accum) {
    void *pa = nullptr, *pw = nullptr;
    e = cudaGetSymbolAddress(&pa, g_noalloc_accum);
    if (e != cudaSuccess) { err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e); return SFG_ERR_CUDA; }
    e = cudaGetSymbolAddress(&pw, g_noalloc_words);
    if (e != cudaSuccess) { err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e); return SFG_ERR_CUDA; }
    d.accum = static_cast<float *>(pa);
    d.words = static_cast<int *>(pw);
  }
  out = d;
  return SFG_OK;
}

}  // namespace

extern "C" {

int sfg_create2d(const sfg_mesh2d_desc *d, const sfg_options *opt, sfg_handle **out) {
  if (!d || !out) { g_create_error = "null argument"; return SFG_ERR_ARG; }
  *out = nullptr;
  sfg_handle *h = nullptr;
  try {
    h = make_handle(opt);
    sfg::Mesh2D &m = h->mesh;
    if (d->nspec <= 0 || d->npgeo <= 0 || (d->ngnod != 4 && d->ngnod != 9) || d->numat <= 0 ||
        !d->coorg || !d->knods || !d->kmato || !d->mat_medium || !d->mat_rho || !d->mat_vp || !d->mat_vs)
      throw std::runtime_error("incomplete mesh description");
    m.nspec = d->nspec; m.npgeo = d->npgeo; m.ngnod = d->ngnod; m.numat = d->numat;
    m.coorg.assign(d->coorg, d->coorg + 2 * size_t(d->npgeo));
    m.knods.assign(d->knods, d->knods + size_t(d->nspec) * d->ngnod);
    m.kmato.assign(d->kmato, d->kmato + d->nspec);
    for (int k : m.knods)
      if (k < 0 || k >= m.npgeo) throw std::runtime_error("knods out of range");
    for (int k : m.kmato)
      if (k < 0 || k >= m.numat) throw std::runtime_error("kmato out of range");
    m.mat_medium.assign(d->mat_medium, d->mat_medium + d->numat);
    m.mat_rho.assign(d->mat_rho, d->mat_rho + d->numat);
    m.mat_vp.assign(d->mat_vp, d->mat_vp + d->numat);
    m.mat_vs.assign(d->mat_vs, d->mat_vs + d->numat);
    if (d->mat_aniso) m.mat_aniso.assign(d->mat_aniso, d->mat_aniso + 6 * size_t(d->numat));
    if (d->mat_cosserat) m.mat_cosserat.assign(d->mat_cosserat, d->mat_cosserat + 8 * size_t(d->numat));
    if (d->mat_poro) m.mat_poro.assign(d->mat_poro, d->mat_poro + 13 * size_t(d->numat));
    if (d->nadj < 0 || (d->nadj > 0 && !d->adjacency)) throw std::runtime_error("bad adjacency records");
    if (d->nadj > 0) m.adjacency.assign(d->adjacency, d->adjacency + 4 * size_t(d->nadj));
    const size_t np = size_t(d->nspec) * sfg::NPTS;
    if (d->point_rho) m.prho.assign(d->point_rho, d->point_rho + np);
    if (d->point_vp) m.pvp.assign(d->point_vp, d->point_vp + np);
    if (d->point_vs) m.pvs.assign(d->point_vs, d->point_vs + np);
    if (d->nabs > 0) {
      m.abs_ispec.assign(d->abs_ispec, d->abs_ispec + d->nabs);
      m.abs_type.assign(d->abs_type, d->abs_type + d->nabs);
    }
    if (d->nfree > 0) {
      m.free_ispec.assign(d->free_ispec, d->free_ispec + d->nfree);
      m.free_type.assign(d->free_type, d->free_type + d->nfree);
    }
    for (size_t i = 0; i < m.abs_ispec.size(); ++i)
      if (m.abs_ispec[i] < 0 || m.abs_ispec[i] >= m.nspec || m.abs_type[i] < 0 || m.abs_type[i] > 3)
        throw std::runtime_error("absorbing edge out of range");
    for (size_t i = 0; i < m.free_ispec.size(); ++i)
      if (m.free_ispec[i] < 0 || m.free_ispec[i] >= m.nspec || m.free_type[i] < 0 || m.free_type[i] > 3)
        throw std::runtime_error("free-surface edge out of range");
    m.elastic_wave = d->elastic_wave;
    finish_create(h);
  } catch (const std::exception &ex) {
    g_create_error = ex.what();
    delete h;
    return SFG_ERR_ARG;
  }
  *out = h;
  return SFG_OK;
}

int sfg_create2d_from_database(const char *path, int elastic_wave, const sfg_options *opt,
                               sfg_handle **out) {
  if (!path || !out) { g_create_error = "null argument"; return SFG_ERR_ARG; }
  *out = nullptr;
  sfg_handle *h = nullptr;
  try {
    h = make_handle(opt);
    std::string err;
    if (!sfg::read_database2d(path, h->mesh, err)) {
      g_create_error = err;
      delete h;
      return SFG_ERR_IO;
    }
    h->mesh.elastic_wave = elastic_wave;
    finish_create(h);
  } catch (const std::exception &ex) {
    g_create_error = ex.what();
    delete h;
    return SFG_ERR_ARG;
  }
  *out = h;
  return SFG_OK;
}

void sfg_destroy(sfg_handle *h) { delete h; }

const char *sfg_last_error(const sfg_handle *h) {
  return h ? h->err.c_str() : g_create_error.c_str();
}

int sfg_set_sources(sfg_handle *h, int nsrc, const sfg_source2d *src) {
  return guarded(h, [&]() {
    if (nsrc < 0 || (nsrc > 0 && !src)) { h->err = "bad source array"; return int(SFG_ERR_ARG); }
    if (h->initialized && nsrc != h->asmb.nsrc) {
      h->err = "after sfg_initialize the number of sources is fixed";
      return int(SFG_ERR_STATE);
    }
    h->sources.clear();
    for (int i = 0; i < nsrc; ++i)
      h->sources.push_back({src[i].x, src[i].z, src[i].shot, src[i].stf, src[i].f0, src[i].factor,
                            src[i].tshift, src[i].angle, src[i].kind, src[i].mxx, src[i].mzz,
                            src[i].mxz, src[i].hdur});
    try {
      sfg::set_sources2d(h->mesh, h->asmb, h->sources);
    } catch (const std::exception &ex) {
      h->err = ex.what();
      return int(SFG_ERR_LOCATE);
    }
    h->have_sources = true;
    if (h->initialized) {
      // same source count: the device tables keep their sizes (and the step
      // graphs their pointers); refill them in place
      const sfg::Assembly2D &a = h->asmb;
      auto put = [&](auto *d, const auto &v) {
        if (d && !v.empty()) SFG_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice));
      };
      SFG_CUDA(cudaStreamSynchronize(h->stream));
      if (h->el.nspec) put(h->el.src_head, a.el_src_head);
      if (h->ac.nspec) put(h->ac.src_head, a.ac_src_head);
      put(h->d_src_next, a.src_next);
      put(h->d_src_shot, a.src_shot);
      put(h->d_src_arr, a.src_arr);
      put(h->d_src_arr2, a.src_arr2);
      put(h->d_stf, a.stf);
      refresh_tile_records(h);
      h->adj.forward_done = false;
    }
    return int(SFG_OK);
  });
}

int sfg_set_stf_table(sfg_handle *h, const float *table, int nstep, int nsrc) {
  return guarded(h, [&]() {
    if (!h->have_sources || nsrc != h->asmb.nsrc || nstep != h->asmb.nstep || !table) {
      h->err = "STF table must match [nstep][nsrc] of the sources already set";
      return int(SFG_ERR_ARG);
    }
    for (int i = 0; i < nstep; ++i)
      for (int s = 0; s < nsrc; ++s) {
        const float v = table[size_t(i) * nsrc + s];
        h->asmb.stf[size_t(i) * nsrc + s] = h->asmb.src_medium[s] == 0 ? -v : v;
      }
    return int(SFG_OK);
  });
}

int sfg_set_receivers(sfg_handle *h, int nrec, const double *x, const double *z, double angle,
                      int ntypes, const int *types) {
  return guarded(h, [&]() {
    if (h->initialized) { h->err = "receivers must be set before sfg_initialize"; return int(SFG_ERR_STATE); }
    if (nrec < 0 || (nrec > 0 && (!x || !z)) || ntypes < 1 || ntypes > 7 || !types) {
      h->err = "bad receiver arguments";
      return int(SFG_ERR_ARG);
    }
    for (int t = 0; t < ntypes; ++t)
      if (types[t] < 0 || types[t] > 6) { h->err = "unknown seismogram type"; return int(SFG_ERR_ARG); }
    h->rec_x.assign(x, x + nrec);
    h->rec_z.assign(z, z + nrec);
    try {
      sfg::set_receivers2d(h->mesh, h->asmb, h->rec_x, h->rec_z, angle, std::vector<int>(types, types + ntypes));
    } catch (const std::exception &ex) {
      h->err = ex.what();
      return int(SFG_ERR_LOCATE);
    }
    h->have_receivers = true;
    return int(SFG_OK);
  });
}

int sfg_initialize(sfg_handle *h) {
  return guarded(h, [&]() {
    if (h->initialized) return int(SFG_OK);
    sfg::Assembly2D &a = h->asmb;
    if (!h->have_sources) sfg::set_sources2d(h->mesh, a, {});
    if (!h->have_receivers) { a.nrec = 0; a.ntypes = 1; a.types = {0}; }
    if (a.el.aniso)
      for (int t : a.types)
        if (t == SFG_SEIS_PRESSURE) {
          h->err = "pressure seismograms are defined for isotropic media only";
          return int(SFG_ERR_UNSUPPORTED);
        }
    for (int t : a.types)
      if (t >= SFG_SEIS_ROTATION && !a.el.cosserat) {
        h->err = "rotation, intrinsic rotation and curl seismograms need a Cosserat medium";
        return int(SFG_ERR_UNSUPPORTED);
      }
    a.nsig = (a.nstep + a.nsb - 1) / a.nsb;
    SFG_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    SFG_CUDA(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
    SFG_CUDA(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    SFG_CUDA(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    SFG_CUDA(cudaEventCreate(&h->ev0));
    SFG_CUDA(cudaEventCreate(&h->ev1));
    for (int i = 0; i < sfg::NPTS; ++i) { h->quad.hp[i] = a.hprime[i]; h->quad.hpw[i] = a.hpw[i]; }
    for (int i = 0; i < sfg::NGLL; ++i) h->quad.w[i] = a.wgll[i];
    upload_medium(h, a.el, h->el);
    upload_medium(h, a.ac, h->ac);
    if (h->el.nspec) h->el.src_head = h->mem.upload(a.el_src_head);
    if (h->ac.nspec) h->ac.src_head = h->mem.upload(a.ac_src_head);
    h->d_src_next = h->mem.upload(a.src_next);
    h->d_src_shot = h->mem.upload(a.src_shot);
    SFG_CUDA(cudaMemcpyToSymbol(sfg::dev::c_hp, a.hprime, sizeof(a.hprime)));
    SFG_CUDA(cudaMemcpyToSymbol(sfg::dev::c_hpw, a.hpw, sizeof(a.hpw)));
    SFG_CUDA(cudaMemcpyToSymbol(sfg::dev::c_w, a.wgll, sizeof(a.wgll)));
    h->d_src_arr = h->mem.upload(a.src_arr);
    h->d_src_arr2 = a.src_arr2.empty() ? nullptr : h->mem.upload(a.src_arr2);
    h->d_stf = h->mem.upload(a.stf);
    h->d_rec_elem = h->mem.upload(a.rec_elem);
    h->d_rec_h = h->mem.upload(a.rec_h);
    std::vector<int> rl_el, rl_ac;
    for (int r = 0; r < a.nrec; ++r) (a.rec_medium[r] == 1 ? rl_el : rl_ac).push_back(r);
    h->el.rec_list = h->mem.upload(rl_el);
    h->el.nrec = int(rl_el.size());
    h->ac.rec_list = h->mem.upload(rl_ac);
    h->ac.nrec = int(rl_ac.size());
    h->d_seis = h->mem.zeros<float>(size_t(a.nshots) * a.nsig * a.ntypes * std::max(a.nrec, 1) * 2);
    h->d_step = h->mem.zeros<int>(1);
    h->d_flag = h->mem.zeros<int>(1);
    SFG_CUDA(cudaDeviceSynchronize());
    {
      int dev = 0;
      SFG_CUDA(cudaGetDevice(&dev));
      SFG_CUDA(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, dev));
    }
    {
      // interface points paired one to one, one shot, P-SV: fused updates
      const sfg::MediumData &E = a.el, &C = a.ac;
      bool ok = E.nspec && C.nspec && a.nshots == 1 && E.ncomp == 2 && E.niface == C.niface &&
                E.cp_start.empty() && C.cp_start.empty();
      for (int i = 0; ok && i < E.niface; ++i) {
        const int j = E.cp_other[i];
        ok = j >= 0 && j < C.niface && C.cp_other[j] == i;
      }
      h->fuse_ok = ok;
    }
    h->tile_ok = compute_tile_ok(h);
    if (h->tile_ok) upload_tiles(h);
    h->btile_ok = compute_btile_ok(h);
    if (h->btile_ok) upload_btiles(h);
    autotune(h);
    h->graph_steps = std::max(1, h->opt.steps_per_graph);
    h->graph_k = capture(h, h->graph_steps, true);
    h->graph_1 = capture(h, 1, true);
    h->graph_e = capture(h, 1, false);
    h->initialized = true;
    return int(SFG_OK);
  });
}

int sfg_step(sfg_handle *h) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    resume(h);
    enqueue_step(h, h->stream, false);
    h->state_final = true;
    SFG_CUDA(cudaGetLastError());
    ++h->host_step;
    return int(SFG_OK);
  });
}

int sfg_run(sfg_handle *h, int nsteps) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    if (nsteps < 0) return int(SFG_ERR_ARG);
    run_steps(h, nsteps);
    return int(SFG_OK);
  });
}

int sfg_synchronize(sfg_handle *h) {
  return guarded(h, [&]() {
    if (h->stream) SFG_CUDA(cudaStreamSynchronize(h->stream));
    return int(SFG_OK);
  });
}

int sfg_reset_fields(sfg_handle *h) {
  return guarded(h, [&]() {
    if (!h->initialized) return int(SFG_ERR_STATE);
    for (DevMedium *D : {&h->el, &h->ac}) {
      if (!D->nspec) continue;
      const size_t n = (D->values() + 4) * sizeof(float);
      SFG_CUDA(cudaMemsetAsync(D->u, 0, n, h->stream));
      SFG_CUDA(cudaMemsetAsync(D->v, 0, n, h->stream));
      SFG_CUDA(cudaMemsetAsync(D->accum, 0, n, h->stream));
      SFG_CUDA(cudaMemsetAsync(D->a, 0, n, h->stream));
    }
    const sfg::Assembly2D &a = h->asmb;
    SFG_CUDA(cudaMemsetAsync(h->d_seis, 0,
                             size_t(a.nshots) * a.nsig * a.ntypes * std::max(a.nrec, 1) * 2 * sizeof(float),
                             h->stream));
    SFG_CUDA(cudaMemsetAsync(h->d_step, 0, sizeof(int), h->stream));
    SFG_CUDA(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    SFG_CUDA(cudaStreamSynchronize(h->stream));
    h->host_step = 0;
    h->state_final = true;
    return int(SFG_OK);
  });
}

int sfg_run_timed(sfg_handle *h, int nsteps, float *ms) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    SFG_CUDA(cudaEventRecord(h->ev0, h->stream));
    run_steps(h, nsteps);
    SFG_CUDA(cudaEventRecord(h->ev1, h->stream));
    SFG_CUDA(cudaEventSynchronize(h->ev1));
    float t = 0;
    SFG_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
    if (ms) *ms = t;
    return int(SFG_OK);
  });
}

int sfg_run_timed_flushed(sfg_handle *h, int nsteps, size_t flush_bytes, float *ms) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    if (nsteps < 0) return int(SFG_ERR_ARG);
    const int batch = 256;
    std::vector<cudaEvent_t> ev(2 * batch);
    for (auto &e : ev) SFG_CUDA(cudaEventCreate(&e));
    double total = 0.0;
    int done = 0;
    resume(h);
    try {
      while (done < nsteps) {
        const int n = std::min(batch, nsteps - done);
        for (int i = 0; i < n; ++i) {
          if (flush_bytes) flush_l2(h, flush_bytes, i);
          SFG_CUDA(cudaEventRecord(ev[2 * i], h->stream));
          SFG_CUDA(cudaGraphLaunch(h->graph_1, h->stream));
          SFG_CUDA(cudaEventRecord(ev[2 * i + 1], h->stream));
        }
        SFG_CUDA(cudaStreamSynchronize(h->stream));
        for (int i = 0; i < n; ++i) {
          float t = 0;
          SFG_CUDA(cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]));
          total += t;
        }
        done += n;
        h->host_step += n;
      }
    } catch (...) {
      for (auto &e : ev) cudaEventDestroy(e);
      throw;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    // every timed step fused the next predictor: the fields are mid-step
    h->state_final = false;
    if (ms) *ms = float(total);
    return int(SFG_OK);
  });
}

int sfg_step_io(sfg_handle *h, const float *stf_row, float *seis_row) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    const sfg::Assembly2D &a = h->asmb;
    const int step = h->host_step;
    const int rowlen = a.ntypes * a.nrec * 2;
    const size_t io_bytes = 16 + 4 * size_t(a.nsrc) + 4 * size_t(a.nshots) * rowlen;
    if (!h->graph_io) {
      SFG_CUDA(cudaHostAlloc(&h->io_host, io_bytes, cudaHostAllocMapped));
      std::memset(h->io_host, 0, io_bytes);
      SFG_CUDA(cudaHostGetDevicePointer(&h->io_dev, h->io_host, 0));
      const int *io_d = static_cast<const int *>(h->io_dev);
      float *seis_d = reinterpret_cast<float *>(static_cast<char *>(h->io_dev) + 16 + 4 * size_t(a.nsrc));
      // one fused step (the next step's predictor applied in the update)
      // between the row copies; the step's seismograms are complete before
      // its update runs
      cudaGraph_t g = nullptr;
      SFG_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      k_io_in<<<1, 128, 0, h->stream>>>(io_d, h->d_stf, h->d_step, a.nsrc, a.nstep);
      enqueue_step(h, h->stream, true);
      if (a.nrec > 0)
        k_io_out<<<std::max(1, std::min(64, (a.nshots * rowlen + 255) / 256)), 256, 0, h->stream>>>(
            h->d_seis, seis_d, h->d_step, a.nsb, a.nsig, a.nshots, rowlen);
      SFG_CUDA(cudaStreamEndCapture(h->stream, &g));
      SFG_CUDA(cudaGraphInstantiate(&h->graph_io, g, 0));
      cudaGraphDestroy(g);
    }
    int *io = static_cast<int *>(h->io_host);
    io[0] = 0;
    if (stf_row && a.nsrc > 0 && step < a.nstep) {
      // the table stores the acoustic (pressure) sign convention already applied
      float *row = reinterpret_cast<float *>(io + 4);
      for (int s = 0; s < a.nsrc; ++s) row[s] = a.src_medium[s] == 0 ? -stf_row[s] : stf_row[s];
      io[0] = 1;
    }
    std::atomic_thread_fence(std::memory_order_seq_cst);
    resume(h);
    SFG_CUDA(cudaGraphLaunch(h->graph_io, h->stream));
    h->state_final = false;
    ++h->host_step;
    SFG_CUDA(cudaStreamSynchronize(h->stream));
    if (seis_row && a.nrec > 0 && step % a.nsb == 0 && step / a.nsb < a.nsig)
      std::memcpy(seis_row, static_cast<char *>(h->io_host) + 16 + 4 * size_t(a.nsrc),
                  sizeof(float) * size_t(a.nshots) * rowlen);
    return int(SFG_OK);
  });
}

int sfg_time_kernel(sfg_handle *h, int which, int iters, float *ms) {
  return sfg_time_kernel_flushed(h, which, iters, 0, ms);
}

int sfg_time_kernel_flushed(sfg_handle *h, int which, int iters, size_t flush_bytes, float *ms) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    if (iters <= 0 || which < 0 || which > 3) return int(SFG_ERR_ARG);
    const int medium = which == 2 ? SFG_MEDIUM_ACOUSTIC : SFG_MEDIUM_ELASTIC;
    DevMedium &D = medium == SFG_MEDIUM_ELASTIC ? h->el : h->ac;
    if (which != 0 && D.nspec == 0) { if (ms) *ms = 0; return int(SFG_OK); }
    auto launch = [&]() {
      if (h->variant == 5) {
        // fused tile kernel: 0 the tile kernel, 1 the boundary points, 3 receivers
        if (which == 0) launch_tile_kernel(h, true, h->stream);
        else if (which == 1) launch_tile_boundary(h, true, h->stream);
        else if (which == 3) launch_tile_receivers(h, h->stream);
        return;
      }
      if (h->variant == 7) {
        // batched tiles: 0 the tile kernel, 1 the shared points, 3 receivers
        if (which == 0) launch_btile(h, true, h->stream);
        else if (which == 1) launch_btile_shared(h, true, h->stream);
        else if (which == 3) launch_receivers(h, SFG_MEDIUM_ELASTIC, h->stream);
        return;
      }
      if (which == 0) launch_stiffness(h, h->stream);
      else if (which == 3) { launch_receivers(h, SFG_MEDIUM_ACOUSTIC, h->stream);
                             launch_receivers(h, SFG_MEDIUM_ELASTIC, h->stream); }
      else launch_update(h, medium, true, false, h->stream);
    };
    h->state_final = false;
    for (int i = 0; i < 3; ++i) launch();
    float t = 0;
    if (flush_bytes == 0) {
      // back to back
      SFG_CUDA(cudaEventRecord(h->ev0, h->stream));
      for (int i = 0; i < iters; ++i) launch();
      SFG_CUDA(cudaEventRecord(h->ev1, h->stream));
      SFG_CUDA(cudaEventSynchronize(h->ev1));
      SFG_CUDA(cudaGetLastError());
      SFG_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
    } else {
      // each launch after an L2 flush (the cache holds none of its inputs)
      for (int i = 0; i < iters; ++i) {
        flush_l2(h, flush_bytes, i);
        SFG_CUDA(cudaEventRecord(h->ev0, h->stream));
        launch();
        SFG_CUDA(cudaEventRecord(h->ev1, h->stream));
        SFG_CUDA(cudaEventSynchronize(h->ev1));
        float ti = 0;
        SFG_CUDA(cudaEventElapsedTime(&ti, h->ev0, h->ev1));
        t += ti;
      }
      SFG_CUDA(cudaGetLastError());
    }
    if (ms) *ms = t / iters;
    return int(SFG_OK);
  });
}

int sfg_get_info(const sfg_handle *h, sfg_info *info) {
  if (!h || !info) return SFG_ERR_ARG;
  const sfg::Assembly2D &a = h->asmb;
  std::memset(info, 0, sizeof(*info));
  info->nspec = a.nspec;
  info->nspec_elastic = a.el.nspec;
  info->nspec_acoustic = a.ac.nspec;
  info->nglob = a.nglob;
  info->nglob_elastic = a.el.nglob;
  info->nglob_acoustic = a.ac.nglob;
  info->ncolors_elastic = a.el.color_start.empty() ? 0 : int(a.el.color_start.size()) - 1;
  info->ncolors_acoustic = a.ac.color_start.empty() ? 0 : int(a.ac.color_start.size()) - 1;
  info->nshots = a.nshots;
  info->nsig = a.nsig ? a.nsig : (a.nstep + a.nsb - 1) / a.nsb;
  info->nrec = a.nrec;
  info->ntypes = a.ntypes;
  info->nstep = a.nstep;
  info->istep = h->host_step;
  info->t0 = a.t0;
  info->device_bytes = h->mem.bytes;
  info->kernels_per_step = h->initialized ? kernels_per_step(h) : 0;
  info->elements_per_block = h->epb;
  info->kernel_variant = h->variant;
  info->ncomp_elastic = a.el.ncomp;
  return SFG_OK;
}

int sfg_get_seismograms(sfg_handle *h, float *out, size_t count) {
  return guarded(h, [&]() {
    if (!h->initialized) return int(SFG_ERR_STATE);
    const sfg::Assembly2D &a = h->asmb;
    const size_t n = size_t(a.nshots) * a.nsig * a.ntypes * a.nrec * 2;
    if (count < n || !out) { h->err = "output buffer too small"; return int(SFG_ERR_ARG); }
    if (n == 0) return int(SFG_OK);
    std::vector<float> raw(n);
    SFG_CUDA(cudaStreamSynchronize(h->stream));
    SFG_CUDA(cudaMemcpy(raw.data(), h->d_seis, n * sizeof(float), cudaMemcpyDeviceToHost));
    // receiver-angle rotation (seismogram_iterator.hpp:40-49)
    const float ca = std::cos(float(M_PI) / 180.f * float(a.rec_angle));
    const float sa = std::sin(float(M_PI) / 180.f * float(a.rec_angle));
    for (size_t i = 0; i < n; i += 2) {
      out[i] = ca * raw[i] - sa * raw[i + 1];
      out[i + 1] = sa * raw[i] + ca * raw[i + 1];
    }
    return int(SFG_OK);
  });
}

int sfg_get_field(sfg_handle *h, int medium, int which, float *out, size_t count) {
  return guarded(h, [&]() {
    if (!h->initialized) return int(SFG_ERR_STATE);
    DevMedium &D = medium == SFG_MEDIUM_ELASTIC ? h->el : h->ac;
    const size_t n = D.values();
    if (!out || count < n) { h->err = "output buffer too small"; return int(SFG_ERR_ARG); }
    if (!h->state_final) {
      h->err = "fields are mid-step after a timing call; run a step first";
      return int(SFG_ERR_STATE);
    }
    const float *src = which == 0 ? D.u : which == 1 ? D.v : D.a;
    if (n == 0) return int(SFG_OK);
    SFG_CUDA(cudaStreamSynchronize(h->stream));
    if (D.S == 1) {
      SFG_CUDA(cudaMemcpy(out, src, n * sizeof(float), cudaMemcpyDeviceToHost));
      return int(SFG_OK);
    }
    // device layout [point][comp][shot] -> [shot][point][comp]
    std::vector<float> tmp(n);
    SFG_CUDA(cudaMemcpy(tmp.data(), src, n * sizeof(float), cudaMemcpyDeviceToHost));
    const size_t pc = size_t(D.nglob) * D.ncomp;
    for (size_t k = 0; k < pc; ++k)
      for (int sh = 0; sh < D.S; ++sh) out[size_t(sh) * pc + k] = tmp[k * D.S + sh];
    return int(SFG_OK);
  });
}

int sfg_get_numbering(sfg_handle *h, int *ibool_global, int *g2e, int *g2a) {
  if (!h) return SFG_ERR_ARG;
  const sfg::Assembly2D &a = h->asmb;
  if (ibool_global) std::copy(a.ibool_global.begin(), a.ibool_global.end(), ibool_global);
  if (g2e) std::copy(a.glob_to_el.begin(), a.glob_to_el.end(), g2e);
  if (g2a) std::copy(a.glob_to_ac.begin(), a.glob_to_ac.end(), g2a);
  return SFG_OK;
}

int sfg_get_geometry(sfg_handle *h, double *x, double *z, double *jac, int *medium) {
  if (!h) return SFG_ERR_ARG;
  const sfg::Assembly2D &a = h->asmb;
  if (x) std::copy(a.gx.begin(), a.gx.end(), x);
  if (z) std::copy(a.gz.begin(), a.gz.end(), z);
  if (jac) std::copy(a.jac_d.begin(), a.jac_d.end(), jac);
  if (medium) std::copy(a.mesh_medium.begin(), a.mesh_medium.end(), medium);
  return SFG_OK;
}

int sfg_check_finite(sfg_handle *h) {
  if (!h || !h->initialized) return 0;
  int f = 0;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return SFG_ERR_CUDA;
  if (cudaMemcpy(&f, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SFG_ERR_CUDA;
  if (f == 2) {
    h->err = "an element kernel gave up waiting for its staged element data";
    return SFG_ERR_CUDA;
  }
  return f ? SFG_ERR_NONFINITE : 0;
}

int sfg_step_noalloc(sfg_handle *h, int istep, float *u, float *v, float *a) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    if (h->ac.nspec != 0 || h->el.nspec == 0 || h->el.S != 1 || h->el.ncomp > 2 || h->el.aniso) {
      h->err = "sfg_step_noalloc advances single-shot, single-medium isotropic elastic (P-SV or SH) models only";
      return int(SFG_ERR_UNSUPPORTED);
    }
    if (!u || !v || !a || istep < 0) { h->err = "null field pointer or negative step"; return int(SFG_ERR_ARG); }
    const size_t n = size_t(h->el.nglob) * h->el.ncomp;
    if (n > NOALLOC_MAX_VALUES) {
      h->err = "sfg_step_noalloc: the model has " + std::to_string(n) +
               " point values, above the fixed scratch of " + std::to_string(NOALLOC_MAX_VALUES);
      return int(SFG_ERR_ARG);
    }
    // the kernels read and write the fields as float2 / float4 vectors
    for (const float *p : {u, v, a})
      if (reinterpret_cast<uintptr_t>(p) % 16 != 0) {
        h->err = "sfg_step_noalloc: u, v and a must start on a 16-byte boundary";
        return int(SFG_ERR_ARG);
      }
    NoallocDevice nd;
    const int rc = noalloc_device(nd, h->err);
    if (rc != SFG_OK) return rc;
    cudaStream_t s = h->stream;
    // the caller's fields replace the handle's, the fixed array its accumulator
    DevMedium el = h->el;
    el.u = u;
    el.v = v;
    el.a = a;
    el.accum = nd.accum;
    SFG_CUDA(cudaMemsetAsync(nd.accum, 0, (n + 4) * sizeof(float), s));
    const int words[2] = {istep, 0};
    SFG_CUDA(cudaMemcpyAsync(nd.words, words, sizeof(words), cudaMemcpyHostToDevice, s));
    // predictor, element launches, corrector: the kernels of sfg_step
    launch_predict_medium(h, el, s);
    // colour passes into the fixed accumulator (every launch shape gives the same bits)
    launch_stiffness(h, el, h->ac, nd.words, s, h->variant == 2 ? 2 : 1);
    sfg::dev::UpdateArgs U = update_args(h, el, h->ac, SFG_MEDIUM_ELASTIC, false, false);
    U.inv_start = nullptr;
    U.r = nullptr;
    U.a_store = a;
    U.flag = nd.words + 1;
    U.step = nd.words;
    sfg::dev::k_update<<<grid_for(U.n / 4), 256, 0, s>>>(U);
    SFG_CUDA(cudaGetLastError());
    SFG_CUDA(cudaStreamSynchronize(s));
    // the update's non-finite flag lives in the fixed words: read it back
    int flag = 0;
    SFG_CUDA(cudaMemcpy(&flag, nd.words + 1, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
      h->err = "sfg_step_noalloc: the displacement became NaN or Inf";
      return int(SFG_ERR_NONFINITE);
    }
    return int(SFG_OK);
  });
}

// ------------------------------------------------- step-wise interface ---
// The granularity of the reference's kernel facade: Newmark predictor and
// corrector phases per medium (newmark.tpp:10-128), update_wavefields per
// medium (domain_kernels.hpp:72-141: coupling, sources, stiffness, division
// by the mass matrix) and compute_seismograms (:189-203).  They run the
// owner-computes element kernel restricted to one medium and keep the fields
// in the reference's phase states, so a host loop that calls them in the
// reference's order reproduces sfg_run bit for bit.

int sfg_predictor(sfg_handle *h, int medium) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    if (h->asmb.nshots != 1) { h->err = "the step-wise interface runs single-shot handles"; return int(SFG_ERR_UNSUPPORTED); }
    if (medium != SFG_MEDIUM_ACOUSTIC && medium != SFG_MEDIUM_ELASTIC) return int(SFG_ERR_ARG);
    if (!h->state_final) { h->err = "fields are mid-step; end the run with sfg_step first"; return int(SFG_ERR_STATE); }
    DevMedium &D = medium == SFG_MEDIUM_ELASTIC ? h->el : h->ac;
    if (D.nspec == 0) return 0;
    launch_predict_medium(h, D, h->stream);
    SFG_CUDA(cudaMemsetAsync(D.a, 0, D.values() * sizeof(float), h->stream));
    SFG_CUDA(cudaGetLastError());
    return int(D.values());
  });
}

int sfg_update_wavefields(sfg_handle *h, int medium, int istep) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    if (h->asmb.nshots != 1) { h->err = "the step-wise interface runs single-shot handles"; return int(SFG_ERR_UNSUPPORTED); }
    if ((medium != SFG_MEDIUM_ACOUSTIC && medium != SFG_MEDIUM_ELASTIC) || istep < 0) return int(SFG_ERR_ARG);
    DevMedium &D = medium == SFG_MEDIUM_ELASTIC ? h->el : h->ac;
    DevMedium &O = medium == SFG_MEDIUM_ELASTIC ? h->ac : h->el;
    if (D.nspec == 0) return 0;
    cudaStream_t s = h->stream;
    sfg::dev::k_set_step<<<1, 1, 0, s>>>(h->d_step, istep);
    // element contributions of this medium only (sources and Stacey in the epilogue)
    const DevMedium none{};
    if (medium == SFG_MEDIUM_ELASTIC) launch_stiffness(h, h->el, none, h->d_step, s, 3);
    else launch_stiffness(h, none, h->ac, h->d_step, s, 3);
    // coupling and division by the mass matrix: a stored for the corrector
    sfg::dev::UpdateArgs U = update_args(h, D, O, medium, false, false);
    U.inv_start = D.inv_start;
    U.r = D.r;
    U.a_store = D.a;
    const int npts = int(D.values()) / D.ncomp;
    switch (D.ncomp) {
      case 1: sfg::dev::k_accel_gather<1><<<grid_for(npts), 256, 0, s>>>(U); break;
      case 2: sfg::dev::k_accel_gather<2><<<grid_for(npts), 256, 0, s>>>(U); break;
      case 3: sfg::dev::k_accel_gather<3><<<grid_for(npts), 256, 0, s>>>(U); break;
      default: sfg::dev::k_accel_gather<4><<<grid_for(npts), 256, 0, s>>>(U); break;
    }
    SFG_CUDA(cudaGetLastError());
    return D.nspec;
  });
}

int sfg_corrector(sfg_handle *h, int medium) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    if (h->asmb.nshots != 1) { h->err = "the step-wise interface runs single-shot handles"; return int(SFG_ERR_UNSUPPORTED); }
    if (medium != SFG_MEDIUM_ACOUSTIC && medium != SFG_MEDIUM_ELASTIC) return int(SFG_ERR_ARG);
    DevMedium &D = medium == SFG_MEDIUM_ELASTIC ? h->el : h->ac;
    if (D.nspec == 0) return 0;
    const int n = int(D.values());
    sfg::dev::k_correct<<<grid_for(n), 256, 0, h->stream>>>(D.v, D.a, n, float(h->asmb.dt) / 2.0f);
    SFG_CUDA(cudaGetLastError());
    return n;
  });
}

int sfg_compute_seismograms(sfg_handle *h, int isig) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg_initialize first"; return int(SFG_ERR_STATE); }
    if (h->asmb.nshots != 1) { h->err = "the step-wise interface runs single-shot handles"; return int(SFG_ERR_UNSUPPORTED); }
    if (isig < 0 || isig >= h->asmb.nsig) { h->err = "seismogram sample index out of range"; return int(SFG_ERR_ARG); }
    for (int medium : {SFG_MEDIUM_ACOUSTIC, SFG_MEDIUM_ELASTIC}) {
      const DevMedium &D = medium == SFG_MEDIUM_ELASTIC ? h->el : h->ac;
      if (D.nspec == 0 || D.nrec == 0) continue;
      sfg::dev::RecArgs R = rec_args(h, medium);
      R.final_fields = 1;
      R.isig_fixed = isig;
      sfg::dev::k_receivers<<<D.nrec, 32, 0, h->stream>>>(R);
    }
    SFG_CUDA(cudaGetLastError());
    return int(SFG_OK);
  });
}

// ---------------------------------------------------------------- adjoint ---

int sfg_set_model2d(sfg_handle *h, const float *rho, const float *kappa, const float *mu) {
  return guarded(h, [&]() {
    if (!rho || !kappa || !mu) return int(SFG_ERR_ARG);
    sfg::set_model2d(h->mesh, h->asmb, rho, kappa, mu);
    // pressure sources in acoustic elements carry l / kappa: rebuild them
    const bool ac_src = h->have_sources && h->asmb.ac.nspec > 0 && h->asmb.nsrc > 0;
    if (ac_src) sfg::set_sources2d(h->mesh, h->asmb, h->sources);
    if (h->initialized) {
      if (ac_src)
        SFG_CUDA(cudaMemcpy(h->d_src_arr, h->asmb.src_arr.data(), h->asmb.src_arr.size() * sizeof(float),
                            cudaMemcpyHostToDevice));
      for (int med = 0; med < 2; ++med) {
        const sfg::MediumData &M = med == 1 ? h->asmb.el : h->asmb.ac;
        DevMedium &D = med == 1 ? h->el : h->ac;
        if (!D.nspec) continue;
        auto put = [&](float *d, const std::vector<float> &v) {
          if (d && !v.empty()) SFG_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice));
        };
        put(D.prop0, M.prop0); put(D.prop1, M.prop1);
        put(D.bc_imp0, M.bc_imp0); put(D.bc_imp1, M.bc_imp1);
        put(D.minv, M.minv);
      }
      refresh_tile_records(h);
      if (h->adj.st_c && !h->asmb.el.stacey_c.empty())
        SFG_CUDA(cudaMemcpy(h->adj.st_c, h->asmb.el.stacey_c.data(), h->asmb.el.stacey_c.size() * sizeof(float),
                            cudaMemcpyHostToDevice));
      h->adj.forward_done = false;
    }
    return int(SFG_OK);
  });
}

}  // extern "C"

namespace {

// The medium of an adjoint run: the model has exactly one.
DevMedium &adj_dev(sfg_handle *h) { return h->el.nspec ? h->el : h->ac; }
const sfg::MediumData &adj_data(const sfg_handle *h) { return h->el.nspec ? h->asmb.el : h->asmb.ac; }
bool adj_acoustic(const sfg_handle *h) { return h->el.nspec == 0; }

// A coupled model's two interface point lists pair one to one (conforming
// edges): every acoustic interface point p has the elastic partner q =
// ac.cp_other[p] whose partner is p again.
bool conforming_pairs(const sfg::Assembly2D &a) {
  const sfg::MediumData &E = a.el, &A = a.ac;
  if (!E.cp_start.empty() || !A.cp_start.empty() || E.niface != A.niface) return false;
  for (int p = 0; p < A.niface; ++p) {
    const int q = A.cp_other[p];
    if (q < 0 || q >= E.niface || E.cp_other[q] != p) return false;
  }
  return true;
}

int adjoint_checks(sfg_handle *h) {
  if (!h->initialized) { h->err = "sfg_initialize first"; return SFG_ERR_STATE; }
  const sfg::Assembly2D &a = h->asmb;
  if (h->el.nspec > 0 && h->ac.nspec > 0) {
    // coupled acoustic-elastic model: isotropic P-SV, conforming interfaces,
    // displacement seismograms at elastic receivers or pressure seismograms
    // at acoustic receivers
    bool ok = !h->el.aniso && h->el.ncomp == 2 && h->el.S == 1 && a.nsb == 1 && a.ntypes == 1 &&
              conforming_pairs(a) &&
              (a.types[0] == SFG_SEIS_DISPLACEMENT || a.types[0] == SFG_SEIS_PRESSURE);
    const int rec_medium = ok && a.types[0] == SFG_SEIS_PRESSURE ? SFG_MEDIUM_ACOUSTIC : SFG_MEDIUM_ELASTIC;
    for (int r = 0; ok && r < a.nrec; ++r) ok = a.rec_medium[r] == rec_medium;
    if (!ok) {
      h->err = "the coupled adjoint needs isotropic elastic P-SV and acoustic media with conforming interfaces, "
               "one shot, seismograms sampled every step: displacement at receivers in the elastic medium or "
               "pressure at receivers in the acoustic medium";
      return SFG_ERR_UNSUPPORTED;
    }
    h->adj_coupled = true;
    return SFG_OK;
  }
  const int want = h->el.nspec ? SFG_SEIS_DISPLACEMENT : SFG_SEIS_PRESSURE;
  if (h->el.aniso || h->el.ncomp >= 3 || adj_dev(h).S != 1 || a.nsb != 1 || a.ntypes != 1 || a.types[0] != want) {
    h->err = "the adjoint needs one medium (isotropic elastic P-SV or SH with displacement seismograms, "
             "or acoustic with pressure seismograms) or a coupled pair, one shot, seismograms sampled every step";
    return SFG_ERR_UNSUPPORTED;
  }
  h->adj_coupled = false;
  return SFG_OK;
}

template <typename T>
T *dalloc(size_t n) {
  T *p = nullptr;
  SFG_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  SFG_CUDA(cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T)));
  return p;
}

// Sizes of one medium's adjoint arrays.
void adj_medium_sizes(AdjointState &A, const DevMedium &D, const sfg::MediumData &M) {
  A.nvals = D.values();
  A.nloc = size_t(D.nspec) * sfg::NPTS;
  A.stride = ((A.nvals + 3) / 4) * 4 + 4;
  A.nglob = size_t(D.nglob);
  A.vstride = ((2 * M.stacey_pt.size() + 3) / 4) * 4 + 4;
}

size_t adj_segment_bytes(const AdjointState &A, int interval) {
  return size_t(interval) * (2 * A.stride + A.vstride) * sizeof(float);
}

// Checkpoints and segment buffers of one medium.
void adj_medium_segments(AdjointState &A, int ncheck, int nbuf, int interval) {
  for (float **p : {&A.ckpt, &A.seg_u, &A.seg_a, &A.seg_v})
    if (*p) { cudaFree(*p); *p = nullptr; }
  A.ckpt = dalloc<float>(size_t(ncheck) * 3 * (A.nvals + 4));
  A.seg_u = dalloc<float>(size_t(nbuf) * interval * A.stride);
  A.seg_a = dalloc<float>(size_t(nbuf) * interval * A.stride);
  A.seg_v = dalloc<float>(size_t(nbuf) * interval * A.vstride);
}

template <typename T>
T *dupload(const std::vector<T> &v) {
  T *p = dalloc<T>(v.size());
  if (!v.empty()) SFG_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return p;
}

// One medium's sweep state (once per handle): adjoint fields, element-point
// results, gradient sums, the element-local Stacey points, receivers as
// adjoint sources (displacement: per element chain; pressure: per point
// CSR), the acoustic sources' columns and, in a coupled model, the
// transposed coupling of the interface points.
void adj_medium_init(sfg_handle *h, AdjointState &A, const DevMedium &D, const sfg::MediumData &M, int medium) {
  const sfg::Assembly2D &as = h->asmb;
  const bool acoustic = medium == SFG_MEDIUM_ACOUSTIC;
  const size_t nvals = A.nvals, nloc = A.nloc;
  A.lu = dalloc<float>(nvals + 4); A.lv = dalloc<float>(nvals + 4); A.mu = dalloc<float>(nvals + 4);
  A.r = dalloc<float>(2 * nloc);
  // element-local Stacey points: global point, Stacey slot, geometry
  std::unordered_map<int, int> slot;
  for (size_t j = 0; j < M.stacey_pt.size(); ++j) slot[M.stacey_pt[j]] = int(j);
  std::vector<int> lg, lj;
  std::vector<float> geo;
  A.lb_k.clear();
  A.lb_pm.clear();
  for (int ce = 0; ce < M.nspec; ++ce) {
    if (M.bc_slot[ce] < 0) continue;
    for (int q = 0; q < sfg::NPTS; ++q) {
      const size_t k = size_t(M.bc_slot[ce]) * sfg::NPTS + q;
      if (M.bc_w[k] == 0.0f) continue;
      const int g = M.ibool[size_t(ce) * sfg::NPTS + q];
      lg.push_back(g);
      lj.push_back(slot.at(g));
      // P-SV: the normal; SH and acoustic: x is the free-surface mask (1 in SH)
      geo.insert(geo.end(), {M.ncomp == 2 ? M.bc_nx[k] : M.bc_keep[k], M.bc_nz[k], M.bc_j1[k], M.bc_w[k]});
      A.lb_k.push_back(k);
      A.lb_pm.push_back(size_t(M.elem_mesh[ce]) * sfg::NPTS + q);
    }
  }
  A.nlb = int(lg.size());
  A.off_lb = ((2 * nloc + A.nglob + 3) / 4) * 4;
  // acoustic sources (their STF columns)
  A.src_list.clear();
  if (acoustic)
    for (int si = 0; si < as.nsrc; ++si)
      if (as.src_medium[si] == SFG_MEDIUM_ACOUSTIC) A.src_list.push_back(si);
  A.nsrc_t = int(A.src_list.size());
  A.src_ce = dalloc<int>(std::max(A.nsrc_t, 1));
  A.src_id = dupload(A.src_list);
  A.lb_g = dupload(lg); A.lb_j = dupload(lj); A.lb_geo = dupload(geo);
  A.sum = dalloc<float>(A.nsum()); A.comp = dalloc<float>(A.nsum()); A.seg = dalloc<float>(A.nsum());
  // displacement receivers of this medium as adjoint sources: chain per
  // compute element
  const bool disp = as.ntypes > 0 && as.types[0] == SFG_SEIS_DISPLACEMENT;
  std::vector<int> head(D.nspec, -1), next(std::max(as.nrec, 1), -1);
  for (int r = 0; r < as.nrec; ++r) {
    if (!disp || as.rec_medium[r] != medium) continue;
    next[r] = head[as.rec_elem[r]];
    head[as.rec_elem[r]] = r;
  }
  A.ad_head = dupload(head);
  A.ad_next = dupload(next);
  // pressure receivers (acoustic): points they touch, with receiver and weight
  A.pressure = acoustic && as.ntypes > 0 && as.types[0] == SFG_SEIS_PRESSURE;
  if (A.pressure) {
    std::vector<std::vector<std::pair<int, float>>> by_pt(D.nglob);
    for (int r = 0; r < as.nrec; ++r) {
      if (as.rec_medium[r] != SFG_MEDIUM_ACOUSTIC) continue;
      for (int q = 0; q < sfg::NPTS; ++q) {
        const float hq = as.rec_h[size_t(r) * sfg::NPTS + q];
        if (hq != 0.0f) by_pt[M.ibool[size_t(as.rec_elem[r]) * sfg::NPTS + q]].push_back({r, hq});
      }
    }
    std::vector<int> pt, start{0}, rr;
    std::vector<float> hw;
    for (int g = 0; g < D.nglob; ++g) {
      if (by_pt[g].empty()) continue;
      pt.push_back(g);
      for (auto &[r, hq] : by_pt[g]) { rr.push_back(r); hw.push_back(hq); }
      start.push_back(int(rr.size()));
    }
    A.nps = int(pt.size());
    A.ps_pt = dupload(pt); A.ps_start = dupload(start); A.ps_rec = dupload(rr); A.ps_h = dupload(hw);
  }
  A.nst = int(M.stacey_pt.size());
  A.st_pt = dupload(M.stacey_pt);
  A.st_c = dupload(M.stacey_c);
  if (h->adj_coupled) {
    // partner of each interface point and the partner side's normal
    const sfg::MediumData &O = acoustic ? as.el : as.ac;
    std::vector<int> other(M.niface);
    std::vector<float> nx(M.niface), nz(M.niface);
    for (int i = 0; i < M.niface; ++i) {
      other[i] = M.cp_other[i];
      nx[i] = O.cp_nx[other[i]];
      nz[i] = O.cp_nz[other[i]];
    }
    A.cp_other = dupload(other); A.cp_nx = dupload(nx); A.cp_nz = dupload(nz);
  }
  A.d_rec = dalloc<sfg::dev::SegRecord>(1);
}

void adj_write_record(AdjointState &A) {
  sfg::dev::SegRecord rec{A.seg_u, A.seg_a, A.stride, 0, A.seg_v, A.vstride, A.st_pt, A.nst, 0};
  SFG_CUDA(cudaMemcpy(A.d_rec, &rec, sizeof(rec), cudaMemcpyHostToDevice));
}

void adjoint_alloc(sfg_handle *h, int nstep, int interval) {
  AdjointState &A = h->adj;
  AdjointState &A2 = h->adj2;
  const bool cpl = h->adj_coupled;
  const DevMedium &D = adj_dev(h);
  const int ncheck = (nstep + interval - 1) / interval;
  const size_t old_nvals = A.nvals;
  const size_t old_bytes = A.seg_u ? size_t(A.nbuf) * (adj_segment_bytes(A, A.interval) +
                                                       (A2.seg_u ? adj_segment_bytes(A2, A.interval) : 0)) : 0;
  adj_medium_sizes(A, D, adj_data(h));
  if (cpl) adj_medium_sizes(A2, h->ac, h->asmb.ac);
  // segment buffers: as many as the budget holds (default: 75% of the device
  // memory free before they are allocated), at least 2, at most ncheck
  const size_t seg_bytes = adj_segment_bytes(A, interval) + (cpl ? adj_segment_bytes(A2, interval) : 0);
  size_t budget = A.budget;
  if (budget == 0) {
    size_t fr = 0, tot = 0;
    SFG_CUDA(cudaMemGetInfo(&fr, &tot));
    budget = size_t(0.75 * double(fr + old_bytes));
  }
  const int nbuf = int(std::max<size_t>(2, std::min<size_t>(size_t(std::max(ncheck, 2)), budget / seg_bytes)));
  if (old_nvals != A.nvals || A.interval != interval || A.ncheck < ncheck || A.nbuf != nbuf ||
      (cpl && !A2.seg_u)) {
    adj_medium_segments(A, ncheck, nbuf, interval);
    if (cpl) adj_medium_segments(A2, ncheck, nbuf, interval);
    A.rec_from = -1;
    if (A.graph_rseg) { cudaGraphExecDestroy(A.graph_rseg); A.graph_rseg = nullptr; }
    for (cudaGraphExec_t &g : A.graph_rev)
      if (g) cudaGraphExecDestroy(g);
    A.graph_rev.assign(nbuf, nullptr);
    for (auto *ev : {&A.ev_rec, &A.ev_rev}) {
      for (cudaEvent_t e : *ev)
        if (e) cudaEventDestroy(e);
      ev->assign(nbuf, nullptr);
      for (cudaEvent_t &e : *ev) SFG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    A.nbuf = nbuf;
  }
  for (AdjointState *X : {&A, &A2}) {
    X->interval = interval;
    X->ncheck = ncheck;
    X->nstep = nstep;
    X->nbuf = nbuf;
  }
  if (!A.lu) {
    adj_medium_init(h, A, D, adj_data(h), h->el.nspec ? SFG_MEDIUM_ELASTIC : SFG_MEDIUM_ACOUSTIC);
    A.d_k0 = dalloc<int>(1);
    SFG_CUDA(cudaStreamCreateWithFlags(&A.rstream, cudaStreamNonBlocking));
  }
  if (cpl && !A2.lu) adj_medium_init(h, A2, h->ac, h->asmb.ac, SFG_MEDIUM_ACOUSTIC);
  adj_write_record(A);
  if (cpl) adj_write_record(A2);
  if (!A.graph_r1) {
    // one recording step with the next predictor fused, and one ending on
    // the corrector (the segment's last step)
    h->recording = 1;
    A.graph_r1 = capture(h, 1, true);
    A.graph_re = capture(h, 1, false);
    h->recording = 0;
  }
  if (!A.graph_rseg && interval > 1) {
    h->recording = 2;
    A.graph_rseg = capture(h, interval - 1, true);
    h->recording = 0;
  }
}

// Checkpoint c of every medium in the sweep: u, v, a at the segment's start.
void save_state(sfg_handle *h, int c) {
  for (int m = 0; m < (h->adj_coupled ? 2 : 1); ++m) {
    const AdjointState &A = m ? h->adj2 : h->adj;
    const DevMedium &D = m ? h->ac : adj_dev(h);
    const size_t n = D.values() + 4;
    float *dst = A.ckpt + size_t(c) * 3 * n;
    SFG_CUDA(cudaMemcpyAsync(dst, D.u, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    SFG_CUDA(cudaMemcpyAsync(dst + n, D.v, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    SFG_CUDA(cudaMemcpyAsync(dst + 2 * n, D.a, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
  }
}

// Segments held from the forward run (the last min(nbuf, ncheck)) and the
// buffer of segment c: a held segment has its own buffer; a recomputed one
// takes, alternately, the buffers of the last two held segments, which are
// the first the reverse sweep frees.
int held_from(const AdjointState &A) { return A.ncheck - std::min(A.nbuf, A.ncheck); }
int seg_buffer(const AdjointState &A, int c) {
  const int c_r = held_from(A), R = A.ncheck - c_r;
  if (c >= c_r) return c - c_r;
  return R - 1 - ((c_r - 1 - c) & 1);
}

// Recompute (or, in the forward run, compute: `seismograms`) segment c from
// the state in the fields, recording u~, a' and the Stacey v~ of each step
// into segment buffer b.  Stream-ordered on the handle's stream.
void record_segment(sfg_handle *h, int c, bool seismograms, int b) {
  AdjointState &A = h->adj;
  const int k0 = c * A.interval, k1 = std::min(k0 + A.interval, A.nstep);
  const size_t ob = size_t(b) * A.interval;
  sfg::dev::k_set_segment<<<1, 1, 0, h->stream>>>(A.d_rec, h->d_step, A.seg_u + ob * A.stride,
                                                  A.seg_a + ob * A.stride, A.seg_v + ob * A.vstride, k0);
  if (h->adj_coupled) {
    const AdjointState &A2 = h->adj2;
    sfg::dev::k_set_segment<<<1, 1, 0, h->stream>>>(A2.d_rec, h->d_step, A2.seg_u + ob * A2.stride,
                                                    A2.seg_a + ob * A2.stride, A2.seg_v + ob * A2.vstride, k0);
  }
  resume(h);
  if (!seismograms && k1 - k0 == A.interval && A.graph_rseg) {
    SFG_CUDA(cudaGraphLaunch(A.graph_rseg, h->stream));
  } else {
    for (int k = k0; k + 1 < k1; ++k) SFG_CUDA(cudaGraphLaunch(A.graph_r1, h->stream));
  }
  SFG_CUDA(cudaGraphLaunch(A.graph_re, h->stream));
  sfg::dev::k_set_step<<<1, 1, 0, h->stream>>>(h->d_step, k1);
  h->state_final = true;
  h->host_step = k1;
}

// Reverse sweep over one segment of n steps held in buffer b (slots n-1 ..
// 0), then the Kahan fold of its sums.  `last`: the run's final segment,
// whose final step starts from mu = 0 (no Stacey term) unless pressure
// seismograms set mu there.
template <int E, bool ROW = false>
void reverse_segment_E(sfg_handle *h, int b, int n, bool last, cudaStream_t rs) {
  AdjointState &A = h->adj;
  const DevMedium &D = adj_dev(h);
  const float dt = float(h->asmb.dt), dt2 = dt / 2.0f, dtsq2 = dt * dt / 2.0f;
  auto args = [&](AdjointState &X, const DevMedium &M) {
    sfg::dev::AdjArgs J{};
    J.ibool = M.ibool; J.xix = M.xix; J.xiz = M.xiz; J.gax = M.gax; J.gaz = M.gaz; J.jac = M.jac;
    J.prop0 = M.prop0; J.prop1 = M.prop1;
    J.mu = X.mu; J.r = X.r; J.pslot = M.slot; J.seg = X.seg;
    J.ad_head = X.ad_head; J.ad_next = X.ad_next; J.ad_h = h->d_rec_h;
    J.gtab = A.gtab; J.seg_k0 = A.d_k0; J.nrec = h->asmb.nrec;
    J.nspec = M.nspec;
    J.bc_slot = M.bc_slot; J.bc_keep = M.bc_keep;
    J.quad = h->quad;
    return J;
  };
  auto stacey_args = [&](AdjointState &X) {
    sfg::dev::AdjStaceyArgs St{};
    St.lb_g = X.lb_g; St.lb_j = X.lb_j; St.geo = reinterpret_cast<const float4 *>(X.lb_geo);
    St.mu = X.mu; St.acc = X.seg + X.off_lb; St.nlb = X.nlb;
    St.lv = X.lv; St.pt = X.st_pt; St.cm = X.st_c; St.nst = X.nst;
    St.nb_grad = grid_for(X.nlb);
    return St;
  };
  sfg::dev::AdjArgs J = args(A, D);
  sfg::dev::AdjStaceyArgs St = stacey_args(A);
  const int eblocks = (D.nspec + E - 1) / E;
  const size_t ob = size_t(b) * A.interval;
  auto psrc = [&](AdjointState &X, const DevMedium &M, int slot) {
    if (X.nps)
      sfg::dev::k_adj_psrc<<<std::min(grid_for(X.nps), 64), 128, 0, rs>>>(
          X.mu, M.minv, X.ps_pt, X.ps_start, X.ps_rec, X.ps_h, A.gtab, A.d_k0, slot, h->asmb.nrec, X.nps);
  };
  auto srcterm = [&](AdjointState &X, const DevMedium &M, int slot) {
    if (X.nsrc_t)
      sfg::dev::k_adj_srcterm<<<(X.nsrc_t * sfg::NPTS + 127) / 128, 128, 0, rs>>>(
          X.seg + X.off_src(), X.mu, M.ibool, X.src_ce, h->d_stf, A.d_k0, slot, X.nsrc_t, h->asmb.nstep,
          X.src_id, h->asmb.nsrc);
  };
  if (h->adj_coupled) {
    // coupled P-SV + acoustic step in reverse: both media's Stacey and
    // element terms with their own mu_k, then the elastic post (lu~ takes the
    // acoustic mu_k through the interface) and the acoustic post (its
    // adjoint acceleration takes the elastic mu_(k-1)), in that order
    AdjointState &C = h->adj2;
    const DevMedium &Ac = h->ac;
    sfg::dev::AdjArgs Ja = args(C, Ac);
    sfg::dev::AdjStaceyArgs Sa = stacey_args(C);
    const int ablocks = (Ac.nspec + E - 1) / E;
    const sfg::dev::AdjCoupling cp_el{A.cp_other, A.cp_nx, A.cp_nz, C.mu, D.niface};
    const sfg::dev::AdjCoupling cp_ac{C.cp_other, C.cp_nx, C.cp_nz, A.mu, Ac.niface};
    if (last && C.pressure) psrc(C, Ac, n - 1);
    for (int i = n - 1; i >= 0; --i) {
      const size_t sl = ob + size_t(i);
      if (A.nst) {
        St.vst = A.seg_v + sl * A.vstride;
        St.af = A.seg_a + sl * A.stride;
        sfg::dev::k_adj_stacey<2><<<St.nb_grad + grid_for(A.nst), 256, 0, rs>>>(St);
      }
      if (C.nst) {
        Sa.vst = C.seg_v + sl * C.vstride;
        Sa.af = C.seg_a + sl * C.stride;
        sfg::dev::k_adj_stacey<1><<<Sa.nb_grad + grid_for(C.nst), 256, 0, rs>>>(Sa);
      }
      J.uf = A.seg_u + sl * A.stride;
      J.slot = i;
      if (ROW) sfg::dev::k_adj_elem_row<32><<<(D.nspec + 31) / 32, sfg::dev::NG * 32, 0, rs>>>(J);
      else sfg::dev::k_adj_elem<E><<<eblocks, sfg::dev::NP * E, 0, rs>>>(J);
      Ja.uf = C.seg_u + sl * C.stride;
      Ja.slot = i;
      sfg::dev::k_adj_elem_ac<E><<<ablocks, sfg::dev::NP * E, 0, rs>>>(Ja);
      srcterm(C, Ac, i);
      sfg::dev::k_adj_post<2, true><<<grid_for(D.nglob), 256, 0, rs>>>(
          A.lu, A.lv, A.mu, A.seg + 2 * A.nloc, A.seg_a + sl * A.stride, D.minv, A.r, D.inv_start,
          D.nglob, dt, dt2, dtsq2, cp_el);
      sfg::dev::k_adj_post<1, true><<<grid_for(Ac.nglob), 256, 0, rs>>>(
          C.lu, C.lv, C.mu, C.seg + 2 * C.nloc, C.seg_a + sl * C.stride, Ac.minv, C.r, Ac.inv_start,
          Ac.nglob, dt, dt2, dtsq2, cp_ac);
      psrc(C, Ac, i - 1);
    }
    sfg::dev::k_kahan_fold<<<grid_for(int(A.nsum())), 256, 0, rs>>>(A.sum, A.comp, A.seg, int(A.nsum()));
    sfg::dev::k_kahan_fold<<<grid_for(int(C.nsum())), 256, 0, rs>>>(C.sum, C.comp, C.seg, int(C.nsum()));
    return;
  }
  if (last && A.pressure) psrc(A, D, n - 1);      // mu of the final step: B (-R^T g)
  for (int i = n - 1; i >= 0; --i) {
    const size_t sl = ob + size_t(i);
    const bool sh = D.ncomp == 1;
    if (A.nst && !(last && i == n - 1 && !A.pressure)) {
      St.vst = A.seg_v + sl * A.vstride;
      St.af = A.seg_a + sl * A.stride;
      if (sh) sfg::dev::k_adj_stacey<1><<<St.nb_grad + grid_for(A.nst), 256, 0, rs>>>(St);
      else sfg::dev::k_adj_stacey<2><<<St.nb_grad + grid_for(A.nst), 256, 0, rs>>>(St);
    }
    J.uf = A.seg_u + sl * A.stride;
    J.slot = i;
    if (A.pressure) {
      sfg::dev::k_adj_elem_ac<E><<<eblocks, sfg::dev::NP * E, 0, rs>>>(J);
      srcterm(A, D, i);
      sfg::dev::k_adj_post<1><<<grid_for(D.nglob), 256, 0, rs>>>(
          A.lu, A.lv, A.mu, A.seg + 2 * A.nloc, A.seg_a + sl * A.stride, D.minv, A.r, D.inv_start,
          D.nglob, dt, dt2, dtsq2);
      psrc(A, D, i - 1);                      // mu of the previous step gets its source
    } else if (sh) {
      sfg::dev::k_adj_elem_sh<E><<<eblocks, sfg::dev::NP * E, 0, rs>>>(J);
      sfg::dev::k_adj_post<1><<<grid_for(D.nglob), 256, 0, rs>>>(
          A.lu, A.lv, A.mu, A.seg + 2 * A.nloc, A.seg_a + sl * A.stride, D.minv, A.r, D.inv_start,
          D.nglob, dt, dt2, dtsq2);
    } else {
      if (ROW) sfg::dev::k_adj_elem_row<32><<<(D.nspec + 31) / 32, sfg::dev::NG * 32, 0, rs>>>(J);
      else sfg::dev::k_adj_elem<E><<<eblocks, sfg::dev::NP * E, 0, rs>>>(J);
      sfg::dev::k_adj_post<2><<<grid_for(D.nglob), 256, 0, rs>>>(
          A.lu, A.lv, A.mu, A.seg + 2 * A.nloc, A.seg_a + sl * A.stride, D.minv, A.r, D.inv_start,
          D.nglob, dt, dt2, dtsq2);
    }
  }
  sfg::dev::k_kahan_fold<<<grid_for(int(A.nsum())), 256, 0, rs>>>(A.sum, A.comp, A.seg, int(A.nsum()));
}

void reverse_segment(sfg_handle *h, int b, int n, bool last, cudaStream_t rs);

// Launch shape of the reverse element kernel: 8, 16 or 32 elements per block
// of the point form, or (code 1) the P-SV row form; each timed over a few
// launches on the live buffers (before the sums are cleared), the fastest
// kept.  All shapes give the same bits.  A forward kernel_variant fixed to 6
// fixes the row form, 1 to 5 the point form.
void tune_reverse(sfg_handle *h, cudaStream_t rs) {
  AdjointState &A = h->adj;
  if (A.epb) return;
  const bool row = adj_dev(h).ncomp == 2 && !A.pressure;
  if (row && h->opt.kernel_variant == 6) { A.epb = 1; return; }
  std::vector<int> cand{8, 16, 32};
  if (row && h->opt.kernel_variant == 0) cand.push_back(1);
  float best = 1e30f;
  A.epb = 8;
  for (int e : cand) {
    const int save = A.epb;
    A.epb = e;
    for (int rep = 0; rep < 2; ++rep) {
      if (rep == 1) SFG_CUDA(cudaEventRecord(h->ev0, rs));
      for (int i = 0; i < 3; ++i) reverse_segment(h, 0, 1, true, rs);
    }
    SFG_CUDA(cudaEventRecord(h->ev1, rs));
    SFG_CUDA(cudaEventSynchronize(h->ev1));
    float t = 0;
    SFG_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
    if (t < best) best = t;
    else A.epb = save;
  }
}

void reverse_segment(sfg_handle *h, int b, int n, bool last, cudaStream_t rs) {
  switch (h->adj.epb) {
    case 1: reverse_segment_E<32, true>(h, b, n, last, rs); break;
    case 16: reverse_segment_E<16>(h, b, n, last, rs); break;
    case 32: reverse_segment_E<32>(h, b, n, last, rs); break;
    default: reverse_segment_E<8>(h, b, n, last, rs); break;
  }
}

void restore_state(sfg_handle *h, int c) {
  for (int m = 0; m < (h->adj_coupled ? 2 : 1); ++m) {
    const AdjointState &A = m ? h->adj2 : h->adj;
    const DevMedium &D = m ? h->ac : adj_dev(h);
    const size_t n = D.values() + 4;
    const float *src = A.ckpt + size_t(c) * 3 * n;
    SFG_CUDA(cudaMemcpyAsync(D.u, src, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    SFG_CUDA(cudaMemcpyAsync(D.v, src + n, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    SFG_CUDA(cudaMemcpyAsync(D.a, src + 2 * n, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
  }
  h->state_final = true;
}

}  // namespace

extern "C" {

int sfg_forward_checkpointed(sfg_handle *h, int nsteps, int interval) {
  return guarded(h, [&]() {
    const int rc = adjoint_checks(h);
    if (rc != SFG_OK) return rc;
    if (nsteps <= 0 || nsteps > h->asmb.nstep || interval <= 0) {
      h->err = "need 0 < nsteps <= nstep and interval > 0";
      return int(SFG_ERR_ARG);
    }
    adjoint_alloc(h, nsteps, std::min(interval, nsteps));
    AdjointState &A = h->adj;
    const int ret = sfg_reset_fields(h);
    if (ret != SFG_OK) return ret;
    const int c_r = held_from(A);
    for (int c = 0; c < A.ncheck; ++c) {
      save_state(h, c);
      // the last nbuf segments are recorded on the way: the reverse sweep
      // recomputes only the earlier ones
      if (c >= c_r) record_segment(h, c, true, seg_buffer(A, c));
      else run_steps(h, std::min(A.interval, nsteps - c * A.interval));
    }
    SFG_CUDA(cudaStreamSynchronize(h->stream));
    A.rec_from = c_r;
    A.forward_done = true;
    return int(SFG_OK);
  });
}

int sfg_set_adjoint_budget(sfg_handle *h, size_t bytes) {
  return guarded(h, [&]() {
    h->adj.budget = bytes;
    return int(SFG_OK);
  });
}

int sfg_adjoint_buffers(sfg_handle *h) {
  return guarded(h, [&]() { return h->adj.seg_u ? h->adj.nbuf : 0; });
}

int sfg_adjoint_gradient(sfg_handle *h, const float *seis_grad, float *grad_rho, float *grad_kappa,
                         float *grad_mu) {
  return guarded(h, [&]() {
    const int rc = adjoint_checks(h);
    if (rc != SFG_OK) return rc;
    AdjointState &A = h->adj;
    if (!A.forward_done) { h->err = "run sfg_forward_checkpointed first"; return int(SFG_ERR_STATE); }
    if (!seis_grad) return int(SFG_ERR_ARG);
    const sfg::Assembly2D &as = h->asmb;
    const int nrec = as.nrec;
    cudaStream_t s = h->stream;
    // dL/d(seismogram) of every step on the device: [nstep][nrec][2]
    const size_t ng = std::max<size_t>(size_t(A.nstep) * nrec * 2, 1);
    if (ng > A.gtab_cap) {
      // the reverse-sweep graphs hold the table's address: drop them with it
      SFG_CUDA(cudaStreamSynchronize(s));
      if (A.rstream) SFG_CUDA(cudaStreamSynchronize(A.rstream));
      if (A.gtab) cudaFree(A.gtab);
      A.gtab = dalloc<float>(ng);
      A.gtab_cap = ng;
      for (cudaGraphExec_t &g : A.graph_rev)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }
    AdjointState &A2 = h->adj2;
    const bool cpl = h->adj_coupled;
    const size_t nstage = std::max({ng, A.nsum(), cpl ? A2.nsum() : size_t(0)});
    if (nstage > A.h_stage_cap) {
      if (A.h_stage) cudaFreeHost(A.h_stage);
      SFG_CUDA(cudaMallocHost(&A.h_stage, nstage * sizeof(float)));
      A.h_stage_cap = nstage;
    }
    if (nrec) {
      // the seismograms leave the library rotated by the receiver angle
      // (sfg_get_seismograms); the adjoint sources are rotated back
      float *g = A.h_stage;
      const float ca = std::cos(float(M_PI) / 180.f * float(as.rec_angle));
      const float sa = std::sin(float(M_PI) / 180.f * float(as.rec_angle));
      for (size_t i = 0; i + 1 < size_t(A.nstep) * nrec * 2; i += 2) {
        g[i] = ca * seis_grad[i] + sa * seis_grad[i + 1];
        g[i + 1] = -sa * seis_grad[i] + ca * seis_grad[i + 1];
      }
      SFG_CUDA(cudaMemcpyAsync(A.gtab, g, size_t(A.nstep) * nrec * 2 * sizeof(float), cudaMemcpyHostToDevice, s));
    }
    for (AdjointState *X : {&A, &A2}) {
      if (!X->nsrc_t || (X == &A2 && !cpl)) continue;
      // the acoustic sources' elements (they may have moved since the last call)
      X->src_ce_h.resize(X->nsrc_t);
      for (int j = 0; j < X->nsrc_t; ++j) X->src_ce_h[j] = as.src_elem[X->src_list[j]];
      SFG_CUDA(cudaMemcpyAsync(X->src_ce, X->src_ce_h.data(), X->nsrc_t * sizeof(int), cudaMemcpyHostToDevice, s));
    }
    tune_reverse(h, s);
    for (AdjointState *X : {&A, &A2}) {
      if (X == &A2 && !cpl) continue;
      for (float *p : {X->lu, X->lv, X->mu})
        SFG_CUDA(cudaMemsetAsync(p, 0, (X->nvals + 4) * sizeof(float), s));
      for (float *p : {X->sum, X->comp, X->seg})
        SFG_CUDA(cudaMemsetAsync(p, 0, X->nsum() * sizeof(float), s));
    }
    cudaStream_t rs = A.rstream;
    // the reverse stream starts after the set-up above
    SFG_CUDA(cudaEventRecord(A.ev_rec[0], s));
    SFG_CUDA(cudaStreamWaitEvent(rs, A.ev_rec[0], 0));
    for (int c = A.ncheck - 1; c >= 0; --c) {
      const int b = seg_buffer(A, c), k0 = c * A.interval, k1 = std::min(k0 + A.interval, A.nstep);
      if (A.rec_from < 0 || c < A.rec_from) {
        // buffer b is free once the reverse sweep of its last segment is done
        SFG_CUDA(cudaStreamWaitEvent(s, A.ev_rev[b], 0));
        restore_state(h, c);
        record_segment(h, c, false, b);
      }
      SFG_CUDA(cudaEventRecord(A.ev_rec[b], s));
      SFG_CUDA(cudaStreamWaitEvent(rs, A.ev_rec[b], 0));
      sfg::dev::k_set_step<<<1, 1, 0, rs>>>(A.d_k0, k0);
      if (c + 1 < A.ncheck && k1 - k0 == A.interval) {
        // full segment, not the run's last: one graph per buffer
        if (!A.graph_rev[b]) {
          cudaGraph_t g = nullptr;
          SFG_CUDA(cudaStreamBeginCapture(rs, cudaStreamCaptureModeThreadLocal));
          reverse_segment(h, b, k1 - k0, false, rs);
          SFG_CUDA(cudaStreamEndCapture(rs, &g));
          SFG_CUDA(cudaGraphInstantiate(&A.graph_rev[b], g, 0));
          cudaGraphDestroy(g);
        }
        SFG_CUDA(cudaGraphLaunch(A.graph_rev[b], rs));
      } else {
        reverse_segment(h, b, k1 - k0, c + 1 == A.ncheck, rs);
      }
      SFG_CUDA(cudaEventRecord(A.ev_rev[b], rs));
      SFG_CUDA(cudaGetLastError());
    }
    A.rec_from = -1;
    SFG_CUDA(cudaStreamSynchronize(rs));
    SFG_CUDA(cudaStreamSynchronize(s));
    h->host_step = A.nstep;
    const float dt2 = float(as.dt) / 2.0f;
    // per medium of the sweep (a coupled model: elastic, then acoustic)
    auto extract = [&](AdjointState &A, const DevMedium &D, const sfg::MediumData &M, bool acoustic) {
      // compute order -> mesh order.  Elastic: kappa and mu terms, rho from the
      // mass, -W_p G(g_p).  Acoustic: the stiffness term is d/d(rho^-1) (rho:
      // times -rho^-2), the mass W / kappa gives kappa: +W_p G(g_p) / kappa^2.
      const float *tot = h->adj.h_stage;
      SFG_CUDA(cudaMemcpy(h->adj.h_stage, A.sum, A.nsum() * sizeof(float), cudaMemcpyDeviceToHost));
      const float *grho = tot + 2 * A.nloc;
      for (int ce = 0; ce < D.nspec; ++ce) {
        const int e = M.elem_mesh[ce];
        for (int q = 0; q < sfg::NPTS; ++q) {
          const size_t pc = size_t(ce) * sfg::NPTS + q, pm = size_t(e) * sfg::NPTS + q;
          const double W = as.wgll_d[q % sfg::NGLL] * as.wgll_d[q / sfg::NGLL] * as.jac_d[pm];
          const double G = double(grho[M.ibool[pc]]);
          if (acoustic) {
            const double ri = double(M.prop0[pc]), kap = double(M.prop1[pc]);
            if (grad_rho) grad_rho[pm] = float(-ri * ri * double(tot[2 * pc + 1]));
            if (grad_kappa) grad_kappa[pm] = float(W * G / (kap * kap));
            continue;
          }
          if (grad_kappa) grad_kappa[pm] = tot[2 * pc];
          if (grad_mu) grad_mu[pm] = tot[2 * pc + 1];
          if (grad_rho) grad_rho[pm] = float(-W * G);
        }
      }
      // Stacey impedances rvp = sqrt(rho (kappa + 4/3 mu)), rvs = sqrt(rho mu);
      // acoustic: 1 / (rho vp) = (rho kappa)^-1/2
      const float *lbs = tot + A.off_lb;
      for (int i = 0; i < A.nlb; ++i) {
        const size_t k = A.lb_k[i];
        const double A1 = lbs[4 * i], A2 = lbs[4 * i + 1], A3 = lbs[4 * i + 2], A4 = lbs[4 * i + 3];
        const double wj = double(M.bc_w[k]) * double(M.bc_j1[k]);
        const double g_vp = -wj * (A1 + double(dt2) * A3);
        const double g_vs = -wj * (A2 - A1 + double(dt2) * (A4 - A3));
        const size_t pm = A.lb_pm[i];
        if (acoustic) {
          const size_t pc = size_t(as.mesh_to_compute[pm / sfg::NPTS]) * sfg::NPTS + pm % sfg::NPTS;
          const double imp = M.bc_imp0[k], rho = 1.0 / double(M.prop0[pc]), kap = double(M.prop1[pc]);
          if (grad_rho) grad_rho[pm] += float(g_vs * (-imp / (2 * rho)));
          if (grad_kappa) grad_kappa[pm] += float(g_vs * (-imp / (2 * kap)));
          continue;
        }
        const double rho = h->mesh.prho.empty() ? h->mesh.mat_rho[h->mesh.kmato[pm / sfg::NPTS]] : h->mesh.prho[pm];
        const double rvp = M.bc_imp0[k], rvs = M.bc_imp1[k];
        double dr = 0, dk = 0, dm = 0;
        if (rvp > 0) {      // P-SV only: SH has no P impedance (g_vp is 0 there)
          dr = g_vp * rvp / (2 * rho);
          dk = g_vp * rho / (2 * rvp);
          dm = g_vp * (2.0 / 3.0) * rho / rvp;
        }
        if (rvs > 0) {
          dr += g_vs * rvs / (2 * rho);
          dm += g_vs * rho / (2 * rvs);
        }
        if (grad_rho) grad_rho[pm] += float(dr);
        if (grad_kappa) grad_kappa[pm] += float(dk);
        if (grad_mu) grad_mu[pm] += float(dm);
      }
      if (acoustic && grad_kappa) {
        // kappa in the pressure sources' arrays l / kappa
        const float *ss = tot + A.off_src();
        for (int j = 0; j < A.nsrc_t; ++j) {
          const int si = A.src_list[j];
          const int ce = as.src_elem[si];
          for (int q = 0; q < sfg::NPTS; ++q) {
            const size_t pc = size_t(ce) * sfg::NPTS + q, pm = size_t(M.elem_mesh[ce]) * sfg::NPTS + q;
            const double sa = as.src_arr[(size_t(si) * 2) * sfg::NPTS + q];
            grad_kappa[pm] += float(-double(ss[size_t(j) * sfg::NPTS + q]) * sa / double(M.prop1[pc]));
          }
        }
      }
      if (acoustic && grad_mu) {
        // the acoustic medium uses kappa + 4/3 mu as its bulk modulus
        for (int ce = 0; ce < D.nspec; ++ce)
          for (int q = 0; q < sfg::NPTS; ++q) {
            const size_t pm = size_t(M.elem_mesh[ce]) * sfg::NPTS + q;
            grad_mu[pm] = grad_kappa ? float(4.0 / 3.0 * grad_kappa[pm]) : 0.0f;
          }
      }
    };
    extract(A, adj_dev(h), adj_data(h), adj_acoustic(h));
    if (cpl) extract(A2, h->ac, as.ac, true);
    return int(SFG_OK);
  });
}

}  // extern "C"
