// libsfg, 3D elastic: host set-up of structured hexahedral meshes and the
// extern "C" entry points declared in include/sfg3d.h.
//
// Set-up (FP64, rounded to FP32): lattice numbering of the GLL points,
// 8-node trilinear geometry (core/specfem/shape_function/dim3,
// core/specfem/jacobian/dim3), isotropic properties (lambda + 2 mu = kappa +
// 4/3 mu, kappa = rho (vp^2 - 4/3 vs^2)), mass matrix rho w w w |J|
// (include/medium/dim3/elastic/isotropic/mass_matrix.tpp:5-15), absorbing
// faces, source arrays (compute_source_array/dim3/impl/*) and receiver
// interpolants; the point-major contribution slots of the owner-computes
// assembly.
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sfg3d.h"
#include "kernels3d.cuh"

namespace sfg3 {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define SFG3_CUDA(call)                                                                  \
  do {                                                                                   \
    cudaError_t _e = (call);                                                             \
    if (_e != cudaSuccess) throw sfg3::CudaError(std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

constexpr int NG = 5, NQ = 125;

struct DevMem {
  std::vector<void *> ptrs;
  size_t bytes = 0;
  template <typename T>
  T *upload(const std::vector<T> &h) {
    if (h.empty()) return nullptr;
    T *d = nullptr;
    SFG3_CUDA(cudaMalloc(&d, h.size() * sizeof(T)));
    ptrs.push_back(d);
    bytes += h.size() * sizeof(T);
    SFG3_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
  }
  template <typename T>
  T *zeros(size_t n) {
    if (n == 0) return nullptr;
    T *d = nullptr;
    SFG3_CUDA(cudaMalloc(&d, n * sizeof(T)));
    ptrs.push_back(d);
    bytes += n * sizeof(T);
    SFG3_CUDA(cudaMemset(d, 0, n * sizeof(T)));
    return d;
  }
  ~DevMem() {
    for (void *p : ptrs) cudaFree(p);
  }
};

// ------------------------------------------------------------ geometry ---
void gll5(double z[NG], double w[NG], double hp[NG][NG]) {
  const double r = std::sqrt(3.0 / 7.0);
  const double zz[NG] = {-1.0, -r, 0.0, r, 1.0};
  const double ww[NG] = {0.1, 49.0 / 90.0, 32.0 / 45.0, 49.0 / 90.0, 0.1};
  auto P4 = [](double x) { return (35 * x * x * x * x - 30 * x * x + 3) / 8.0; };
  for (int i = 0; i < NG; ++i) { z[i] = zz[i]; w[i] = ww[i]; }
  for (int i = 0; i < NG; ++i)
    for (int j = 0; j < NG; ++j) {
      if (i == j) hp[i][j] = i == 0 ? -5.0 : (i == NG - 1 ? 5.0 : 0.0);
      else hp[i][j] = P4(z[i]) / (P4(z[j]) * (z[i] - z[j]));
    }
}

void lagrange(double x, const double z[NG], double h[NG], double hp[NG]) {
  for (int d = 0; d < NG; ++d) {
    double num = 1, den = 1, sum = 0;
    for (int i = 0; i < NG; ++i) {
      if (i == d) continue;
      num *= x - z[i];
      den *= z[d] - z[i];
      double p = 1;
      for (int j = 0; j < NG; ++j)
        if (j != d && j != i) p *= x - z[j];
      sum += p;
    }
    h[d] = num / den;
    hp[d] = sum / den;
  }
}

// 8-node hexahedron, corners (xi, eta, gamma) in {-1, 1}^3 (same order as the
// mesh description: bottom face counter-clockwise, then top face)
const int CS[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                      {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

struct Geo {
  double x[3];
  double inv[3][3];  // d xi_k / d x_j
  double jac;
};

Geo map_point(const double cn[8][3], double xi, double eta, double ga) {
  double dx[3][3] = {{0}};
  Geo G{};
  for (int a = 0; a < 8; ++a) {
    const double sx = 1 + CS[a][0] * xi, sy = 1 + CS[a][1] * eta, sz = 1 + CS[a][2] * ga;
    const double N = 0.125 * sx * sy * sz;
    const double dN[3] = {0.125 * CS[a][0] * sy * sz, 0.125 * sx * CS[a][1] * sz, 0.125 * sx * sy * CS[a][2]};
    for (int j = 0; j < 3; ++j) {
      G.x[j] += N * cn[a][j];
      for (int k = 0; k < 3; ++k) dx[j][k] += dN[k] * cn[a][j];
    }
  }
  const double det = dx[0][0] * (dx[1][1] * dx[2][2] - dx[1][2] * dx[2][1]) -
                     dx[0][1] * (dx[1][0] * dx[2][2] - dx[1][2] * dx[2][0]) +
                     dx[0][2] * (dx[1][0] * dx[2][1] - dx[1][1] * dx[2][0]);
  G.jac = det;
  G.inv[0][0] = (dx[1][1] * dx[2][2] - dx[1][2] * dx[2][1]) / det;
  G.inv[0][1] = (dx[0][2] * dx[2][1] - dx[0][1] * dx[2][2]) / det;
  G.inv[0][2] = (dx[0][1] * dx[1][2] - dx[0][2] * dx[1][1]) / det;
  G.inv[1][0] = (dx[1][2] * dx[2][0] - dx[1][0] * dx[2][2]) / det;
  G.inv[1][1] = (dx[0][0] * dx[2][2] - dx[0][2] * dx[2][0]) / det;
  G.inv[1][2] = (dx[0][2] * dx[1][0] - dx[0][0] * dx[1][2]) / det;
  G.inv[2][0] = (dx[1][0] * dx[2][1] - dx[1][1] * dx[2][0]) / det;
  G.inv[2][1] = (dx[0][1] * dx[2][0] - dx[0][0] * dx[2][1]) / det;
  G.inv[2][2] = (dx[0][0] * dx[1][1] - dx[0][1] * dx[1][0]) / det;
  return G;
}

}  // namespace sfg3

struct sfg_handle3d {
  std::string err;
  sfg_options opt{};
  int nex = 0, ney = 0, nez = 0, nspec = 0, nglob = 0;
  size_t nloc = 0;
  std::vector<double> nodes;
  std::vector<float> rho, vp, vs;
  int absorbing[6] = {0, 0, 0, 0, 0, 0};
  double zd[5], wd[5], hpd[5][5];
  // host set-up
  std::vector<float> g9;  // [9][nloc]
  std::vector<float> jac, c0, mu;
  std::vector<int> slot, inv_start, bc_slot;
  std::vector<float> bc_c, minv;
  // sources / receivers
  std::vector<sfg_source3d> sources;
  int nsrc = 0;
  std::vector<int> src_elem, src_next, src_head;
  std::vector<float> src_arr, stf;
  double t0 = 0;
  int nrec = 0, ntypes = 1;
  std::vector<int> rec_elem, types{0};
  std::vector<float> rec_h;
  bool have_sources = false, initialized = false, state_final = true;
  int host_step = 0;
  // device
  std::unique_ptr<sfg3::DevMem> mem;
  sfg3::dev::Elem3Args EA{};
  int *d_step = nullptr, *d_flag = nullptr;
  float *d_u = nullptr, *d_v = nullptr, *d_a = nullptr, *d_minv = nullptr, *d_r = nullptr;
  int *d_inv_start = nullptr, *d_ibool = nullptr, *d_rec_elem = nullptr, *d_types = nullptr;
  float *d_rec_h = nullptr, *d_seis = nullptr, *d_stf = nullptr;
  float *flush = nullptr;
  size_t flush_bytes = 0;
  int epb = 4;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraphExec_t graph_k = nullptr, graph_1 = nullptr, graph_e = nullptr;
  int graph_steps = 20;
  int sm_count = 148;
  ~sfg_handle3d() {
    for (cudaGraphExec_t g : {graph_k, graph_1, graph_e})
      if (g) cudaGraphExecDestroy(g);
    if (flush) cudaFree(flush);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    mem.reset();
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

using sfg3::NG;
using sfg3::NQ;

static std::string g_create_error3;

template <typename F>
int guarded(sfg_handle3d *h, F &&fn) {
  if (!h) return SFG_ERR_ARG;
  try {
    return fn();
  } catch (const sfg3::CudaError &ex) {
    h->err = ex.what();
    return SFG_ERR_CUDA;
  } catch (const std::exception &ex) {
    h->err = ex.what();
    return SFG_ERR_ARG;
  }
}

void corners(const sfg_handle3d *h, int e, double cn[8][3]) {
  const int ex = e % h->nex, ey = (e / h->nex) % h->ney, ez = e / (h->nex * h->ney);
  for (int a = 0; a < 8; ++a) {
    const int i = ex + (sfg3::CS[a][0] > 0), j = ey + (sfg3::CS[a][1] > 0), k = ez + (sfg3::CS[a][2] > 0);
    const double *p = &h->nodes[3 * ((size_t(k) * (h->ney + 1) + j) * (h->nex + 1) + i)];
    for (int c = 0; c < 3; ++c) cn[a][c] = p[c];
  }
}

// Element and local coordinates of a point: nearest control node, Newton in
// the elements around it, first element within 1e-9 of the best.
void locate(const sfg_handle3d *h, const double *X, int &elem, double xi[3]) {
  const size_t nn = size_t(h->nex + 1) * (h->ney + 1) * (h->nez + 1);
  size_t best = 0;
  double bd = 1e300;
  for (size_t i = 0; i < nn; ++i) {
    double d = 0;
    for (int c = 0; c < 3; ++c) d += (h->nodes[3 * i + c] - X[c]) * (h->nodes[3 * i + c] - X[c]);
    if (d < bd) { bd = d; best = i; }
  }
  const int ni = int(best % (h->nex + 1)), nj = int((best / (h->nex + 1)) % (h->ney + 1)),
            nk = int(best / (size_t(h->nex + 1) * (h->ney + 1)));
  double bestv = 1e300;
  elem = -1;
  for (int dk = -1; dk <= 0; ++dk)
    for (int dj = -1; dj <= 0; ++dj)
      for (int di = -1; di <= 0; ++di) {
        const int ex = ni + di, ey = nj + dj, ez = nk + dk;
        if (ex < 0 || ey < 0 || ez < 0 || ex >= h->nex || ey >= h->ney || ez >= h->nez) continue;
        const int e = (ez * h->ney + ey) * h->nex + ex;
        double cn[8][3];
        corners(h, e, cn);
        double s[3] = {0, 0, 0};
        for (int it = 0; it < 20; ++it) {
          const sfg3::Geo G = sfg3::map_point(cn, s[0], s[1], s[2]);
          double r[3];
          for (int c = 0; c < 3; ++c) r[c] = X[c] - G.x[c];
          for (int k = 0; k < 3; ++k) {
            double ds = 0;
            for (int j = 0; j < 3; ++j) ds += G.inv[k][j] * r[j];
            s[k] += ds;
          }
        }
        const double m = std::max({std::fabs(s[0]), std::fabs(s[1]), std::fabs(s[2])});
        if (m < bestv - 1e-9) {
          bestv = m;
          elem = e;
          for (int c = 0; c < 3; ++c) xi[c] = std::min(1.0, std::max(-1.0, s[c]));
        }
      }
  if (elem < 0 || bestv > 1.0 + 1e-6) throw std::runtime_error("point outside the mesh");
}

void setup_geometry(sfg_handle3d *h) {
  const size_t nloc = h->nloc;
  const int NX = 4 * h->nex + 1, NY = 4 * h->ney + 1;
  h->g9.assign(9 * nloc, 0.0f);
  h->jac.assign(nloc, 0.0f);
  h->c0.assign(nloc, 0.0f);
  h->mu.assign(nloc, 0.0f);
  std::vector<int> ibool(nloc);
  std::vector<double> mass(size_t(h->nglob), 0.0);
  bool bad = false;
#pragma omp parallel for schedule(static) reduction(|| : bad)
  for (int e = 0; e < h->nspec; ++e) {
    double cn[8][3];
    corners(h, e, cn);
    const int ex = e % h->nex, ey = (e / h->nex) % h->ney, ez = e / (h->nex * h->ney);
    for (int q = 0; q < NQ; ++q) {
      const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
      const size_t p = size_t(e) * NQ + q;
      ibool[p] = ((4 * ez + iz) * NY + 4 * ey + iy) * NX + 4 * ex + ix;
      const sfg3::Geo G = sfg3::map_point(cn, h->zd[ix], h->zd[iy], h->zd[iz]);
      if (!(G.jac > 0)) bad = true;
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) h->g9[size_t(k * 3 + j) * nloc + p] = float(G.inv[k][j]);
      h->jac[p] = float(G.jac);
      const double rho = h->rho[p], vp = h->vp[p], vs = h->vs[p];
      const double m = rho * vs * vs, kappa = rho * (vp * vp - 4.0 / 3.0 * vs * vs);
      h->c0[p] = float(kappa + 4.0 / 3.0 * m);
      h->mu[p] = float(m);
    }
  }
  if (bad) throw std::runtime_error("non-positive Jacobian in the mesh");
  // mass (serial: fixed summation order)
  for (int e = 0; e < h->nspec; ++e)
    for (int q = 0; q < NQ; ++q) {
      const size_t p = size_t(e) * NQ + q;
      const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
      mass[size_t(ibool[p])] += double(h->rho[p]) * h->wd[ix] * h->wd[iy] * h->wd[iz] * double(h->jac[p]);
    }
  // absorbing faces: per element point C = sum over the element's absorbing
  // faces of w_a w_b [(rvp - rvs) n n^T / |n| + rvs |n| I]; implicit mass term
  std::vector<double> mst(size_t(h->nglob) * 3, 0.0);
  h->bc_slot.assign(size_t(h->nspec), -1);
  h->bc_c.clear();
  int nbc = 0;
  for (int e = 0; e < h->nspec; ++e) {
    const int ex = e % h->nex, ey = (e / h->nex) % h->ney, ez = e / (h->nex * h->ney);
    const bool on[6] = {ex == 0, ex == h->nex - 1, ey == 0, ey == h->ney - 1, ez == 0, ez == h->nez - 1};
    bool any = false;
    for (int f = 0; f < 6; ++f) any |= on[f] && h->absorbing[f];
    if (!any) continue;
    h->bc_slot[size_t(e)] = nbc++;
    h->bc_c.resize(size_t(nbc) * 6 * NQ, 0.0f);
    std::vector<double> C(6 * NQ, 0.0);
    for (int f = 0; f < 6; ++f) {
      if (!on[f] || !h->absorbing[f]) continue;
      const int k = f / 2, fix = (f % 2) ? NG - 1 : 0;
      const double sgn = (f % 2) ? 1.0 : -1.0;
      for (int b = 0; b < NG; ++b)
        for (int c = 0; c < NG; ++c) {
          int idx[3];
          idx[k] = fix;
          idx[(k + 1) % 3] = b;
          idx[(k + 2) % 3] = c;
          const int q = (idx[2] * NG + idx[1]) * NG + idx[0];
          const size_t p = size_t(e) * NQ + q;
          double n[3];
          for (int j = 0; j < 3; ++j) n[j] = sgn * double(h->g9[size_t(k * 3 + j) * h->nloc + p]) * double(h->jac[p]);
          const double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
          const double rho = h->rho[p], rvp = rho * double(h->vp[p]), rvs = rho * double(h->vs[p]);
          const double wab = h->wd[b] * h->wd[c];
          const double d = (rvp - rvs) / nn * wab, s = rvs * nn * wab;
          C[0 * NQ + q] += d * n[0] * n[0] + s;
          C[1 * NQ + q] += d * n[1] * n[1] + s;
          C[2 * NQ + q] += d * n[2] * n[2] + s;
          C[3 * NQ + q] += d * n[0] * n[1];
          C[4 * NQ + q] += d * n[0] * n[2];
          C[5 * NQ + q] += d * n[1] * n[2];
          // implicit term: -traction at the velocity stand-in -dt/2 (1, 1, 1)
          const double vv = -h->opt.dt * 0.5, vn = vv * (n[0] + n[1] + n[2]);
          for (int j = 0; j < 3; ++j) {
            const double fj = (vn * n[j] / (nn * nn)) * (rvp - rvs) + vv * rvs;
            mst[size_t(ibool[p]) * 3 + j] += -1.0 * fj * nn * wab;
          }
        }
    }
    for (int i = 0; i < 6 * NQ; ++i) h->bc_c[size_t(nbc - 1) * 6 * NQ + i] = float(C[i]);
  }
  h->minv.assign(size_t(h->nglob) * 3, 0.0f);
  for (size_t g = 0; g < size_t(h->nglob); ++g)
    for (int j = 0; j < 3; ++j) h->minv[g * 3 + j] = float(1.0 / (mass[g] + mst[g * 3 + j]));
  // point-major slots: each point's contributions in increasing element order
  h->inv_start.assign(size_t(h->nglob) + 1, 0);
  for (size_t p = 0; p < nloc; ++p) h->inv_start[size_t(ibool[p]) + 1]++;
  for (size_t g = 0; g < size_t(h->nglob); ++g) h->inv_start[g + 1] += h->inv_start[g];
  std::vector<int> fill(h->inv_start.begin(), h->inv_start.end() - 1);
  h->slot.resize(nloc);
  for (size_t p = 0; p < nloc; ++p) h->slot[p] = fill[size_t(ibool[p])]++;
  h->EA.nloc = nloc;
  h->mem.reset(new sfg3::DevMem());
  h->d_ibool = h->mem->upload(ibool);
}

void setup_sources(sfg_handle3d *h) {
  h->nsrc = int(h->sources.size());
  h->src_elem.assign(size_t(h->nsrc), 0);
  h->src_next.assign(size_t(std::max(h->nsrc, 1)), -1);
  h->src_head.assign(size_t(h->nspec), -1);
  h->src_arr.assign(size_t(std::max(h->nsrc, 1)) * 3 * NQ, 0.0f);
  const int nstep = h->opt.nstep;
  h->stf.assign(size_t(nstep) * std::max(h->nsrc, 1), 0.0f);
  std::vector<double> ts(size_t(h->nsrc));
  h->t0 = 0;
  for (int s = 0; s < h->nsrc; ++s) {
    const sfg_source3d &S = h->sources[size_t(s)];
    if (!(S.f0 > 0)) throw std::runtime_error("source f0 must be positive");
    ts[size_t(s)] = double(-1.2f * (1.0f / float(S.f0)) + float(S.tshift));
    h->t0 = s == 0 ? ts[0] : std::min(h->t0, ts[size_t(s)]);
  }
  for (int s = 0; s < h->nsrc; ++s) {
    const sfg_source3d &S = h->sources[size_t(s)];
    const double X[3] = {S.x, S.y, S.z};
    int e;
    double xi[3];
    locate(h, X, e, xi);
    h->src_elem[size_t(s)] = e;
    h->src_next[size_t(s)] = h->src_head[size_t(e)];
    h->src_head[size_t(e)] = s;
    double hh[3][NG], hd[3][NG];
    for (int k = 0; k < 3; ++k) sfg3::lagrange(xi[k], h->zd, hh[k], hd[k]);
    float *arr = &h->src_arr[size_t(s) * 3 * NQ];
    if (S.kind == SFG_SOURCE_FORCE) {
      for (int q = 0; q < NQ; ++q) {
        const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
        const double hl = hh[0][ix] * hh[1][iy] * hh[2][iz];
        for (int c = 0; c < 3; ++c) arr[c * NQ + q] = float(hl * S.comp[c]);
      }
    } else if (S.kind == SFG_SOURCE_MOMENT_TENSOR) {
      double J[3][3] = {{0}};
      for (int q = 0; q < NQ; ++q) {
        const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
        const double hl = hh[0][ix] * hh[1][iy] * hh[2][iz];
        for (int k = 0; k < 3; ++k)
          for (int j = 0; j < 3; ++j) J[k][j] += hl * double(h->g9[size_t(k * 3 + j) * h->nloc + size_t(e) * NQ + q]);
      }
      const double *cp = S.comp;
      const double M[3][3] = {{cp[0], cp[3], cp[4]}, {cp[3], cp[1], cp[5]}, {cp[4], cp[5], cp[2]}};
      for (int q = 0; q < NQ; ++q) {
        const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
        const double dxi[3] = {hd[0][ix] * hh[1][iy] * hh[2][iz], hh[0][ix] * hd[1][iy] * hh[2][iz],
                               hh[0][ix] * hh[1][iy] * hd[2][iz]};
        double dsx[3] = {0, 0, 0};
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) dsx[j] += dxi[k] * J[k][j];
        for (int c = 0; c < 3; ++c) arr[c * NQ + q] = float(M[c][0] * dsx[0] + M[c][1] * dsx[1] + M[c][2] * dsx[2]);
      }
    } else {
      throw std::runtime_error("unknown source kind");
    }
    // Ricker table in FP32 (ricker.cpp:40-63)
    const float tsh = float(ts[size_t(s)] - h->t0), t0 = float(h->t0);
    const float f0 = float(S.f0), fac = float(S.factor), pi = float(M_PI), aa = pi * pi * f0 * f0;
    const float dt = float(h->opt.dt);
    for (int i = 0; i < nstep; ++i) {
      const float t = t0 + float(i) * dt - tsh;
      h->stf[size_t(i) * h->nsrc + s] = fac * ((1.0f - 2.0f * aa * t * t) * std::exp(-aa * t * t));
    }
  }
}

// Element kernel launch: 1, 2 or 4 elements per block run the point form
// (one thread per element point), 6 or 8 the column form (one thread per
// column of five points).
int col3_smem(int E) { return E * 9 * 25 * sfg3::dev::RP3 * int(sizeof(float)); }

void launch_elem(sfg_handle3d *h, const sfg3::dev::Elem3Args &A, cudaStream_t s) {
  const int E = h->epb;
  const int grid = (h->nspec + E - 1) / E;
  switch (E) {
    case 1: sfg3::dev::k_stiffness3d<1><<<grid, NQ * 1, 0, s>>>(A); break;
    case 2: sfg3::dev::k_stiffness3d<2><<<grid, NQ * 2, 0, s>>>(A); break;
    case 6: sfg3::dev::k_stiffness3d_col<6><<<grid, 25 * 6, col3_smem(6), s>>>(A); break;
    case 8: sfg3::dev::k_stiffness3d_col<8><<<grid, 25 * 8, col3_smem(8), s>>>(A); break;
    default: sfg3::dev::k_stiffness3d<4><<<grid, NQ * 4, 0, s>>>(A); break;
  }
}

bool valid_epb3(int e) { return e == 1 || e == 2 || e == 4 || e == 6 || e == 8; }

void launch_step(sfg_handle3d *h, cudaStream_t s, bool predict) {
  sfg3::dev::Elem3Args A = h->EA;
  A.step = h->d_step;
  launch_elem(h, A, s);
  if (h->nrec) {
    sfg3::dev::Rec3Args R{};
    R.ibool = h->d_ibool; R.rec_elem = h->d_rec_elem; R.rec_h = h->d_rec_h; R.types = h->d_types;
    R.ntypes = h->ntypes; R.nrec = h->nrec; R.nsig = h->opt.nstep;
    R.u = h->d_u; R.v = h->d_v; R.minv = h->d_minv; R.r = h->d_r; R.inv_start = h->d_inv_start;
    R.dt2 = float(h->opt.dt) / 2.0f;
    R.step = h->d_step; R.seis = h->d_seis;
    sfg3::dev::k_receivers3d<<<h->nrec, 128, 0, s>>>(R);
  }
  sfg3::dev::Update3Args U{};
  U.u = h->d_u; U.v = h->d_v; U.a_store = predict ? nullptr : h->d_a;
  U.minv = h->d_minv; U.inv_start = h->d_inv_start; U.r = h->d_r; U.npts = h->nglob;
  const float dt = float(h->opt.dt);
  U.dt = dt; U.dt2 = dt / 2.0f; U.dtsq2 = dt * dt / 2.0f;
  U.predict = predict ? 1 : 0;
  U.flag = h->d_flag; U.step = h->d_step; U.advance = 1;
  const int ug = std::max(1, std::min((h->nglob + 255) / 256, h->sm_count * 8));
  sfg3::dev::k_update3d<<<ug, 256, 0, s>>>(U);
}

cudaGraphExec_t capture(sfg_handle3d *h, int n, bool last_predicts) {
  cudaGraph_t g = nullptr;
  SFG3_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < n; ++i) launch_step(h, h->stream, i + 1 < n || last_predicts);
  SFG3_CUDA(cudaStreamEndCapture(h->stream, &g));
  cudaGraphExec_t ex = nullptr;
  SFG3_CUDA(cudaGraphInstantiate(&ex, g, 0));
  cudaGraphDestroy(g);
  return ex;
}

void resume(sfg_handle3d *h) {
  if (h->state_final) {
    const float dt = float(h->opt.dt);
    const size_t n = size_t(h->nglob) * 3;
    sfg3::dev::k_predict3d<<<h->sm_count * 8, 256, 0, h->stream>>>(h->d_u, h->d_v, h->d_a, n, dt, dt / 2.0f,
                                                                      dt * dt / 2.0f);
    h->state_final = false;
  }
}

void run_steps(sfg_handle3d *h, int n) {
  if (n <= 0) return;
  resume(h);
  int fused = n - 1;
  while (fused >= h->graph_steps) {
    SFG3_CUDA(cudaGraphLaunch(h->graph_k, h->stream));
    fused -= h->graph_steps;
  }
  for (; fused > 0; --fused) SFG3_CUDA(cudaGraphLaunch(h->graph_1, h->stream));
  SFG3_CUDA(cudaGraphLaunch(h->graph_e, h->stream));
  h->state_final = true;
  h->host_step += n;
  SFG3_CUDA(cudaGetLastError());
}

}  // namespace

extern "C" {

const char *sfg3d_last_error(const sfg_handle3d *h) { return h ? h->err.c_str() : g_create_error3.c_str(); }

int sfg3d_create(const sfg_mesh3d_desc *mesh, const sfg_options *opt, sfg_handle3d **out) {
  if (!mesh || !opt || !out) { g_create_error3 = "null argument"; return SFG_ERR_ARG; }
  *out = nullptr;
  if (mesh->nex <= 0 || mesh->ney <= 0 || mesh->nez <= 0 || !mesh->nodes || !mesh->rho || !mesh->vp ||
      !mesh->vs || !(opt->dt > 0) || opt->nstep <= 0) {
    g_create_error3 = "invalid mesh or options";
    return SFG_ERR_ARG;
  }
  if (opt->nshots > 1 || opt->nstep_between_samples > 1) {
    g_create_error3 = "3D runs one shot sampled every step";
    return SFG_ERR_UNSUPPORTED;
  }
  const long long nsp = (long long)mesh->nex * mesh->ney * mesh->nez;
  const long long ng = (4LL * mesh->nex + 1) * (4LL * mesh->ney + 1) * (4LL * mesh->nez + 1);
  if (nsp * NQ >= (1LL << 31) || ng >= (1LL << 31)) {
    g_create_error3 = "mesh too large for 32-bit point indices";
    return SFG_ERR_ARG;
  }
  auto h = std::make_unique<sfg_handle3d>();
  h->opt = *opt;
  h->nex = mesh->nex; h->ney = mesh->ney; h->nez = mesh->nez;
  h->nspec = int(nsp);
  h->nglob = int(ng);
  h->nloc = size_t(nsp) * NQ;
  h->nodes.assign(mesh->nodes, mesh->nodes + 3 * size_t(mesh->nex + 1) * (mesh->ney + 1) * (mesh->nez + 1));
  h->rho.assign(mesh->rho, mesh->rho + h->nloc);
  h->vp.assign(mesh->vp, mesh->vp + h->nloc);
  h->vs.assign(mesh->vs, mesh->vs + h->nloc);
  for (int f = 0; f < 6; ++f) h->absorbing[f] = mesh->absorbing[f] ? 1 : 0;
  sfg3::gll5(h->zd, h->wd, h->hpd);
  for (size_t p = 0; p < h->nloc; ++p)
    if (!(h->rho[p] > 0) || !(h->vs[p] >= 0) || !(h->vp[p] > h->vs[p] * 1.1547f)) {
      g_create_error3 = "model values must give rho > 0, vs >= 0, lambda + 2 mu > 0";
      return SFG_ERR_ARG;
    }
  if (valid_epb3(opt->elements_per_block)) h->epb = opt->elements_per_block;
  if (opt->steps_per_graph > 0) h->graph_steps = opt->steps_per_graph;
  *out = h.release();
  return SFG_OK;
}

void sfg3d_destroy(sfg_handle3d *h) { delete h; }

int sfg3d_set_sources(sfg_handle3d *h, int nsrc, const sfg_source3d *src) {
  return guarded(h, [&]() {
    if (h->initialized) { h->err = "sources must be set before sfg3d_initialize"; return int(SFG_ERR_STATE); }
    if (nsrc < 0 || (nsrc > 0 && !src)) { h->err = "bad source array"; return int(SFG_ERR_ARG); }
    h->sources.assign(src, src + nsrc);
    h->have_sources = true;
    return int(SFG_OK);
  });
}

int sfg3d_set_receivers(sfg_handle3d *h, int nrec, const double *xyz, int ntypes, const int *types) {
  return guarded(h, [&]() {
    if (h->initialized) { h->err = "receivers must be set before sfg3d_initialize"; return int(SFG_ERR_STATE); }
    if (nrec < 0 || (nrec > 0 && !xyz) || ntypes < 1 || ntypes > 3 || !types) {
      h->err = "bad receiver arrays";
      return int(SFG_ERR_ARG);
    }
    h->nrec = nrec;
    h->ntypes = ntypes;
    h->types.assign(types, types + ntypes);
    for (int t : h->types)
      if (t < 0 || t > 2) { h->err = "3D seismograms: displacement, velocity or acceleration"; return int(SFG_ERR_ARG); }
    h->rec_elem.assign(size_t(nrec), 0);
    h->rec_h.assign(size_t(std::max(nrec, 1)) * NQ, 0.0f);
    for (int r = 0; r < nrec; ++r) {
      int e;
      double xi[3];
      try {
        locate(h, xyz + 3 * r, e, xi);
      } catch (const std::exception &ex) {
        h->err = ex.what();
        return int(SFG_ERR_LOCATE);
      }
      h->rec_elem[size_t(r)] = e;
      double hh[3][NG], hd[3][NG];
      for (int k = 0; k < 3; ++k) sfg3::lagrange(xi[k], h->zd, hh[k], hd[k]);
      for (int q = 0; q < NQ; ++q) {
        const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
        h->rec_h[size_t(r) * NQ + q] = float(hh[0][ix] * hh[1][iy] * hh[2][iz]);
      }
    }
    return int(SFG_OK);
  });
}

int sfg3d_initialize(sfg_handle3d *h) {
  return guarded(h, [&]() {
    if (h->initialized) return int(SFG_OK);
    omp_set_num_threads(std::max(1, omp_get_num_procs()));
    setup_geometry(h);
    try {
      setup_sources(h);
    } catch (const std::exception &ex) {
      h->err = ex.what();
      return int(SFG_ERR_LOCATE);
    }
    SFG3_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    SFG3_CUDA(cudaEventCreate(&h->ev0));
    SFG3_CUDA(cudaEventCreate(&h->ev1));
    {
      int dev = 0;
      SFG3_CUDA(cudaGetDevice(&dev));
      SFG3_CUDA(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, dev));
    }
    float hp[25], hpw[25], w[5];
    for (int i = 0; i < NG; ++i) {
      w[i] = float(h->wd[i]);
      for (int j = 0; j < NG; ++j) {
        hp[i * NG + j] = float(h->hpd[i][j]);
        hpw[i * NG + j] = float(h->hpd[i][j] * h->wd[i]);
      }
    }
    SFG3_CUDA(cudaMemcpyToSymbol(sfg3::dev::c3_hp, hp, sizeof(hp)));
    SFG3_CUDA(cudaMemcpyToSymbol(sfg3::dev::c3_hpw, hpw, sizeof(hpw)));
    SFG3_CUDA(cudaMemcpyToSymbol(sfg3::dev::c3_w, w, sizeof(w)));
    sfg3::DevMem &m = *h->mem;
    sfg3::dev::Elem3Args &A = h->EA;
    A.ibool = h->d_ibool;
    A.g9 = m.upload(h->g9);
    A.jac = m.upload(h->jac);
    A.c0 = m.upload(h->c0);
    A.mu = m.upload(h->mu);
    A.slot = m.upload(h->slot);
    A.bc_slot = m.upload(h->bc_slot);
    A.bc_c = h->bc_c.empty() ? nullptr : m.upload(h->bc_c);
    A.src_head = m.upload(h->src_head);
    A.src_next = m.upload(h->src_next);
    A.src_arr = m.upload(h->src_arr);
    h->d_stf = m.upload(h->stf);
    A.stf = h->d_stf;
    A.nsrc = std::max(h->nsrc, 1);
    A.nstep = h->opt.nstep;
    A.nspec = h->nspec;
    A.nloc = h->nloc;
    const size_t n = size_t(h->nglob) * 3 + 4;
    h->d_u = m.zeros<float>(n);
    h->d_v = m.zeros<float>(n);
    h->d_a = m.zeros<float>(n);
    h->d_r = m.zeros<float>(h->nloc * 3 + 4);
    h->d_minv = m.upload(h->minv);
    h->d_inv_start = m.upload(h->inv_start);
    A.u = h->d_u; A.v = h->d_v; A.r = h->d_r;
    if (h->nsrc == 0) A.src_head = m.upload(std::vector<int>(size_t(h->nspec), -1));
    h->d_rec_elem = m.upload(h->rec_elem);
    h->d_rec_h = m.upload(h->rec_h);
    h->d_types = m.upload(h->types);
    h->d_seis = m.zeros<float>(size_t(h->opt.nstep) * h->ntypes * std::max(h->nrec, 1) * 3);
    h->d_step = m.zeros<int>(1);
    h->d_flag = m.zeros<int>(1);
    // host copies no longer needed
    std::vector<float>().swap(h->g9);
    std::vector<float>().swap(h->jac);
    std::vector<float>().swap(h->c0);
    std::vector<float>().swap(h->mu);
    std::vector<int>().swap(h->slot);
    SFG3_CUDA(cudaDeviceSynchronize());
    SFG3_CUDA(cudaFuncSetAttribute(sfg3::dev::k_stiffness3d_col<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   col3_smem(8)));
    SFG3_CUDA(cudaFuncSetAttribute(sfg3::dev::k_stiffness3d_col<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   col3_smem(6)));
    if (!valid_epb3(h->opt.elements_per_block)) {
      // launch-shape autotuner: elements per block and form of the element
      // kernel, whole steps timed on this mesh (all shapes give the same bits)
      float best = 1e30f;
      int pick = h->epb;
      for (int e : {1, 2, 4, 6, 8}) {
        h->epb = e;
        for (int i = 0; i < 2; ++i) launch_step(h, h->stream, true);
        SFG3_CUDA(cudaEventRecord(h->ev0, h->stream));
        for (int i = 0; i < 3; ++i) launch_step(h, h->stream, true);
        SFG3_CUDA(cudaEventRecord(h->ev1, h->stream));
        SFG3_CUDA(cudaEventSynchronize(h->ev1));
        float t = 0;
        SFG3_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
        if (t < best) { best = t; pick = e; }
      }
      h->epb = pick;
      const size_t nb = n * sizeof(float);
      SFG3_CUDA(cudaMemset(h->d_u, 0, nb));
      SFG3_CUDA(cudaMemset(h->d_v, 0, nb));
      SFG3_CUDA(cudaMemset(h->d_a, 0, nb));
      SFG3_CUDA(cudaMemset(h->d_step, 0, sizeof(int)));
      SFG3_CUDA(cudaMemset(h->d_flag, 0, sizeof(int)));
      SFG3_CUDA(cudaMemset(h->d_seis, 0, size_t(h->opt.nstep) * h->ntypes * std::max(h->nrec, 1) * 3 * sizeof(float)));
      SFG3_CUDA(cudaDeviceSynchronize());
    }
    h->graph_k = capture(h, h->graph_steps, true);
    h->graph_1 = capture(h, 1, true);
    h->graph_e = capture(h, 1, false);
    h->initialized = true;
    h->state_final = true;
    h->host_step = 0;
    return int(SFG_OK);
  });
}

int sfg3d_reset_fields(sfg_handle3d *h) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg3d_initialize first"; return int(SFG_ERR_STATE); }
    const size_t n = (size_t(h->nglob) * 3 + 4) * sizeof(float);
    SFG3_CUDA(cudaMemsetAsync(h->d_u, 0, n, h->stream));
    SFG3_CUDA(cudaMemsetAsync(h->d_v, 0, n, h->stream));
    SFG3_CUDA(cudaMemsetAsync(h->d_a, 0, n, h->stream));
    SFG3_CUDA(cudaMemsetAsync(h->d_step, 0, sizeof(int), h->stream));
    SFG3_CUDA(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    SFG3_CUDA(cudaMemsetAsync(h->d_seis, 0, size_t(h->opt.nstep) * h->ntypes * std::max(h->nrec, 1) * 3 * sizeof(float),
                              h->stream));
    SFG3_CUDA(cudaStreamSynchronize(h->stream));
    h->state_final = true;
    h->host_step = 0;
    return int(SFG_OK);
  });
}

int sfg3d_run(sfg_handle3d *h, int nsteps) {
  return guarded(h, [&]() {
    if (!h->initialized) { h->err = "sfg3d_initialize first"; return int(SFG_ERR_STATE); }
    if (nsteps < 0 || h->host_step + nsteps > h->opt.nstep) { h->err = "beyond nstep"; return int(SFG_ERR_ARG); }
    run_steps(h, nsteps);
    SFG3_CUDA(cudaStreamSynchronize(h->stream));
    return int(SFG_OK);
  });
}

int sfg3d_run_timed(sfg_handle3d *h, int nsteps, float *ms) {
  return guarded(h, [&]() {
    if (!h->initialized || !ms) return int(SFG_ERR_STATE);
    if (nsteps <= 0 || h->host_step + nsteps > h->opt.nstep) { h->err = "beyond nstep"; return int(SFG_ERR_ARG); }
    resume(h);
    SFG3_CUDA(cudaEventRecord(h->ev0, h->stream));
    int left = nsteps;
    while (left >= h->graph_steps) { SFG3_CUDA(cudaGraphLaunch(h->graph_k, h->stream)); left -= h->graph_steps; }
    for (; left > 0; --left) SFG3_CUDA(cudaGraphLaunch(h->graph_1, h->stream));
    SFG3_CUDA(cudaEventRecord(h->ev1, h->stream));
    SFG3_CUDA(cudaEventSynchronize(h->ev1));
    SFG3_CUDA(cudaEventElapsedTime(ms, h->ev0, h->ev1));
    h->host_step += nsteps;
    return int(SFG_OK);
  });
}

// Reads a buffer so that the L2 afterwards holds its clean lines (the sink is
// written only on a value the zero-filled buffer never has).
__global__ void __launch_bounds__(256) k_read_flush3(const float4 *__restrict__ b, size_t n4, float *sink) {
  float acc = 0.f;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n4; i += size_t(gridDim.x) * blockDim.x) {
    const float4 v = b[i];
    acc += v.x + v.y + v.z + v.w;
  }
  if (acc == 1234.5f) *sink = acc;
}

int sfg3d_run_timed_flushed(sfg_handle3d *h, int nsteps, size_t flush_bytes, float *ms) {
  return guarded(h, [&]() {
    if (!h->initialized || !ms) return int(SFG_ERR_STATE);
    if (nsteps <= 0 || h->host_step + nsteps > h->opt.nstep) { h->err = "beyond nstep"; return int(SFG_ERR_ARG); }
    if (h->flush_bytes < flush_bytes) {
      if (h->flush) cudaFree(h->flush);
      h->flush = nullptr;
      h->flush_bytes = 0;
      SFG3_CUDA(cudaMalloc(&h->flush, 2 * flush_bytes + 16));
      SFG3_CUDA(cudaMemset(h->flush, 0, 2 * flush_bytes + 16));
      h->flush_bytes = flush_bytes;
    }
    resume(h);
    float total = 0;
    char *fb = reinterpret_cast<char *>(h->flush);
    for (int i = 0; i < nsteps; ++i) {
      // L2 flush outside the timed interval: a write of flush_bytes, then a
      // read of a second buffer, so that no dirty line is left in the cache
      SFG3_CUDA(cudaMemsetAsync(fb, i & 0xff, flush_bytes, h->stream));
      k_read_flush3<<<148 * 8, 256, 0, h->stream>>>(reinterpret_cast<const float4 *>(fb + h->flush_bytes),
                                                    flush_bytes / 16,
                                                    reinterpret_cast<float *>(fb + 2 * h->flush_bytes));
      SFG3_CUDA(cudaEventRecord(h->ev0, h->stream));
      SFG3_CUDA(cudaGraphLaunch(h->graph_1, h->stream));
      SFG3_CUDA(cudaEventRecord(h->ev1, h->stream));
      SFG3_CUDA(cudaEventSynchronize(h->ev1));
      float t = 0;
      SFG3_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
      total += t;
    }
    *ms = total;
    h->host_step += nsteps;
    return int(SFG_OK);
  });
}

int sfg3d_step_io(sfg_handle3d *h, const float *stf_row, float *seis_row) {
  return guarded(h, [&]() {
    if (!h->initialized) return int(SFG_ERR_STATE);
    const int step = h->host_step;
    if (step >= h->opt.nstep) { h->err = "beyond nstep"; return int(SFG_ERR_ARG); }
    if (stf_row && h->nsrc > 0)
      SFG3_CUDA(cudaMemcpyAsync(h->d_stf + size_t(step) * h->nsrc, stf_row, size_t(h->nsrc) * sizeof(float),
                                cudaMemcpyHostToDevice, h->stream));
    resume(h);
    SFG3_CUDA(cudaGraphLaunch(h->graph_1, h->stream));
    h->host_step += 1;
    if (seis_row && h->nrec > 0)
      SFG3_CUDA(cudaMemcpyAsync(seis_row, h->d_seis + size_t(step) * h->ntypes * h->nrec * 3,
                                size_t(h->ntypes) * h->nrec * 3 * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    SFG3_CUDA(cudaStreamSynchronize(h->stream));
    return int(SFG_OK);
  });
}

int sfg3d_time_kernel(sfg_handle3d *h, int which, int reps, float *ms) {
  return guarded(h, [&]() {
    if (!h->initialized || !ms || reps <= 0) return int(SFG_ERR_ARG);
    // time on scratch copies of the mutable state: the fields are saved and restored
    const size_t n = (size_t(h->nglob) * 3 + 4) * sizeof(float);
    float *save = nullptr;
    SFG3_CUDA(cudaMalloc(&save, 2 * n));
    SFG3_CUDA(cudaMemcpyAsync(save, h->d_u, n, cudaMemcpyDeviceToDevice, h->stream));
    SFG3_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(save) + n, h->d_v, n, cudaMemcpyDeviceToDevice, h->stream));
    int step0 = 0;
    SFG3_CUDA(cudaMemcpy(&step0, h->d_step, sizeof(int), cudaMemcpyDeviceToHost));
    SFG3_CUDA(cudaEventRecord(h->ev0, h->stream));
    for (int i = 0; i < reps; ++i) {
      if (which == 0) {
        sfg3::dev::Elem3Args A = h->EA;
        A.step = h->d_step;
        launch_elem(h, A, h->stream);
      } else {
        sfg3::dev::Update3Args U{};
        U.u = h->d_u; U.v = h->d_v; U.minv = h->d_minv; U.inv_start = h->d_inv_start; U.r = h->d_r;
        U.npts = h->nglob; U.dt = float(h->opt.dt); U.dt2 = U.dt / 2; U.dtsq2 = U.dt * U.dt / 2;
        U.predict = 1; U.flag = h->d_flag; U.step = h->d_step; U.advance = 0;
        const int ug = std::max(1, std::min((h->nglob + 255) / 256, h->sm_count * 8));
        sfg3::dev::k_update3d<<<ug, 256, 0, h->stream>>>(U);
      }
    }
    SFG3_CUDA(cudaEventRecord(h->ev1, h->stream));
    SFG3_CUDA(cudaEventSynchronize(h->ev1));
    float t = 0;
    SFG3_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
    *ms = t / reps;
    SFG3_CUDA(cudaMemcpyAsync(h->d_u, save, n, cudaMemcpyDeviceToDevice, h->stream));
    SFG3_CUDA(cudaMemcpyAsync(h->d_v, reinterpret_cast<char *>(save) + n, n, cudaMemcpyDeviceToDevice, h->stream));
    SFG3_CUDA(cudaMemcpyAsync(h->d_step, &step0, sizeof(int), cudaMemcpyHostToDevice, h->stream));
    SFG3_CUDA(cudaStreamSynchronize(h->stream));
    cudaFree(save);
    return int(SFG_OK);
  });
}

int sfg3d_get_info(sfg_handle3d *h, sfg_info3d *info) {
  return guarded(h, [&]() {
    if (!info) return int(SFG_ERR_ARG);
    info->nspec = h->nspec; info->nglob = h->nglob; info->nstep = h->opt.nstep; info->istep = h->host_step;
    info->nrec = h->nrec; info->ntypes = h->ntypes; info->nsig = h->opt.nstep; info->nsrc = h->nsrc;
    info->t0 = h->t0;
    info->device_bytes = h->mem ? h->mem->bytes : 0;
    info->elements_per_block = h->epb;
    info->kernels_per_step = 2 + (h->nrec > 0 ? 1 : 0);
    info->kernel_variant = h->epb >= 6 ? 2 : 1;
    return int(SFG_OK);
  });
}

int sfg3d_get_seismograms(sfg_handle3d *h, float *out, size_t count) {
  return guarded(h, [&]() {
    if (!h->initialized) return int(SFG_ERR_STATE);
    const size_t n = size_t(h->opt.nstep) * h->ntypes * h->nrec * 3;
    if (!out || count < n) { h->err = "output buffer too small"; return int(SFG_ERR_ARG); }
    if (n == 0) return int(SFG_OK);
    SFG3_CUDA(cudaStreamSynchronize(h->stream));
    SFG3_CUDA(cudaMemcpy(out, h->d_seis, n * sizeof(float), cudaMemcpyDeviceToHost));
    return int(SFG_OK);
  });
}

int sfg3d_get_field(sfg_handle3d *h, int which, float *out, size_t count) {
  return guarded(h, [&]() {
    if (!h->initialized) return int(SFG_ERR_STATE);
    const size_t n = size_t(h->nglob) * 3;
    if (!out || count < n) { h->err = "output buffer too small"; return int(SFG_ERR_ARG); }
    if (!h->state_final) { h->err = "fields are mid-step after a timing call; run a step first"; return int(SFG_ERR_STATE); }
    const float *src = which == 0 ? h->d_u : which == 1 ? h->d_v : h->d_a;
    SFG3_CUDA(cudaStreamSynchronize(h->stream));
    SFG3_CUDA(cudaMemcpy(out, src, n * sizeof(float), cudaMemcpyDeviceToHost));
    return int(SFG_OK);
  });
}

int sfg3d_check_finite(sfg_handle3d *h) {
  if (!h || !h->initialized) return 0;
  int f = 0;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return SFG_ERR_CUDA;
  if (cudaMemcpy(&f, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SFG_ERR_CUDA;
  return f ? SFG_ERR_NONFINITE : 0;
}

}  // extern "C"
