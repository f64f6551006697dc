// CPU oracle for the SPECFEM++ 2D per-time-step spectral-element update.
//
// TEST INFRASTRUCTURE ONLY.  This file is a plain C++ restatement of the
// reference algorithm, used as the checker by tests/, by the smoke test and
// as the CPU baseline of bench.py.  The product (libsfg) never links it.
//
// Everything is templated on the arithmetic type so that the same code runs
// in FP32 (the reference's type_real = float) and FP64.  With one thread the
// assembly is serial in element order.  With nthreads > 1 the elements of
// each medium are split into colours (greedy, in element order: no two
// elements of a colour share a global point) and each colour is one OpenMP
// loop with plain adds, colour after colour: every point's contributions are
// summed in colour order whatever the thread count, so a multithreaded FP32
// run is deterministic too.  The reference sums with atomic adds in
// whatever order its threads arrive (compute_stiffness_interaction.tpp:
// 244-245), so no single order is the reference's.
//
// Reference files restated (paths inside the SPECFEM++ tree):
//   GLL points / weights        src/quadrature/gll/gll_library.cpp:102-190
//   hprime(i,j) = l'_j(xi_i)    src/quadrature/gll/lagrange_poly.cpp:161-191
//   Lagrange interpolants       src/quadrature/gll/lagrange_poly.cpp:11-43
//   shape functions (4/9 node)  core/specfem/shape_function/dim2/*.cpp
//   Jacobian                    core/specfem/jacobian/dim2/jacobian.cpp
//   point location              src/algorithms/dim2/locate_point_impl.cpp
//   properties                  include/medium/dim2/elastic/isotropic/material.hpp:66-69,
//                               include/medium/dim2/elastic/isotropic/properties.hpp:71-91,
//                               include/medium/dim2/acoustic/isotropic/properties.hpp:62-72
//   mass matrix                 include/kokkos_kernels/impl/compute_mass_matrix.tpp:95-121
//   Stacey (traction + mass)    include/boundary_conditions/stacey/stacey.tpp:50-80,130-146,296-326,817-853
//   Stacey edge data            core/specfem/assembly/boundaries/dim2/impl/stacey.tpp,
//                               core/specfem/assembly/boundaries/dim2/impl/utilities.hpp
//   edge normals                core/specfem/point/jacobian_matrix.hpp:424-449
//   free surface                include/boundary_conditions/dirichlet/dirichlet.hpp:38-62
//   stiffness                   include/kokkos_kernels/impl/compute_stiffness_interaction.tpp:140-247
//   gradient / divergence       include/algorithms/gradient.hpp:40-82, divergence.hpp:41-74
//   stress                      include/medium/dim2/elastic/isotropic/stress.hpp:38-129,
//                               include/medium/dim2/acoustic/isotropic/stress.hpp:33-53
//   F = J sigma dxi/dx          core/specfem/point/stress.hpp:166-183
//   sources                     include/kokkos_kernels/impl/compute_source_interaction.tpp,
//                               include/medium/dim2/{elastic,acoustic}/isotropic/source.hpp,
//                               core/specfem/assembly/compute_source_array/dim2/impl/compute_source_array_from_vector.cpp,
//                               core/specfem/source/dim2/vector_source/force_source.cpp
//   Ricker STF                  core/specfem/source_time_functions/ricker.cpp, impl/time_functions.hpp:78
//   coupling                    include/kokkos_kernels/impl/compute_coupling.tpp:21-115,
//                               include/medium/dim2/coupling_terms/{acoustic_elastic,elastic_acoustic}.hpp,
//                               core/specfem/assembly/conforming_interfaces/dim2/impl/interface_container.tpp
//   nonconforming coupling      include/kokkos_kernels/impl/compute_coupling.tpp:117-249,
//                               include/algorithms/{transfer.hpp,integrate/coupling_integral1d.hpp},
//                               core/specfem/assembly/nonconforming_interfaces/dim2/impl/*,
//                               core/specfem/assembly/edge_types/dim2/edge_types.cpp,
//                               src/algorithms/dim2/locate_point_impl.cpp:126-198
//   Newmark                     core/specfem/timescheme/newmark.tpp:10-128
//   step order                  core/specfem/solver/time_marching.tpp:33-83
//   seismograms                 include/kokkos_kernels/impl/compute_seismogram.tpp,
//                               include/medium/dim2/acoustic/isotropic/wavefield.hpp,
//                               core/specfem/assembly/receivers/dim2/impl/seismogram_iterator.hpp:37-53
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle2d.h"

namespace {

constexpr int NG = 5;
constexpr int NP = NG * NG;

// ---------------------------------------------------------------- GLL ---
double legendre(double x, int n) {
  double p0 = 1.0, p1 = x;
  if (n == 0) return 1.0;
  for (int k = 1; k < n; ++k) {
    double p2 = ((2.0 * k + 1.0) * x * p1 - k * p0) / (k + 1.0);
    p0 = p1;
    p1 = p2;
  }
  return p1;
}

// GLL nodes of degree N=4: the roots of (1-x^2) P'_4(x); closed form for NGLL=5.
void gll_nodes(double z[NG], double w[NG]) {
  const double a = std::sqrt(3.0 / 7.0);
  z[0] = -1.0; z[1] = -a; z[2] = 0.0; z[3] = a; z[4] = 1.0;
  const int N = NG - 1;
  for (int i = 0; i < NG; ++i) {
    double p = legendre(z[i], N);
    w[i] = 2.0 / (N * (N + 1.0) * p * p);
  }
}

// hprime[i][j] = l'_j(xi_i): derivative of the j-th Lagrange polynomial at node i.
void gll_hprime(const double z[NG], double hp[NG][NG]) {
  const int N = NG - 1;
  for (int i = 0; i < NG; ++i)
    for (int j = 0; j < NG; ++j) {
      if (i == 0 && j == 0) hp[i][j] = -0.25 * N * (N + 1.0);
      else if (i == N && j == N) hp[i][j] = 0.25 * N * (N + 1.0);
      else if (i == j) hp[i][j] = 0.0;
      else hp[i][j] = legendre(z[i], N) / (legendre(z[j], N) * (z[i] - z[j]));
    }
}

template <typename T>
void lagrange_interp(T xi, const T z[NG], T h[NG], T hp[NG]) {
  for (int d = 0; d < NG; ++d) {
    T p1 = 1, p2 = 1, sum = 0;
    for (int i = 0; i < NG; ++i) {
      if (i == d) continue;
      p1 *= (xi - z[i]);
      p2 *= (z[d] - z[i]);
      T p3 = 1;
      for (int j = 0; j < NG; ++j)
        if (j != d && j != i) p3 *= (xi - z[j]);
      sum += p3;
    }
    T inv = T(1) / p2;
    h[d] = p1 * inv;
    hp[d] = sum * inv;
  }
}

// ------------------------------------------------------ shape functions ---
template <typename T>
void shape2d(T xi, T ga, int ngnod, T *s) {
  if (ngnod == 4) {
    s[0] = T(0.25) * (xi - 1) * (ga - 1);
    s[1] = T(-0.25) * (xi + 1) * (ga - 1);
    s[2] = T(0.25) * (xi + 1) * (ga + 1);
    s[3] = T(-0.25) * (xi - 1) * (ga + 1);
  } else {
    s[0] = T(0.25) * (xi - 1) * xi * (ga - 1) * ga;
    s[1] = T(0.25) * (xi + 1) * xi * (ga - 1) * ga;
    s[2] = T(0.25) * (xi + 1) * xi * (ga + 1) * ga;
    s[3] = T(0.25) * (xi - 1) * xi * (ga + 1) * ga;
    s[4] = T(0.5) * (1 - xi * xi) * (ga - 1) * ga;
    s[5] = T(0.5) * (xi + 1) * xi * (1 - ga * ga);
    s[6] = T(0.5) * (1 - xi * xi) * (ga + 1) * ga;
    s[7] = T(0.5) * (xi - 1) * xi * (1 - ga * ga);
    s[8] = (1 - xi * xi) * (1 - ga * ga);
  }
}

template <typename T>
void dshape2d(T xi, T ga, int ngnod, T *dx, T *dg) {
  if (ngnod == 4) {
    const T sp = xi + 1, sm = xi - 1, tp = ga + 1, tm = ga - 1;
    dx[0] = T(0.25) * tm; dx[1] = T(-0.25) * tm; dx[2] = T(0.25) * tp; dx[3] = T(-0.25) * tp;
    dg[0] = T(0.25) * sm; dg[1] = T(-0.25) * sp; dg[2] = T(0.25) * sp; dg[3] = T(-0.25) * sm;
  } else {
    const T sp = xi + 1, sm = xi - 1, tp = ga + 1, tm = ga - 1;
    const T s2 = xi * 2, t2 = ga * 2, ss = xi * xi, tt = ga * ga, st = xi * ga;
    dx[0] = T(0.25) * tm * ga * (s2 - 1); dx[1] = T(0.25) * tm * ga * (s2 + 1);
    dx[2] = T(0.25) * tp * ga * (s2 + 1); dx[3] = T(0.25) * tp * ga * (s2 - 1);
    dg[0] = T(0.25) * sm * xi * (t2 - 1); dg[1] = T(0.25) * sp * xi * (t2 - 1);
    dg[2] = T(0.25) * sp * xi * (t2 + 1); dg[3] = T(0.25) * sm * xi * (t2 + 1);
    dx[4] = -st * tm; dx[5] = T(0.5) * (1 - tt) * (s2 + 1);
    dx[6] = -st * tp; dx[7] = T(0.5) * (1 - tt) * (s2 - 1);
    dg[4] = T(0.5) * (1 - ss) * (t2 - 1); dg[5] = -st * sp;
    dg[6] = T(0.5) * (1 - ss) * (t2 + 1); dg[7] = -st * sm;
    dx[8] = -s2 * (1 - tt); dg[8] = -t2 * (1 - ss);
  }
}

template <typename T>
struct Jac {
  T xix, gammax, xiz, gammaz, jac;
};

template <typename T>
Jac<T> jacobian_at(const T *cx, const T *cz, int ngnod, T xi, T ga) {
  T dx[9], dg[9];
  dshape2d<T>(xi, ga, ngnod, dx, dg);
  T xxi = 0, zxi = 0, xga = 0, zga = 0;
  for (int n = 0; n < ngnod; ++n) {
    xxi += dx[n] * cx[n]; zxi += dx[n] * cz[n];
    xga += dg[n] * cx[n]; zga += dg[n] * cz[n];
  }
  T j = xxi * zga - xga * zxi;
  return {zga / j, -zxi / j, -xga / j, xxi / j, j};
}

template <typename T>
void location_at(const T *cx, const T *cz, int ngnod, T xi, T ga, T &x, T &z) {
  T s[9];
  shape2d<T>(xi, ga, ngnod, s);
  x = 0; z = 0;
  for (int n = 0; n < ngnod; ++n) { x += s[n] * cx[n]; z += s[n] * cz[n]; }
}

// -------------------------------------------------------------- model ---
enum { BOTTOM = 0, RIGHT = 1, TOP = 2, LEFT = 3 };
enum { MED_ACOUSTIC = 0, MED_ELASTIC = 1 };

bool on_edge(int type, int iz, int ix) {
  return (type == TOP && iz == NG - 1) || (type == BOTTOM && iz == 0) ||
         (type == LEFT && ix == 0) || (type == RIGHT && ix == NG - 1);
}

// (xi, gamma) of the point at local coordinate c along an edge: xi runs along
// bottom and top, gamma along left and right.
template <typename S>
void edge_local(int type, S c, S &xi, S &ga) {
  if (type == BOTTOM) { xi = c; ga = S(-1); }
  else if (type == RIGHT) { xi = S(1); ga = c; }
  else if (type == TOP) { xi = c; ga = S(1); }
  else { xi = S(-1); ga = c; }
}

// Local coordinate along one edge of an element of the point closest to
// (X, Z): Newton steps on the edge coordinate from 0 with the inverse
// Jacobian row of that coordinate, clamped to [-1, 1], stopping at an end
// whose step points outside (src/algorithms/dim2/locate_point_impl.cpp:126-198).
template <typename S>
S edge_coordinate(S X, S Z, const S *cx, const S *cz, int ngnod, int type) {
  const S deriv_eps = S(1e-12);
  S xi, ga;
  edge_local<S>(type, S(0), xi, ga);
  S &c = (type == BOTTOM || type == TOP) ? xi : ga;
  for (int it = 0; it < 100; ++it) {
    S x, z;
    location_at<S>(cx, cz, ngnod, xi, ga, x, z);
    const Jac<S> J = jacobian_at<S>(cx, cz, ngnod, xi, ga);
    const S dx = -(x - X), dz = -(z - Z);
    const S d = (type == BOTTOM || type == TOP) ? J.xix * dx + J.xiz * dz
                                                : J.gammax * dx + J.gammaz * dz;
    if (c == S(-1) && d < -deriv_eps) return S(-1);
    if (c == S(1) && d > deriv_eps) return S(1);
    c += d;
    if (c > S(1)) c = S(1);
    else if (c < S(-1)) c = S(-1);
    if (std::abs(d) < deriv_eps) break;
  }
  return c;
}

template <typename T>
struct Sim {
  const OracleInput2D &in;
  int nspec, nglob = 0, ngnod;
  T z[NG], w[NG], hp[NG][NG];
  T hpw[NG][NG];                    // hp[l][i] * w[l] rounded once (device evaluation order)
  std::vector<int> ibool;           // [nspec][25]
  std::vector<T> xix, xiz, gax, gaz, jac;  // [nspec][25]
  std::vector<T> gx, gz;            // coordinates of local points
  std::vector<int> medium;          // [nspec]
  // elastic: kappa, mu, rho; acoustic: rho_inverse, kappa
  std::vector<T> p_kappa, p_mu, p_rho, p_rhoinv;
  // anisotropic elastic (when in.aniso): c11, c13, c15, c33, c35, c55 per point
  std::vector<T> p_c[6];
  // Cosserat (when in.cosserat): rho, kappa, mu, nu, j, lambda_c, mu_c, nu_c
  std::vector<T> p_cs[8];
  // poroelastic (when in.poro): phi, rho_s, rho_f, tortuosity, mu_G, H_Biot,
  // C_Biot, M_Biot, permxx, permxz, permzz, eta_f
  std::vector<T> p_po[12];
  // Stacey point data per element (dense, tag 0/1)
  std::vector<uint8_t> st_tag, fs_tag;   // [nspec][25]
  std::vector<T> st_nx, st_nz, st_w;     // [nspec][25]
  // fields: acoustic (1 comp) and elastic (ncomp_el comps), indexed by global id
  int ncomp_el;
  std::vector<T> ua, va, aa, minv_a;
  std::vector<T> ue, ve, ae, minv_e;    // [nglob][ncomp_el]
  std::vector<uint8_t> is_ac_glob, is_el_glob;
  // coupling point lists
  struct CPoint { int ispec, iz, ix, iglob; T nx, nz, fac; };
  std::vector<CPoint> cpl_ac, cpl_el;   // self acoustic / self elastic
  // nonconforming acoustic-elastic edge pairs: the self edge's points, the
  // coupled edge's points, and on the NG-point intersection quadrature the
  // self / coupled transfer functions, weight * |dx/dxi| and the self
  // element's outward unit normal
  struct NCEdge {
    int self_e, self_t, cpl_e, cpl_t;
    int gs[NG], gc[NG];
    uint8_t fs[NG];
    T ts[NG][NG], tc[NG][NG];   // [quadrature point][edge point]
    T fac[NG], nx[NG], nz[NG];
  };
  std::vector<NCEdge> nc_ac, nc_el;     // self acoustic / self elastic
  // sources
  struct Src { int ispec; int medium; T arr[4][NP]; int ncomp; std::vector<T> stf; };
  std::vector<Src> srcs;
  struct Rec { int ispec; T h[NP]; };
  std::vector<Rec> recs;
  T dt;

  explicit Sim(const OracleInput2D &in_) : in(in_), nspec(in_.nspec), ngnod(in_.ngnod) {}

  void setup() {
    double zd[NG], wd[NG], hpd[NG][NG];
    gll_nodes(zd, wd);
    gll_hprime(zd, hpd);
    for (int i = 0; i < NG; ++i) {
      z[i] = T(zd[i]); w[i] = T(wd[i]);
      for (int j = 0; j < NG; ++j) { hp[i][j] = T(hpd[i][j]); hpw[i][j] = T(hpd[i][j] * wd[i]); }
    }
    dt = T(in.dt);
    ncomp_el = in.poro ? 4 : in.cosserat ? 3 : in.elastic_sh ? 1 : 2;
    number_points();
    geometry();
    properties();
    boundaries();
    coupling();
    nonconforming();
    mass();
    sources();
    receivers();
  }

  void setup_geometry_only() {
    double zd[NG], wd[NG], hpd[NG][NG];
    gll_nodes(zd, wd);
    gll_hprime(zd, hpd);
    for (int i = 0; i < NG; ++i) {
      z[i] = T(zd[i]); w[i] = T(wd[i]);
      for (int j = 0; j < NG; ++j) hp[i][j] = T(hpd[i][j]);
    }
    number_points();
    geometry();
  }

  // Global numbering by element topology: corners by control-node id, edge
  // points by (corner pair, position), element-interior points unique.
  void number_points() {
    ibool.assign(size_t(nspec) * NP, -1);
    std::map<int, int> corner_id;
    std::map<std::tuple<int, int, int>, int> edge_id;
    const int cz[4] = {0, 0, NG - 1, NG - 1}, cxx[4] = {0, NG - 1, NG - 1, 0};
    for (int e = 0; e < nspec; ++e) {
      const int *kn = in.knods + size_t(e) * ngnod;
      for (int c = 0; c < 4; ++c) {
        auto it = corner_id.find(kn[c]);
        int id;
        if (it == corner_id.end()) { id = nglob++; corner_id[kn[c]] = id; }
        else id = it->second;
        ibool[size_t(e) * NP + cz[c] * NG + cxx[c]] = id;
      }
      // edges: (corner A at position 0, corner B at position 4, point(t))
      for (int ed = 0; ed < 4; ++ed) {
        int A, B;
        if (ed == BOTTOM) { A = 0; B = 1; } else if (ed == RIGHT) { A = 1; B = 2; }
        else if (ed == TOP) { A = 3; B = 2; } else { A = 0; B = 3; }
        for (int t = 1; t < NG - 1; ++t) {
          int iz, ix;
          if (ed == BOTTOM) { iz = 0; ix = t; } else if (ed == RIGHT) { iz = t; ix = NG - 1; }
          else if (ed == TOP) { iz = NG - 1; ix = t; } else { iz = t; ix = 0; }
          int na = kn[A], nb = kn[B];
          int k = na < nb ? t : NG - 1 - t;
          auto key = std::make_tuple(std::min(na, nb), std::max(na, nb), k);
          auto it = edge_id.find(key);
          int id;
          if (it == edge_id.end()) { id = nglob++; edge_id[key] = id; }
          else id = it->second;
          ibool[size_t(e) * NP + iz * NG + ix] = id;
        }
      }
      for (int iz = 1; iz < NG - 1; ++iz)
        for (int ix = 1; ix < NG - 1; ++ix) ibool[size_t(e) * NP + iz * NG + ix] = nglob++;
    }
  }

  template <typename S>
  void ctrl(int e, S *cx, S *cz) const {
    for (int n = 0; n < ngnod; ++n) {
      int id = in.knods[size_t(e) * ngnod + n];
      cx[n] = S(in.coorg[2 * size_t(id)]);
      cz[n] = S(in.coorg[2 * size_t(id) + 1]);
    }
  }

  template <typename S>
  void geometry_in() {
    size_t n = size_t(nspec) * NP;
    xix.resize(n); xiz.resize(n); gax.resize(n); gaz.resize(n); jac.resize(n);
    gx.resize(n); gz.resize(n);
    S zs[NG];
    for (int i = 0; i < NG; ++i) zs[i] = setup_z<S>(i);
    for (int e = 0; e < nspec; ++e) {
      S cx[9], cz[9];
      ctrl<S>(e, cx, cz);
      for (int iz = 0; iz < NG; ++iz)
        for (int ix = 0; ix < NG; ++ix) {
          size_t p = size_t(e) * NP + iz * NG + ix;
          Jac<S> J = jacobian_at<S>(cx, cz, ngnod, zs[ix], zs[iz]);
          xix[p] = T(J.xix); gax[p] = T(J.gammax); xiz[p] = T(J.xiz); gaz[p] = T(J.gammaz);
          jac[p] = T(J.jac);
          S x, zz;
          location_at<S>(cx, cz, ngnod, zs[ix], zs[iz], x, zz);
          gx[p] = T(x); gz[p] = T(zz);
        }
    }
  }

  template <typename S>
  S setup_z(int i) const {
    double zd[NG], wd[NG];
    gll_nodes(zd, wd);
    return S(zd[i]);
  }

  void geometry() {
    if (in.setup_in_run_precision) geometry_in<T>();
    else geometry_in<double>();
  }

  void properties() {
    size_t n = size_t(nspec) * NP;
    medium.assign(in.medium, in.medium + nspec);
    p_kappa.resize(n); p_mu.resize(n); p_rho.resize(n); p_rhoinv.resize(n);
    for (size_t p = 0; p < n; ++p) {
      const T rho = T(in.rho[p]), vp = T(in.vp[p]), vs = T(in.vs[p]);
      if (medium[p / NP] == MED_ELASTIC) {
        p_mu[p] = rho * vs * vs;
        p_kappa[p] = rho * (vp * vp - T(4.0 / 3.0) * vs * vs);
        p_rho[p] = rho;
      } else {
        p_rhoinv[p] = T(1) / rho;
        p_kappa[p] = rho * vp * vp;
        p_rho[p] = rho;
      }
    }
    if (in.cosserat) {
      if (in.elastic_sh || in.aniso) throw std::runtime_error("Cosserat media are P-SV-T only");
      for (int k = 0; k < 8; ++k) {
        p_cs[k].resize(n);
        for (size_t p = 0; p < n; ++p) p_cs[k][p] = T(in.cosserat[p * 8 + k]);
      }
      for (size_t p = 0; p < n; ++p)
        if (medium[p / NP] == MED_ELASTIC) {
          p_rho[p] = p_cs[0][p]; p_kappa[p] = p_cs[1][p]; p_mu[p] = p_cs[2][p];
        }
    }
    if (in.poro) {
      if (in.elastic_sh || in.aniso || in.cosserat)
        throw std::runtime_error("poroelastic media are P-SV isotropic only");
      for (int k = 0; k < 12; ++k) p_po[k].assign(n, T(0));
      for (size_t p = 0; p < n; ++p) {
        if (medium[p / NP] != MED_ELASTIC) continue;
        const double *v = in.poro + p * 13;
        // material.hpp: Q_mu must be 9999 (no attenuation); Biot coefficients
        // with the reference's mixed float / double literal arithmetic
        if (std::abs(T(v[12]) - 9999.0) > 1e-6)
          throw std::runtime_error("poroelastic attenuation is not implemented");
        const T rhos = T(v[0]), rhof = T(v[1]), phi = T(v[2]), tort = T(v[3]);
        const T ks = T(v[7]), kf = T(v[8]), kfr = T(v[9]), etaf = T(v[10]), mufr = T(v[11]);
        const T D = T(double(ks) * (1.0 + double(phi) * (double(ks / kf) - 1.0)));
        const T fac = T(1.0 / double(D - kfr));
        const T H = T(double((ks - kfr) * (ks - kfr) * fac + kfr) + 4.0 / 3.0 * double(mufr));
        const T C = ks * (ks - kfr) * fac;
        const T M = ks * ks * fac;
        const T vals[12] = {phi, rhos, rhof, tort, mufr, H, C, M, T(v[4]), T(v[5]), T(v[6]), etaf};
        for (int k = 0; k < 12; ++k) p_po[k][p] = vals[k];
      }
    }
    if (in.aniso) {
      if (in.elastic_sh) throw std::runtime_error("anisotropic SH is outside this path");
      for (int k = 0; k < 6; ++k) {
        p_c[k].resize(n);
        for (size_t p = 0; p < n; ++p) p_c[k][p] = T(in.aniso[p * 6 + k]);
      }
    }
  }

  T lp2m(size_t p) const { return p_kappa[p] + T(4.0 / 3.0) * p_mu[p]; }
  // poroelastic rho_bar = (1 - phi) rho_s + phi rho_f (poroelastic/isotropic/properties.hpp)
  T rho_bar(size_t p) const { return ((T(1) - p_po[0][p]) * p_po[1][p]) + (p_po[0][p] * p_po[2][p]); }
  // anisotropic: rho vp = sqrt(rho c33), rho vs = sqrt(rho c55)
  // (include/medium/dim2/elastic/anisotropic/properties.hpp:88-94)
  T rho_vp(size_t p) const {
    return in.aniso ? std::sqrt(p_rho[p] * p_c[3][p]) : std::sqrt(lp2m(p) / p_rho[p]) * p_rho[p];
  }
  T rho_vs(size_t p) const {
    if (in.cosserat)   // rho sqrt((mu + nu) / rho) (stacey.tpp:183-230)
      return p_rho[p] * std::sqrt((p_mu[p] + p_cs[3][p]) / p_rho[p]);
    return in.aniso ? std::sqrt(p_rho[p] * p_c[5][p]) : std::sqrt(p_rho[p] * p_mu[p]);
  }
  // Cosserat rotational impedance j sqrt((mu_c + nu_c) / j)
  T j_vt(size_t p) const { return p_cs[4][p] * std::sqrt((p_cs[6][p] + p_cs[7][p]) / p_cs[4][p]); }
  T rho_vpinv(size_t p) const { return std::sqrt(p_rhoinv[p] * (T(1) / p_kappa[p])); }

  void normal(size_t p, int type, T &nx, T &nz) const {
    if (type == BOTTOM) { nx = T(-1) * gax[p] * jac[p]; nz = T(-1) * gaz[p] * jac[p]; }
    else if (type == TOP) { nx = gax[p] * jac[p]; nz = gaz[p] * jac[p]; }
    else if (type == LEFT) { nx = T(-1) * xix[p] * jac[p]; nz = T(-1) * xiz[p] * jac[p]; }
    else { nx = xix[p] * jac[p]; nz = xiz[p] * jac[p]; }
  }

  void boundaries() {
    size_t n = size_t(nspec) * NP;
    st_tag.assign(n, 0); fs_tag.assign(n, 0);
    st_nx.assign(n, 0); st_nz.assign(n, 0); st_w.assign(n, 0);
    // entries applied in order of appearance; a later edge of the same element
    // overwrites the normal/weight of a shared corner point (stacey.tpp).
    for (int i = 0; i < in.nabs; ++i) {
      int e = in.abs_ispec[i], type = in.abs_type[i];
      for (int iz = 0; iz < NG; ++iz)
        for (int ix = 0; ix < NG; ++ix) {
          if (!on_edge(type, iz, ix)) continue;
          size_t p = size_t(e) * NP + iz * NG + ix;
          st_tag[p] = 1;
          normal(p, type, st_nx[p], st_nz[p]);
          st_w[p] = (type == LEFT || type == RIGHT) ? w[iz] : w[ix];
        }
    }
    for (int i = 0; i < in.nfree; ++i) {
      int e = in.free_ispec[i], type = in.free_type[i];
      for (int iz = 0; iz < NG; ++iz)
        for (int ix = 0; ix < NG; ++ix)
          if (on_edge(type, iz, ix)) fs_tag[size_t(e) * NP + iz * NG + ix] = 1;
    }
  }

  // acoustic/elastic shared edges: for each element pair sharing an edge,
  // one self point list per side (interface_container.tpp).
  void coupling() {
    std::map<std::pair<int, int>, std::vector<std::pair<int, int>>> edges;  // corner pair -> (elem, type)
    for (int e = 0; e < nspec; ++e) {
      const int *kn = in.knods + size_t(e) * ngnod;
      const int ends[4][2] = {{0, 1}, {1, 2}, {3, 2}, {0, 3}};
      for (int ed = 0; ed < 4; ++ed) {
        int a = kn[ends[ed][0]], b = kn[ends[ed][1]];
        edges[{std::min(a, b), std::max(a, b)}].push_back({e, ed});
      }
    }
    for (auto &kv : edges) {
      if (kv.second.size() != 2) continue;
      auto [e1, t1] = kv.second[0];
      auto [e2, t2] = kv.second[1];
      if (medium[e1] == medium[e2]) continue;
      if (ncomp_el >= 3)
        throw std::runtime_error("Cosserat and poroelastic media are not coupled to acoustic ones here");
      for (auto [e, t] : {std::make_pair(e1, t1), std::make_pair(e2, t2)}) {
        for (int iz = 0; iz < NG; ++iz)
          for (int ix = 0; ix < NG; ++ix) {
            if (!on_edge(t, iz, ix)) continue;
            size_t p = size_t(e) * NP + iz * NG + ix;
            CPoint c;
            c.ispec = e; c.iz = iz; c.ix = ix; c.iglob = ibool[p];
            normal(p, t, c.nx, c.nz);
            c.fac = (t == BOTTOM || t == TOP) ? w[ix] : w[iz];
            (medium[e] == MED_ACOUSTIC ? cpl_ac : cpl_el).push_back(c);
          }
      }
    }
  }

  // Nonconforming acoustic-elastic edges from the mesh adjacency records
  // (core/specfem/assembly/edge_types/dim2/edge_types.cpp: a nonconforming
  // record between different media and its reverse record give the self and
  // coupled edges).  Per pair, the intersection of the two edges in the self
  // edge's local coordinate carries an NG-point GLL quadrature mapped
  // linearly onto it; its points are located on the coupled edge, and the
  // Lagrange interpolants there are the transfer functions
  // (nonconforming_interfaces/dim2/impl/compute_intersection.cpp:49-167,
  // compute_intersection.tpp:13-122).  The quadrature factor w_q |dx/dxi|
  // and the self element's outward normal come from the derivative of the
  // mapped quadrature points (impl/interface_container.tpp:20-180).
  template <typename S>
  void nonconforming_in() {
    if (!in.adjacency || in.nadj <= 0) return;
    std::map<std::pair<int, int>, int> orient;
    for (int r = 0; r < in.nadj; ++r) {
      const int *a = in.adjacency + 4 * size_t(r);
      if (a[2] == 3) orient[{a[0], a[1]}] = a[3];
      else if (a[2] != 1) throw std::runtime_error("Unknown connection type in adjacency graph.");
    }
    S zs[NG], ws[NG], hps[NG][NG];
    {
      double zd[NG], wd[NG], hpd[NG][NG];
      gll_nodes(zd, wd);
      gll_hprime(zd, hpd);
      for (int i = 0; i < NG; ++i) {
        zs[i] = S(zd[i]); ws[i] = S(wd[i]);
        for (int j = 0; j < NG; ++j) hps[i][j] = S(hpd[i][j]);
      }
    }
    auto ends = [](int t, int &a, int &b) {
      if (t == BOTTOM) { a = 0; b = 1; } else if (t == RIGHT) { a = 1; b = 2; }
      else if (t == TOP) { a = 3; b = 2; } else { a = 0; b = 3; }
    };
    auto edge_point = [](int t, int k) {
      return t == BOTTOM ? k : t == RIGHT ? k * NG + NG - 1 : t == TOP ? (NG - 1) * NG + k : k * NG;
    };
    for (const auto &kv : orient) {
      const int e1 = kv.first.first, e2 = kv.first.second, t1 = kv.second;
      if (medium[e1] == medium[e2]) continue;
      const auto back = orient.find({e2, e1});
      if (back == orient.end())
        throw std::runtime_error("Non-symmetric adjacency graph detected in `compute_intersection`.");
      const int t2 = back->second;
      if (t1 > LEFT || t2 > LEFT) throw std::runtime_error("compute_intersection must be given edges");
      if (ncomp_el != 2)
        throw std::runtime_error("nonconforming coupling: P-SV elastic media only");
      NCEdge E;
      E.self_e = e1; E.self_t = t1; E.cpl_e = e2; E.cpl_t = t2;
      S c1x[9], c1z[9], c2x[9], c2z[9];
      ctrl<S>(e1, c1x, c1z);
      ctrl<S>(e2, c2x, c2z);
      int a1, b1, a2, b2;
      ends(t1, a1, b1);
      ends(t2, a2, b2);
      const S p2lo = edge_coordinate<S>(c2x[a2], c2z[a2], c1x, c1z, ngnod, t1);
      const S p2hi = edge_coordinate<S>(c2x[b2], c2z[b2], c1x, c1z, ngnod, t1);
      const S p1lo = edge_coordinate<S>(c1x[a1], c1z[a1], c2x, c2z, ngnod, t2);
      const S p1hi = edge_coordinate<S>(c1x[b1], c1z[b1], c2x, c2z, ngnod, t2);
      const S min1 = std::min(p2lo, p2hi), max1 = std::max(p2lo, p2hi);
      const S min2 = std::min(p1lo, p1hi), max2 = std::max(p1lo, p1hi);
      if (min1 > max1 - S(1e-5) || min2 > max2 - S(1e-5))
        throw std::runtime_error("nonconforming edges without an intersection");
      S ts[NG][NG], tc[NG][NG], hdum[NG];
      for (int q = 0; q < NG; ++q) {
        const S c1 = S(0.5) * ((max1 - min1) * zs[q] + (max1 + min1));
        S xi, ga, X, Z;
        edge_local<S>(t1, c1, xi, ga);
        location_at<S>(c1x, c1z, ngnod, xi, ga, X, Z);
        const S c2 = edge_coordinate<S>(X, Z, c2x, c2z, ngnod, t2);
        lagrange_interp<S>(c1, zs, ts[q], hdum);
        lagrange_interp<S>(c2, zs, tc[q], hdum);
      }
      S lx[NG], lz[NG];
      for (int k = 0; k < NG; ++k) {
        S lc = 0;
        for (int i = 0; i < NG; ++i) lc += ts[k][i] * zs[i];
        S xi, ga;
        edge_local<S>(t1, lc, xi, ga);
        location_at<S>(c1x, c1z, ngnod, xi, ga, lx[k], lz[k]);
      }
      for (int q = 0; q < NG; ++q) {
        S drx = 0, drz = 0;
        for (int k = 0; k < NG; ++k) { drx += hps[q][k] * lx[k]; drz += hps[q][k] * lz[k]; }
        const S fac = ws[q] * std::sqrt(drx * drx + drz * drz);
        S nx = drz, nz = -drx;
        S mag = std::sqrt(nx * nx + nz * nz);
        if (t1 == TOP || t1 == LEFT) mag *= S(-1);
        E.fac[q] = T(fac); E.nx[q] = T(nx / mag); E.nz[q] = T(nz / mag);
        for (int i = 0; i < NG; ++i) { E.ts[q][i] = T(ts[q][i]); E.tc[q][i] = T(tc[q][i]); }
      }
      for (int k = 0; k < NG; ++k) {
        const size_t ps = size_t(e1) * NP + edge_point(t1, k);
        E.gs[k] = ibool[ps];
        E.fs[k] = fs_tag[ps];
        E.gc[k] = ibool[size_t(e2) * NP + edge_point(t2, k)];
      }
      (medium[e1] == MED_ACOUSTIC ? nc_ac : nc_el).push_back(E);
    }
  }

  void nonconforming() {
    if (in.setup_in_run_precision) nonconforming_in<T>();
    else nonconforming_in<double>();
  }

  // Stacey traction (stacey.tpp:50-80 P-SV, :130-146 SH, :296-326 acoustic)
  void stacey(size_t p, const T *vel, T *acc) const {
    const T nx = st_nx[p], nz = st_nz[p];
    const T j1 = std::sqrt(nx * nx + nz * nz);
    if (medium[p / NP] == MED_ACOUSTIC) {
      const T f = st_w[p] * j1;
      acc[0] += T(-1) * f * rho_vpinv(p) * vel[0];
    } else if (ncomp_el == 1) {
      const T f = st_w[p] * j1;
      acc[0] += T(-1) * f * rho_vs(p) * vel[0];
    } else {
      const T vn = vel[0] * nx + vel[1] * nz;
      const T dn[2] = {nx, nz};
      T fac[2];
      for (int c = 0; c < 2; ++c)
        fac[c] = ((vn * dn[c] / (j1 * j1)) * (rho_vp(p) - rho_vs(p))) + vel[c] * rho_vs(p);
      acc[0] += T(-1) * fac[0] * j1 * st_w[p];
      acc[1] += T(-1) * fac[1] * j1 * st_w[p];
      if (ncomp_el == 3) acc[2] += T(-1) * j_vt(p) * vel[2] * j1 * st_w[p];
    }
  }

  void mass() {
    ua.assign(nglob, 0); va.assign(nglob, 0); aa.assign(nglob, 0); minv_a.assign(nglob, 0);
    size_t ne = size_t(nglob) * ncomp_el;
    ue.assign(ne, 0); ve.assign(ne, 0); ae.assign(ne, 0); minv_e.assign(ne, 0);
    is_ac_glob.assign(nglob, 0); is_el_glob.assign(nglob, 0);
    for (int e = 0; e < nspec; ++e)
      for (int iz = 0; iz < NG; ++iz)
        for (int ix = 0; ix < NG; ++ix) {
          size_t p = size_t(e) * NP + iz * NG + ix;
          int g = ibool[p];
          T fac = w[ix] * w[iz] * jac[p];
          if (medium[e] == MED_ACOUSTIC) {
            is_ac_glob[g] = 1;
            T m = (T(1) / p_kappa[p]) * fac;
            if (st_tag[p]) {
              T v = T(-1) * dt * T(0.5);
              T acc = m;
              stacey(p, &v, &acc);
              m = acc;
            }
            minv_a[g] += m;
          } else {
            is_el_glob[g] = 1;
            // Cosserat: rho, rho, j (isotropic_cosserat/mass_matrix.tpp);
            // poroelastic: rho_bar - phi rho_f / tort twice, then
            // (rho_f tort rho_bar - phi rho_f^2) / (phi rho_bar) twice
            // (poroelastic/isotropic/mass_matrix.tpp)
            T m[4] = {p_rho[p] * fac, p_rho[p] * fac, ncomp_el == 3 ? p_cs[4][p] * fac : T(0), T(0)};
            if (ncomp_el == 4) {
              const T phi = p_po[0][p], rhof = p_po[2][p], tort = p_po[3][p], rb = rho_bar(p);
              const T solid = rb - phi * rhof / tort;
              const T fluid = (rhof * tort * rb - phi * rhof * rhof) / (phi * rb);
              m[0] = solid * fac; m[1] = solid * fac; m[2] = fluid * fac; m[3] = fluid * fac;
            }
            if (st_tag[p]) {
              if (ncomp_el == 4) throw std::runtime_error("Stacey edges on poroelastic media are outside this path");
              T v[3] = {T(-1) * dt * T(0.5), T(-1) * dt * T(0.5), T(-1) * dt * T(0.5)};
              stacey(p, v, m);
            }
            for (int c = 0; c < ncomp_el; ++c) minv_e[size_t(g) * ncomp_el + c] += m[c];
          }
        }
    for (int g = 0; g < nglob; ++g) {
      if (is_ac_glob[g]) minv_a[g] = T(1) / minv_a[g];
      if (is_el_glob[g])
        for (int c = 0; c < ncomp_el; ++c)
          minv_e[size_t(g) * ncomp_el + c] = T(1) / minv_e[size_t(g) * ncomp_el + c];
    }
  }

  // ------------------------------------------------- point location ---
  // Closest GLL point, then Newton iterations from the element centre in that
  // element and the elements sharing a corner with it (locate_point_impl.cpp).
  // Ties (a point on an edge or corner shared by several elements) go to the
  // first element in mesh order: a candidate replaces the current choice only
  // when it is closer by more than 1e-9 of the mesh extent.
  template <typename S>
  std::tuple<int, double, double> locate_in(double X, double Z) const {
    const S x = S(X), zz = S(Z);
    double xmin = 1e300, xmax = -1e300, zmin = 1e300, zmax = -1e300;
    for (int i = 0; i < in.npgeo; ++i) {
      xmin = std::min(xmin, in.coorg[2 * i]); xmax = std::max(xmax, in.coorg[2 * i]);
      zmin = std::min(zmin, in.coorg[2 * i + 1]); zmax = std::max(zmax, in.coorg[2 * i + 1]);
    }
    const S tol = S(1e-9 * std::max(xmax - xmin, zmax - zmin));
    S best = std::numeric_limits<S>::max();
    int eg = -1;
    for (int e = 0; e < nspec; ++e)
      for (int q = 0; q < NP; ++q) {
        size_t p = size_t(e) * NP + q;
        S dx = S(gx[p]) - x, dz = S(gz[p]) - zz;
        S d = std::sqrt(dx * dx + dz * dz);
        if (d < best - tol) { best = d; eg = e; }
      }
    std::vector<int> cand{eg};
    const int *kg = in.knods + size_t(eg) * ngnod;
    for (int e = 0; e < nspec; ++e) {
      if (e == eg) continue;
      const int *ke = in.knods + size_t(e) * ngnod;
      bool share = false;
      for (int a = 0; a < 4 && !share; ++a)
        for (int b = 0; b < 4; ++b)
          if (kg[a] == ke[b]) { share = true; break; }
      if (share) cand.push_back(e);
    }
    S fd = std::numeric_limits<S>::max();
    int es = -1; S xs = -9999, gs = -9999;
    for (int e : cand) {
      S cx[9], cz[9];
      ctrl<S>(e, cx, cz);
      S xi = 0, ga = 0;
      for (int it = 0; it < 100; ++it) {
        S lx, lz;
        location_at<S>(cx, cz, ngnod, xi, ga, lx, lz);
        Jac<S> J = jacobian_at<S>(cx, cz, ngnod, xi, ga);
        S dx = -(lx - x), dz = -(lz - zz);
        S dxi = J.xix * dx + J.xiz * dz, dga = J.gammax * dx + J.gammaz * dz;
        xi += dxi; ga += dga;
        xi = std::min(std::max(xi, S(-1.01)), S(1.01));
        ga = std::min(std::max(ga, S(-1.01)), S(1.01));
        if (std::abs(dxi) < 1e-12 && std::abs(dga) < 1e-12) break;
      }
      S lx, lz;
      location_at<S>(cx, cz, ngnod, xi, ga, lx, lz);
      S d = std::sqrt((lx - x) * (lx - x) + (lz - zz) * (lz - zz));
      if (d < fd - tol) { fd = d; es = e; xs = xi; gs = ga; }
    }
    if (es < 0 || std::abs(std::abs(xs) - S(1.01)) < S(1e-6) || std::abs(std::abs(gs) - S(1.01)) < S(1e-6))
      throw std::runtime_error("Failed to locate point in the mesh");
    return {es, double(xs), double(gs)};
  }

  std::tuple<int, double, double> locate(double X, double Z) const {
    return in.setup_in_run_precision ? locate_in<T>(X, Z) : locate_in<double>(X, Z);
  }

  // Lagrange interpolants at a located point, in the setup precision.
  void interpolants(double xi, double ga, T out[NP], T dx_out[NP] = nullptr, T dg_out[NP] = nullptr) const {
    double zd[NG], wd[NG];
    gll_nodes(zd, wd);
    if (in.setup_in_run_precision) {
      T hx[NG], hpx[NG], hg[NG], hpg[NG], zt[NG];
      for (int i = 0; i < NG; ++i) zt[i] = T(zd[i]);
      lagrange_interp<T>(T(xi), zt, hx, hpx);
      lagrange_interp<T>(T(ga), zt, hg, hpg);
      for (int iz = 0; iz < NG; ++iz)
        for (int ix = 0; ix < NG; ++ix) out[iz * NG + ix] = hx[ix] * hg[iz];
    } else {
      double hx[NG], hpx[NG], hg[NG], hpg[NG];
      lagrange_interp<double>(xi, zd, hx, hpx);
      lagrange_interp<double>(ga, zd, hg, hpg);
      for (int iz = 0; iz < NG; ++iz)
        for (int ix = 0; ix < NG; ++ix) out[iz * NG + ix] = T(hx[ix] * hg[iz]);
    }
  }

  // Moment-tensor source array (P-SV): M . grad(l_x(xi) l_z(gamma)) with the
  // stored Jacobian interpolated at the source
  // (core/specfem/assembly/compute_source_array/dim2/impl/compute_source_array_from_tensor.cpp:17-86;
  //  tensor [[Mxx, Mxz], [Mxz, Mzz]], core/specfem/source/dim2/tensor_source/moment_tensor_source.cpp:22-35).
  // Interpolants and products in the setup precision.
  void moment_tensor_array(Src &S, int e, double xi, double ga, double mxx, double mzz, double mxz) {
    if (S.medium != MED_ELASTIC || ncomp_el != 2)
      throw std::runtime_error("moment-tensor sources need an elastic P-SV element");
    for (int q = 0; q < NP; ++q) S.arr[2][q] = 0;
    S.ncomp = 2;
    double zd[NG], wd[NG], hx[NG], hpx[NG], hg[NG], hpg[NG];
    gll_nodes(zd, wd);
    lagrange_interp<double>(xi, zd, hx, hpx);
    lagrange_interp<double>(ga, zd, hg, hpg);
    double jx[4] = {0, 0, 0, 0};
    for (int iz = 0; iz < NG; ++iz)
      for (int ix = 0; ix < NG; ++ix) {
        const size_t p = size_t(e) * NP + iz * NG + ix;
        const double h = hx[ix] * hg[iz];
        jx[0] += h * double(xix[p]); jx[1] += h * double(xiz[p]);
        jx[2] += h * double(gax[p]); jx[3] += h * double(gaz[p]);
      }
    for (int iz = 0; iz < NG; ++iz)
      for (int ix = 0; ix < NG; ++ix) {
        const int q = iz * NG + ix;
        const double dsx = (hpx[ix] * jx[0]) * hg[iz] + hx[ix] * (hpg[iz] * jx[2]);
        const double dsz = (hpx[ix] * jx[1]) * hg[iz] + hx[ix] * (hpg[iz] * jx[3]);
        S.arr[0][q] = T(mxx * dsx + mxz * dsz);
        S.arr[1][q] = T(mxz * dsx + mzz * dsz);
      }
  }

  void sources() {
    const int nstep = in.nstep;
    for (int s = 0; s < in.nsrc; ++s) {
      auto [e, xi, ga] = locate(in.src_x[s], in.src_z[s]);
      Src S;
      S.ispec = e;
      S.medium = medium[e];
      T h[NP];
      interpolants(xi, ga, h);
      if (in.src_kind && in.src_kind[s] == 1) {
        if (ncomp_el == 4 && S.medium == MED_ELASTIC)
          throw std::runtime_error("moment-tensor sources in poroelastic media are outside this path");
        moment_tensor_array(S, e, xi, ga, in.src_mxx[s], in.src_mzz[s], in.src_mxz[s]);
      } else {
        T fv[4] = {0, 0, 0, 0};
        if (S.medium == MED_ACOUSTIC || ncomp_el == 1) { S.ncomp = 1; fv[0] = 1; }
        else {
          // Cosserat: (sin, cos, 0); poroelastic: (sin, cos, sin, cos)
          // (vector_source/force_source.cpp:53-67)
          S.ncomp = ncomp_el;
          T ang = T(in.src_angle[s]) * T(M_PI) / T(180.0);
          fv[0] = std::sin(ang); fv[1] = std::cos(ang);
          if (ncomp_el == 4) { fv[2] = fv[0]; fv[3] = fv[1]; }
        }
        for (int q = 0; q < NP; ++q)
          for (int c = 0; c < S.ncomp; ++c) S.arr[c][q] = h[q] * fv[c];
      }
      S.stf.resize(size_t(nstep));
      if (in.stf_table) {
        for (int i = 0; i < nstep; ++i) S.stf[i] = T(in.stf_table[size_t(i) * in.nsrc + s]);
      } else {
        const T f0 = T(in.src_f0[s]), fac = T(in.src_factor[s]), tsh = T(in.src_tshift[s]);
        const T t0 = T(in.t0);
        const T pi = T(M_PI);
        for (int i = 0; i < nstep; ++i) {
          T t = t0 + T(i) * dt - tsh;
          T a = pi * pi * f0 * f0;
          S.stf[i] = fac * ((T(1) - T(2) * a * t * t) * std::exp(-a * t * t));
        }
      }
      srcs.push_back(S);
    }
  }

  void receivers() {
    for (int r = 0; r < in.nrec; ++r) {
      auto [e, xi, ga] = locate(in.rec_x[r], in.rec_z[r]);
      Rec R;
      R.ispec = e;
      interpolants(xi, ga, R.h);
      recs.push_back(R);
    }
  }

  // --------------------------------------------------------- kernels ---
  // One element's forces for a medium of ncomp components.  The body is
  // instantiated per component count (the loops then have fixed trip counts);
  // the arithmetic and its order are the same for every count.
  template <typename AddFn>
  void stiffness_element(int e, int ncomp, const std::vector<T> &u, const std::vector<T> &v,
                         AddFn add) const {
    switch (ncomp) {
      case 1: stiffness_element_nc<1>(e, u, v, add); return;
      case 2: stiffness_element_nc<2>(e, u, v, add); return;
      case 3: stiffness_element_nc<3>(e, u, v, add); return;
      default: stiffness_element_nc<4>(e, u, v, add); return;
    }
  }

  template <int NC, typename AddFn>
  void stiffness_element_nc(int e, const std::vector<T> &u, const std::vector<T> &v, AddFn add) const {
    constexpr int ncomp = NC;
    T fu[NP][4], F[NP][4][2], Sa[NP][2];   // Sa: Cosserat sigma_xz, sigma_zx
    const int *ib = &ibool[size_t(e) * NP];
    for (int q = 0; q < NP; ++q)
      for (int c = 0; c < ncomp; ++c) fu[q][c] = u[size_t(ib[q]) * ncomp + c];
    const bool acoustic = medium[e] == MED_ACOUSTIC;
    for (int iz = 0; iz < NG; ++iz)
      for (int ix = 0; ix < NG; ++ix) {
        const int q = iz * NG + ix;
        const size_t p = size_t(e) * NP + q;
        T dxi[4] = {0, 0, 0, 0}, dga[4] = {0, 0, 0, 0};
        if (in.device_order) {
          for (int l = 0; l < NG; ++l)
            for (int c = 0; c < ncomp; ++c) {
              dxi[c] = std::fma(hp[ix][l], fu[iz * NG + l][c], dxi[c]);
              dga[c] = std::fma(hp[iz][l], fu[l * NG + ix][c], dga[c]);
            }
        } else {
          for (int l = 0; l < NG; ++l)
            for (int c = 0; c < ncomp; ++c) {
              dxi[c] += hp[ix][l] * fu[iz * NG + l][c];
              dga[c] += hp[iz][l] * fu[l * NG + ix][c];
            }
        }
        T du[4][2];
        for (int c = 0; c < ncomp; ++c) {
          du[c][0] = xix[p] * dxi[c] + gax[p] * dga[c];
          du[c][1] = xiz[p] * dxi[c] + gaz[p] * dga[c];
        }
        T S[4][2];
        if (!acoustic && ncomp == 4) {
          // poroelastic/isotropic/stress.hpp: solid stresses with lambda_G =
          // H - 2 mu_G, fluid pressure sigma_p; rows u_s: sigma - phi/tort
          // sigma_p, rows w: sigma_p delta - rho_f/rho_bar sigma
          const T mu = p_po[4][p], C = p_po[6][p], M = p_po[7][p];
          const T lam = p_po[5][p] - T(2.0) * mu, l2m = lam + T(2.0) * mu;
          const T dw = du[2][0] + du[3][1];
          const T sxx = l2m * du[0][0] + lam * du[1][1] + C * dw;
          const T szz = l2m * du[1][1] + lam * du[0][0] + C * dw;
          const T sxz = mu * (du[0][1] + du[1][0]);
          const T sp = C * (du[0][0] + du[1][1]) + M * dw;
          const T pt = p_po[0][p] / p_po[3][p], rr = p_po[2][p] / rho_bar(p);
          S[0][0] = sxx - pt * sp; S[0][1] = sxz;
          S[1][0] = sxz; S[1][1] = szz - pt * sp;
          S[2][0] = sp - rr * sxx; S[2][1] = T(-1.0) * rr * sxz;
          S[3][0] = T(-1.0) * rr * sxz; S[3][1] = sp - rr * szz;
        } else if (!acoustic && ncomp == 3) {
          // Cosserat P-SV-T stress (isotropic_cosserat/stress.hpp, cosserat_stress.hpp):
          // lambda = kappa - 2/3 mu; rows u_x: (sxx, szx), u_z: (sxz, szz),
          // rotation: (mu_c + nu_c) grad(phi); sxz += 2 nu phi, szx -= 2 nu phi
          const T mu = p_mu[p], nu = p_cs[3][p], lam = p_kappa[p] - T(2.0 / 3.0) * mu;
          const T phi = fu[q][2];
          const T dv = du[0][0] + du[1][1];
          const T sxx = lam * dv + T(2) * mu * du[0][0];
          const T szz = lam * dv + T(2) * mu * du[1][1];
          T sxz = mu * (du[1][0] + du[0][1]) + nu * (du[1][0] - du[0][1]);
          T szx = mu * (du[0][1] + du[1][0]) + nu * (du[0][1] - du[1][0]);
          szx -= T(2) * nu * phi;
          sxz += T(2) * nu * phi;
          const T mc = p_cs[6][p] + p_cs[7][p];
          S[0][0] = sxx; S[0][1] = szx; S[1][0] = sxz; S[1][1] = szz;
          S[2][0] = mc * du[2][0]; S[2][1] = mc * du[2][1];
          Sa[q][0] = sxz; Sa[q][1] = szx;
        } else if (acoustic) {
          S[0][0] = p_rhoinv[p] * du[0][0];
          S[0][1] = p_rhoinv[p] * du[0][1];
        } else if (ncomp == 1) {
          S[0][0] = p_mu[p] * du[0][0];
          S[0][1] = p_mu[p] * du[0][1];
        } else if (in.aniso) {
          // include/medium/dim2/elastic/anisotropic/stress.hpp
          const T sh = du[1][0] + du[0][1];
          const T sxx = p_c[0][p] * du[0][0] + p_c[1][p] * du[1][1] + p_c[2][p] * sh;
          const T szz = p_c[1][p] * du[0][0] + p_c[3][p] * du[1][1] + p_c[4][p] * sh;
          const T sxz = p_c[2][p] * du[0][0] + p_c[4][p] * du[1][1] + p_c[5][p] * sh;
          S[0][0] = sxx; S[0][1] = sxz; S[1][0] = sxz; S[1][1] = szz;
        } else {
          const T l2m = lp2m(p), lam = l2m - T(2) * p_mu[p];
          const T sxx = l2m * du[0][0] + lam * du[1][1];
          const T szz = l2m * du[1][1] + lam * du[0][0];
          const T sxz = p_mu[p] * (du[0][1] + du[1][0]);
          S[0][0] = sxx; S[0][1] = sxz; S[1][0] = sxz; S[1][1] = szz;
        }
        for (int c = 0; c < ncomp; ++c) {
          F[q][c][0] = jac[p] * (S[c][0] * xix[p] + S[c][1] * xiz[p]);
          F[q][c][1] = jac[p] * (S[c][0] * gax[p] + S[c][1] * gaz[p]);
        }
      }
    for (int iz = 0; iz < NG; ++iz)
      for (int ix = 0; ix < NG; ++ix) {
        const int q = iz * NG + ix;
        const size_t p = size_t(e) * NP + q;
        T t1[4] = {0, 0, 0, 0}, t2[4] = {0, 0, 0, 0};
        if (in.device_order) {
          for (int l = 0; l < NG; ++l)
            for (int c = 0; c < ncomp; ++c) {
              t1[c] = std::fma(F[iz * NG + l][c][0], hpw[l][ix], t1[c]);
              t2[c] = std::fma(F[l * NG + ix][c][1], hpw[l][iz], t2[c]);
            }
        } else {
          for (int l = 0; l < NG; ++l) {
            for (int c = 0; c < ncomp; ++c) t1[c] += F[iz * NG + l][c][0] * hp[l][ix] * w[l];
            for (int c = 0; c < ncomp; ++c) t2[c] += F[l * NG + ix][c][1] * hp[l][iz] * w[l];
          }
        }
        T acc[4];
        for (int c = 0; c < ncomp; ++c) acc[c] = T(-1) * (w[iz] * t1[c] + w[ix] * t2[c]);
        if (!acoustic && ncomp == 4) {
          // viscous damping of the relative fluid motion (poroelastic/isotropic/damping.hpp,
          // compute_stiffness_interaction.tpp:216-223): factor = w_x w_z |J|
          const T fac = w[ix] * w[iz] * jac[p];
          const T kxx = p_po[8][p], kxz = p_po[9][p], kzz = p_po[10][p], eta = p_po[11][p];
          const T det = kxx * kzz - kxz * kxz;
          const T ixx = kzz / det, ixz = T(-1.0) * kxz / det, izz = kxx / det;
          const T v2 = v[size_t(ib[q]) * 4 + 2], v3 = v[size_t(ib[q]) * 4 + 3];
          const T viscx = fac * ((eta * ixx * v2) + (eta * ixz * v3));
          const T viscz = fac * ((eta * ixz * v2) + (eta * izz * v3));
          const T pt = p_po[0][p] / p_po[3][p];
          acc[0] += pt * viscx;
          acc[1] += pt * viscz;
          acc[2] -= viscx;
          acc[3] -= viscz;
        }
        // Cosserat couple stress: -W (sigma_xz - sigma_zx) on the rotation
        // (compute_stiffness_interaction.tpp:216-229, cosserat_couple_stress.hpp)
        if (!acoustic && ncomp == 3) acc[2] -= (Sa[q][0] - Sa[q][1]) * (w[ix] * w[iz] * jac[p]);
        if (st_tag[p]) {
          T vel[4];
          for (int c = 0; c < ncomp; ++c) vel[c] = v[size_t(ib[q]) * ncomp + c];
          stacey(p, vel, acc);
        }
        if (acoustic && fs_tag[p]) acc[0] = 0;
        add(ib[q], acc);
      }
  }

  // Threads of the point-wise loops below (element-wise arithmetic: the
  // thread count changes no bit); set by run().
  int nthr = 1;
  void predictor(std::vector<T> &u, std::vector<T> &v, std::vector<T> &a) {
    const T dt2 = dt / T(2.0), dtsq2 = dt * dt / T(2.0);
    const long long n = (long long)u.size();
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static) if (nthr > 1 && n > 65536)
#endif
    for (long long i = 0; i < n; ++i) {
      u[size_t(i)] += dt * v[size_t(i)] + dtsq2 * a[size_t(i)];
      v[size_t(i)] += dt2 * a[size_t(i)];
      a[size_t(i)] = 0;
    }
  }
  void corrector(std::vector<T> &v, const std::vector<T> &a) {
    const T dt2 = dt / T(2.0);
    const long long n = (long long)v.size();
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static) if (nthr > 1 && n > 65536)
#endif
    for (long long i = 0; i < n; ++i) v[size_t(i)] += dt2 * a[size_t(i)];
  }

  // Greedy colouring of one medium's elements, in element order (built once).
  std::vector<std::vector<int>> colour_lists[2];
  const std::vector<std::vector<int>> &colours(int med) {
    std::vector<std::vector<int>> &out = colour_lists[med == MED_ACOUSTIC ? 0 : 1];
    if (!out.empty() || nspec == 0) return out;
    std::vector<uint32_t> used(nglob, 0u);
    for (int e = 0; e < nspec; ++e) {
      if (medium[e] != med) continue;
      uint32_t mask = 0;
      for (int q = 0; q < NP; ++q) mask |= used[ibool[size_t(e) * NP + q]];
      int c = 0;
      while (c < 32 && (mask >> c & 1u)) ++c;
      if (c == 32) throw std::runtime_error("mesh needs more than 32 colours");
      for (int q = 0; q < NP; ++q) used[ibool[size_t(e) * NP + q]] |= 1u << c;
      if (int(out.size()) <= c) out.resize(c + 1);
      out[size_t(c)].push_back(e);
    }
    return out;
  }

  void update_medium(int med, int istep, int nthreads) {
    const int ncomp = med == MED_ACOUSTIC ? 1 : ncomp_el;
    std::vector<T> &u = med == MED_ACOUSTIC ? ua : ue;
    std::vector<T> &v = med == MED_ACOUSTIC ? va : ve;
    std::vector<T> &a = med == MED_ACOUSTIC ? aa : ae;
    const std::vector<T> &minv = med == MED_ACOUSTIC ? minv_a : minv_e;
    // coupling (domain_kernels.hpp:77-94)
    if (med == MED_ACOUSTIC) {
      for (const auto &c : cpl_ac) {
        T val = c.fac * (c.nx * ue[size_t(c.iglob) * ncomp_el + 0] + c.nz * ue[size_t(c.iglob) * ncomp_el + 1]);
        if (fs_tag[size_t(c.ispec) * NP + c.iz * NG + c.ix]) val = 0;
        a[c.iglob] += val;
      }
    } else if (ncomp_el == 2) {
      for (const auto &c : cpl_el) {
        a[size_t(c.iglob) * 2 + 0] += c.fac * c.nx * aa[c.iglob];
        a[size_t(c.iglob) * 2 + 1] += c.fac * c.nz * aa[c.iglob];
      }
    }
    // nonconforming coupling (compute_coupling.tpp:117-249): the coupled
    // field interpolated to the intersection quadrature (algorithms/transfer.hpp),
    // times the self normal (coupling_terms/*.hpp), integrated against the
    // self edge's transfer functions (integrate/coupling_integral1d.hpp)
    if (med == MED_ACOUSTIC) {
      for (const auto &E : nc_ac) {
        T f[NG];
        for (int q = 0; q < NG; ++q) {
          T u0 = 0, u1 = 0;
          for (int j = 0; j < NG; ++j) {
            u0 += ue[size_t(E.gc[j]) * 2 + 0] * E.tc[q][j];
            u1 += ue[size_t(E.gc[j]) * 2 + 1] * E.tc[q][j];
          }
          f[q] = E.nx[q] * u0 + E.nz[q] * u1;
        }
        for (int i = 0; i < NG; ++i) {
          T r = 0;
          for (int q = 0; q < NG; ++q) r += f[q] * E.fac[q] * E.ts[q][i];
          if (E.fs[i]) r = 0;
          a[E.gs[i]] += r;
        }
      }
    } else if (ncomp_el == 2) {
      for (const auto &E : nc_el) {
        T f0[NG], f1[NG];
        for (int q = 0; q < NG; ++q) {
          T p = 0;
          for (int j = 0; j < NG; ++j) p += aa[E.gc[j]] * E.tc[q][j];
          f0[q] = E.nx[q] * p;
          f1[q] = E.nz[q] * p;
        }
        for (int i = 0; i < NG; ++i) {
          T r0 = 0, r1 = 0;
          for (int q = 0; q < NG; ++q) {
            r0 += f0[q] * E.fac[q] * E.ts[q][i];
            r1 += f1[q] * E.fac[q] * E.ts[q][i];
          }
          a[size_t(E.gs[i]) * 2 + 0] += r0;
          a[size_t(E.gs[i]) * 2 + 1] += r1;
        }
      }
    }
    // sources (:96-110)
    for (const auto &S : srcs) {
      if (S.medium != med) continue;
      const int *ib = &ibool[size_t(S.ispec) * NP];
      for (int q = 0; q < NP; ++q) {
        size_t p = size_t(S.ispec) * NP + q;
        if (med == MED_ACOUSTIC)
          a[ib[q]] += -S.stf[istep] * S.arr[0][q] / p_kappa[p];
        else if (ncomp == 4) {
          // poroelastic/isotropic/source.hpp: solid rows times (1 - phi / tort),
          // fluid rows times (1 - rho_f / rho_bar), double literals
          const double fs = 1.0 - double(p_po[0][p] / p_po[3][p]);
          const double ff = 1.0 - double(p_po[2][p] / rho_bar(p));
          for (int c = 0; c < 4; ++c)
            a[size_t(ib[q]) * 4 + c] += T(double(S.stf[istep] * S.arr[c][q]) * (c < 2 ? fs : ff));
        } else
          for (int c = 0; c < ncomp; ++c) a[size_t(ib[q]) * ncomp + c] += S.stf[istep] * S.arr[c][q];
      }
    }
    // stiffness (:112-126)
#ifdef _OPENMP
    if (nthreads > 1) {
      const std::vector<std::vector<int>> &col = colours(med);
      for (const std::vector<int> &L : col) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long long k = 0; k < (long long)L.size(); ++k)
          stiffness_element(L[size_t(k)], ncomp, u, v, [&](int g, const T *acc) {
            for (int c = 0; c < ncomp; ++c) a[size_t(g) * ncomp + c] += acc[c];
          });
      }
    } else
#endif
    {
      for (int e = 0; e < nspec; ++e) {
        if (medium[e] != med) continue;
        stiffness_element(e, ncomp, u, v, [&](int g, const T *acc) {
          for (int c = 0; c < ncomp; ++c) a[size_t(g) * ncomp + c] += acc[c];
        });
      }
    }
    // divide by mass (:128-138), only on this medium's points
    const std::vector<uint8_t> &own = med == MED_ACOUSTIC ? is_ac_glob : is_el_glob;
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static) if (nthr > 1 && nglob > 65536)
#endif
    for (int g = 0; g < nglob; ++g)
      if (own[g])
        for (int c = 0; c < ncomp; ++c) a[size_t(g) * ncomp + c] *= minv[size_t(g) * ncomp + c];
  }

  // seismogram value of one receiver for one type (compute_seismogram.tpp)
  void seismo(const Rec &R, int type, T out[2]) const {
    const int e = R.ispec;
    const int *ib = &ibool[size_t(e) * NP];
    out[0] = out[1] = 0;
    if (medium[e] == MED_ACOUSTIC) {
      const std::vector<T> &f = type == 0 ? ua : type == 1 ? va : aa;
      if (type == 3) {
        for (int q = 0; q < NP; ++q) out[0] += R.h[q] * (T(-1.0) * aa[ib[q]]);
        return;
      }
      for (int iz = 0; iz < NG; ++iz)
        for (int ix = 0; ix < NG; ++ix) {
          const int q = iz * NG + ix;
          const size_t p = size_t(e) * NP + q;
          T dxi = 0, dga = 0;
          for (int l = 0; l < NG; ++l) {
            dxi += hp[ix][l] * f[ib[iz * NG + l]];
            dga += hp[iz][l] * f[ib[l * NG + ix]];
          }
          T dx = xix[p] * dxi + gax[p] * dga, dz = xiz[p] * dxi + gaz[p] * dga;
          out[0] += R.h[q] * (p_rhoinv[p] * dx);
          out[1] += R.h[q] * (p_rhoinv[p] * dz);
        }
      return;
    }
    const int nc = ncomp_el;
    if (type == 3 || type == 5 || type == 6) {
      // elastic pressure -(lambda + 2/3 mu) div u (elastic/isotropic/wavefield.hpp:57-89;
      // Cosserat: -kappa div u); Cosserat curl du_x/dz - du_z/dx and intrinsic
      // rotation phi - curl / 2 (isotropic_cosserat/wavefield.hpp)
      if (nc == 1) return;
      if ((type == 5 || type == 6) && nc != 3) return;
      for (int iz = 0; iz < NG; ++iz)
        for (int ix = 0; ix < NG; ++ix) {
          const int q = iz * NG + ix;
          const size_t p = size_t(e) * NP + q;
          T dxi[2] = {0, 0}, dga[2] = {0, 0};
          for (int l = 0; l < NG; ++l)
            for (int c = 0; c < 2; ++c) {
              dxi[c] += hp[ix][l] * ue[size_t(ib[iz * NG + l]) * nc + c];
              dga[c] += hp[iz][l] * ue[size_t(ib[l * NG + ix]) * nc + c];
            }
          if (type == 3 && nc == 4) {
            // poroelastic/isotropic/wavefield.hpp: -(C div u_s + M div w)
            T dxf[2] = {0, 0}, dgf[2] = {0, 0};
            for (int l = 0; l < NG; ++l)
              for (int c = 0; c < 2; ++c) {
                dxf[c] += hp[ix][l] * ue[size_t(ib[iz * NG + l]) * nc + 2 + c];
                dgf[c] += hp[iz][l] * ue[size_t(ib[l * NG + ix]) * nc + 2 + c];
              }
            const T dux = xix[p] * dxi[0] + gax[p] * dga[0];
            const T duz = xiz[p] * dxi[1] + gaz[p] * dga[1];
            const T dwx = xix[p] * dxf[0] + gax[p] * dgf[0];
            const T dwz = xiz[p] * dxf[1] + gaz[p] * dgf[1];
            out[0] += R.h[q] * (T(-1.0) * (p_po[6][p] * (dux + duz) + p_po[7][p] * (dwx + dwz)));
          } else if (type == 3) {
            const T dux = xix[p] * dxi[0] + gax[p] * dga[0];
            const T duz = xiz[p] * dxi[1] + gaz[p] * dga[1];
            const T k = nc == 3 ? p_kappa[p] : (lp2m(p) - T(2) * p_mu[p]) + T(2.0 / 3.0) * p_mu[p];
            out[0] += R.h[q] * (T(-1.0) * (k * (dux + duz)));
          } else {
            const T duxz = xiz[p] * dxi[0] + gaz[p] * dga[0];   // d u_x / dz
            const T duzx = xix[p] * dxi[1] + gax[p] * dga[1];   // d u_z / dx
            const T curl = duxz - duzx;
            out[0] += R.h[q] * (type == 6 ? curl : ue[size_t(ib[q]) * nc + 2] - T(0.5) * curl);
          }
        }
      return;
    }
    if (type == 4) {                       // Cosserat rotation
      if (nc != 3) return;
      for (int q = 0; q < NP; ++q) out[0] += R.h[q] * ue[size_t(ib[q]) * nc + 2];
      return;
    }
    const std::vector<T> &f = type == 0 ? ue : type == 1 ? ve : ae;
    for (int q = 0; q < NP; ++q)
      for (int c = 0; c < std::min(nc, 2); ++c) out[c] += R.h[q] * f[size_t(ib[q]) * nc + c];
  }

  // ---------------------------------------------------------------------
  // The reference's combined (adjoint + backward) simulation of an isotropic
  // elastic P-SV model and its Frechet kernels
  // (core/specfem/solver/time_marching.tpp:133-264,
  //  include/kokkos_kernels/impl/compute_material_derivatives.tpp:14-153,
  //  include/medium/dim2/elastic/isotropic/frechet_derivative.hpp:55-181).
  //
  // One elastic update on fields (u, v, a): the given sources at istep, the
  // element forces, M^-1.  mode 0: plain; 1: record the contributions of the
  // elements that carry Stacey points (forward run); 2: replay them instead
  // of computing those elements (backward run,
  // compute_stiffness_interaction.tpp:123-137, stored at :238-242).
  std::vector<uint8_t> st_elem;                 // element carries Stacey points
  std::vector<int> st_slot;                     // its slot in the replay buffer
  std::vector<T> replay;                        // [nstep][nst_elem][25][2]
  int nst_elem = 0;

  void update_elastic(std::vector<T> &u, std::vector<T> &v, std::vector<T> &a, int istep,
                      const std::vector<Src> &sources, int mode) {
    for (const auto &S : sources) {
      const int *ib = &ibool[size_t(S.ispec) * NP];
      for (int q = 0; q < NP; ++q)
        for (int c = 0; c < 2; ++c) a[size_t(ib[q]) * 2 + c] += S.stf[istep] * S.arr[c][q];
    }
    for (int e = 0; e < nspec; ++e) {
      if (medium[e] != MED_ELASTIC) continue;
      T *rec = nullptr;
      if (mode != 0 && st_elem[e]) rec = &replay[((size_t(istep) * nst_elem + st_slot[e]) * NP) * 2];
      if (mode == 2 && rec) {
        for (int q = 0; q < NP; ++q)
          for (int c = 0; c < 2; ++c) a[size_t(ibool[size_t(e) * NP + q]) * 2 + c] += rec[q * 2 + c];
        continue;
      }
      int q = 0;
      stiffness_element(e, 2, u, v, [&](int g, const T *acc) {
        for (int c = 0; c < 2; ++c) {
          a[size_t(g) * 2 + c] += acc[c];
          if (rec) rec[q * 2 + c] = acc[c];
        }
        ++q;
      });
    }
    for (int g = 0; g < nglob; ++g)
      if (is_el_glob[g])
        for (int c = 0; c < 2; ++c) a[size_t(g) * 2 + c] *= minv_e[size_t(g) * 2 + c];
  }

  // Element gradient of a field at every point of element e: du[q][c][j] =
  // d u_c / d x_j (include/algorithms/gradient.hpp:40-82).  With `add` the
  // xi / gamma derivatives of `add` are summed in before the Jacobian map, as
  // the reference's two-field gradient does with its shared accumulators
  // (gradient.hpp:296-317).
  void element_grad(int e, const std::vector<T> &f, const std::vector<T> *add, T du[NP][2][2]) const {
    const int *ib = &ibool[size_t(e) * NP];
    for (int iz = 0; iz < NG; ++iz)
      for (int ix = 0; ix < NG; ++ix) {
        const int q = iz * NG + ix;
        const size_t p = size_t(e) * NP + q;
        T dxi[2] = {0, 0}, dga[2] = {0, 0};
        for (int l = 0; l < NG; ++l)
          for (int c = 0; c < 2; ++c) {
            dxi[c] += hp[ix][l] * f[size_t(ib[iz * NG + l]) * 2 + c];
            dga[c] += hp[iz][l] * f[size_t(ib[l * NG + ix]) * 2 + c];
            if (add) {
              dxi[c] += hp[ix][l] * (*add)[size_t(ib[iz * NG + l]) * 2 + c];
              dga[c] += hp[iz][l] * (*add)[size_t(ib[l * NG + ix]) * 2 + c];
            }
          }
        for (int c = 0; c < 2; ++c) {
          du[q][c][0] = xix[p] * dxi[c] + gax[p] * dga[c];
          du[q][c][1] = xiz[p] * dxi[c] + gaz[p] * dga[c];
        }
      }
  }

  // adj [nstep][nrec][2]: adjoint source time functions of the receivers
  // (point forces at the receiver locations, applied at step istep as the
  // iteration runs istep = nstep-1 .. 0).  quirk: the backward derivatives
  // include the adjoint field's (the reference's two-field gradient).
  // reconstruct: the reference's reverse-time backward field; else the
  // forward run's own snapshots (to separate reconstruction error).
  // Out: kernels rho, mu, kappa [nspec][25] and the quadrature weight
  // w_x w_z |J| of every element point.
  void adjoint_compat(const double *adj, int quirk, int reconstruct, double *out_rho, double *out_mu,
                      double *out_kappa, double *out_w) {
    if (ncomp_el != 2 || in.aniso || in.cosserat || in.poro)
      throw std::runtime_error("the reference-compatible adjoint covers isotropic elastic P-SV media");
    for (int e = 0; e < nspec; ++e)
      if (medium[e] != MED_ELASTIC) throw std::runtime_error("the reference-compatible adjoint covers one elastic medium");
    const int nstep = in.nstep;
    st_elem.assign(nspec, 0);
    st_slot.assign(nspec, -1);
    nst_elem = 0;
    for (int e = 0; e < nspec; ++e) {
      for (int q = 0; q < NP; ++q) st_elem[e] |= st_tag[size_t(e) * NP + q];
      if (st_elem[e]) st_slot[e] = nst_elem++;
    }
    replay.assign(size_t(nstep) * nst_elem * NP * 2, T(0));
    std::vector<std::vector<T>> snaps;
    // forward run (sources of the configuration), recording the Stacey elements
    for (int istep = 0; istep < nstep; ++istep) {
      predictor(ue, ve, ae);
      update_elastic(ue, ve, ae, istep, srcs, 1);
      corrector(ve, ae);
      if (!reconstruct) snaps.push_back(ue);
    }
    const std::vector<T> fu = ue, fv = ve, fa = ae;   // the forward wavefield buffer
    // adjoint sources: one point force per receiver and component
    std::vector<Src> asrc;
    for (int r = 0; r < in.nrec; ++r)
      for (int c = 0; c < 2; ++c) {
        Src S{};
        S.ispec = recs[r].ispec;
        S.medium = MED_ELASTIC;
        S.ncomp = 2;
        for (int q = 0; q < NP; ++q) { S.arr[c][q] = recs[r].h[q]; S.arr[1 - c][q] = T(0); }
        S.stf.resize(nstep);
        for (int k = 0; k < nstep; ++k) S.stf[k] = T(adj[(size_t(k) * in.nrec + r) * 2 + c]);
        asrc.push_back(S);
      }
    const size_t ne = size_t(nglob) * 2;
    std::vector<T> uA(ne, T(0)), vA(ne, T(0)), aA(ne, T(0)), uB(ne, T(0)), vB(ne, T(0)), aB(ne, T(0));
    const size_t nloc = size_t(nspec) * NP;
    std::vector<double> krho(nloc, 0.0), kmu(nloc, 0.0), kkap(nloc, 0.0);
    const T dt2 = dt / T(2.0), dtsq2 = dt * dt / T(2.0);
    T dA[NP][2][2], dB[NP][2][2];
    for (int istep = nstep - 1; istep >= 0; --istep) {
      // adjoint time step (newmark.tpp apply_*_phase_forward on the adjoint field)
      predictor(uA, vA, aA);
      update_elastic(uA, vA, aA, istep, asrc, 0);
      corrector(vA, aA);
      // backward time step: -dt, -dt/2, +dt^2/2 (newmark.tpp:222-267)
      if (reconstruct) {
        for (size_t i = 0; i < ne; ++i) {
          uB[i] += T(-1) * dt * vB[i] + dtsq2 * aB[i];
          vB[i] += T(-1) * dt2 * aB[i];
          aB[i] = 0;
        }
        update_elastic(uB, vB, aB, istep, srcs, 2);
        for (size_t i = 0; i < ne; ++i) vB[i] += T(-1) * dt2 * aB[i];
        if (istep == nstep - 1) { uB = fu; vB = fv; aB = fa; }   // the buffer copy (time_marching.tpp:214-216)
      } else {
        uB = snaps[size_t(istep)];
      }
      // Frechet kernels of this step
      for (int e = 0; e < nspec; ++e) {
        element_grad(e, uA, nullptr, dA);
        element_grad(e, uB, quirk ? &uA : nullptr, dB);
        const int *ib = &ibool[size_t(e) * NP];
        for (int q = 0; q < NP; ++q) {
          const size_t p = size_t(e) * NP + q;
          const T kap = lp2m(p) - p_mu[p];           // kappa2D = lambda + mu (frechet_derivative.hpp:77)
          const T ad_xx = dA[q][0][0], ad_zz = dA[q][1][1], ad_xz = T(0.5) * (dA[q][1][0] + dA[q][0][1]);
          const T b_xx = dB[q][0][0], b_zz = dB[q][1][1], b_xz = T(0.5) * (dB[q][1][0] + dB[q][0][1]);
          const T kk = (ad_xx + ad_zz) * (b_xx + b_zz);
          const T mm = ad_xx * b_xx + ad_zz * b_zz + T(2.0) * ad_xz * b_xz - T(1.0 / 3.0) * kk;
          const size_t g = size_t(ib[q]) * 2;
          const T rr = aA[g] * uB[g] + aA[g + 1] * uB[g + 1];
          kkap[p] += double(T(-1.0) * kap * dt * kk);
          kmu[p] += double(T(-2.0) * p_mu[p] * dt * mm);
          krho[p] += double(T(-1.0) * p_rho[p] * dt * rr);
        }
      }
    }
    for (size_t p = 0; p < nloc; ++p) {
      out_rho[p] = krho[p]; out_mu[p] = kmu[p]; out_kappa[p] = kkap[p];
      const int q = int(p % NP), iz = q / NG, ix = q - iz * NG;
      out_w[p] = double(w[ix]) * double(w[iz]) * double(jac[p]);
    }
  }

  void run(double *seis, int nthreads) {
    nthr = std::max(1, nthreads);
    const int nsb = std::max(1, in.nstep_between_samples);
    int isig = 0;
    const T ca = std::cos(T(M_PI) / T(180) * T(in.rec_angle));
    const T sa = std::sin(T(M_PI) / T(180) * T(in.rec_angle));
    for (int istep = 0; istep < in.nstep; ++istep) {
      predictor(ua, va, aa);
      predictor(ue, ve, ae);
      update_medium(MED_ACOUSTIC, istep, nthreads);
      corrector(va, aa);
      update_medium(MED_ELASTIC, istep, nthreads);
      corrector(ve, ae);
      if (istep % nsb == 0 && seis) {
        for (int t = 0; t < in.ntypes; ++t)
          for (int r = 0; r < in.nrec; ++r) {
            T o[2];
            seismo(recs[r], in.seis_types[t], o);
            size_t k = ((size_t(isig) * in.ntypes + t) * in.nrec + r) * 2;
            seis[k + 0] = double(ca * o[0] - sa * o[1]);
            seis[k + 1] = double(sa * o[0] + ca * o[1]);
          }
        ++isig;
      }
    }
  }
};

template <typename T>
int run_impl(const OracleInput2D *in, OracleOutput2D *out, int nthreads) {
  try {
    Sim<T> s(*in);
    s.setup();
    const auto t0 = std::chrono::steady_clock::now();
    s.run(out->seismograms, nthreads);
    out->loop_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    out->nglob = s.nglob;
    if (out->final_u_elastic) {
      for (size_t i = 0; i < s.ue.size(); ++i) out->final_u_elastic[i] = double(s.ue[i]);
    }
    if (out->final_u_acoustic) {
      for (size_t i = 0; i < s.ua.size(); ++i) out->final_u_acoustic[i] = double(s.ua[i]);
    }
    if (out->ibool) std::copy(s.ibool.begin(), s.ibool.end(), out->ibool);
    return 0;
  } catch (const std::exception &ex) {
    std::snprintf(out->error, sizeof(out->error), "%s", ex.what());
    return -1;
  }
}

}  // namespace

extern "C" {

int oracle2d_run_f32(const OracleInput2D *in, OracleOutput2D *out, int nthreads) {
  return run_impl<float>(in, out, nthreads);
}

int oracle2d_run_f64(const OracleInput2D *in, OracleOutput2D *out, int nthreads) {
  return run_impl<double>(in, out, nthreads);
}

// Element and local coordinates the oracle assigns to a physical point.
int oracle2d_locate(const OracleInput2D *in, int precision64, double x, double z, int *ispec,
                    double *xi, double *gamma) {
  try {
    if (precision64) {
      Sim<double> s(*in);
      s.setup_geometry_only();
      auto [e, a, b] = s.locate(x, z);
      *ispec = e; *xi = a; *gamma = b;
    } else {
      Sim<float> s(*in);
      s.setup_geometry_only();
      auto [e, a, b] = s.locate(x, z);
      *ispec = e; *xi = a; *gamma = b;
    }
    return 0;
  } catch (const std::exception &) {
    return -1;
  }
}

// The reference's combined adjoint simulation and Frechet kernels (FP64).
int oracle2d_adjoint_compat_f64(const OracleInput2D *in, const double *adj, int quirk, int reconstruct,
                                double *rho_kl, double *mu_kl, double *kappa_kl, double *weight,
                                char *error, int error_len) {
  try {
    Sim<double> s(*in);
    s.setup();
    s.adjoint_compat(adj, quirk, reconstruct, rho_kl, mu_kl, kappa_kl, weight);
    return 0;
  } catch (const std::exception &ex) {
    if (error && error_len > 0) std::snprintf(error, size_t(error_len), "%s", ex.what());
    return -1;
  }
}

// Count global points of a mesh (so callers can size final-field buffers).
int oracle2d_count_nglob(const OracleInput2D *in) {
  Sim<double> s(*in);
  s.number_points();
  return s.nglob;
}

// Known-answer helpers used by the unit tests.
void oracle_gll(double *z, double *w, double *hprime) {
  double zz[NG], ww[NG], hp[NG][NG];
  gll_nodes(zz, ww);
  gll_hprime(zz, hp);
  for (int i = 0; i < NG; ++i) {
    z[i] = zz[i]; w[i] = ww[i];
    for (int j = 0; j < NG; ++j) hprime[i * NG + j] = hp[i][j];
  }
}

double oracle_legendre(double x, int n) { return legendre(x, n); }

// 2D elastic isotropic P-SV stress (stress.hpp:38-78); du row-major [2][2].
void oracle_stress_psv(double kappa, double mu, const double *du, double *sigma) {
  double l2m = kappa + 4.0 / 3.0 * mu, lam = l2m - 2.0 * mu;
  sigma[0] = l2m * du[0] + lam * du[3];
  sigma[1] = mu * (du[1] + du[2]);
  sigma[2] = sigma[1];
  sigma[3] = l2m * du[3] + lam * du[0];
}

}  // extern "C"
