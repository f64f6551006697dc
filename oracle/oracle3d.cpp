// CPU oracle of the 3D elastic spectral-element time step (test
// infrastructure: the checker of the CUDA path, never part of the product).
//
// Restates, for structured hexahedral meshes (an (nex x ney x nez) lattice of
// 8-node elements with arbitrary control-node coordinates), the reference's 3D
// elastic isotropic forward step:
//   GLL nodes/weights/derivatives   src/quadrature/gll/gll_library.cpp, lagrange_poly.cpp
//   8-node shape functions, Jacobian core/specfem/shape_function/dim3, core/specfem/jacobian/dim3
//   gradient (3D)                   include/algorithms/gradient.hpp:103-156
//   stress (3D isotropic)           include/medium/dim3/elastic/isotropic/stress.hpp:46-99
//   F = |J| sigma . grad(xi)        core/specfem/point/stress.hpp:217-240
//   divergence (3D)                 include/algorithms/divergence.hpp:90-137
//   mass matrix                     include/medium/dim3/elastic/isotropic/mass_matrix.tpp:5-15
//   Newmark predictor/corrector     core/specfem/timescheme/newmark.tpp:10-128
//   force / moment-tensor sources   core/specfem/assembly/compute_source_array/dim3/impl/*
//   receivers (Lagrange interp.)    include/kokkos_kernels/impl/compute_seismogram.tpp
// Stacey absorbing faces are not part of the reference's 3D path; the oracle
// holds the 3D form of its 2D P-SV condition (stacey.tpp:50-80): traction
// -[(rho vp - rho vs)(v.n)n/|n|^2 + rho vs v] |n| w_a w_b on each absorbing
// face point (n = |J| grad(xi_k), outward), and the implicit mass term
// evaluated with the velocity stand-in -dt/2 in every component
// (stacey.tpp:817-853 in 2D).
//
// Global numbering is the lattice of GLL points; elements are assembled in 8
// colour passes (parity of the element indices), so the order of every sum is
// fixed.  Setup (Jacobians, location, interpolants) in FP64, rounded to the
// run precision; the time loop in the run precision (float or double).
#include "oracle3d.h"

#include <omp.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

constexpr int NG = 5, NP3 = 125;

void gll5(double z[NG], double w[NG], double hp[NG][NG]) {
  const double r = std::sqrt(3.0 / 7.0);
  const double zz[NG] = {-1.0, -r, 0.0, r, 1.0};
  const double ww[NG] = {0.1, 49.0 / 90.0, 32.0 / 45.0, 49.0 / 90.0, 0.1};
  for (int i = 0; i < NG; ++i) { z[i] = zz[i]; w[i] = ww[i]; }
  // Legendre P4 and the GLL derivative matrix (lagrange_poly.cpp:45-72)
  auto P4 = [](double x) { return (35 * x * x * x * x - 30 * x * x + 3) / 8.0; };
  const int N = NG - 1;
  for (int i = 0; i < NG; ++i)
    for (int j = 0; j < NG; ++j) {
      if (i == j) hp[i][j] = i == 0 ? -0.25 * N * (N + 1.0) : (i == N ? 0.25 * N * (N + 1.0) : 0.0);
      else hp[i][j] = P4(z[i]) / (P4(z[j]) * (z[i] - z[j]));
    }
}

// Lagrange interpolants h and derivatives hp at x (lagrange_poly.cpp:12-44).
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

// 8-node hexahedron, corners (xi, eta, gamma) in {-1, 1}^3:
// 0 (-,-,-) 1 (+,-,-) 2 (+,+,-) 3 (-,+,-) 4 (-,-,+) 5 (+,-,+) 6 (+,+,+) 7 (-,+,+)
const int CS[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                      {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

struct Geo {
  double x[3];
  double inv[3][3];  // inv[k][j] = d xi_k / d x_j
  double jac;
};

Geo map_point(const double cn[8][3], double xi, double eta, double ga) {
  double dx[3][3] = {{0}};  // dx[j][k] = d x_j / d xi_k
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
  // inverse of dx (xi derivatives of x): inv = dx^-1
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

template <typename T>
struct Sim3D {
  const OracleInput3D &in;
  int nex, ney, nez, nspec, NX, NY, NZ, nglob;
  double zd[NG], wd[NG], hpd[NG][NG];
  T w[NG], hp[NG][NG];
  T hpw[NG][NG];   // hp[l][i] * w[l] rounded once (device evaluation order)
  std::vector<int> ibool;                           // [nspec][125]
  std::vector<T> g9, jac, c0, mu;                   // g9: [nspec][125][9]
  std::vector<T> u, v, a, minv;                     // [nglob][3]
  struct Face { int e, q; T n[3]; T rvp, rvs, w; };   // one absorbing face point
  std::vector<Face> faces;
  std::vector<std::vector<int>> face_of_elem;       // indices into faces per element
  struct Src { int e; T arr[3][NP3]; std::vector<T> stf; };
  std::vector<Src> srcs;
  struct Rec { int e; T h[NP3]; };
  std::vector<Rec> recs;
  T dt;

  explicit Sim3D(const OracleInput3D &i) : in(i) {
    nex = in.nex; ney = in.ney; nez = in.nez;
    nspec = nex * ney * nez;
    NX = 4 * nex + 1; NY = 4 * ney + 1; NZ = 4 * nez + 1;
    nglob = NX * NY * NZ;
    gll5(zd, wd, hpd);
    for (int i = 0; i < NG; ++i) {
      w[i] = T(wd[i]);
      for (int j = 0; j < NG; ++j) { hp[i][j] = T(hpd[i][j]); hpw[i][j] = T(hpd[i][j] * wd[i]); }
    }
    dt = T(in.dt);
  }

  void corners(int e, double cn[8][3]) const {
    const int ex = e % nex, ey = (e / nex) % ney, ez = e / (nex * ney);
    for (int a = 0; a < 8; ++a) {
      const int i = ex + (CS[a][0] > 0), j = ey + (CS[a][1] > 0), k = ez + (CS[a][2] > 0);
      const double *p = in.nodes + 3 * ((size_t(k) * (ney + 1) + j) * (nex + 1) + i);
      for (int c = 0; c < 3; ++c) cn[a][c] = p[c];
    }
  }

  void setup() {
    const size_t nloc = size_t(nspec) * NP3;
    ibool.resize(nloc); g9.resize(nloc * 9); jac.resize(nloc); c0.resize(nloc); mu.resize(nloc);
    std::vector<double> mass(size_t(nglob), 0.0);
    for (int e = 0; e < nspec; ++e) {
      double cn[8][3];
      corners(e, cn);
      const int ex = e % nex, ey = (e / nex) % ney, ez = e / (nex * ney);
      for (int iz = 0; iz < NG; ++iz)
        for (int iy = 0; iy < NG; ++iy)
          for (int ix = 0; ix < NG; ++ix) {
            const int q = (iz * NG + iy) * NG + ix;
            const size_t p = size_t(e) * NP3 + q;
            ibool[p] = ((4 * ez + iz) * NY + 4 * ey + iy) * NX + 4 * ex + ix;
            const Geo G = map_point(cn, zd[ix], zd[iy], zd[iz]);
            if (!(G.jac > 0)) throw std::runtime_error("non-positive Jacobian");
            for (int k = 0; k < 3; ++k)
              for (int j = 0; j < 3; ++j) g9[p * 9 + k * 3 + j] = T(G.inv[k][j]);
            jac[p] = T(G.jac);
            const double rho = in.rho[p], vp = in.vp[p], vs = in.vs[p];
            const double m = rho * vs * vs;
            const double kappa = rho * (vp * vp - 4.0 / 3.0 * vs * vs);
            c0[p] = T(kappa + 4.0 / 3.0 * m);
            mu[p] = T(m);
            mass[size_t(ibool[p])] += rho * wd[ix] * wd[iy] * wd[iz] * G.jac;
          }
    }
    // Stacey faces (3D form of the 2D P-SV condition)
    std::vector<std::array<double, 3>> mstacey(size_t(nglob), {0.0, 0.0, 0.0});
    face_of_elem.assign(size_t(nspec), {});
    for (int e = 0; e < nspec; ++e) {
      const int ex = e % nex, ey = (e / nex) % ney, ez = e / (nex * ney);
      const bool on[6] = {ex == 0, ex == nex - 1, ey == 0, ey == ney - 1, ez == 0, ez == nez - 1};
      for (int f = 0; f < 6; ++f) {
        if (!on[f] || !in.absorbing[f]) continue;
        const int k = f / 2;                 // xi, eta or gamma face
        const int fix = (f % 2) ? NG - 1 : 0;
        const double sgn = (f % 2) ? 1.0 : -1.0;
        for (int b = 0; b < NG; ++b)
          for (int c = 0; c < NG; ++c) {
            int idx[3];
            idx[k] = fix;
            idx[(k + 1) % 3] = b;
            idx[(k + 2) % 3] = c;
            const int q = (idx[2] * NG + idx[1]) * NG + idx[0];
            const size_t p = size_t(e) * NP3 + q;
            double n[3];
            for (int j = 0; j < 3; ++j) n[j] = sgn * double(g9[p * 9 + k * 3 + j]) * double(jac[p]);
            const double rho = in.rho[p], vp = in.vp[p], vs = in.vs[p];
            const double wab = wd[b] * wd[c];
            Face F{e, q, {T(n[0]), T(n[1]), T(n[2])}, T(rho * vp), T(rho * vs), T(wab)};
            face_of_elem[size_t(e)].push_back(int(faces.size()));
            faces.push_back(F);
            // implicit mass term, velocity stand-in -dt/2 in every component
            const double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            const double vv = -double(in.dt) * 0.5;
            const double vn = vv * (n[0] + n[1] + n[2]);
            for (int j = 0; j < 3; ++j) {
              const double fj = (vn * n[j] / (nn * nn)) * (rho * vp - rho * vs) + vv * rho * vs;
              mstacey[size_t(ibool[p])][j] += -1.0 * fj * nn * wab;
            }
          }
      }
    }
    minv.assign(size_t(nglob) * 3, T(0));
    for (int g = 0; g < nglob; ++g)
      for (int j = 0; j < 3; ++j) minv[size_t(g) * 3 + j] = T(1.0 / (mass[g] + mstacey[g][j]));
    u.assign(size_t(nglob) * 3, T(0));
    v = u;
    a = u;
  }

  // element containing (x, y, z) and its local coordinates
  void locate(const double *X, int &elem, double xi[3]) const {
    // nearest control node, then Newton in the (up to 8) elements around it
    size_t best = 0;
    double bd = 1e300;
    const size_t nn = size_t(nex + 1) * (ney + 1) * (nez + 1);
    for (size_t i = 0; i < nn; ++i) {
      double d = 0;
      for (int c = 0; c < 3; ++c) d += (in.nodes[3 * i + c] - X[c]) * (in.nodes[3 * i + c] - X[c]);
      if (d < bd) { bd = d; best = i; }
    }
    const int ni = int(best % (nex + 1)), nj = int((best / (nex + 1)) % (ney + 1)),
              nk = int(best / (size_t(nex + 1) * (ney + 1)));
    double bestv = 1e300;
    elem = -1;
    for (int dk = -1; dk <= 0; ++dk)
      for (int dj = -1; dj <= 0; ++dj)
        for (int di = -1; di <= 0; ++di) {
          const int ex = ni + di, ey = nj + dj, ez = nk + dk;
          if (ex < 0 || ey < 0 || ez < 0 || ex >= nex || ey >= ney || ez >= nez) continue;
          const int e = (ez * ney + ey) * nex + ex;
          double cn[8][3];
          corners(e, cn);
          double s[3] = {0, 0, 0};
          for (int it = 0; it < 20; ++it) {
            const Geo G = map_point(cn, s[0], s[1], s[2]);
            double r[3];
            for (int c = 0; c < 3; ++c) r[c] = X[c] - G.x[c];
            for (int k = 0; k < 3; ++k) {
              double ds = 0;
              for (int j = 0; j < 3; ++j) ds += G.inv[k][j] * r[j];
              s[k] += ds;
            }
          }
          const double m = std::max({std::fabs(s[0]), std::fabs(s[1]), std::fabs(s[2])});
          // canonical choice on shared faces: the first element within 1e-9
          if (m < bestv - 1e-9) {
            bestv = m;
            elem = e;
            for (int c = 0; c < 3; ++c) xi[c] = std::min(1.0, std::max(-1.0, s[c]));
          }
        }
    if (elem < 0 || bestv > 1.0 + 1e-6) throw std::runtime_error("point outside the mesh");
  }

  void sources() {
    for (int s = 0; s < in.nsrc; ++s) {
      Src S;
      double xi[3];
      locate(in.src_xyz + 3 * s, S.e, xi);
      double h[3][NG], hd[3][NG];
      for (int k = 0; k < 3; ++k) lagrange(xi[k], zd, h[k], hd[k]);
      const double *cp = in.src_comp + 6 * s;
      if (in.src_kind[s] == 0) {
        for (int q = 0; q < NP3; ++q) {
          const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
          const double hl = h[0][ix] * h[1][iy] * h[2][iz];
          for (int c = 0; c < 3; ++c) S.arr[c][q] = T(hl * cp[c]);
        }
      } else {
        // M . grad(l l l) with the Jacobian interpolated at the source
        double J[3][3] = {{0}};
        for (int q = 0; q < NP3; ++q) {
          const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
          const double hl = h[0][ix] * h[1][iy] * h[2][iz];
          for (int k = 0; k < 3; ++k)
            for (int j = 0; j < 3; ++j) J[k][j] += hl * double(g9[(size_t(S.e) * NP3 + q) * 9 + k * 3 + j]);
        }
        const double M[3][3] = {{cp[0], cp[3], cp[4]}, {cp[3], cp[1], cp[5]}, {cp[4], cp[5], cp[2]}};
        for (int q = 0; q < NP3; ++q) {
          const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
          const double dxi[3] = {hd[0][ix] * h[1][iy] * h[2][iz], h[0][ix] * hd[1][iy] * h[2][iz],
                                 h[0][ix] * h[1][iy] * hd[2][iz]};
          double dsx[3] = {0, 0, 0};
          for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) dsx[j] += dxi[k] * J[k][j];
          for (int c = 0; c < 3; ++c) S.arr[c][q] = T(M[c][0] * dsx[0] + M[c][1] * dsx[1] + M[c][2] * dsx[2]);
        }
      }
      S.stf.resize(size_t(in.nstep));
      const T f0 = T(in.src_f0[s]), fac = T(in.src_factor[s]), tsh = T(in.src_tshift[s]);
      const T pi = T(M_PI);
      for (int i = 0; i < in.nstep; ++i) {
        const T t = T(in.t0) + T(i) * dt - tsh;
        const T aa = pi * pi * f0 * f0;
        S.stf[size_t(i)] = fac * ((T(1) - T(2) * aa * t * t) * std::exp(-aa * t * t));
      }
      srcs.push_back(std::move(S));
    }
  }

  void receivers() {
    for (int r = 0; r < in.nrec; ++r) {
      Rec R;
      double xi[3];
      locate(in.rec_xyz + 3 * r, R.e, xi);
      double h[3][NG], hd[3][NG];
      for (int k = 0; k < 3; ++k) lagrange(xi[k], zd, h[k], hd[k]);
      for (int q = 0; q < NP3; ++q) {
        const int ix = q % NG, iy = (q / NG) % NG, iz = q / (NG * NG);
        R.h[q] = T(h[0][ix] * h[1][iy] * h[2][iz]);
      }
      recs.push_back(R);
    }
  }

  // -K u (+ Stacey traction) of element e added into acc
  void element(int e, std::vector<T> &acc) const {
    T fu[NP3][3], F[NP3][3][3];
    const size_t base = size_t(e) * NP3;
    for (int q = 0; q < NP3; ++q)
      for (int c = 0; c < 3; ++c) fu[q][c] = u[size_t(ibool[base + q]) * 3 + c];
    for (int iz = 0; iz < NG; ++iz)
      for (int iy = 0; iy < NG; ++iy)
        for (int ix = 0; ix < NG; ++ix) {
          const int q = (iz * NG + iy) * NG + ix;
          const size_t p = base + q;
          T dxi[3][3];  // [comp][xi, eta, gamma]
          for (int c = 0; c < 3; ++c) {
            T s0 = 0, s1 = 0, s2 = 0;
            if (in.device_order) {
              for (int l = 0; l < NG; ++l) {
                s0 = std::fma(hp[ix][l], fu[(iz * NG + iy) * NG + l][c], s0);
                s1 = std::fma(hp[iy][l], fu[(iz * NG + l) * NG + ix][c], s1);
                s2 = std::fma(hp[iz][l], fu[(l * NG + iy) * NG + ix][c], s2);
              }
            } else {
              for (int l = 0; l < NG; ++l) {
                s0 += hp[ix][l] * fu[(iz * NG + iy) * NG + l][c];
                s1 += hp[iy][l] * fu[(iz * NG + l) * NG + ix][c];
                s2 += hp[iz][l] * fu[(l * NG + iy) * NG + ix][c];
              }
            }
            dxi[c][0] = s0; dxi[c][1] = s1; dxi[c][2] = s2;
          }
          const T *gi = &g9[p * 9];
          // device order: the map, the normal stresses and F as FMA chains,
          // as the CUDA element kernels compute them (dot3 / stress3)
          const bool dv = in.device_order;
          auto dot3 = [dv](T a0, T b0, T a1, T b1, T a2, T b2) {
            return dv ? T(std::fma(a2, b2, std::fma(a1, b1, a0 * b0))) : a0 * b0 + a1 * b1 + a2 * b2;
          };
          T du[3][3];  // du[c][j] = d u_c / d x_j
          for (int c = 0; c < 3; ++c)
            for (int j = 0; j < 3; ++j)
              du[c][j] = dot3(dxi[c][0], gi[0 * 3 + j], dxi[c][1], gi[1 * 3 + j], dxi[c][2], gi[2 * 3 + j]);
          const T l2m = c0[p], m = mu[p], lam = l2m - T(2) * m;
          T sig[3][3];
          if (dv) {
            sig[0][0] = std::fma(l2m, du[0][0], lam * (du[1][1] + du[2][2]));
            sig[1][1] = std::fma(l2m, du[1][1], lam * (du[0][0] + du[2][2]));
            sig[2][2] = std::fma(l2m, du[2][2], lam * (du[0][0] + du[1][1]));
          } else {
            sig[0][0] = l2m * du[0][0] + lam * (du[1][1] + du[2][2]);
            sig[1][1] = l2m * du[1][1] + lam * (du[0][0] + du[2][2]);
            sig[2][2] = l2m * du[2][2] + lam * (du[0][0] + du[1][1]);
          }
          sig[0][1] = sig[1][0] = m * (du[0][1] + du[1][0]);
          sig[0][2] = sig[2][0] = m * (du[0][2] + du[2][0]);
          sig[1][2] = sig[2][1] = m * (du[1][2] + du[2][1]);
          for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 3; ++k)
              F[q][c][k] = jac[p] * dot3(sig[c][0], gi[k * 3 + 0], sig[c][1], gi[k * 3 + 1], sig[c][2], gi[k * 3 + 2]);
        }
    T r[NP3][3];
    for (int iz = 0; iz < NG; ++iz)
      for (int iy = 0; iy < NG; ++iy)
        for (int ix = 0; ix < NG; ++ix) {
          const int q = (iz * NG + iy) * NG + ix;
          for (int c = 0; c < 3; ++c) {
            T t1 = 0, t2 = 0, t3 = 0;
            if (in.device_order) {
              for (int l = 0; l < NG; ++l) {
                t1 = std::fma(F[(iz * NG + iy) * NG + l][c][0], hpw[l][ix], t1);
                t2 = std::fma(F[(iz * NG + l) * NG + ix][c][1], hpw[l][iy], t2);
                t3 = std::fma(F[(l * NG + iy) * NG + ix][c][2], hpw[l][iz], t3);
              }
            } else {
              for (int l = 0; l < NG; ++l) {
                t1 += F[(iz * NG + iy) * NG + l][c][0] * hp[l][ix] * w[l];
                t2 += F[(iz * NG + l) * NG + ix][c][1] * hp[l][iy] * w[l];
                t3 += F[(l * NG + iy) * NG + ix][c][2] * hp[l][iz] * w[l];
              }
            }
            if (in.device_order) {
              const T wzy = w[iz] * w[iy], wzx = w[iz] * w[ix], wyx = w[iy] * w[ix];
              r[q][c] = -T(std::fma(wyx, t3, std::fma(wzx, t2, wzy * t1)));
            } else {
              r[q][c] = T(-1) * (w[iz] * w[iy] * t1 + w[iz] * w[ix] * t2 + w[iy] * w[ix] * t3);
            }
          }
        }
    for (int fi : face_of_elem[size_t(e)]) {
      const Face &F0 = faces[size_t(fi)];
      const T *vv = &v[size_t(ibool[base + F0.q]) * 3];
      const T nn2 = F0.n[0] * F0.n[0] + F0.n[1] * F0.n[1] + F0.n[2] * F0.n[2];
      const T nn = std::sqrt(nn2);
      const T vn = vv[0] * F0.n[0] + vv[1] * F0.n[1] + vv[2] * F0.n[2];
      for (int c = 0; c < 3; ++c) {
        const T f = ((vn * F0.n[c] / nn2) * (F0.rvp - F0.rvs)) + vv[c] * F0.rvs;
        r[F0.q][c] += T(-1) * f * nn * F0.w;
      }
    }
    for (int q = 0; q < NP3; ++q)
      for (int c = 0; c < 3; ++c) acc[size_t(ibool[base + q]) * 3 + c] += r[q][c];
  }

  void run(double *seis, double *final_u, int nthreads) {
    setup();
    sources();
    receivers();
    const T dt2 = dt / T(2), dtsq2 = dt * dt / T(2);
    const size_t n = size_t(nglob) * 3;
    std::vector<std::vector<int>> color(8);
    for (int e = 0; e < nspec; ++e) {
      const int ex = e % nex, ey = (e / nex) % ney, ez = e / (nex * ney);
      color[size_t((ex & 1) + 2 * (ey & 1) + 4 * (ez & 1))].push_back(e);
    }
    omp_set_num_threads(std::max(1, nthreads));
    const auto tl = std::chrono::steady_clock::now();
    for (int istep = 0; istep < in.nstep; ++istep) {
#pragma omp parallel for schedule(static)
      for (long long i = 0; i < (long long)n; ++i) {
        u[i] = u[i] + (dt * v[i] + dtsq2 * a[i]);
        v[i] = v[i] + dt2 * a[i];
        a[i] = T(0);
      }
      for (int c = 0; c < 8; ++c) {
        const auto &L = color[size_t(c)];
#pragma omp parallel for schedule(static)
        for (long long k = 0; k < (long long)L.size(); ++k) element(L[size_t(k)], a);
      }
      for (const Src &S : srcs)
        for (int q = 0; q < NP3; ++q)
          for (int c = 0; c < 3; ++c)
            a[size_t(ibool[size_t(S.e) * NP3 + q]) * 3 + c] += S.stf[size_t(istep)] * S.arr[c][q];
#pragma omp parallel for schedule(static)
      for (long long i = 0; i < (long long)n; ++i) {
        a[i] = a[i] * minv[i];
        v[i] = v[i] + dt2 * a[i];
      }
      for (int t = 0; t < in.ntypes; ++t) {
        const std::vector<T> &f = in.seis_types[t] == 0 ? u : (in.seis_types[t] == 1 ? v : a);
        for (int r = 0; r < in.nrec; ++r) {
          const Rec &R = recs[size_t(r)];
          for (int c = 0; c < 3; ++c) {
            T s = 0;
            for (int q = 0; q < NP3; ++q) s += R.h[q] * f[size_t(ibool[size_t(R.e) * NP3 + q]) * 3 + c];
            seis[((size_t(istep) * in.ntypes + t) * in.nrec + r) * 3 + c] = double(s);
          }
        }
      }
    }
    loop_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tl).count();
    if (final_u)
      for (size_t i = 0; i < n; ++i) final_u[i] = double(u[i]);
  }
  double loop_seconds = 0;
};

template <typename T>
int run_impl(const OracleInput3D *in, OracleOutput3D *out, int nthreads) {
  try {
    Sim3D<T> S(*in);
    out->nglob = S.nglob;
    S.run(out->seismograms, out->final_u, nthreads);
    out->seconds = S.loop_seconds;
    return 0;
  } catch (const std::exception &e) {
    std::snprintf(out->error, sizeof(out->error), "%s", e.what());
    return -1;
  }
}

}  // namespace

extern "C" {
int oracle3d_run_f32(const OracleInput3D *in, OracleOutput3D *out, int nthreads) {
  return run_impl<float>(in, out, nthreads);
}
int oracle3d_run_f64(const OracleInput3D *in, OracleOutput3D *out, int nthreads) {
  return run_impl<double>(in, out, nthreads);
}
}
