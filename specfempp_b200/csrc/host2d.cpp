// Host-side assembly of libsfg (see host2d.hpp).  Plain C++17, no CUDA.
#include "host2d.hpp"

#include <algorithm>
#include <map>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <stdexcept>
#include <unordered_map>

namespace sfg {

namespace {

constexpr int BOTTOM = 0, RIGHT = 1, TOP = 2, LEFT = 3;

// ----------------------------------------------------------- database.bin ---
// Record layout per src/io/mesh/impl/fortran/dim2/{read_mesh_database,
// read_parameters,read_material_properties,read_boundaries,read_elements,
// read_adjacency_graph}.cpp and mesh.cpp:26-215.
struct RecordReader {
  std::vector<char> buf;
  size_t pos = 0;
  std::vector<std::pair<size_t, int>> recs;  // offset, length
  size_t cur = 0;
  bool load(const std::string &path, std::string &err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "Could not open database file: " + path; return false; }
    buf.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    while (pos < buf.size()) {
      if (pos + 4 > buf.size()) { err = "truncated record header"; return false; }
      int n;
      std::memcpy(&n, &buf[pos], 4);
      if (n < 0 || pos + 8 + size_t(n) > buf.size()) { err = "truncated database record"; return false; }
      int n2;
      std::memcpy(&n2, &buf[pos + 4 + n], 4);
      if (n2 != n) { err = "record length markers differ"; return false; }
      recs.push_back({pos + 4, n});
      pos += 8 + size_t(n);
    }
    return true;
  }
  bool more() const { return cur < recs.size(); }
  int len() const { return recs[cur].second; }
  const char *next(int expect_min = 0) {
    if (cur >= recs.size()) throw std::runtime_error("database ended early");
    if (recs[cur].second < expect_min) throw std::runtime_error("short database record");
    return &buf[recs[cur++].first];
  }
};

template <typename T>
T rd(const char *&p) {
  T v;
  std::memcpy(&v, p, sizeof(T));
  p += sizeof(T);
  return v;
}

// -------------------------------------------------------------- GLL ---
double legendre(double x, int n) {
  double p0 = 1.0, p1 = x;
  for (int k = 1; k < n; ++k) {
    double p2 = ((2.0 * k + 1.0) * x * p1 - k * p0) / (k + 1.0);
    p0 = p1;
    p1 = p2;
  }
  return n == 0 ? 1.0 : p1;
}

void gll(double z[NGLL], double w[NGLL], double hp[NGLL][NGLL]) {
  const int N = NGLL - 1;
  // nodes: +-1 and the roots of P'_4; for degree 4 these are 0 and +-sqrt(3/7)
  const double r = std::sqrt(3.0 / 7.0);
  const double zz[NGLL] = {-1.0, -r, 0.0, r, 1.0};
  for (int i = 0; i < NGLL; ++i) {
    z[i] = zz[i];
    const double p = legendre(z[i], N);
    w[i] = 2.0 / (N * (N + 1.0) * p * p);
  }
  for (int i = 0; i < NGLL; ++i)
    for (int j = 0; j < NGLL; ++j) {
      if (i == j) hp[i][j] = (i == 0) ? -0.25 * N * (N + 1.0) : (i == N ? 0.25 * N * (N + 1.0) : 0.0);
      else hp[i][j] = legendre(z[i], N) / (legendre(z[j], N) * (z[i] - z[j]));
    }
}

void lagrange(double xi, const double z[NGLL], double h[NGLL]) {
  for (int d = 0; d < NGLL; ++d) {
    double num = 1, den = 1;
    for (int i = 0; i < NGLL; ++i)
      if (i != d) { num *= xi - z[i]; den *= z[d] - z[i]; }
    h[d] = num / den;
  }
}

// Lagrange interpolants and their derivatives at xi
// (src/quadrature/gll/lagrange_poly.cpp:12-44).
void lagrange_d(double xi, const double z[NGLL], double h[NGLL], double hp[NGLL]) {
  lagrange(xi, z, h);
  for (int d = 0; d < NGLL; ++d) {
    double den = 1, sum = 0;
    for (int i = 0; i < NGLL; ++i) {
      if (i == d) continue;
      den *= z[d] - z[i];
      double p = 1;
      for (int j = 0; j < NGLL; ++j)
        if (j != d && j != i) p *= xi - z[j];
      sum += p;
    }
    hp[d] = sum / den;
  }
}

// ----------------------------------------------------- shape functions ---
void shape(int ngnod, double xi, double ga, double *s, double *dx, double *dg) {
  if (ngnod == 4) {
    s[0] = 0.25 * (xi - 1) * (ga - 1); s[1] = -0.25 * (xi + 1) * (ga - 1);
    s[2] = 0.25 * (xi + 1) * (ga + 1); s[3] = -0.25 * (xi - 1) * (ga + 1);
    dx[0] = 0.25 * (ga - 1); dx[1] = -0.25 * (ga - 1); dx[2] = 0.25 * (ga + 1); dx[3] = -0.25 * (ga + 1);
    dg[0] = 0.25 * (xi - 1); dg[1] = -0.25 * (xi + 1); dg[2] = 0.25 * (xi + 1); dg[3] = -0.25 * (xi - 1);
    return;
  }
  // 9-node Lagrange quadrilateral (corners, edge mid-points, centre)
  const double lx[3] = {0.5 * xi * (xi - 1), 1 - xi * xi, 0.5 * xi * (xi + 1)};
  const double lg[3] = {0.5 * ga * (ga - 1), 1 - ga * ga, 0.5 * ga * (ga + 1)};
  const double dlx[3] = {xi - 0.5, -2 * xi, xi + 0.5};
  const double dlg[3] = {ga - 0.5, -2 * ga, ga + 0.5};
  // node n -> (index along xi, index along gamma)
  const int ix[9] = {0, 2, 2, 0, 1, 2, 1, 0, 1};
  const int ig[9] = {0, 0, 2, 2, 0, 1, 2, 1, 1};
  for (int n = 0; n < 9; ++n) {
    s[n] = lx[ix[n]] * lg[ig[n]];
    dx[n] = dlx[ix[n]] * lg[ig[n]];
    dg[n] = lx[ix[n]] * dlg[ig[n]];
  }
}

struct JacD {
  double xix, xiz, gax, gaz, jac, x, z;
};

JacD jacobian(const Mesh2D &m, int e, double xi, double ga) {
  double s[9], dx[9], dg[9];
  shape(m.ngnod, xi, ga, s, dx, dg);
  double xxi = 0, zxi = 0, xga = 0, zga = 0, x = 0, z = 0;
  for (int n = 0; n < m.ngnod; ++n) {
    const int id = m.knods[size_t(e) * m.ngnod + n];
    const double cx = m.coorg[2 * size_t(id)], cz = m.coorg[2 * size_t(id) + 1];
    xxi += dx[n] * cx; zxi += dx[n] * cz; xga += dg[n] * cx; zga += dg[n] * cz;
    x += s[n] * cx; z += s[n] * cz;
  }
  const double j = xxi * zga - xga * zxi;
  return {zga / j, -xga / j, -zxi / j, xxi / j, j, x, z};
}

bool on_edge(int type, int iz, int ix) {
  return (type == TOP && iz == NGLL - 1) || (type == BOTTOM && iz == 0) ||
         (type == LEFT && ix == 0) || (type == RIGHT && ix == NGLL - 1);
}

// outward (unnormalised) edge normal of an element at a point, scaled by |J|
// (core/specfem/point/jacobian_matrix.hpp:424-449)
void edge_normal(const JacD &J, int type, double &nx, double &nz) {
  switch (type) {
    case BOTTOM: nx = -J.gax * J.jac; nz = -J.gaz * J.jac; break;
    case TOP: nx = J.gax * J.jac; nz = J.gaz * J.jac; break;
    case LEFT: nx = -J.xix * J.jac; nz = -J.xiz * J.jac; break;
    default: nx = J.xix * J.jac; nz = J.xiz * J.jac; break;
  }
}

// Per-point words of an isotropic poroelastic material
// (include/medium/dim2/poroelastic/isotropic/material.hpp: Biot coefficients
// evaluated as the reference does, FP32 values with double literals;
// properties.hpp: rho_bar, the inverse permeability).
struct PoroWords {
  float H, mu, C, M, phi_tort, rhof_rhobar, exx, exz, ezz;
};

PoroWords poro_words(const double *v) {
  if (std::abs(float(v[12]) - 9999.0) > 1e-6)
    throw std::runtime_error("poroelastic attenuation (Q_mu != 9999) is not implemented");
  const float rhos = float(v[0]), rhof = float(v[1]), phi = float(v[2]), tort = float(v[3]);
  const float kxx = float(v[4]), kxz = float(v[5]), kzz = float(v[6]);
  const float ks = float(v[7]), kf = float(v[8]), kfr = float(v[9]), eta = float(v[10]), mufr = float(v[11]);
  const float D = float(double(ks) * (1.0 + double(phi) * (double(ks / kf) - 1.0)));
  const float fac = float(1.0 / double(D - kfr));
  PoroWords P;
  P.H = float(double((ks - kfr) * (ks - kfr) * fac + kfr) + 4.0 / 3.0 * double(mufr));
  P.C = ks * (ks - kfr) * fac;
  P.M = ks * ks * fac;
  P.mu = mufr;
  P.phi_tort = phi / tort;
  const float rb = ((1.0f - phi) * rhos) + (phi * rhof);
  P.rhof_rhobar = rhof / rb;
  const float det = kxx * kzz - kxz * kxz;
  P.exx = eta * (kzz / det);
  P.exz = eta * (-1.0f * kxz / det);
  P.ezz = eta * (kxx / det);
  return P;
}

// (xi, gamma) of local coordinate c along an edge: xi runs along bottom and
// top, gamma along left and right.
void edge_local(int t, double c, double &xi, double &ga) {
  if (t == BOTTOM) { xi = c; ga = -1; }
  else if (t == RIGHT) { xi = 1; ga = c; }
  else if (t == TOP) { xi = c; ga = 1; }
  else { xi = -1; ga = c; }
}

// Local coordinate along edge t of element e of the point closest to
// (X, Z): Newton steps from 0 on the edge coordinate, clamped to [-1, 1],
// stopping at an end whose step points outside
// (src/algorithms/dim2/locate_point_impl.cpp:126-198).
double edge_coordinate(const Mesh2D &m, int e, int t, double X, double Z) {
  double xi, ga;
  edge_local(t, 0.0, xi, ga);
  double &c = (t == BOTTOM || t == TOP) ? xi : ga;
  for (int it = 0; it < 100; ++it) {
    const JacD J = jacobian(m, e, xi, ga);
    const double dx = -(J.x - X), dz = -(J.z - Z);
    const double d = (t == BOTTOM || t == TOP) ? J.xix * dx + J.xiz * dz : J.gax * dx + J.gaz * dz;
    if (c == -1.0 && d < -1e-12) return -1.0;
    if (c == 1.0 && d > 1e-12) return 1.0;
    c = std::min(1.0, std::max(-1.0, c + d));
    if (std::abs(d) < 1e-12) break;
  }
  return c;
}

int edge_point(int t, int k) {
  return t == BOTTOM ? k : t == RIGHT ? k * NGLL + NGLL - 1 : t == TOP ? (NGLL - 1) * NGLL + k : k * NGLL;
}

// Coupling weights of one nonconforming edge pair: the self edge (e1, t1)
// receives at its point i sum_j W[i][j] * (field of the coupled edge (e2,
// t2) at its point j), W[i][j] = sum_q T1[q][i] f[q] n[q] T2[q][j] over an
// NGLL-point GLL quadrature mapped linearly onto the edges' intersection in
// the self edge's local coordinate; T1, T2 are the Lagrange interpolants at
// the quadrature points on each edge, f[q] = w_q |dx/dxi| and n[q] the self
// element's outward unit normal from the derivative of the mapped points
// (core/specfem/assembly/nonconforming_interfaces/dim2/impl/compute_intersection.cpp:49-167,
// impl/interface_container.tpp:20-180; applied as in
// include/kokkos_kernels/impl/compute_coupling.tpp:117-249).
void nonconforming_weights(const Mesh2D &m, const double z[NGLL], const double w[NGLL],
                           const double hp[NGLL][NGLL], int e1, int t1, int e2, int t2,
                           double W[NGLL][NGLL][2]) {
  auto corner = [&](int e, int k, double &x, double &zz) {
    const int id = m.knods[size_t(e) * m.ngnod + k];
    x = m.coorg[2 * size_t(id)];
    zz = m.coorg[2 * size_t(id) + 1];
  };
  auto ends = [](int t, int &a, int &b) {
    if (t == BOTTOM) { a = 0; b = 1; } else if (t == RIGHT) { a = 1; b = 2; }
    else if (t == TOP) { a = 3; b = 2; } else { a = 0; b = 3; }
  };
  int a1, b1, a2, b2;
  ends(t1, a1, b1);
  ends(t2, a2, b2);
  double x, zz;
  corner(e2, a2, x, zz); const double p2lo = edge_coordinate(m, e1, t1, x, zz);
  corner(e2, b2, x, zz); const double p2hi = edge_coordinate(m, e1, t1, x, zz);
  corner(e1, a1, x, zz); const double p1lo = edge_coordinate(m, e2, t2, x, zz);
  corner(e1, b1, x, zz); const double p1hi = edge_coordinate(m, e2, t2, x, zz);
  const double min1 = std::min(p2lo, p2hi), max1 = std::max(p2lo, p2hi);
  const double min2 = std::min(p1lo, p1hi), max2 = std::max(p1lo, p1hi);
  if (min1 > max1 - 1e-5 || min2 > max2 - 1e-5)
    throw std::runtime_error("nonconforming edges without an intersection");
  double T1[NGLL][NGLL], T2[NGLL][NGLL], lx[NGLL], lz[NGLL];
  for (int q = 0; q < NGLL; ++q) {
    const double c1 = 0.5 * ((max1 - min1) * z[q] + (max1 + min1));
    double xi, ga;
    edge_local(t1, c1, xi, ga);
    const JacD J = jacobian(m, e1, xi, ga);
    lagrange(c1, z, T1[q]);
    lagrange(edge_coordinate(m, e2, t2, J.x, J.z), z, T2[q]);
  }
  for (int k = 0; k < NGLL; ++k) {
    double lc = 0, xi, ga;
    for (int i = 0; i < NGLL; ++i) lc += T1[k][i] * z[i];
    edge_local(t1, lc, xi, ga);
    const JacD J = jacobian(m, e1, xi, ga);
    lx[k] = J.x;
    lz[k] = J.z;
  }
  for (int i = 0; i < NGLL; ++i)
    for (int j = 0; j < NGLL; ++j) W[i][j][0] = W[i][j][1] = 0.0;
  for (int q = 0; q < NGLL; ++q) {
    double drx = 0, drz = 0;
    for (int k = 0; k < NGLL; ++k) { drx += hp[q][k] * lx[k]; drz += hp[q][k] * lz[k]; }
    const double f = w[q] * std::sqrt(drx * drx + drz * drz);
    double mag = std::sqrt(drx * drx + drz * drz);
    if (t1 == TOP || t1 == LEFT) mag = -mag;
    const double nx = drz / mag, nz = -drx / mag;
    for (int i = 0; i < NGLL; ++i)
      for (int j = 0; j < NGLL; ++j) {
        const double c = T1[q][i] * f * T2[q][j];
        W[i][j][0] += c * nx;
        W[i][j][1] += c * nz;
      }
  }
}

// Spread the low 32 bits of x to the even bits of a 64-bit word.
uint64_t spread_bits(uint64_t x) {
  x &= 0xffffffffull;
  x = (x | (x << 16)) & 0x0000ffff0000ffffull;
  x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
  x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}

// Tiles of TILE_E compute elements of one medium: the elements sorted by the
// Morton code of their centre on a grid whose cell is the median element
// extent (on a structured mesh the cell indices are the element's column and
// row, and every aligned run of 16 codes is a 4 x 4 block of elements), then
// cut into consecutive runs.  Returns [ntiles][TILE_E] compute elements, -1
// past the last element.
std::vector<int> make_tiles(const Assembly2D &a, const std::vector<int> &elem_mesh) {
  const int n = int(elem_mesh.size());
  if (n == 0) return {};
  std::vector<double> cx(n), cz(n), ext(n);
  for (int ce = 0; ce < n; ++ce) {
    const size_t p = size_t(elem_mesh[ce]) * NPTS;
    double x0 = 1e300, x1 = -1e300, z0 = 1e300, z1 = -1e300;
    for (int q = 0; q < NPTS; ++q) {
      x0 = std::min(x0, a.gx[p + q]); x1 = std::max(x1, a.gx[p + q]);
      z0 = std::min(z0, a.gz[p + q]); z1 = std::max(z1, a.gz[p + q]);
    }
    cx[ce] = 0.25 * (a.gx[p] + a.gx[p + 4] + a.gx[p + 20] + a.gx[p + 24]);
    cz[ce] = 0.25 * (a.gz[p] + a.gz[p + 4] + a.gz[p + 20] + a.gz[p + 24]);
    ext[ce] = std::max(x1 - x0, z1 - z0);
  }
  std::vector<double> e2 = ext;
  std::nth_element(e2.begin(), e2.begin() + n / 2, e2.end());
  const double cell = e2[n / 2] > 0 ? e2[n / 2] : 1.0;
  const double xmin = *std::min_element(cx.begin(), cx.end());
  const double zmin = *std::min_element(cz.begin(), cz.end());
  std::vector<std::pair<uint64_t, int>> key(n);
  for (int ce = 0; ce < n; ++ce) {
    const double fx = std::floor((cx[ce] - xmin) / cell + 0.5), fz = std::floor((cz[ce] - zmin) / cell + 0.5);
    const uint64_t ix = uint64_t(std::min(std::max(fx, 0.0), 4.0e9));
    const uint64_t iz = uint64_t(std::min(std::max(fz, 0.0), 4.0e9));
    key[ce] = {spread_bits(ix) | (spread_bits(iz) << 1), ce};
  }
  std::sort(key.begin(), key.end());
  const int ntiles = (n + TILE_E - 1) / TILE_E;
  std::vector<int> tiles(size_t(ntiles) * TILE_E, -1);
  for (int i = 0; i < n; ++i) tiles[i] = key[i].second;
  return tiles;
}

}  // namespace

bool read_database2d(const std::string &path, Mesh2D &m, std::string &err) {
  RecordReader r;
  if (!r.load(path, err)) return false;
  try {
    r.next();                                   // title
    r.next();                                   // noise tomography, PML flags
    { const char *p = r.next(4); m.nspec = rd<int>(p); }
    { const char *p = r.next(8); m.npgeo = rd<int>(p); }
    for (int i = 0; i < 38; ++i) r.next();
    if (r.len() == 16) r.next();                // optional electromagnetic record
    for (int i = 0; i < 22; ++i) r.next();
    m.coorg.assign(2 * size_t(m.npgeo), 0.0);
    for (int i = 0; i < m.npgeo; ++i) {
      const char *p = r.next(20);
      int ip = rd<int>(p);
      double x = rd<double>(p), z = rd<double>(p);
      if (ip < 1 || ip > m.npgeo) throw std::runtime_error("Error reading coordinates");
      m.coorg[2 * size_t(ip - 1)] = x;
      m.coorg[2 * size_t(ip - 1) + 1] = z;
    }
    int nelemabs, nacforcing, nacsurf, nfs, nfp, nsp, ntang, naxis;
    {
      const char *p = r.next(20);
      m.numat = rd<int>(p); m.ngnod = rd<int>(p);
      int ns = rd<int>(p);
      if (ns != m.nspec) throw std::runtime_error("nspec mismatch");
    }
    {
      const char *p = r.next(32);
      nelemabs = rd<int>(p); nacforcing = rd<int>(p); nacsurf = rd<int>(p); nfs = rd<int>(p);
      nfp = rd<int>(p); nsp = rd<int>(p); ntang = rd<int>(p); naxis = rd<int>(p);
    }
    if (m.ngnod != 4 && m.ngnod != 9) throw std::runtime_error("ngnod must be 4 or 9");
    r.next();                                   // attenuation
    m.mat_medium.resize(m.numat); m.mat_rho.resize(m.numat);
    m.mat_vp.resize(m.numat); m.mat_vs.resize(m.numat);
    for (int i = 0; i < m.numat; ++i) {
      const char *p = r.next(112);
      int n = rd<int>(p), indic = rd<int>(p);
      double v[13];
      for (double &x : v) x = rd<double>(p);
      if (n != i + 1) throw std::runtime_error("Wrong material set number");
      if (indic == 2) {
        // anisotropic elastic: rho, c11, c13, c15, c33, c35, c55, c12, c23, c25
        // (src/io/mesh/impl/fortran/dim2/read_material_properties.cpp:252-291)
        if (m.mat_aniso.empty()) m.mat_aniso.assign(size_t(m.numat) * 6, std::nan(""));
        for (int k = 0; k < 6; ++k) m.mat_aniso[size_t(i) * 6 + k] = v[1 + k];
        m.mat_rho[i] = v[0];
        m.mat_vp[i] = std::sqrt(v[4] / v[0]);
        m.mat_vs[i] = std::sqrt(v[6] / v[0]);
        m.mat_medium[i] = 1;
        continue;
      }
      if (indic == 5) {
        // isotropic Cosserat elastic (P-SV-T): rho, kappa, mu, nu, j, lambda_c,
        // mu_c, nu_c (read_material_properties.cpp:366-395)
        if (m.mat_cosserat.empty()) m.mat_cosserat.assign(size_t(m.numat) * 8, std::nan(""));
        for (int k = 0; k < 8; ++k) m.mat_cosserat[size_t(i) * 8 + k] = v[k];
        m.mat_rho[i] = v[0];
        m.mat_vp[i] = std::sqrt((v[1] + 4.0 / 3.0 * v[2]) / v[0]);
        m.mat_vs[i] = std::sqrt(v[2] / v[0]);
        m.mat_medium[i] = 1;
        continue;
      }
      if (indic == 3) {
        // isotropic poroelastic: rho_s, rho_f, phi, tortuosity, kxx, kxz, kzz,
        // kappa_s, kappa_f, kappa_fr, eta_f, mu_fr, Q_mu
        // (read_material_properties.cpp:303-332)
        if (m.mat_poro.empty()) m.mat_poro.assign(size_t(m.numat) * 13, std::nan(""));
        for (int k = 0; k < 13; ++k) m.mat_poro[size_t(i) * 13 + k] = v[k];
        m.mat_rho[i] = (1.0 - v[2]) * v[0] + v[2] * v[1];
        m.mat_vp[i] = m.mat_vs[i] = 0.0;
        m.mat_medium[i] = 1;
        continue;
      }
      if (indic != 1)
        throw std::runtime_error("only isotropic, anisotropic, Cosserat and poroelastic elastic and acoustic materials are supported");
      m.mat_rho[i] = v[0]; m.mat_vp[i] = v[1]; m.mat_vs[i] = v[2];
      m.mat_medium[i] = (v[2] == 0.0) ? 0 : 1;
    }
    m.knods.assign(size_t(m.nspec) * m.ngnod, -1);
    m.kmato.assign(m.nspec, -1);
    for (int i = 0; i < m.nspec; ++i) {
      const char *p = r.next(4 * (3 + m.ngnod));
      int n = rd<int>(p), km = rd<int>(p);
      if (n < 1 || n > m.nspec || km < 1 || km > m.numat) throw std::runtime_error("bad element record");
      for (int k = 0; k < m.ngnod; ++k) {
        int id = rd<int>(p);
        if (id < 1 || id > m.npgeo) throw std::runtime_error("Error reading knods (node_id) values");
        m.knods[size_t(n - 1) * m.ngnod + k] = id - 1;
      }
      m.kmato[n - 1] = km - 1;
    }
    r.next();                                   // ninterfaces, max_interface_size
    for (int i = 0; i < std::max(nelemabs, 0); ++i) {
      const char *p = r.next(56);
      int num = rd<int>(p);
      int c[4];
      for (int &x : c) x = rd<int>(p);
      int cnt = (c[0] != 0) + (c[1] != 0) + (c[2] != 0) + (c[3] != 0);
      if (cnt != 1) throw std::runtime_error("must have one and only one absorbing edge per absorbing line cited");
      if (num < 1 || num > m.nspec) throw std::runtime_error("Wrong absorbing element number");
      m.abs_ispec.push_back(num - 1);
      m.abs_type.push_back(c[0] ? BOTTOM : c[1] ? RIGHT : c[2] ? TOP : LEFT);
    }
    for (int i = 0; i < nacsurf; ++i) {
      const char *p = r.next(16);
      int isp = rd<int>(p), kind = rd<int>(p), e1 = rd<int>(p) - 1, e2 = rd<int>(p) - 1;
      if (isp < 1 || isp > m.nspec) throw std::runtime_error("bad free-surface element");
      if (kind == 1) throw std::runtime_error("single-node acoustic free surface records are not supported");
      const int *kn = &m.knods[size_t(isp - 1) * m.ngnod];
      auto is = [&](int a, int b) { return (e1 == kn[a] && e2 == kn[b]) || (e1 == kn[b] && e2 == kn[a]); };
      int t = is(0, 1) ? BOTTOM : is(0, 3) ? LEFT : is(1, 2) ? RIGHT : is(2, 3) ? TOP : -1;
      if (t < 0) throw std::runtime_error("Could not generate type of acoustic free surface boundary");
      m.free_ispec.push_back(isp - 1);
      m.free_type.push_back(t);
    }
    for (int i = 0; i < nacforcing; ++i) r.next();
    for (int i = 0; i < nfs + nfp + nsp; ++i) r.next();
    r.next();                                   // tangential flags
    for (int i = 0; i < ntang; ++i) r.next();
    for (int i = 0; i < naxis; ++i) r.next();
    if (r.more()) {
      // adjacency graph (src/io/mesh/impl/fortran/dim2/read_adjacency_graph.cpp:11-40)
      const char *p = r.next(4);
      int nadj = rd<int>(p);
      m.adjacency.reserve(4 * size_t(std::max(nadj, 0)));
      for (int i = 0; i < nadj; ++i) {
        const char *q = r.next(16);
        const int e = rd<int>(q), nb = rd<int>(q), conn = rd<int>(q), orient = rd<int>(q);
        if (conn != 1 && conn != 3) throw std::runtime_error("Unknown connection type in adjacency graph.");
        if (e < 1 || e > m.nspec || nb < 1 || nb > m.nspec || orient < 1 || orient > 8)
          throw std::runtime_error("bad adjacency record");
        m.adjacency.insert(m.adjacency.end(), {e - 1, nb - 1, conn, orient - 1});
      }
    }
    if (r.more()) throw std::runtime_error("The Database file wasn't fully read");
  } catch (const std::exception &ex) {
    err = ex.what();
    return false;
  }
  return true;
}

// --------------------------------------------------- model-dependent part ---
// Material words, Stacey impedances, the assembled Stacey matrices and the
// inverse mass matrix: everything that changes when the model changes.
void assemble_model2d(const Mesh2D &m, Assembly2D &a) {
  const double dt = a.dt;
  double w[NGLL];
  for (int i = 0; i < NGLL; ++i) w[i] = double(a.wgll_d[i]);
  auto model = [&](int e, size_t pm, double &rho, double &vp, double &vs) {
    const int mat = m.kmato[e];
    rho = m.prho.empty() ? m.mat_rho[mat] : m.prho[pm];
    vp = m.pvp.empty() ? m.mat_vp[mat] : m.pvp[pm];
    vs = m.pvs.empty() ? m.mat_vs[mat] : m.pvs[pm];
  };
  auto aniso_of = [&](int e) -> const double * {
    if (m.mat_aniso.empty()) return nullptr;
    const double *c = &m.mat_aniso[size_t(m.kmato[e]) * 6];
    return std::isfinite(c[0]) ? c : nullptr;
  };
  a.el.aniso = false;
  for (int ce = 0; ce < a.el.nspec; ++ce) a.el.aniso |= aniso_of(a.el.elem_mesh[ce]) != nullptr;
  a.el.cosserat = a.el.ncomp == 3;
  a.el.poro = a.el.ncomp == 4;
  if (a.el.poro && (a.el.niface > 0 || a.el.aniso || !m.prho.empty()))
    throw std::runtime_error("poroelastic media: material constants only, not coupled to acoustic media");
  auto poro_of = [&](int e) { return &m.mat_poro[size_t(m.kmato[e]) * 13]; };
  if (a.el.cosserat && a.el.niface > 0)
    throw std::runtime_error("Cosserat media are not coupled to acoustic ones here");
  if (a.el.cosserat && (a.el.aniso || !m.prho.empty()))
    throw std::runtime_error("Cosserat media: material constants only (no anisotropy, no point models)");
  auto cos_of = [&](int e) { return &m.mat_cosserat[size_t(m.kmato[e]) * 8]; };
  if (a.el.aniso && (a.el.ncomp != 2 || !m.prho.empty()))
    throw std::runtime_error("anisotropic media: P-SV with material constants only (no SH, no point models)");
  for (int med = 0; med < 2; ++med) {
    MediumData &D = med == 1 ? a.el : a.ac;
    const size_t n = size_t(D.nspec) * NPTS;
    D.prop0.resize(n);
    D.prop1.resize(n);
    for (auto *v : {&D.prop2, &D.prop3, &D.prop4, &D.prop5}) v->assign(med == 1 && D.aniso ? n : 0, 0.0f);
    if (med == 1 && D.cosserat) for (auto *v : {&D.prop2, &D.prop3}) v->assign(n, 0.0f);
    for (auto *v : {&D.prop6, &D.prop7, &D.prop8}) v->assign(med == 1 && D.poro ? n : 0, 0.0f);
    if (med == 1 && D.poro)
      for (auto *v : {&D.prop2, &D.prop3, &D.prop4, &D.prop5}) v->assign(n, 0.0f);
    for (int ce = 0; ce < D.nspec; ++ce) {
      const int e = D.elem_mesh[ce];
      for (int q = 0; q < NPTS; ++q) {
        const size_t pm = size_t(e) * NPTS + q, pc = size_t(ce) * NPTS + q;
        double rho, vp, vs;
        model(e, pm, rho, vp, vs);
        if (med == 1 && D.poro) {
          const PoroWords P = poro_words(poro_of(e));
          D.prop0[pc] = P.H; D.prop1[pc] = P.mu; D.prop2[pc] = P.C; D.prop3[pc] = P.M;
          D.prop4[pc] = P.phi_tort; D.prop5[pc] = P.rhof_rhobar;
          D.prop6[pc] = P.exx; D.prop7[pc] = P.exz; D.prop8[pc] = P.ezz;
        } else if (med == 1 && D.cosserat) {
          // lambda = kappa - 2/3 mu, mu, nu, mu_c + nu_c
          // (include/medium/dim2/elastic/isotropic_cosserat/properties.hpp, stress.hpp)
          const double *c = cos_of(e);
          D.prop0[pc] = float(c[1] - 2.0 / 3.0 * c[2]);
          D.prop1[pc] = float(c[2]);
          D.prop2[pc] = float(c[3]);
          D.prop3[pc] = float(c[6] + c[7]);
        } else if (med == 1 && D.aniso) {
          // c11, c13, c15, c33, c35, c55 (include/medium/dim2/elastic/anisotropic/
          // properties.hpp); isotropic elements of the medium in the same form
          const double *c = aniso_of(e);
          const double mu = rho * vs * vs, l2m = rho * vp * vp;
          const double iso[6] = {l2m, l2m - 2.0 * mu, 0.0, l2m, 0.0, mu};
          const double *cc = c ? c : iso;
          D.prop0[pc] = float(cc[0]); D.prop1[pc] = float(cc[1]); D.prop2[pc] = float(cc[2]);
          D.prop3[pc] = float(cc[3]); D.prop4[pc] = float(cc[4]); D.prop5[pc] = float(cc[5]);
        } else if (med == 1) {
          // kappa = rho (vp^2 - 4/3 vs^2), mu = rho vs^2; lambda+2mu = kappa + 4/3 mu
          // (include/medium/dim2/elastic/isotropic/material.hpp:66-69, properties.hpp:71-91)
          const double mu = rho * vs * vs;
          const double kappa = rho * (vp * vp - 4.0 / 3.0 * vs * vs);
          D.prop0[pc] = float(kappa + 4.0 / 3.0 * mu);
          D.prop1[pc] = float(mu);
        } else {
          D.prop0[pc] = float(1.0 / rho);            // rho_inverse
          D.prop1[pc] = float(rho * vp * vp);        // kappa
        }
      }
    }
    // Stacey impedances
    for (int ce = 0; ce < D.nspec; ++ce) {
      if (D.bc_slot[ce] < 0) continue;
      const int e = D.elem_mesh[ce];
      for (int q = 0; q < NPTS; ++q) {
        const size_t k = size_t(D.bc_slot[ce]) * NPTS + q;
        if (D.bc_w[k] == 0.0f) continue;
        const size_t pm = size_t(e) * NPTS + q, pc = size_t(ce) * NPTS + q;
        double rho, vp, vs;
        model(e, pm, rho, vp, vs);
        if (med == 1 && D.poro) throw std::runtime_error("Stacey edges on poroelastic media are not supported");
        if (med == 1 && D.cosserat) {
          // rho vp = sqrt((kappa + 4/3 mu) rho), rho vs = rho sqrt((mu + nu) / rho),
          // j sqrt((mu_c + nu_c) / j) (stacey.tpp:183-230)
          const double *c = cos_of(e);
          D.bc_imp0[k] = float(std::sqrt((c[1] + 4.0 / 3.0 * c[2]) * c[0]));
          D.bc_imp1[k] = float(c[0] * std::sqrt((c[2] + c[3]) / c[0]));
          D.bc_imp2[k] = float(c[4] * std::sqrt((c[6] + c[7]) / c[4]));
        } else if (med == 1 && D.aniso) {
          // rho vp = sqrt(rho c33), rho vs = sqrt(rho c55)
          // (include/medium/dim2/elastic/anisotropic/properties.hpp:88-94)
          D.bc_imp0[k] = float(std::sqrt(rho * double(D.prop3[pc])));
          D.bc_imp1[k] = float(std::sqrt(rho * double(D.prop5[pc])));
        } else if (med == 1) {
          // rho*vp = sqrt((lambda+2mu)/rho)*rho, rho*vs = sqrt(rho*mu) (properties.hpp:77-87)
          const double l2m = D.prop0[pc], mu = D.prop1[pc];
          D.bc_imp0[k] = float(std::sqrt(l2m / rho) * rho);
          D.bc_imp1[k] = float(std::sqrt(rho * mu));
        } else {
          // 1/(rho vp) = sqrt(rho_inverse / kappa) (acoustic properties.hpp:69-72)
          D.bc_imp0[k] = float(std::sqrt(double(D.prop0[pc]) / double(D.prop1[pc])));
        }
      }
    }
  }
  // assembled per-point Stacey matrices of the elastic medium: the traction
  // of an element point is -C_e v with C_e = w |n| [(rho vp - rho vs) n n^T /
  // |n|^2 + rho vs I] in P-SV (stacey.tpp:50-80) and w |n| rho vs in SH
  // (stacey.tpp:126-146, stored in the xx slot); acoustic: w |n| / (rho vp)
  // times the free-surface mask of the element point (stacey.tpp:296-326,
  // dirichlet.hpp:38-62), in the xx slot; the adjoint applies C^T = C
  for (MediumData *Dp : {&a.el, &a.ac}) {
    MediumData &D = *Dp;
    D.stacey_pt.clear();
    D.stacey_c.clear();
    if (D.nspec && !D.aniso && !D.cosserat && !D.poro) {
      std::unordered_map<int, size_t> slot;
      for (int ce = 0; ce < D.nspec; ++ce) {
        if (D.bc_slot[ce] < 0) continue;
        for (int q = 0; q < NPTS; ++q) {
          const size_t k = size_t(D.bc_slot[ce]) * NPTS + q;
          if (D.bc_w[k] == 0.0f) continue;
          const int g = D.ibool[size_t(ce) * NPTS + q];
          auto it = slot.find(g);
          size_t j;
          if (it == slot.end()) {
            j = D.stacey_pt.size();
            slot[g] = j;
            D.stacey_pt.push_back(g);
            D.stacey_c.resize(3 * (j + 1), 0.0f);
          } else {
            j = it->second;
          }
          const double nx = D.bc_nx[k], nz = D.bc_nz[k], j1 = D.bc_j1[k], wq = D.bc_w[k];
          const double rvp = D.bc_imp0[k], rvs = D.bc_imp1[k];
          const double f = wq * j1, d = (rvp - rvs) / (j1 * j1);
          if (Dp == &a.ac) {
            D.stacey_c[3 * j + 0] += float(f * rvp * double(D.bc_keep[k]));
            continue;
          }
          if (D.ncomp == 1) {
            D.stacey_c[3 * j + 0] += float(f * rvs);
            continue;
          }
          D.stacey_c[3 * j + 0] += float(f * (d * nx * nx + rvs));
          D.stacey_c[3 * j + 1] += float(f * (d * nx * nz));
          D.stacey_c[3 * j + 2] += float(f * (d * nz * nz + rvs));
        }
      }
    }
  }
  // --- mass matrix (+ Stacey implicit term), inverted -------------
  // M = sum rho w_x w_z |J| (acoustic: 1/kappa), plus (dt/2) C on Stacey points
  // (compute_mass_matrix.tpp:95-121, stacey.tpp:817-853), then 1/M.
  for (int med = 0; med < 2; ++med) {
    MediumData &D = med == 1 ? a.el : a.ac;
    std::vector<double> M(size_t(D.nglob) * D.ncomp, 0.0);
    for (int ce = 0; ce < D.nspec; ++ce) {
      const int e = D.elem_mesh[ce];
      for (int iz = 0; iz < NGLL; ++iz)
        for (int ix = 0; ix < NGLL; ++ix) {
          const int q = iz * NGLL + ix;
          const size_t pc = size_t(ce) * NPTS + q, pm = size_t(e) * NPTS + q;
          const double fac = w[ix] * w[iz] * a.jac_d[pm];
          double rho, vp, vs;
          model(e, pm, rho, vp, vs);
          double mc[4] = {0, 0, 0, 0};
          if (med == 1) mc[0] = mc[1] = rho * fac;
          else mc[0] = (1.0 / double(D.prop1[pc])) * fac;
          if (med == 1 && D.poro) {
            // solid rho_bar - phi rho_f / tort, fluid (rho_f tort rho_bar -
            // phi rho_f^2) / (phi rho_bar) (poroelastic/isotropic/mass_matrix.tpp)
            const double *v = poro_of(e);
            const double phi = v[2], rhof = v[1], tort = v[3], rb = (1.0 - phi) * v[0] + phi * rhof;
            mc[0] = mc[1] = (rb - phi * rhof / tort) * fac;
            mc[2] = mc[3] = ((rhof * tort * rb - phi * rhof * rhof) / (phi * rb)) * fac;
          }
          // Cosserat: rho, rho, j (isotropic_cosserat/mass_matrix.tpp)
          if (med == 1 && D.cosserat) mc[2] = m.mat_cosserat[size_t(m.kmato[e]) * 8 + 4] * fac;
          if (D.bc_slot[ce] >= 0) {
            const size_t k = size_t(D.bc_slot[ce]) * NPTS + q;
            if (D.bc_w[k] != 0.0f) {
              const double vv = -dt * 0.5;  // velocity stand-in of the implicit term
              const double nx = D.bc_nx[k], nz = D.bc_nz[k], j1 = D.bc_j1[k], wq = D.bc_w[k];
              if (med == 0) {
                mc[0] += -1.0 * wq * j1 * double(D.bc_imp0[k]) * vv;
              } else if (D.ncomp == 1) {
                mc[0] += -1.0 * wq * j1 * double(D.bc_imp1[k]) * vv;
              } else {
                const double vn = vv * nx + vv * nz;
                const double dn[2] = {nx, nz};
                for (int c = 0; c < 2; ++c) {
                  const double f = ((vn * dn[c] / (j1 * j1)) * (double(D.bc_imp0[k]) - double(D.bc_imp1[k]))) +
                                   vv * double(D.bc_imp1[k]);
                  mc[c] += -1.0 * f * j1 * wq;
                }
                if (D.cosserat) mc[2] += -1.0 * double(D.bc_imp2[k]) * vv * j1 * wq;
              }
            }
          }
          const int g = D.ibool[pc];
          for (int c = 0; c < D.ncomp; ++c) M[size_t(g) * D.ncomp + c] += mc[c];
        }
    }
    D.minv.resize(M.size());
    for (size_t i = 0; i < M.size(); ++i) D.minv[i] = float(1.0 / M[i]);
  }
}

void set_model2d(Mesh2D &m, Assembly2D &a, const float *rho, const float *kappa, const float *mu) {
  const size_t n = size_t(m.nspec) * NPTS;
  m.prho.resize(n);
  m.pvp.resize(n);
  m.pvs.resize(n);
  for (size_t p = 0; p < n; ++p) {
    if (!(rho[p] > 0) || !(mu[p] >= 0) || !(kappa[p] + 4.0 / 3.0 * mu[p] > 0))
      throw std::runtime_error("model values must give rho > 0, mu >= 0, lambda + 2 mu > 0");
    m.prho[p] = rho[p];
    m.pvs[p] = float(std::sqrt(double(mu[p]) / rho[p]));
    m.pvp[p] = float(std::sqrt((double(kappa[p]) + 4.0 / 3.0 * double(mu[p])) / rho[p]));
  }
  assemble_model2d(m, a);
}

// ------------------------------------------------------------ assembly ---
void assemble2d(const Mesh2D &m, double dt, Assembly2D &a) {
  const int nspec = m.nspec;
  if (nspec <= 0 || (m.ngnod != 4 && m.ngnod != 9)) throw std::runtime_error("invalid mesh");
  a.nspec = nspec;
  a.dt = dt;
  a.elastic_wave = m.elastic_wave;
  double z[NGLL], w[NGLL], hp[NGLL][NGLL];
  gll(z, w, hp);
  for (int i = 0; i < NGLL; ++i) { a.zgll[i] = z[i]; a.wgll[i] = float(w[i]); a.wgll_d[i] = w[i]; }
  for (int i = 0; i < NGLL; ++i)
    for (int j = 0; j < NGLL; ++j) {
      a.hprime[i * NGLL + j] = float(hp[i][j]);
      a.hpw[i * NGLL + j] = float(hp[i][j] * w[i]);
    }

  // --- global numbering from element topology -----------------------
  // key: corners (node), edge points (min node, max node, position), interior
  const size_t nloc = size_t(nspec) * NPTS;
  std::vector<uint64_t> key(nloc);
  const int cz[4] = {0, 0, NGLL - 1, NGLL - 1}, cx[4] = {0, NGLL - 1, NGLL - 1, 0};
  const uint64_t npg = uint64_t(m.npgeo);
  for (int e = 0; e < nspec; ++e) {
    const int *kn = &m.knods[size_t(e) * m.ngnod];
    for (int iz = 0; iz < NGLL; ++iz)
      for (int ix = 0; ix < NGLL; ++ix) {
        const size_t p = size_t(e) * NPTS + iz * NGLL + ix;
        uint64_t k = ~0ull;
        for (int c = 0; c < 4; ++c)
          if (iz == cz[c] && ix == cx[c]) k = uint64_t(kn[c]);
        if (k == ~0ull) {
          int A = -1, B = -1, t = 0;
          if (iz == 0) { A = 0; B = 1; t = ix; }
          else if (iz == NGLL - 1) { A = 3; B = 2; t = ix; }
          else if (ix == 0) { A = 0; B = 3; t = iz; }
          else if (ix == NGLL - 1) { A = 1; B = 2; t = iz; }
          if (A >= 0) {
            uint64_t na = kn[A], nb = kn[B];
            uint64_t pos = na < nb ? uint64_t(t) : uint64_t(NGLL - 1 - t);
            k = npg + (std::min(na, nb) * npg + std::max(na, nb)) * NGLL + pos;
          } else {
            k = npg + npg * npg * NGLL + p;  // interior: unique
          }
        }
        key[p] = k;
      }
  }
  std::vector<uint32_t> order(nloc);
  std::iota(order.begin(), order.end(), 0u);
  std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return key[x] < key[y]; });
  std::vector<int> gid(nloc);
  int ng = -1;
  for (size_t i = 0; i < nloc; ++i) {
    if (i == 0 || key[order[i]] != key[order[i - 1]]) ++ng;
    gid[order[i]] = ng;
  }
  a.nglob = ng + 1;
  // renumber by first touch in element order (locality)
  {
    std::vector<int> remap(a.nglob, -1);
    int next = 0;
    for (size_t p = 0; p < nloc; ++p)
      if (remap[gid[p]] < 0) remap[gid[p]] = next++;
    for (size_t p = 0; p < nloc; ++p) gid[p] = remap[gid[p]];
  }
  a.ibool_global = gid;

  // --- geometry in mesh order --------------------------------------
  std::vector<JacD> J(nloc);
  a.gx.resize(nloc);
  a.gz.resize(nloc);
  for (int e = 0; e < nspec; ++e)
    for (int iz = 0; iz < NGLL; ++iz)
      for (int ix = 0; ix < NGLL; ++ix) {
        const size_t p = size_t(e) * NPTS + iz * NGLL + ix;
        J[p] = jacobian(m, e, z[ix], z[iz]);
        if (!(J[p].jac > 0)) throw std::runtime_error("non-positive Jacobian: check element orientation");
        a.gx[p] = J[p].x;
        a.gz[p] = J[p].z;
      }

  // --- media and colouring ------------------------------------------
  a.mesh_medium.resize(nspec);
  for (int e = 0; e < nspec; ++e) a.mesh_medium[e] = m.mat_medium[m.kmato[e]];
  a.mesh_to_compute.assign(nspec, -1);
  // greedy colouring: no two elements of a colour share a global point
  std::vector<int> color(nspec, 0);
  {
    std::vector<uint32_t> used(a.nglob, 0u);
    for (int e = 0; e < nspec; ++e) {
      uint32_t mask = 0;
      for (int q = 0; q < NPTS; ++q) mask |= used[gid[size_t(e) * NPTS + q]];
      int c = 0;
      while (c < 32 && (mask >> c & 1u)) ++c;
      if (c == 32) throw std::runtime_error("mesh needs more than 32 colours");
      color[e] = c;
      for (int q = 0; q < NPTS; ++q) used[gid[size_t(e) * NPTS + q]] |= 1u << c;
    }
  }

  // --- Stacey and free-surface point data (mesh order) ----------------
  // Absorbing entries are applied in database order; on a corner shared by
  // two absorbing edges of one element the later entry's normal and weight
  // win (core/specfem/assembly/boundaries/dim2/impl/stacey.tpp).
  struct BcPt { double w = 0, nx = 0, nz = 0; bool st = false, fs = false; };
  std::unordered_map<int, std::vector<BcPt>> bc;  // mesh element -> 25 points
  for (size_t i = 0; i < m.abs_ispec.size(); ++i) {
    const int e = m.abs_ispec[i], t = m.abs_type[i];
    auto &v = bc[e];
    v.resize(NPTS);
    for (int iz = 0; iz < NGLL; ++iz)
      for (int ix = 0; ix < NGLL; ++ix) {
        if (!on_edge(t, iz, ix)) continue;
        BcPt &b = v[iz * NGLL + ix];
        b.st = true;
        edge_normal(J[size_t(e) * NPTS + iz * NGLL + ix], t, b.nx, b.nz);
        b.w = (t == LEFT || t == RIGHT) ? w[iz] : w[ix];
      }
  }
  for (size_t i = 0; i < m.free_ispec.size(); ++i) {
    const int e = m.free_ispec[i], t = m.free_type[i];
    if (a.mesh_medium[e] != 0) continue;      // free surface acts on acoustic media
    auto &v = bc[e];
    v.resize(NPTS);
    for (int iz = 0; iz < NGLL; ++iz)
      for (int ix = 0; ix < NGLL; ++ix)
        if (on_edge(t, iz, ix)) v[iz * NGLL + ix].fs = true;
  }

  // --- acoustic/elastic coupling -------------------------------------
  // Each element pair sharing an edge across media contributes, on the self
  // side, GLL weight * outward normal of the self element at the edge points
  // (core/specfem/assembly/conforming_interfaces/dim2/impl/interface_container.tpp);
  // the contribution of an acoustic point on the free surface is dropped
  // (compute_coupling.tpp:101-106).  The term is linear in the other medium's
  // field at the same global point, so the edge contributions of a point are
  // summed once here and applied per point in the update kernels.
  std::vector<double> cpl[2];                 // [medium][glob][2]
  std::vector<uint8_t> is_iface[2];
  cpl[0].assign(2 * size_t(a.nglob), 0.0); cpl[1].assign(2 * size_t(a.nglob), 0.0);
  is_iface[0].assign(a.nglob, 0); is_iface[1].assign(a.nglob, 0);
  {
    std::unordered_map<uint64_t, std::vector<std::pair<int, int>>> edges;
    const int ends[4][2] = {{0, 1}, {1, 2}, {3, 2}, {0, 3}};
    for (int e = 0; e < nspec; ++e) {
      const int *kn = &m.knods[size_t(e) * m.ngnod];
      for (int t = 0; t < 4; ++t) {
        uint64_t na = kn[ends[t][0]], nb = kn[ends[t][1]];
        edges[std::min(na, nb) * npg + std::max(na, nb)].push_back({e, t});
      }
    }
    std::vector<std::pair<uint64_t, std::vector<std::pair<int, int>>>> sorted(edges.begin(), edges.end());
    std::sort(sorted.begin(), sorted.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
    for (auto &kv : sorted) {
      if (kv.second.size() != 2) continue;
      const auto [e1, t1] = kv.second[0];
      const auto [e2, t2] = kv.second[1];
      if (a.mesh_medium[e1] == a.mesh_medium[e2]) continue;
      for (auto [e, t] : {std::make_pair(e1, t1), std::make_pair(e2, t2)}) {
        const int med = a.mesh_medium[e];
        const auto it = bc.find(e);
        for (int iz = 0; iz < NGLL; ++iz)
          for (int ix = 0; ix < NGLL; ++ix) {
            if (!on_edge(t, iz, ix)) continue;
            const int q = iz * NGLL + ix;
            const int g = gid[size_t(e) * NPTS + q];
            is_iface[med][g] = 1;
            if (it != bc.end() && it->second[q].fs) continue;
            double nx, nz;
            edge_normal(J[size_t(e) * NPTS + q], t, nx, nz);
            const double f = (t == BOTTOM || t == TOP) ? w[ix] : w[iz];
            cpl[med][2 * size_t(g)] += f * nx;
            cpl[med][2 * size_t(g) + 1] += f * nz;
          }
      }
    }
  }

  // --- nonconforming acoustic-elastic coupling ----------------------
  // A nonconforming record between different media and its reverse record
  // give a self and a coupled edge (core/specfem/assembly/edge_types/dim2/edge_types.cpp);
  // the self points receive weighted sums of the coupled edge's points
  // (nonconforming_weights).  Contributions of acoustic points on the free
  // surface are dropped as for conforming edges.
  std::vector<std::unordered_map<int, std::map<int, std::array<double, 2>>>> ncw(2);
  if (!m.adjacency.empty()) {
    std::map<std::pair<int, int>, int> orient;
    const size_t nadj = m.adjacency.size() / 4;
    for (size_t r = 0; r < nadj; ++r) {
      const int *rec = &m.adjacency[4 * r];
      if (rec[2] == 3) orient[{rec[0], rec[1]}] = rec[3];
      else if (rec[2] != 1) throw std::runtime_error("Unknown connection type in adjacency graph.");
    }
    for (const auto &kv : orient) {
      const int e1 = kv.first.first, e2 = kv.first.second, t1 = kv.second;
      if (e1 < 0 || e1 >= nspec || e2 < 0 || e2 >= nspec) throw std::runtime_error("bad adjacency record");
      if (a.mesh_medium[e1] == a.mesh_medium[e2]) continue;
      const auto back = orient.find({e2, e1});
      if (back == orient.end())
        throw std::runtime_error("Non-symmetric adjacency graph detected in `compute_intersection`.");
      const int t2 = back->second;
      if (t1 > LEFT || t2 > LEFT) throw std::runtime_error("compute_intersection must be given edges");
      if (m.elastic_wave == 1 || !m.mat_cosserat.empty())
        throw std::runtime_error("nonconforming coupling: P-SV isotropic or anisotropic elastic media only");
      double W[NGLL][NGLL][2];
      nonconforming_weights(m, z, w, hp, e1, t1, e2, t2, W);
      const int med = a.mesh_medium[e1];
      const auto it = bc.find(e1);
      for (int i = 0; i < NGLL; ++i) {
        const int q1 = edge_point(t1, i);
        const int g = gid[size_t(e1) * NPTS + q1];
        auto &row = ncw[med][g];      // marks the point as coupled
        if (it != bc.end() && it->second[q1].fs) continue;
        for (int j = 0; j < NGLL; ++j) {
          auto &acc = row[gid[size_t(e2) * NPTS + edge_point(t2, j)]];
          acc[0] += W[i][j][0];
          acc[1] += W[i][j][1];
        }
      }
    }
  }
  const bool nonconforming = !ncw[0].empty() || !ncw[1].empty();

  // --- compute order, per-medium numbering, element arrays -----------
  for (int med = 0; med < 2; ++med) {
    MediumData &D = med == 1 ? a.el : a.ac;
    D.ncomp = med == 1 ? (m.elastic_wave == 1 ? 1 : 2) : 1;
    if (med == 1 && !m.mat_cosserat.empty()) {
      // a Cosserat elastic medium: every elastic element Cosserat, P-SV-T
      bool any = false, all = true;
      for (int e = 0; e < nspec; ++e)
        if (a.mesh_medium[e] == 1) {
          const bool c = std::isfinite(m.mat_cosserat[size_t(m.kmato[e]) * 8]);
          any |= c; all &= c;
        }
      if (any && (!all || m.elastic_wave == 1))
        throw std::runtime_error("Cosserat media: every elastic element Cosserat, P-SV only");
      if (any) D.ncomp = 3;
    }
    if (med == 1 && !m.mat_poro.empty()) {
      // a poroelastic medium: every elastic element poroelastic, four components
      bool any = false, all = true;
      for (int e = 0; e < nspec; ++e)
        if (a.mesh_medium[e] == 1) {
          const bool c = std::isfinite(m.mat_poro[size_t(m.kmato[e]) * 13]);
          any |= c; all &= c;
        }
      if (any && (!all || m.elastic_wave == 1 || D.ncomp == 3))
        throw std::runtime_error("poroelastic media: every elastic element poroelastic, P-SV only");
      if (any) D.ncomp = 4;
    }
    int ncol = 0;
    for (int e = 0; e < nspec; ++e)
      if (a.mesh_medium[e] == med) ncol = std::max(ncol, color[e] + 1);
    D.color_start.assign(1, 0);
    for (int c = 0; c < ncol; ++c) {
      for (int e = 0; e < nspec; ++e)
        if (a.mesh_medium[e] == med && color[e] == c) {
          a.mesh_to_compute[e] = int(D.elem_mesh.size());
          D.elem_mesh.push_back(e);
        }
      D.color_start.push_back(int(D.elem_mesh.size()));
    }
    D.nspec = int(D.elem_mesh.size());
    D.elem_color.assign(D.nspec, 0);
    for (int c = 0; c < ncol; ++c)
      for (int ce = D.color_start[c]; ce < D.color_start[c + 1]; ++ce) D.elem_color[ce] = c;
    // tiles of the fused tile kernel
    D.tile_elem = make_tiles(a, D.elem_mesh);
    D.ntiles = int(D.tile_elem.size()) / TILE_E;
    // per-medium point numbering (every assembly variant sums a point's
    // contributions in colour order, so the numbering changes no result; it
    // sets the locality of the gathers and the tiles' contiguous ranges):
    // coupled-interface points first (by first touch in compute order), then
    // the interior points of each tile in tile order (first touch inside the
    // tile), then the points several tiles share (first touch in tile order)
    std::vector<int> &g2m = med == 1 ? a.glob_to_el : a.glob_to_ac;
    g2m.assign(a.nglob, -1);
    D.ibool.resize(size_t(D.nspec) * NPTS);
    for (int ce = 0; ce < D.nspec; ++ce) {
      const int e = D.elem_mesh[ce];
      for (int q = 0; q < NPTS; ++q) {
        const int g = gid[size_t(e) * NPTS + q];
        const bool iface = is_iface[med][g] || (nonconforming && ncw[med].count(g));
        if (g2m[g] >= 0 || !iface) continue;
        g2m[g] = D.nglob++;
        D.glob_of_point.push_back(g);
      }
    }
    D.niface = D.nglob;
    {
      std::vector<int> tcount(a.nglob, 0), tlast(a.nglob, -1);
      for (int t = 0; t < D.ntiles; ++t)
        for (int s = 0; s < TILE_E; ++s) {
          const int ce = D.tile_elem[size_t(t) * TILE_E + s];
          if (ce < 0) continue;
          for (int q = 0; q < NPTS; ++q) {
            const int g = gid[size_t(D.elem_mesh[ce]) * NPTS + q];
            if (tlast[g] != t) { tlast[g] = t; ++tcount[g]; }
          }
        }
      D.tile_ibeg.assign(D.ntiles, 0);
      D.tile_nint.assign(D.ntiles, 0);
      for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) D.sh0 = D.nglob;
        for (int t = 0; t < D.ntiles; ++t) {
          if (pass == 0) D.tile_ibeg[t] = D.nglob;
          for (int s = 0; s < TILE_E; ++s) {
            const int ce = D.tile_elem[size_t(t) * TILE_E + s];
            if (ce < 0) continue;
            for (int q = 0; q < NPTS; ++q) {
              const int g = gid[size_t(D.elem_mesh[ce]) * NPTS + q];
              if (g2m[g] >= 0 || (pass == 0 && tcount[g] != 1)) continue;
              g2m[g] = D.nglob++;
              D.glob_of_point.push_back(g);
            }
          }
          if (pass == 0) D.tile_nint[t] = D.nglob - D.tile_ibeg[t];
        }
      }
    }
    if (D.nspec == 0) D.niface = D.sh0 = 0;
    for (int ce = 0; ce < D.nspec; ++ce) {
      const int e = D.elem_mesh[ce];
      for (int q = 0; q < NPTS; ++q) D.ibool[size_t(ce) * NPTS + q] = g2m[gid[size_t(e) * NPTS + q]];
    }
    // tile-local indices: interior point k = point - tile_ibeg; the tile's
    // shared points follow, in first-touch order
    D.tile_lidx.assign(size_t(D.ntiles) * TILE_E * NPTS, 0);
    D.tile_nsh.assign(D.ntiles, 0);
    D.tile_sh_off.assign(D.ntiles, 0);
    D.tile_sh.clear();
    for (int t = 0; t < D.ntiles; ++t) {
      const int ib = D.tile_ibeg[t], ni = D.tile_nint[t];
      std::vector<int> shl;
      std::unordered_map<int, int> pos;
      for (int s = 0; s < TILE_E; ++s) {
        const int ce = D.tile_elem[size_t(t) * TILE_E + s];
        if (ce < 0) continue;
        for (int q = 0; q < NPTS; ++q) {
          const int pt = D.ibool[size_t(ce) * NPTS + q];
          int k;
          if (pt >= ib && pt < ib + ni) {
            k = pt - ib;
          } else {
            auto it = pos.find(pt);
            if (it == pos.end()) { it = pos.emplace(pt, int(shl.size())).first; shl.push_back(pt); }
            k = ni + it->second;
          }
          if (k > 65535) throw std::runtime_error("tile with more than 65536 local points");
          D.tile_lidx[(size_t(t) * TILE_E + s) * NPTS + q] = uint16_t(k);
        }
      }
      D.tile_sh_off[t] = int(D.tile_sh.size());
      D.tile_nsh[t] = int(shl.size());
      D.tile_sh.insert(D.tile_sh.end(), shl.begin(), shl.end());
      while (D.tile_sh.size() % 4) D.tile_sh.push_back(0);
    }
    D.inv_start.assign(D.nglob + 1, 0);
    for (int v : D.ibool) ++D.inv_start[v + 1];
    for (int i = 0; i < D.nglob; ++i) D.inv_start[i + 1] += D.inv_start[i];
    D.inv_idx.resize(D.ibool.size());
    {
      std::vector<int> fill(D.inv_start.begin(), D.inv_start.end() - 1);
      for (size_t pl = 0; pl < D.ibool.size(); ++pl) D.inv_idx[fill[D.ibool[pl]]++] = int(pl);
    }
    const size_t n = size_t(D.nspec) * NPTS;
    D.xix.resize(n); D.xiz.resize(n); D.gax.resize(n); D.gaz.resize(n); D.jac.resize(n);
    for (int ce = 0; ce < D.nspec; ++ce) {
      const int e = D.elem_mesh[ce];
      for (int q = 0; q < NPTS; ++q) {
        const size_t pm = size_t(e) * NPTS + q, pc = size_t(ce) * NPTS + q;
        D.xix[pc] = float(J[pm].xix); D.xiz[pc] = float(J[pm].xiz);
        D.gax[pc] = float(J[pm].gax); D.gaz[pc] = float(J[pm].gaz);
        D.jac[pc] = float(J[pm].jac);
      }
    }
  }
  // per-point coupling coefficients of the interface points of each medium
  for (int med = 0; med < 2; ++med) {
    MediumData &D = med == 1 ? a.el : a.ac;
    const std::vector<int> &other = med == 1 ? a.glob_to_ac : a.glob_to_el;
    if (nonconforming) {
      // several entries per point: the conforming one (same global point)
      // and the nonconforming ones, merged per point of the other medium
      D.cp_start.assign(D.niface + 1, 0);
      D.cp_nx.clear(); D.cp_nz.clear(); D.cp_other.clear();
      for (int i = 0; i < D.niface; ++i) {
        const int g = D.glob_of_point[i];
        std::map<int, std::array<double, 2>> ent;
        if (is_iface[med][g]) {
          if (other[g] < 0) throw std::runtime_error("coupled point missing in the other medium");
          auto &e = ent[other[g]];
          e[0] += cpl[med][2 * size_t(g)];
          e[1] += cpl[med][2 * size_t(g) + 1];
        }
        const auto it = ncw[med].find(g);
        if (it != ncw[med].end())
          for (const auto &kv : it->second) {
            const int o = other[kv.first];
            if (o < 0) throw std::runtime_error("coupled point missing in the other medium");
            auto &e = ent[o];
            e[0] += kv.second[0];
            e[1] += kv.second[1];
          }
        for (const auto &kv : ent) {
          D.cp_other.push_back(kv.first);
          D.cp_nx.push_back(float(kv.second[0]));
          D.cp_nz.push_back(float(kv.second[1]));
        }
        D.cp_start[i + 1] = int(D.cp_other.size());
      }
      continue;
    }
    D.cp_nx.assign(D.niface, 0.f); D.cp_nz.assign(D.niface, 0.f); D.cp_other.assign(D.niface, -1);
    for (int i = 0; i < D.niface; ++i) {
      const int g = D.glob_of_point[i];
      D.cp_nx[i] = float(cpl[med][2 * size_t(g)]);
      D.cp_nz[i] = float(cpl[med][2 * size_t(g) + 1]);
      D.cp_other[i] = other[g];
      if (D.cp_other[i] < 0) throw std::runtime_error("coupled point missing in the other medium");
    }
  }

  // --- Stacey / free-surface arrays in compute order -----------------
  for (int med = 0; med < 2; ++med) {
    MediumData &D = med == 1 ? a.el : a.ac;
    D.bc_slot.assign(D.nspec, -1);
    int ns = 0;
    for (int ce = 0; ce < D.nspec; ++ce)
      if (bc.count(D.elem_mesh[ce])) D.bc_slot[ce] = ns++;
    const size_t n = size_t(ns) * NPTS;
    D.bc_w.assign(n, 0); D.bc_nx.assign(n, 0); D.bc_nz.assign(n, 0); D.bc_j1.assign(n, 0);
    D.bc_imp0.assign(n, 0); D.bc_imp1.assign(n, 0); D.bc_keep.assign(n, 1.0f); D.bc_imp2.assign(n, 0);
    for (int ce = 0; ce < D.nspec; ++ce) {
      if (D.bc_slot[ce] < 0) continue;
      const auto &v = bc[D.elem_mesh[ce]];
      for (int q = 0; q < NPTS; ++q) {
        const size_t k = size_t(D.bc_slot[ce]) * NPTS + q;
        if (v[q].st) {
          D.bc_w[k] = float(v[q].w);
          D.bc_nx[k] = float(v[q].nx);
          D.bc_nz[k] = float(v[q].nz);
          D.bc_j1[k] = float(std::sqrt(v[q].nx * v[q].nx + v[q].nz * v[q].nz));
        }
        if (v[q].fs) D.bc_keep[k] = 0.0f;
      }
    }
  }

  a.jac_d.resize(nloc);
  for (size_t p = 0; p < nloc; ++p) a.jac_d[p] = J[p].jac;
  assemble_model2d(m, a);
}

// ------------------------------------------------------ point location ---
// Closest GLL point, then Newton iterations from the element centre in that
// element and its corner-sharing neighbours; the candidate whose mapped point
// is closest wins (src/algorithms/dim2/locate_point_impl.cpp).
namespace {

void build_locate_index(const Mesh2D &m, Assembly2D &a) {
  Assembly2D::LocateIndex &L = a.loc;
  double xmin = 1e300, xmax = -1e300, zmin = 1e300, zmax = -1e300;
  for (int i = 0; i < m.npgeo; ++i) {
    xmin = std::min(xmin, m.coorg[2 * i]); xmax = std::max(xmax, m.coorg[2 * i]);
    zmin = std::min(zmin, m.coorg[2 * i + 1]); zmax = std::max(zmax, m.coorg[2 * i + 1]);
  }
  L.tol = 1e-9 * std::max(xmax - xmin, zmax - zmin);
  // cell size: the largest element bounding-box extent, so the GLL point
  // nearest to any point inside the mesh lies in the 3x3 cells around it
  double h = 0;
  for (int e = 0; e < m.nspec; ++e) {
    double ex0 = 1e300, ex1 = -1e300, ez0 = 1e300, ez1 = -1e300;
    for (int k = 0; k < m.ngnod; ++k) {
      const int id = m.knods[size_t(e) * m.ngnod + k];
      ex0 = std::min(ex0, m.coorg[2 * id]); ex1 = std::max(ex1, m.coorg[2 * id]);
      ez0 = std::min(ez0, m.coorg[2 * id + 1]); ez1 = std::max(ez1, m.coorg[2 * id + 1]);
    }
    h = std::max(h, std::max(ex1 - ex0, ez1 - ez0));
  }
  L.h = h > 0 ? h : 1.0;
  L.x0 = xmin;
  L.z0 = zmin;
  L.nx = int((xmax - xmin) / L.h) + 1;
  L.nz = int((zmax - zmin) / L.h) + 1;
  const size_t ncell = size_t(L.nx) * L.nz;
  auto cell_of = [&](double x, double z) {
    int cx = std::min(std::max(int((x - L.x0) / L.h), 0), L.nx - 1);
    int cz = std::min(std::max(int((z - L.z0) / L.h), 0), L.nz - 1);
    return size_t(cz) * L.nx + cx;
  };
  L.cell_start.assign(ncell + 1, 0);
  for (size_t p = 0; p < a.gx.size(); ++p) ++L.cell_start[cell_of(a.gx[p], a.gz[p]) + 1];
  for (size_t c = 0; c < ncell; ++c) L.cell_start[c + 1] += L.cell_start[c];
  L.cell_pts.resize(a.gx.size());
  std::vector<int> fill(L.cell_start.begin(), L.cell_start.end() - 1);
  for (size_t p = 0; p < a.gx.size(); ++p) L.cell_pts[fill[cell_of(a.gx[p], a.gz[p])]++] = int(p);
  L.node_start.assign(m.npgeo + 1, 0);
  for (int e = 0; e < m.nspec; ++e)
    for (int k = 0; k < 4; ++k) ++L.node_start[m.knods[size_t(e) * m.ngnod + k] + 1];
  for (int i = 0; i < m.npgeo; ++i) L.node_start[i + 1] += L.node_start[i];
  L.node_elems.resize(L.node_start[m.npgeo]);
  std::vector<int> nf(L.node_start.begin(), L.node_start.end() - 1);
  for (int e = 0; e < m.nspec; ++e)
    for (int k = 0; k < 4; ++k) L.node_elems[nf[m.knods[size_t(e) * m.ngnod + k]]++] = e;
  L.built = true;
}

}  // namespace

// Closest GLL point, then Newton iterations from the element centre in that
// element and its corner-sharing neighbours; the candidate whose mapped point
// is closest wins (src/algorithms/dim2/locate_point_impl.cpp).  A point on an
// edge or corner shared by several elements goes to the first element in mesh
// order: a candidate replaces the current choice only when it is closer by
// more than 1e-9 of the mesh extent.  Candidates are scanned in mesh order;
// the grid index only narrows the scan.
bool locate_point2d(const Mesh2D &m, Assembly2D &a, double x, double z, int &ispec, double &xi,
                    double &gamma) {
  if (!a.loc.built) build_locate_index(m, a);
  const Assembly2D::LocateIndex &L = a.loc;
  const double tol = L.tol;
  std::vector<int> pts;
  const int cx = int(std::floor((x - L.x0) / L.h)), cz = int(std::floor((z - L.z0) / L.h));
  for (int jz = cz - 1; jz <= cz + 1; ++jz)
    for (int jx = cx - 1; jx <= cx + 1; ++jx) {
      if (jx < 0 || jz < 0 || jx >= L.nx || jz >= L.nz) continue;
      const size_t c = size_t(jz) * L.nx + jx;
      pts.insert(pts.end(), L.cell_pts.begin() + L.cell_start[c], L.cell_pts.begin() + L.cell_start[c + 1]);
    }
  if (pts.empty()) {  // outside the gridded area: scan everything
    pts.resize(a.gx.size());
    std::iota(pts.begin(), pts.end(), 0);
  }
  std::sort(pts.begin(), pts.end());
  double best = 1e300;
  size_t pb = 0;
  for (int p : pts) {
    const double d = std::sqrt((a.gx[p] - x) * (a.gx[p] - x) + (a.gz[p] - z) * (a.gz[p] - z));
    if (d < best - tol) { best = d; pb = size_t(p); }
  }
  const int eg = int(pb / NPTS);
  std::vector<int> cand;
  for (int k = 0; k < 4; ++k) {
    const int node = m.knods[size_t(eg) * m.ngnod + k];
    for (int i = L.node_start[node]; i < L.node_start[node + 1]; ++i)
      if (L.node_elems[i] != eg) cand.push_back(L.node_elems[i]);
  }
  std::sort(cand.begin(), cand.end());
  cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
  cand.insert(cand.begin(), eg);
  double fd = 1e300;
  ispec = -1;
  for (int e : cand) {
    double s = 0, g = 0;
    for (int it = 0; it < 100; ++it) {
      JacD J = jacobian(m, e, s, g);
      const double dx = x - J.x, dz = z - J.z;
      const double ds = J.xix * dx + J.xiz * dz, dg = J.gax * dx + J.gaz * dz;
      s = std::min(std::max(s + ds, -1.01), 1.01);
      g = std::min(std::max(g + dg, -1.01), 1.01);
      if (std::abs(ds) < 1e-12 && std::abs(dg) < 1e-12) break;
    }
    JacD J = jacobian(m, e, s, g);
    const double d = std::sqrt((J.x - x) * (J.x - x) + (J.z - z) * (J.z - z));
    if (d < fd - tol) { fd = d; ispec = e; xi = s; gamma = g; }
  }
  if (ispec < 0 || std::abs(std::abs(xi) - 1.01) < 1e-6 || std::abs(std::abs(gamma) - 1.01) < 1e-6)
    return false;
  return true;
}

void set_sources2d(const Mesh2D &m, Assembly2D &a, const std::vector<Source2D> &src) {
  a.nsrc = int(src.size());
  a.src_medium.resize(a.nsrc); a.src_elem.resize(a.nsrc); a.src_shot.resize(a.nsrc);
  a.src_next.assign(a.nsrc, -1);
  a.src_arr.assign(size_t(a.nsrc) * 2 * NPTS, 0.0f);
  a.src_arr2.assign(a.el.poro ? size_t(a.nsrc) * 2 * NPTS : 0, 0.0f);
  a.el_src_head.assign(a.el.nspec, -1);
  a.ac_src_head.assign(a.ac.nspec, -1);
  // start time per shot: t0 = min over the shot's sources of their start
  // times, and each source's shift becomes t0_source - t0
  // (read_sources.cpp:142-172).  Start times, FP32 like the reference:
  // Ricker, Dirac (f0 = 1/(10 dt), dirac.cpp:25) and dGaussian -1.2/f0 +
  // tshift; Gaussian -2/f0 + tshift; Gaussian by hdur and Heaviside, with hdur
  // raised to 5 dt, -2 hdur + tshift, then evaluated with hdur / 1.628
  // (ricker.cpp, gaussian.cpp, dgaussian.cpp, gaussianhdur.cpp, heaviside.cpp;
  // the factor 2 is the 2D one of core/specfem/source/source.tpp:17-62).
  std::vector<double> f0(a.nsrc), t0s(a.nsrc);
  a.shot_t0.assign(a.nshots, 1e300);
  for (int s = 0; s < a.nsrc; ++s) {
    const Source2D &S = src[s];
    if (S.shot < 0 || S.shot >= a.nshots) throw std::runtime_error("source shot index out of range");
    if (S.stf < 0 || S.stf > 5) throw std::runtime_error("unknown source time function");
    if (S.stf == 3 || S.stf == 5) {
      if (!(S.hdur > 0)) throw std::runtime_error("source hdur must be positive");
      const float hd = std::max(float(S.hdur), 5.0f * float(a.dt));
      t0s[s] = double(-2.0f * hd + float(S.tshift));
      f0[s] = double(hd / 1.628f);                // evaluation half duration
    } else {
      f0[s] = S.stf == 1 ? double(1.0f / (10.0f * float(a.dt))) : S.f0;
      if (!(f0[s] > 0)) throw std::runtime_error("source f0 must be positive");
      const float fac = S.stf == 2 ? 2.0f : 1.2f;
      t0s[s] = double(-fac * (1.0f / float(f0[s])) + float(S.tshift));
    }
    a.shot_t0[S.shot] = std::min(a.shot_t0[S.shot], t0s[s]);
  }
  for (double &t : a.shot_t0)
    if (t > 1e299) t = 0.0;
  if (a.user_t0) {
    // a given start time: it must not come after the earliest start (less the
    // smallest shift), and every source keeps its own tshift
    // (read_sources.cpp:155-161)
    float min_t0 = 3.4e38f, min_tshift = 3.4e38f;
    for (int s = 0; s < a.nsrc; ++s) {
      min_t0 = std::min(min_t0, float(t0s[s]));
      min_tshift = std::min(min_tshift, float(src[s].tshift));
    }
    if (a.nsrc && float(a.user_t0_value) > min_t0 - min_tshift)
      throw std::runtime_error("User defined start time is less than minimum required for stability");
    a.shot_t0.assign(a.nshots, double(float(a.user_t0_value)));
  }
  a.t0 = *std::min_element(a.shot_t0.begin(), a.shot_t0.end());
  a.stf.assign(size_t(a.nstep) * a.nsrc, 0.0f);
  for (int s = 0; s < a.nsrc; ++s) {
    const Source2D &S = src[s];
    int e;
    double xi, ga;
    if (!locate_point2d(m, a, S.x, S.z, e, xi, ga)) throw std::runtime_error("Failed to locate source in the mesh");
    const int med = a.mesh_medium[e];
    const int ce = a.mesh_to_compute[e];
    a.src_medium[s] = med; a.src_elem[s] = ce; a.src_shot[s] = S.shot;
    std::vector<int> &head = med == 1 ? a.el_src_head : a.ac_src_head;
    a.src_next[s] = head[ce];
    head[ce] = s;
    double hx[NGLL], hg[NGLL], hpx[NGLL], hpg[NGLL];
    lagrange_d(xi, a.zgll, hx, hpx);
    lagrange_d(ga, a.zgll, hg, hpg);
    const MediumData &D = med == 1 ? a.el : a.ac;
    const double ang = S.angle * M_PI / 180.0;
    if (S.kind == 1) {
      // moment tensor: source array M . grad(l_x l_z) with the Jacobian
      // interpolated at the source (compute_source_array_from_tensor.cpp:17-86,
      // moment_tensor_source.cpp:22-35); elastic P-SV only
      if (med != 1 || D.ncomp != 2)
        throw std::runtime_error("moment-tensor sources need an elastic P-SV element");
      double jx[4] = {0, 0, 0, 0};  // xi_x, xi_z, gamma_x, gamma_z at the source
      for (int iz = 0; iz < NGLL; ++iz)
        for (int ix = 0; ix < NGLL; ++ix) {
          const size_t p = size_t(ce) * NPTS + iz * NGLL + ix;
          const double h = hx[ix] * hg[iz];
          jx[0] += h * D.xix[p]; jx[1] += h * D.xiz[p]; jx[2] += h * D.gax[p]; jx[3] += h * D.gaz[p];
        }
      for (int iz = 0; iz < NGLL; ++iz)
        for (int ix = 0; ix < NGLL; ++ix) {
          const int q = iz * NGLL + ix;
          const double dsx = (hpx[ix] * jx[0]) * hg[iz] + hx[ix] * (hpg[iz] * jx[2]);
          const double dsz = (hpx[ix] * jx[1]) * hg[iz] + hx[ix] * (hpg[iz] * jx[3]);
          a.src_arr[(size_t(s) * 2) * NPTS + q] = float(S.mxx * dsx + S.mxz * dsz);
          a.src_arr[(size_t(s) * 2 + 1) * NPTS + q] = float(S.mxz * dsx + S.mzz * dsz);
        }
    }
    for (int iz = 0; iz < NGLL && S.kind == 0; ++iz)
      for (int ix = 0; ix < NGLL; ++ix) {
        const int q = iz * NGLL + ix;
        const double h = hx[ix] * hg[iz];
        if (med == 0) {
          // pressure source: -stf * l / kappa (acoustic source.hpp:65); the
          // sign is applied to the STF column below
          a.src_arr[(size_t(s) * 2) * NPTS + q] = float(h / double(D.prop1[size_t(ce) * NPTS + q]));
        } else if (D.ncomp == 1) {
          a.src_arr[(size_t(s) * 2) * NPTS + q] = float(h);
        } else if (D.poro) {
          // force on both phases, (sin, cos) each, the solid rows times
          // (1 - phi / tort), the fluid rows times (1 - rho_f / rho_bar)
          // (vector_source/force_source.cpp:53-60, poroelastic/isotropic/source.hpp)
          const size_t pc = size_t(ce) * NPTS + q;
          const double fs = 1.0 - double(D.prop4[pc]), ff = 1.0 - double(D.prop5[pc]);
          a.src_arr[(size_t(s) * 2) * NPTS + q] = float(h * std::sin(ang) * fs);
          a.src_arr[(size_t(s) * 2 + 1) * NPTS + q] = float(h * std::cos(ang) * fs);
          a.src_arr2[(size_t(s) * 2) * NPTS + q] = float(h * std::sin(ang) * ff);
          a.src_arr2[(size_t(s) * 2 + 1) * NPTS + q] = float(h * std::cos(ang) * ff);
        } else {
          a.src_arr[(size_t(s) * 2) * NPTS + q] = float(h * std::sin(ang));
          a.src_arr[(size_t(s) * 2 + 1) * NPTS + q] = float(h * std::cos(ang));
        }
      }
    // STF on the shot's own time axis, FP32 like the reference tables
    const float tsh = a.user_t0 ? float(S.tshift) : float(t0s[s] - a.shot_t0[S.shot]);
    const float t0 = float(a.shot_t0[S.shot]);
    const float fz = float(f0[s]), fac = float(S.factor);
    const float pi = float(M_PI);
    const float aa = pi * pi * fz * fz;
    for (int i = 0; i < a.nstep; ++i) {
      const float t = t0 + float(i) * float(a.dt) - tsh;
      float v;
      switch (S.stf) {
        case 1:                  // Dirac and Gaussian: -exp(-a t^2) / (2a)
        case 2: v = fac * (-1.0f * std::exp(-aa * t * t) / (2.0f * aa)); break;
        case 3: {                // Gaussian by hdur: exp(-t^2/h^2) / (sqrt(pi) h)
          const float h = fz, ah = 1.0f / (h * h);
          v = fac * (std::exp(-ah * t * t) / (std::sqrt(pi) * h));
          break;
        }
        case 4: v = fac * (t * std::exp(-aa * t * t)); break;      // dGaussian
        case 5: v = fac * (0.5f * (1.0f + std::erf(t / fz))); break;  // Heaviside
        default: v = fac * ((1.0f - 2.0f * aa * t * t) * std::exp(-aa * t * t));  // Ricker
      }
      a.stf[size_t(i) * a.nsrc + s] = med == 0 ? -v : v;
    }
  }
}

void set_receivers2d(const Mesh2D &m, Assembly2D &a, const std::vector<double> &x,
                     const std::vector<double> &z, double angle, const std::vector<int> &types) {
  a.nrec = int(x.size());
  a.types = types;
  a.ntypes = int(types.size());
  a.rec_angle = angle;
  a.rec_medium.resize(a.nrec); a.rec_elem.resize(a.nrec);
  a.rec_h.assign(size_t(a.nrec) * NPTS, 0.0f);
  for (int r = 0; r < a.nrec; ++r) {
    int e;
    double xi, ga;
    if (!locate_point2d(m, a, x[r], z[r], e, xi, ga)) throw std::runtime_error("Failed to locate receiver in the mesh");
    a.rec_medium[r] = a.mesh_medium[e];
    a.rec_elem[r] = a.mesh_to_compute[e];
    double hx[NGLL], hg[NGLL];
    lagrange(xi, a.zgll, hx);
    lagrange(ga, a.zgll, hg);
    for (int iz = 0; iz < NGLL; ++iz)
      for (int ix = 0; ix < NGLL; ++ix) a.rec_h[size_t(r) * NPTS + iz * NGLL + ix] = float(hx[ix] * hg[iz]);
  }
}

}  // namespace sfg
