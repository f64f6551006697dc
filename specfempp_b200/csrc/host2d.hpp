// Host-side (Kokkos-free) 2D mesh and assembly data model of libsfg.
//
// Mirrors the reference's specfem::mesh::mesh<dim2> (include/mesh/dim2/mesh.hpp)
// and the parts of specfem::assembly::assembly<dim2> that the time step reads
// (core/specfem/assembly/*), laid out for the device: elements are reordered by
// medium and colour, element-local arrays are [element][25] in that order, and
// each medium has its own global point numbering (the reference's per-medium
// assembly_index_mapping, core/specfem/assembly/fields/impl/field_impl.tpp:18-62).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace sfg {

constexpr int NGLL = 5;
constexpr int NPTS = NGLL * NGLL;

struct Mesh2D {
  int nspec = 0, npgeo = 0, ngnod = 0;
  std::vector<double> coorg;          // [npgeo][2]
  std::vector<int> knods;             // [nspec][ngnod]
  std::vector<int> kmato;             // [nspec]
  int numat = 0;
  std::vector<int> mat_medium;        // [numat]
  std::vector<double> mat_rho, mat_vp, mat_vs;
  // optional anisotropic elastic constants [numat][6] (c11, c13, c15, c33,
  // c35, c55); rows of NaN for isotropic materials
  std::vector<double> mat_aniso;
  // optional isotropic Cosserat constants [numat][8] (rho, kappa, mu, nu, j,
  // lambda_c, mu_c, nu_c); rows of NaN for other materials
  std::vector<double> mat_cosserat;
  // optional isotropic poroelastic constants [numat][13] (rho_s, rho_f, phi,
  // tortuosity, kxx, kxz, kzz, kappa_s, kappa_f, kappa_fr, eta_f, mu_fr,
  // Q_mu); rows of NaN for other materials
  std::vector<double> mat_poro;
  std::vector<float> prho, pvp, pvs;  // optional [nspec][25]
  std::vector<int> abs_ispec, abs_type, free_ispec, free_type;
  int elastic_wave = 0;               // 0 P-SV, 1 SH
  // adjacency records [n][4] (element, neighbour, connection 1 strongly
  // conforming / 3 nonconforming, orientation 0..7), 0-based
  std::vector<int> adjacency;
};

// Reads a SPECFEM2D database.bin (Fortran unformatted records).
bool read_database2d(const std::string &path, Mesh2D &m, std::string &err);

struct Source2D {
  double x, z;
  int shot, stf;
  double f0, factor, tshift, angle;
  int kind = 0;                   // 0 force, 1 moment tensor
  double mxx = 0, mzz = 0, mxz = 0;
  double hdur = 0;                // half duration (Gaussian by hdur, Heaviside)
};

// Per-medium device-ready arrays (element order = compute order of that medium).
struct MediumData {
  int nspec = 0, nglob = 0, ncomp = 0;
  std::vector<int> color_start;       // [ncolors+1] element ranges
  std::vector<int> elem_mesh;         // compute element -> mesh element
  std::vector<int> ibool;             // [nspec][25] -> medium point id
  std::vector<float> xix, xiz, gax, gaz, jac;  // [nspec][25]
  std::vector<float> prop0, prop1;    // elastic: lambda+2mu, mu; acoustic: 1/rho, kappa
  // anisotropic elastic medium: prop0..prop5 = c11, c13, c15, c33, c35, c55
  bool aniso = false;
  std::vector<float> prop2, prop3, prop4, prop5;
  // isotropic Cosserat medium (ncomp 3: u_x, u_z, rotation): prop0 = lambda =
  // kappa - 2/3 mu, prop1 = mu, prop2 = nu, prop3 = mu_c + nu_c; bc_imp2 the
  // rotational Stacey impedance j sqrt((mu_c + nu_c) / j)
  bool cosserat = false;
  // isotropic poroelastic medium (ncomp 4: solid u_x, u_z, fluid w_x, w_z):
  // prop0 = H_Biot, prop1 = mu_G, prop2 = C_Biot, prop3 = M_Biot, prop4 =
  // phi / tortuosity, prop5 = rho_f / rho_bar, prop6..prop8 = eta_f times the
  // inverse permeability (xx, xz, zz)
  bool poro = false;
  std::vector<float> prop6, prop7, prop8;
  std::vector<float> minv;            // [nglob][ncomp]
  // Stacey / free-surface: slot per element (-1 none), compact [nslot][25]
  std::vector<int> bc_slot;
  std::vector<float> bc_w, bc_nx, bc_nz, bc_j1, bc_imp0, bc_imp1, bc_keep, bc_imp2;
  // coupling with the other medium: the first niface points of the medium's
  // numbering lie on coupled edges; per point the sum over the coupled edges
  // of GLL weight * outward normal, and the other medium's id of the point.
  // With nonconforming interfaces a point couples to several points of the
  // other medium: cp_start [niface + 1] then gives each point's range of
  // (cp_nx, cp_nz, cp_other) entries; empty = one entry per point.
  int niface = 0;
  std::vector<float> cp_nx, cp_nz;    // [niface] or [cp_start[niface]]
  std::vector<int> cp_other;          // [niface] or [cp_start[niface]]
  std::vector<int> cp_start;          // empty or [niface + 1]
  std::vector<int> glob_of_point;     // medium point id -> mesh global id
  // owner-computes assembly: for every medium point, the element-local
  // indices (compute element * 25 + GLL point) that contribute to it, in
  // increasing compute order (= colour order)
  std::vector<int> inv_start, inv_idx;
  // assembled Stacey matrices (elastic P-SV): point ids and (Cxx, Cxz, Czz)
  std::vector<int> stacey_pt;
  std::vector<float> stacey_c;
  // Tiles of the fused tile kernel: the medium's compute elements in groups of
  // TILE_E that lie close together (Morton order of the element centres).  A
  // point that only one tile touches and that is on no coupled edge is
  // interior to that tile; the point numbering gives every tile's interior
  // points one contiguous range [tile_ibeg, tile_ibeg + tile_nint).  The
  // points that several tiles touch are numbered after all interior ranges,
  // from sh0 on; with the interface points [0, niface) they are the boundary
  // points, finished outside the tiles.
  int ntiles = 0, sh0 = 0;
  std::vector<int> elem_color;        // [nspec] colour of each compute element
  std::vector<int> tile_elem;         // [ntiles][TILE_E] compute element, -1 past the tile's end
  std::vector<int> tile_ibeg, tile_nint, tile_nsh, tile_sh_off;
  std::vector<int> tile_sh;           // each tile's shared points (lists padded to 4 entries)
  std::vector<uint16_t> tile_lidx;    // [ntiles][TILE_E][25] tile-local point index
};

constexpr int TILE_E = 16;          // elements per tile of the fused tile kernel

struct Assembly2D {
  int nspec = 0, nglob = 0, nshots = 1, elastic_wave = 0;
  double dt = 0;
  int nstep = 0, nsb = 1;
  bool user_t0 = false;               // start time given by the caller
  double user_t0_value = 0;
  float hprime[NPTS];                 // hprime[i*5+j] = l'_j(xi_i)
  float hpw[NPTS];                    // hprime[l*5+i] * w[l]  (divergence form)
  float wgll[NGLL];
  double wgll_d[NGLL];
  double zgll[NGLL];
  std::vector<double> jac_d;          // [nspec][25] mesh order, |J| in FP64
  std::vector<int> ibool_global;      // [nspec][25] mesh order
  std::vector<double> gx, gz;         // [nspec][25] mesh order, GLL point coordinates
  MediumData el, ac;
  std::vector<int> mesh_medium;       // [nspec]
  std::vector<int> mesh_to_compute;   // [nspec] index inside its medium
  std::vector<int> glob_to_el, glob_to_ac;
  // sources (compute-order element of their medium)
  int nsrc = 0;
  std::vector<int> src_medium, src_elem, src_shot, src_next, el_src_head, ac_src_head;
  std::vector<float> src_arr;         // [nsrc][2][25]
  std::vector<float> src_arr2;        // poroelastic fluid rows [nsrc][2][25] (else empty)
  std::vector<float> stf;             // [nstep][nsrc]
  std::vector<double> shot_t0;        // per shot
  double t0 = 0;
  // receivers
  int nrec = 0, ntypes = 0, nsig = 0;
  std::vector<int> rec_medium, rec_elem, types;
  std::vector<float> rec_h;           // [nrec][25]
  double rec_angle = 0;
  // point-location index (built on first use): GLL points bucketed on a
  // uniform grid, and the elements around every control node
  struct LocateIndex {
    bool built = false;
    double x0 = 0, z0 = 0, h = 1, tol = 0;
    int nx = 0, nz = 0;
    std::vector<int> cell_start, cell_pts;    // CSR over cells -> local point
    std::vector<int> node_start, node_elems;  // CSR over control nodes -> elements
  } loc;
};

// Build everything but sources/receivers (numbering, geometry, colouring,
// boundaries, coupling, mass matrix).  Throws std::runtime_error on error.
void assemble2d(const Mesh2D &m, double dt, Assembly2D &a);
// Model-dependent arrays (material words, Stacey impedances and matrices, M^-1).
void assemble_model2d(const Mesh2D &m, Assembly2D &a);
// Replace the model by per-GLL-point rho, kappa, mu ([nspec][25], mesh order).
void set_model2d(Mesh2D &m, Assembly2D &a, const float *rho, const float *kappa, const float *mu);
void set_sources2d(const Mesh2D &m, Assembly2D &a, const std::vector<Source2D> &src);
void set_receivers2d(const Mesh2D &m, Assembly2D &a, const std::vector<double> &x,
                     const std::vector<double> &z, double angle, const std::vector<int> &types);
// locate a physical point: returns mesh element and (xi, gamma)
bool locate_point2d(const Mesh2D &m, Assembly2D &a, double x, double z, int &ispec,
                    double &xi, double &gamma);

}  // namespace sfg
