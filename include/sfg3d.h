/* libsfg — 3D elastic spectral-element time stepping on B200 (sm_100a), FP32.
 *
 * The 3D counterpart of the 2D interface in sfg.h: a structured lattice of
 * 8-node hexahedra (arbitrary control-node coordinates), isotropic elastic
 * media given per GLL point, force and moment-tensor sources, receivers, the
 * Newmark time loop captured in CUDA graphs.  Status codes and sfg_options
 * are those of sfg.h (elements_per_block fixes the element kernel's launch
 * shape: 1, 2 or 4 elements per block with one thread per element GLL point,
 * 6 or 8 with one thread per column of five points; 0 lets the autotuner
 * choose; all give the same bits; kernel_variant is ignored).
 *
 * It replaces, for this mesh class, the reference's dim3 forward path:
 * the assembly (core/specfem/assembly/ dim3 containers), the element kernel
 * compute_stiffness_interaction<dim3, ...> (include/kokkos_kernels/impl/
 * compute_stiffness_interaction.tpp:26-253 with gradient.hpp:103-156,
 * divergence.hpp:90-137, dim3 elastic stress.hpp:46-99), the dim3 mass matrix,
 * source arrays (core/specfem/assembly/compute_source_array/dim3/impl/*),
 * seismograms (compute_seismogram.tpp) and the Newmark loop
 * (core/specfem/solver/time_marching.tpp:8-131).  Absorbing (Stacey) faces
 * extend the reference's 2D condition (stacey.tpp:50-80) to 3D; the
 * reference's dim3 path has no absorbing boundary.
 */
#ifndef SFG3D_H
#define SFG3D_H

#include "sfg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sfg_handle3d sfg_handle3d;

typedef struct sfg_mesh3d_desc {
  int nex, ney, nez;            /* element e = (ez*ney + ey)*nex + ex */
  const double *nodes;          /* [(nez+1)*(ney+1)*(nex+1)][3] control nodes (x, y, z),
                                   node (i, j, k) at (k*(ney+1) + j)*(nex+1) + i */
  const float *rho, *vp, *vs;   /* [nspec][125], point q = (iz*5 + iy)*5 + ix */
  int absorbing[6];             /* Stacey on faces xmin, xmax, ymin, ymax, zmin, zmax */
} sfg_mesh3d_desc;

typedef struct sfg_source3d {
  double x, y, z;
  int kind;                     /* SFG_SOURCE_FORCE or SFG_SOURCE_MOMENT_TENSOR */
  int stf;                      /* SFG_STF_RICKER */
  double f0, factor, tshift;
  double comp[6];               /* force (fx, fy, fz, 0, 0, 0) or (Mxx, Myy, Mzz, Mxy, Mxz, Myz) */
} sfg_source3d;

typedef struct sfg_info3d {
  int nspec, nglob, nstep, istep, nrec, ntypes, nsig, nsrc;
  double t0;
  size_t device_bytes;
  int elements_per_block;
  int kernels_per_step;
  int kernel_variant;           /* element-kernel form in use: 1 point form, 2 column form */
} sfg_info3d;

/* Reference: specfem::assembly::assembly<dim3> construction from the mesh. */
int sfg3d_create(const sfg_mesh3d_desc *mesh, const sfg_options *opt, sfg_handle3d **out);
void sfg3d_destroy(sfg_handle3d *h);
const char *sfg3d_last_error(const sfg_handle3d *h);
/* Reference: read_sources (src/io/sources/dim3/read_sources.cpp) + source arrays. */
int sfg3d_set_sources(sfg_handle3d *h, int nsrc, const sfg_source3d *src);
/* Receivers [nrec][3] (x, y, z); types SFG_SEIS_DISPLACEMENT/VELOCITY/ACCELERATION.
 * Reference: src/io/receivers/dim3/read_receivers.cpp, receiver interpolants. */
int sfg3d_set_receivers(sfg_handle3d *h, int nrec, const double *xyz, int ntypes, const int *types);
/* Mass matrix (+ Stacey term), upload, step graphs. */
int sfg3d_initialize(sfg_handle3d *h);
/* nsteps time steps (time_marching.tpp:8-131). */
int sfg3d_run(sfg_handle3d *h, int nsteps);
/* nsteps steps timed with CUDA events on the handle's stream (ms). */
int sfg3d_run_timed(sfg_handle3d *h, int nsteps, float *ms);
/* The same with an L2 flush before every step (a write of flush_bytes,
 * larger than L2, then a read of a second buffer of that size, so that the
 * cache holds no dirty lines when the step starts), timing the steps only. */
int sfg3d_run_timed_flushed(sfg_handle3d *h, int nsteps, size_t flush_bytes, float *ms);
/* One step with host input/output: stf_row [nsrc] (pinned host memory, this
 * step's source-time values) copied in, the step's seismogram row
 * [ntypes][nrec][3] copied out; synchronous. */
int sfg3d_step_io(sfg_handle3d *h, const float *stf_row, float *seis_row);
/* Average duration of one launch of kernel `which` (0 element, 1 update). */
int sfg3d_time_kernel(sfg_handle3d *h, int which, int reps, float *ms);
int sfg3d_reset_fields(sfg_handle3d *h);
int sfg3d_get_info(sfg_handle3d *h, sfg_info3d *info);
/* [nsig][ntypes][nrec][3] */
int sfg3d_get_seismograms(sfg_handle3d *h, float *out, size_t count);
/* field [nglob][3] (lattice numbering); which 0 u, 1 v, 2 a */
int sfg3d_get_field(sfg_handle3d *h, int which, float *out, size_t count);
int sfg3d_check_finite(sfg_handle3d *h);

#ifdef __cplusplus
}
#endif
#endif
