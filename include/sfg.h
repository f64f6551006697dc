/*
 * sfg.h — C ABI of libsfg, the B200 (sm_100a) spectral-element time-step
 * engine that stands in for SPECFEM++'s per-time-step kernels.
 *
 * All functions return 0 on success or a negative SFG_ERR_* code; the text of
 * the last error of a handle is returned by sfg_last_error().  No torch or
 * CUDA types appear in the signatures: meshes, sources and receivers are plain
 * host arrays, results are copied into caller-owned host buffers.  A handle is
 * used by one host thread at a time; separate handles are independent.
 *
 * Reference interfaces that each group replaces (paths in SPECFEM++):
 *   sfg_create2d / sfg_create2d_from_database
 *       specfem::io::read_2d_mesh          src/io/mesh/impl/fortran/dim2/mesh.cpp:26-215
 *       specfem::assembly::assembly<dim2>  core/specfem/assembly/assembly/dim2/assembly.cpp
 *   sfg_set_sources     specfem::io::read_2d_sources src/io/sources/dim2/read_sources.cpp:29-172,
 *                       assembly sources  core/specfem/assembly/sources/dim2/sources.cpp
 *   sfg_set_receivers   specfem::io::read_2d_receivers, assembly receivers
 *                       core/specfem/assembly/receivers/dim2/receivers.cpp
 *   sfg_initialize      domain_kernels::initialize  include/kokkos_kernels/domain_kernels.hpp:151-179
 *                       (compute_mass_matrix + invert_mass_matrix)
 *   sfg_step / sfg_run  time_marching<forward>::run core/specfem/solver/time_marching.tpp:33-90:
 *                       newmark predictor/corrector core/specfem/timescheme/newmark.tpp:10-128,
 *                       domain_kernels::update_wavefields include/kokkos_kernels/domain_kernels.hpp:72-141
 *                       (compute_coupling, compute_source_interaction,
 *                        compute_stiffness_interaction, divide_mass_matrix),
 *                       domain_kernels::compute_seismograms :189-203
 *   sfg_get_seismograms receivers.sync_seismograms() + seismogram iterator
 *                       core/specfem/assembly/receivers/dim2/impl/seismogram_iterator.hpp:37-53
 *   sfg_get_field       simulation_field copy_to_host (include/io/wavefield/writer.tpp)
 */
#ifndef SFG_H
#define SFG_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SFG_OK = 0,
  SFG_ERR_ARG = -1,       /* invalid argument / inconsistent sizes */
  SFG_ERR_IO = -2,        /* database file missing or malformed */
  SFG_ERR_CUDA = -3,      /* a CUDA runtime call failed */
  SFG_ERR_LOCATE = -4,    /* a source or receiver lies outside the mesh */
  SFG_ERR_STATE = -5,     /* call out of order (e.g. sfg_run before sfg_initialize) */
  SFG_ERR_NONFINITE = -6, /* the wavefield became NaN/Inf */
  SFG_ERR_UNSUPPORTED = -7
};

/* Edge types, the reference's mesh_entity order for absorbing records. */
enum { SFG_EDGE_BOTTOM = 0, SFG_EDGE_RIGHT = 1, SFG_EDGE_TOP = 2, SFG_EDGE_LEFT = 3 };
enum { SFG_MEDIUM_ACOUSTIC = 0, SFG_MEDIUM_ELASTIC = 1 };
enum { SFG_WAVE_PSV = 0, SFG_WAVE_SH = 1 };
/* Seismogram types; rotation, intrinsic rotation (rotation minus half the
 * curl) and curl (du_x/dz - du_z/dx) exist in Cosserat media
 * (include/medium/dim2/elastic/isotropic_cosserat/wavefield.hpp); scalar
 * types fill the first component. */
enum { SFG_SEIS_DISPLACEMENT = 0, SFG_SEIS_VELOCITY = 1, SFG_SEIS_ACCELERATION = 2,
       SFG_SEIS_PRESSURE = 3, SFG_SEIS_ROTATION = 4, SFG_SEIS_INTRINSIC_ROTATION = 5,
       SFG_SEIS_CURL = 6 };
/* Source-time functions (core/specfem/source_time_functions): Ricker, Dirac
 * (f0 = 1/(10 dt)), Gaussian and its derivative by f0, Gaussian and Heaviside
 * (error function) by half duration hdur (at least 5 dt; start time
 * -2 hdur + tshift, evaluated with hdur / 1.628). */
enum { SFG_STF_RICKER = 0, SFG_STF_DIRAC = 1, SFG_STF_GAUSSIAN = 2, SFG_STF_GAUSSIAN_HDUR = 3,
       SFG_STF_DGAUSSIAN = 4, SFG_STF_HEAVISIDE = 5 };
enum { SFG_FIELD_DISPLACEMENT = 0, SFG_FIELD_VELOCITY = 1, SFG_FIELD_ACCELERATION = 2 };

typedef struct sfg_handle sfg_handle;

/* In-memory 2D mesh, the content of a SPECFEM2D database.bin
 * (specfem::mesh::mesh<dim2>, include/mesh/dim2/mesh.hpp). */
typedef struct sfg_mesh2d_desc {
  int nspec, npgeo, ngnod;       /* ngnod = 4 or 9 control nodes */
  const double *coorg;           /* [npgeo][2] control-node (x, z) */
  const int *knods;              /* [nspec][ngnod], 0-based */
  const int *kmato;              /* [nspec] material index, 0-based */
  int numat;
  const int *mat_medium;         /* [numat] SFG_MEDIUM_* */
  const double *mat_rho, *mat_vp, *mat_vs; /* [numat] */
  const float *point_rho, *point_vp, *point_vs; /* optional [nspec][25] GLL-point models */
  int nabs;
  const int *abs_ispec, *abs_type;   /* absorbing (Stacey) edges */
  int nfree;
  const int *free_ispec, *free_type; /* acoustic free-surface edges */
  int elastic_wave;              /* SFG_WAVE_PSV or SFG_WAVE_SH */
  const double *mat_aniso;       /* optional [numat][6] anisotropic elastic constants
                                    (c11, c13, c15, c33, c35, c55; NaN rows: isotropic);
                                    mat_vp = sqrt(c33/rho), mat_vs = sqrt(c55/rho) there */
  const double *mat_cosserat;    /* optional [numat][8] isotropic Cosserat constants (rho,
                                    kappa, mu, nu, j, lambda_c, mu_c, nu_c; NaN rows: other
                                    materials); the elastic medium then has three
                                    components (u_x, u_z, rotation), P-SV only */
  int nadj;                      /* adjacency records (0: none) */
  const int *adjacency;          /* optional [nadj][4] (element, neighbour, connection 1
                                    strongly conforming / 3 nonconforming, orientation of
                                    the shared entity on the element 0 bottom 1 right 2 top
                                    3 left 4..7 corners), 0-based: the mesh's adjacency
                                    graph (src/io/mesh/impl/fortran/dim2/read_adjacency_graph.cpp).
                                    A nonconforming acoustic-elastic record and its
                                    reverse couple the two media through the edges'
                                    intersection (P-SV elastic media); strongly
                                    conforming records are implied by shared control nodes */
  const double *mat_poro;        /* optional [numat][13] isotropic poroelastic constants
                                    (rho_s, rho_f, phi, tortuosity, kxx, kxz, kzz, kappa_s,
                                    kappa_f, kappa_fr, eta_f, mu_fr, Q_mu = 9999; NaN rows:
                                    other materials); the elastic medium then has four
                                    components (solid u_x, u_z, fluid w_x, w_z), P-SV, no
                                    Stacey edges, no acoustic coupling; seismograms give
                                    the solid motion and the pore pressure */
} sfg_mesh2d_desc;

typedef struct sfg_options {
  double dt;
  int nstep;                     /* steps the source tables cover */
  int nshots;                    /* independent shots advanced together (>= 1) */
  int nstep_between_samples;     /* seismogram sampling (>= 1) */
  int steps_per_graph;           /* time steps per captured CUDA graph (0 = default) */
  int elements_per_block;        /* elements per block of the element kernel: 8, 16, 32
                                    (the row form: 16 or 32; 0 = chosen by the autotuner
                                    at sfg_initialize) */
  int kernel_variant;            /* assembly / element kernel: 1 colour passes (one block
                                    per chunk), 2 colour passes with a persistent
                                    prefetching kernel, 3 owner-computes (one element
                                    launch, per-point sum in colour order), 4 owner-computes
                                    with the element arrays staged by bulk copies, 5 fused
                                    tile kernel (element forces, assembly in shared memory
                                    and the point update of tile-interior points in one
                                    launch; isotropic P-SV / SH / acoustic media, or
                                    batched shots in fours on one elastic medium, others
                                    fall back to 3); with batched shots 2 is 1 and 4 is
                                    owner-computes with the row-form element kernel (one
                                    thread per element row and quad of shots; shots in
                                    fours); 6 owner-computes with the row-form element
                                    kernel of one shot (one thread per element row;
                                    isotropic P-SV and acoustic media, 16 or 32 elements
                                    per block, others fall back to 3); with batched shots
                                    in fours and displacement receivers, 7 assembles and
                                    finishes each four-element tile's interior points in
                                    the element kernel (others fall back to 3); all give
                                    the same bits (0 = chosen by the autotuner) */
  int store_acceleration;        /* also keep the elastic acceleration inside runs */
  int has_start_time;            /* 1: the run starts at start_time (the configuration's
                                    time-scheme t0) and sources keep their own tshift;
                                    0: start at the earliest source start, shifts relative
                                    to it (src/io/sources/dim2/read_sources.cpp:142-172) */
  double start_time;
} sfg_options;

typedef struct sfg_source2d {
  double x, z;
  int shot;                      /* shot this source belongs to (0..nshots-1) */
  int stf;                       /* SFG_STF_* */
  double f0, factor, tshift, angle;
  int kind;                      /* SFG_SOURCE_FORCE or SFG_SOURCE_MOMENT_TENSOR */
  double mxx, mzz, mxz;          /* moment tensor (kind SFG_SOURCE_MOMENT_TENSOR) */
  double hdur;                   /* half duration (SFG_STF_GAUSSIAN_HDUR, SFG_STF_HEAVISIDE) */
} sfg_source2d;

enum { SFG_SOURCE_FORCE = 0, SFG_SOURCE_MOMENT_TENSOR = 1 };

typedef struct sfg_info {
  int nspec, nspec_elastic, nspec_acoustic;
  int nglob, nglob_elastic, nglob_acoustic;
  int ncolors_elastic, ncolors_acoustic;
  int nshots, nsig, nrec, ntypes, nstep;
  int istep;                     /* next step to be run */
  double t0;                     /* time of step 0 (earliest shot) */
  size_t device_bytes;
  int kernels_per_step;
  int elements_per_block, kernel_variant; /* launch shape in use */
  int ncomp_elastic;             /* components of the elastic fields: 2 P-SV, 1 SH,
                                    3 Cosserat (u_x, u_z, rotation), 4 poroelastic
                                    (solid u_x, u_z, fluid w_x, w_z) */
} sfg_info;

/* ---- life cycle ---- */
int sfg_create2d(const sfg_mesh2d_desc *mesh, const sfg_options *opt, sfg_handle **out);
int sfg_create2d_from_database(const char *database_path, int elastic_wave,
                               const sfg_options *opt, sfg_handle **out);
void sfg_destroy(sfg_handle *h);
const char *sfg_last_error(const sfg_handle *h);   /* NULL handle: last create error */

/* ---- sources / receivers (before sfg_initialize) ---- */
/* After sfg_initialize, sources may be replaced by as many new ones (next
 * shot of a sequential survey, e.g. one source per adjoint gradient). */
int sfg_set_sources(sfg_handle *h, int nsrc, const sfg_source2d *src);
/* Optional external source-time table [nstep][nsrc] (overrides the analytic STFs). */
int sfg_set_stf_table(sfg_handle *h, const float *table, int nstep, int nsrc);
int sfg_set_receivers(sfg_handle *h, int nrec, const double *x, const double *z,
                      double angle_deg, int ntypes, const int *types);

/* ---- mass matrix, upload, graph build ---- */
int sfg_initialize(sfg_handle *h);

/* ---- time stepping ---- */
/* After sfg_step and sfg_run the fields hold the reference's end-of-step
 * state (displacement after the predictor, velocity after the corrector). */
int sfg_step(sfg_handle *h);                        /* one step */
int sfg_run(sfg_handle *h, int nsteps);             /* nsteps steps via CUDA graphs */
int sfg_synchronize(sfg_handle *h);
int sfg_reset_fields(sfg_handle *h);                /* zero wavefields, istep = 0 */
/* Device time of nsteps graph-replayed steps, measured with CUDA events on the
 * handle's stream (inputs resident); ms_total receives the elapsed time. */
int sfg_run_timed(sfg_handle *h, int nsteps, float *ms_total);
/* Device time of nsteps steps, each launched separately after an L2 flush
 * outside the timed interval (a write of flush_bytes to a scratch buffer, then
 * a read of a second scratch buffer of flush_bytes, so that the cache holds
 * none of the model's data and no dirty lines); returns the sum of the
 * per-step times measured with CUDA events on the handle's stream. */
int sfg_run_timed_flushed(sfg_handle *h, int nsteps, size_t flush_bytes, float *ms_total);
/* One step with host buffers: copies this step's source-time values
 * stf_row[nsrc] (host, may be NULL to keep the table) to the device, runs the
 * step, and copies the seismogram sample of the step (when the step is a
 * sampling step) into seis_row[nshots][ntypes][nrec][2] (host, may be NULL);
 * returns after the copy has landed.  This is the per-step path a host driver
 * that streams sources in and traces out would call.  The step is the fused
 * one of a run: afterwards the fields hold the next step's predictor, and
 * sfg_get_field refuses them until sfg_step or sfg_run ends on the exact
 * end-of-step state. */
int sfg_step_io(sfg_handle *h, const float *stf_row, float *seis_row);
/* Average device time of one launch of a named kernel family, timed alone with
 * CUDA events: which = 0 element (stiffness) launches of one step, all colours
 * and both media; 1 elastic point update; 2 acoustic point update;
 * 3 receiver kernels.  With the fused tile kernel (variant 5): 0 the tile
 * kernel (elements and tile-interior points of both media), 1 the boundary
 * points of both media, 2 nothing (0 ms), 3 receivers.  Leaves the fields
 * mid-step (sfg_reset_fields after). */
int sfg_time_kernel(sfg_handle *h, int which, int iters, float *ms_per_launch);
/* The same with the L2 cache flushed before every launch, outside the timed
 * interval, as sfg_run_timed_flushed does before a step, so that the launch
 * reads all its inputs from HBM; flush_bytes = 0 is sfg_time_kernel. */
int sfg_time_kernel_flushed(sfg_handle *h, int which, int iters, size_t flush_bytes, float *ms_per_launch);

/* ---- step-wise interface: the reference's kernel facade ----
 * One phase per call, in the reference's granularity, on the handle's own
 * fields; a host loop that calls them in time_marching<forward>::run's order
 * (predictor of every medium, update_wavefields and corrector of the acoustic
 * medium, then of the elastic medium, then compute_seismograms) gives
 * sfg_run's seismograms and fields bit for bit.  Single-shot handles; the
 * calls are asynchronous on the handle's stream (sfg_synchronize to wait);
 * the handle's own step count is not advanced (the caller passes istep).
 *   sfg_predictor        newmark_impl::predictor_phase_impl
 *                        core/specfem/timescheme/newmark.tpp:64-128: u += dt v +
 *                        dt^2/2 a, v += dt/2 a, a = 0; returns the degrees of
 *                        freedom updated (nglob * ncomp of the medium, 0 when absent)
 *   sfg_update_wavefields domain_kernels::update_wavefields<medium>(istep)
 *                        include/kokkos_kernels/domain_kernels.hpp:72-141: coupling
 *                        with the other medium, sources of step istep, stiffness
 *                        with Stacey / free surface, division by the mass matrix;
 *                        returns the elements updated (the medium's nspec)
 *   sfg_corrector        newmark_impl::corrector_phase_impl newmark.tpp:10-62:
 *                        v += dt/2 a; returns nglob * ncomp
 *   sfg_compute_seismograms domain_kernels::compute_seismograms(isig_step)
 *                        domain_kernels.hpp:189-203: sample isig of every receiver
 * frechet_kernels::compute_derivatives (include/kokkos_kernels/frechet_kernels.hpp:
 * 37-49) has no step-wise counterpart: it accumulates per step against a
 * backward wavefield that the reference reconstructs by running Newmark
 * backwards, which the discrete adjoint here replaces by checkpoints and
 * recomputation; sfg_adjoint_gradient runs the whole combined simulation. */
int sfg_predictor(sfg_handle *h, int medium);
int sfg_update_wavefields(sfg_handle *h, int medium, int istep);
int sfg_corrector(sfg_handle *h, int medium);
int sfg_compute_seismograms(sfg_handle *h, int isig);

/* ---- results ---- */
int sfg_get_info(const sfg_handle *h, sfg_info *info);
/* Seismograms [nshots][nsig][ntypes][nrec][2], receiver-angle rotation applied. */
int sfg_get_seismograms(sfg_handle *h, float *out, size_t count);
/* Wavefield of one medium, in the handle's per-medium point numbering:
 * elastic [nshots][nglob_elastic][ncomp], acoustic [nshots][nglob_acoustic]. */
int sfg_get_field(sfg_handle *h, int medium, int which, float *out, size_t count);
/* Global (mesh) id of every element GLL point in database element order,
 * and the per-medium index of each global point (-1 if absent). */
int sfg_get_numbering(sfg_handle *h, int *ibool_global, int *glob_to_elastic,
                      int *glob_to_acoustic);
/* Coordinates x, z and |J| of every element GLL point [nspec][25] (database
 * element order, point q = iz*5 + ix; FP64) and the medium of every element
 * (SFG_MEDIUM_*); any pointer may be NULL.  What the reference's kernel and
 * wavefield writers take from its mesh (include/io/impl/medium_writer.tpp,
 * include/io/wavefield/writer.tpp). */
int sfg_get_geometry(sfg_handle *h, double *x, double *z, double *jac, int *medium);
/* Non-zero once a non-finite value was seen in the elastic/acoustic update. */
int sfg_check_finite(sfg_handle *h);

/* ---- adjoint (one 2D medium, one shot, seismograms every step: isotropic
 * elastic P-SV or SH with displacement seismograms (in SH the gradient with
 * respect to kappa is zero), or acoustic with pressure seismograms (there the
 * bulk modulus is kappa + 4/3 mu, so dL/dmu = 4/3 dL/dkappa)) ----
 * Replace the model by per-GLL-point rho, kappa, mu ([nspec][25], database
 * element order; kappa = lambda + 2/3 mu as the reference stores it).
 * Reference: the property container, core/specfem/assembly/properties. */
int sfg_set_model2d(sfg_handle *h, const float *rho, const float *kappa, const float *mu);
/* Forward run of nsteps steps from rest that keeps the state every `interval`
 * steps on the device (seismograms as sfg_run).  Replaces the reference's
 * forward-wavefield dump for adjoint runs (include/io/wavefield/writer.tpp). */
int sfg_forward_checkpointed(sfg_handle *h, int nsteps, int interval);
/* Device memory for the adjoint's segment buffers (each holds one checkpoint
 * interval of recorded forward states).  The forward run records its last
 * segments into them on the way, as many as the buffers hold, so that the
 * reverse sweep recomputes only the earlier segments; bytes = 0 (the
 * default) takes 75% of the device memory free when the buffers are
 * allocated (at the next sfg_forward_checkpointed); at least two buffers are
 * always kept.  Gradients do not depend on it (bit for bit).  No counterpart
 * in the reference, whose combined run reads the whole forward wavefield
 * back from storage. */
int sfg_set_adjoint_budget(sfg_handle *h, size_t bytes);
/* Segment buffers allocated by the last sfg_forward_checkpointed (0 before). */
int sfg_adjoint_buffers(sfg_handle *h);
/* Gradient of a misfit L with respect to rho, kappa, mu at every GLL point
 * ([nspec][25], database element order) given seis_grad = dL/d(seismogram)
 * [nsteps][nrec][2]: the reverse sweep recomputes each checkpoint segment
 * that the forward run did not keep and runs the discrete adjoint of the
 * time step.  Models: one isotropic elastic (P-SV or SH, displacement
 * seismograms) or acoustic (pressure seismograms) medium, or a coupled
 * acoustic-elastic model with conforming interfaces and either displacement
 * seismograms at receivers in the elastic medium or pressure seismograms at
 * receivers in the acoustic medium; else SFG_ERR_UNSUPPORTED.  Replaces the reference's
 * combined adjoint/backward run and compute_material_derivatives
 * (core/specfem/solver/time_marching.tpp:133-264,
 *  include/kokkos_kernels/impl/compute_material_derivatives.tpp:14-153). */
int sfg_adjoint_gradient(sfg_handle *h, const float *seis_grad, float *grad_rho, float *grad_kappa,
                         float *grad_mu);

/* One time step of the handle's elastic model on device buffers the caller
 * owns, with no device memory allocated by the call.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc while they step: a host framework that owns and budgets all
 * device memory itself (as the reference's Kokkos runtime does), or a time
 * loop that runs after the device memory has been sized and frozen.  The
 * handle must be initialised (that is where its read-only mesh arrays were
 * uploaded) and hold a single isotropic elastic medium (P-SV or SH; other
 * media are refused with SFG_ERR_UNSUPPORTED).  u, v, a are the displacement,
 * velocity and acceleration in the handle's elastic point numbering
 * ([nglob_elastic][ncomp] floats on the handle's device, each starting on a
 * 16-byte boundary, else SFG_ERR_ARG before any launch), in the end-of-step
 * state that sfg_step leaves; the call applies the predictor, the element
 * kernel and the corrector exactly as sfg_step does and writes the new state
 * back into u, v, a, using source-time values of step istep.  It records no
 * seismogram sample (sfg_step does).  The work runs on the handle's stream,
 * which does not wait for other streams: finish every write to u, v, a (for
 * example with a device or stream synchronize) before the call.  The element
 * kernel's accumulator lives in a fixed array inside the library, limited to
 * 4,194,304 point values (2,097,152 two-component points); larger models are
 * rejected with SFG_ERR_ARG.  All calls share that array (it is cleared at
 * the start of every call), so calls that overlap on the GPU race.  The first
 * call on a device looks up the array's device address; make that first call
 * before any stream capture.  The handle's own fields and step count are not
 * touched; the call returns after the step has finished on the GPU, with
 * SFG_ERR_NONFINITE when the new displacement holds a NaN or Inf. */
int sfg_step_noalloc(sfg_handle *h, int istep, float *u, float *v, float *a);

#ifdef __cplusplus
}
#endif
#endif /* SFG_H */
