/* CPU oracle of the 3D elastic step (test infrastructure only). */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleInput3D {
  int nex, ney, nez;          /* structured lattice of 8-node hexahedra */
  const double *nodes;        /* [(nez+1)][(ney+1)][(nex+1)][3] control nodes (x, y, z) */
  const double *rho, *vp, *vs; /* [nspec][125] per GLL point; element e = (ez*ney + ey)*nex + ex */
  int absorbing[6];           /* Stacey on face: xmin xmax ymin ymax zmin zmax */
  int nsrc;
  const int *src_kind;        /* 0 force, 1 moment tensor */
  const double *src_xyz;      /* [nsrc][3] */
  const double *src_comp;     /* [nsrc][6]: (fx, fy, fz, 0, 0, 0) or (Mxx, Myy, Mzz, Mxy, Mxz, Myz) */
  const double *src_f0, *src_factor, *src_tshift;
  double t0;                  /* time of step 0 */
  int nrec;
  const double *rec_xyz;      /* [nrec][3] */
  int ntypes;
  const int *seis_types;      /* 0 displacement 1 velocity 2 acceleration */
  double dt;
  int nstep;
  /* 0: the reference's evaluation order; 1: the device kernels' order (the
   * 5-term contractions as fused multiply-adds, hprime * w rounded once) */
  int device_order;
} OracleInput3D;

typedef struct OracleOutput3D {
  double *seismograms;        /* [nstep][ntypes][nrec][3] */
  double *final_u;            /* optional [nglob][3] (lattice numbering) */
  int nglob;
  double seconds;             /* wall time of the time loop */
  char error[256];
} OracleOutput3D;

int oracle3d_run_f32(const OracleInput3D *in, OracleOutput3D *out, int nthreads);
int oracle3d_run_f64(const OracleInput3D *in, OracleOutput3D *out, int nthreads);

#ifdef __cplusplus
}
#endif
