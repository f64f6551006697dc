/* CPU oracle for the SPECFEM++ 2D time step (test infrastructure only). */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleInput2D {
  int nspec, npgeo, ngnod;
  const double *coorg;   /* [npgeo][2] */
  const int *knods;      /* [nspec][ngnod], 0-based */
  const int *medium;     /* [nspec]: 0 acoustic, 1 elastic */
  const double *rho, *vp, *vs; /* [nspec][25] per GLL point */
  int elastic_sh;        /* 0: P-SV, 1: SH */
  int nabs;
  const int *abs_ispec, *abs_type;   /* type: 0 bottom 1 right 2 top 3 left */
  int nfree;
  const int *free_ispec, *free_type;
  int nsrc;
  const double *src_x, *src_z, *src_angle, *src_f0, *src_factor, *src_tshift;
  const double *stf_table; /* optional [nstep][nsrc]; overrides Ricker */
  double t0;
  int nrec;
  const double *rec_x, *rec_z;
  double rec_angle;
  int ntypes;
  const int *seis_types;   /* 0 displacement 1 velocity 2 acceleration 3 pressure
                              4 rotation 5 intrinsic rotation 6 curl (Cosserat) */
  double dt;
  int nstep, nstep_between_samples;
  /* 0: setup geometry (Jacobians, point location, interpolants) in FP64 and
   * rounded to the run precision; 1: setup in the run precision, as the
   * reference does with type_real. */
  int setup_in_run_precision;
  /* optional per-source kind (NULL: all force sources): 0 force, 1 moment
   * tensor with components src_mxx, src_mzz, src_mxz */
  const int *src_kind;
  const double *src_mxx, *src_mzz, *src_mxz;
  /* optional anisotropic elastic constants per GLL point [nspec][25][6]
   * (c11, c13, c15, c33, c35, c55); NULL: isotropic from rho, vp, vs */
  const double *aniso;
  /* optional Cosserat elastic constants per GLL point [nspec][25][8] (rho,
   * kappa, mu, nu, j, lambda_c, mu_c, nu_c): three components (u_x, u_z,
   * rotation); NULL: none */
  const double *cosserat;
  /* optional mesh adjacency records [nadj][4]: (element, neighbour,
   * connection 1 strongly conforming / 3 nonconforming, orientation of the
   * shared entity on the element 0 bottom 1 right 2 top 3 left, 4..7
   * corners), 0-based.  Nonconforming acoustic-elastic records couple the
   * two media through an intersection quadrature; NULL or nadj 0: none */
  int nadj;
  const int *adjacency;
  /* optional isotropic poroelastic materials per GLL point [nspec][25][13]
   * (rho_s, rho_f, phi, tortuosity, kxx, kxz, kzz, kappa_s, kappa_f,
   * kappa_fr, eta_f, mu_fr, Q_mu): four components (solid u_x, u_z, fluid
   * w_x, w_z); NULL: none */
  const double *poro;
  /* 0: the reference's evaluation order (products and sums rounded
   * separately); 1: the device kernels' order (the 5-term contractions as
   * fused multiply-adds, the divergence weights hprime * w rounded once).
   * Both restate the same algorithm; they differ only in FP32 rounding. */
  int device_order;
} OracleInput2D;

typedef struct OracleOutput2D {
  double *seismograms;       /* [nsig][ntypes][nrec][2] */
  double *final_u_elastic;   /* optional [nglob][ncomp] */
  double *final_u_acoustic;  /* optional [nglob] */
  int *ibool;                /* optional [nspec][25] */
  int nglob;
  double loop_seconds;       /* wall time of the time loop alone */
  char error[256];
} OracleOutput2D;

int oracle2d_run_f32(const OracleInput2D *in, OracleOutput2D *out, int nthreads);
int oracle2d_run_f64(const OracleInput2D *in, OracleOutput2D *out, int nthreads);
int oracle2d_count_nglob(const OracleInput2D *in);
/* The reference's combined simulation (adjoint field from the adjoint
 * sources adj [nstep][nrec][2] at the receivers, backward field by reverse
 * Newmark with Stacey replay, or the forward snapshots when reconstruct = 0)
 * and its Frechet kernels rho, mu, kappa per element GLL point [nspec][25];
 * quirk = 1 adds the adjoint derivatives into the backward ones as the
 * reference's two-field gradient does.  weight: w_x w_z |J| per point.
 * Isotropic elastic P-SV models; FP64. */
int oracle2d_adjoint_compat_f64(const OracleInput2D *in, const double *adj, int quirk, int reconstruct,
                                double *rho_kl, double *mu_kl, double *kappa_kl, double *weight,
                                char *error, int error_len);
int oracle2d_locate(const OracleInput2D *in, int precision64, double x, double z, int *ispec,
                    double *xi, double *gamma);
void oracle_gll(double *z, double *w, double *hprime);
double oracle_legendre(double x, int n);
void oracle_stress_psv(double kappa, double mu, const double *du, double *sigma);

#ifdef __cplusplus
}
#endif
