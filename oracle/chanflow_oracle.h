/*
 * chanflow_oracle.h -- CPU FP64 restatement of the reference channel-flow
 * solver's per-timestep hot path.  TEST INFRASTRUCTURE ONLY: this library is
 * the checker that the CUDA product is compared against.  Nothing in the
 * product links, loads or calls it.
 *
 * The reference (Fortran 90 + MPI + FFTW3) cannot be compiled here (no Fortran
 * compiler, MPI or FFTW).  This file restates its arithmetic in C, citing the
 * Fortran routine each function follows (paths relative to the reference
 * project, PFC = ParallelFortran-Code/).
 *
 * Pinning: the restatement is pinned against the reference's own known-answer
 * data: PFC/makegrid.m (y/yh at ny=200, stretch 2.75), the which_test=6
 * analytic decaying-vortex solution (PFC/main_mpi.f90:121-161), the constant
 * bulk flux Q=4/3 under fix_mass (PFC/diagnostics.txt:111,138) and
 * round-off divergence (PFC/pass2.f90:380-419).  FFTW's own rounding is not
 * pinned (no FFTW outputs ship with the reference); the DFT here is checked
 * against numpy.fft.
 *
 * Array layouts are the reference's Fortran (column-major) layouts:
 *   data1 (nz, nx/2+1, ny+1, 3)   complex   PFC/data.f90:9, PFC/setup.f90:447
 *   data2 (ny+1, 3, nz, nx/2+1)   complex   PFC/setup.f90:448
 *   data4 (ny+1, nz, nx/2+1)      complex   PFC/setup.f90:449
 *   cbc_top/cbc_bot (nz, nx/2+1, 3) complex PFC/setup.f90:565-566
 *   physical planes (nx2, nz2)    real
 */
#ifndef CHANFLOW_ORACLE_H
#define CHANFLOW_ORACLE_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
  int nx, ny, nz, nx2, nz2;
  double re, lx, lz, beta;      /* beta already in radians */
  double dt, cfl_max;
  int fix_mass, dt_flag;
  double ctrlu, ctrlw;
  double stretch;               /* tanh stretching, PFC/setup.f90:545 */
  int uniform_grid;             /* which_test=6 uniform grid on [-1/2,1/2] */
  int nthreads;                 /* OpenMP threads (0 = default) */
} orc_params;

typedef struct orc_ctx orc_ctx;

orc_ctx *orc_create(const orc_params *p);
void orc_destroy(orc_ctx *c);

/* accessors (pointers into the context; sizes follow the reference) */
double *orc_grid(orc_ctx *c, const char *name, int *len);
double complex *orc_data1(orc_ctx *c);
double complex *orc_data2(orc_ctx *c);
double complex *orc_data4(orc_ctx *c);
double complex *orc_cbc_top(orc_ctx *c);
double complex *orc_cbc_bot(orc_ctx *c);
double *orc_buffer(orc_ctx *c);          /* fringe damping (nx2, nz2) */
double *orc_target_inflow(orc_ctx *c);   /* (ny+1, 3) */
double *orc_baseflow(orc_ctx *c);        /* linearized baseflow profile (ny+1, 3) */
double *orc_d_um_dy(orc_ctx *c);         /* (ny) */
double *orc_cfl(orc_ctx *c);             /* (ny+1) per-plane CFL of last rk1 */
void orc_get_scalars(orc_ctx *c, double *t_total, double *dt, double *p_grad);
void orc_set_scalars(orc_ctx *c, double t_total, double dt, double p_grad);
void orc_set_step(orc_ctx *c, int step, int rk_step);
int orc_status(orc_ctx *c);              /* 0 ok, <0 the reference would STOP */

/* transforms, PFC/transform.f90 */
void orc_fft(int n, int sign, const double complex *in, double complex *out);
void orc_xz_c2r(orc_ctx *c, const double complex *cdata, double *data);
void orc_xz_r2c(orc_ctx *c, const double *data, double complex *cdata);
void orc_div_fluxes(orc_ctx *c, const double *dx, const double *dy,
                    const double *dz, double complex *cdata);
void orc_small_r2c(orc_ctx *c, const double *data, double complex *cdata);
void orc_small_c2r(orc_ctx *c, const double complex *cdata, double *data);

/* hot path */
void orc_nonlinear(orc_ctx *c);            /* PFC/pass1.f90:26-124 */
void orc_nonlinear_linearized(orc_ctx *c); /* PFC/pass1_linearized.f90:135-250 */
void orc_rhs_solve(orc_ctx *c);            /* PFC/pass2.f90:29-180 */
void orc_boundary(orc_ctx *c);             /* PFC/read_write.f90:1465-1532 */
void orc_l2_norm(orc_ctx *c, double *l2, double *drag); /* PFC/read_write.f90:1432 */

/* initial field, PFC/init_vel.f90 */
void orc_init_field(orc_ctx *c, int which_test, unsigned long long seed,
                    double ampl);
void orc_initial_velocity(orc_ctx *c, int which_test, unsigned long long seed,
                          double ampl);
double orc_rng_u01(unsigned long long seed, int x, int z, int j, int col);
void orc_remove_initial_divergence(orc_ctx *c);
void orc_init_from_velocity(orc_ctx *c);   /* PFC/init_vel.f90:325-351 on a caller-set data1 */
void orc_compute_d_um_dy(orc_ctx *c);
void orc_compute_initial_pressure(orc_ctx *c, int linearized);
void orc_strip_divergence_column(orc_ctx *c, double complex *cu /*(ny+1,3)*/,
                                 double complex *cp /*(ny+1)*/, double coef,
                                 int x, int z);

/* time loop, PFC/main_mpi.f90:70-86 */
void orc_timestep(orc_ctx *c, int nsteps, int linearized);

/* diagnostics */
double orc_bulk_flux(orc_ctx *c);          /* Q, PFC/pass2.f90:106-108 */
double orc_max_divergence(orc_ctx *c);     /* PFC/pass2.f90:380-419 */

/* wall forcing (cbc(:,:,2)), PFC/pass2.f90:423-673.  Index 0 is the bottom
 * wall, 1 the top; a wall is forced when its jetmag is nonzero (:494,517). */
typedef struct orc_jet {
  int mode;               /* 0 none, 1 reference tanh jet, 2 gaussian slot */
  double xjet[2], zjet[2];        /* jet centre (absolute x, z) */
  double jetmag[2];               /* jet velocity (mode 2: slot peak velocity) */
  double forcing[2], for_freq[2]; /* amplitude modulation, mode 1 */
  double jet_diam;                /* mode 1 */
  double width, freq;             /* gaussian slot: v = jetmag exp(-(d/width)^2) (1+sin 2 pi freq t)/2 */
  double frac_xbuff;      /* suction region (PFC/pass2.f90:553-609) */
  int filter_jet_profile;
  double jet_forcing[24];       /* (3,2,4) Freund forcing parameters */
  double jet_forcing_incr[24];  /* (3,2,4) their random-walk increments */
  unsigned long long seed;      /* random walk RNG seed (0: parameters fixed) */
} orc_jet;
/* crossflow == 1: rhs_solve calls jet_profile at every substep with the
 * end-of-substep time (PFC/pass2.f90:37-44).  NULL switches it off. */
void orc_set_jet(orc_ctx *c, const orc_jet *j);
/* jet_profile(time, time_incr): random walk of the forcing parameters
 * (:454-477, RANDOM_NUMBER replaced by the counter RNG, draw n of call k is
 * orc_rng_u01(seed, k, 0, n, 7)), then the wall profile into cbc(:,:,2). */
void orc_jet_profile(orc_ctx *c, double time, double time_incr);
/* current forcing parameters and increments (24 each, may be NULL) */
void orc_get_jet_forcing(orc_ctx *c, double *jet_forcing, double *jet_forcing_incr);

/* Arnoldi propagator matvec, PFC/arnoldi.f90:485-567 */
void orc_arnoldi_matvec(orc_ctx *c, int tend, const double *v, double *w);

#ifdef __cplusplus
}
#endif
#endif
