/*
 * chanflow_host.h -- host-side C++ mirror of the reference's setup module
 * (PFC/setup.f90) and initial-field generator (PFC/init_vel.f90) for callers
 * without a Fortran host: parses flow.dat, computes the grid operators and
 * wavenumbers that cfg_create takes, and builds seeded initial fields.
 * A Fortran host keeps its own setup.f90 and only needs chanflow.h.
 */
#ifndef CHANFLOW_HOST_H
#define CHANFLOW_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

/* flow.dat run parameters (PFC/setup.f90:45-160) plus the extension block
 * that may follow line 95 (lines "value  name": stretch, dt, seed,
 * precision, uniform_grid, jet_mode, jet_width, jet_peak, jet_freq). */
typedef struct cfh_run {
  double re, ctrlu, ctrlw, lx, lz, beta, disturb_ampl;
  int nx, ny, nz, nx2, nz2;
  int tend, output_step, save_step, l2_step;
  int read_vel, save_vel, vel_out, which_test;
  int fix_mass, dt_flag, divg_check;
  int bl_grid, crossflow, filter_jet_profile;
  double jet_diam, xjet_top, zjet_top, jetmag_top, forcing_top, for_freq_top;
  double xjet_bot, zjet_bot, jetmag_bot, forcing_bot, for_freq_bot;
  int xfringe, zfringe;
  double frac_xbuff;
  /* extension block */
  double stretch;         /* default 2.75 (PFC/setup.f90:545) */
  double dt;              /* <= 0: define_parameters default 0.25*lx/nx */
  unsigned long long seed;
  int precision;          /* CFG_FP64 / CFG_MIXED */
  int uniform_grid;       /* which_test 6 grid */
  int jet_mode;           /* 0 none, 1 reference tanh jet, 2 gaussian slot */
  double jet_width, jet_peak, jet_freq;
  /* fringe parameters, flow.dat lines 88-95 */
  double fringe_gain, buff_xrise, buff_xfall, frac_zbuff, buff_zrise, buff_zfall;
} cfh_run;

/* Grid operators in reference layout, owned by the caller (sizes as in
 * chanflow.h's cfg_grid).  cfh_grid_alloc/free manage the arrays. */
typedef struct cfh_grid {
  int nx, ny, nz, nx2, nz2;
  double *y, *yh, *hh, *hn, *dh, *dn, *iu, *dm, *d2h, *d2n, *dyh, *dy, *kx, *kz;
  double *buffer, *target_inflow, *xcoord, *zcoord;
} cfh_grid;

void cfh_run_defaults(cfh_run *r);
/* read_parms: 0 on success, <0 on a malformed or short file */
int cfh_read_flow_dat(const char *path, cfh_run *r, char *err, int errlen);

cfh_grid *cfh_grid_alloc(int nx, int ny, int nz, int nx2, int nz2);
void cfh_grid_free(cfh_grid *g);
/* define_coordinates (channel branch, PFC/setup.f90:541-754) and the
 * wavenumbers of define_parameters (:1439-1466). */
int cfh_define_grid(cfh_grid *g, double lx, double lz, double stretch, int uniform);

/* Seeded initial field in data1 layout (nz, nx/2+1, ny+1, 3), complex
 * interleaved: which_test 1, 4, 6 (PFC/init_vel.f90:88-244) and 10
 * (laminar 1-y^2 plus k^-2 divergence-free noise).  The divergence removal
 * and initial pressure run on the device (cfg_remove_initial_divergence,
 * cfg_compute_initial_pressure). */
int cfh_initial_field(const cfh_grid *g, int which_test, unsigned long long seed,
                      double ampl, double beta, double *data1);

/* The Orr-Sommerfeld initial fields, which_test 2, 5 and 8
 * (PFC/init_vel.f90:95-159).
 *
 * cfh_read_efn: efn.m as READ_EIGENFUNCTION reads it (PFC/init_vel.f90:565-572):
 * 4 x 65 numbers, one per line, column after column -- Re u, Im u, Re v, Im v
 * at the Chebyshev-Gauss-Lobatto points y_j = cos(pi j / 64), j = 0..64 --
 * into uin (65, 4) column-major.  Fortran D exponents are accepted.  Returns
 * 0, -1 when the file cannot be opened, -2 when it is short or malformed.
 *
 * cfh_interp_eigenfunction: the rest of READ_EIGENFUNCTION (:583-633): the
 * Chebyshev coefficients of the four columns, u summed onto yh(2..ny) with
 * u(1) = u(ny+1) = 0, v onto y(1..ny) with v(ny+1) = 0.  u, v: (ny+1)
 * complex, interleaved.
 *
 * cfh_initial_field_mode: the which_test 2 / 5 / 8 velocity before the
 * divergence removal: the laminar profile plus ampl times the mode in
 * Fourier column (kz 1, kx 2) for 2, (kz 2 and its conjugate kz nz, kx 1)
 * for 5 and (kz 2, kx 2) for 8, rotated by beta as the reference does.
 * data1 (nz, nx/2+1, ny+1, 3) complex interleaved.  Returns -1 for another
 * which_test. */
int cfh_read_efn(const char *path, double *uin);
int cfh_interp_eigenfunction(const cfh_grid *g, const double *uin, double *u, double *v);
int cfh_initial_field_mode(const cfh_grid *g, int which_test, double ampl, double beta,
                           const double *u, const double *v, double *data1);

/* read_write::save_velocity / read_velocity (PFC/read_write.f90:21-292) on
 * host arrays in data1 layout (nz, nx/2+1, ny+1, 3): the reference's restart
 * file, Fortran unformatted sequential (4-byte record markers, native byte
 * order): a header record NX, NY, NZ, LX, LZ, RE, DT, T_TOTAL, one record
 * per kx holding data1(1:nz, kx, 1:ny+1, 1:3), and a closing record 0, 0
 * (no dynamic SGS coefficients).  cfh_read_velocity applies read_velocity's
 * checks (NX, NY, NZ equal; LX, LZ within EPSILON) and returns CFG_E_ARG
 * with the reference's message in err otherwise; a changed RE is reported
 * on stderr and accepted, as the reference does.  It returns the file's DT
 * and T_TOTAL (the caller keeps its own dt unless dt_flag, :75-78). */
int cfh_save_velocity(const char *path, int nx, int ny, int nz, double lx, double lz, double re,
                      double dt, double t_total, const double *data1, char *err, int errlen);
int cfh_read_velocity(const char *path, int nx, int ny, int nz, double lx, double lz, double re,
                      double *dt, double *t_total, double *data1, char *err, int errlen);

/* The seeded counter-based generator replacing RANDOM_NUMBER. */
double cfh_rng_u01(unsigned long long seed, int x, int z, int j, int col);

#ifdef __cplusplus
}
#endif
#endif
