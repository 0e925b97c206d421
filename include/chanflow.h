/*
 * chanflow.h -- C ABI of the B200 (sm_100a) channel-flow hot path.
 *
 * A drop-in for the per-timestep routines of the reference Fortran solver
 * (PFC = ParallelFortran-Code/).  The reference has no FFI layer of its own:
 * its boundary is a set of Fortran module procedures that talk through module
 * globals.  Each entry point below replaces one of them; a Fortran caller
 * binds them with ISO_C_BINDING and keeps its module
 * interfaces, flow.dat parameters and read_write file layouts unchanged.
 *
 * Conventions
 *  - Every call returns 0 on success or a negative CFG_E_* code; the message
 *    is available from cfg_last_error().  The device never traps: device-side
 *    failures (CFL abort) set a flag that the host reads (cfg_status).
 *  - Host arrays use the reference's Fortran (column-major) layouts; complex
 *    values are interleaved (re, im) doubles, i.e. C_DOUBLE_COMPLEX.
 *      data1 (nz, nx/2+1, ny+1, 3)   PFC/data.f90:9,   PFC/setup.f90:447
 *      data2 (ny+1, 3, nz, nx/2+1)   PFC/data.f90:9,   PFC/setup.f90:448
 *      data4 (ny+1, nz, nx/2+1)      PFC/data.f90:10,  PFC/setup.f90:449
 *      cbc_top/cbc_bot (nz, nx/2+1, 3)  PFC/gridparms.f90:59, PFC/setup.f90:565
 *  - State lives on the device between calls; upload/download are the only
 *    host<->device copies of the fields.  Calls on one context are issued in
 *    order on the context's CUDA stream and are not re-entrant.
 */
#ifndef CHANFLOW_H
#define CHANFLOW_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFG_OK 0
#define CFG_E_ARG (-1)        /* invalid argument / unsupported size */
#define CFG_E_CUDA (-2)       /* CUDA runtime error */
#define CFG_E_NOMEM (-3)      /* device allocation failed */
#define CFG_E_CFL (-4)        /* 'CFL IS TOO BIG', PFC/pass1.f90:235-244 */
#define CFG_E_DT (-5)         /* 'DT IS TOO BIG', PFC/pass1.f90:228-233 */
#define CFG_E_STATE (-6)      /* call out of sequence */
#define CFG_E_SIZE (-7)       /* size beyond a fixed scratch capacity */

#define CFG_FP64 0            /* every kernel in FP64 */
#define CFG_MIXED 1           /* FP32 transforms/products/solves, FP64 mean mode */

typedef struct cfg_ctx cfg_ctx;

/* Run parameters: the runparms/gridparms scalars the hot path reads
 * (PFC/runparms.f90:20-53, PFC/gridparms.f90:26-40). */
typedef struct cfg_params {
  int nx, ny, nz, nx2, nz2;     /* flow.dat lines 10-14 */
  double re, lx, lz, beta;      /* beta in radians (PFC/setup.f90:105) */
  double dt, cfl_max;           /* PFC/setup.f90:1377-1378 */
  int fix_mass, dt_flag;        /* flow.dat lines 46-47 */
  double ctrlu, ctrlw;          /* feedback gains, flow.dat lines 5-6 */
  int precision;                /* CFG_FP64 or CFG_MIXED */
  int device;                   /* CUDA device ordinal */
} cfg_params;

/* Grid operators and wavenumbers computed by define_coordinates and
 * define_parameters (PFC/setup.f90:541-837, 1439-1466).  All pointers are
 * host arrays in reference layout; buffer and target_inflow may be NULL
 * (no fringe). */
typedef struct cfg_grid {
  const double *y;              /* (ny) */
  const double *yh;             /* (ny+1) */
  const double *hn;             /* (ny) */
  const double *dh;             /* (ny+1) */
  const double *dn;             /* (ny) */
  const double *iu;             /* (2, ny) */
  const double *dm;             /* (3, 4) */
  const double *d2h;            /* (3, ny+1) */
  const double *d2n;            /* (3, ny) */
  const double *dyh;            /* (ny+1) */
  const double *dy;             /* (ny+1) */
  const double *kx;             /* (nx/2+1) */
  const double *kz;             /* (nz) FFT order */
  const double *buffer;         /* (nx2, nz2) fringe damping, or NULL */
  const double *target_inflow;  /* (ny+1, 3) fringe target, or NULL */
} cfg_grid;

/* initialize_fft + allocate_data_arrays (PFC/transform.f90:60-160,
 * PFC/setup.f90:441-514): allocates the device state and plans. */
int cfg_create(const cfg_params *p, const cfg_grid *g, cfg_ctx **out);
/* finalize_fft + deallocate_data_arrays (PFC/transform.f90:164-191). */
void cfg_destroy(cfg_ctx *c);
const char *cfg_last_error(const cfg_ctx *c);

/* Copy data1/data2/data4 host <-> device (any pointer may be NULL). */
int cfg_upload_state(cfg_ctx *c, const double *data1, const double *data2,
                     const double *data4);
int cfg_download_state(cfg_ctx *c, double *data1, double *data2, double *data4);

/* Scalar state: t_total, dt, p_grad (runparms) and d_um_dy(ny) (gridparms).
 * d_um_dy may be NULL.  cfg_get_scalars synchronises; cfl_max (nullable)
 * returns MAXVAL(cfl(2:ny)) of the last rk_step=1 nonlinear call. */
int cfg_set_scalars(cfg_ctx *c, double t_total, double dt, double p_grad,
                    const double *d_um_dy);
int cfg_get_scalars(cfg_ctx *c, double *t_total, double *dt, double *p_grad,
                    double *d_um_dy, double *cfl_max);

/* Inhomogeneous wall values cbc_top/cbc_bot (nz, nx/2+1, 3); either may be
 * NULL.  They are read by rhs_solve exactly like the module arrays. */
int cfg_set_wall_bc(cfg_ctx *c, const double *cbc_top, const double *cbc_bot);
int cfg_get_wall_bc(cfg_ctx *c, double *cbc_top, double *cbc_bot);

/* read_write::boundary, PFC/read_write.f90:1465-1532: zeroes cbc_top/cbc_bot
 * and applies the wall-shear feedback law for nonzero ctrlu/ctrlw. */
int cfg_boundary(cfg_ctx *c);

/* pass1::nonlinear, PFC/pass1.f90:26-124: replaces the velocity in data1 by
 * the dealiased nonlinear term; on rk_step==1 computes the per-plane CFL
 * (check_cfl, :202-250) and, if dt_flag, adapts dt on the device. */
int cfg_nonlinear(cfg_ctx *c, int step, int rk_step);

/* pass1_linearized::nonlinear_linearized, PFC/pass1_linearized.f90:135-250,
 * about the baseflow set by cfg_set_baseflow (uniform in x and z). */
int cfg_nonlinear_linearized(cfg_ctx *c, int step, int rk_step);
/* Baseflow profile (ny+1, 3) for the linearized term (init_baseflow,
 * PFC/pass1_linearized.f90:20-131). */
int cfg_set_baseflow(cfg_ctx *c, const double *profile);

/* pass2::rhs_solve, PFC/pass2.f90:29-180: per-(kx,kz) RK3/Crank-Nicolson
 * substep (PHASE1 :184-352) with the Helmholtz and pressure solves of
 * PFC/solve.f90; the mean mode updates p_grad and d_um_dy on the device. */
int cfg_rhs_solve(cfg_ctx *c, int step, int rk_step);

/* The body of the timestep loop, PFC/main_mpi.f90:70-86, for nsteps steps:
 * boundary, then three (nonlinear, rhs_solve) substeps, then
 * t_total = t_total + dt.  No host synchronisation. */
int cfg_timestep(cfg_ctx *c, int nsteps);
/* Same with nonlinear_linearized (the arnoldi.f90 matvec loop, :540-547). */
int cfg_timestep_linearized(cfg_ctx *c, int nsteps);

/* arnoldi::compute_time_deriv, PFC/arnoldi.f90:485-567: the propagator
 * matvec w = Phi_T v of the Arnoldi stability solver (the OP*x step of the
 * pdnaupd reverse-communication loop, :257-300).  v and w are host vectors
 * (nx, nz, ny+1, 3) of physical velocity planes.  v is scaled by
 * eps/max|v| (eps = 1e-8) and sqrt(dyh) (u, w) or sqrt(dy) (v) weights,
 * transformed with small_fft_real_to_complex into data1 = data2, p_grad and
 * d_um_dy are zeroed, the initial pressure is computed with the linearized
 * term, tend linearized steps are taken from t_total = 0, and the result is
 * unweighted and transformed back.  Overwrites the context's state. */
int cfg_arnoldi_matvec(cfg_ctx *c, int tend, const double *v, double *w);

/* transform::xz_fft_complex_to_real / xz_fft_real_to_complex,
 * PFC/transform.f90:195-227,258-409: one plane, host arrays
 * cdata (nz, nx/2+1) complex and data (nx2, nz2) real. */
int cfg_xz_c2r(cfg_ctx *c, const double *cdata, double *data);
int cfg_xz_r2c(cfg_ctx *c, const double *data, double *cdata);
/* transform::small_fft_real_to_complex / small_fft_complex_to_real,
 * PFC/transform.f90:950-1142: nx x nz grid, no dealiasing, nplanes planes
 * (data (nx, nz, nplanes), cdata (nz, nx/2+1, nplanes)); forward scaled by
 * 1/(nx*nz).  Computed in the context's precision.  Up to about 3*(ny+1)
 * planes per call (CFG_E_ARG beyond). */
int cfg_small_r2c(cfg_ctx *c, const double *data, double *cdata, int nplanes);
int cfg_small_c2r(cfg_ctx *c, const double *cdata, double *data, int nplanes);

/* Crossflow wall forcing, the cbc_top/cbc_bot(:,:,2) slot (jet_profile,
 * PFC/pass2.f90:423-673, closed channel).  Index 0 of each pair is the
 * bottom wall, 1 the top; a wall is forced when its jetmag is nonzero
 * (:494,517).  Mode 1 is the reference's tanh jet with Freund forcing
 * (define_jet_profile, :611-656); mode 2 a Gaussian spanwise slot at x = xjet,
 * v = jetmag exp(-(d/width)^2) (1 + sin(2 pi freq t))/2, written to the same
 * slot.  Both subtract the suction profile (define_suction_profile, :553-609)
 * that balances the jet's mass flux.  The Freund parameters random-walk on
 * every call (:454-477) with RANDOM_NUMBER replaced by the counter RNG of the
 * initial field: draw n (0..23) of call k is u01(seed, k, 0, n, 7);
 * seed 0 keeps them fixed. */
typedef struct cfg_jet {
  int mode;                        /* 0 off, 1 tanh jet, 2 Gaussian slot */
  double xjet[2], zjet[2];         /* jet centre (absolute x, z) */
  double jetmag[2];                /* jet velocity (mode 2: slot peak) */
  double forcing[2], for_freq[2];  /* mode 1 amplitude modulation */
  double jet_diam;                 /* mode 1 */
  double width, freq;              /* mode 2 */
  double frac_xbuff;               /* suction band (flow.dat frac_xbuff) */
  int filter_jet_profile;          /* raised-cosine filter passes */
  double jet_forcing[24];          /* (3,2,4) Freund A, St, phi, psi */
  double jet_forcing_incr[24];     /* (3,2,4) their random-walk increments */
  unsigned long long seed;         /* random-walk seed, 0: fixed parameters */
} cfg_jet;
/* crossflow = 1 (jet != NULL, mode != 0): every cfg_rhs_solve / cfg_timestep
 * substep first calls jet_profile with the end-of-substep time
 * t_total + dt*SUM(rkc(1:rk)+rkd(1:rk)) and increment dt*(rkc(rk)+rkd(rk))
 * (PFC/pass2.f90:37-44), from the device-resident t_total and dt.  Resets
 * the forcing parameters and the call counter.  NULL: crossflow = 0. */
int cfg_set_jet(cfg_ctx *c, const cfg_jet *jet);
/* pass2::jet_profile(time, time_incr, ctop, cbot) with host-given time:
 * random walk, then cbc_top/cbc_bot(:,:,2).  Needs cfg_set_jet. */
int cfg_jet_profile(cfg_ctx *c, double time, double time_incr);
/* The current forcing parameters and increments (24 each; NULL skips). */
int cfg_get_jet_forcing(cfg_ctx *c, double *jet_forcing, double *jet_forcing_incr);

/* Fringe (buffer) region, init_buffer (PFC/init_jet_buffer.f90:358-483),
 * computed on the device: the nx x nz profile (define_fringe_region ramps
 * in x and, with zfringe, at both z ends), transformed with
 * small_fft_real_to_complex and interpolated onto the dealiased nx2 x nz2
 * grid with xz_fft_complex_to_real, times fringe_gain; target_inflow
 * (ny+1, 3) = 0.75 (1 - yh^8) (cos beta, 0, sin beta) of the closed
 * channel.  The nonlinear step then adds buffer*(u - target) (pass1.f90).
 * xfringe = zfringe = 0 switches the fringe off. */
typedef struct cfg_fringe {
  double fringe_gain;
  int xfringe, zfringe;
  double frac_xbuff, buff_xrise, buff_xfall;   /* x band: last frac_xbuff of lx */
  double frac_zbuff;                           /* z bands at both ends */
} cfg_fringe;
int cfg_init_buffer(cfg_ctx *c, const cfg_fringe *f);
/* The device's buffer (nx2, nz2) and target_inflow (ny+1, 3); NULL skips. */
int cfg_get_buffer(cfg_ctx *c, double *buffer, double *target_inflow);

/* read_write::l2_norm, PFC/read_write.f90:1432-1462: perturbation L2 norm
 * about U=1-y^2 and the wall-shear difference d_um_dy(1)-d_um_dy(ny). */
int cfg_l2_norm(cfg_ctx *c, double *l2, double *drag);

/* init_vel: remove_initial_divergence (PFC/init_vel.f90:518-536) followed by
 * the d_um_dy initialisation (:333-342) and data2 = data1 (:344-348). */
int cfg_remove_initial_divergence(cfg_ctx *c);
/* init_vel::compute_initial_pressure (PFC/init_vel.f90:437-514); linearized
 * selects nonlinear_linearized as in arnoldi.f90:528-535. */
int cfg_compute_initial_pressure(cfg_ctx *c, int linearized);

/* Output that does not stall the step.  Each call converts the device state
 * to the file's order with one kernel on the context stream, copies it to
 * pinned host memory on a second stream and writes the file on a host thread;
 * it returns at once and later steps may be issued meanwhile.  At most one
 * write is in flight: the next output call (or cfg_wait_io) waits for it.
 * cfg_wait_io returns that write's status (CFG_E_ARG with the message in
 * cfg_last_error on an I/O failure).  cfg_destroy waits too.
 *
 * read_write::save_velocity (PFC/read_write.f90:211-292): the restart file
 * (Fortran unformatted sequential: header NX, NY, NZ, LX, LZ, RE, DT,
 * T_TOTAL; one record per kx with data1(1:nz, kx, 1:ny+1, 1:3); a closing
 * record 0, 0), DT and T_TOTAL taken at the call. */
int cfg_save_velocity(cfg_ctx *c, const char *path);
/* read_write::output_hdf_dfsd's VTK snapshot (PFC/read_write.f90:296-500,
 * xskip = yskip = zskip = 1): u, v, w on the nx x (ny+1) x nz grid of
 * (x, yh, z) points -- v averaged onto yh, small_fft_complex_to_real per
 * plane -- as a legacy binary big-endian float32 rectilinear grid. */
int cfg_write_vtk(cfg_ctx *c, const char *path);
/* Post-processing on the same grid (x, yh, z): the velocity-gradient tensor
 * A_ij = du_i/dx_j (x and z derivatives spectral, y by 3-point Lagrange
 * differences on yh -- the stencils of PFC/stats.f90's setup_diff), the
 * vorticity, the Q-criterion -tr(A^2)/2 and the discriminant
 * D = (6 (tr A^3)^2 - (tr A^2)^3)/8 of the ParaView Calculator in
 * ParaView-Code/DiscriminantFilter.cpd:17, computed on the device and
 * written behind the velocity as VECTORS vorticity, SCALARS Q and SCALARS D
 * (background write, as cfg_write_vtk). */
int cfg_write_vtk_derived(cfg_ctx *c, const char *path);
/* Per-plane moments of one snapshot (compute_velocity_moments and
 * compute_vorticity_moments, PFC/stats.f90:423-456, with weight 1): stats is
 * (ny+1, 27) column-major: mean u, v, w; variance; skewness m3/(m2^1.5+eps);
 * flatness m4/(m2^2+eps); the fluxes <u'v'>, <v'v'>, <w'v'>; then mean,
 * variance, skewness and flatness of the three vorticity components, on the
 * planes yh(1..ny+1).  Synchronous. */
int cfg_plane_statistics(cfg_ctx *c, double *stats);
int cfg_wait_io(cfg_ctx *c);
/* read_write::read_velocity (PFC/read_write.f90:21-209): checks NX, NY, NZ,
 * LX, LZ against the context (CFG_E_ARG with the reference's message),
 * reports a changed RE on stderr, uploads data1 and sets t_total (and dt
 * when dt_flag).  The caller then removes the divergence and computes the
 * initial pressure as define_initial_field does.  Synchronous. */
int cfg_read_velocity(cfg_ctx *c, const char *path);

/* Bulk flux Q = sum dyh*Re(u_mean) (PFC/pass2.f90:106-108) and the maximum
 * |divergence| over all wavenumbers (check_divergence, :380-419). */
int cfg_diagnostics(cfg_ctx *c, double *bulk_flux, double *max_divergence);

/* Device error flag: 0, CFG_E_CFL or CFG_E_DT.  Synchronises. */
int cfg_status(cfg_ctx *c);
int cfg_synchronize(cfg_ctx *c);

/* The CUDA stream (cudaStream_t) every call of this context is issued on,
 * for callers that order their own work or timing events against it. */
void *cfg_stream(cfg_ctx *c);

/* Number of kernel launches this context has issued (for accounting). */
long long cfg_launch_count(const cfg_ctx *c);

/* Per-kernel timing with CUDA events recorded on the context's stream around
 * each hot-path launch.  cfg_profile_enable(c, 1) clears and starts the
 * record; cfg_profile_read(c, -1, ...) returns the number of distinct
 * kernels, cfg_profile_read(c, i, name, len, &launches, &ms) the i-th one's
 * launch count and summed device time.  Both synchronise. */
int cfg_profile_enable(cfg_ctx *c, int on);
int cfg_profile_read(cfg_ctx *c, int idx, char *name, int namelen, int *launches,
                     double *total_ms);

/* ---- multi-rank runs (slab decomposition of one field) ----------------
 *
 * distribute_data (PFC/setup.f90:298-437): the split of the nx/2+1 Fourier
 * columns (nx_proc, x_start), of the nz2 physical z rows (nz_proc, z_start)
 * and of the nz undealiased z rows (nz_small_proc, z_small_start) among
 * nproc ranks -- the first (n mod nproc) ranks take one more.  Each output
 * array has nproc entries; any may be NULL. */
int cfg_partition(int nx, int nz, int nz2, int nproc, int *nx_proc, int *x_start,
                  int *nz_proc, int *z_start, int *nz_small_proc, int *z_small_start);

/* A group of nranks contexts that advance one field together, rank i owning
 * the Fourier columns [x_start[i], x_start[i] + nx_proc[i]) of the state and
 * the z2 rows [z_start[i], ...) of the physical planes, as the reference's
 * MPI ranks do (PFC/main_mpi.f90 under mpirun).  It replaces the MPI
 * decomposition of pass1::nonlinear: the two MPI_ALLTOALLV transposes of
 * the x-z transforms (PFC/transform.f90:345-409, 573-690) become stores of
 * the z and flux kernels straight into the owning rank's buffers (peer
 * memory when the ranks are on different GPUs, peer access enabled here),
 * and the CFL MPI_ALLREDUCE (PFC/pass1.f90:202-250) a fold of the other
 * ranks' per-plane maxima.  devices[i] is rank i's GPU (NULL: p->device
 * for all; ranks may share a GPU).  Each rank needs >= 1 kx column and a
 * multiple of 8 z2 rows; ctrlu = ctrlw = 0 (the wall feedback transforms
 * whole planes).  cfg_group_rank gives rank i's context for
 * cfg_upload_state / cfg_download_state (arrays of the rank's local sizes,
 * data1(nz, nx_proc[i], ny+1, 3) as in PFC/setup.f90:447-449),
 * cfg_set_scalars, cfg_get_scalars, cfg_set_wall_bc, cfg_rhs_solve,
 * cfg_status; entry points that need whole planes return CFG_E_ARG on a
 * rank of a group of two or more. */
typedef struct cfg_group cfg_group;
int cfg_group_create(const cfg_params *p, const cfg_grid *g, int nranks, const int *devices,
                     cfg_group **out);
int cfg_group_size(const cfg_group *grp);
cfg_ctx *cfg_group_rank(cfg_group *grp, int rank);
/* timestep (PFC/main_mpi.f90:55-116) of all ranks: per RK substep the
 * inverse z transforms, a barrier, the x stages, a barrier, the forward z
 * transforms and rhs_solve.  Asynchronous. */
int cfg_group_timestep(cfg_group *grp, int nsteps);
int cfg_group_synchronize(cfg_group *grp);
void cfg_group_destroy(cfg_group *grp);

/* The same decomposition with one process per rank (one per GPU, as the
 * reference runs under mpirun; PFC/setup.f90:298-437 in each process).
 * cfg_rank_create makes rank `rank`'s context (its slabs, on p->device);
 * cfg_rank_export writes a record of cfg_rank_record_size() bytes (CUDA IPC
 * handles of the rank's transpose targets and CFL maxima, its slabs); the
 * caller all-gathers the nranks records in rank order (MPI_ALLGATHER,
 * torch.distributed) and passes them to cfg_rank_connect, which maps the
 * other ranks' buffers (once per context; CFG_E_STATE after that).
 * cfg_rank_timestep then advances this rank; between
 * the phases of each substep it completes its own stores and calls
 * barrier(user), which must return 0 once every rank has called it
 * (MPI_BARRIER) -- the exchange of the MPI_ALLTOALLV transposes of
 * PFC/transform.f90:345-409, 573-690.  Same limits as cfg_group_create. */
typedef int (*cfg_barrier_fn)(void *user);
size_t cfg_rank_record_size(void);
int cfg_rank_create(const cfg_params *p, const cfg_grid *g, int rank, int nranks, cfg_ctx **out);
int cfg_rank_export(cfg_ctx *c, void *record);
int cfg_rank_connect(cfg_ctx *c, const void *records);
int cfg_rank_timestep(cfg_ctx *c, int nsteps, cfg_barrier_fn barrier, void *user);
/* The same without the host synchronisation: barrier(user) must enqueue a
 * barrier on this context's stream (cfg_stream) that completes only after
 * every rank's stream has reached it -- e.g. an NCCL all-reduce of one word
 * on that stream -- so the host never waits between the phases. */
int cfg_rank_timestep_ordered(cfg_ctx *c, int nsteps, cfg_barrier_fn barrier, void *user);

/* ---- launch shapes and ensembles (no counterpart in the reference) -----
 *
 * cfg_autotune: times trial_steps steps of this context's own state per
 * candidate tile setting -- warps per rhs block, z rows per flux block,
 * planes per z-transform block, one parameter at a time -- keeps the fastest
 * and restores the state, scalars, wall values and jet walk afterwards.
 * Results do not depend on the tiles (bit for bit).  choice (nullable, 4
 * ints) receives the tiles; cfg_set_tiles sets them directly. */
int cfg_autotune(cfg_ctx *c, int trial_steps, int *choice);
int cfg_set_tiles(cfg_ctx *c, const int *tiles);
int cfg_get_tiles(const cfg_ctx *c, int *tiles);   /* the current 4 tiles */

/* An ensemble of independent contexts on one GPU (different grids,
 * Reynolds numbers, seeds, forcing): members of one run of the reference
 * each, advanced together.  cfg_ensemble_timestep runs the first step
 * eagerly and captures one step of the ensemble into a CUDA graph; every
 * further step is one graph launch on the ensemble's stream.  autotune != 0
 * tunes the tiles once per distinct grid.  The members stay owned by the
 * caller and must outlive the ensemble; call cfg_ensemble_synchronize before
 * reading or changing a member, and do not change a member's parameters
 * (jet, baseflow, fringe, tiles) once the ensemble has stepped (the graph
 * and the member tables hold them).
 *
 * Step layout.  Batched (the default when every member allows it: mixed
 * precision, one rank, the register-FFT transforms with the v2 rhs kernel,
 * no LES, no wall feedback): the members fall into classes of the same grid
 * and tiles, and every kernel of the step runs once per class over a table
 * of the members' arguments in device memory.  Otherwise, or after
 * cfg_ensemble_set_batched(e, 0): one graph branch per member.  The results
 * are the same bit for bit.  cfg_ensemble_set_batched(e, 1) returns
 * CFG_E_ARG when a member does not allow it; cfg_ensemble_batched tells the
 * current layout. */
typedef struct cfg_ensemble cfg_ensemble;
int cfg_ensemble_create(int nmembers, cfg_ctx *const *members, int autotune, cfg_ensemble **out);
int cfg_ensemble_timestep(cfg_ensemble *e, int nsteps);
int cfg_ensemble_synchronize(cfg_ensemble *e);
void *cfg_ensemble_stream(cfg_ensemble *e);
int cfg_ensemble_set_batched(cfg_ensemble *e, int on);
int cfg_ensemble_batched(const cfg_ensemble *e);
void cfg_ensemble_destroy(cfg_ensemble *e);

/* Learned subgrid-stress closure network (the LES mode of the reference's
 * subgrid = 1 runs, PFC/main_mpi.f90:10-13,74-78, whose modules are not in
 * the reference): a perceptron 10 -> 64 -> 64 -> 64 -> 6 with GELU (tanh
 * form, hardware tanh) on the hidden layers, BF16 weights and activations
 * and FP32 accumulation on the sm_100 tensor cores (tcgen05, accumulators in
 * tensor memory).  Inputs per
 * point: the 9 resolved velocity-gradient components and the wall distance,
 * normalised by the caller; outputs: the 6 subgrid-stress components
 * (11, 22, 33, 12, 13, 23), normalised.
 *
 * Parameters: cfg_mlp_nparams() FP32 values, W0[64][10] b0[64] W1[64][64]
 * b1[64] W2[64][64] b2[64] W3[6][64] b3[6] (y = W x + b per layer).
 * cfg_mlp_set_params also clears the gradient and the Adam moments.
 *
 * cfg_mlp_forward: x device [n][10] FP32 -> y device [n][6] FP32, on stream.
 * cfg_mlp_accumulate_grad: one batch of training samples, rows idx[0..batch)
 *   of x [.][10] and targets t [.][6] (device): adds the gradient of the
 *   mean-square loss (mean over batch x 6) and the loss itself to the
 *   network's accumulators, summed in a fixed order (the same bits on every
 *   run); calls on one network run in stream order, since they share its
 *   per-tile gradient buffer, which grows (cudaFree, cudaMalloc) the first
 *   time a batch exceeds 65536 rows.  cfg_mlp_get_grads copies them to the host
 *   (synchronises); cfg_mlp_adam_step applies one Adam update (bias
 *   corrected) from them and clears them; cfg_mlp_zero_grads clears them.
 * cfg_mlp_status: CFG_E_STATE if a kernel gave up waiting for the tensor
 *   cores (a bounded wait), else CFG_OK.  Needs an sm_100 device
 *   (CFG_E_ARG otherwise). */
typedef struct cfg_mlp cfg_mlp;
int cfg_mlp_nparams(void);
int cfg_mlp_create(int device, cfg_mlp **out);
void cfg_mlp_destroy(cfg_mlp *m);
int cfg_mlp_set_params(cfg_mlp *m, const float *params);
int cfg_mlp_get_params(cfg_mlp *m, float *params);
int cfg_mlp_forward(cfg_mlp *m, const float *x, float *y, long long n, void *stream);
int cfg_mlp_accumulate_grad(cfg_mlp *m, const float *x, const float *t, const int *idx, int batch, void *stream);
int cfg_mlp_get_grads(cfg_mlp *m, float *grads, float *loss);
int cfg_mlp_zero_grads(cfg_mlp *m, void *stream);
int cfg_mlp_adam_step(cfg_mlp *m, float lr, float beta1, float beta2, float eps, void *stream);
int cfg_mlp_status(cfg_mlp *m);

/* LES mode (the reference's subgrid = 1 branch, PFC/main_mpi.f90:74-78; its
 * model modules are not in the reference): subgrid stresses added to the
 * momentum fluxes of every nonlinear step.
 *   model 1: eddy viscosity, Smagorinsky constant cs with van Driest damping
 *     (1 - exp(-y+/aplus)), filter width (lx/nx * dy * lz/nz)^(1/3), u_tau
 *     from the mean wall shear;
 *   model 2: the learned closure (mlp, cfg_mlp_*) on the features
 *     (G_ij = du_i/dx_j row by row and 1 - |y|, in the lower half-channel's
 *     frame) normalised as (f - in_shift) / in_scale, its outputs mapped as
 *     out_shift + out_scale * y; it falls back to model 1 at every point whose
 *     stress tensor is not realizable or whose backscatter -tau:S is below
 *     -beta times the eddy viscosity's dissipation.
 * Needs the register-FFT x stage and one rank (CFG_E_ARG otherwise).  The
 * network stays owned by the caller and must outlive the context's steps.
 * cfg_les_features writes the model-2 features of the current state
 * (device, [(ny-1) * nz2 * nx2][10], planes 2..ny, z2, x2 fastest) without a
 * step; cfg_les_fallbacks returns the fallback count since cfg_set_les and
 * the points per substep (synchronises); cfg_les_stresses below. */
typedef struct cfg_les {
  int model;
  double cs, aplus, beta;
  cfg_mlp *mlp;
  float in_shift[10], in_scale[10], out_shift[6], out_scale[6];
} cfg_les;
int cfg_set_les(cfg_ctx *c, const cfg_les *les);
int cfg_les_features(cfg_ctx *c, float *features);
int cfg_les_fallbacks(cfg_ctx *c, unsigned long long *fallbacks, unsigned long long *points);
/* the subgrid stresses of the last nonlinear step (or cfg_les_features
 * call), host [ny+1][6][nz2][nx2] FP64, yh planes 1..ny+1, components 11,
 * 22, 33, 12, 13, 23 (synchronises) */
int cfg_les_stresses(cfg_ctx *c, double *S);

/* cfg_xz_c2r_noalloc -- no counterpart in the reference.  The inverse x-z
 * transform of one plane (the semantics of cfg_xz_c2r /
 * xz_fft_complex_to_real) for callers that cannot allocate device memory:
 * hosts whose device memory is pre-assigned at start-up by another owner (a
 * framework's caching allocator, a communication library's registered
 * buffers), where one more cudaMalloc would fail or fragment that pool, and
 * step loops that cannot take the device-wide synchronisation that
 * cudaMalloc/cudaFree imply.  It allocates nothing and needs no context.
 *
 *   cdata  device pointer, (nz, nx/2+1) complex FP64 (interleaved re, im)
 *   data   device pointer, (nx2, nz2) real FP64 (written)
 *   stream cudaStream_t to run on (NULL: the legacy default stream)
 *
 * Its intermediate plane and twiddle tables live in one fixed file-scope
 * device array of 4.06 MiB that every GPU loading the library holds until
 * exit.  Limits: (nx/2+1)*nz2 <= 262144 and nx2, nz2 <= 2048 (2^a 3^b, even);
 * larger planes return CFG_E_SIZE.  Every call shares that array and it keeps
 * the previous call's contents: each call rewrites the intermediate plane it
 * reads (nothing must start at zero), and the twiddle tables are rewritten
 * only when nx2 or nz2 differs from the previous call's on that device.  So
 * calls whose executions overlap on the GPU -- other streams, other host
 * threads -- race; serialise them.  The kernels' shared-memory limits are
 * only ever raised, never lowered.  The first call on a
 * device performs a one-time set-up (it looks up the array's device address
 * with that device current); make that first call before any stream capture.
 * Returns CFG_OK, CFG_E_ARG, CFG_E_SIZE or CFG_E_CUDA. */
int cfg_xz_c2r_noalloc(int nx, int nz, int nx2, int nz2, const double *cdata,
                       double *data, void *stream);

#ifdef __cplusplus
}
#endif
#endif
