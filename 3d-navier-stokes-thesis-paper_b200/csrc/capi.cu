// capi.cu -- the C ABI of include/chanflow.h: device state, plans, kernel
// orchestration for one channel-flow context on one B200.
//
// Sections, in order: layout-conversion kernels (Fortran arrays <-> device
// state); the context (cfg_ctx) and its per-launch timing; Impl<T>, the
// step's orchestration per precision (set-up, the three nonlinear phases,
// the rhs solve with its side streams, plane transforms, jet, boundary,
// l2); the entry points of one context (create, state, step, transforms,
// diagnostics, Arnoldi matvec); background file output and
// post-processing; the fringe; multi-rank runs (partition, one-process
// groups, one process per rank); the launch-shape autotuner; ensembles
// stepped by CUDA graphs.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "chanflow.h"
#include "pass1.cuh"
#include "pass2.cuh"
#include "pass1_fast.h"
#include "arnoldi.cuh"
#include "io.cuh"
#include "jet.cuh"
#include "les.cuh"
#include "mlp_les.h"
#include "pass2v2.h"
#include "planes.cuh"
#include "restart.h"
#include "regfft.cuh"

using namespace cfd;

// ----------------------------------------------------------------------------
// layout conversion kernels between the reference's Fortran arrays (FP64) and
// the device state ([kx][kz][comp][y], precision T)
template <typename T>
__global__ void k_data1_in(const double2* __restrict__ src, cplx_t<T>* __restrict__ vel,
                           double2* __restrict__ mvel64, Geom g) {
  // src (nz, nxh, ny+1, 3): element (z, x, j, c) at z + nz*(x + nxh*(j + ny1*c))
  const size_t n = (size_t)g.nw * 3 * g.ny1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(i % g.ny1);
    const int c = (int)((i / g.ny1) % 3);
    const size_t w = i / ((size_t)3 * g.ny1);
    const double2 v = src[w + (size_t)g.nw * (j + (size_t)g.ny1 * c)];
    vel[i] = mk<cplx_t<T>>((T)v.x, (T)v.y);
    if (mvel64 && w == 0) mvel64[c * g.ny1 + j] = v;
  }
}
template <typename T>
__global__ void k_data1_out(const cplx_t<T>* __restrict__ vel, const double2* __restrict__ mvel64,
                            double2* __restrict__ dst, Geom g) {
  const size_t n = (size_t)g.nw * 3 * g.ny1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(i % g.ny1);
    const int c = (int)((i / g.ny1) % 3);
    const size_t w = i / ((size_t)3 * g.ny1);
    double2 v;
    if (mvel64 && w == 0) v = mvel64[c * g.ny1 + j];
    else { const cplx_t<T> s = vel[i]; v = make_double2((double)s.x, (double)s.y); }
    dst[w + (size_t)g.nw * (j + (size_t)g.ny1 * c)] = v;
  }
}
template <typename T>
__global__ void k_conv_in(const double2* __restrict__ src, cplx_t<T>* __restrict__ dst, size_t n,
                          double2* __restrict__ side, size_t nside) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = src[i];
    dst[i] = mk<cplx_t<T>>((T)v.x, (T)v.y);
    if (side && i < nside) side[i] = v;
  }
}
template <typename T>
__global__ void k_conv_out(const cplx_t<T>* __restrict__ src, double2* __restrict__ dst, size_t n,
                           const double2* __restrict__ side, size_t nside) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if (side && i < nside) dst[i] = side[i];
    else { const cplx_t<T> s = src[i]; dst[i] = make_double2((double)s.x, (double)s.y); }
  }
}
template <typename T>
__global__ void k_real_in(const double* __restrict__ src, T* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) dst[i] = (T)src[i];
}
template <typename T>
__global__ void k_real_out(const T* __restrict__ src, double* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) dst[i] = (double)src[i];
}
__global__ void k_advance_time(DevScalars* sc) { sc->t_total = sc->t_total + sc->dt; }

// max |divergence| (check_divergence, PFC/pass2.f90:380-419), warp per wavenumber
template <typename T>
__global__ void k_divergence(const cplx_t<T>* __restrict__ vel, Geom g, GridDev gd,
                             unsigned long long* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= g.nw) return;
  const int n1 = g.ny1, ny = g.ny;
  const double kx = gd.kx[w / g.nz], kz = gd.kz[w % g.nz];
  const cplx_t<T>* c = vel + (size_t)w * 3 * n1;
  double m = 0;
  for (int j = 1 + lane; j <= ny - 1; j += 32) {
    const double dvx = gd.dh[j] * ((double)c[n1 + j].x - (double)c[n1 + j - 1].x);
    const double dvy = gd.dh[j] * ((double)c[n1 + j].y - (double)c[n1 + j - 1].y);
    const double re = -kx * (double)c[j].y + dvx - kz * (double)c[2 * n1 + j].y;
    const double im = kx * (double)c[j].x + dvy + kz * (double)c[2 * n1 + j].x;
    m = fmax(m, sqrt(re * re + im * im));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// ----------------------------------------------------------------------------
struct cfg_ctx {
  cfg_params p{};
  Geom g{};
  bool mixed = false;
  int dev = 0;
  cudaStream_t st = nullptr;
  // side stream: the small mean-mode and FP64 low-|k| solves run beside the
  // main per-wavenumber kernel; joined back with events
  cudaStream_t st2 = nullptr, st3 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join3 = nullptr;
  // background file output (restart file, VTK snapshot): the layout kernel
  // runs on st, the copy to pinned host memory on st_io, the file write on
  // io_thread
  cudaStream_t st_io = nullptr;
  cudaEvent_t ev_io_start = nullptr, ev_io_done = nullptr;
  void* io_dev = nullptr;
  void* io_host = nullptr;
  size_t io_bytes = 0;
  DevScalars* sc_snap = nullptr;   // device copy of the scalars at the snapshot
  DevScalars* sc_host = nullptr;   // pinned
  std::thread io_thread;
  int io_status = 0;
  std::string io_err;
  std::vector<double> hyh;
  // post-processing: y-derivative weights/stencils on yh, per-plane sums
  double* pp_wy = nullptr;
  int* pp_sy = nullptr;
  double* pp_acc = nullptr;
  cudaStream_t prof_stream = nullptr;
  std::string err;
  long long launches = 0;
  int step = 0;
  // grid
  double* dgrid = nullptr;
  GridDev gd{};
  void* fringe = nullptr;
  int has_fringe = 0;
  // state
  void *vel = nullptr, *cru = nullptr, *prs = nullptr;
  double2 *mvel64 = nullptr, *mcru64 = nullptr;
  void *T1 = nullptr, *T2 = nullptr;
  // physical planes of the split x stage (k_xinv_r -> k_flux_r)
  void* P = nullptr;
  bool split_x = false;
  int flux_zr = 4;
  void* cbc = nullptr;   // [bot, top][3][nw]
  DevScalars* sc = nullptr;
  double* d_um_dy = nullptr;
  double* cflp = nullptr;
  unsigned long long* cflbits = nullptr;
  double* l2acc = nullptr;
  unsigned long long* divbits = nullptr;
  // lane-major grid coefficients of k_rhs2 (storage precision, rhs2_lanes
  // lanes) and in FP64 for 32 lanes (the FP64 list and the mean mode)
  void* rhs2_tbl = nullptr;
  void* rhs2_tbl64 = nullptr;
  // crossflow jet (cfg_set_jet): parameters, device walk state
  bool crossflow = false;
  JetParams jp{};
  JetState* jst = nullptr;
  int* plist = nullptr;
  // plane work buffers
  void *pw_H = nullptr, *pw_phys = nullptr, *pw_phys2 = nullptr, *pw_in = nullptr;
  size_t pw_planes = 0;
  // staging for FP64 host <-> device conversion
  double2* stage = nullptr;
  size_t stage_elems = 0;
  // twiddles and plans
  void *twx = nullptr, *twz = nullptr, *twxs = nullptr, *twzs = nullptr;
  FftPlan px{}, pz{}, pxs{}, pzs{};
  // launch shapes
  int YB1 = 1, YB3 = 1, ZR = 1, KC = 4, M = 2;
  size_t sm_zinv = 0, sm_xflux = 0, sm_zfwd = 0, sm_rhs = 0;
  RkTab rkt{};
  double hdm[12] = {0};
  std::vector<double> hdy;
  // mixed precision: whether mvel64 holds the current data1 mean column (it
  // does not while data1 holds the nonlinear term)
  bool mean64_valid = true;
  // wavenumber lists for the rhs kernels: fast (arithmetic in the storage
  // precision) and, in mixed precision, |k| < 4 solved in FP64
  int* wl_fast = nullptr;
  int* wl_prec = nullptr;
  int n_fast = 0, n_prec = 0;
  size_t sm_rhs64 = 0;
  // register-FFT pass-1 kernels (when the lengths are compiled in)
  bool fast_z = false, fast_x = false;
  bool use_rhs2 = true;
  int rhs2_lanes = 32;
  int rhs2_warps = 3;   // warps (wavenumbers) per k_rhs2 block
  int fYB1 = 1, fYB3 = 1, fZR = 1;
  int xinv_zb = 0;      // z2 rows per k_xinv_r block (0: 16 in FP32, 8 in FP64), tuned
  // optional per-launch CUDA-event timing on the context stream
  bool prof_on = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  struct Rec { const char* name; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  const char* cur_name = nullptr;
  cudaEvent_t cur_a = nullptr;
  // rank of a multi-rank run (cfg_group): kx slab [g.kx0, g.kx0 + g.nxh) in
  // Fourier space, z2 slab [z0s, z0s + gP.nz2) in physical space
  // (distribute_data, PFC/setup.f90:298-437)
  int rank = 0, nranks = 1, z0s = 0;
  Geom gP{};              // geometry of the x stage: all kx, this rank's z2 rows
  GridDev gd_all{};       // grid operators with the global kx table
  Scatter scat{};         // transpose targets (n == 0: one rank)
  void* scat_tab = nullptr;
  unsigned long long** cfl_peers = nullptr;   // the other ranks' cflbits
  int n_cfl_peers = 0;
  std::vector<void*> ipc_open;   // other processes' buffers mapped by cfg_rank_connect
  // LES mode (cfg_set_les): subgrid stresses S[ny+1][6][nz2][nx2] (storage
  // precision) added by the flux kernel; the learned closure's features and
  // outputs (FP32) and its fallback counter
  // mean split of the mixed path's nonlinear products (k_zinv_r drops the
  // mean column, k_flux_r adds its products from mean_base, FP64 (ny+1, 3))
  bool mean_split = false;
  double* mean_base = nullptr;
  bool les_on = false;
  LesDev les{};
  cfg_mlp* les_mlp = nullptr;
  void* les_S = nullptr;
  float* les_F = nullptr;
  double* les_len = nullptr;   // the eddy viscosity's length per plane (model 2)
  unsigned long long* les_nfall = nullptr;
  unsigned long long les_points = 0;
};

// slab of one rank (cfg_group_create); one rank: the whole grid
struct SlabPart {
  int rank, nranks, x0, nxl, z0, nzl;
};

static cudaEvent_t prof_event(cfg_ctx* c) {
  if (c->ev_used == c->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c->ev_pool.push_back(e);
  }
  return c->ev_pool[c->ev_used++];
}
static void prof_begin(cfg_ctx* c, const char* name) {
  if (!c->prof_on) return;
  c->cur_name = name;
  c->cur_a = prof_event(c);
  cudaEventRecord(c->cur_a, c->prof_stream ? c->prof_stream : c->st);
}
static void prof_end(cfg_ctx* c) {
  if (!c->prof_on || !c->cur_name) return;
  cudaEvent_t b = prof_event(c);
  cudaEventRecord(b, c->prof_stream ? c->prof_stream : c->st);
  c->recs.push_back({c->cur_name, c->cur_a, b});
  c->cur_name = nullptr;
}

static int fail(cfg_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}
#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) return fail(c, CFG_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)
#define CKL()                                                                            \
  do {                                                                                   \
    c->launches++;                                                                       \
    prof_end(c);                                                                         \
    cudaError_t e_ = cudaGetLastError();                                                 \
    if (e_ != cudaSuccess) return fail(c, CFG_E_CUDA, "launch: %s", cudaGetErrorString(e_)); \
  } while (0)

static bool make_plan(int n, FftPlan& p) {
  memset(&p, 0, sizeof(p));
  p.n = n;
  int m = n, k = 0;
  while (m % 8 == 0) { p.radix[k++] = 8; m /= 8; }
  while (m % 4 == 0) { p.radix[k++] = 4; m /= 4; }
  while (m % 2 == 0) { p.radix[k++] = 2; m /= 2; }
  while (m % 3 == 0) { p.radix[k++] = 3; m /= 3; }
  if (m != 1 || k > 16) return false;
  p.npass = k;
  int ns = 1;
  for (int q = 0; q < k; ++q) { p.ns[q] = ns; ns *= p.radix[q]; }
  return true;
}

template <typename T>
static void* make_twiddles(int n) {
  std::vector<cplx_t<T>> h(n);
  for (int m = 0; m < n; ++m) {
    const double a = -2.0 * M_PI * (double)m / (double)n;
    h[m].x = (T)cos(a);
    h[m].y = (T)sin(a);
  }
  void* d = nullptr;
  if (cudaMalloc(&d, sizeof(cplx_t<T>) * n) != cudaSuccess) return nullptr;
  cudaMemcpy(d, h.data(), sizeof(cplx_t<T>) * n, cudaMemcpyHostToDevice);
  return d;
}

static dim3 grid1d(size_t n, int bs = 256) {
  size_t b = (n + bs - 1) / bs;
  if (b > 148 * 32) b = 148 * 32;
  if (b < 1) b = 1;
  return dim3((unsigned)b);
}

// ----------------------------------------------------------------------------
// global CFL maxima of a multi-rank run: each rank folds the other ranks'
// per-plane maxima (peer memory) into its own before k_cfl_finalize, so that
// every rank takes the same dt (the MPI_ALLREDUCE of check_cfl,
// PFC/pass1.f90:202-250).  Values are non-negative doubles as bit patterns.
__global__ void k_cfl_merge(unsigned long long* __restrict__ own, unsigned long long* const* __restrict__ peers,
                            int npeers, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned long long m = own[i];
    for (int r = 0; r < npeers; ++r) {
      const unsigned long long v = *((volatile const unsigned long long*)peers[r] + i);
      m = v > m ? v : m;
    }
    own[i] = m;
  }
}

// Lets a kernel take as much dynamic shared memory as the device allows.
// The limit is an attribute of the kernel on its device, shared by every
// context there, so contexts only ever raise it (to the device maximum) and
// never lower it under another context's launches.
template <typename K>
static cudaError_t allow_smem(K kernel) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  cudaFuncAttributes fa;
  if ((e = cudaFuncGetAttributes(&fa, kernel)) != cudaSuccess) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

// the real parts of the mean column (kx = kz = 0) of the velocity as the
// (ny+1, 3) FP64 profile the mean-split flux kernel reads: from the FP64 side
// copy m64 when given, else from the FP32 state
__global__ void k_mean_base(const double2* __restrict__ m64, const float2* __restrict__ v32, double* __restrict__ base,
                            int ny1) {
  for (int i = threadIdx.x; i < 3 * ny1; i += blockDim.x) base[i] = m64 ? m64[i].x : (double)v32[i].x;
}

template <typename T>
struct Impl {
  using C = cplx_t<T>;

  static int setup(cfg_ctx* c) {
    const Geom& g = c->g;
    const size_t cs = sizeof(C);
    const size_t budget = 110 * 1024;
    c->YB1 = (int)std::max<size_t>(1, std::min<size_t>(8, (budget / cs / g.nz2 - 1) / 6));
    c->YB3 = (int)std::max<size_t>(1, std::min<size_t>(8, (budget / cs / g.nz2 - 1) / 12));
    c->sm_zinv = cs * (g.nz2 + 6 * c->YB1 * g.nz2);
    c->sm_zfwd = cs * (g.nz2 + 12 * c->YB3 * g.nz2);
    auto xsm = [&](int zr) {
      const int nseq = 4 * zr + (zr + 1) / 2;
      return cs * g.nx2 + sizeof(T) * 9 * zr * g.nx2 + 2 * cs * nseq * g.nx2;
    };
    c->ZR = 1;
    for (int zr : {4, 2}) if (g.nz2 % zr == 0 && xsm(zr) <= budget) { c->ZR = zr; break; }
    c->sm_xflux = xsm(c->ZR);
    long kc = (long)(g.ny - 1) * (g.nz2 / c->ZR) / 592;
    c->KC = (int)std::max(2L, std::min(16L, kc));
    c->M = (g.ny1 + 31) / 32;
    if (c->M < 2) c->M = 2;
    if (c->M > 8) return fail(c, CFG_E_ARG, "ny+1 = %d exceeds 256 rows", g.ny1);
    if (c->sm_zinv > 200 * 1024 || c->sm_zfwd > 200 * 1024 || c->sm_xflux > 200 * 1024)
      return fail(c, CFG_E_ARG, "transform lengths too large for shared memory");
    CK(allow_smem(k_zinv<T>));
    CK(allow_smem(k_zfwd<T>));
    CK(allow_smem(k_xflux<T, false>));
    CK(allow_smem(k_xflux<T, true>));
    CK(allow_smem(k_pz_inv<T>));
    CK(allow_smem(k_pz_fwd<T>));
    CK(allow_smem(k_px_inv<T>));
    CK(allow_smem(k_px_fwd<T>));
    CK(allow_smem(k_l2_rows<T>));
    c->sm_rhs = 0;
    switch (c->M) {
#define RHS_ATTR(MM)                                                                              \
  case MM:                                                                                        \
    c->sm_rhs = 4 * 5 * ColIdx<MM>::SIZE * cs;                                                   \
    c->sm_rhs64 = 4 * 5 * ColIdx<MM>::SIZE * sizeof(double2);                                    \
    CK(allow_smem(k_rhs<T, T, MM>));                                                              \
    CK(allow_smem(k_rhs<double, T, MM>));                                                         \
    break;
      RHS_ATTR(2) RHS_ATTR(3) RHS_ATTR(4) RHS_ATTR(5) RHS_ATTR(6) RHS_ATTR(7) RHS_ATTR(8)
#undef RHS_ATTR
    }
    // register-FFT kernels: z-kernel tiles that keep four (FP32) or two (FP64)
    // blocks per SM, matching their launch bounds
    const bool f32 = sizeof(T) == 4;
    c->fast_z = regfft_supported(g.nz2);
    c->fast_x = regfft_supported(g.nx2);
    if (c->fast_z) {
      const size_t zb = f32 ? 52 * 1024 : 108 * 1024;
      // z inverse: three blocks per SM with the raw tile and the exchange
      // (FP32); one plane per block in FP64 (measured best at 256x193x256)
      c->fYB1 = 1;
      for (int yb = f32 ? 4 : 1; yb >= 1; --yb)
        if (p1_fast_smem(0, g.nz2, f32, yb, g.nxh, g.nz) <= 74 * 1024) { c->fYB1 = yb; break; }
      c->fYB3 = 1;
      for (int yb = 4; yb >= 1; --yb)
        if (p1_fast_smem(2, g.nz2, f32, yb, g.nxh, g.nz) <= zb) { c->fYB3 = yb; break; }
    }
    if (c->fast_x) {
      c->fZR = 1;
      for (int zr : {4, 2})
        if (g.nz2 % zr == 0 && p1_fast_smem(1, g.nx2, f32, zr, g.nxh, g.nz) <= budget) { c->fZR = zr; break; }
      if (p1_fast_smem(1, g.nx2, f32, c->fZR, g.nxh, g.nz) > 220 * 1024) c->fast_x = false;
    }
    if (getenv("CHANFLOW_GENERIC_FFT")) c->fast_x = c->fast_z = false;
    // split x stage: physical planes written once, fluxes read three of them
    // z rows per flux block: 4 (FP32) or 2 (FP64, half the shared memory)
    // z2 rows per inverse-x block: the default rule unless CHANFLOW_XINV_ROWS
    // sets 8, 16 or 24 (the tuners also try them)
    c->xinv_zb = getenv("CHANFLOW_XINV_ROWS") ? atoi(getenv("CHANFLOW_XINV_ROWS")) : 0;
    if (c->xinv_zb != 8 && !(f32 && (c->xinv_zb == 16 || c->xinv_zb == 24))) c->xinv_zb = 0;
    c->flux_zr = getenv("CHANFLOW_FLUX_ZR") ? atoi(getenv("CHANFLOW_FLUX_ZR")) : (f32 ? 4 : 2);
    if (c->flux_zr != 2 && !(c->flux_zr == 8 && f32)) c->flux_zr = 4;   // 8 rows: FP32 only
    // (gP: the x stage's geometry, all kx and this rank's z2 rows)
    const Geom& gp = c->gP;
    if (c->xinv_zb && gp.nz2 % c->xinv_zb) c->xinv_zb = 0;
    c->split_x = c->fast_x && (!getenv("CHANFLOW_FUSED_XFLUX") || c->nranks > 1) && gp.nz2 % 8 == 0 &&
                 gp.nz2 % c->flux_zr == 0 && p1_fast_smem(3, g.nx2, f32, gp.nz2, gp.nxh, g.nz) <= 200 * 1024 &&
                 p1_fast_smem(4, g.nx2, f32, c->flux_zr, gp.nxh, g.nz) <= 200 * 1024;
    if (c->split_x &&
        cudaMalloc(&c->P, sizeof(T) * (size_t)(g.ny + 1) * 3 * gp.nz2 * g.nx2) != cudaSuccess) {
      cudaGetLastError();
      c->split_x = false;
    }
    // mixed precision, one rank, register transforms: the FP32 transforms
    // carry the fluctuation only and the mean's products come from its FP64
    // copy (CHANFLOW_NO_MEAN_SPLIT=1 keeps the whole velocity in the
    // transforms)
    c->mean_split = f32 && c->split_x && c->fast_z && c->nranks == 1 && !getenv("CHANFLOW_NO_MEAN_SPLIT");
    if (c->mean_split && cudaMalloc(&c->mean_base, sizeof(double) * 3 * (size_t)g.ny1) != cudaSuccess) {
      cudaGetLastError();
      c->mean_split = false;
    }
    c->use_rhs2 = rhs2_supported(g.ny1) && !getenv("CHANFLOW_RHS_V1");
    // lanes per wavenumber in FP32: 8 (four wavenumbers per warp) up to 64
    // rows, 16 (two) up to 128 -- fewer idle rows and fewer cyclic-reduction
    // levels than 32; 32 for taller columns (fewer lanes would hold more
    // than 8 rows each) and in FP64 (its kernel and coefficient table exist
    // for 32 only).
    // CHANFLOW_RHS2_LANES=8 (up to 64 rows), 16 (up to 256) or 32 overrides
    // the choice in FP32.  Not a tuned tile: the lane count sets the
    // reduction order of the solves, so it changes the rounding.
    c->rhs2_lanes = !f32 ? 32 : (g.ny1 <= 64 ? 8 : (g.ny1 <= 128 ? 16 : 32));
    if (f32 && getenv("CHANFLOW_RHS2_LANES")) {
      const int l = atoi(getenv("CHANFLOW_RHS2_LANES"));
      if (l == 32 || (l == 16 && g.ny1 <= 256) || (l == 8 && g.ny1 <= 64)) c->rhs2_lanes = l;
    }
    c->rhs2_warps = f32 ? 3 : 2;
    c->twx = make_twiddles<T>(g.nx2);
    c->twz = make_twiddles<T>(g.nz2);
    c->twxs = make_twiddles<T>(g.nx);
    c->twzs = make_twiddles<T>(g.nz);
    if (!c->twx || !c->twz || !c->twxs || !c->twzs) return fail(c, CFG_E_NOMEM, "twiddles");
    return CFG_OK;
  }

  static int nonlinear(cfg_ctx* c, int step, int rk, bool lin) {
    for (int ph = 1; ph <= 3; ++ph) {
      const int r = nl_phase(c, step, rk, lin, ph);
      if (r) return r;
    }
    return CFG_OK;
  }

  // the launch record of register-FFT pass-1 kernel `which` (0 k_zinv_r, 1
  // k_xflux_r, 2 k_zfwd_r, 3 k_xinv_r, 4 k_flux_r) in substep rk
  static P1Launch p1_args(const cfg_ctx* c, int rk, bool lin, int which) {
    const Geom& g = c->g;
    P1Launch a{};
    a.vel = c->vel; a.T1 = c->T1; a.T2 = c->T2; a.velout = c->vel; a.g = g; a.twx = c->twx; a.twz = c->twz;
    a.gd = c->gd; a.fringe = c->fringe; a.has_fringe = c->has_fringe; a.YB1 = c->fYB1; a.YB3 = c->fYB3;
    a.ZR = c->fZR; a.cflbits = c->cflbits; a.do_cfl = (rk == 1); a.lin = lin ? 1 : 0; a.st = c->st;
    a.KC = (int)std::max(2L, std::min(16L, (long)(g.ny - 1) * (g.nz2 / c->fZR) / 592));
    a.P = c->P;
    a.FZR = c->flux_zr;
    a.sc = c->scat;
    a.split = (c->mean_split && !lin && !c->les_on) ? 1 : 0;
    a.XZB = c->xinv_zb;
    if (which == 3 || which == 4) {
      // x stage of the split path on this rank's z2 rows, all kx
      a.g = c->gP;
      a.gd = c->gd_all;
      if (c->fringe) a.fringe = (const T*)c->fringe + (size_t)c->z0s * g.nx2;
      if (which == 4 && a.split) a.gd.baseflow = c->mean_base;
    }
    return a;
  }

  // nonlinear (PFC/pass1.f90:26-124) in three phases; a multi-rank run puts
  // a barrier between them: 1 the inverse z transform, scattered to the z2
  // slabs; 2 the x stage (inverse x, fluxes, forward x), scattered to the kx
  // slabs; 3 the forward z transform and the CFL / dt update
  static int nl_phase(cfg_ctx* c, int step, int rk, bool lin, int phase) {
    const Geom& g = c->g;
    const int do_cfl = (rk == 1);
    const bool f32 = sizeof(T) == 4;
    P1Launch a = p1_args(c, rk, lin, 0);
    if (phase == 1) {
      if (a.split) {
        // the current mean velocity (the FP64 side copy when it holds it)
        prof_begin(c, "k_mean_base");
        k_mean_base<<<1, 256, 0, c->st>>>(c->mean64_valid ? c->mvel64 : nullptr, (const float2*)c->vel, c->mean_base,
                                         g.ny1);
        CKL();
      }
      c->mean64_valid = false;
      if (do_cfl) CK(cudaMemsetAsync(c->cflbits, 0, sizeof(unsigned long long) * 3 * g.ny1, c->st));
      dim3 g1(g.nxh, (g.ny1 + c->YB1 - 1) / c->YB1);
      prof_begin(c, "k_zinv");
      if (c->fast_z) {
        if (p1_fast_launch(0, g.nz2, f32, a) != 0) return fail(c, CFG_E_CUDA, "k_zinv_r launch");
      } else
        k_zinv<T><<<g1, 256, c->sm_zinv, c->st>>>((const C*)c->vel, (C*)c->T1, g, c->pz, (const C*)c->twz,
                                                   c->YB1, 0, g.ny1);
      CKL();
      return CFG_OK;
    }
    if (phase == 2) {
      dim3 g2(g.nz2 / c->ZR, (g.ny - 1 + c->KC - 1) / c->KC);
      if (c->split_x) {
        a = p1_args(c, rk, lin, 3);
        prof_begin(c, "k_xinv");
        if (p1_fast_launch(3, g.nx2, f32, a) != 0) return fail(c, CFG_E_CUDA, "k_xinv_r launch");
        CKL();
        a = p1_args(c, rk, lin, 4);
        if (c->les_on && !lin) {
          const int r = les_stresses(c, c->les_F);
          if (r) return r;
          a.sgs = c->les_S;
        }
        prof_begin(c, "k_flux");
        if (p1_fast_launch(4, g.nx2, f32, a) != 0) return fail(c, CFG_E_CUDA, "k_flux_r launch");
      } else if (c->fast_x) {
        prof_begin(c, "k_xflux");
        if (p1_fast_launch(1, g.nx2, f32, a) != 0) return fail(c, CFG_E_CUDA, "k_xflux_r launch");
      } else if (lin) {
        prof_begin(c, "k_xflux");
        k_xflux<T, true><<<g2, 256, c->sm_xflux, c->st>>>((const C*)c->T1, (C*)c->T2, g, c->px, (const C*)c->twx,
                                                           c->gd, (const T*)c->fringe, c->has_fringe, c->ZR, c->KC,
                                                           c->cflbits, do_cfl);
      } else {
        prof_begin(c, "k_xflux");
        k_xflux<T, false><<<g2, 256, c->sm_xflux, c->st>>>((const C*)c->T1, (C*)c->T2, g, c->px, (const C*)c->twx,
                                                            c->gd, (const T*)c->fringe, c->has_fringe, c->ZR, c->KC,
                                                            c->cflbits, do_cfl);
      }
      CKL();
      return CFG_OK;
    }
    if (do_cfl && c->n_cfl_peers > 0) {
      prof_begin(c, "k_cfl_merge");
      k_cfl_merge<<<1, 256, 0, c->st>>>(c->cflbits, c->cfl_peers, c->n_cfl_peers, 3 * g.ny1);
      CKL();
    }
    dim3 g3(g.nxh, (g.ny1 + c->YB3 - 1) / c->YB3);
    prof_begin(c, "k_zfwd");
    if (c->fast_z) {
      if (p1_fast_launch(2, g.nz2, f32, a) != 0) return fail(c, CFG_E_CUDA, "k_zfwd_r launch");
    } else
      k_zfwd<T><<<g3, 256, c->sm_zfwd, c->st>>>((const C*)c->T2, (C*)c->vel, g, c->pz, (const C*)c->twz, c->gd, c->YB3);
    CKL();
    if (do_cfl) {
      prof_begin(c, "k_cfl_finalize");
      if (lin)
        k_cfl_finalize<true><<<1, 256, 0, c->st>>>(c->cflbits, g, c->gd, c->sc, c->cflp, c->p.lx, c->p.lz,
                                                    c->p.dt_flag, c->p.cfl_max, step);
      else
        k_cfl_finalize<false><<<1, 256, 0, c->st>>>(c->cflbits, g, c->gd, c->sc, c->cflp, c->p.lx, c->p.lz,
                                                     c->p.dt_flag, c->p.cfl_max, step);
      CKL();
    }
    return CFG_OK;
  }

  // the LES mode's subgrid stresses from the physical planes P (after
  // k_xinv_r): eddy viscosity, and for model 2 the network and the checks
  static int les_stresses(cfg_ctx* c, float* F) {
    const Geom& g = c->g;
    dim3 gr((g.nx2 + 127) / 128, g.nz2, g.ny - 1);
    prof_begin(c, "k_les_sgs");
    k_les_sgs<T><<<gr, 128, 0, c->st>>>((const T*)c->P, (T*)c->les_S, F, g, c->gd, c->les, c->d_um_dy);
    CKL();
    if (c->les.model == 2 && F == c->les_F) {
      // the planes' eddy-viscosity lengths, then the network with the checks
      // and the blend in its output layer's epilogue (the outputs never go
      // to memory)
      k_les_lengths<<<1, 128, 0, c->st>>>(c->les_len, c->gd, c->les, c->d_um_dy, g.ny);
      CKL();
      prof_begin(c, "k_mlp_fwd");
      const LesBlend<T> b{(T*)c->les_S, c->les_F, c->les_len, c->gd, c->les, g.nx2, g.nz2, c->les_nfall};
      if (mlp_forward_blend<T>(c->les_mlp, (long long)c->les_points, b, c->st) != CFG_OK)
        return fail(c, CFG_E_CUDA, "closure network launch");
      c->launches++;
      prof_end(c);
    }
    return CFG_OK;
  }

  // the closure's input features of the current state into F (device):
  // the inverse transforms and the feature kernel, without a step
  static int les_features(cfg_ctx* c, float* F) {
    const Geom& g = c->g;
    const bool f32 = sizeof(T) == 4;
    P1Launch a{};
    a.vel = c->vel; a.T1 = c->T1; a.g = g; a.twx = c->twx; a.twz = c->twz; a.gd = c->gd; a.YB1 = c->fYB1;
    a.st = c->st; a.P = c->P; a.FZR = c->flux_zr; a.sc = c->scat;
    if (p1_fast_launch(0, g.nz2, f32, a) != 0) return fail(c, CFG_E_CUDA, "k_zinv_r launch");
    c->launches++;
    a.g = c->gP;
    a.gd = c->gd_all;
    if (p1_fast_launch(3, g.nx2, f32, a) != 0) return fail(c, CFG_E_CUDA, "k_xinv_r launch");
    c->launches++;
    return les_stresses(c, F);
  }

  // launch records of k_rhs2: the fast list (storage precision) or, prec,
  // the mixed path's |k| < 4 list in FP64 on the side stream st2
  static Rhs2Launch rhs2_args(const cfg_ctx* c, int rk, bool prec) {
    const Geom& g = c->g;
    Rhs2Launch a{};
    a.vel = c->vel; a.cru = c->cru; a.prs = c->prs;
    a.cbc_top = (const C*)c->cbc + 3 * (size_t)g.nw; a.cbc_bot = c->cbc;
    a.g = g; a.gd = c->gd; a.sc = c->sc; a.rkt = c->rkt; a.rk = rk; a.re = c->p.re;
    if (prec) {
      a.wlist = c->wl_prec; a.nlist = c->n_prec; a.warps = 1; a.lanes = 32; a.tbl = c->rhs2_tbl64;
      a.st = c->st2;
    } else {
      a.wlist = c->wl_fast; a.nlist = c->n_fast; a.warps = c->rhs2_warps; a.lanes = c->rhs2_lanes;
      a.tbl = c->rhs2_tbl;
      a.st = c->st;
    }
    return a;
  }
  // launch record of the mean mode (k_rhs_mean2) on the side stream st3
  static RhsMeanLaunch mean_args(const cfg_ctx* c, int rk) {
    const Geom& g = c->g;
    RhsMeanLaunch m{};
    m.vel = c->vel; m.cru = c->cru; m.prs = c->prs; m.mvel64 = c->mvel64; m.mcru64 = c->mcru64;
    m.cbc_top = (const C*)c->cbc + 3 * (size_t)g.nw; m.cbc_bot = c->cbc;
    m.g = g; m.gd = c->gd; m.sc = c->sc; m.d_um_dy = c->d_um_dy; m.rkt = c->rkt; m.rk = rk;
    m.re = c->p.re; m.beta = c->p.beta; m.fix_mass = c->p.fix_mass; m.tbl64 = (const double*)c->rhs2_tbl64;
    m.st = c->st3;
    return m;
  }

  template <int MM>
  static int rhs_m(cfg_ctx* c, int rk, int mode) {
    const Geom& g = c->g;
    // crossflow == 1: the wall jet of this substep (PFC/pass2.f90:41-43)
    if (c->crossflow && mode == 0) {
      const int r = jet(c, rk, 0.0, 0.0, 1);
      if (r) return r;
    }
    // fork: the FP64 low-|k| list and the mean mode on two side streams, one
    // warp per wavenumber so that they spread over many SMs beside the main
    // kernel
    CK(cudaEventRecord(c->ev_fork, c->st));
    CK(cudaStreamWaitEvent(c->st2, c->ev_fork, 0));
    CK(cudaStreamWaitEvent(c->st3, c->ev_fork, 0));
    const bool v2 = c->use_rhs2 && c->rhs2_tbl64 && mode == 0;
    if (c->n_prec > 0) {
      c->prof_stream = c->st2;
      prof_begin(c, "k_rhs_fp64");
      if (v2 && sizeof(T) == 4) {
        if (rhs2_launch_prec(rhs2_args(c, rk, true)) != 0) return fail(c, CFG_E_CUDA, "k_rhs2 (FP64 list) launch");
      } else {
        k_rhs<double, T, MM><<<c->n_prec, 32, c->sm_rhs64 / 4, c->st2>>>((C*)c->vel, (C*)c->cru, (C*)c->prs,
                                                                       (const C*)c->cbc + 3 * (size_t)g.nw,
                                                                       (const C*)c->cbc, g, c->gd, c->sc, c->rkt, rk,
                                                                       c->p.re, mode, c->wl_prec, c->n_prec);
      }
      CKL();
    }
    if (mode == 0) c->mean64_valid = true;
    c->prof_stream = c->st3;
    prof_begin(c, "k_rhs_mean");
    if (g.kx0 != 0) {
      // the mean mode lives on the rank that holds kx = 0
    } else if (v2) {
      if (rhs_mean2_launch(sizeof(T) == 4, mean_args(c, rk)) != 0) return fail(c, CFG_E_CUDA, "k_rhs_mean2 launch");
    } else {
      k_rhs_mean<T, MM><<<1, 32, 0, c->st3>>>((C*)c->vel, (C*)c->cru, (C*)c->prs, c->mvel64, c->mcru64,
                                             (const C*)c->cbc + 3 * (size_t)g.nw, (const C*)c->cbc, g, c->gd, c->sc,
                                             c->d_um_dy, c->rkt, rk, c->p.re, c->p.beta, c->p.fix_mass, mode);
    }
    CKL();
    c->prof_stream = nullptr;
    CK(cudaEventRecord(c->ev_join, c->st2));
    CK(cudaEventRecord(c->ev_join3, c->st3));
    if (c->n_fast > 0 && mode == 0 && c->use_rhs2) {
      prof_begin(c, "k_rhs");
      if (rhs2_launch(sizeof(T) == 4, rhs2_args(c, rk, false)) != 0) return fail(c, CFG_E_CUDA, "k_rhs2 launch");
      CKL();
    } else if (c->n_fast > 0) {
      dim3 gr((c->n_fast + 3) / 4);
      prof_begin(c, "k_rhs");
      k_rhs<T, T, MM><<<gr, 128, c->sm_rhs, c->st>>>((C*)c->vel, (C*)c->cru, (C*)c->prs,
                                                     (const C*)c->cbc + 3 * (size_t)g.nw, (const C*)c->cbc, g,
                                                     c->gd, c->sc, c->rkt, rk, c->p.re, mode, c->wl_fast, c->n_fast);
      CKL();
    }
    // join
    CK(cudaStreamWaitEvent(c->st, c->ev_join, 0));
    CK(cudaStreamWaitEvent(c->st, c->ev_join3, 0));
    return CFG_OK;
  }
  static int rhs(cfg_ctx* c, int rk, int mode) {
    switch (c->M) {
      case 2: return rhs_m<2>(c, rk, mode);
      case 3: return rhs_m<3>(c, rk, mode);
      case 4: return rhs_m<4>(c, rk, mode);
      case 5: return rhs_m<5>(c, rk, mode);
      case 6: return rhs_m<6>(c, rk, mode);
      case 7: return rhs_m<7>(c, rk, mode);
      default: return rhs_m<8>(c, rk, mode);
    }
  }

  // inverse transforms of `np` spectral planes to physical rows
  static int planes_c2r(cfg_ctx* c, const C* in, PlaneIn L, const int* plist_dev, int np, T* phys) {
    const Geom& g = c->g;
    const int smp = (int)(sizeof(C) * (g.nz2 + 2 * L.nc * g.nz2));
    prof_begin(c, "k_pz_inv");
    k_pz_inv<T><<<dim3(g.nxh, np), 128, smp, c->st>>>(in, L, plist_dev, np, (C*)c->pw_H, g.nxh, g.nz, g.nz2, 1,
                                                       g.nx2 > g.nx, c->pz, (const C*)c->twz);
    CKL();
    const int smx = (int)(sizeof(C) * 3 * g.nx2);
    prof_begin(c, "k_px_inv");
    k_px_inv<T><<<dim3((g.nz2 + 1) / 2, np * L.nc), 128, smx, c->st>>>((const C*)c->pw_H, phys, g.nxh, g.nz2, g.nx2,
                                                                        c->px, (const C*)c->twx);
    CKL();
    return CFG_OK;
  }
  static int planes_r2c(cfg_ctx* c, const T* phys, int np, C* out, size_t osp, size_t oskx, size_t oskz) {
    const Geom& g = c->g;
    const int smx = (int)(sizeof(C) * 3 * g.nx2);
    prof_begin(c, "k_px_fwd");
    k_px_fwd<T><<<dim3((g.nz2 + 1) / 2, np), 128, smx, c->st>>>(phys, (C*)c->pw_H, g.nxh, g.nz2, g.nx2, c->px,
                                                                (const C*)c->twx);
    CKL();
    const int smz = (int)(sizeof(C) * 3 * g.nz2);
    const T scale = (T)(1.0 / ((double)g.nx2 * (double)g.nz2));
    prof_begin(c, "k_pz_fwd");
    k_pz_fwd<T><<<dim3(g.nxh, np), 128, smz, c->st>>>((const C*)c->pw_H, out, osp, oskx, oskz, g.nxh, g.nz2, g.nz, 1,
                                                      scale, c->pz, (const C*)c->twz);
    CKL();
    return CFG_OK;
  }

  // small (nx x nz, no dealiasing) transforms of np planes,
  // small_fft_real_to_complex / small_fft_complex_to_real
  // (PFC/transform.f90:950-1142); H is a scratch of np*nxh*nz complex values
  static int small_r2c(cfg_ctx* c, const T* phys, int np, C* out, size_t osp, size_t oskx, size_t oskz, C* H) {
    const Geom& g = c->g;
    const int smx = (int)(sizeof(C) * 3 * g.nx);
    prof_begin(c, "k_px_fwd");
    k_px_fwd<T><<<dim3((g.nz + 1) / 2, np), 128, smx, c->st>>>(phys, H, g.nxh, g.nz, g.nx, c->pxs, (const C*)c->twxs);
    CKL();
    const int smz = (int)(sizeof(C) * 3 * g.nz);
    const T scale = (T)(1.0 / ((double)g.nx * (double)g.nz));
    prof_begin(c, "k_pz_fwd");
    k_pz_fwd<T><<<dim3(g.nxh, np), 128, smz, c->st>>>(H, out, osp, oskx, oskz, g.nxh, g.nz, g.nz, 0, scale, c->pzs,
                                                      (const C*)c->twzs);
    CKL();
    return CFG_OK;
  }
  static int small_c2r(cfg_ctx* c, const C* in, PlaneIn L, int np, T* phys, C* H) {
    const Geom& g = c->g;
    const int smp = (int)(sizeof(C) * (g.nz + 2 * L.nc * g.nz));
    prof_begin(c, "k_pz_inv");
    k_pz_inv<T><<<dim3(g.nxh, np), 128, smp, c->st>>>(in, L, nullptr, np, H, g.nxh, g.nz, g.nz, 0, 0, c->pzs,
                                                      (const C*)c->twzs);
    CKL();
    const int smx = (int)(sizeof(C) * 3 * g.nx);
    prof_begin(c, "k_px_inv");
    k_px_inv<T><<<dim3((g.nz + 1) / 2, np * L.nc), 128, smx, c->st>>>(H, phys, g.nxh, g.nz, g.nx, c->pxs,
                                                                       (const C*)c->twxs);
    CKL();
    return CFG_OK;
  }

  // jet_profile (PFC/pass2.f90:423-673) into cbc(:,:,2): use_sc takes the
  // end-of-substep time of substep rk from the device scalars
  static int jet(cfg_ctx* c, int rk, double time, double incr, int use_sc) {
    const Geom& g = c->g;
    prof_begin(c, "k_jet_walk");
    k_jet_walk<<<1, 32, 0, c->st>>>(c->jst, c->jp, c->sc, c->rkt, rk, time, incr, use_sc);
    CKL();
    prof_begin(c, "k_jet_field");
    k_jet_field<T><<<dim3(g.nz, 3), 128, 0, c->st>>>((T*)c->pw_phys, c->jp, c->jst, g.nx, g.nz, c->p.lx, c->p.lz);
    CKL();
    int r = small_r2c(c, (const T*)c->pw_phys, 3, (C*)c->pw_in, (size_t)g.nw, g.nz, 1, (C*)c->pw_H);
    if (r) return r;
    prof_begin(c, "k_jet_combine");
    k_jet_combine<T><<<(g.nw + 255) / 256, 256, 0, c->st>>>((const C*)c->pw_in, (C*)c->cbc, c->jp, c->gd, g.nx,
                                                             g.nz, g.nxh, c->p.lx, c->p.lz);
    CKL();
    return CFG_OK;
  }

  static int boundary(cfg_ctx* c) {
    const Geom& g = c->g;
    CK(cudaMemsetAsync(c->cbc, 0, sizeof(C) * 6 * (size_t)g.nw, c->st));
    const size_t np = (size_t)g.nx2 * g.nz2;
    for (int q = 0; q < 3; q += 2) {
      const double gain = q == 0 ? c->p.ctrlu : c->p.ctrlw;
      if (gain == 0.0) continue;
      const double off = q == 0 ? 2.0 : 0.0;
      PlaneIn L{1, (size_t)g.ny1, (size_t)g.nz * 3 * g.ny1, (size_t)3 * g.ny1, 1};
      int r = planes_c2r(c, (const C*)c->vel + (size_t)q * g.ny1, L, c->plist, 4, (T*)c->pw_phys);
      if (r) return r;
      const double* dm = nullptr;
      (void)dm;
      prof_begin(c, "k_feedback");
      k_feedback<T><<<grid1d(np), 256, 0, c->st>>>((const T*)c->pw_phys, (T*)c->pw_phys2, np, c->hdm[0], c->hdm[1],
                                                   c->hdm[2], c->hdm[3], c->hdm[4], c->hdm[5], gain, off);
      CKL();
      r = planes_r2c(c, (const T*)c->pw_phys2, 2, (C*)c->cbc + (size_t)q * g.nw, 3 * (size_t)g.nw, g.nz, 1);
      if (r) return r;
    }
    return CFG_OK;
  }

  static int l2(cfg_ctx* c, double* l2, double* drag) {
    const Geom& g = c->g;
    CK(cudaMemsetAsync(c->l2acc, 0, sizeof(double) * g.ny1, c->st));
    const int smp = (int)(sizeof(C) * (g.nz2 + 2 * 3 * g.nz2));
    PlaneIn L{1, (size_t)g.ny1, (size_t)g.nz * 3 * g.ny1, (size_t)3 * g.ny1, 3};
    prof_begin(c, "k_pz_inv");
    k_pz_inv<T><<<dim3(g.nxh, g.ny), 128, smp, c->st>>>((const C*)c->vel, L, nullptr, g.ny, (C*)c->T1, g.nxh, g.nz,
                                                        g.nz2, 1, g.nx2 > g.nx, c->pz, (const C*)c->twz);
    CKL();
    const int smx = (int)(sizeof(C) * 3 * g.nx2);
    prof_begin(c, "k_l2_rows");
    k_l2_rows<T><<<dim3((g.nz2 + 1) / 2, 3 * g.ny), 128, smx, c->st>>>((const C*)c->T1, g.nxh, g.nz2, g.nx2, c->px,
                                                                       (const C*)c->twx, c->gd.y, g.ny, c->l2acc);
    CKL();
    std::vector<double> acc(g.ny1), dmd(g.ny);
    CK(cudaMemcpyAsync(acc.data(), c->l2acc, sizeof(double) * g.ny, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(dmd.data(), c->d_um_dy, sizeof(double) * g.ny, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    double s = 0;
    for (int j = 0; j < g.ny; ++j) s += acc[j] * c->hdy[j];
    if (l2) *l2 = sqrt(s / (double)g.nx2 / (double)g.nz2 / 2.0);
    if (drag) *drag = dmd[0] - dmd[g.ny - 1];
    return CFG_OK;
  }
};


// ----------------------------------------------------------------------------
#define DISPATCH(c, call) ((c)->mixed ? Impl<float>::call : Impl<double>::call)

static size_t csize(const cfg_ctx* c) { return c->mixed ? sizeof(float2) : sizeof(double2); }
static size_t rsize(const cfg_ctx* c) { return c->mixed ? sizeof(float) : sizeof(double); }

static int ensure_stage(cfg_ctx* c, size_t elems) {
  if (c->stage_elems >= elems) return CFG_OK;
  if (c->stage) cudaFree(c->stage);
  c->stage = nullptr;
  c->stage_elems = 0;
  CK(cudaMalloc(&c->stage, sizeof(double2) * elems));
  c->stage_elems = elems;
  return CFG_OK;
}

// the FP64 side copy of the mean column, on the rank that holds kx = 0
static double2* mean_side(const cfg_ctx* c, double2* p) { return c->g.kx0 == 0 ? p : nullptr; }

// entry points that need the whole grid on one context
static int single_only(cfg_ctx* c, const char* what) {
  return fail(c, CFG_E_ARG, "%s: not available on one rank of a multi-rank group", what);
}

static int check_status(cfg_ctx* c) {
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->sc, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (h.status == CFG_E_CFL) return fail(c, CFG_E_CFL, "CFL IS TOO BIG");
  if (h.status == CFG_E_DT) return fail(c, CFG_E_DT, "DT IS TOO BIG");
  return CFG_OK;
}

extern "C" {

const char* cfg_last_error(const cfg_ctx* c) { return c ? c->err.c_str() : "null context"; }
long long cfg_launch_count(const cfg_ctx* c) { return c ? c->launches : 0; }
void* cfg_stream(cfg_ctx* c) { return c ? (void*)c->st : nullptr; }

// one context: the whole grid (sp == nullptr) or one rank's slabs of it
static int create_impl(const cfg_params* p, const cfg_grid* gr, const SlabPart* sp, cfg_ctx** out) {
  if (!p || !gr || !out) return CFG_E_ARG;
  *out = nullptr;
  cfg_ctx* c = new cfg_ctx();
  c->p = *p;
  auto bad = [&](int code) { cfg_destroy(c); return code; };
  if (p->nx < 4 || p->nz < 4 || p->ny < 5 || (p->nx & 1) || (p->nz & 1) || p->nx2 < p->nx || p->nz2 < p->nz ||
      (p->nx2 & 1) || (p->nz2 & 1)) {
    fprintf(stderr, "cfg_create: unsupported grid %d x %d x %d (%d, %d)\n", p->nx, p->ny, p->nz, p->nx2, p->nz2);
    delete c;
    return CFG_E_ARG;
  }
  if (p->precision != CFG_FP64 && p->precision != CFG_MIXED) { delete c; return CFG_E_ARG; }
  c->mixed = (p->precision == CFG_MIXED);
  Geom& g = c->g;
  g.nx = p->nx; g.ny = p->ny; g.nz = p->nz; g.nx2 = p->nx2; g.nz2 = p->nz2;
  g.nxh_all = p->nx / 2 + 1;
  g.nxh = sp ? sp->nxl : g.nxh_all;
  g.kx0 = sp ? sp->x0 : 0;
  g.ny1 = p->ny + 1;
  g.nw = g.nz * g.nxh;
  c->gP = g;
  c->gP.nxh = g.nxh_all;
  c->gP.kx0 = 0;
  c->gP.nz2 = sp ? sp->nzl : g.nz2;
  c->gP.nw = g.nz * g.nxh_all;
  if (sp) {
    c->rank = sp->rank;
    c->nranks = sp->nranks;
    c->z0s = sp->z0;
  }
  if (!make_plan(g.nx2, c->px) || !make_plan(g.nz2, c->pz) || !make_plan(g.nx, c->pxs) || !make_plan(g.nz, c->pzs)) {
    fprintf(stderr, "cfg_create: transform lengths must be 2^a 3^b\n");
    delete c;
    return CFG_E_ARG;
  }
  c->dev = p->device;
  if (cudaSetDevice(c->dev) != cudaSuccess) { fail(c, CFG_E_CUDA, "cudaSetDevice"); delete c; return CFG_E_CUDA; }
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->st3, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join3, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    delete c;
    return CFG_E_CUDA;
  }
  // RK constants: single-precision literals widened (PFC/pass2.f90:14-18)
  const float ra[3] = {0.0f, -17.0f / 60.0f, -5.0f / 12.0f}, rb[3] = {8.0f / 15.0f, 5.0f / 12.0f, 3.0f / 4.0f};
  const float rc[3] = {29.0f / 96.0f, -3.0f / 40.0f, 1.0f / 6.0f}, rd[3] = {37.0f / 160.0f, 5.0f / 24.0f, 1.0f / 6.0f};
  for (int i = 0; i < 3; ++i) {
    c->rkt.a[i + 1] = ra[i]; c->rkt.b[i + 1] = rb[i]; c->rkt.c[i + 1] = rc[i]; c->rkt.d[i + 1] = rd[i];
  }
  // grid operators (FP64 on the device)
  const int ny = g.ny, n1 = g.ny1;
  struct Part { const double* src; size_t n; const double** dst; };
  std::vector<double> zeros3((size_t)3 * n1, 0.0);
  const double* tgt = gr->target_inflow ? gr->target_inflow : zeros3.data();
  Part parts[] = {{gr->y, (size_t)ny, &c->gd.y},       {gr->yh, (size_t)n1, &c->gd.yh},
                  {gr->hn, (size_t)ny, &c->gd.hn},     {gr->dh, (size_t)n1, &c->gd.dh},
                  {gr->dn, (size_t)ny, &c->gd.dn},     {gr->iu, (size_t)2 * ny, &c->gd.iu},
                  {gr->dm, 12, &c->gd.dm},             {gr->d2h, (size_t)3 * n1, &c->gd.d2h},
                  {gr->d2n, (size_t)3 * ny, &c->gd.d2n}, {gr->dyh, (size_t)n1, &c->gd.dyh},
                  {gr->dy, (size_t)n1, &c->gd.dy},     {gr->kx, (size_t)g.nxh_all, &c->gd.kx},
                  {gr->kz, (size_t)g.nz, &c->gd.kz},   {tgt, (size_t)3 * n1, &c->gd.target},
                  {zeros3.data(), (size_t)3 * n1, &c->gd.baseflow}};
  size_t tot = 0;
  for (auto& pt : parts) {
    if (!pt.src) { fprintf(stderr, "cfg_create: missing grid array\n"); return bad(CFG_E_ARG); }
    tot += pt.n;
  }
  // the end rows of d2h/d2n must be the copied neighbours (PFC/setup.f90:720-726)
  for (int i = 0; i < 3; ++i) {
    if (gr->d2h[i] != gr->d2h[3 + i] || gr->d2h[3 * ny + i] != gr->d2h[3 * (ny - 1) + i] ||
        gr->d2n[i] != gr->d2n[3 + i] || gr->d2n[3 * (ny - 1) + i] != gr->d2n[3 * (ny - 2) + i]) {
      fail(c, CFG_E_ARG, "d2h/d2n end rows are not copies of their neighbours");
      fprintf(stderr, "cfg_create: %s\n", c->err.c_str());
      return bad(CFG_E_ARG);
    }
  }
  if (cudaMalloc(&c->dgrid, sizeof(double) * tot) != cudaSuccess) return bad(CFG_E_NOMEM);
  {
    std::vector<double> h(tot);
    size_t off = 0;
    for (auto& pt : parts) {
      memcpy(h.data() + off, pt.src, sizeof(double) * pt.n);
      *pt.dst = c->dgrid + off;
      off += pt.n;
    }
    cudaMemcpy(c->dgrid, h.data(), sizeof(double) * tot, cudaMemcpyHostToDevice);
  }
  // the x stage reads the global kx table; the Fourier-space kernels this
  // rank's slab of it
  c->gd_all = c->gd;
  c->gd.kx = c->gd_all.kx + g.kx0;
  memcpy(c->hdm, gr->dm, sizeof(double) * 12);
  c->hdy.assign(gr->dy, gr->dy + n1);
  c->hyh.assign(gr->yh, gr->yh + n1);
  // state and work buffers
  const size_t cs = csize(c), nf = (size_t)g.nw * 3 * n1;
  // T1: hybrid rows of this rank's z2 slab for all kx (the z transform's
  // scatter target); T2: x-transformed fluxes of this rank's kx slab for all
  // z2 (the flux kernel's scatter target)
  const size_t t1 = (size_t)n1 * 3 * g.nxh_all * c->gP.nz2, t2 = (size_t)n1 * 6 * g.nxh * g.nz2;
  bool ok = cudaMalloc(&c->vel, cs * nf) == cudaSuccess && cudaMalloc(&c->cru, cs * nf) == cudaSuccess &&
            cudaMalloc(&c->prs, cs * (size_t)g.nw * n1) == cudaSuccess && cudaMalloc(&c->T1, cs * t1) == cudaSuccess &&
            cudaMalloc(&c->T2, cs * t2) == cudaSuccess && cudaMalloc(&c->cbc, cs * 6 * (size_t)g.nw) == cudaSuccess &&
            cudaMalloc(&c->sc, sizeof(DevScalars)) == cudaSuccess &&
            cudaMalloc(&c->d_um_dy, sizeof(double) * ny) == cudaSuccess &&
            cudaMalloc(&c->cflp, sizeof(double) * n1) == cudaSuccess &&
            cudaMalloc(&c->cflbits, sizeof(unsigned long long) * 3 * n1) == cudaSuccess &&
            cudaMalloc(&c->l2acc, sizeof(double) * n1) == cudaSuccess &&
            cudaMalloc(&c->divbits, sizeof(unsigned long long)) == cudaSuccess &&
            cudaMalloc(&c->plist, sizeof(int) * 8) == cudaSuccess;
  const size_t npl = 4;
  ok = ok && cudaMalloc(&c->pw_H, cs * npl * 3 * g.nxh * g.nz2) == cudaSuccess &&
       cudaMalloc(&c->pw_phys, rsize(c) * npl * g.nx2 * g.nz2) == cudaSuccess &&
       cudaMalloc(&c->pw_phys2, rsize(c) * npl * g.nx2 * g.nz2) == cudaSuccess &&
       cudaMalloc(&c->pw_in, cs * npl * g.nw) == cudaSuccess;
  if (c->mixed)
    ok = ok && cudaMalloc(&c->mvel64, sizeof(double2) * 3 * n1) == cudaSuccess &&
         cudaMalloc(&c->mcru64, sizeof(double2) * 3 * n1) == cudaSuccess;
  if (!ok) return bad(CFG_E_NOMEM);
  cudaMemset(c->vel, 0, cs * nf);
  cudaMemset(c->cru, 0, cs * nf);
  cudaMemset(c->prs, 0, cs * (size_t)g.nw * n1);
  cudaMemset(c->cbc, 0, cs * 6 * (size_t)g.nw);
  cudaMemset(c->d_um_dy, 0, sizeof(double) * ny);
  cudaMemset(c->cflp, 0, sizeof(double) * n1);
  if (c->mixed) {
    cudaMemset(c->mvel64, 0, sizeof(double2) * 3 * n1);
    cudaMemset(c->mcru64, 0, sizeof(double2) * 3 * n1);
  }
  DevScalars h{};
  h.t_total = 0.0;
  h.dt = p->dt;
  h.p_grad = -2.0 / p->re;   // PFC/setup.f90:1384
  cudaMemcpy(c->sc, &h, sizeof(h), cudaMemcpyHostToDevice);
  int pl[4] = {1, 2, ny - 1, ny - 2};   // planes 2, 3, ny, ny-1 (boundary)
  cudaMemcpy(c->plist, pl, sizeof(pl), cudaMemcpyHostToDevice);
  {
    // wavenumber lists: the mean mode has its own kernel; in mixed precision
    // the wavenumbers with |k| < 4 (ill-conditioned pressure solves on the
    // stretched grid) run with FP64 arithmetic
    std::vector<int> fast, prec;
    for (int w = (g.kx0 == 0 ? 1 : 0); w < g.nw; ++w) {
      const double kx = gr->kx[g.kx0 + w / g.nz], kz = gr->kz[w % g.nz];
      const double k2 = kx * kx + kz * kz;
      if (c->mixed && k2 < 16.0) prec.push_back(w);
      else fast.push_back(w);
    }
    c->n_fast = (int)fast.size();
    c->n_prec = (int)prec.size();
    if (cudaMalloc(&c->wl_fast, sizeof(int) * std::max<size_t>(1, fast.size())) != cudaSuccess ||
        cudaMalloc(&c->wl_prec, sizeof(int) * std::max<size_t>(1, prec.size())) != cudaSuccess)
      return bad(CFG_E_NOMEM);
    if (!fast.empty()) cudaMemcpy(c->wl_fast, fast.data(), sizeof(int) * fast.size(), cudaMemcpyHostToDevice);
    if (!prec.empty()) cudaMemcpy(c->wl_prec, prec.data(), sizeof(int) * prec.size(), cudaMemcpyHostToDevice);
  }
  if (gr->buffer) {
    bool any = false;
    for (size_t i = 0; i < (size_t)g.nx2 * g.nz2; ++i) any = any || gr->buffer[i] != 0.0;
    if (any) {
      c->has_fringe = 1;
      if (cudaMalloc(&c->fringe, rsize(c) * g.nx2 * g.nz2) != cudaSuccess) return bad(CFG_E_NOMEM);
      std::vector<float> hf(g.nx2 * (size_t)g.nz2);
      if (c->mixed) {
        for (size_t i = 0; i < hf.size(); ++i) hf[i] = (float)gr->buffer[i];
        cudaMemcpy(c->fringe, hf.data(), sizeof(float) * hf.size(), cudaMemcpyHostToDevice);
      } else {
        cudaMemcpy(c->fringe, gr->buffer, sizeof(double) * hf.size(), cudaMemcpyHostToDevice);
      }
    }
  }
  int r = DISPATCH(c, setup(c));
  if (r) {
    fprintf(stderr, "cfg_create: %s\n", c->err.c_str());
    return bad(r);
  }
  if (c->use_rhs2) {
    const size_t tb = rhs2_table_bytes(c->mixed, g.ny1, c->rhs2_lanes);
    std::vector<unsigned char> ht(tb);
    rhs2_table(c->mixed, ny, c->rhs2_lanes, gr->dh, gr->dn, gr->d2h, gr->d2n, ht.data());
    if (cudaMalloc(&c->rhs2_tbl, tb) != cudaSuccess) return bad(CFG_E_NOMEM);
    cudaMemcpy(c->rhs2_tbl, ht.data(), tb, cudaMemcpyHostToDevice);
    const size_t tb64 = rhs2_table_bytes(false, g.ny1, 32);
    std::vector<unsigned char> h64(tb64);
    rhs2_table(false, ny, 32, gr->dh, gr->dn, gr->d2h, gr->d2n, h64.data());
    if (cudaMalloc(&c->rhs2_tbl64, tb64) != cudaSuccess) return bad(CFG_E_NOMEM);
    cudaMemcpy(c->rhs2_tbl64, h64.data(), tb64, cudaMemcpyHostToDevice);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return bad(CFG_E_CUDA);
  *out = c;
  return CFG_OK;
}

int cfg_create(const cfg_params* p, const cfg_grid* gr, cfg_ctx** out) { return create_impl(p, gr, nullptr, out); }

void cfg_destroy(cfg_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  if (c->io_thread.joinable()) c->io_thread.join();
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->st_io) cudaStreamSynchronize(c->st_io);
  if (c->io_dev) cudaFree(c->io_dev);
  if (c->sc_snap) cudaFree(c->sc_snap);
  if (c->io_host) cudaFreeHost(c->io_host);
  if (c->sc_host) cudaFreeHost(c->sc_host);
  if (c->ev_io_start) cudaEventDestroy(c->ev_io_start);
  if (c->ev_io_done) cudaEventDestroy(c->ev_io_done);
  if (c->st_io) cudaStreamDestroy(c->st_io);
  for (void* q : c->ipc_open) cudaIpcCloseMemHandle(q);
  void* bufs[] = {c->dgrid, c->fringe, c->vel, c->cru, c->prs, c->mvel64, c->mcru64, c->T1, c->T2, c->P,
                  c->rhs2_tbl, c->rhs2_tbl64, c->jst, c->pp_wy, c->pp_sy, c->pp_acc, c->cbc,
                  c->sc, c->d_um_dy, c->cflp, c->cflbits, c->l2acc, c->divbits, c->plist, c->pw_H,
                  c->pw_phys, c->pw_phys2, c->pw_in, c->stage, c->twx, c->twz, c->twxs, c->twzs,
                  c->wl_fast, c->wl_prec, c->scat_tab, c->cfl_peers, c->les_S, c->les_F, c->les_len,
                  c->les_nfall, c->mean_base};
  for (void* b : bufs)
    if (b) cudaFree(b);
  for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->ev_join3) cudaEventDestroy(c->ev_join3);
  if (c->st2) cudaStreamDestroy(c->st2);
  if (c->st3) cudaStreamDestroy(c->st3);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

int cfg_upload_state(cfg_ctx* c, const double* d1, const double* d2, const double* d4) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t nf = (size_t)g.nw * 3 * g.ny1;
  int r = ensure_stage(c, nf);
  if (r) return r;
  if (d1) {
    CK(cudaMemcpyAsync(c->stage, d1, sizeof(double2) * nf, cudaMemcpyHostToDevice, c->st));
    c->mean64_valid = true;
    if (c->mixed) k_data1_in<float><<<grid1d(nf), 256, 0, c->st>>>(c->stage, (float2*)c->vel, mean_side(c, c->mvel64), g);
    else k_data1_in<double><<<grid1d(nf), 256, 0, c->st>>>(c->stage, (double2*)c->vel, nullptr, g);
    CKL();
  }
  if (d2) {
    CK(cudaMemcpyAsync(c->stage, d2, sizeof(double2) * nf, cudaMemcpyHostToDevice, c->st));
    if (c->mixed) k_conv_in<float><<<grid1d(nf), 256, 0, c->st>>>(c->stage, (float2*)c->cru, nf, mean_side(c, c->mcru64), 3 * (size_t)g.ny1);
    else k_conv_in<double><<<grid1d(nf), 256, 0, c->st>>>(c->stage, (double2*)c->cru, nf, nullptr, 0);
    CKL();
  }
  if (d4) {
    const size_t n = (size_t)g.nw * g.ny1;
    CK(cudaMemcpyAsync(c->stage, d4, sizeof(double2) * n, cudaMemcpyHostToDevice, c->st));
    if (c->mixed) k_conv_in<float><<<grid1d(n), 256, 0, c->st>>>(c->stage, (float2*)c->prs, n, nullptr, 0);
    else k_conv_in<double><<<grid1d(n), 256, 0, c->st>>>(c->stage, (double2*)c->prs, n, nullptr, 0);
    CKL();
  }
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}

int cfg_download_state(cfg_ctx* c, double* d1, double* d2, double* d4) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t nf = (size_t)g.nw * 3 * g.ny1;
  int r = ensure_stage(c, nf);
  if (r) return r;
  if (d1) {
    if (c->mixed) k_data1_out<float><<<grid1d(nf), 256, 0, c->st>>>((const float2*)c->vel, c->mean64_valid ? mean_side(c, c->mvel64) : nullptr, c->stage, g);
    else k_data1_out<double><<<grid1d(nf), 256, 0, c->st>>>((const double2*)c->vel, nullptr, c->stage, g);
    CKL();
    CK(cudaMemcpyAsync(d1, c->stage, sizeof(double2) * nf, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  if (d2) {
    if (c->mixed) k_conv_out<float><<<grid1d(nf), 256, 0, c->st>>>((const float2*)c->cru, c->stage, nf, mean_side(c, c->mcru64), 3 * (size_t)g.ny1);
    else k_conv_out<double><<<grid1d(nf), 256, 0, c->st>>>((const double2*)c->cru, c->stage, nf, nullptr, 0);
    CKL();
    CK(cudaMemcpyAsync(d2, c->stage, sizeof(double2) * nf, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  if (d4) {
    const size_t n = (size_t)g.nw * g.ny1;
    if (c->mixed) k_conv_out<float><<<grid1d(n), 256, 0, c->st>>>((const float2*)c->prs, c->stage, n, nullptr, 0);
    else k_conv_out<double><<<grid1d(n), 256, 0, c->st>>>((const double2*)c->prs, c->stage, n, nullptr, 0);
    CKL();
    CK(cudaMemcpyAsync(d4, c->stage, sizeof(double2) * n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  return CFG_OK;
}

int cfg_set_scalars(cfg_ctx* c, double t_total, double dt, double p_grad, const double* d_um_dy) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->sc, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  h.t_total = t_total;
  h.dt = dt;
  h.p_grad = p_grad;
  CK(cudaMemcpyAsync(c->sc, &h, sizeof(h), cudaMemcpyHostToDevice, c->st));
  if (d_um_dy) CK(cudaMemcpyAsync(c->d_um_dy, d_um_dy, sizeof(double) * c->g.ny, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}

int cfg_get_scalars(cfg_ctx* c, double* t_total, double* dt, double* p_grad, double* d_um_dy, double* cfl_max) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->sc, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  if (d_um_dy) CK(cudaMemcpyAsync(d_um_dy, c->d_um_dy, sizeof(double) * c->g.ny, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (t_total) *t_total = h.t_total;
  if (dt) *dt = h.dt;
  if (p_grad) *p_grad = h.p_grad;
  if (cfl_max) *cfl_max = h.cfl_max;
  return CFG_OK;
}

int cfg_set_wall_bc(cfg_ctx* c, const double* top, const double* bot) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  const size_t n = 3 * (size_t)c->g.nw;
  int r = ensure_stage(c, 2 * n);
  if (r) return r;
  const double* src[2] = {bot, top};
  for (int k = 0; k < 2; ++k) {
    if (!src[k]) continue;
    CK(cudaMemcpyAsync(c->stage, src[k], sizeof(double2) * n, cudaMemcpyHostToDevice, c->st));
    if (c->mixed) k_conv_in<float><<<grid1d(n), 256, 0, c->st>>>(c->stage, (float2*)c->cbc + k * n, n, nullptr, 0);
    else k_conv_in<double><<<grid1d(n), 256, 0, c->st>>>(c->stage, (double2*)c->cbc + k * n, n, nullptr, 0);
    CKL();
    CK(cudaStreamSynchronize(c->st));
  }
  return CFG_OK;
}

int cfg_get_wall_bc(cfg_ctx* c, double* top, double* bot) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  const size_t n = 3 * (size_t)c->g.nw;
  int r = ensure_stage(c, 2 * n);
  if (r) return r;
  double* dst[2] = {bot, top};
  for (int k = 0; k < 2; ++k) {
    if (!dst[k]) continue;
    if (c->mixed) k_conv_out<float><<<grid1d(n), 256, 0, c->st>>>((const float2*)c->cbc + k * n, c->stage, n, nullptr, 0);
    else k_conv_out<double><<<grid1d(n), 256, 0, c->st>>>((const double2*)c->cbc + k * n, c->stage, n, nullptr, 0);
    CKL();
    CK(cudaMemcpyAsync(dst[k], c->stage, sizeof(double2) * n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  return CFG_OK;
}

int cfg_set_baseflow(cfg_ctx* c, const double* profile) {
  if (!c || !profile) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  CK(cudaMemcpyAsync((void*)c->gd.baseflow, profile, sizeof(double) * 3 * c->g.ny1, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}

int cfg_boundary(cfg_ctx* c) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  return DISPATCH(c, boundary(c));
}

int cfg_nonlinear(cfg_ctx* c, int step, int rk_step) {
  if (!c || rk_step < 1 || rk_step > 3) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_nonlinear");
  cudaSetDevice(c->dev);
  c->step = step;
  return DISPATCH(c, nonlinear(c, step, rk_step, false));
}

int cfg_nonlinear_linearized(cfg_ctx* c, int step, int rk_step) {
  if (!c || rk_step < 1 || rk_step > 3) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_nonlinear_linearized");
  cudaSetDevice(c->dev);
  c->step = step;
  return DISPATCH(c, nonlinear(c, step, rk_step, true));
}

int cfg_rhs_solve(cfg_ctx* c, int step, int rk_step) {
  if (!c || rk_step < 1 || rk_step > 3) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  (void)step;
  return DISPATCH(c, rhs(c, rk_step, 0));
}

// one time step (PFC/main_mpi.f90:70-86), enqueued only: boundary, three
// (nonlinear, rhs_solve) substeps, t_total += dt
static int step_enqueue(cfg_ctx* c, bool lin) {
  c->step = c->step < 0 ? 1 : c->step + 1;
  int r;
  if (!lin) {
    r = DISPATCH(c, boundary(c));
    if (r) return r;
  }
  for (int rk = 1; rk <= 3; ++rk) {
    r = DISPATCH(c, nonlinear(c, c->step, rk, lin));
    if (r) return r;
    r = DISPATCH(c, rhs(c, rk, 0));
    if (r) return r;
  }
  prof_begin(c, "k_advance_time");
  k_advance_time<<<1, 1, 0, c->st>>>(c->sc);
  CKL();
  return CFG_OK;
}

static int timestep_impl(cfg_ctx* c, int nsteps, bool lin) {
  if (!c || nsteps < 0) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_timestep");
  cudaSetDevice(c->dev);
  for (int s = 0; s < nsteps; ++s) {
    const int r = step_enqueue(c, lin);
    if (r) return r;
  }
  return CFG_OK;
}

int cfg_timestep(cfg_ctx* c, int nsteps) { return timestep_impl(c, nsteps, false); }


int cfg_timestep_linearized(cfg_ctx* c, int nsteps) { return timestep_impl(c, nsteps, true); }

int cfg_remove_initial_divergence(cfg_ctx* c) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  int r = DISPATCH(c, rhs(c, 1, 1));
  if (r) return r;
  const size_t nf = (size_t)c->g.nw * 3 * c->g.ny1;
  CK(cudaMemcpyAsync(c->cru, c->vel, csize(c) * nf, cudaMemcpyDeviceToDevice, c->st));
  return CFG_OK;
}

int cfg_compute_initial_pressure(cfg_ctx* c, int linearized) {
  if (!c) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_compute_initial_pressure");
  cudaSetDevice(c->dev);
  // step = -1, rk_step = 3 (PFC/init_vel.f90:444-445): no CFL, no dt change
  int r = DISPATCH(c, nonlinear(c, -1, 3, linearized != 0));
  if (r) return r;
  r = DISPATCH(c, rhs(c, 3, 2));
  if (r) return r;
  // data1 = data2 (the velocity copy), PFC/init_vel.f90:469-473
  const size_t nf = (size_t)c->g.nw * 3 * c->g.ny1;
  CK(cudaMemcpyAsync(c->vel, c->cru, csize(c) * nf, cudaMemcpyDeviceToDevice, c->st));
  if (c->mixed) CK(cudaMemcpyAsync(c->mvel64, c->mcru64, sizeof(double2) * 3 * c->g.ny1, cudaMemcpyDeviceToDevice, c->st));
  c->mean64_valid = true;
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}

int cfg_xz_c2r(cfg_ctx* c, const double* cdata, double* data) {
  if (!c || !cdata || !data) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_xz_c2r");
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t nin = (size_t)g.nw, nout = (size_t)g.nx2 * g.nz2;
  int r = ensure_stage(c, std::max(nin, nout));
  if (r) return r;
  CK(cudaMemcpyAsync(c->stage, cdata, sizeof(double2) * nin, cudaMemcpyHostToDevice, c->st));
  PlaneIn L{0, 0, (size_t)g.nz, 1, 1};
  if (c->mixed) {
    k_conv_in<float><<<grid1d(nin), 256, 0, c->st>>>(c->stage, (float2*)c->pw_in, nin, nullptr, 0);
    CKL();
    r = Impl<float>::planes_c2r(c, (const float2*)c->pw_in, L, nullptr, 1, (float*)c->pw_phys);
    if (r) return r;
    k_real_out<float><<<grid1d(nout), 256, 0, c->st>>>((const float*)c->pw_phys, (double*)c->stage, nout);
  } else {
    k_conv_in<double><<<grid1d(nin), 256, 0, c->st>>>(c->stage, (double2*)c->pw_in, nin, nullptr, 0);
    CKL();
    r = Impl<double>::planes_c2r(c, (const double2*)c->pw_in, L, nullptr, 1, (double*)c->pw_phys);
    if (r) return r;
    k_real_out<double><<<grid1d(nout), 256, 0, c->st>>>((const double*)c->pw_phys, (double*)c->stage, nout);
  }
  CKL();
  CK(cudaMemcpyAsync(data, c->stage, sizeof(double) * nout, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}

int cfg_xz_r2c(cfg_ctx* c, const double* data, double* cdata) {
  if (!c || !cdata || !data) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_xz_r2c");
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t nin = (size_t)g.nx2 * g.nz2, nout = (size_t)g.nw;
  int r = ensure_stage(c, std::max(nin, nout));
  if (r) return r;
  CK(cudaMemcpyAsync(c->stage, data, sizeof(double) * nin, cudaMemcpyHostToDevice, c->st));
  if (c->mixed) {
    k_real_in<float><<<grid1d(nin), 256, 0, c->st>>>((const double*)c->stage, (float*)c->pw_phys, nin);
    CKL();
    r = Impl<float>::planes_r2c(c, (const float*)c->pw_phys, 1, (float2*)c->pw_in, 0, g.nz, 1);
    if (r) return r;
    k_conv_out<float><<<grid1d(nout), 256, 0, c->st>>>((const float2*)c->pw_in, c->stage, nout, nullptr, 0);
  } else {
    k_real_in<double><<<grid1d(nin), 256, 0, c->st>>>((const double*)c->stage, (double*)c->pw_phys, nin);
    CKL();
    r = Impl<double>::planes_r2c(c, (const double*)c->pw_phys, 1, (double2*)c->pw_in, 0, g.nz, 1);
    if (r) return r;
    k_conv_out<double><<<grid1d(nout), 256, 0, c->st>>>((const double2*)c->pw_in, c->stage, nout, nullptr, 0);
  }
  CKL();
  CK(cudaMemcpyAsync(cdata, c->stage, sizeof(double2) * nout, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}

// the small transforms use the hybrid and flux work arrays as device scratch
// (T1 holds the spectral planes; T2 the physical planes and, behind them, the
// hybrid intermediate)
static int small_capacity(cfg_ctx* c) {
  const Geom& g = c->g;
  const size_t t1 = (size_t)g.ny1 * 3 * g.nxh * g.nz2, t2 = (size_t)g.ny1 * 6 * g.nxh * g.nz2;
  const size_t per_t2 = ((size_t)g.nx * g.nz + 1) / 2 + (size_t)g.nxh * g.nz + 1;
  return (int)std::min<size_t>(std::min(t1 / g.nw, t2 / per_t2), 65535);
}

int cfg_small_r2c(cfg_ctx* c, const double* data, double* cdata, int nplanes) {
  if (!c || !cdata || !data || nplanes < 1) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_small_r2c");
  if (nplanes > small_capacity(c)) return fail(c, CFG_E_ARG, "cfg_small_r2c: more than %d planes", small_capacity(c));
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t nin = (size_t)g.nx * g.nz * nplanes, nout = (size_t)g.nw * nplanes;
  int r = ensure_stage(c, std::max(nin, nout));
  if (r) return r;
  CK(cudaMemcpyAsync(c->stage, data, sizeof(double) * nin, cudaMemcpyHostToDevice, c->st));
  if (c->mixed) {
    k_real_in<float><<<grid1d(nin), 256, 0, c->st>>>((const double*)c->stage, (float*)c->T2, nin);
    CKL();
    r = Impl<float>::small_r2c(c, (const float*)c->T2, nplanes, (float2*)c->T1, (size_t)g.nw, g.nz, 1,
                               (float2*)c->T2 + (nin + 1) / 2);
    if (r) return r;
    k_conv_out<float><<<grid1d(nout), 256, 0, c->st>>>((const float2*)c->T1, c->stage, nout, nullptr, 0);
  } else {
    k_real_in<double><<<grid1d(nin), 256, 0, c->st>>>((const double*)c->stage, (double*)c->T2, nin);
    CKL();
    r = Impl<double>::small_r2c(c, (const double*)c->T2, nplanes, (double2*)c->T1, (size_t)g.nw, g.nz, 1,
                                (double2*)c->T2 + (nin + 1) / 2);
    if (r) return r;
    k_conv_out<double><<<grid1d(nout), 256, 0, c->st>>>((const double2*)c->T1, c->stage, nout, nullptr, 0);
  }
  CKL();
  CK(cudaMemcpyAsync(cdata, c->stage, sizeof(double2) * nout, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}

int cfg_small_c2r(cfg_ctx* c, const double* cdata, double* data, int nplanes) {
  if (!c || !cdata || !data || nplanes < 1) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_small_c2r");
  if (nplanes > small_capacity(c)) return fail(c, CFG_E_ARG, "cfg_small_c2r: more than %d planes", small_capacity(c));
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t nin = (size_t)g.nw * nplanes, nout = (size_t)g.nx * g.nz * nplanes;
  int r = ensure_stage(c, std::max(nin, nout));
  if (r) return r;
  CK(cudaMemcpyAsync(c->stage, cdata, sizeof(double2) * nin, cudaMemcpyHostToDevice, c->st));
  PlaneIn L{(size_t)g.nw, 0, (size_t)g.nz, 1, 1};
  if (c->mixed) {
    k_conv_in<float><<<grid1d(nin), 256, 0, c->st>>>(c->stage, (float2*)c->T1, nin, nullptr, 0);
    CKL();
    r = Impl<float>::small_c2r(c, (const float2*)c->T1, L, nplanes, (float*)c->T2, (float2*)c->T2 + (nout + 1) / 2);
    if (r) return r;
    k_real_out<float><<<grid1d(nout), 256, 0, c->st>>>((const float*)c->T2, (double*)c->stage, nout);
  } else {
    k_conv_in<double><<<grid1d(nin), 256, 0, c->st>>>(c->stage, (double2*)c->T1, nin, nullptr, 0);
    CKL();
    r = Impl<double>::small_c2r(c, (const double2*)c->T1, L, nplanes, (double*)c->T2,
                                (double2*)c->T2 + (nout + 1) / 2);
    if (r) return r;
    k_real_out<double><<<grid1d(nout), 256, 0, c->st>>>((const double*)c->T2, (double*)c->stage, nout);
  }
  CKL();
  CK(cudaMemcpyAsync(data, c->stage, sizeof(double) * nout, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}

int cfg_set_les(cfg_ctx* c, const cfg_les* l) {
  if (!c) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_set_les");
  cudaSetDevice(c->dev);
  if (!l || l->model == 0) {
    c->les_on = false;
    return CFG_OK;
  }
  if (l->model != 1 && l->model != 2) return fail(c, CFG_E_ARG, "cfg_set_les: model %d", l->model);
  if (!c->split_x) return fail(c, CFG_E_ARG, "cfg_set_les: needs the register-FFT x stage (nx2 of 24 .. 576)");
  if (l->model == 2 && !l->mlp) return fail(c, CFG_E_ARG, "cfg_set_les: model 2 needs the network");
  if (!(l->cs >= 0.0) || !(l->aplus > 0.0) || !(l->beta >= 0.0)) return fail(c, CFG_E_ARG, "cfg_set_les: cs, aplus, beta");
  for (int i = 0; i < 10; ++i)
    if (!(l->in_scale[i] != 0.0f) && l->model == 2) return fail(c, CFG_E_ARG, "cfg_set_les: in_scale[%d] = 0", i);
  const Geom& g = c->g;
  const size_t cs = (size_t)g.nz2 * g.nx2;
  const size_t tsz = c->mixed ? sizeof(float) : sizeof(double);
  c->les_points = (unsigned long long)(g.ny - 1) * cs;
  if (!c->les_S) {
    if (cudaMalloc(&c->les_S, tsz * 6 * cs * g.ny1) != cudaSuccess || cudaMalloc(&c->les_nfall, 8) != cudaSuccess)
      return fail(c, CFG_E_NOMEM, "LES stresses");
    CK(cudaMemsetAsync(c->les_S, 0, tsz * 6 * cs * g.ny1, c->st));   // wall planes stay zero
  }
  if (l->model == 2 && !c->les_F) {
    if (cudaMalloc(&c->les_F, sizeof(float) * 10 * c->les_points) != cudaSuccess ||
        cudaMalloc(&c->les_len, sizeof(double) * (g.ny + 1)) != cudaSuccess)
      return fail(c, CFG_E_NOMEM, "LES closure buffers");
  }
  CK(cudaMemsetAsync(c->les_nfall, 0, 8, c->st));
  LesDev& d = c->les;
  d.model = l->model;
  d.cs = l->cs;
  d.aplus = l->aplus;
  d.beta = l->beta;
  d.dx = c->p.lx / g.nx;
  d.dz = c->p.lz / g.nz;
  d.hx = c->p.lx / g.nx2;
  d.hz = c->p.lz / g.nz2;
  d.re = c->p.re;
  for (int i = 0; i < 10; ++i) {
    d.in_shift[i] = l->in_shift[i];
    d.in_scale[i] = l->model == 2 ? l->in_scale[i] : 1.0f;
    d.in_iscale[i] = 1.0 / (double)d.in_scale[i];
  }
  for (int i = 0; i < 6; ++i) {
    d.out_shift[i] = l->out_shift[i];
    d.out_scale[i] = l->out_scale[i];
  }
  c->les_mlp = l->mlp;
  CK(cudaStreamSynchronize(c->st));
  c->les_on = true;
  return CFG_OK;
}

int cfg_les_features(cfg_ctx* c, float* features) {
  if (!c || !features) return CFG_E_ARG;
  if (!c->les_on || c->les.model != 2) return fail(c, CFG_E_STATE, "cfg_les_features: set the LES model 2 first");
  cudaSetDevice(c->dev);
  return DISPATCH(c, les_features(c, features));
}

int cfg_les_stresses(cfg_ctx* c, double* S) {
  if (!c || !S) return CFG_E_ARG;
  if (!c->les_S) return fail(c, CFG_E_STATE, "cfg_les_stresses: no LES model set");
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t n = (size_t)g.ny1 * 6 * g.nz2 * g.nx2;
  if (c->mixed) {
    std::vector<float> h(n);
    CK(cudaMemcpyAsync(h.data(), c->les_S, n * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (size_t i = 0; i < n; ++i) S[i] = h[i];
  } else {
    CK(cudaMemcpyAsync(S, c->les_S, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  return CFG_OK;
}

int cfg_les_fallbacks(cfg_ctx* c, unsigned long long* fallbacks, unsigned long long* points) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  unsigned long long h = 0;
  if (c->les_nfall) {
    CK(cudaMemcpyAsync(&h, c->les_nfall, 8, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  if (fallbacks) *fallbacks = h;
  if (points) *points = c->les_points;
  return CFG_OK;
}

int cfg_set_jet(cfg_ctx* c, const cfg_jet* j) {
  if (!c) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_set_jet");
  cudaSetDevice(c->dev);
  if (!j || j->mode == 0) {
    c->crossflow = false;
    return CFG_OK;
  }
  if (j->mode != 1 && j->mode != 2) return fail(c, CFG_E_ARG, "cfg_set_jet: mode %d", j->mode);
  if (j->filter_jet_profile < 0) return fail(c, CFG_E_ARG, "cfg_set_jet: filter_jet_profile < 0");
  if (j->mode == 1 && !(j->jet_diam > 0.0)) return fail(c, CFG_E_ARG, "cfg_set_jet: jet_diam must be positive");
  if (j->mode == 2 && !(j->width > 0.0)) return fail(c, CFG_E_ARG, "cfg_set_jet: width must be positive");
  // define_suction_profile (PFC/pass2.f90:565-567)
  const double frac_suct = 0.5 * j->frac_xbuff, xend = c->p.lx * (1.0 - j->frac_xbuff) + c->p.lx * frac_suct;
  if (!(j->frac_xbuff > 0.0) || xend > c->p.lx) return fail(c, CFG_E_ARG, "Suction must end inside box.");
  JetParams& p = c->jp;
  p.mode = j->mode;
  for (int w = 0; w < 2; ++w) {
    p.xjet[w] = j->xjet[w]; p.zjet[w] = j->zjet[w]; p.jetmag[w] = j->jetmag[w];
    p.forcing[w] = j->forcing[w]; p.for_freq[w] = j->for_freq[w];
  }
  p.jet_diam = j->jet_diam; p.width = j->width; p.freq = j->freq; p.frac_xbuff = j->frac_xbuff;
  p.filter = j->filter_jet_profile; p.seed = j->seed;
  if (!c->jst && cudaMalloc(&c->jst, sizeof(JetState)) != cudaSuccess) return fail(c, CFG_E_NOMEM, "jet state");
  JetState h{};
  memcpy(h.jf, j->jet_forcing, sizeof(h.jf));
  memcpy(h.inc, j->jet_forcing_incr, sizeof(h.inc));
  CK(cudaMemcpyAsync(c->jst, &h, sizeof(h), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->crossflow = true;
  return CFG_OK;
}

int cfg_jet_profile(cfg_ctx* c, double time, double time_incr) {
  if (!c) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_jet_profile");
  if (!c->crossflow) return fail(c, CFG_E_STATE, "cfg_jet_profile: no jet set (cfg_set_jet)");
  cudaSetDevice(c->dev);
  return DISPATCH(c, jet(c, 0, time, time_incr, 0));
}

int cfg_get_jet_forcing(cfg_ctx* c, double* jet_forcing, double* jet_forcing_incr) {
  if (!c) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_get_jet_forcing");
  if (!c->jst) return fail(c, CFG_E_STATE, "cfg_get_jet_forcing: no jet set (cfg_set_jet)");
  cudaSetDevice(c->dev);
  JetState h{};
  CK(cudaMemcpyAsync(&h, c->jst, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (jet_forcing) memcpy(jet_forcing, h.jf, sizeof(h.jf));
  if (jet_forcing_incr) memcpy(jet_forcing_incr, h.inc, sizeof(h.inc));
  return CFG_OK;
}

int cfg_l2_norm(cfg_ctx* c, double* l2, double* drag) {
  if (!c) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_l2_norm");
  cudaSetDevice(c->dev);
  return DISPATCH(c, l2(c, l2, drag));
}

int cfg_diagnostics(cfg_ctx* c, double* bulk_flux, double* max_div) {
  if (!c) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_diagnostics");
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  CK(cudaMemsetAsync(c->divbits, 0, sizeof(unsigned long long), c->st));
  const int nb = (g.nw + 3) / 4;
  if (c->mixed) k_divergence<float><<<nb, 128, 0, c->st>>>((const float2*)c->vel, g, c->gd, c->divbits);
  else k_divergence<double><<<nb, 128, 0, c->st>>>((const double2*)c->vel, g, c->gd, c->divbits);
  CKL();
  std::vector<double2> mean(g.ny1);
  if (c->mixed) CK(cudaMemcpyAsync(mean.data(), c->mvel64, sizeof(double2) * g.ny1, cudaMemcpyDeviceToHost, c->st));
  else CK(cudaMemcpyAsync(mean.data(), c->vel, sizeof(double2) * g.ny1, cudaMemcpyDeviceToHost, c->st));
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, c->divbits, sizeof(bits), cudaMemcpyDeviceToHost, c->st));
  std::vector<double> dyh(g.ny1);
  CK(cudaMemcpyAsync(dyh.data(), c->gd.dyh, sizeof(double) * g.ny1, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (bulk_flux) {
    double s = 0;
    for (int j = 0; j < g.ny1; ++j) s += dyh[j] * mean[j].x;
    *bulk_flux = s;
  }
  if (max_div) {
    double d;
    memcpy(&d, &bits, sizeof(d));
    *max_div = d;
  }
  return CFG_OK;
}

int cfg_status(cfg_ctx* c) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  return check_status(c);
}

int cfg_profile_enable(cfg_ctx* c, int on) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  CK(cudaStreamSynchronize(c->st));
  c->recs.clear();
  c->ev_used = 0;
  c->prof_on = on != 0;
  return CFG_OK;
}

int cfg_profile_read(cfg_ctx* c, int idx, char* name, int namelen, int* launches, double* total_ms) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  CK(cudaStreamSynchronize(c->st));
  // distinct kernel names in first-seen order
  std::vector<const char*> names;
  for (auto& r : c->recs) {
    bool seen = false;
    for (const char* n : names) seen = seen || strcmp(n, r.name) == 0;
    if (!seen) names.push_back(r.name);
  }
  if (idx < 0) return (int)names.size();
  if (idx >= (int)names.size()) return CFG_E_ARG;
  int n = 0;
  double ms = 0;
  for (auto& r : c->recs) {
    if (strcmp(r.name, names[idx]) != 0) continue;
    float t = 0;
    CK(cudaEventElapsedTime(&t, r.a, r.b));
    ms += t;
    ++n;
  }
  if (name && namelen > 0) snprintf(name, namelen, "%s", names[idx]);
  if (launches) *launches = n;
  if (total_ms) *total_ms = ms;
  return CFG_OK;
}

int cfg_synchronize(cfg_ctx* c) {
  if (!c) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}

}  // extern "C"

// compute_time_deriv (PFC/arnoldi.f90:485-567) on the device; see chanflow.h
int cfg_arnoldi_matvec(cfg_ctx* c, int tend, const double* v, double* w) {
  if (!c || !v || !w || tend < 0) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_arnoldi_matvec");
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const int np = 3 * g.ny1;
  if (np > small_capacity(c)) return fail(c, CFG_E_ARG, "cfg_arnoldi_matvec: %d planes exceed the scratch", np);
  const size_t nvec = (size_t)g.nx * g.nz * np, nf = (size_t)g.nw * np;
  int r = ensure_stage(c, nvec);
  if (r) return r;
  CK(cudaMemcpyAsync(c->stage, v, sizeof(double) * nvec, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemsetAsync(c->divbits, 0, sizeof(unsigned long long), c->st));
  k_absmax<<<std::min<size_t>(1184, (nvec + 255) / 256), 256, 0, c->st>>>((const double*)c->stage, nvec, c->divbits);
  CKL();
  unsigned long long mb = 0;
  CK(cudaMemcpyAsync(&mb, c->divbits, sizeof(mb), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (mb == 0) return fail(c, CFG_E_ARG, "cfg_arnoldi_matvec: zero vector");
  const double eps = 1.0e-8;   // PFC/arnoldi.f90:500
  PlaneIn L{1, 0, (size_t)g.nz * np, (size_t)np, 1};
  if (c->mixed) {
    using C = float2;
    k_real_in<float><<<grid1d(nvec), 256, 0, c->st>>>((const double*)c->stage, (float*)c->T2, nvec);
    CKL();
    r = Impl<float>::small_r2c(c, (const float*)c->T2, np, (C*)c->vel, 1, (size_t)g.nz * np, np, (C*)c->T1);
    if (r) return r;
    k_arnoldi_scale<float><<<grid1d(nf), 256, 0, c->st>>>((C*)c->vel, g, c->gd, c->divbits, eps, 0);
    CKL();
    k_mean_widen<float><<<1, 256, 0, c->st>>>((const C*)c->vel, c->mvel64, g.ny1);
    CKL();
    CK(cudaMemcpyAsync(c->mcru64, c->mvel64, sizeof(double2) * 3 * g.ny1, cudaMemcpyDeviceToDevice, c->st));
  } else {
    using C = double2;
    k_real_in<double><<<grid1d(nvec), 256, 0, c->st>>>((const double*)c->stage, (double*)c->T2, nvec);
    CKL();
    r = Impl<double>::small_r2c(c, (const double*)c->T2, np, (C*)c->vel, 1, (size_t)g.nz * np, np, (C*)c->T1);
    if (r) return r;
    k_arnoldi_scale<double><<<grid1d(nf), 256, 0, c->st>>>((C*)c->vel, g, c->gd, c->divbits, eps, 0);
    CKL();
  }
  c->mean64_valid = true;
  // data2 = data1, p_grad = 0, d_um_dy = 0, initial pressure, t_total = 0
  CK(cudaMemcpyAsync(c->cru, c->vel, csize(c) * nf, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaMemsetAsync(c->d_um_dy, 0, sizeof(double) * g.ny, c->st));
  k_arnoldi_reset<<<1, 1, 0, c->st>>>(c->sc);
  CKL();
  r = cfg_compute_initial_pressure(c, 1);
  if (r) return r;
  c->step = 0;
  r = timestep_impl(c, tend, true);
  if (r) return r;
  if (c->mixed) {
    using C = float2;
    k_arnoldi_scale<float><<<grid1d(nf), 256, 0, c->st>>>((C*)c->vel, g, c->gd, c->divbits, eps, 1);
    CKL();
    r = Impl<float>::small_c2r(c, (const C*)c->vel, L, np, (float*)c->T2, (C*)c->T1);
    if (r) return r;
    k_real_out<float><<<grid1d(nvec), 256, 0, c->st>>>((const float*)c->T2, (double*)c->stage, nvec);
  } else {
    using C = double2;
    k_arnoldi_scale<double><<<grid1d(nf), 256, 0, c->st>>>((C*)c->vel, g, c->gd, c->divbits, eps, 1);
    CKL();
    r = Impl<double>::small_c2r(c, (const C*)c->vel, L, np, (double*)c->T2, (C*)c->T1);
    if (r) return r;
    k_real_out<double><<<grid1d(nvec), 256, 0, c->st>>>((const double*)c->T2, (double*)c->stage, nvec);
  }
  CKL();
  CK(cudaMemcpyAsync(w, c->stage, sizeof(double) * nvec, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return cfg_status(c);
}

// ---------------------------------------------------------------------------
// Restart file and VTK snapshot (PFC/read_write.f90:21-292, 296-500)

int cfg_wait_io(cfg_ctx* c) {
  if (!c) return CFG_E_ARG;
  if (c->io_thread.joinable()) c->io_thread.join();
  const int r = c->io_status;
  c->io_status = 0;
  if (r) {
    c->err = c->io_err;
    fprintf(stderr, "chanflow: %s\n", c->io_err.c_str());
  }
  return r;
}

// device and pinned host buffers of the background output, grown on demand
static int ensure_io(cfg_ctx* c, size_t bytes) {
  if (!c->st_io) {
    CK(cudaStreamCreateWithFlags(&c->st_io, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_io_start, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_io_done, cudaEventDisableTiming));
    CK(cudaMalloc(&c->sc_snap, sizeof(DevScalars)));
    CK(cudaMallocHost(&c->sc_host, sizeof(DevScalars)));
  }
  if (c->io_bytes >= bytes) return CFG_OK;
  CK(cudaStreamSynchronize(c->st_io));
  if (c->io_dev) cudaFree(c->io_dev);
  if (c->io_host) cudaFreeHost(c->io_host);
  c->io_dev = c->io_host = nullptr;
  c->io_bytes = 0;
  if (cudaMalloc(&c->io_dev, bytes) != cudaSuccess || cudaMallocHost(&c->io_host, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, CFG_E_NOMEM, "output buffers of %zu bytes", bytes);
  }
  c->io_bytes = bytes;
  return CFG_OK;
}

// after the layout kernel on st: snapshot the scalars, copy the io buffer to
// the host on st_io and start the file writer, which waits for that copy
template <typename F>
static int start_io(cfg_ctx* c, size_t bytes, F write) {
  CK(cudaMemcpyAsync(c->sc_snap, c->sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, c->st));
  CK(cudaEventRecord(c->ev_io_start, c->st));
  CK(cudaStreamWaitEvent(c->st_io, c->ev_io_start, 0));
  CK(cudaMemcpyAsync(c->io_host, c->io_dev, bytes, cudaMemcpyDeviceToHost, c->st_io));
  CK(cudaMemcpyAsync(c->sc_host, c->sc_snap, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->st_io));
  CK(cudaEventRecord(c->ev_io_done, c->st_io));
  const int dev = c->dev;
  c->io_thread = std::thread([c, dev, write]() {
    cudaSetDevice(dev);
    if (cudaEventSynchronize(c->ev_io_done) != cudaSuccess) {
      c->io_status = CFG_E_CUDA;
      c->io_err = "output copy failed";
      return;
    }
    std::string why;
    c->io_status = write(why);
    c->io_err = why;
  });
  return CFG_OK;
}

int cfg_save_velocity(cfg_ctx* c, const char* path) {
  if (!c || !path) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_save_velocity");
  cudaSetDevice(c->dev);
  int r = cfg_wait_io(c);
  if (r) return r;
  const Geom& g = c->g;
  const size_t nf = (size_t)g.nw * 3 * g.ny1, bytes = nf * sizeof(double2);
  r = ensure_io(c, bytes);
  if (r) return r;
  if (c->mixed)
    k_restart_out<float><<<grid1d(nf), 256, 0, c->st>>>((const float2*)c->vel, c->mean64_valid ? c->mvel64 : nullptr,
                                                        (double2*)c->io_dev, g);
  else
    k_restart_out<double><<<grid1d(nf), 256, 0, c->st>>>((const double2*)c->vel, nullptr, (double2*)c->io_dev, g);
  CKL();
  const std::string p(path);
  const cfg_params prm = c->p;
  return start_io(c, bytes, [c, p, prm](std::string& why) {
    return cfd_io::write_restart_slabs(p.c_str(), prm.nx, prm.ny, prm.nz, prm.lx, prm.lz, prm.re, c->sc_host->dt,
                                       c->sc_host->t_total, (const double*)c->io_host, why);
  });
}

int cfg_read_velocity(cfg_ctx* c, const char* path) {
  if (!c || !path) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_read_velocity");
  cudaSetDevice(c->dev);
  int r = cfg_wait_io(c);
  if (r) return r;
  const Geom& g = c->g;
  const size_t nf = (size_t)g.nw * 3 * g.ny1, bytes = nf * sizeof(double2);
  r = ensure_io(c, bytes);
  if (r) return r;
  CK(cudaStreamSynchronize(c->st_io));
  double dt = 0, t_total = 0;
  std::string why;
  r = cfd_io::read_restart_slabs(path, c->p.nx, c->p.ny, c->p.nz, c->p.lx, c->p.lz, c->p.re, &dt, &t_total,
                                 (double*)c->io_host, why);
  if (r) return fail(c, r, "%s", why.c_str());
  CK(cudaMemcpyAsync(c->io_dev, c->io_host, bytes, cudaMemcpyHostToDevice, c->st));
  if (c->mixed)
    k_restart_in<float><<<grid1d(nf), 256, 0, c->st>>>((const double2*)c->io_dev, (float2*)c->vel, c->mvel64, g);
  else
    k_restart_in<double><<<grid1d(nf), 256, 0, c->st>>>((const double2*)c->io_dev, (double2*)c->vel, nullptr, g);
  CKL();
  c->mean64_valid = true;
  // t_total from the file; dt too when dt_flag (PFC/read_write.f90:75-79)
  DevScalars h;
  CK(cudaMemcpyAsync(&h, c->sc, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  h.t_total = t_total;
  if (c->p.dt_flag == 1) h.dt = dt;
  CK(cudaMemcpyAsync(c->sc, &h, sizeof(h), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}

int cfg_write_vtk(cfg_ctx* c, const char* path) {
  if (!c || !path) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_write_vtk");
  cudaSetDevice(c->dev);
  int r = cfg_wait_io(c);
  if (r) return r;
  const Geom& g = c->g;
  const int np = 3 * g.ny1;
  const size_t nvec = (size_t)g.nx * g.ny1 * g.nz * 3, bytes = nvec * 4;
  const size_t nspec = (size_t)g.nw * np, nh = (size_t)np * g.nxh * g.nz;
  r = ensure_io(c, bytes);
  if (r) return r;
  PlaneIn L{(size_t)g.nw, 0, (size_t)g.nz, 1, 1};
  if (c->mixed) {
    using C = float2;
    k_vtk_planes<float><<<grid1d(nspec), 256, 0, c->st>>>((const C*)c->vel, c->mean64_valid ? c->mvel64 : nullptr,
                                                          (C*)c->T1, g);
    CKL();
    float* phys = (float*)((C*)c->T2 + nh);
    r = Impl<float>::small_c2r(c, (const C*)c->T1, L, np, phys, (C*)c->T2);
    if (r) return r;
    k_vtk_pack<float><<<grid1d(nvec), 256, 0, c->st>>>(phys, (uint32_t*)c->io_dev, g.nx, g.ny1, g.nz);
  } else {
    using C = double2;
    k_vtk_planes<double><<<grid1d(nspec), 256, 0, c->st>>>((const C*)c->vel, nullptr, (C*)c->T1, g);
    CKL();
    double* phys = (double*)((C*)c->T2 + nh);
    r = Impl<double>::small_c2r(c, (const C*)c->T1, L, np, phys, (C*)c->T2);
    if (r) return r;
    k_vtk_pack<double><<<grid1d(nvec), 256, 0, c->st>>>(phys, (uint32_t*)c->io_dev, g.nx, g.ny1, g.nz);
  }
  CKL();
  const std::string p(path);
  const cfg_params prm = c->p;
  return start_io(c, bytes, [c, p, prm](std::string& why) {
    return cfd_io::write_vtk(p.c_str(), prm.nx, prm.ny, prm.nz, prm.lx, prm.lz, c->hyh.data(),
                             (const unsigned char*)c->io_host, 0, why);
  });
}

// ---------------------------------------------------------------------------
// Post-processing: velocity-gradient tensor, vorticity, Q-criterion and
// discriminant on the snapshot grid, and per-plane moments (the arithmetic of
// ParaView-Code/DiscriminantFilter.cpd:17 and PFC/stats.f90:120-251)

// 3-point Lagrange first-derivative weights on yh (stats.f90's setup_diff
// stencils: planes j-1, j, j+1; one-sided at the ends)
static int ensure_postproc(cfg_ctx* c) {
  if (c->pp_wy) return CFG_OK;
  const int n1 = c->g.ny1;
  std::vector<double> w(3 * n1);
  std::vector<int> sidx(3 * n1);
  const std::vector<double>& y = c->hyh;
  for (int j = 0; j < n1; ++j) {
    const int a = (j == 0) ? 0 : (j == n1 - 1 ? n1 - 3 : j - 1);
    const int nd[3] = {a, a + 1, a + 2};
    const double x0 = y[j];
    for (int q = 0; q < 3; ++q) {
      const double xq = y[nd[q]], xr = y[nd[(q + 1) % 3]], xs = y[nd[(q + 2) % 3]];
      w[3 * j + q] = ((x0 - xr) + (x0 - xs)) / ((xq - xr) * (xq - xs));
      sidx[3 * j + q] = nd[q];
    }
  }
  CK(cudaMalloc(&c->pp_wy, sizeof(double) * 3 * n1));
  CK(cudaMalloc(&c->pp_sy, sizeof(int) * 3 * n1));
  CK(cudaMalloc(&c->pp_acc, sizeof(double) * 30 * n1));
  CK(cudaMemcpy(c->pp_wy, w.data(), sizeof(double) * 3 * n1, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->pp_sy, sidx.data(), sizeof(int) * 3 * n1, cudaMemcpyHostToDevice));
  return CFG_OK;
}

template <typename T>
static int postproc(cfg_ctx* c, uint32_t* out) {
  using C = cplx_t<T>;
  const Geom& g = c->g;
  const int n1 = g.ny1;
  const size_t nw = (size_t)g.nw;
  const double2* m64 = (c->mixed && c->mean64_valid) ? c->mvel64 : nullptr;
  double* accV = c->pp_acc;
  double* accW = c->pp_acc + 15 * (size_t)n1;
  CK(cudaMemsetAsync(c->pp_acc, 0, sizeof(double) * 30 * n1, c->st));
  // velocity on the yh planes
  const int np3 = 3 * n1;
  PlaneIn L{nw, 0, (size_t)g.nz, 1, 1};
  k_vtk_planes<T><<<grid1d(nw * np3), 256, 0, c->st>>>((const C*)c->vel, m64, (C*)c->T1, g);
  CKL();
  T* physU = (T*)((C*)c->T2 + (size_t)np3 * g.nxh * g.nz);
  int r = Impl<T>::small_c2r(c, (const C*)c->T1, L, np3, physU, (C*)c->T2);
  if (r) return r;
  if (out) {
    k_vtk_pack<T><<<grid1d((size_t)g.nx * n1 * g.nz * 3), 256, 0, c->st>>>(physU, out, g.nx, n1, g.nz);
    CKL();
  }
  k_stats_vel<T><<<dim3(g.nz, n1), 128, 0, c->st>>>(physU, (const C*)c->T1, g.nx, g.nz, n1, nw, accV);
  CKL();
  // the gradient tensor in chunks of planes that fit the work arrays
  const int NP = std::max(1, std::min(32, (int)((size_t)n1 * g.nz2 / (3 * (size_t)g.nz))));
  for (int p0 = 0; p0 < n1; p0 += NP) {
    const int np = std::min(NP, n1 - p0);
    k_grad_spec<T><<<grid1d(nw * 3 * np), 256, 0, c->st>>>((const C*)c->vel, m64, (C*)c->T1, g, c->gd, c->pp_wy,
                                                           c->pp_sy, p0, np);
    CKL();
    T* physA = (T*)((C*)c->T2 + (size_t)9 * np * g.nxh * g.nz);
    r = Impl<T>::small_c2r(c, (const C*)c->T1, L, 9 * np, physA, (C*)c->T2);
    if (r) return r;
    k_derived<T><<<dim3(g.nz, np), 128, 0, c->st>>>(physA, (const C*)c->T1, g.nx, g.nz, n1, nw, p0, out, accW);
    CKL();
  }
  return CFG_OK;
}

int cfg_write_vtk_derived(cfg_ctx* c, const char* path) {
  if (!c || !path) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_write_vtk_derived");
  cudaSetDevice(c->dev);
  int r = cfg_wait_io(c);
  if (r) return r;
  r = ensure_postproc(c);
  if (r) return r;
  const Geom& g = c->g;
  const size_t npts = (size_t)g.nx * g.ny1 * g.nz, bytes = npts * 8 * 4;
  r = ensure_io(c, bytes);
  if (r) return r;
  r = c->mixed ? postproc<float>(c, (uint32_t*)c->io_dev) : postproc<double>(c, (uint32_t*)c->io_dev);
  if (r) return r;
  const std::string p(path);
  const cfg_params prm = c->p;
  return start_io(c, bytes, [c, p, prm](std::string& why) {
    return cfd_io::write_vtk(p.c_str(), prm.nx, prm.ny, prm.nz, prm.lx, prm.lz, c->hyh.data(),
                             (const unsigned char*)c->io_host, 1, why);
  });
}

int cfg_plane_statistics(cfg_ctx* c, double* stats) {
  if (!c || !stats) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_plane_statistics");
  cudaSetDevice(c->dev);
  int r = ensure_postproc(c);
  if (r) return r;
  r = c->mixed ? postproc<float>(c, nullptr) : postproc<double>(c, nullptr);
  if (r) return r;
  const int n1 = c->g.ny1;
  std::vector<double> acc(30 * (size_t)n1);
  CK(cudaMemcpyAsync(acc.data(), c->pp_acc, sizeof(double) * acc.size(), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const double scale = 1.0 / ((double)c->g.nx * (double)c->g.nz), eps = 2.220446049250313e-16;
  auto col = [&](int k) { return stats + (size_t)k * n1; };
  for (int j = 0; j < n1; ++j) {
    const double* v = &acc[(size_t)j * 15];
    const double* w = &acc[(size_t)(n1 + j) * 15];
    for (int q = 0; q < 3; ++q) {
      const double var = scale * v[q], var_w = scale * w[q];
      col(q)[j] = v[12 + q];
      col(3 + q)[j] = var;
      col(6 + q)[j] = scale * v[3 + q] / (std::pow(var, 1.5) + eps);
      col(9 + q)[j] = scale * v[6 + q] / (var * var + eps);
      col(12 + q)[j] = scale * v[9 + q];
      col(15 + q)[j] = w[12 + q];
      col(18 + q)[j] = var_w;
      col(21 + q)[j] = scale * w[3 + q] / (std::pow(var_w, 1.5) + eps);
      col(24 + q)[j] = scale * w[6 + q] / (var_w * var_w + eps);
    }
  }
  return CFG_OK;
}

// ---------------------------------------------------------------------------
// init_buffer (PFC/init_jet_buffer.f90:358-483) on the device
int cfg_init_buffer(cfg_ctx* c, const cfg_fringe* f) {
  if (!c || !f) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_init_buffer");
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  if (f->xfringe == 0 && f->zfringe == 0) {
    c->has_fringe = 0;
    return CFG_OK;
  }
  if (!c->fringe && cudaMalloc(&c->fringe, rsize(c) * g.nx2 * g.nz2) != cudaSuccess)
    return fail(c, CFG_E_NOMEM, "fringe buffer");
  FringeParams fp{f->xfringe, f->zfringe, f->frac_xbuff, f->buff_xrise, f->buff_xfall, f->frac_zbuff};
  const size_t np = (size_t)g.nx2 * g.nz2;
  PlaneIn L{0, 0, (size_t)g.nz, 1, 1};
  int r;
  if (c->mixed) {
    using T = float;
    using C = float2;
    k_fringe_profile<T><<<g.nz, 128, 0, c->st>>>((T*)c->pw_phys, fp, g.nx, g.nz, c->p.lx, c->p.lz);
    CKL();
    r = Impl<T>::small_r2c(c, (const T*)c->pw_phys, 1, (C*)c->pw_in, 0, g.nz, 1, (C*)c->pw_H);
    if (r) return r;
    r = Impl<T>::planes_c2r(c, (const C*)c->pw_in, L, nullptr, 1, (T*)c->pw_phys2);
    if (r) return r;
    k_scale_real<T><<<grid1d(np), 256, 0, c->st>>>((const T*)c->pw_phys2, (T*)c->fringe, np, f->fringe_gain);
  } else {
    using T = double;
    using C = double2;
    k_fringe_profile<T><<<g.nz, 128, 0, c->st>>>((T*)c->pw_phys, fp, g.nx, g.nz, c->p.lx, c->p.lz);
    CKL();
    r = Impl<T>::small_r2c(c, (const T*)c->pw_phys, 1, (C*)c->pw_in, 0, g.nz, 1, (C*)c->pw_H);
    if (r) return r;
    r = Impl<T>::planes_c2r(c, (const C*)c->pw_in, L, nullptr, 1, (T*)c->pw_phys2);
    if (r) return r;
    k_scale_real<T><<<grid1d(np), 256, 0, c->st>>>((const T*)c->pw_phys2, (T*)c->fringe, np, f->fringe_gain);
  }
  CKL();
  // target_inflow for the closed channel: 0.75 (1 - yh^8) (cos beta, 0, sin beta)
  const int n1 = g.ny1;
  std::vector<double> tgt(3 * (size_t)n1, 0.0);
  for (int j = 0; j < n1; ++j) {
    const double p = 0.75 * (1.0 - std::pow(c->hyh[j], 8));
    tgt[j] = p * std::cos(c->p.beta);
    tgt[2 * (size_t)n1 + j] = p * std::sin(c->p.beta);
  }
  CK(cudaMemcpyAsync((void*)c->gd.target, tgt.data(), sizeof(double) * tgt.size(), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->has_fringe = 1;
  return CFG_OK;
}

int cfg_get_buffer(cfg_ctx* c, double* buffer, double* target_inflow) {
  if (!c) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_get_buffer");
  cudaSetDevice(c->dev);
  const Geom& g = c->g;
  const size_t np = (size_t)g.nx2 * g.nz2;
  if (buffer) {
    if (!c->has_fringe || !c->fringe) {
      memset(buffer, 0, sizeof(double) * np);
    } else if (c->mixed) {
      std::vector<float> h(np);
      CK(cudaMemcpyAsync(h.data(), c->fringe, sizeof(float) * np, cudaMemcpyDeviceToHost, c->st));
      CK(cudaStreamSynchronize(c->st));
      for (size_t i = 0; i < np; ++i) buffer[i] = h[i];
    } else {
      CK(cudaMemcpyAsync(buffer, c->fringe, sizeof(double) * np, cudaMemcpyDeviceToHost, c->st));
    }
  }
  if (target_inflow)
    CK(cudaMemcpyAsync(target_inflow, c->gd.target, sizeof(double) * 3 * g.ny1, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFG_OK;
}


// ----------------------------------------------------------------------------
// Multi-rank runs: one context per rank, each holding a kx slab of the
// spectral state and a z2 slab of the physical planes (distribute_data,
// PFC/setup.f90:298-437).  The two MPI_ALLTOALLV transposes of the reference's
// x-z transforms (PFC/transform.f90:345-409, 573-690) are the scatter stores
// of k_zinv_r and k_flux_r into the owners' buffers (peer memory when the
// ranks sit on different GPUs); a barrier of events separates the phases.

// what one rank needs of another: where its T1 / T2 / CFL maxima live (a
// pointer valid on this rank's GPU: the peer's own, or an IPC mapping) and
// its slabs
struct PeerView {
  const void *T1, *T2;
  unsigned long long* cfl;
  int x0, nxl, z0, nzl;
};

static PeerView view_of(const cfg_ctx* o) {
  return PeerView{o->T1, o->T2, o->cflbits, o->g.kx0, o->g.nxh, o->z0s, o->gP.nz2};
}

// scatter tables and CFL peer list of rank c from the views of all ranks
static int build_scatter(cfg_ctx* c, const std::vector<PeerView>& v) {
  const int n = (int)v.size(), nz2 = c->g.nz2, nxh = c->g.nxh_all;
  const size_t cs = csize(c);
  std::vector<int> zown(nz2, -1), xown(nxh, -1);
  for (int i = 0; i < n; ++i) {
    for (int z = v[i].z0; z < v[i].z0 + v[i].nzl && z < nz2; ++z) zown[z] = i;
    for (int x = v[i].x0; x < v[i].x0 + v[i].nxl && x < nxh; ++x) xown[x] = i;
  }
  for (int z = 0; z < nz2; ++z)
    if (zown[z] < 0) return fail(c, CFG_E_ARG, "z2 row %d has no owner", z);
  for (int x = 0; x < nxh; ++x)
    if (xown[x] < 0) return fail(c, CFG_E_ARG, "kx column %d has no owner", x);
  std::vector<unsigned long long> tab((size_t)2 * nz2 + 2 * nxh);
  unsigned long long* zdst = tab.data();
  long long* zpitch = reinterpret_cast<long long*>(zdst + nz2);
  unsigned long long* xdst = zdst + 2 * nz2;
  long long* xpitch = reinterpret_cast<long long*>(xdst + nxh);
  for (int z = 0; z < nz2; ++z) {
    const PeerView& o = v[zown[z]];
    zdst[z] = (unsigned long long)((const char*)o.T1 + cs * (size_t)(z - o.z0));
    zpitch[z] = o.nzl;
  }
  for (int x = 0; x < nxh; ++x) {
    const PeerView& o = v[xown[x]];
    xdst[x] = (unsigned long long)((const char*)o.T2 + cs * ((size_t)(x - o.x0) * nz2 + c->z0s));
    xpitch[x] = (long long)o.nxl * nz2;
  }
  std::vector<unsigned long long*> peers;
  for (int i = 0; i < n; ++i)
    if (i != c->rank) peers.push_back(v[i].cfl);
  cudaSetDevice(c->dev);
  if (c->scat_tab) cudaFree(c->scat_tab);
  if (c->cfl_peers) cudaFree(c->cfl_peers);
  c->scat_tab = nullptr;
  c->cfl_peers = nullptr;
  if (cudaMalloc(&c->scat_tab, sizeof(unsigned long long) * tab.size()) != cudaSuccess ||
      cudaMalloc(&c->cfl_peers, sizeof(unsigned long long*) * std::max<size_t>(1, peers.size())) != cudaSuccess)
    return fail(c, CFG_E_NOMEM, "scatter tables");
  CK(cudaMemcpy(c->scat_tab, tab.data(), sizeof(unsigned long long) * tab.size(), cudaMemcpyHostToDevice));
  if (!peers.empty())
    CK(cudaMemcpy(c->cfl_peers, peers.data(), sizeof(unsigned long long*) * peers.size(), cudaMemcpyHostToDevice));
  const unsigned long long* d = (const unsigned long long*)c->scat_tab;
  c->scat.n = n;
  c->scat.zdst = d;
  c->scat.zpitch = reinterpret_cast<const long long*>(d + nz2);
  c->scat.xdst = d + 2 * nz2;
  c->scat.xpitch = reinterpret_cast<const long long*>(d + 2 * nz2 + nxh);
  c->n_cfl_peers = n - 1;
  return CFG_OK;
}

struct cfg_group {
  std::vector<cfg_ctx*> r;
  std::vector<cudaEvent_t> ev;
  std::vector<int> nx_proc, x_start, nz_proc, z_start;
};

int cfg_partition(int nx, int nz, int nz2, int nproc, int* nx_proc, int* x_start, int* nz_proc, int* z_start,
                  int* nz_small_proc, int* z_small_start) {
  if (nx < 2 || nz < 1 || nz2 < nz || nproc < 1) return CFG_E_ARG;
  // the first (n mod nproc) ranks take one more column / row
  const int nxh = nx / 2 + 1;
  const int xl = nxh % nproc, zl = nz2 % nproc, sl = nz % nproc;
  int xs = 0, zs = 0, ss = 0;
  for (int n = 0; n < nproc; ++n) {
    const int a = (nxh - xl) / nproc + (n < xl ? 1 : 0);
    const int b = (nz2 - zl) / nproc + (n < zl ? 1 : 0);
    const int d = (nz - sl) / nproc + (n < sl ? 1 : 0);
    if (nx_proc) nx_proc[n] = a;
    if (x_start) x_start[n] = xs;
    if (nz_proc) nz_proc[n] = b;
    if (z_start) z_start[n] = zs;
    if (nz_small_proc) nz_small_proc[n] = d;
    if (z_small_start) z_small_start[n] = ss;
    xs += a;
    zs += b;
    ss += d;
  }
  return CFG_OK;
}

static int group_barrier(cfg_group* G) {
  const int n = (int)G->r.size();
  if (n < 2) return CFG_OK;
  for (int i = 0; i < n; ++i) {
    cudaSetDevice(G->r[i]->dev);
    if (cudaEventRecord(G->ev[i], G->r[i]->st) != cudaSuccess) return fail(G->r[i], CFG_E_CUDA, "barrier record");
  }
  for (int s = 0; s < n; ++s) {
    cudaSetDevice(G->r[s]->dev);
    for (int i = 0; i < n; ++i)
      if (i != s && cudaStreamWaitEvent(G->r[s]->st, G->ev[i], 0) != cudaSuccess)
        return fail(G->r[s], CFG_E_CUDA, "barrier wait");
  }
  return CFG_OK;
}

void cfg_group_destroy(cfg_group* G) {
  if (!G) return;
  for (size_t i = 0; i < G->r.size(); ++i) {
    if (!G->r[i]) continue;
    cudaSetDevice(G->r[i]->dev);
    cudaStreamSynchronize(G->r[i]->st);
  }
  for (size_t i = 0; i < G->ev.size(); ++i)
    if (G->ev[i]) {
      cudaSetDevice(G->r[i]->dev);
      cudaEventDestroy(G->ev[i]);
    }
  for (cfg_ctx* c : G->r) cfg_destroy(c);
  delete G;
}

int cfg_group_create(const cfg_params* p, const cfg_grid* gr, int nranks, const int* devices, cfg_group** out) {
  if (!p || !gr || !out || nranks < 1 || nranks > 64) return CFG_E_ARG;
  *out = nullptr;
  if (p->ctrlu != 0.0 || p->ctrlw != 0.0) {
    fprintf(stderr, "cfg_group_create: wall feedback (ctrlu, ctrlw) needs a single context\n");
    return CFG_E_ARG;
  }
  cfg_group* G = new cfg_group();
  const int n = nranks;
  G->nx_proc.resize(n); G->x_start.resize(n); G->nz_proc.resize(n); G->z_start.resize(n);
  cfg_partition(p->nx, p->nz, p->nz2, n, G->nx_proc.data(), G->x_start.data(), G->nz_proc.data(), G->z_start.data(),
                nullptr, nullptr);
  for (int i = 0; i < n; ++i) {
    // every rank needs a kx column, and its z2 rows in whole tiles of the
    // x-stage kernels (8 rows)
    if (G->nx_proc[i] < 1 || G->nz_proc[i] < 8 || G->nz_proc[i] % 8 != 0) {
      fprintf(stderr, "cfg_group_create: rank %d gets %d kx columns and %d z2 rows (needs >= 1 and a multiple of 8)\n",
              i, G->nx_proc[i], G->nz_proc[i]);
      delete G;
      return CFG_E_ARG;
    }
  }
  G->r.assign(n, nullptr);
  G->ev.assign(n, nullptr);
  for (int i = 0; i < n; ++i) {
    cfg_params pi = *p;
    pi.device = devices ? devices[i] : p->device;
    SlabPart sp{i, n, G->x_start[i], G->nx_proc[i], G->z_start[i], G->nz_proc[i]};
    int r = create_impl(&pi, gr, &sp, &G->r[i]);
    if (r) { cfg_group_destroy(G); return r; }
    cfg_ctx* c = G->r[i];
    if (n > 1 && !(c->split_x && c->fast_z)) {
      fprintf(stderr, "cfg_group_create: transform lengths %d x %d have no register-FFT kernels\n", p->nx2, p->nz2);
      cfg_group_destroy(G);
      return CFG_E_ARG;
    }
    cudaSetDevice(c->dev);
    if (cudaEventCreateWithFlags(&G->ev[i], cudaEventDisableTiming) != cudaSuccess) {
      cfg_group_destroy(G);
      return CFG_E_CUDA;
    }
  }
  if (n > 1) {
    // peer access between the ranks' GPUs
    for (int s = 0; s < n; ++s)
      for (int i = 0; i < n; ++i) {
        const int ds = G->r[s]->dev, di = G->r[i]->dev;
        if (ds == di) continue;
        int can = 0;
        cudaDeviceCanAccessPeer(&can, ds, di);
        if (!can) {
          fprintf(stderr, "cfg_group_create: GPU %d cannot reach GPU %d\n", ds, di);
          cfg_group_destroy(G);
          return CFG_E_CUDA;
        }
        cudaSetDevice(ds);
        const cudaError_t e = cudaDeviceEnablePeerAccess(di, 0);
        if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) {
          cudaGetLastError();
          fprintf(stderr, "cfg_group_create: peer access %d -> %d failed\n", ds, di);
          cfg_group_destroy(G);
          return CFG_E_CUDA;
        }
        cudaGetLastError();
      }
    std::vector<PeerView> views(n);
    for (int i = 0; i < n; ++i) views[i] = view_of(G->r[i]);
    for (int s = 0; s < n; ++s) {
      const int r = build_scatter(G->r[s], views);
      if (r) { cfg_group_destroy(G); return r; }
    }
  }
  *out = G;
  return CFG_OK;
}

int cfg_group_size(const cfg_group* G) { return G ? (int)G->r.size() : 0; }

cfg_ctx* cfg_group_rank(cfg_group* G, int rank) {
  if (!G || rank < 0 || rank >= (int)G->r.size()) return nullptr;
  return G->r[rank];
}

int cfg_group_timestep(cfg_group* G, int nsteps) {
  if (!G || nsteps < 0) return CFG_E_ARG;
  const int n = (int)G->r.size();
  int r;
  for (int s = 0; s < nsteps; ++s) {
    for (cfg_ctx* c : G->r) {
      cudaSetDevice(c->dev);
      c->step = c->step < 0 ? 1 : c->step + 1;
      if ((r = DISPATCH(c, boundary(c)))) return r;
    }
    for (int rk = 1; rk <= 3; ++rk) {
      for (int ph = 1; ph <= 3; ++ph) {
        for (cfg_ctx* c : G->r) {
          cudaSetDevice(c->dev);
          if ((r = DISPATCH(c, nl_phase(c, c->step, rk, false, ph)))) return r;
          if (ph == 3 && (r = DISPATCH(c, rhs(c, rk, 0)))) return r;
        }
        if (ph < 3 && (r = group_barrier(G))) return r;
      }
    }
    for (cfg_ctx* c : G->r) {
      cudaSetDevice(c->dev);
      prof_begin(c, "k_advance_time");
      k_advance_time<<<1, 1, 0, c->st>>>(c->sc);
      CKL();
    }
  }
  (void)n;
  return CFG_OK;
}

int cfg_group_synchronize(cfg_group* G) {
  if (!G) return CFG_E_ARG;
  for (cfg_ctx* c : G->r) {
    const int r = cfg_synchronize(c);
    if (r) return r;
  }
  return CFG_OK;
}

// ---- one process per rank ---------------------------------------------------
// The same decomposition with each rank in its own process (one per GPU, as
// under mpirun): the ranks exchange CUDA IPC handles of their T1, T2 and CFL
// buffers through the host (any all-gather: MPI, torch.distributed), map the
// others' buffers, and step with a host barrier between the phases.

struct cfg_rank_rec {
  int magic, rank, nranks, x0, nxl, z0, nzl, elem;
  cudaIpcMemHandle_t t1, t2, cfl;
};
static const int RANK_MAGIC = 0x43464752;

size_t cfg_rank_record_size(void) { return sizeof(cfg_rank_rec); }

int cfg_rank_create(const cfg_params* p, const cfg_grid* gr, int rank, int nranks, cfg_ctx** out) {
  if (!p || !gr || !out || nranks < 1 || nranks > 64 || rank < 0 || rank >= nranks) return CFG_E_ARG;
  *out = nullptr;
  if (p->ctrlu != 0.0 || p->ctrlw != 0.0) {
    fprintf(stderr, "cfg_rank_create: wall feedback (ctrlu, ctrlw) needs a single context\n");
    return CFG_E_ARG;
  }
  std::vector<int> nxp(nranks), xs(nranks), nzp(nranks), zs(nranks);
  cfg_partition(p->nx, p->nz, p->nz2, nranks, nxp.data(), xs.data(), nzp.data(), zs.data(), nullptr, nullptr);
  for (int i = 0; i < nranks; ++i)
    if (nxp[i] < 1 || nzp[i] < 8 || nzp[i] % 8 != 0) {
      fprintf(stderr, "cfg_rank_create: rank %d gets %d kx columns and %d z2 rows (needs >= 1 and a multiple of 8)\n",
              i, nxp[i], nzp[i]);
      return CFG_E_ARG;
    }
  SlabPart sp{rank, nranks, xs[rank], nxp[rank], zs[rank], nzp[rank]};
  int r = create_impl(p, gr, &sp, out);
  if (r) return r;
  if (nranks > 1 && !((*out)->split_x && (*out)->fast_z)) {
    fprintf(stderr, "cfg_rank_create: transform lengths %d x %d have no register-FFT kernels\n", p->nx2, p->nz2);
    cfg_destroy(*out);
    *out = nullptr;
    return CFG_E_ARG;
  }
  return CFG_OK;
}

int cfg_rank_export(cfg_ctx* c, void* record) {
  if (!c || !record) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  cfg_rank_rec h{};
  h.magic = RANK_MAGIC; h.rank = c->rank; h.nranks = c->nranks;
  h.x0 = c->g.kx0; h.nxl = c->g.nxh; h.z0 = c->z0s; h.nzl = c->gP.nz2; h.elem = (int)csize(c);
  CK(cudaIpcGetMemHandle(&h.t1, c->T1));
  CK(cudaIpcGetMemHandle(&h.t2, c->T2));
  CK(cudaIpcGetMemHandle(&h.cfl, c->cflbits));
  memcpy(record, &h, sizeof(h));
  return CFG_OK;
}

int cfg_rank_connect(cfg_ctx* c, const void* records) {
  if (!c || !records) return CFG_E_ARG;
  if (c->scat.n != 0 || !c->ipc_open.empty()) return fail(c, CFG_E_STATE, "cfg_rank_connect: already connected");
  cudaSetDevice(c->dev);
  const int n = c->nranks;
  std::vector<cfg_rank_rec> h(n);
  memcpy(h.data(), records, sizeof(cfg_rank_rec) * n);
  std::vector<PeerView> v(n);
  for (int i = 0; i < n; ++i) {
    if (h[i].magic != RANK_MAGIC || h[i].rank != i || h[i].nranks != n || h[i].elem != (int)csize(c))
      return fail(c, CFG_E_ARG, "rank record %d does not belong to this run", i);
    if (i == c->rank) {
      v[i] = view_of(c);
      continue;
    }
    void* m[3] = {nullptr, nullptr, nullptr};
    const cudaIpcMemHandle_t* hh[3] = {&h[i].t1, &h[i].t2, &h[i].cfl};
    for (int k = 0; k < 3; ++k) {
      CK(cudaIpcOpenMemHandle(&m[k], *hh[k], cudaIpcMemLazyEnablePeerAccess));
      c->ipc_open.push_back(m[k]);
    }
    v[i] = PeerView{m[0], m[1], (unsigned long long*)m[2], h[i].x0, h[i].nxl, h[i].z0, h[i].nzl};
  }
  return build_scatter(c, v);
}

static int rank_timestep(cfg_ctx* c, int nsteps, cfg_barrier_fn barrier, void* user, bool host_sync) {
  if (!c || nsteps < 0 || (c->nranks > 1 && (!barrier || !c->scat.n))) return CFG_E_ARG;
  cudaSetDevice(c->dev);
  int r;
  for (int s = 0; s < nsteps; ++s) {
    c->step = c->step < 0 ? 1 : c->step + 1;
    if ((r = DISPATCH(c, boundary(c)))) return r;
    for (int rk = 1; rk <= 3; ++rk)
      for (int ph = 1; ph <= 3; ++ph) {
        if ((r = DISPATCH(c, nl_phase(c, c->step, rk, false, ph)))) return r;
        if (ph == 3) {
          if ((r = DISPATCH(c, rhs(c, rk, 0)))) return r;
        } else if (c->nranks > 1) {
          // host barrier: this rank's stores into the others' buffers are
          // complete, then every rank's; stream-ordered barrier: the callback
          // enqueues it on this context's stream
          if (host_sync) CK(cudaStreamSynchronize(c->st));
          if (barrier(user) != 0) return fail(c, CFG_E_ARG, "barrier callback failed");
        }
      }
    prof_begin(c, "k_advance_time");
    k_advance_time<<<1, 1, 0, c->st>>>(c->sc);
    CKL();
  }
  return CFG_OK;
}


// ---- launch-shape autotuner ------------------------------------------------
// Tries the tile parameters of the step's kernels on this context's own
// grid -- warps per k_rhs2 block, z rows per k_flux_r block, planes per
// k_zinv_r / k_zfwd_r block -- one at a time (coordinate descent), timing a
// few steps of the real state with CUDA events, and keeps the fastest.  The
// state, the scalars, the wall values and the jet walk are restored after
// every trial, so the run continues as if nothing had happened.  Every
// choice gives the same results bit for bit (each wavenumber, row and plane
// goes through the same arithmetic whatever the tile), only the time differs.

struct TuneSnap {
  std::vector<std::pair<void*, void*>> bufs;   // (live, copy)
  std::vector<size_t> bytes;
};

static int snap_take(cfg_ctx* c, TuneSnap& s) {
  const Geom& g = c->g;
  const size_t cs = csize(c), nf = (size_t)g.nw * 3 * g.ny1;
  std::vector<std::pair<void*, size_t>> live = {
      {c->vel, cs * nf}, {c->cru, cs * nf}, {c->prs, cs * (size_t)g.nw * g.ny1}, {c->cbc, cs * 6 * (size_t)g.nw},
      {c->sc, sizeof(DevScalars)}, {c->d_um_dy, sizeof(double) * g.ny}};
  if (c->mvel64) live.push_back({c->mvel64, sizeof(double2) * 3 * g.ny1});
  if (c->mcru64) live.push_back({c->mcru64, sizeof(double2) * 3 * g.ny1});
  if (c->jst) live.push_back({c->jst, sizeof(JetState)});
  for (auto& l : live) {
    void* d = nullptr;
    if (cudaMalloc(&d, l.second) != cudaSuccess) return fail(c, CFG_E_NOMEM, "autotune snapshot");
    s.bufs.push_back({l.first, d});
    s.bytes.push_back(l.second);
    CK(cudaMemcpyAsync(d, l.first, l.second, cudaMemcpyDeviceToDevice, c->st));
  }
  return CFG_OK;
}
static int snap_restore(cfg_ctx* c, TuneSnap& s) {
  for (size_t i = 0; i < s.bufs.size(); ++i)
    CK(cudaMemcpyAsync(s.bufs[i].first, s.bufs[i].second, s.bytes[i], cudaMemcpyDeviceToDevice, c->st));
  return CFG_OK;
}
static void snap_free(TuneSnap& s) {
  for (auto& b : s.bufs) cudaFree(b.second);
  s.bufs.clear();
}

int cfg_autotune(cfg_ctx* c, int trial_steps, int* choice) {
  if (!c || trial_steps < 1) return CFG_E_ARG;
  if (c->nranks > 1) return single_only(c, "cfg_autotune");
  if (c->prof_on) return fail(c, CFG_E_STATE, "cfg_autotune: profiling is on");
  cudaSetDevice(c->dev);
  CK(cudaStreamSynchronize(c->st));
  TuneSnap snap;
  int r = snap_take(c, snap);
  if (r) { snap_free(snap); return r; }
  const int step0 = c->step;
  const long long launches0 = c->launches;
  const bool mean_ok = c->mean64_valid;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // one trial: restore, one untimed step, trial_steps timed steps; a
  // failing launch or a device error flag disqualifies the setting
  auto trial = [&]() -> float {
    if (snap_restore(c, snap)) return -1.f;
    c->step = step0;
    if (step_enqueue(c, false)) { cudaGetLastError(); return -1.f; }
    cudaEventRecord(e0, c->st);
    for (int i = 0; i < trial_steps; ++i)
      if (step_enqueue(c, false)) { cudaGetLastError(); cudaStreamSynchronize(c->st); return -1.f; }
    cudaEventRecord(e1, c->st);
    if (cudaEventSynchronize(e1) != cudaSuccess) { cudaGetLastError(); return -1.f; }
    DevScalars h;
    cudaMemcpy(&h, c->sc, sizeof(h), cudaMemcpyDeviceToHost);
    if (h.status != 0) return -1.f;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
  };
  float best = trial();
  if (best < 0.f) {
    snap_restore(c, snap);
    cudaStreamSynchronize(c->st);
    snap_free(snap);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->step = step0;
    c->launches = launches0;
    return fail(c, CFG_E_STATE, "cfg_autotune: the current settings do not run");
  }
  const bool f32 = c->mixed;
  auto tune = [&](int* knob, std::initializer_list<int> vals) {
    const int keep = *knob;
    int bestv = keep;
    for (int v : vals) {
      if (v == keep) continue;
      *knob = v;
      const float t = trial();
      if (t >= 0.f && t < best) { best = t; bestv = v; }
    }
    *knob = bestv;
  };
  if (c->use_rhs2) {
    if (f32) tune(&c->rhs2_warps, {2, 3, 4});
    else tune(&c->rhs2_warps, {1, 2});
  }

  // a row count that does not split, or the 8-row block outside the
  // FP32 nonlinear products, fails its trial
  if (c->split_x) tune(&c->flux_zr, {2, 4, 8});
  if (c->fast_z) {
    // planes per z-transform block (a block too large for its launch fails
    // its trial)
    tune(&c->fYB1, {1, 2, 3, 4, 6, 8});
    tune(&c->fYB3, {1, 2, 3, 4, 6, 8});
  }
  // z2 rows per inverse-x block (not one of the four public tiles; a row
  // count that does not divide the slab fails its trial)
  if (c->split_x) tune(&c->xinv_zb, {8, 16, 24});
  snap_restore(c, snap);
  CK(cudaStreamSynchronize(c->st));
  snap_free(snap);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->step = step0;
  c->launches = launches0;
  c->mean64_valid = mean_ok;
  if (choice) {
    choice[0] = c->rhs2_warps;
    choice[1] = c->flux_zr;
    choice[2] = c->fYB1;
    choice[3] = c->fYB3;
  }
  return CFG_OK;
}

int cfg_get_tiles(const cfg_ctx* c, int* tiles) {
  if (!c || !tiles) return CFG_E_ARG;
  tiles[0] = c->rhs2_warps;
  tiles[1] = c->flux_zr;
  tiles[2] = c->fYB1;
  tiles[3] = c->fYB3;
  return CFG_OK;
}

int cfg_set_tiles(cfg_ctx* c, const int* tiles) {
  if (!c || !tiles) return CFG_E_ARG;
  const int w = tiles[0], fz = tiles[1], y1 = tiles[2], y3 = tiles[3];
  if (w < 1 || w > 4 || (fz != 2 && fz != 4 && !(fz == 8 && c->mixed)) || y1 < 1 || y1 > 8 || y3 < 1 || y3 > 8 ||
      (c->split_x && c->gP.nz2 % fz != 0))
    return fail(c, CFG_E_ARG, "cfg_set_tiles: unsupported tiles");
  c->rhs2_warps = w;
  c->flux_zr = fz;
  c->fYB1 = y1;
  c->fYB3 = y3;
  return CFG_OK;
}

// ---- ensembles: many independent contexts stepped by one graph ------------
// Configuration C5: members of different grids, Reynolds numbers, seeds and
// forcing on one GPU.  One time step of every member is captured once into a
// CUDA graph, so a step of the whole ensemble is one graph launch.  Two ways
// to lay the step out:
//   batched (the default where every member allows it): the members fall
//     into classes of the same grid and launch tiles, and every kernel of
//     the step runs once per class -- blockIdx.x runs over the class's
//     members, each member's arguments come from a table in device memory
//     (the *_b kernels of pass1_fast.inc, pass2v2.cu and below) -- one
//     branch of the graph per class;
//   branches: each member's step on its own branch, forked from and joined
//     to the ensemble stream.
// The arithmetic is the same either way: the batched kernels run the same
// bodies on the same arguments.

// per-member arguments of the batched small kernels (mixed precision)
struct EnsMember {
  // substep prologue: the mean-split base and the CFL maxima
  const double2* m64;
  const float2* v32;
  double* base;
  int ny1, split;
  unsigned long long* cflbits;
  // boundary: the wall values, zeroed at every step
  float2* cbc;
  size_t ncbc;
  // check_cfl and the dt update
  Geom g;
  GridDev gd;
  DevScalars* sc;
  double* cflp;
  double lx, lz, cfl_max;
  int dt_flag;
};

// per-member arguments of the batched wall jet (members with crossflow)
struct EnsJet {
  JetState* st;
  JetParams jp;
  const DevScalars* sc;
  RkTab rkt;
  float* phys;
  float2 *H, *spec, *cbc;
  GridDev gd;
  FftPlan px, pz;
  const float2 *twx, *twz;
  int nx, nz, nxh;
  size_t nw;
  double lx, lz;
};

// k_mean_base and, at rk 1, the zeroed CFL maxima of every member; one block
// per member
__global__ void k_ens_prologue(const EnsMember* __restrict__ tab, int do_cfl) {
  const EnsMember& a = tab[blockIdx.x];
  const int n = 3 * a.ny1;
  if (a.split)
    for (int i = threadIdx.x; i < n; i += blockDim.x) a.base[i] = a.m64 ? a.m64[i].x : (double)a.v32[i].x;
  if (do_cfl)
    for (int i = threadIdx.x; i < n; i += blockDim.x) a.cflbits[i] = 0ull;
}

// the wall values zeroed (boundary without feedback); grid (blocks, members)
__global__ void k_ens_zero_cbc(const EnsMember* __restrict__ tab) {
  const EnsMember& a = tab[blockIdx.y];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.ncbc; i += (size_t)gridDim.x * blockDim.x)
    a.cbc[i] = make_float2(0.f, 0.f);
}

__global__ void k_cfl_finalize_b(const EnsMember* __restrict__ tab, int step) {
  const EnsMember& a = tab[blockIdx.x];
  k_cfl_finalize_body<false>(make_uint3(0, 0, 0), a.cflbits, a.g, a.gd, a.sc, a.cflp, a.lx, a.lz, a.dt_flag,
                             a.cfl_max, step);
}

__global__ void k_ens_advance(const EnsMember* __restrict__ tab, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) tab[m].sc->t_total = tab[m].sc->t_total + tab[m].sc->dt;
}

__global__ void k_jet_walk_b(const EnsJet* __restrict__ tab, int rk) {
  const EnsJet& a = tab[blockIdx.x];
  k_jet_walk_body(make_uint3(0, 0, 0), a.st, a.jp, a.sc, a.rkt, rk, 0.0, 0.0, 1);
}

__global__ void k_jet_field_b(const EnsJet* __restrict__ tab, unsigned gx) {
  const unsigned m = blockIdx.x / gx;
  const EnsJet& a = tab[m];
  k_jet_field_body<float>(make_uint3(blockIdx.x - m * gx, blockIdx.y, 0), a.phys, a.jp, a.st, a.nx, a.nz, a.lx,
                          a.lz);
}

__global__ void k_px_fwd_b(const EnsJet* __restrict__ tab, unsigned gx) {
  const unsigned m = blockIdx.x / gx;
  const EnsJet& a = tab[m];
  k_px_fwd_body<float>(make_uint3(blockIdx.x - m * gx, blockIdx.y, 0), a.phys, a.H, a.nxh, a.nz, a.nx, a.px, a.twx);
}

__global__ void k_pz_fwd_b(const EnsJet* __restrict__ tab, unsigned gx) {
  const unsigned m = blockIdx.x / gx;
  const EnsJet& a = tab[m];
  const float scale = (float)(1.0 / ((double)a.nx * (double)a.nz));
  k_pz_fwd_body<float>(make_uint3(blockIdx.x - m * gx, blockIdx.y, 0), a.H, a.spec, a.nw, (size_t)a.nz, 1, a.nxh,
                       a.nz, a.nz, 0, scale, a.pz, a.twz);
}

__global__ void k_jet_combine_b(const EnsJet* __restrict__ tab, unsigned gx) {
  const unsigned m = blockIdx.x / gx;
  const EnsJet& a = tab[m];
  k_jet_combine_body<float>(make_uint3(blockIdx.x - m * gx, 0, 0), a.spec, a.cbc, a.jp, a.gd, a.nx, a.nz, a.nxh,
                            a.lx, a.lz);
}

// one class of a batched ensemble: members with the same grid and tiles
struct EnsClass {
  std::vector<int> mem, jet;   // member indices; those with the wall jet
  cudaStream_t st = nullptr, st2 = nullptr, st3 = nullptr;
  cudaEvent_t ev_start = nullptr, ev_fork = nullptr, ev_j2 = nullptr, ev_j3 = nullptr, ev_done = nullptr;
  void* dtab = nullptr;        // every table below, one allocation
  P1Launch *zinv = nullptr, *xinv = nullptr, *zfwd = nullptr, *flux[3] = {};
  Rhs2Launch *r2[3] = {}, *r2p[3] = {};
  RhsMeanLaunch* rm[3] = {};
  EnsMember* sm = nullptr;
  EnsJet* jt = nullptr;
  // the first member's records: launch shapes, on the class's streams
  P1Launch h_zinv{}, h_xinv{}, h_zfwd{}, h_flux[3] = {};
  Rhs2Launch h_r2[3] = {}, h_r2p[3] = {};
  RhsMeanLaunch h_rm[3] = {};
  int nx = 0, nz = 0, nxh = 0, nx2 = 0, nz2 = 0;
  size_t ncbc = 0;
};

struct cfg_ensemble {
  std::vector<cfg_ctx*> m;
  int dev = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_done;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<long long> launches_per_step;
  bool batched = false;        // step layout of the next capture
  bool last_batched = false;   // layout of the last enqueued step
  std::vector<EnsClass> cls;   // batched: the classes (built on first use)
};

static void ens_free_classes(cfg_ensemble* e) {
  for (EnsClass& k : e->cls) {
    if (k.dtab) cudaFree(k.dtab);
    for (cudaEvent_t v : {k.ev_start, k.ev_fork, k.ev_j2, k.ev_j3, k.ev_done})
      if (v) cudaEventDestroy(v);
    for (cudaStream_t v : {k.st, k.st2, k.st3})
      if (v) cudaStreamDestroy(v);
  }
  e->cls.clear();
}

static void ens_drop_graph(cfg_ensemble* e) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->exec = nullptr;
  e->graph = nullptr;
}

void cfg_ensemble_destroy(cfg_ensemble* e) {
  if (!e) return;
  cudaSetDevice(e->dev);
  if (e->st) cudaStreamSynchronize(e->st);
  ens_drop_graph(e);
  ens_free_classes(e);
  for (cudaEvent_t v : e->ev_done) cudaEventDestroy(v);
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  if (e->st) cudaStreamDestroy(e->st);
  delete e;
}

// whether a member's step can run in the batched layout
static bool ens_batchable(const cfg_ctx* c) {
  return c->mixed && c->nranks == 1 && c->g.kx0 == 0 && c->split_x && c->fast_z && c->use_rhs2 && c->rhs2_tbl64 &&
         c->n_fast > 0 && !c->les_on && c->p.ctrlu == 0.0 && c->p.ctrlw == 0.0 && !c->prof_on;
}

// same class: everything that sets a batched launch's shape or kernel
static bool ens_same_class(const cfg_ctx* a, const cfg_ctx* b) {
  const Geom &x = a->g, &y = b->g;
  return x.nx == y.nx && x.ny == y.ny && x.nz == y.nz && x.nx2 == y.nx2 && x.nz2 == y.nz2 && x.nxh == y.nxh &&
         x.ny1 == y.ny1 && x.nw == y.nw && a->gP.nz2 == b->gP.nz2 && a->fYB1 == b->fYB1 && a->fYB3 == b->fYB3 &&
         a->flux_zr == b->flux_zr && a->rhs2_warps == b->rhs2_warps && a->rhs2_lanes == b->rhs2_lanes &&
         a->mean_split == b->mean_split && a->n_fast == b->n_fast && a->n_prec == b->n_prec &&
         a->xinv_zb == b->xinv_zb;
}

// the classes, their streams and their member tables
static int ens_build_classes(cfg_ensemble* e) {
  using I = Impl<float>;
  ens_free_classes(e);
  for (int i = 0; i < (int)e->m.size(); ++i) {
    bool placed = false;
    for (EnsClass& k : e->cls)
      if (ens_same_class(e->m[k.mem[0]], e->m[i])) {
        k.mem.push_back(i);
        placed = true;
        break;
      }
    if (!placed) {
      e->cls.emplace_back();
      e->cls.back().mem.push_back(i);
    }
  }
  for (EnsClass& k : e->cls) {
    for (int i : k.mem)
      if (e->m[i]->crossflow) k.jet.push_back(i);
    bool ok = true;
    for (cudaStream_t* v : {&k.st, &k.st2, &k.st3})
      ok = ok && cudaStreamCreateWithFlags(v, cudaStreamNonBlocking) == cudaSuccess;
    for (cudaEvent_t* v : {&k.ev_start, &k.ev_fork, &k.ev_j2, &k.ev_j3, &k.ev_done})
      ok = ok && cudaEventCreateWithFlags(v, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) return CFG_E_CUDA;
    const int n = (int)k.mem.size(), nj = (int)k.jet.size();
    std::vector<P1Launch> zinv(n), xinv(n), zfwd(n), flux(3 * n);
    std::vector<Rhs2Launch> r2(3 * n), r2p(3 * n);
    std::vector<RhsMeanLaunch> rm(3 * n);
    std::vector<EnsMember> sm(n);
    std::vector<EnsJet> jt(nj);
    for (int q = 0; q < n; ++q) {
      const cfg_ctx* c = e->m[k.mem[q]];
      zinv[q] = I::p1_args(c, 1, false, 0);
      xinv[q] = I::p1_args(c, 1, false, 3);
      zfwd[q] = I::p1_args(c, 1, false, 2);
      for (int rk = 1; rk <= 3; ++rk) {
        flux[(rk - 1) * n + q] = I::p1_args(c, rk, false, 4);
        r2[(rk - 1) * n + q] = I::rhs2_args(c, rk, false);
        r2p[(rk - 1) * n + q] = I::rhs2_args(c, rk, true);
        rm[(rk - 1) * n + q] = I::mean_args(c, rk);
      }
      EnsMember& a = sm[q];
      a.m64 = c->mvel64;
      a.v32 = (const float2*)c->vel;
      a.base = c->mean_base;
      a.ny1 = c->g.ny1;
      a.split = (c->mean_split && !c->les_on) ? 1 : 0;
      a.cflbits = c->cflbits;
      a.cbc = (float2*)c->cbc;
      a.ncbc = 6 * (size_t)c->g.nw;
      a.g = c->g;
      a.gd = c->gd;
      a.sc = c->sc;
      a.cflp = c->cflp;
      a.lx = c->p.lx;
      a.lz = c->p.lz;
      a.cfl_max = c->p.cfl_max;
      a.dt_flag = c->p.dt_flag;
    }
    for (int q = 0; q < nj; ++q) {
      const cfg_ctx* c = e->m[k.jet[q]];
      EnsJet& a = jt[q];
      a.st = c->jst;
      a.jp = c->jp;
      a.sc = c->sc;
      a.rkt = c->rkt;
      a.phys = (float*)c->pw_phys;
      a.H = (float2*)c->pw_H;
      a.spec = (float2*)c->pw_in;
      a.cbc = (float2*)c->cbc;
      a.gd = c->gd;
      a.px = c->pxs;
      a.pz = c->pzs;
      a.twx = (const float2*)c->twxs;
      a.twz = (const float2*)c->twzs;
      a.nx = c->g.nx;
      a.nz = c->g.nz;
      a.nxh = c->g.nxh;
      a.nw = (size_t)c->g.nw;
      a.lx = c->p.lx;
      a.lz = c->p.lz;
    }
    // one device allocation, 256-byte aligned pieces
    size_t off = 0;
    auto take = [&](size_t bytes) {
      const size_t o = off;
      off += (bytes + 255) & ~(size_t)255;
      return o;
    };
    const size_t o_zinv = take(sizeof(P1Launch) * n), o_xinv = take(sizeof(P1Launch) * n),
                 o_zfwd = take(sizeof(P1Launch) * n), o_flux = take(sizeof(P1Launch) * 3 * n),
                 o_r2 = take(sizeof(Rhs2Launch) * 3 * n), o_r2p = take(sizeof(Rhs2Launch) * 3 * n),
                 o_rm = take(sizeof(RhsMeanLaunch) * 3 * n), o_sm = take(sizeof(EnsMember) * n),
                 o_jt = take(sizeof(EnsJet) * (nj > 0 ? nj : 1));
    if (cudaMalloc(&k.dtab, off) != cudaSuccess) {
      cudaGetLastError();
      k.dtab = nullptr;
      return CFG_E_NOMEM;
    }
    char* b = (char*)k.dtab;
    auto put = [&](size_t o, const void* src, size_t bytes) {
      return bytes == 0 || cudaMemcpy(b + o, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    ok = put(o_zinv, zinv.data(), sizeof(P1Launch) * n) && put(o_xinv, xinv.data(), sizeof(P1Launch) * n) &&
         put(o_zfwd, zfwd.data(), sizeof(P1Launch) * n) && put(o_flux, flux.data(), sizeof(P1Launch) * 3 * n) &&
         put(o_r2, r2.data(), sizeof(Rhs2Launch) * 3 * n) && put(o_r2p, r2p.data(), sizeof(Rhs2Launch) * 3 * n) &&
         put(o_rm, rm.data(), sizeof(RhsMeanLaunch) * 3 * n) && put(o_sm, sm.data(), sizeof(EnsMember) * n) &&
         put(o_jt, jt.data(), sizeof(EnsJet) * nj);
    if (!ok) return CFG_E_CUDA;
    k.zinv = (P1Launch*)(b + o_zinv);
    k.xinv = (P1Launch*)(b + o_xinv);
    k.zfwd = (P1Launch*)(b + o_zfwd);
    for (int r = 0; r < 3; ++r) {
      k.flux[r] = (P1Launch*)(b + o_flux) + r * n;
      k.r2[r] = (Rhs2Launch*)(b + o_r2) + r * n;
      k.r2p[r] = (Rhs2Launch*)(b + o_r2p) + r * n;
      k.rm[r] = (RhsMeanLaunch*)(b + o_rm) + r * n;
      k.h_flux[r] = flux[r * n];
      k.h_flux[r].st = k.st;
      k.h_r2[r] = r2[r * n];
      k.h_r2[r].st = k.st;
      k.h_r2p[r] = r2p[r * n];
      k.h_r2p[r].st = k.st2;
      k.h_rm[r] = rm[r * n];
      k.h_rm[r].st = k.st3;
    }
    k.sm = (EnsMember*)(b + o_sm);
    k.jt = (EnsJet*)(b + o_jt);
    k.h_zinv = zinv[0];
    k.h_zinv.st = k.st;
    k.h_xinv = xinv[0];
    k.h_xinv.st = k.st;
    k.h_zfwd = zfwd[0];
    k.h_zfwd.st = k.st;
    const cfg_ctx* c0 = e->m[k.mem[0]];
    k.nx = c0->g.nx;
    k.nz = c0->g.nz;
    k.nxh = c0->g.nxh;
    k.nx2 = c0->g.nx2;
    k.nz2 = c0->g.nz2;
    k.ncbc = 6 * (size_t)c0->g.nw;
  }
  return CFG_OK;
}

// one time step of one class: the sequence of step_enqueue (boundary, three
// nonlinear + rhs substeps, t_total += dt), each kernel once for all members
static int ens_class_enqueue(cfg_ensemble* e, EnsClass& k) {
  const int n = (int)k.mem.size(), nj = (int)k.jet.size();
  cfg_ctx* c0 = e->m[k.mem[0]];
  int launches = 0;
  auto ck = [&](bool ok, const char* what) {
    return ok && cudaGetLastError() == cudaSuccess ? 0 : fail(c0, CFG_E_CUDA, "%s", what);
  };
  const unsigned zb = (unsigned)std::min<size_t>(64, (k.ncbc + 255) / 256);
  k_ens_zero_cbc<<<dim3(zb, n), 256, 0, k.st>>>(k.sm);
  ++launches;
  if (int r = ck(true, "batched boundary")) return r;
  for (int rk = 1; rk <= 3; ++rk) {
    k_ens_prologue<<<n, 256, 0, k.st>>>(k.sm, rk == 1);
    ++launches;
    if (int r = ck(true, "batched substep prologue")) return r;
    if (int r = ck(p1_fast_launch_batch(0, k.nz2, true, k.h_zinv, k.zinv, n) == 0, "batched k_zinv_r")) return r;
    if (int r = ck(p1_fast_launch_batch(3, k.nx2, true, k.h_xinv, k.xinv, n) == 0, "batched k_xinv_r")) return r;
    if (int r = ck(p1_fast_launch_batch(4, k.nx2, true, k.h_flux[rk - 1], k.flux[rk - 1], n) == 0, "batched k_flux_r"))
      return r;
    if (int r = ck(p1_fast_launch_batch(2, k.nz2, true, k.h_zfwd, k.zfwd, n) == 0, "batched k_zfwd_r")) return r;
    launches += 4;
    if (rk == 1) {
      k_cfl_finalize_b<<<n, 256, 0, k.st>>>(k.sm, c0->step);
      ++launches;
      if (int r = ck(true, "batched k_cfl_finalize")) return r;
    }
    if (nj > 0) {
      // the wall jet of this substep (PFC/pass2.f90:41-43); beside the
      // nonlinear term on a side stream (from rk 2, when dt is final) it
      // measured slower: 8.70 against 8.62 ms per 64-member step
      k_jet_walk_b<<<nj, 32, 0, k.st>>>(k.jt, rk);
      k_jet_field_b<<<dim3(k.nz * nj, 3), 128, 0, k.st>>>(k.jt, (unsigned)k.nz);
      const unsigned gxx = (unsigned)(k.nz + 1) / 2;
      k_px_fwd_b<<<dim3(gxx * nj, 3), 128, sizeof(float2) * 3 * k.nx, k.st>>>(k.jt, gxx);
      k_pz_fwd_b<<<dim3((unsigned)k.nxh * nj, 3), 128, sizeof(float2) * 3 * k.nz, k.st>>>(k.jt, (unsigned)k.nxh);
      const unsigned gxc = (unsigned)((k.ncbc / 6 + 255) / 256);
      k_jet_combine_b<<<gxc * nj, 256, 0, k.st>>>(k.jt, gxc);
      launches += 5;
      if (int r = ck(true, "batched wall jet")) return r;
    }
    // the FP64 |k| < 4 list and the mean mode beside the main kernel
    if (int r = ck(cudaEventRecord(k.ev_fork, k.st) == cudaSuccess &&
                       cudaStreamWaitEvent(k.st2, k.ev_fork, 0) == cudaSuccess &&
                       cudaStreamWaitEvent(k.st3, k.ev_fork, 0) == cudaSuccess,
                   "batched fork"))
      return r;
    if (k.h_r2p[rk - 1].nlist > 0) {
      if (int r = ck(rhs2_launch_prec_batch(k.h_r2p[rk - 1], k.r2p[rk - 1], n) == 0, "batched k_rhs2 (FP64 list)"))
        return r;
      ++launches;
    }
    if (int r = ck(rhs_mean2_launch_batch(true, k.h_rm[rk - 1], k.rm[rk - 1], n) == 0, "batched k_rhs_mean2")) return r;
    if (int r = ck(rhs2_launch_batch(true, k.h_r2[rk - 1], k.r2[rk - 1], n) == 0, "batched k_rhs2")) return r;
    launches += 2;
    if (int r = ck(cudaEventRecord(k.ev_j2, k.st2) == cudaSuccess && cudaEventRecord(k.ev_j3, k.st3) == cudaSuccess &&
                       cudaStreamWaitEvent(k.st, k.ev_j2, 0) == cudaSuccess &&
                       cudaStreamWaitEvent(k.st, k.ev_j3, 0) == cudaSuccess,
                   "batched join"))
      return r;
  }
  k_ens_advance<<<(n + 63) / 64, 64, 0, k.st>>>(k.sm, n);
  ++launches;
  if (int r = ck(true, "batched advance time")) return r;
  // the members' host bookkeeping, as step_enqueue keeps it (the batched
  // launches are shared: each member is credited with its share)
  for (int q = 0; q < n; ++q) {
    cfg_ctx* c = e->m[k.mem[q]];
    c->step = c->step < 0 ? 1 : c->step + 1;
    c->mean64_valid = true;
    c->launches += (launches + q) / n;
  }
  return CFG_OK;
}

static int ens_batched_enqueue(cfg_ensemble* e) {
  if (e->cls.empty()) {
    const int r = ens_build_classes(e);
    if (r) return r;
  }
  if (cudaEventRecord(e->ev_fork, e->st) != cudaSuccess) return CFG_E_CUDA;
  for (EnsClass& k : e->cls) {
    if (cudaStreamWaitEvent(k.st, e->ev_fork, 0) != cudaSuccess) return CFG_E_CUDA;
    const int r = ens_class_enqueue(e, k);
    if (r) return r;
    if (cudaEventRecord(k.ev_done, k.st) != cudaSuccess || cudaStreamWaitEvent(e->st, k.ev_done, 0) != cudaSuccess)
      return CFG_E_CUDA;
  }
  return CFG_OK;
}

// The launch tiles of a batched ensemble, tuned per class on the batched
// step of the whole ensemble: coordinate descent over warps per rhs block,
// z rows per flux block, planes per z-transform block and z rows per
// inverse-x block, one class at a time, every member's state, scalars, wall
// values and jet walk restored before each trial and at the end.  A setting whose launch fails or that sets a device error flag is
// skipped.
static int ens_tune_batched(cfg_ensemble* e, int trial_steps) {
  const int n = (int)e->m.size();
  int r = ens_build_classes(e);
  if (r) return r;
  std::vector<std::vector<int>> groups;
  for (const EnsClass& k : e->cls) groups.push_back(k.mem);
  std::vector<TuneSnap> snaps(n);
  std::vector<int> step0(n);
  std::vector<long long> launches0(n);
  for (int i = 0; i < n && !r; ++i) {
    cfg_ctx* c = e->m[i];
    step0[i] = c->step;
    launches0[i] = c->launches;
    r = snap_take(c, snaps[i]);
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!r && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) r = CFG_E_CUDA;
  if (!r && cudaDeviceSynchronize() != cudaSuccess) r = CFG_E_CUDA;
  // one trial of class q's current tiles: the whole batched step, every
  // class at once as the graph runs them, so that a class's tiles are judged
  // by what they cost beside the others (alone, a small class favours many
  // small blocks that only fill an otherwise idle GPU)
  auto trial = [&](int q) -> float {
    for (int i = 0; i < n; ++i) {
      snap_restore(e->m[i], snaps[i]);
      e->m[i]->step = step0[i];
    }
    if (cudaDeviceSynchronize() != cudaSuccess || ens_build_classes(e)) {
      cudaGetLastError();
      return -1.f;
    }
    bool found = false;
    for (const EnsClass& x : e->cls) found = found || x.mem == groups[q];
    if (!found) return -1.f;
    bool ok = ens_batched_enqueue(e) == CFG_OK && cudaEventRecord(e0, e->st) == cudaSuccess;
    for (int s = 0; s < trial_steps && ok; ++s) ok = ens_batched_enqueue(e) == CFG_OK;
    ok = ok && cudaEventRecord(e1, e->st) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      cudaDeviceSynchronize();
      cudaGetLastError();
      return -1.f;
    }
    for (int i = 0; i < n; ++i) {
      DevScalars h;
      if (cudaMemcpy(&h, e->m[i]->sc, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess || h.status != 0) return -1.f;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
  };
  for (int q = 0; q < (int)groups.size() && !r; ++q) {
    float best = trial(q);
    if (best < 0.f) continue;   // the class keeps its tiles
    auto tune = [&](int cfg_ctx::*knob, std::initializer_list<int> vals) {
      const int keep = e->m[groups[q][0]]->*knob;
      int bestv = keep;
      for (int v : vals) {
        if (v == keep) continue;
        for (int i : groups[q]) e->m[i]->*knob = v;
        const float t = trial(q);
        if (t >= 0.f && t < best) {
          best = t;
          bestv = v;
        }
      }
      for (int i : groups[q]) e->m[i]->*knob = bestv;
    };
    tune(&cfg_ctx::rhs2_warps, {2, 3, 4});
    tune(&cfg_ctx::flux_zr, {2, 4, 8});
    tune(&cfg_ctx::fYB1, {1, 2, 3, 4, 6, 8});
    tune(&cfg_ctx::fYB3, {1, 2, 3, 4, 6, 8});
    tune(&cfg_ctx::xinv_zb, {8, 16, 24});
  }
  for (int i = 0; i < n; ++i) {
    cfg_ctx* c = e->m[i];
    if (!snaps[i].bufs.empty()) snap_restore(c, snaps[i]);
    c->step = step0[i];
    c->launches = launches0[i];
    c->mean64_valid = true;
  }
  if (cudaDeviceSynchronize() != cudaSuccess && !r) r = CFG_E_CUDA;
  for (TuneSnap& sn : snaps) snap_free(sn);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  ens_free_classes(e);   // rebuilt by the first step with the chosen tiles
  return r;
}

int cfg_ensemble_create(int n, cfg_ctx* const* members, int autotune, cfg_ensemble** out) {
  if (n < 1 || !members || !out) return CFG_E_ARG;
  *out = nullptr;
  for (int i = 0; i < n; ++i)
    if (!members[i] || members[i]->nranks > 1 || members[i]->dev != members[0]->dev || members[i]->prof_on)
      return CFG_E_ARG;
  cfg_ensemble* e = new cfg_ensemble();
  e->m.assign(members, members + n);
  e->dev = members[0]->dev;
  cudaSetDevice(e->dev);
  e->ev_done.assign(n, nullptr);
  bool ok = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < n && ok; ++i) ok = cudaEventCreateWithFlags(&e->ev_done[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) { cfg_ensemble_destroy(e); return CFG_E_CUDA; }
  e->batched = true;
  for (int i = 0; i < n; ++i) e->batched = e->batched && ens_batchable(members[i]);
  bool tune_batched = e->batched && autotune;
  for (int i = 0; i < n; ++i) tune_batched = tune_batched && members[i]->mean64_valid;
  if (tune_batched) {
    // one class per grid first (each grid's default tiles), tuned one class
    // at a time on the whole batched step
    const int r = ens_tune_batched(e, 3);
    if (r) { cfg_ensemble_destroy(e); return r; }
  } else if (autotune) {
    // one trial run per distinct grid and precision; the others take its tiles
    for (int i = 0; i < n; ++i) {
      cfg_ctx* c = e->m[i];
      int first = -1;
      for (int j = 0; j < i && first < 0; ++j) {
        const cfg_ctx* o = e->m[j];
        if (o->mixed == c->mixed && o->p.nx == c->p.nx && o->p.ny == c->p.ny && o->p.nz == c->p.nz &&
            o->p.nx2 == c->p.nx2 && o->p.nz2 == c->p.nz2)
          first = j;
      }
      if (first >= 0) {
        const cfg_ctx* o = e->m[first];
        const int t[4] = {o->rhs2_warps, o->flux_zr, o->fYB1, o->fYB3};
        c->xinv_zb = o->xinv_zb;
        const int r = cfg_set_tiles(c, t);
        if (r) { cfg_ensemble_destroy(e); return r; }
      } else {
        const int r = cfg_autotune(c, 3, nullptr);
        if (r) { cfg_ensemble_destroy(e); return r; }
      }
    }
  }
  *out = e;
  return CFG_OK;
}

// one step of the ensemble (eagerly, or under stream capture): batched, or
// every member on its own stream, forked from and joined to the ensemble
// stream.  A batched step needs every member's FP64 mean copy current (it is
// after any whole step).
static int ensemble_enqueue(cfg_ensemble* e) {
  bool batched = e->batched;
  for (const cfg_ctx* c : e->m) batched = batched && c->mean64_valid;
  e->last_batched = batched;
  if (batched) return ens_batched_enqueue(e);
  if (cudaEventRecord(e->ev_fork, e->st) != cudaSuccess) return CFG_E_CUDA;
  for (size_t i = 0; i < e->m.size(); ++i) {
    cfg_ctx* c = e->m[i];
    if (cudaStreamWaitEvent(c->st, e->ev_fork, 0) != cudaSuccess) return fail(c, CFG_E_CUDA, "ensemble fork");
    const int r = step_enqueue(c, false);
    if (r) return r;
    if (cudaEventRecord(e->ev_done[i], c->st) != cudaSuccess ||
        cudaStreamWaitEvent(e->st, e->ev_done[i], 0) != cudaSuccess)
      return fail(c, CFG_E_CUDA, "ensemble join");
  }
  return CFG_OK;
}

int cfg_ensemble_timestep(cfg_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return CFG_E_ARG;
  cudaSetDevice(e->dev);
  int r;
  if (!e->exec && nsteps > 0) {
    // the first step runs eagerly (it also sets every kernel's shared-memory
    // limit; a second one when the first could not run batched), the next
    // one is captured
    if ((r = ensemble_enqueue(e))) return r;
    --nsteps;
    if (e->batched && !e->last_batched && nsteps > 0) {
      if ((r = ensemble_enqueue(e))) return r;
      --nsteps;
    }
    if (nsteps == 0) return CFG_OK;
    std::vector<long long> before(e->m.size());
    for (size_t i = 0; i < e->m.size(); ++i) before[i] = e->m[i]->launches;
    if (cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return CFG_E_CUDA;
    r = ensemble_enqueue(e);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e->st, &g);
    if (r || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return r ? r : CFG_E_CUDA;
    }
    e->graph = g;
    if (cudaGraphInstantiate(&e->exec, e->graph, 0) != cudaSuccess) {
      cudaGetLastError();
      return CFG_E_CUDA;
    }
    e->launches_per_step.resize(e->m.size());
    for (size_t i = 0; i < e->m.size(); ++i) {
      e->launches_per_step[i] = e->m[i]->launches - before[i];
      // the capture advanced the host step counters without running a step
      e->m[i]->step -= 1;
      e->m[i]->launches = before[i];
    }
  }
  for (int s = 0; s < nsteps; ++s) {
    if (cudaGraphLaunch(e->exec, e->st) != cudaSuccess) return CFG_E_CUDA;
    for (size_t i = 0; i < e->m.size(); ++i) {
      e->m[i]->step += 1;
      e->m[i]->launches += e->launches_per_step[i];
    }
  }
  return CFG_OK;
}

int cfg_ensemble_synchronize(cfg_ensemble* e) {
  if (!e) return CFG_E_ARG;
  cudaSetDevice(e->dev);
  return cudaStreamSynchronize(e->st) == cudaSuccess ? CFG_OK : CFG_E_CUDA;
}

void* cfg_ensemble_stream(cfg_ensemble* e) { return e ? (void*)e->st : nullptr; }

int cfg_ensemble_set_batched(cfg_ensemble* e, int on) {
  if (!e) return CFG_E_ARG;
  if (on)
    for (const cfg_ctx* c : e->m)
      if (!ens_batchable(c)) return CFG_E_ARG;
  cudaSetDevice(e->dev);
  if (cudaStreamSynchronize(e->st) != cudaSuccess) return CFG_E_CUDA;
  // the next step is captured again in the new layout; the classes are
  // rebuilt then (tiles may have changed)
  ens_drop_graph(e);
  ens_free_classes(e);
  e->batched = on != 0;
  return CFG_OK;
}

int cfg_ensemble_batched(const cfg_ensemble* e) { return e && e->batched ? 1 : 0; }

int cfg_rank_timestep(cfg_ctx* c, int nsteps, cfg_barrier_fn barrier, void* user) {
  return rank_timestep(c, nsteps, barrier, user, true);
}

int cfg_rank_timestep_ordered(cfg_ctx* c, int nsteps, cfg_barrier_fn barrier, void* user) {
  return rank_timestep(c, nsteps, barrier, user, false);
}

