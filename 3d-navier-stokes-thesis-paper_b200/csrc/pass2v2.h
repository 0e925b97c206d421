// pass2v2.h -- launch interface of the v2 RK substep kernel.
#pragma once
#include <cuda_runtime.h>

#include "pass1.cuh"
#include "pass2.cuh"

namespace cfd {

struct Rhs2Launch {
  void *vel, *cru, *prs;
  const void *cbc_top, *cbc_bot;
  Geom g;
  GridDev gd;
  const DevScalars* sc;
  RkTab rkt;
  int rk;
  double re;
  const int* wlist;
  int nlist;
  int warps;   // warps per block
  int lanes;   // lanes per wavenumber: 32, or 16 or 8 (FP32 only)
  const void* tbl;   // coefficient table of rhs2_table for these lanes
  cudaStream_t st;
};

// 0 on success, -1 unsupported size, -2 launch error
int rhs2_launch(bool f32, const Rhs2Launch& a);
// the mixed path's |k| < 4 list: FP64 arithmetic over FP32 storage, tbl the
// FP64 table for 32 lanes
int rhs2_launch_prec(const Rhs2Launch& a);
// the same kernels for nmem members of one grid in one launch: tab is the
// members' launch records in device memory, a the first member's (host)
// copy, which sets the launch shape and stream
int rhs2_launch_batch(bool f32, const Rhs2Launch& a, const Rhs2Launch* tab, int nmem);
int rhs2_launch_prec_batch(const Rhs2Launch& a, const Rhs2Launch* tab, int nmem);

// the mean mode (k_rhs_mean2)
struct RhsMeanLaunch {
  void *vel, *cru, *prs;
  double2 *mvel64, *mcru64;   // FP64 mean columns (mixed), or null
  const void *cbc_top, *cbc_bot;
  Geom g;
  GridDev gd;
  DevScalars* sc;
  double* d_um_dy;
  RkTab rkt;
  int rk;
  double re, beta;
  int fix_mass;
  const double* tbl64;        // FP64 coefficient table for 32 lanes
  cudaStream_t st;
};
int rhs_mean2_launch(bool f32, const RhsMeanLaunch& a);
int rhs_mean2_launch_batch(bool f32, const RhsMeanLaunch& a, const RhsMeanLaunch* tab, int nmem);
bool rhs2_supported(int ny1);
// the lane-major grid-coefficient table the kernel reads (host side)
size_t rhs2_table_bytes(bool f32, int ny1, int lanes);
void rhs2_table(bool f32, int ny, int lanes, const double* dh, const double* dn, const double* d2h,
                const double* d2n, void* out);

}  // namespace cfd
