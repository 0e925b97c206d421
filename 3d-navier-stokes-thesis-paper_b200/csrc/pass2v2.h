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
  int lanes;   // lanes per wavenumber: 32, or 16 (FP32 only)
  const void* tbl;   // coefficient table of rhs2_table for these lanes
  cudaStream_t st;
};

// 0 on success, -1 unsupported size, -2 launch error
int rhs2_launch(bool f32, const Rhs2Launch& a);
bool rhs2_supported(int ny1);
// the lane-major grid-coefficient table the kernel reads (host side)
size_t rhs2_table_bytes(bool f32, int ny1, int lanes);
void rhs2_table(bool f32, int ny, int lanes, const double* dh, const double* dn, const double* d2h,
                const double* d2n, void* out);

}  // namespace cfd
