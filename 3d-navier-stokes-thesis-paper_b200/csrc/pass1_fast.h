// pass1_fast.h -- launch interface of the register-FFT pass-1 kernels, one
// translation unit per transform length (pass1_n<N>.cu).
#pragma once
#include <cuda_runtime.h>

#include "pass1.cuh"

namespace cfd {

struct P1Launch {
  const void* vel;      // spectral velocity (k_zinv input)
  void* T1;             // hybrid planes
  void* T2;             // x-transformed fluxes
  void* velout;         // nonlinear term (k_zfwd output)
  Geom g;
  const void* twx;      // W_nx2^m
  const void* twz;      // W_nz2^m
  GridDev gd;
  const void* fringe;
  int has_fringe;
  int YB1, YB3, ZR, KC;
  unsigned long long* cflbits;
  int do_cfl;
  int lin;
  void* P;              // physical planes (split x stage)
  int FZR;              // z rows per k_flux_r block (2 or 4)
  Scatter sc;           // transposes of a multi-rank run (n == 0: one rank)
  const void* sgs;      // LES subgrid stresses [ny+1][6][nz2][nx2] for k_flux_r, or null
  int split;            // mean split: k_zinv_r drops the mean column, k_flux_r adds it from gd.baseflow
  int XZB;              // z2 rows per k_xinv_r block: 8, 16 or 24 (FP32), 0 for the default
  cudaStream_t st;
};

// which: 0 k_zinv_r, 1 k_xflux_r, 2 k_zfwd_r, 3 k_xinv_r, 4 k_flux_r.
// Returns 0, or -1 when the length is not compiled in, or -2 on a launch error.
int p1_fast_launch(int which, int n, bool f32, const P1Launch& a);
// the same kernel for nmem members of one grid and tiles in one launch: tab
// is the members' P1Launch array in device memory, a the first member's
// (host) copy, which sets the launch shape and stream; which 0, 2, 3 or 4
int p1_fast_launch_batch(int which, int n, bool f32, const P1Launch& a, const P1Launch* tab, int nmem);
// shared memory bytes of kernel `which` at length n with its tile parameter
// (YB for 0/2, ZR for 1 and 4, the z2 row count for 3); 0 when unsupported.
size_t p1_fast_smem(int which, int n, bool f32, int param, int nxh, int nz);

}  // namespace cfd
