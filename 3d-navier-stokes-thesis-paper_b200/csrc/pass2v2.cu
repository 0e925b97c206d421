// pass2v2.cu -- launcher of the v2 RK substep kernel (pass2v2.cuh) for the
// supported rows-per-lane values.
#include "pass2v2.cuh"
#include "pass2v2.h"

#include <algorithm>


namespace cfd {

// Batched launches over a member table (the ensemble mode): member m of a
// class of identical grids takes blocks m*gx ... m*gx + gx - 1 of the main
// kernel (one block each of the mean kernel) and reads its arguments from its
// launch record in device memory.  Same bodies, same arithmetic.
template <typename T, typename S, int M, int G>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 5 : 1)
k_rhs2_b(const Rhs2Launch* __restrict__ tab, unsigned gx) {
  using CS = cplx_t<S>;
  const unsigned m = blockIdx.x / gx;
  const Rhs2Launch& a = tab[m];
  k_rhs2_body<T, S, M, G>(make_uint3(blockIdx.x - m * gx, 0, 0), (CS*)a.vel, (CS*)a.cru, (CS*)a.prs,
                          (const CS*)a.cbc_top, (const CS*)a.cbc_bot, a.g, a.gd, a.sc, a.rkt, a.rk, a.re, a.wlist,
                          a.nlist, (const T*)a.tbl);
}

template <typename S, int M>
__global__ void __launch_bounds__(32) k_rhs_mean2_b(const RhsMeanLaunch* __restrict__ tab) {
  using CS = cplx_t<S>;
  const RhsMeanLaunch& a = tab[blockIdx.x];
  k_rhs_mean2_body<S, M>(make_uint3(0, 0, 0), (CS*)a.vel, (CS*)a.cru, (CS*)a.prs, a.mvel64, a.mcru64,
                         (const CS*)a.cbc_top, (const CS*)a.cbc_bot, a.g, a.gd, a.sc, a.d_um_dy, a.rkt, a.rk, a.re,
                         a.beta, a.fix_mass, a.tbl64);
}

// tab: null for one domain (arguments from a), else the device table of nmem
// members whose launch shapes equal a's
template <typename T, int M, int G>
static int launch_m(const Rhs2Launch& a, const Rhs2Launch* tab, int nmem) {
  const size_t sm = rhs2_smem<T, M, G>(a.warps, a.g.ny1);
  // the limit raised so far on each device (the attribute is per device)
  static size_t cur_dev[64][2];   // single-domain and batched kernel
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return -2;
  size_t& cur = cur_dev[dev][tab ? 1 : 0];
  if (cur == 0) cur = 48 * 1024;
  if (sm > cur) {
    const cudaError_t e =
        tab ? cudaFuncSetAttribute(k_rhs2_b<T, T, M, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)
            : cudaFuncSetAttribute(k_rhs2<T, T, M, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return -2;
    }
    cur = sm;
  }
  const int per_block = a.warps * (32 / G);
  dim3 gr((a.nlist + per_block - 1) / per_block);
  using C = cplx_t<T>;
  if (tab)
    k_rhs2_b<T, T, M, G><<<gr.x * (unsigned)nmem, 32 * a.warps, sm, a.st>>>(tab, gr.x);
  else
    k_rhs2<T, T, M, G><<<gr, 32 * a.warps, sm, a.st>>>((C*)a.vel, (C*)a.cru, (C*)a.prs, (const C*)a.cbc_top,
                                                    (const C*)a.cbc_bot, a.g, a.gd, a.sc, a.rkt, a.rk, a.re, a.wlist,
                                                    a.nlist, (const T*)a.tbl);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// 32 lanes per wavenumber: M = ceil(ny1/32) <= 8 rows per lane
template <typename T>
static int launch_g32(const Rhs2Launch& a, const Rhs2Launch* tab, int nmem) {
  const int M = (a.g.ny1 + 31) / 32;
  switch (M < 2 ? 2 : M) {
    case 2: return launch_m<T, 2, 32>(a, tab, nmem);
    case 3: return launch_m<T, 3, 32>(a, tab, nmem);
    case 4: return launch_m<T, 4, 32>(a, tab, nmem);
    case 5: return launch_m<T, 5, 32>(a, tab, nmem);
    case 6: return launch_m<T, 6, 32>(a, tab, nmem);
    case 7: return launch_m<T, 7, 32>(a, tab, nmem);
    case 8: return launch_m<T, 8, 32>(a, tab, nmem);
    default: return -1;
  }
}

// 8 lanes per wavenumber (FP32 only): M = ceil(ny1/8) <= 8
static int launch_g8(const Rhs2Launch& a, const Rhs2Launch* tab, int nmem) {
  const int M = (a.g.ny1 + 7) / 8;
  switch (M < 2 ? 2 : M) {
    case 2: return launch_m<float, 2, 8>(a, tab, nmem);
    case 3: return launch_m<float, 3, 8>(a, tab, nmem);
    case 4: return launch_m<float, 4, 8>(a, tab, nmem);
    case 5: return launch_m<float, 5, 8>(a, tab, nmem);
    case 6: return launch_m<float, 6, 8>(a, tab, nmem);
    case 7: return launch_m<float, 7, 8>(a, tab, nmem);
    case 8: return launch_m<float, 8, 8>(a, tab, nmem);
    default: return -1;
  }
}

// 16 lanes per wavenumber (FP32 only): M = ceil(ny1/16) <= 16
static int launch_g16(const Rhs2Launch& a, const Rhs2Launch* tab, int nmem) {
  const int M = (a.g.ny1 + 15) / 16;
  switch (M < 2 ? 2 : M) {
    case 2: return launch_m<float, 2, 16>(a, tab, nmem);
    case 3: return launch_m<float, 3, 16>(a, tab, nmem);
    case 4: return launch_m<float, 4, 16>(a, tab, nmem);
    case 5: return launch_m<float, 5, 16>(a, tab, nmem);
    case 6: return launch_m<float, 6, 16>(a, tab, nmem);
    case 7: return launch_m<float, 7, 16>(a, tab, nmem);
    case 8: return launch_m<float, 8, 16>(a, tab, nmem);
    case 9: return launch_m<float, 9, 16>(a, tab, nmem);
    case 10: return launch_m<float, 10, 16>(a, tab, nmem);
    case 11: return launch_m<float, 11, 16>(a, tab, nmem);
    case 12: return launch_m<float, 12, 16>(a, tab, nmem);
    case 13: return launch_m<float, 13, 16>(a, tab, nmem);
    case 14: return launch_m<float, 14, 16>(a, tab, nmem);
    case 15: return launch_m<float, 15, 16>(a, tab, nmem);
    case 16: return launch_m<float, 16, 16>(a, tab, nmem);
    default: return -1;
  }
}

// FP64 arithmetic over FP32 storage, one warp (one wavenumber) per block
template <int M>
static int launch_prec_m(const Rhs2Launch& a, const Rhs2Launch* tab, int nmem) {
  const size_t sm = rhs2_smem<double, M, 32>(1, a.g.ny1);
  if (sm > 48 * 1024) return -1;
  if (tab)
    k_rhs2_b<double, float, M, 32><<<(unsigned)a.nlist * (unsigned)nmem, 32, sm, a.st>>>(tab, (unsigned)a.nlist);
  else
    k_rhs2<double, float, M, 32><<<a.nlist, 32, sm, a.st>>>((float2*)a.vel, (float2*)a.cru, (float2*)a.prs,
                                                           (const float2*)a.cbc_top, (const float2*)a.cbc_bot, a.g,
                                                           a.gd, a.sc, a.rkt, a.rk, a.re, a.wlist, a.nlist,
                                                           (const double*)a.tbl);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int rhs2_launch_prec(const Rhs2Launch& a) { return rhs2_launch_prec_batch(a, nullptr, 0); }

int rhs2_launch_prec_batch(const Rhs2Launch& a, const Rhs2Launch* tab, int nmem) {
  const int M = (a.g.ny1 + 31) / 32;
  switch (M < 2 ? 2 : M) {
    case 2: return launch_prec_m<2>(a, tab, nmem);
    case 3: return launch_prec_m<3>(a, tab, nmem);
    case 4: return launch_prec_m<4>(a, tab, nmem);
    case 5: return launch_prec_m<5>(a, tab, nmem);
    case 6: return launch_prec_m<6>(a, tab, nmem);
    case 7: return launch_prec_m<7>(a, tab, nmem);
    case 8: return launch_prec_m<8>(a, tab, nmem);
    default: return -1;
  }
}

template <typename S, int M>
static int launch_mean_m(const RhsMeanLaunch& a, const RhsMeanLaunch* tab, int nmem) {
  using CS = cplx_t<S>;
  const size_t sm = rhs_mean2_smem<M>(a.g.ny1);
  if (sm > 48 * 1024) return -1;
  if (tab)
    k_rhs_mean2_b<S, M><<<(unsigned)nmem, 32, sm, a.st>>>(tab);
  else
    k_rhs_mean2<S, M><<<1, 32, sm, a.st>>>((CS*)a.vel, (CS*)a.cru, (CS*)a.prs, a.mvel64, a.mcru64,
                                           (const CS*)a.cbc_top, (const CS*)a.cbc_bot, a.g, a.gd, a.sc, a.d_um_dy,
                                           a.rkt, a.rk, a.re, a.beta, a.fix_mass, a.tbl64);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename S>
static int launch_mean_t(const RhsMeanLaunch& a, const RhsMeanLaunch* tab, int nmem) {
  const int M = (a.g.ny1 + 31) / 32;
  switch (M < 2 ? 2 : M) {
    case 2: return launch_mean_m<S, 2>(a, tab, nmem);
    case 3: return launch_mean_m<S, 3>(a, tab, nmem);
    case 4: return launch_mean_m<S, 4>(a, tab, nmem);
    case 5: return launch_mean_m<S, 5>(a, tab, nmem);
    case 6: return launch_mean_m<S, 6>(a, tab, nmem);
    case 7: return launch_mean_m<S, 7>(a, tab, nmem);
    case 8: return launch_mean_m<S, 8>(a, tab, nmem);
    default: return -1;
  }
}

int rhs_mean2_launch(bool f32, const RhsMeanLaunch& a) { return rhs_mean2_launch_batch(f32, a, nullptr, 0); }

int rhs_mean2_launch_batch(bool f32, const RhsMeanLaunch& a, const RhsMeanLaunch* tab, int nmem) {
  return f32 ? launch_mean_t<float>(a, tab, nmem) : launch_mean_t<double>(a, tab, nmem);
}

int rhs2_launch(bool f32, const Rhs2Launch& a) { return rhs2_launch_batch(f32, a, nullptr, 0); }

int rhs2_launch_batch(bool f32, const Rhs2Launch& a, const Rhs2Launch* tab, int nmem) {
  if (tab && nmem < 1) return -1;
  if (f32 && a.lanes == 16) return launch_g16(a, tab, nmem);
  if (f32 && a.lanes == 8) return launch_g8(a, tab, nmem);
  return f32 ? launch_g32<float>(a, tab, nmem) : launch_g32<double>(a, tab, nmem);
}

bool rhs2_supported(int ny1) { return ny1 <= 256; }

int rhs2_rows_per_lane(int ny1, int lanes) { return std::max(2, (ny1 + lanes - 1) / lanes); }

size_t rhs2_table_bytes(bool f32, int ny1, int lanes) {
  return (f32 ? sizeof(float) : sizeof(double)) * (size_t)RC_NUM * rhs2_rows_per_lane(ny1, lanes) * lanes;
}

void rhs2_table(bool f32, int ny, int lanes, const double* dh, const double* dn, const double* d2h,
                const double* d2n, void* out) {
  const int M = rhs2_rows_per_lane(ny + 1, lanes);
  if (f32) rhs2_fill_table<float>((float*)out, M, lanes, ny, dh, dn, d2h, d2n);
  else rhs2_fill_table<double>((double*)out, M, lanes, ny, dh, dn, d2h, d2n);
}

}  // namespace cfd
