// pass2v2.cu -- launcher of the v2 RK substep kernel (pass2v2.cuh) for the
// supported rows-per-lane values.
#include "pass2v2.cuh"
#include "pass2v2.h"

namespace cfd {

template <typename T, int M>
static int launch_m(const Rhs2Launch& a) {
  // FP32: 16 lanes per wavenumber; FP64: 32 (keeps the FP64 registers in bounds)
  constexpr int G = sizeof(T) == 4 ? 16 : 32;
  const size_t sm = rhs2_smem<T, M, G>(a.warps);
  static size_t cur = 48 * 1024;
  if (sm > cur) {
    if (cudaFuncSetAttribute(k_rhs2<T, M, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) {
      cudaGetLastError();
      return -2;
    }
    cur = sm;
  }
  const int per_block = a.warps * (32 / G);
  dim3 gr((a.nlist + per_block - 1) / per_block);
  using C = cplx_t<T>;
  k_rhs2<T, M, G><<<gr, 32 * a.warps, sm, a.st>>>((C*)a.vel, (C*)a.cru, (C*)a.prs, (const C*)a.cbc_top,
                                                  (const C*)a.cbc_bot, a.g, a.gd, a.sc, a.rkt, a.rk, a.re, a.wlist,
                                                  a.nlist);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename T>
static int launch_big(const Rhs2Launch& a, int M) {
  if constexpr (sizeof(T) == 4) {
    switch (M) {
      case 9: return launch_m<T, 9>(a);
      case 10: return launch_m<T, 10>(a);
      case 11: return launch_m<T, 11>(a);
      case 12: return launch_m<T, 12>(a);
      case 13: return launch_m<T, 13>(a);
      case 14: return launch_m<T, 14>(a);
      case 15: return launch_m<T, 15>(a);
      case 16: return launch_m<T, 16>(a);
      default: return -1;
    }
  }
  return -1;
}

template <typename T>
static int launch_t(const Rhs2Launch& a) {
  const int G = sizeof(T) == 4 ? 16 : 32;
  const int M = (a.g.ny1 + G - 1) / G;
  if (sizeof(T) == 8 && M > 8) return -1;
  switch (M < 2 ? 2 : M) {
    case 2: return launch_m<T, 2>(a);
    case 3: return launch_m<T, 3>(a);
    case 4: return launch_m<T, 4>(a);
    case 5: return launch_m<T, 5>(a);
    case 6: return launch_m<T, 6>(a);
    case 7: return launch_m<T, 7>(a);
    case 8: return launch_m<T, 8>(a);
    default: return sizeof(T) == 4 ? launch_big<T>(a, M) : -1;
  }
}

int rhs2_launch(bool f32, const Rhs2Launch& a) { return f32 ? launch_t<float>(a) : launch_t<double>(a); }

bool rhs2_supported(int ny1) { return ny1 <= 256; }

}  // namespace cfd
