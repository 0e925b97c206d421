// noalloc.cu -- cfg_xz_c2r_noalloc: the single-plane inverse x-z transform of
// cfg_xz_c2r with its intermediate (the hybrid plane, z physical / x spectral)
// and twiddle tables held in a fixed, file-scope device array instead of
// memory allocated per context.  It allocates nothing: no cudaMalloc,
// cudaFree or allocating library call, on any call.
//
// Who needs it: hosts that cannot call cudaMalloc at the point where they
// transform a plane.  Examples are a Fortran driver whose device memory is
// pre-assigned at start-up by another owner (a framework's caching allocator
// or a communication library holding registered buffers), where a further
// cudaMalloc would fail or fragment the pool, and step loops that must not
// take the device-wide synchronisation cudaMalloc/cudaFree imply.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "chanflow.h"
#include "planes.cuh"

using namespace cfd;

namespace {

// Capacity of the fixed scratch: the hybrid plane holds (nx/2+1)*nz2 complex
// values, the twiddle tables nx2 + nz2 more.
constexpr size_t kMaxHybrid = (size_t)1 << 18;   // 262144 complex FP64 = 4 MiB
constexpr int kMaxLen = 2048;                    // nx2, nz2 upper bound

// The scratch array.  Every GPU that loads this library holds it (4.06 MiB)
// until the process exits; every call shares it and it keeps the last call's
// contents.
static __device__ __align__(256) double2 g_scratch[kMaxHybrid + 2 * (size_t)kMaxLen];

// Per device, with that device current at the first call: the device address
// of g_scratch, and the transform lengths whose twiddle tables the array holds
// now (0: none), so that a call of the same lengths does not rewrite them.
constexpr int kMaxDevices = 64;
double2* g_scratch_addr[kMaxDevices] = {nullptr};
int g_tw_len[kMaxDevices][2] = {};
std::mutex g_setup_mutex;

// Raise a kernel's dynamic shared-memory limit on the current device to
// `need` bytes if it is lower; never lower it (other contexts may have raised
// it for larger launches of the same kernel).
template <typename K>
cudaError_t raise_smem(K kernel, size_t need) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  if ((size_t)fa.maxDynamicSharedSizeBytes >= need) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
}

bool plan_2_3(int n, FftPlan& p) {
  p = FftPlan{};
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

// W_n^m = exp(-2 pi i m / n)
__global__ void k_twiddles(double2* tw, int n) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)m / (double)n, &s, &c);
    tw[m] = make_double2(c, s);
  }
}

}  // namespace

extern "C" int cfg_xz_c2r_noalloc(int nx, int nz, int nx2, int nz2, const double* cdata, double* data,
                                  void* stream) {
  if (!cdata || !data || nx < 2 || nz < 2 || (nx & 1) || (nz & 1) || (nx2 & 1) || (nz2 & 1) || nx2 < nx ||
      nz2 < nz)
    return CFG_E_ARG;
  FftPlan px, pz;
  if (!plan_2_3(nx2, px) || !plan_2_3(nz2, pz)) return CFG_E_ARG;
  const int nxh = nx / 2 + 1;
  if (nx2 > kMaxLen || nz2 > kMaxLen || (size_t)nxh * nz2 > kMaxHybrid) {
    fprintf(stderr,
            "cfg_xz_c2r_noalloc: plane %d x %d (dealiased %d x %d) exceeds the fixed scratch "
            "((nx/2+1)*nz2 <= %zu, nx2, nz2 <= %d)\n",
            nx, nz, nx2, nz2, kMaxHybrid, kMaxLen);
    return CFG_E_SIZE;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CFG_E_CUDA;
  const size_t smz = sizeof(double2) * 3 * (size_t)nz2, smx = sizeof(double2) * 3 * (size_t)nx2;
  double2* base = nullptr;
  bool write_twx = false, write_twz = false;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
      // once per device, with that device current: the host-side symbol is a
      // stand-in, the kernels need the device address
      double2* p = nullptr;
      if (cudaGetSymbolAddress((void**)&p, g_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return CFG_E_CUDA;
      }
      g_scratch_addr[dev] = p;
    }
    base = g_scratch_addr[dev];
    if (raise_smem(k_pz_inv<double>, smz) != cudaSuccess || raise_smem(k_px_inv<double>, smx) != cudaSuccess) {
      cudaGetLastError();
      return CFG_E_CUDA;
    }
    write_twx = g_tw_len[dev][0] != nx2;
    write_twz = g_tw_len[dev][1] != nz2;
    g_tw_len[dev][0] = nx2;
    g_tw_len[dev][1] = nz2;
  }
  cudaStream_t st = (cudaStream_t)stream;
  double2* H = base;                 // hybrid plane (nx/2+1, nz2): fully rewritten below
  double2* twx = base + kMaxHybrid;  // W_nx2
  double2* twz = twx + kMaxLen;      // W_nz2
  // the twiddle tables are written when the lengths change and kept otherwise
  if (write_twx) k_twiddles<<<8, 256, 0, st>>>(twx, nx2);
  if (write_twz) k_twiddles<<<8, 256, 0, st>>>(twz, nz2);
  PlaneIn L{0, 0, (size_t)nz, 1, 1};
  k_pz_inv<double><<<dim3(nxh, 1), 128, smz, st>>>(reinterpret_cast<const double2*>(cdata), L, nullptr, 1, H, nxh,
                                                   nz, nz2, 1, nx2 > nx, pz, twz);
  k_px_inv<double><<<dim3((nz2 + 1) / 2, 1), 128, smx, st>>>(H, data, nxh, nz2, nx2, px, twx);
  if (cudaGetLastError() != cudaSuccess) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    g_tw_len[dev][0] = g_tw_len[dev][1] = 0;  // the tables may not have been written
    return CFG_E_CUDA;
  }
  return CFG_OK;
}
