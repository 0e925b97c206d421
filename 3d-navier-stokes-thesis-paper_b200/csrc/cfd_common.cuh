// cfd_common.cuh -- complex types, device geometry and launch helpers shared
// by the channel-flow kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cfd {

template <typename T> struct CT;
template <> struct CT<float> { using type = float2; };
template <> struct CT<double> { using type = double2; };
template <typename T> using cplx_t = typename CT<T>::type;

template <typename C> __host__ __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) { C r; r.x = a; r.y = b; return r; }
template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) { return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
template <typename C, typename T> __host__ __device__ __forceinline__ C cscale(T s, C a) { return mk<C>(s * a.x, s * a.y); }
// (i*k) * a for real k
template <typename C, typename T> __host__ __device__ __forceinline__ C cimul(T k, C a) { return mk<C>(-k * a.y, k * a.x); }
template <typename C> __host__ __device__ __forceinline__ C czero() { return mk<C>(0, 0); }

// Geometry of one context, by value in every launch.
struct Geom {
  int nx, ny, nz, nx2, nz2;
  int nxh;   // nx/2+1 Fourier columns in x
  int ny1;   // ny+1 planes
  int nw;    // nz*nxh wavenumbers
};

// FFT plan for one length: Stockham passes, radices in {2,3,4,8}.
struct FftPlan {
  int n, npass;
  int radix[16];
  int ns[16];
};

}  // namespace cfd
