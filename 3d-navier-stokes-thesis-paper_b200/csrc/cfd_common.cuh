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

// FP32 complex additions, subtractions and real scalings as one packed
// two-lane instruction (add/sub/mul.rn.f32x2, sm_100): the same IEEE results
// as the two scalar operations, half the issued instructions.
#if !defined(CFD_NO_F32X2)
template <> __host__ __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  float2 r;
  asm("{.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "add.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
#else
  return mk<float2>(a.x + b.x, a.y + b.y);
#endif
}
template <> __host__ __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  float2 r;
  asm("{.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
#else
  return mk<float2>(a.x - b.x, a.y - b.y);
#endif
}
template <> __host__ __device__ __forceinline__ float2 cscale<float2, float>(float s, float2 a) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  float2 r;
  asm("{.reg .b64 pa, ps, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 ps, {%4, %4};\n\t"
      "mul.rn.f32x2 pr, ps, pa;\n\tmov.b64 {%0, %1}, pr;}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(s));
  return r;
#else
  return mk<float2>(s * a.x, s * a.y);
#endif
}
#endif
// (i*k) * a for real k
template <typename C, typename T> __host__ __device__ __forceinline__ C cimul(T k, C a) { return mk<C>(-k * a.y, k * a.x); }
template <typename C> __host__ __device__ __forceinline__ C czero() { return mk<C>(0, 0); }

// Geometry of one context, by value in every launch.
struct Geom {
  int nx, ny, nz, nx2, nz2;
  int nxh;   // nx/2+1 Fourier columns in x
  int ny1;   // ny+1 planes
  int nw;    // nz*nxh wavenumbers
  // slab of a multi-rank run (PFC/setup.f90:298-437 split kx in Fourier
  // space): global index of the first local kx column and the global column
  // count; 0 and nxh for one rank
  int kx0, nxh_all;
};

// Scatter targets of the two transposes of a multi-rank run.  The inverse z
// transform of each rank writes element z2 of hybrid row R to the rank that
// owns z2, at zdst[z2] + R * zpitch[z2] (complex elements); the flux kernel
// writes column kx of x-transformed row R to the rank that owns kx, at
// xdst[kx] + R * xpitch[kx].  Addresses are byte addresses in the owners'
// buffers (peer memory on other GPUs).  n == 0: one rank, local layouts.
struct Scatter {
  int n;
  const unsigned long long* zdst;
  const long long* zpitch;
  const unsigned long long* xdst;
  const long long* xpitch;
};

// FFT plan for one length: Stockham passes, radices in {2,3,4,8}.
struct FftPlan {
  int n, npass;
  int radix[16];
  int ns[16];
};

}  // namespace cfd
