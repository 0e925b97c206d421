// fft.cuh -- block-cooperative mixed-radix (2/3/4/8) Stockham FFT on batches
// of sequences held in shared memory.  Replaces the FFTW plans of
// PFC/transform.f90:60-160 (sign -1 forward, +1 backward, unnormalised).
#pragma once
#include "cfd_common.cuh"

namespace cfd {

template <typename C>
__device__ __forceinline__ C mul_si(C a, int sign) {  // (sign * i) * a
  return sign > 0 ? mk<C>(-a.y, a.x) : mk<C>(a.y, -a.x);
}

template <typename C>
__device__ __forceinline__ void dft2(C* v) {
  C a = v[0];
  v[0] = cadd(a, v[1]);
  v[1] = csub(a, v[1]);
}

template <typename C>
__device__ __forceinline__ void dft4(C* v, int sign) {
  C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  C t2 = cadd(v[1], v[3]), t3 = mul_si(csub(v[1], v[3]), sign);
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  v[1] = cadd(t1, t3);
  v[3] = csub(t1, t3);
}

template <typename C, typename T>
__device__ __forceinline__ void dft3(C* v, int sign) {
  const T s3 = (T)0.86602540378443864676;
  C a = v[0], b = v[1], c = v[2];
  C t1 = cadd(b, c);
  C t2 = mk<C>(a.x - (T)0.5 * t1.x, a.y - (T)0.5 * t1.y);
  C d = csub(b, c);
  T t3x = (T)sign * s3 * d.x, t3y = (T)sign * s3 * d.y;
  v[0] = cadd(a, t1);
  v[1] = mk<C>(t2.x - t3y, t2.y + t3x);
  v[2] = mk<C>(t2.x + t3y, t2.y - t3x);
}

template <typename C, typename T>
__device__ __forceinline__ void dft8(C* v, int sign) {
  C e[4] = {v[0], v[2], v[4], v[6]};
  C o[4] = {v[1], v[3], v[5], v[7]};
  dft4(e, sign);
  dft4(o, sign);
  const T r = (T)0.70710678118654752440;
  const T s = (T)sign;
  C o1 = mk<C>(r * (o[1].x - s * o[1].y), r * (o[1].y + s * o[1].x));
  C o2 = mul_si(o[2], sign);
  C o3 = mk<C>(r * (-o[3].x - s * o[3].y), r * (-o[3].y + s * o[3].x));
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], o1);
  v[5] = csub(e[1], o1);
  v[2] = cadd(e[2], o2);
  v[6] = csub(e[2], o2);
  v[3] = cadd(e[3], o3);
  v[7] = csub(e[3], o3);
}

// Transforms nseq sequences of length p.n (sequence s at in + s*stride).
// tw[m] = exp(-2 pi i m / n), m < n, in shared or global memory.  Ping-pongs
// between `in` and `out`; returns the buffer holding the result.  Every
// thread of the block must call it (it synchronises between passes).
template <typename T>
__device__ cplx_t<T>* block_fft(cplx_t<T>* in, cplx_t<T>* out, const FftPlan& p,
                                int nseq, int stride, const cplx_t<T>* tw, int sign) {
  using C = cplx_t<T>;
  const int N = p.n;
  for (int q = 0; q < p.npass; ++q) {
    const int R = p.radix[q], Ns = p.ns[q], NR = N / R, tstep = N / (Ns * R);
    const int total = nseq * NR;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int s = t / NR, j = t - s * NR;
      const C* src = in + s * stride;
      C* dst = out + s * stride;
      const int k = j % Ns;
      C v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        if (r < R) {
          C x = src[j + r * NR];
          if (r > 0 && k > 0) {
            C w = tw[k * r * tstep];
            if (sign > 0) w.y = -w.y;
            x = cmul(x, w);
          }
          v[r] = x;
        }
      }
      switch (R) {
        case 2: dft2(v); break;
        case 3: dft3<C, T>(v, sign); break;
        case 4: dft4(v, sign); break;
        default: dft8<C, T>(v, sign); break;
      }
      const int d = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < R) dst[d + r * Ns] = v[r];
    }
    __syncthreads();
    C* tmp = in;
    in = out;
    out = tmp;
  }
  return in;
}

}  // namespace cfd
