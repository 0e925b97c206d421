// regfft.cuh -- register-resident FFTs for the hot-path transform lengths.
//
// A length N = N1*N2 transform (N1, N2 in {6, 8, 12, 16, 24}) runs in two
// stages with one shared-memory exchange:
//   stage 1: each thread owns one column n2, loads x[N2*n1 + n2] (n1 < N1),
//            does an N1-point FFT in registers and applies W_N^(n2*k1);
//   stage 2: each thread owns one row k1, does an N2-point FFT over n2 and
//            produces X[k1 + N1*k2].
// The small FFTs are compile-time mixed-radix compositions whose twiddles are
// immediate constant-bank operands (W_48 table).  Sign -1 forward, +1 backward,
// unnormalised, as FFTW.
#pragma once
#include <cmath>

#include "cfd_common.cuh"

namespace cfd {

// cos(2 pi m / 48) for m in [0, 12]: the quarter wave, correctly rounded
// to FP64 (checked against 50-digit values).  Literals so that every twiddle
// of the small FFTs folds to an immediate operand.
__host__ __device__ __forceinline__ constexpr double cos48q(int m) {
  return m == 0 ? 1.0
         : m == 1 ? 0.9914448613738104
         : m == 2 ? 0.9659258262890683
         : m == 3 ? 0.9238795325112867
         : m == 4 ? 0.8660254037844386
         : m == 5 ? 0.7933533402912352
         : m == 6 ? 0.7071067811865476
         : m == 7 ? 0.6087614290087207
         : m == 8 ? 0.5
         : m == 9 ? 0.3826834323650898
         : m == 10 ? 0.25881904510252074
         : m == 11 ? 0.1305261922200516
         : 0.0;
}

__host__ __device__ __forceinline__ constexpr double cos48_r(int r) {
  return r <= 12 ? cos48q(r) : r <= 24 ? -cos48q(24 - r) : r <= 36 ? -cos48q(r - 24) : cos48q(48 - r);
}

// cos(2 pi m / 48) for any m, from the quarter wave by the symmetries
// cos(pi - a) = -cos(a) and cos(2 pi - a) = cos(a): every entry is the
// correctly rounded value, exact zeros at m = 12, 36 and exact halves.
__host__ __device__ __forceinline__ constexpr double cos48(int m) {
  return cos48_r(((m % 48) + 48) % 48);
}

// W_N^(m) with the transform sign: sign -1 -> exp(-2 pi i m/N), +1 -> conjugate
template <typename T, int N, int SIGN>
__host__ __device__ __forceinline__ cplx_t<T> wconst(int m) {
  static_assert(48 % N == 0, "small FFT length must divide 48");
  const int q = (m % N) * (48 / N);
  // exp(-2 pi i q/48) = cos - i sin, sin(a) = cos(a - pi/2) = cos48(q - 12)
  return mk<cplx_t<T>>((T)cos48(q), (T)(SIGN > 0 ? 1.0 : -1.0) * (T)cos48((q + 36) % 48));
}

template <typename C, int SIGN>
__host__ __device__ __forceinline__ C mul_i(C a) {   // (SIGN * i) * a
  return SIGN > 0 ? mk<C>(-a.y, a.x) : mk<C>(a.y, -a.x);
}

// x * W_N^m for a twiddle known at compile time after unrolling: the
// quarter turns are sign changes and swaps (IEEE multiplication by an exact
// 0 or 1 is not folded by the compiler), the rest a complex multiply
template <typename T, int N, int SIGN>
__host__ __device__ __forceinline__ cplx_t<T> twmul(cplx_t<T> x, int m) {
  using C = cplx_t<T>;
  const int q = (m % N) * (48 / N);
  if (q == 0) return x;
  if (q == 24) return mk<C>(-x.x, -x.y);
  // W = cos(2 pi q/48) + i SIGN sin(2 pi q/48): SIGN i at q = 12, -SIGN i at 36
  if (q == 12) return mul_i<C, SIGN>(x);
  if (q == 36) return mul_i<C, -SIGN>(x);
  return cmul(x, wconst<T, N, SIGN>(m));
}

template <typename T, int N, int SIGN> struct SmallFFT;

template <typename T, int SIGN> struct SmallFFT<T, 1, SIGN> {
  template <int S> __host__ __device__ static __forceinline__ void run(cplx_t<T>* v) {}
};

template <typename T, int SIGN> struct SmallFFT<T, 2, SIGN> {
  template <int S> __host__ __device__ static __forceinline__ void run(cplx_t<T>* v) {
    const cplx_t<T> a = v[0];
    v[0] = cadd(a, v[S]);
    v[S] = csub(a, v[S]);
  }
};

template <typename T, int SIGN> struct SmallFFT<T, 3, SIGN> {
  template <int S> __host__ __device__ static __forceinline__ void run(cplx_t<T>* v) {
    using C = cplx_t<T>;
    const T s3 = (T)0.86602540378443864676;
    const C a = v[0], b = v[S], c = v[2 * S];
    const C t1 = cadd(b, c);
    const C t2 = mk<C>(a.x - (T)0.5 * t1.x, a.y - (T)0.5 * t1.y);
    const C d = csub(b, c);
    const T t3x = (T)SIGN * s3 * d.x, t3y = (T)SIGN * s3 * d.y;
    v[0] = cadd(a, t1);
    v[S] = mk<C>(t2.x - t3y, t2.y + t3x);
    v[2 * S] = mk<C>(t2.x + t3y, t2.y - t3x);
  }
};

template <typename T, int SIGN> struct SmallFFT<T, 4, SIGN> {
  template <int S> __host__ __device__ static __forceinline__ void run(cplx_t<T>* v) {
    using C = cplx_t<T>;
    const C t0 = cadd(v[0], v[2 * S]), t1 = csub(v[0], v[2 * S]);
    const C t2 = cadd(v[S], v[3 * S]), t3 = mul_i<C, SIGN>(csub(v[S], v[3 * S]));
    v[0] = cadd(t0, t2);
    v[2 * S] = csub(t0, t2);
    v[S] = cadd(t1, t3);
    v[3 * S] = csub(t1, t3);
  }
};

// Composite N = P*Q: decimation in time over p (the "rows" v[p + P*q]).
// Operates in place on v[0], v[S], ..., v[(N-1)*S] and leaves X[k] in v[k*S].
template <typename T, int P, int Q, int SIGN> struct Composite {
  template <int S> __host__ __device__ static __forceinline__ void run(cplx_t<T>* v) {
    using C = cplx_t<T>;
    constexpr int N = P * Q;
    // sub-FFTs of length Q on v[p + P*q]: stride P*S
#pragma unroll
    for (int p = 0; p < P; ++p) SmallFFT<T, Q, SIGN>::template run<P * S>(v + p * S);
    // now v[(p + P*k2)*S] = S_p[k2]; twiddle and length-P FFTs over p
    C t[N];
#pragma unroll
    for (int k2 = 0; k2 < Q; ++k2) {
#pragma unroll
      for (int p = 0; p < P; ++p) {
        t[k2 * P + p] = twmul<T, N, SIGN>(v[(p + P * k2) * S], p * k2);
      }
      SmallFFT<T, P, SIGN>::template run<1>(t + k2 * P);
    }
    // X[k2 + Q*k1] = t[k2*P + k1]
#pragma unroll
    for (int k2 = 0; k2 < Q; ++k2)
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) v[(k2 + Q * k1) * S] = t[k2 * P + k1];
  }
};

template <typename T, int SIGN> struct SmallFFT<T, 6, SIGN> : Composite<T, 2, 3, SIGN> {};
template <typename T, int SIGN> struct SmallFFT<T, 8, SIGN> : Composite<T, 2, 4, SIGN> {};
template <typename T, int SIGN> struct SmallFFT<T, 12, SIGN> : Composite<T, 4, 3, SIGN> {};
template <typename T, int SIGN> struct SmallFFT<T, 16, SIGN> : Composite<T, 4, 4, SIGN> {};
template <typename T, int SIGN> struct SmallFFT<T, 24, SIGN> : Composite<T, 8, 3, SIGN> {};

// Two-stage factorisation of the supported transform lengths.
template <int N> struct Split;
template <> struct Split<24> { static constexpr int N1 = 4, N2 = 6; };
template <> struct Split<48> { static constexpr int N1 = 8, N2 = 6; };
template <> struct Split<72> { static constexpr int N1 = 12, N2 = 6; };
template <> struct Split<96> { static constexpr int N1 = 12, N2 = 8; };
template <> struct Split<144> { static constexpr int N1 = 12, N2 = 12; };
template <> struct Split<192> { static constexpr int N1 = 16, N2 = 12; };
template <> struct Split<288> { static constexpr int N1 = 24, N2 = 12; };
template <> struct Split<384> { static constexpr int N1 = 16, N2 = 24; };
template <> struct Split<576> { static constexpr int N1 = 24, N2 = 24; };

__host__ __device__ constexpr bool regfft_supported(int n) {
  return n == 24 || n == 48 || n == 72 || n == 96 || n == 144 || n == 192 || n == 288 || n == 384 || n == 576;
}

// Shared exchange buffer of one sequence: [k1][n2] with row pitch N2+1.
template <int N> struct XBuf {
  static constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, PITCH = N2 + 1;
  static constexpr int SIZE = N1 * PITCH;
};

// Stage 1 for `nseq` sequences: load(s, m) returns x_s[m]; tw[m] = W_N^m
// (sign -1) in shared memory; writes the exchange buffer Y (nseq * SIZE).
template <typename T, int N, int SIGN, typename Load>
__device__ __forceinline__ void fft_stage1(int nseq, const cplx_t<T>* tw, cplx_t<T>* Y, Load load) {
  using C = cplx_t<T>;
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, PITCH = N2 + 1, SIZE = N1 * PITCH;
  for (int t = threadIdx.x; t < nseq * N2; t += blockDim.x) {
    const int s = t / N2, n2 = t - s * N2;
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = load(s, N2 * n1 + n2);
    SmallFFT<T, N1, SIGN>::template run<1>(v);
    C* y = Y + s * SIZE + n2;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      C x = v[k1];
      if (k1 != 0) {
        C w = tw[n2 * k1];
        if (SIGN > 0) w.y = -w.y;
        x = cmul(x, w);
      }
      y[k1 * PITCH] = x;
    }
  }
}

// Stage 2: store(s, k, X_s[k]) for all k.
template <typename T, int N, int SIGN, typename Store>
__device__ __forceinline__ void fft_stage2(int nseq, const cplx_t<T>* Y, Store store) {
  using C = cplx_t<T>;
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, PITCH = N2 + 1, SIZE = N1 * PITCH;
  for (int t = threadIdx.x; t < nseq * N1; t += blockDim.x) {
    const int s = t / N1, k1 = t - s * N1;
    C u[N2];
    const C* y = Y + s * SIZE + k1 * PITCH;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) u[n2] = y[n2];
    SmallFFT<T, N2, SIGN>::template run<1>(u);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) store(s, k1 + N1 * k2, u[k2]);
  }
}

}  // namespace cfd
