// pass1_reg.cuh -- the pass-1 kernels of pass1.cuh (same arithmetic, same
// layouts) built on the register-resident two-stage FFTs of regfft.cuh for the
// hot-path lengths (48 ... 576).  See pass1.cuh for what each kernel computes
// and which reference routine it replaces.
#pragma once
#include <type_traits>
#include "cfd_common.cuh"
#include "pass1.cuh"
#include "regfft.cuh"

namespace cfd {

// per-sequence stride of the stage exchange buffer (+1 spreads the banks when
// consecutive threads work on consecutive sequences)
template <int N> struct SeqPitch {
  static constexpr int V = Split<N>::N1 * (Split<N>::N2 + 1) + 1;
};

// Stage-1 twiddles W_N^(n2*q) stored as tw2[q*N2 + n2] so that consecutive
// threads (consecutive n2) read consecutive words.
template <typename T, int N>
__device__ __forceinline__ void load_tw2(cplx_t<T>* tw2, const cplx_t<T>* __restrict__ tw) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  for (int i = threadIdx.x; i < N1 * N2; i += blockDim.x) {
    const int q = i / N2, n2 = i - q * N2;
    tw2[i] = tw[n2 * q];
  }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// --------------------------------------------------------------------------
// k_zinv_r: grid (nxh, ceil(ny1/YB)), block zinv_r_threads(N, YB) (one thread
// per stage-1 task).  Inverse z transform of the 3/2-padded columns
// (xz_fft_complex_to_real_parallel, PFC/transform.f90:345-368).  The block's
// input -- YB consecutive planes of all kz and the three components of one kx,
// contiguous YB-value runs of data1 -- is gathered with cp.async into a raw
// tile first, so that all of its loads are in flight at once.
template <int N> __host__ __device__ constexpr int zinv_r_threads(int YB) {
  return ((3 * YB * Split<N>::N2 + 31) / 32) * 32;
}
template <typename T> struct ZRawPad {   // 32 bytes between component blocks
  static constexpr int V = 32 / (int)sizeof(cplx_t<T>);
};

template <typename T, int NZ2>
__device__ __forceinline__ void k_zinv_r_body(const uint3 bid, const cplx_t<T>* __restrict__ vel,
                                              cplx_t<T>* __restrict__ T1, Geom g, const cplx_t<T>* __restrict__ twz,
                                              int YB, Scatter sc, int split) {
  using C = cplx_t<T>;
  constexpr int N1 = Split<NZ2>::N1, N2 = Split<NZ2>::N2, PITCH = N2 + 1, SEQ = SeqPitch<NZ2>::V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NZ = g.nz, NY1 = g.ny1, NXH = g.nxh;
  const int RS = NZ * YB + ZRawPad<T>::V;   // raw stride per component
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* raw = tw + NZ2;                         // [c][kz][jj]
  C* Y = raw + 3 * RS;
  const int kx = bid.x;
  const int j0 = bid.y * YB;
  const int nj = min(YB, NY1 - j0);
  const int nseq = 3 * YB;
  const C* col = vel + (size_t)kx * NZ * 3 * NY1;
  {
    // gather: runs of nj planes at (kz, c), 16-byte pieces when aligned
    // 16-byte pieces need 16-byte aligned sources (data1 run starts) and
    // destinations (raw tile: the kz stride YB and the component stride RS)
    const int rb = nj * (int)sizeof(C);
    const bool v16 = (rb % 16) == 0 && ((size_t)NY1 * sizeof(C)) % 16 == 0 && ((size_t)j0 * sizeof(C)) % 16 == 0 &&
                     ((size_t)YB * sizeof(C)) % 16 == 0 && ((size_t)RS * sizeof(C)) % 16 == 0 &&
                     ((size_t)NZ2 * sizeof(C)) % 16 == 0;
    const int psz = v16 ? 16 : 8, np = rb / psz;
    for (int idx = threadIdx.x; idx < 3 * NZ * np; idx += blockDim.x) {
      const int part = idx % np, r = idx / np, kz = r % NZ, c = r / NZ;
      const char* src = reinterpret_cast<const char*>(col + ((size_t)kz * 3 + c) * NY1 + j0) + part * psz;
      char* dst = reinterpret_cast<char*>(raw + c * RS + kz * YB) + part * psz;
      if (v16) cp_async16(dst, src);
      else cp_async8(dst, src);
    }
    cp_async_commit();
  }
  load_tw2<T, NZ2>(tw, twz);
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  if (split && g.kx0 + kx == 0) {
    // mean split: the kx = kz = 0 column leaves the physical fields (the
    // flux kernel adds the mean's products from its FP64 copy)
    for (int i = threadIdx.x; i < 3 * YB; i += blockDim.x) raw[(i / YB) * RS + (i % YB)] = czero<C>();
    __syncthreads();
  }
  const T half = (T)0.5;
  const bool halve_x = (g.nx2 > g.nx) && (g.kx0 + kx == g.nxh_all - 1) && (NZ2 > NZ);
  // stage 1: consecutive threads take consecutive sequences (planes fastest)
  for (int t = threadIdx.x; t < nseq * N2; t += blockDim.x) {
    const int s = t % nseq, n2 = t / nseq;
    const int jj = s % YB, c = s / YB;
    const C* rc = raw + c * RS + jj;
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int m = N2 * n1 + n2;
      C x = czero<C>();
      if (jj < nj) {
        if (NZ2 > NZ) {
          if (m < NZ / 2) x = rc[m * YB];
          else if (m == NZ / 2) x = cscale(half, rc[(NZ / 2) * YB]);
          else if (m == NZ2 - NZ / 2) x = cscale(half, cconj(rc[(NZ / 2) * YB]));
          else if (m > NZ2 - NZ / 2) x = rc[(m - (NZ2 - NZ)) * YB];
          if (halve_x) x = cscale(half, x);
        } else {
          x = rc[m * YB];
        }
      }
      v[n1] = x;
    }
    SmallFFT<T, N1, +1>::template run<1>(v);
    C* y = Y + s * SEQ + n2;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      C x = v[k1];
      if (k1 != 0) x = cmul(x, cconj(tw[k1 * N2 + n2]));
      y[k1 * PITCH] = x;
    }
  }
  __syncthreads();
  // stage 2: consecutive threads take consecutive rows k1 (coalesced stores)
  for (int t = threadIdx.x; t < nseq * N1; t += blockDim.x) {
    const int k1 = t % N1, s = t / N1;
    const int jj = s % YB, c = s / YB;
    C u[N2];
    const C* y = Y + s * SEQ + k1 * PITCH;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) u[n2] = y[n2];
    SmallFFT<T, N2, +1>::template run<1>(u);
    if (jj < nj && sc.n == 0) {
      C* out = T1 + (((size_t)(j0 + jj) * 3 + c) * NXH + kx) * NZ2;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) out[k1 + N1 * k2] = u[k2];
    } else if (jj < nj) {
      // transpose to z2 slabs: element z2 goes to the rank that owns it
      const long long row = ((long long)(j0 + jj) * 3 + c) * g.nxh_all + g.kx0 + kx;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        const int z = k1 + N1 * k2;
        reinterpret_cast<C*>(__ldg(sc.zdst + z))[row * __ldg(sc.zpitch + z)] = u[k2];
      }
    }
  }
}

template <typename T, int NZ2>
__global__ void __launch_bounds__(288, sizeof(T) == 4 ? 3 : 1)
k_zinv_r(const cplx_t<T>* __restrict__ vel, cplx_t<T>* __restrict__ T1, Geom g, const cplx_t<T>* __restrict__ twz,
         int YB, Scatter sc, int split) {
  k_zinv_r_body<T, NZ2>(blockIdx, vel, T1, g, twz, YB, sc, split);
}

// --------------------------------------------------------------------------
// k_zfwd_r: grid (nxh, ceil(ny1/YB)), block 256.  Forward z transform, fold,
// scale and ikz combine (PFC/transform.f90:317-333, 639-688).
template <typename T, int NZ2>
__device__ __forceinline__ void k_zfwd_r_body(const uint3 bid, const cplx_t<T>* __restrict__ T2,
                                              cplx_t<T>* __restrict__ vel, Geom g, const cplx_t<T>* __restrict__ twz,
                                              GridDev gd, int YB) {
  using C = cplx_t<T>;
  constexpr int N1 = Split<NZ2>::N1, N2 = Split<NZ2>::N2, PITCH = N2 + 1, SEQ = SeqPitch<NZ2>::V;
  constexpr int ZP = NZ2 + 1;   // pitch of the stage-2 output (spreads banks across sequences)
  static_assert(ZP <= SEQ, "stage-2 output must fit in the exchange buffer");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int nseq = 6 * YB;
  C* Y = tw + NZ2;
  C* Z = Y;                      // stage 2 reads Y into registers, then overwrites it
  const int NZ = g.nz, NY1 = g.ny1, NXH = g.nxh, ny = g.ny;
  const int kx = bid.x;
  const int j0 = 1 + bid.y * YB;   // 1-based first plane
  __shared__ T skz[NZ2];                 // kz of the retained rows (nz <= nz2)
  load_tw2<T, NZ2>(tw, twz);
  for (int i = threadIdx.x; i < NZ; i += blockDim.x) skz[i] = (T)gd.kz[i];
  __syncthreads();
  for (int t = threadIdx.x; t < nseq * N2; t += blockDim.x) {
    const int s = t / N2, n2 = t - s * N2;
    const int jj = s / 6, e = (s / 2) % 3, part = s & 1;
    const int j = j0 + jj;
    const bool valid = (j >= 2 && j <= ny) && !(e == 1 && j == ny);
    C v[N1];
    const C* src = T2 + ((((size_t)(j - 1) * 3 + e) * 2 + part) * NXH + kx) * NZ2;
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = valid ? src[N2 * n1 + n2] : czero<C>();
    SmallFFT<T, N1, -1>::template run<1>(v);
    C* y = Y + s * SEQ + n2;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      C x = v[k1];
      if (k1 != 0) x = cmul(x, tw[k1 * N2 + n2]);
      y[k1 * PITCH] = x;
    }
  }
  __syncthreads();
  const int off = NZ2 - NZ;
  // stage 2 in rounds of whole sequences: read all rows of the round, then
  // synchronise before overwriting the exchange buffer with the outputs (the
  // output of sequence s only overlaps exchange rows of sequences <= s)
  const int spr = blockDim.x / N1;
  for (int s0 = 0; s0 < nseq; s0 += spr) {
    const int s = s0 + (int)threadIdx.x / N1, k1 = (int)threadIdx.x % N1;
    const bool act = ((int)threadIdx.x < spr * N1) && s < nseq;
    C u[N2];
    if (act) {
      const C* y = Y + s * SEQ + k1 * PITCH;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) u[n2] = y[n2];
    }
    __syncthreads();
    if (act) {
      SmallFFT<T, N2, -1>::template run<1>(u);
      C* z = Z + s * ZP;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        const int k = k1 + N1 * k2;
        if (k <= NZ / 2 || k >= off + NZ / 2) z[k] = u[k2];
      }
    }
    if (s0 + spr < nseq) __syncthreads();
  }
  __syncthreads();
  const T scale = (T)(1.0 / ((double)g.nx2 * (double)g.nz2));
  const T wsc = (g.kx0 + kx == g.nxh_all - 1) ? (T)2 * scale : scale;
  for (int idx = threadIdx.x; idx < NZ * 3 * YB; idx += blockDim.x) {
    const int jj = idx % YB, e = (idx / YB) % 3, kz = idx / (3 * YB);
    const int j = j0 + jj;
    if (j > NY1) continue;
    const bool valid = (j >= 2 && j <= ny) && !(e == 1 && j == ny);
    C out = czero<C>();
    if (valid) {
      const C* A = Z + ((jj * 3 + e) * 2 + 0) * ZP;
      const C* Zc = Z + ((jj * 3 + e) * 2 + 1) * ZP;
      C fa, fz;
      if (kz < NZ / 2) { fa = A[kz]; fz = Zc[kz]; }
      else if (kz == NZ / 2) {
        fa = cadd(A[NZ / 2], cconj(A[off + NZ / 2]));
        fz = cadd(Zc[NZ / 2], cconj(Zc[off + NZ / 2]));
      } else { fa = A[off + kz]; fz = Zc[off + kz]; }
      const C tz = cscale(wsc, fz);
      out = cadd(cimul<C>(skz[kz], tz), cscale(wsc, fa));
    }
    vel[((size_t)(kx * NZ + kz) * 3 + e) * NY1 + (j - 1)] = out;
  }
}

template <typename T, int NZ2>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2)
k_zfwd_r(const cplx_t<T>* __restrict__ T2, cplx_t<T>* __restrict__ vel, Geom g, const cplx_t<T>* __restrict__ twz,
         GridDev gd, int YB) {
  k_zfwd_r_body<T, NZ2>(blockIdx, T2, vel, g, twz, gd, YB);
}

// --------------------------------------------------------------------------
// k_xflux_r: grid (nz2/ZR, nchunks), block 256.  Same computation as k_xflux.
// Per plane: the T1 rows of the next plane are gathered with cp.async into a
// second buffer while the current plane is transformed; the forward x FFT runs
// in place in a padded buffer (row pitch N2+1), which also hosts the inverse
// transform's exchange.
template <typename T, int NX2, bool LIN>
__global__ void __launch_bounds__(256) k_xflux_r(const cplx_t<T>* __restrict__ T1,
                                                 cplx_t<T>* __restrict__ T2, Geom g,
                                                 const cplx_t<T>* __restrict__ twx, GridDev gd,
                                                 const T* __restrict__ fringe, int has_fringe,
                                                 int ZR, int KC,
                                                 unsigned long long* __restrict__ cflbits,
                                                 int do_cfl) {
  using C = cplx_t<T>;
  constexpr int N1 = Split<NX2>::N1, N2 = Split<NX2>::N2, PITCH = N2 + 1, SEQ = SeqPitch<NX2>::V;
  constexpr int N = NX2, Nh = NX2 / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NXH = g.nxh, NZ2 = g.nz2, ny = g.ny;
  const int NSEQ = 4 * ZR + (ZR + 1) / 2;
  const int NREAL = 3 * ZR, NINV = (3 * ZR + 1) / 2;
  C* tw = reinterpret_cast<C*>(smem_raw);                      // tw2[q*N2 + n2]
  T* win = reinterpret_cast<T*>(tw + N);                       // [3 slots][3][ZR][N]
  C* rawb = reinterpret_cast<C*>(win + 9 * ZR * N);            // 2 x [3][NXH][ZR]
  C* FP = rawb + 2 * 3 * NXH * ZR;                             // [NSEQ][SEQ] padded
  const int z0 = blockIdx.x * ZR;
  const int k0 = 2 + blockIdx.y * KC;
  const int k1e = min(k0 + KC, ny + 1);
  if (k0 > ny) return;
  load_tw2<T, N>(tw, twx);
  __shared__ T red[3][8];
  // position of element x of a sequence in the padded layout
  auto px = [](int x) { return (x / N2) * PITCH + (x % N2); };

  const int chunk_bytes = (int)sizeof(C) * ZR;
  const bool v16 = (chunk_bytes % 16) == 0;
  const int ncp = v16 ? chunk_bytes / 16 : chunk_bytes / 8;
  auto issue_gather = [&](int p, C* raw) {
    const bool vok = (p <= ny);
    for (int idx = threadIdx.x; idx < 3 * NXH * ncp; idx += blockDim.x) {
      const int part = idx % ncp, kx = (idx / ncp) % NXH, c = idx / (ncp * NXH);
      char* dst = reinterpret_cast<char*>(raw + (c * NXH + kx) * ZR) + part * (v16 ? 16 : 8);
      if (c == 1 && !vok) {
        if (v16) *reinterpret_cast<float4*>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
        else *reinterpret_cast<float2*>(dst) = make_float2(0.f, 0.f);
      } else {
        const char* src = reinterpret_cast<const char*>(T1 + (((size_t)(p - 1) * 3 + c) * NXH + kx) * NZ2 + z0) +
                          part * (v16 ? 16 : 8);
        if (v16) cp_async16(dst, src);
        else cp_async8(dst, src);
      }
    }
  };

  // inverse x transform of the gathered plane into window slot `slot`
  auto inverse = [&](const C* raw, int slot) {
    for (int t = threadIdx.x; t < NINV * N2; t += blockDim.x) {
      const int i = t / N2, n2 = t - i * N2;
      const int s1 = 2 * i, s2 = 2 * i + 1;
      const int c1 = s1 / ZR, r1 = s1 % ZR, c2 = s2 / ZR, r2 = s2 % ZR;
      C v[N1];
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) {
        const int k = N2 * n1 + n2;
        const int kk = (k <= Nh) ? k : N - k;
        C x1 = czero<C>(), x2 = czero<C>();
        if (kk < NXH) {
          x1 = raw[(c1 * NXH + kk) * ZR + r1];
          if (s2 < NREAL) x2 = raw[(c2 * NXH + kk) * ZR + r2];
        }
        C z;
        if (k == 0 || k == Nh) z = mk<C>(x1.x, x2.x);
        else if (k < Nh) z = mk<C>(x1.x - x2.y, x1.y + x2.x);
        else z = mk<C>(x1.x + x2.y, -x1.y + x2.x);
        v[n1] = z;
      }
      SmallFFT<T, N1, +1>::template run<1>(v);
      C* y = FP + i * SEQ + n2;
#pragma unroll
      for (int q = 0; q < N1; ++q) {
        C x = v[q];
        if (q != 0) x = cmul(x, cconj(tw[q * N2 + n2]));
        y[q * PITCH] = x;
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < NINV * N1; t += blockDim.x) {
      const int q = t % N1, i = t / N1;
      const int s1 = 2 * i, s2 = 2 * i + 1;
      C u[N2];
      const C* y = FP + i * SEQ + q * PITCH;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) u[n2] = y[n2];
      SmallFFT<T, N2, +1>::template run<1>(u);
      T* w1 = win + ((slot * 3) * ZR + s1) * N;
      T* w2 = win + ((slot * 3) * ZR + s2) * N;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        w1[q + N1 * k2] = u[k2].x;
        if (s2 < NREAL) w2[q + N1 * k2] = u[k2].y;
      }
    }
    __syncthreads();
  };

  const T half = (T)0.5, two = (T)2.0;
  auto flux_plane = [&](int k) {
    const int sm = (k - 1) % 3, s0 = k % 3, sp = (k + 1) % 3;
    const T dhk = (T)gd.dh[k - 1];
    const T dnk = (k <= ny - 1) ? (T)gd.dn[k - 1] : (T)0;
    const T iu1 = (k <= ny - 1) ? (T)gd.iu[2 * (k - 1)] : (T)0;
    const T iu2 = (k <= ny - 1) ? (T)gd.iu[2 * (k - 1) + 1] : (T)0;
    const T tu = (T)gd.target[(k - 1)], tv = (T)gd.target[(ny + 1) + (k - 1)];
    const T tw_ = (T)gd.target[2 * (ny + 1) + (k - 1)];
    T B0[3] = {0, 0, 0}, Bm[3] = {0, 0, 0}, Bp[3] = {0, 0, 0};
    if (LIN) {
      for (int q = 0; q < 3; ++q) {
        B0[q] = (T)gd.baseflow[q * (ny + 1) + k - 1];
        Bm[q] = (T)gd.baseflow[q * (ny + 1) + k - 2];
        Bp[q] = (T)gd.baseflow[q * (ny + 1) + k];
      }
    }
    const bool veq = (k <= ny - 1);
    T ma = 0, mb = 0, mc = 0;
    for (int idx = threadIdx.x; idx < ZR * N; idx += blockDim.x) {
      const int x = idx % N, r = idx / N;
#define WIN(s, c) win[(((s) * 3 + (c)) * ZR + r) * N + x]
      const T U = WIN(s0, 0), V = WIN(s0, 1), W = WIN(s0, 2);
      const T Up = WIN(sp, 0), Wp = WIN(sp, 2);
      const T Vp = (k < ny) ? WIN(sp, 1) : V;
      const T Um = WIN(sm, 0), Vm = WIN(sm, 1), Wm = WIN(sm, 2);
#undef WIN
      const T fr = has_fringe ? fringe[(size_t)(z0 + r) * N + x] : (T)0;
      T fpu0, fpw0, fpu, fpw, xfu, zfu, xfw, zfw;
      if (!LIN) {
        if (k == 2) { fpu0 = Vm * Um; fpw0 = Vm * Wm; }
        else { fpu0 = Vm * half * (Um + U); fpw0 = Vm * half * (Wm + W); }
        if (k < ny) { fpu = V * half * (U + Up); fpw = V * half * (W + Wp); }
        else { fpu = V * Up; fpw = V * Wp; }
        xfu = U * U; zfu = W * U; xfw = U * W; zfw = W * W;
      } else {
        if (k == 2) { fpu0 = Bm[1] * Um + Vm * Bm[0]; fpw0 = Bm[1] * Wm + Vm * Bm[2]; }
        else {
          fpu0 = Bm[1] * half * (Um + U) + Vm * half * (Bm[0] + B0[0]);
          fpw0 = Bm[1] * half * (Wm + W) + Vm * half * (Bm[2] + B0[2]);
        }
        if (k < ny) {
          fpu = B0[1] * half * (U + Up) + V * half * (B0[0] + Bp[0]);
          fpw = B0[1] * half * (W + Wp) + V * half * (B0[2] + Bp[2]);
        } else {
          fpu = B0[1] * Up + V * Bp[0];
          fpw = B0[1] * Wp + V * Bp[2];
        }
        xfu = two * B0[0] * U; zfu = B0[2] * U + W * B0[0];
        xfw = B0[2] * U + W * B0[0]; zfw = two * B0[2] * W;
      }
      const T dyu = dhk * (fpu - fpu0) + fr * (U - tu);
      const T dyw = dhk * (fpw - fpw0) + fr * (W - tw_);
      T xfv = 0, dyv = 0, zfv = 0;
      if (veq) {
        T fp0, fp;
        if (!LIN) {
          const T t0 = half * (Vm + V), t1 = half * (V + Vp);
          fp0 = t0 * t0; fp = t1 * t1;
          xfv = V * (iu1 * U + iu2 * Up);
          zfv = V * (iu1 * W + iu2 * Wp);
        } else {
          const T t0 = half * (Vm + V), b0v = half * (Bm[1] + B0[1]);
          const T t1 = half * (V + Vp), b1v = half * (B0[1] + Bp[1]);
          fp0 = two * t0 * b0v; fp = two * t1 * b1v;
          xfv = B0[1] * (iu1 * U + iu2 * Up) + V * (iu1 * B0[0] + iu2 * Bp[0]);
          zfv = B0[1] * (iu1 * W + iu2 * Wp) + V * (iu1 * B0[2] + iu2 * Bp[2]);
        }
        dyv = dnk * (fp - fp0) + fr * (V - tv);
      }
      const int pxx = px(x);
      FP[(4 * r + 0) * SEQ + pxx] = mk<C>(xfu, dyu);
      FP[(4 * r + 1) * SEQ + pxx] = mk<C>(xfw, dyw);
      FP[(4 * r + 2) * SEQ + pxx] = mk<C>(xfv, dyv);
      FP[(4 * r + 3) * SEQ + pxx] = mk<C>(zfu, zfw);
      T* p4 = reinterpret_cast<T*>(FP + (4 * ZR + r / 2) * SEQ + pxx);
      p4[r & 1] = zfv;
      if ((ZR & 1) && r == ZR - 1) p4[1] = 0;
      if (do_cfl) {
        ma = fmax(ma, fabs(U + Up));
        mb = fmax(mb, fabs(V));
        mc = fmax(mc, fabs(W + Wp));
      }
    }
    if (do_cfl) {
      for (int o = 16; o > 0; o >>= 1) {
        ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
        mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
        mc = fmax(mc, __shfl_xor_sync(0xffffffffu, mc, o));
      }
      const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
      if (lane == 0) { red[0][wid] = ma; red[1][wid] = mb; red[2][wid] = mc; }
    }
    __syncthreads();
    if (do_cfl && threadIdx.x < 3) {
      T m = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[threadIdx.x][w]);
      atomicMax(&cflbits[(size_t)(k - 1) * 3 + threadIdx.x],
                (unsigned long long)__double_as_longlong((double)m));
    }
    // forward x FFT of the NSEQ packed sequences, in place
    for (int t = threadIdx.x; t < NSEQ * N2; t += blockDim.x) {
      const int i = t / N2, n2 = t - i * N2;
      C v[N1];
      C* col = FP + i * SEQ + n2;
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) v[n1] = col[n1 * PITCH];
      SmallFFT<T, N1, -1>::template run<1>(v);
#pragma unroll
      for (int q = 0; q < N1; ++q) {
        C x = v[q];
        if (q != 0) x = cmul(x, tw[q * N2 + n2]);
        col[q * PITCH] = x;
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < NSEQ * N1; t += blockDim.x) {
      const int q = t % N1, i = t / N1;
      C u[N2];
      C* row = FP + i * SEQ + q * PITCH;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) u[n2] = row[n2];
      SmallFFT<T, N2, -1>::template run<1>(u);
      // X[q + N1*k2] is kept at row q, column k2
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) row[k2] = u[k2];
    }
    __syncthreads();
    auto X = [&](int i, int kk) -> C { return FP[i * SEQ + (kk % N1) * PITCH + kk / N1]; };
    for (int idx = threadIdx.x; idx < NXH * ZR; idx += blockDim.x) {
      const int r = idx % ZR, kx = idx / ZR;
      const T kxv = (T)gd.kx[kx];
      const int km = (kx == 0) ? 0 : N - kx;
      const size_t base = (size_t)(k - 1) * 6;
#define OUT(e, part) T2[((base + (e) * 2 + (part)) * NXH + kx) * NZ2 + z0 + r]
      for (int e4 = 0; e4 < 4; ++e4) {
        if (e4 == 2 && !veq) continue;
        const C zk = X(4 * r + e4, kx), zm = X(4 * r + e4, km);
        const C E = mk<C>(half * (zk.x + zm.x), half * (zk.y - zm.y));
        const C O = mk<C>(half * (zk.y + zm.y), -half * (zk.x - zm.x));
        if (e4 < 3) {
          const int e = (e4 == 0) ? 0 : (e4 == 1 ? 2 : 1);
          OUT(e, 0) = cadd(O, cimul<C>(kxv, E));
        } else {
          OUT(0, 1) = E;
          OUT(2, 1) = O;
        }
      }
      if (veq) {
        const int i = 4 * ZR + r / 2;
        const C zk = X(i, kx), zm = X(i, km);
        C v;
        if ((r & 1) == 0) v = mk<C>(half * (zk.x + zm.x), half * (zk.y - zm.y));
        else v = mk<C>(half * (zk.y + zm.y), -half * (zk.x - zm.x));
        OUT(1, 1) = v;
      }
#undef OUT
    }
    __syncthreads();
  };

  // software pipeline over the planes k0-1 .. k1e: gather(p+1) overlaps the
  // inverse transform of p and the fluxes / forward transform of p-1
  const int pfirst = k0 - 1, plast = k1e;
  issue_gather(pfirst, rawb);
  cp_async_commit();
  for (int p = pfirst; p <= plast; ++p) {
    if (p + 1 <= plast) issue_gather(p + 1, rawb + ((p + 1 - pfirst) & 1) * 3 * NXH * ZR);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    inverse(rawb + ((p - pfirst) & 1) * 3 * NXH * ZR, p % 3);
    if (p >= k0 + 1) flux_plane(p - 1);
  }
}

// Packed-sequence layout of k_flux_r: the pitch between sequences,
// N1 (N2 + 1) + D complex values, and their order, component-major
// (sequence e ZR + r for component pair e of row r).  D is chosen per length
// to minimise the shared-memory wavefronts of the kernel's four access
// patterns (the point phase's sequence stores, the two FFT stages, the
// output phase's paired reads) over 2-, 4- and 8-row blocks: a pitch that
// keeps consecutive sequences contiguous modulo the 16 eight-byte bank pairs
// frees the FFT stages of conflicts, and the component-major order keeps the
// output phase's rows apart.  (At 144 points: 24 % fewer wavefronts, 10 %
// off the kernel, measured.)  FP64 elements span twice the banks; at 384 and
// 576 points the row-major layout with a pitch of N1 (N2 + 1) + 1 stays
// ahead there.
template <int N> struct FluxSeqPad;
template <> struct FluxSeqPad<24> { static constexpr int D = 10; };
template <> struct FluxSeqPad<48> { static constexpr int D = 0; };
template <> struct FluxSeqPad<72> { static constexpr int D = 2; };
template <> struct FluxSeqPad<96> { static constexpr int D = 0; };
template <> struct FluxSeqPad<144> { static constexpr int D = 0; };
template <> struct FluxSeqPad<192> { static constexpr int D = 12; };
template <> struct FluxSeqPad<288> { static constexpr int D = 4; };
template <> struct FluxSeqPad<384> { static constexpr int D = 8; };
template <> struct FluxSeqPad<576> { static constexpr int D = 0; };
template <typename T, int N> struct FluxSeq {
  static constexpr bool ROWMAJOR = sizeof(T) == 8 && (N == 384 || N == 576);
  static constexpr int V = ROWMAJOR ? SeqPitch<N>::V : Split<N>::N1 * (Split<N>::N2 + 1) + FluxSeqPad<N>::D;
  static constexpr bool EMAJOR = !ROWMAJOR;
};

// --------------------------------------------------------------------------
// Split x stage: k_xinv_r writes the physical planes once, k_flux_r forms the
// fluxes from three neighbouring physical planes and transforms them forward.
// Physical planes P[(pl*3 + c)*nz2 + z][x], pl = 0 .. ny (plane pl+1 of the
// reference's 1-based y index), c = u, v, w.

__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// row pitch (complex values) of the gathered hybrid rows: 16 bytes of padding
// keeps the 16-byte cp.async destinations aligned and the stage-1 reads
// (consecutive threads on consecutive kx) free of bank conflicts
template <int N, int ZB> __host__ __device__ constexpr int xinv_threads() {
  return ((ZB / 2) * Split<N>::N2 + 31) / 32 * 32 < 128 ? 128
       : (((ZB / 2) * Split<N>::N2 + 31) / 32 * 32 > 256 ? 256 : ((ZB / 2) * Split<N>::N2 + 31) / 32 * 32);
}

template <typename T, int ZB> struct RawPitch {
  static constexpr int V = ZB + 16 / (int)sizeof(cplx_t<T>);
};

// k_xinv_r: grid (nz2/ZB, 3, ny+1), block xinv_threads (one thread per
// stage-1 task, at least 128).  Inverse x transform of ZB
// hybrid rows (one plane, one component) into physical rows, two real rows per
// complex FFT (the x part of xz_fft_complex_to_real_parallel,
// PFC/transform.f90:345-368).  v of plane ny+1 is not formed: no flux reads it.
template <typename T, int NX2, int ZB>
__device__ __forceinline__ void k_xinv_r_body(const uint3 bid, const cplx_t<T>* __restrict__ T1, T* __restrict__ P,
                                              Geom g, const cplx_t<T>* __restrict__ twx) {
  using C = cplx_t<T>;
  constexpr int N1 = Split<NX2>::N1, N2 = Split<NX2>::N2, PITCH = N2 + 1, SEQ = SeqPitch<NX2>::V;
  constexpr int N = NX2, Nh = NX2 / 2, NS = ZB / 2, RP = RawPitch<T, ZB>::V;
  constexpr int CH = ZB * (int)sizeof(C) / 16;   // 16-byte chunks per hybrid row
  static_assert(ZB % 2 == 0 && (ZB * sizeof(C)) % 16 == 0, "ZB rows must pack in pairs and 16-byte chunks");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NXH = g.nxh, NZ2 = g.nz2;
  C* tw = reinterpret_cast<C*>(smem_raw);   // [N]
  C* raw = tw + N;                          // [NXH][RP]
  C* Y = raw + NXH * RP;                    // [NS][SEQ]
  const int z0 = bid.x * ZB, c = bid.y, pl = bid.z;
  if (c == 1 && pl == g.ny) return;
  const C* src = T1 + ((size_t)pl * 3 + c) * NXH * NZ2 + z0;
  for (int idx = threadIdx.x; idx < NXH * CH; idx += blockDim.x) {
    const int kx = idx / CH, part = idx - kx * CH;
    cp_async16(reinterpret_cast<char*>(raw + kx * RP) + part * 16,
               reinterpret_cast<const char*>(src + (size_t)kx * NZ2) + part * 16);
  }
  cp_async_commit();
  load_tw2<T, N>(tw, twx);
  cp_async_wait0();
  __syncthreads();
  for (int t = threadIdx.x; t < NS * N2; t += blockDim.x) {
    const int i = t / N2, n2 = t - i * N2;
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int k = N2 * n1 + n2;
      const int kk = (k <= Nh) ? k : N - k;
      C x1 = czero<C>(), x2 = czero<C>();
      if (kk < NXH) {
        x1 = raw[kk * RP + 2 * i];
        x2 = raw[kk * RP + 2 * i + 1];
      }
      C z;
      if (k == 0 || k == Nh) z = mk<C>(x1.x, x2.x);
      else if (k < Nh) z = mk<C>(x1.x - x2.y, x1.y + x2.x);
      else z = mk<C>(x1.x + x2.y, -x1.y + x2.x);
      v[n1] = z;
    }
    SmallFFT<T, N1, +1>::template run<1>(v);
    C* y = Y + i * SEQ + n2;
#pragma unroll
    for (int q = 0; q < N1; ++q) {
      C x = v[q];
      if (q != 0) x = cmul(x, cconj(tw[q * N2 + n2]));
      y[q * PITCH] = x;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < NS * N1; t += blockDim.x) {
    const int q = t % N1, i = t / N1;
    C u[N2];
    const C* y = Y + i * SEQ + q * PITCH;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) u[n2] = y[n2];
    SmallFFT<T, N2, +1>::template run<1>(u);
    T* w1 = P + (((size_t)pl * 3 + c) * NZ2 + z0 + 2 * i) * N;
    T* w2 = w1 + N;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      w1[q + N1 * k2] = u[k2].x;
      w2[q + N1 * k2] = u[k2].y;
    }
  }
}

template <typename T, int NX2, int ZB>
__global__ void __launch_bounds__(256)
k_xinv_r(const cplx_t<T>* __restrict__ T1, T* __restrict__ P, Geom g, const cplx_t<T>* __restrict__ twx) {
  k_xinv_r_body<T, NX2, ZB>(blockIdx, T1, P, g, twx);
}

// k_flux_r: grid (nz2/ZR, ny-1), block NT.  Fluxes of plane k = 2 + blockIdx.y
// on ZR rows of z from the physical planes k-1, k, k+1, then the forward x
// transform and the Hermitian unpacking into T2 -- the same arithmetic and
// output as k_xflux_r (PFC/pass1.f90:134-226, PFC/transform.f90:287-315).
// MODE 0: the nonlinear products; 1: the linearized products about the
// baseflow (PFC/pass1_linearized.f90:135-509); 3: the nonlinear products of
// a field split into its plane mean B (gd.baseflow, FP64) and the rest u
// (the physical planes, mean column removed): (B + u)(B + u) - B B = the
// linearized products plus u u, the mean-mean products being constant in x
// and z (their divergence is the y derivative of B_i V, zero without net
// transpiration), the fringe and CFL on B + u; 2: the nonlinear products plus
// the subgrid stresses of the LES mode, S[pl][6][nz2][nx2] on the yh planes
// (components 11, 22, 33, 12, 13, 23; zero on the walls), added to the
// momentum fluxes at the same points (y-plane values interpolated as the
// velocities are: half sums for the u and w equations, iu for the v one).
template <typename T, int NX2, int ZR, int NT, int MODE>
__device__ __forceinline__ void k_flux_r_body(const uint3 bid, const T* __restrict__ P, cplx_t<T>* __restrict__ T2,
                                              Geom g, const cplx_t<T>* __restrict__ twx, GridDev gd,
                                              const T* __restrict__ fringe, int has_fringe,
                                              unsigned long long* __restrict__ cflbits, int do_cfl, Scatter sc,
                                              const T* __restrict__ S) {
  constexpr bool LIN = MODE == 1, SGS = MODE == 2, SPLIT = MODE == 3;
  constexpr bool HASB = LIN || SPLIT;
  using C = cplx_t<T>;
  constexpr int N1 = Split<NX2>::N1, N2 = Split<NX2>::N2, PITCH = N2 + 1, SEQ = FluxSeq<T, NX2>::V;
  // sequence of component pair e of row r
  auto sidx = [](int r, int e) { return FluxSeq<T, NX2>::EMAJOR ? e * ZR + r : 4 * r + e; };
  constexpr int N = NX2;
  // four packed sequences per row: (xfu,dyu) (xfw,dyw) (xfv,dyv) (zfw,zfv);
  // zfu = w*u equals xfw = u*w (and likewise in the linearized products), so
  // its transform is taken from the second sequence
  constexpr int NSEQ = 4 * ZR;
  constexpr int NW = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);   // tw2[q*N2 + n2]
  C* FP = tw + N;                           // [NSEQ][SEQ] padded sequences
  __shared__ T red[3][NW];
  __shared__ T skx[NX2 / 2 + 2];             // kx of the retained columns (nx/2+1 <= nx2/2+1)
  const int NXH = g.nxh, NZ2 = g.nz2, ny = g.ny;
  const int z0 = bid.x * ZR;
  const int k = 2 + bid.y;
  load_tw2<T, N>(tw, twx);
  for (int i = threadIdx.x; i < g.nxh; i += NT) skx[i] = (T)gd.kx[i];
  auto px = [](int x) { return (x / N2) * PITCH + (x % N2); };
  const T half = (T)0.5, two = (T)2.0;
  const T dhk = (T)gd.dh[k - 1];
  const bool veq = (k <= ny - 1);
  const T dnk = veq ? (T)gd.dn[k - 1] : (T)0;
  const T iu1 = veq ? (T)gd.iu[2 * (k - 1)] : (T)0;
  const T iu2 = veq ? (T)gd.iu[2 * (k - 1) + 1] : (T)0;
  const T tu = (T)gd.target[(k - 1)], tv = (T)gd.target[(ny + 1) + (k - 1)];
  const T tw_ = (T)gd.target[2 * (ny + 1) + (k - 1)];
  T B0[3] = {0, 0, 0}, Bm[3] = {0, 0, 0}, Bp[3] = {0, 0, 0};
  if (HASB) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      B0[q] = (T)gd.baseflow[q * (ny + 1) + k - 1];
      Bm[q] = (T)gd.baseflow[q * (ny + 1) + k - 2];
      Bp[q] = (T)gd.baseflow[q * (ny + 1) + k];
    }
  }
  // the mean's half sums onto the y planes k-1 and k and its iu-weighted
  // values (mean split)
  T hBm[3], hBp[3], iuB[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    hBm[q] = half * (Bm[q] + B0[q]);
    hBp[q] = half * (B0[q] + Bp[q]);
    iuB[q] = iu1 * B0[q] + iu2 * Bp[q];
  }
  // rows of planes k-1 (index k-2), k, k+1 for component c and row r
  const size_t pstride = (size_t)3 * NZ2 * N;
  const T* Pm = P + (size_t)(k - 2) * pstride + (size_t)z0 * N;
  const T* P0 = Pm + pstride;
  const T* Pp = P0 + pstride;
  const size_t cs = (size_t)NZ2 * N;
  T ma = 0, mb = 0, mc = 0;
  // fluxes of one point (r, x) into the packed sequences; tau: the subgrid
  // stresses of the point (SGS mode): 11, 22, 33, 12, 13, 23 at yh plane k,
  // then 12, 23 at plane k-1 and 12, 22, 23 at plane k+1
  auto point = [&](T U, T V, T W, T Up, T Vp, T Wp, T Um, T Vm, T Wm, T fr, int r, int x, const T* tau) {
  T fpu0 = 0, fpw0 = 0, fpu = 0, fpw = 0, xfu = 0, zfu = 0, xfw = 0, zfw = 0;
  if (SPLIT) {
    // (B + u)(B + u) - B B factored: the fluctuation's products and the
    // mean's in one pass (block constants hold the mean's half sums)
    if (k == 2) { fpu0 = (Vm + Bm[1]) * Um + Vm * Bm[0]; fpw0 = (Vm + Bm[1]) * Wm + Vm * Bm[2]; }
    else { fpu0 = (Vm + Bm[1]) * (half * (Um + U)) + Vm * hBm[0]; fpw0 = (Vm + Bm[1]) * (half * (Wm + W)) + Vm * hBm[2]; }
    if (k < ny) { fpu = (V + B0[1]) * (half * (U + Up)) + V * hBp[0]; fpw = (V + B0[1]) * (half * (W + Wp)) + V * hBp[2]; }
    else { fpu = (V + B0[1]) * Up + V * Bp[0]; fpw = (V + B0[1]) * Wp + V * Bp[2]; }
    xfu = U * (U + two * B0[0]);
    zfu = U * (W + B0[2]) + W * B0[0];
    xfw = zfu;
    zfw = W * (W + two * B0[2]);
  } else if (!LIN) {
    if (k == 2) { fpu0 = Vm * Um; fpw0 = Vm * Wm; }
    else { fpu0 = Vm * half * (Um + U); fpw0 = Vm * half * (Wm + W); }
    if (k < ny) { fpu = V * half * (U + Up); fpw = V * half * (W + Wp); }
    else { fpu = V * Up; fpw = V * Wp; }
    xfu = U * U; zfu = W * U; xfw = U * W; zfw = W * W;
    if (SGS) {
      xfu += tau[0]; zfu += tau[4]; xfw += tau[4]; zfw += tau[2];
      // y-plane k-1 (zero on the bottom wall) and y-plane k (zero on the top one)
      if (k > 2) { fpu0 += half * (tau[6] + tau[3]); fpw0 += half * (tau[7] + tau[5]); }
      if (k < ny) { fpu += half * (tau[3] + tau[8]); fpw += half * (tau[5] + tau[10]); }
    }
  }
  if (LIN) {
    if (k == 2) { fpu0 += Bm[1] * Um + Vm * Bm[0]; fpw0 += Bm[1] * Wm + Vm * Bm[2]; }
    else {
      fpu0 += Bm[1] * half * (Um + U) + Vm * half * (Bm[0] + B0[0]);
      fpw0 += Bm[1] * half * (Wm + W) + Vm * half * (Bm[2] + B0[2]);
    }
    if (k < ny) {
      fpu += B0[1] * half * (U + Up) + V * half * (B0[0] + Bp[0]);
      fpw += B0[1] * half * (W + Wp) + V * half * (B0[2] + Bp[2]);
    } else {
      fpu += B0[1] * Up + V * Bp[0];
      fpw += B0[1] * Wp + V * Bp[2];
    }
    xfu += two * B0[0] * U; zfu += B0[2] * U + W * B0[0];
    xfw += B0[2] * U + W * B0[0]; zfw += two * B0[2] * W;
  }
  // the fringe acts on the whole velocity (its mean included when split)
  const T Uf = SPLIT ? U + B0[0] : U, Wf = SPLIT ? W + B0[2] : W, Vf = SPLIT ? V + B0[1] : V;
  const T dyu = dhk * (fpu - fpu0) + fr * (Uf - tu);
  const T dyw = dhk * (fpw - fpw0) + fr * (Wf - tw_);
  T xfv = 0, dyv = 0, zfv = 0;
  if (veq) {
    T fp0 = 0, fp = 0;
    if (SPLIT) {
      const T t0 = half * (Vm + V), t1 = half * (V + Vp);
      fp0 = t0 * (t0 + two * hBm[1]);
      fp = t1 * (t1 + two * hBp[1]);
      xfv = (V + B0[1]) * (iu1 * U + iu2 * Up) + V * iuB[0];
      zfv = (V + B0[1]) * (iu1 * W + iu2 * Wp) + V * iuB[2];
    } else if (!LIN) {
      const T t0 = half * (Vm + V), t1 = half * (V + Vp);
      fp0 = t0 * t0; fp = t1 * t1;
      xfv = V * (iu1 * U + iu2 * Up);
      zfv = V * (iu1 * W + iu2 * Wp);
      if (SGS) {
        xfv += iu1 * tau[3] + iu2 * tau[8];
        zfv += iu1 * tau[5] + iu2 * tau[10];
        fp0 += tau[1];
        fp += tau[9];
      }
    }
    if (LIN) {
      const T t0 = half * (Vm + V), b0v = half * (Bm[1] + B0[1]);
      const T t1 = half * (V + Vp), b1v = half * (B0[1] + Bp[1]);
      fp0 += two * t0 * b0v; fp += two * t1 * b1v;
      xfv += B0[1] * (iu1 * U + iu2 * Up) + V * (iu1 * B0[0] + iu2 * Bp[0]);
      zfv += B0[1] * (iu1 * W + iu2 * Wp) + V * (iu1 * B0[2] + iu2 * Bp[2]);
    }
    dyv = dnk * (fp - fp0) + fr * (Vf - tv);
  }
  const int pxx = px(x);
  (void)zfu;
  FP[sidx(r, 0) * SEQ + pxx] = mk<C>(xfu, dyu);
  FP[sidx(r, 1) * SEQ + pxx] = mk<C>(xfw, dyw);
  FP[sidx(r, 2) * SEQ + pxx] = mk<C>(xfv, dyv);
  FP[sidx(r, 3) * SEQ + pxx] = mk<C>(zfw, zfv);
    if (do_cfl) {
      if (SPLIT) {
        ma = fmax(ma, fabs(U + Up + B0[0] + Bp[0]));
        mb = fmax(mb, fabs(V + B0[1]));
        mc = fmax(mc, fabs(W + Wp + B0[2] + Bp[2]));
      } else {
        ma = fmax(ma, fabs(U + Up));
        mb = fmax(mb, fabs(V));
        mc = fmax(mc, fabs(W + Wp));
      }
    }
  };
  // two neighbouring x per thread and 8- or 16-byte loads (x even, rows of
  // even length)
  using V2 = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
  static_assert(N % 2 == 0, "even rows");
  constexpr int IT = (ZR * N / 2 + NT - 1) / NT;
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int idx = it * NT + (int)threadIdx.x;
    if ((ZR * N / 2) % NT != 0 && idx >= ZR * N / 2) break;
    const int x = 2 * (idx % (N / 2)), r = idx / (N / 2);
    const size_t o = (size_t)r * N + x;
    auto ld2 = [&](const T* b) { return __ldg(reinterpret_cast<const V2*>(b + o)); };
    const V2 U = ld2(P0), V = ld2(P0 + cs), W = ld2(P0 + 2 * cs);
    const V2 Up = ld2(Pp), Wp = ld2(Pp + 2 * cs);
    const V2 Vp = (k < ny) ? ld2(Pp + cs) : V;
    const V2 Um = ld2(Pm), Vm = ld2(Pm + cs), Wm = ld2(Pm + 2 * cs);
    V2 fr;
    if (has_fringe) fr = __ldg(reinterpret_cast<const V2*>(fringe + (size_t)(z0 + r) * N + x));
    else { fr.x = (T)0; fr.y = (T)0; }
    T ta[11], tb[11];
    if (SGS) {
      // S planes k-1, k, k+1 are S indices k-2, k-1, k (six components each)
      const size_t ss = (size_t)6 * NZ2 * N, so = (size_t)(k - 1) * ss + (size_t)(z0 + r) * N + x;
      const int c0[11] = {0, 1, 2, 3, 4, 5, 3, 5, 3, 1, 5};
      const int pd[11] = {0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 1};
#pragma unroll
      for (int q = 0; q < 11; ++q) {
        const V2 v = __ldg(reinterpret_cast<const V2*>(S + (size_t)((long long)so + (long long)pd[q] * (long long)ss) +
                                                       (size_t)c0[q] * NZ2 * N));
        ta[q] = v.x;
        tb[q] = v.y;
      }
    }
    point(U.x, V.x, W.x, Up.x, Vp.x, Wp.x, Um.x, Vm.x, Wm.x, fr.x, r, x, ta);
    point(U.y, V.y, W.y, Up.y, Vp.y, Wp.y, Um.y, Vm.y, Wm.y, fr.y, r, x + 1, tb);
  }
  if (do_cfl) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
      mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
      mc = fmax(mc, __shfl_xor_sync(0xffffffffu, mc, o));
    }
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { red[0][wid] = ma; red[1][wid] = mb; red[2][wid] = mc; }
  }
  __syncthreads();
  if (do_cfl && threadIdx.x < 3) {
    T m = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) m = fmax(m, red[threadIdx.x][w]);
    atomicMax(&cflbits[(size_t)(k - 1) * 3 + threadIdx.x], (unsigned long long)__double_as_longlong((double)m));
  }
  // forward x FFT of the NSEQ packed sequences, in place
  for (int t = threadIdx.x; t < NSEQ * N2; t += NT) {
    const int i = t / N2, n2 = t - i * N2;
    C v[N1];
    C* col = FP + i * SEQ + n2;
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = col[n1 * PITCH];
    SmallFFT<T, N1, -1>::template run<1>(v);
#pragma unroll
    for (int q = 0; q < N1; ++q) {
      C x = v[q];
      if (q != 0) x = cmul(x, tw[q * N2 + n2]);
      col[q * PITCH] = x;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < NSEQ * N1; t += NT) {
    const int q = t % N1, i = t / N1;
    C u[N2];
    C* row = FP + i * SEQ + q * PITCH;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) u[n2] = row[n2];
    SmallFFT<T, N2, -1>::template run<1>(u);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) row[k2] = u[k2];
  }
  __syncthreads();
  auto X = [&](int i, int kk) -> C { return FP[i * SEQ + (kk % N1) * PITCH + kk / N1]; };
  const size_t base = (size_t)(k - 1) * 6;
  for (int idx = threadIdx.x; idx < NXH * ZR; idx += NT) {
    const int r = idx % ZR, kx = idx / ZR;
    const T kxv = skx[kx];
    const int km = (kx == 0) ? 0 : N - kx;
    // one rank: local layout; several: column kx goes to the rank that owns it
    C* const od = sc.n ? reinterpret_cast<C*>(__ldg(sc.xdst + kx)) + z0 + r : T2 + (size_t)kx * NZ2 + z0 + r;
    const size_t op = sc.n ? (size_t)__ldg(sc.xpitch + kx) : (size_t)NXH * NZ2;
#define OUT(e, part) od[(base + (e) * 2 + (part)) * op]
#pragma unroll
    for (int e4 = 0; e4 < 4; ++e4) {
      if (e4 == 2 && !veq) continue;
      const C zk = X(sidx(r, e4), kx), zm = X(sidx(r, e4), km);
      const C E = mk<C>(half * (zk.x + zm.x), half * (zk.y - zm.y));
      const C O = mk<C>(half * (zk.y + zm.y), -half * (zk.x - zm.x));
      if (e4 < 3) {
        const int e = (e4 == 0) ? 0 : (e4 == 1 ? 2 : 1);
        OUT(e, 0) = cadd(O, cimul<C>(kxv, E));
        if (e4 == 1) OUT(0, 1) = E;
      } else {
        OUT(2, 1) = E;
        if (veq) OUT(1, 1) = O;
      }
    }
#undef OUT
  }
}

template <typename T, int NX2, int ZR, int NT, int MODE>
__global__ void __launch_bounds__(NT, sizeof(T) == 4 ? (NT == 256 ? 4 : 6) : (NT == 256 ? 1 : 3))
k_flux_r(const T* __restrict__ P, cplx_t<T>* __restrict__ T2, Geom g, const cplx_t<T>* __restrict__ twx, GridDev gd,
         const T* __restrict__ fringe, int has_fringe, unsigned long long* __restrict__ cflbits, int do_cfl,
         Scatter sc, const T* __restrict__ S) {
  k_flux_r_body<T, NX2, ZR, NT, MODE>(blockIdx, P, T2, g, twx, gd, fringe, has_fringe, cflbits, do_cfl, sc, S);
}

// smem sizes (bytes) of the three kernels
template <typename T, int N> size_t zinv_r_smem(int YB, int nz) {
  return sizeof(cplx_t<T>) * (N + 3 * ((size_t)nz * YB + ZRawPad<T>::V) + (size_t)3 * YB * SeqPitch<N>::V);
}
template <typename T, int N> constexpr size_t zfwd_r_smem(int YB) {
  return sizeof(cplx_t<T>) * (N + (size_t)6 * YB * SeqPitch<N>::V);
}
template <typename T, int N, int ZB> constexpr size_t xinv_r_smem(int NXH) {
  return sizeof(cplx_t<T>) * (N + (size_t)NXH * RawPitch<T, ZB>::V + (size_t)(ZB / 2) * SeqPitch<N>::V);
}
template <typename T, int N, int ZR> constexpr size_t flux_r_smem() {
  return sizeof(cplx_t<T>) * (N + (size_t)(4 * ZR) * FluxSeq<T, N>::V);
}
template <typename T, int N> constexpr size_t xflux_r_smem(int ZR, int NXH) {
  return sizeof(cplx_t<T>) * N + sizeof(T) * 9 * (size_t)ZR * N + sizeof(cplx_t<T>) * (6 * (size_t)ZR * NXH)
         + sizeof(cplx_t<T>) * (size_t)(4 * ZR + (ZR + 1) / 2) * SeqPitch<N>::V;
}

}  // namespace cfd
