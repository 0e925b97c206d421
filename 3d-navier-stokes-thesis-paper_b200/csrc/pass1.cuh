// pass1.cuh -- dealiased x-z transforms and the nonlinear (or linearized)
// flux divergence of PFC/pass1.f90:26-250, PFC/pass1_linearized.f90:135-508
// and PFC/transform.f90:258-409,573-690, as three sm_100a kernels:
//
//   k_zinv  : spectral velocity  -> hybrid (z physical, kx spectral) planes
//             z-padding to nz2 with the Nyquist split and x-Nyquist halving
//             of xz_fft_complex_to_real_parallel, inverse z FFT.
//   k_xflux : per z-row, sliding up the planes: inverse x c2r of u,v,w,
//             staggered products and y-differences of compute_wall_parallel_
//             flux / compute_wall_normal_flux, fringe term, forward x r2c and
//             ikx combine of parallel_divergence_of_fluxes, CFL maxima.
//   k_zfwd  : forward z FFT, Nyquist fold, truncation, 1/(nx2 nz2) scale,
//             last-kx doubling, ikz combine -> nonlinear term in data1 slots.
//
// Device layouts (y fastest for the spectral state, as data2 in the
// reference):  vel  [kx][kz][comp][y]
//              T1   [plane][comp][kx][z2]           (hybrid, after k_zinv)
//              T2   [plane][eq][part][kx][z2]       (part 0: dY+ikx X, 1: Z)
#pragma once
#include "cfd_common.cuh"
#include "fft.cuh"

namespace cfd {

struct DevScalars {
  double t_total, dt, p_grad, cfl_max;
  int status;
  int pad;
};

struct GridDev {   // device copies of the grid operators (FP64)
  const double *y, *yh, *hn, *dh, *dn, *iu, *dm, *d2h, *d2n, *dyh, *dy, *kx, *kz;
  const double *target;    // (ny+1, 3)
  const double *baseflow;  // (ny+1, 3)
};

// --------------------------------------------------------------------------
// k_zinv: grid (nxh, ceil(ny1/YB)), block 256.
template <typename T>
__global__ void __launch_bounds__(256) k_zinv(const cplx_t<T>* __restrict__ vel,
                                              cplx_t<T>* __restrict__ T1, Geom g,
                                              FftPlan pz, const cplx_t<T>* __restrict__ twz,
                                              int YB, int pl0, int pl1) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int NZ = g.nz, NZ2 = g.nz2, NY1 = g.ny1;
  C* b0 = tw + NZ2;
  const int nseq = 3 * YB;
  C* b1 = b0 + nseq * NZ2;
  const int kx = blockIdx.x;
  const int j0 = pl0 + blockIdx.y * YB;
  const int nj = min(YB, pl1 - j0);
  for (int m = threadIdx.x; m < NZ2; m += blockDim.x) tw[m] = twz[m];
  for (int i = threadIdx.x; i < nseq * NZ2; i += blockDim.x) b0[i] = czero<C>();
  __syncthreads();
  const T half = (T)0.5;
  const bool halve_x = (g.nx2 > g.nx) && (kx == g.nxh - 1) && (NZ2 > NZ);
  for (int idx = threadIdx.x; idx < NZ * 3 * YB; idx += blockDim.x) {
    const int jj = idx % YB, c = (idx / YB) % 3, kz = idx / (3 * YB);
    if (jj >= nj) continue;
    C v = vel[((size_t)(kx * NZ + kz) * 3 + c) * NY1 + j0 + jj];
    C* seq = b0 + (c * YB + jj) * NZ2;
    if (NZ2 > NZ) {
      if (halve_x) v = cscale(half, v);
      if (kz < NZ / 2) seq[kz] = v;
      else if (kz == NZ / 2) {
        seq[NZ / 2] = cscale(half, v);
        seq[NZ2 - NZ / 2] = cscale(half, cconj(v));
      } else seq[kz + NZ2 - NZ] = v;
    } else {
      seq[kz] = v;
    }
  }
  __syncthreads();
  C* res = block_fft<T>(b0, b1, pz, nseq, NZ2, tw, +1);
  for (int idx = threadIdx.x; idx < nseq * NZ2; idx += blockDim.x) {
    const int m = idx % NZ2, s = idx / NZ2, c = s / YB, jj = s % YB;
    if (jj >= nj) continue;
    T1[(((size_t)(j0 + jj) * 3 + c) * g.nxh + kx) * NZ2 + m] = res[idx];
  }
}

// --------------------------------------------------------------------------
// Loads one plane (1-based p) of u, v, w for ZR consecutive z rows from T1 and
// inverse-transforms them in x (FFTW c2r semantics: Im of the DC and Nyquist
// inputs ignored) into window slot `slot`, two real rows per complex FFT.
template <typename T>
__device__ void load_plane_rows(const cplx_t<T>* __restrict__ T1, const Geom& g,
                                const FftPlan& px, const cplx_t<T>* tw, T* win,
                                cplx_t<T>* b0, cplx_t<T>* b1, int p, int slot,
                                int z0, int ZR) {
  using C = cplx_t<T>;
  const int NXH = g.nxh, NX2 = g.nx2, NZ2 = g.nz2;
  const int nreal = 3 * ZR, npair = (nreal + 1) / 2;
  const bool vok = (p <= g.ny);
  C* raw = b1;   // [s][kx], s = c*ZR + r
  for (int idx = threadIdx.x; idx < 3 * NXH * ZR; idx += blockDim.x) {
    const int r = idx % ZR, kx = (idx / ZR) % NXH, c = idx / (ZR * NXH);
    C v = czero<C>();
    if (c != 1 || vok) v = T1[(((size_t)(p - 1) * 3 + c) * NXH + kx) * NZ2 + z0 + r];
    raw[(c * ZR + r) * NXH + kx] = v;
  }
  __syncthreads();
  const int N = NX2, Nh = NX2 / 2;
  for (int idx = threadIdx.x; idx < npair * N; idx += blockDim.x) {
    const int k = idx % N, i = idx / N;
    const int s1 = 2 * i, s2 = 2 * i + 1;
    C x1 = czero<C>(), x2 = czero<C>();
    const int kk = (k <= Nh) ? k : N - k;
    if (kk < NXH) {
      x1 = raw[s1 * NXH + kk];
      if (s2 < nreal) x2 = raw[s2 * NXH + kk];
    }
    C z;
    if (k == 0 || k == Nh) z = mk<C>(x1.x, x2.x);
    else if (k < Nh) z = mk<C>(x1.x - x2.y, x1.y + x2.x);
    else z = mk<C>(x1.x + x2.y, -x1.y + x2.x);
    b0[i * N + k] = z;
  }
  __syncthreads();
  C* res = block_fft<T>(b0, b1, px, npair, N, tw, +1);
  for (int idx = threadIdx.x; idx < npair * N; idx += blockDim.x) {
    const int k = idx % N, i = idx / N;
    const int s1 = 2 * i, s2 = 2 * i + 1;
    C z = res[idx];
    win[((slot * 3) * ZR + s1) * N + k] = z.x;   // s = c*ZR + r maps to [slot][c][r]
    if (s2 < nreal) win[((slot * 3) * ZR + s2) * N + k] = z.y;
  }
  __syncthreads();
}

// k_xflux: grid (nz2/ZR, nchunks), block 256.  Computes the Fourier-x
// transformed fluxes of planes k in [k0, k1) (1-based, 2 <= k <= ny).
template <typename T, bool LIN>
__global__ void __launch_bounds__(256) k_xflux(const cplx_t<T>* __restrict__ T1,
                                               cplx_t<T>* __restrict__ T2, Geom g,
                                               FftPlan px, const cplx_t<T>* __restrict__ twx,
                                               GridDev gd, const T* __restrict__ fringe,
                                               int has_fringe, int ZR, int KC,
                                               unsigned long long* __restrict__ cflbits,
                                               int do_cfl) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NX2 = g.nx2, NXH = g.nxh, NZ2 = g.nz2, ny = g.ny;
  C* tw = reinterpret_cast<C*>(smem_raw);
  T* win = reinterpret_cast<T*>(tw + NX2);             // [3 slots][3][ZR][NX2]
  C* b0 = reinterpret_cast<C*>(win + 9 * ZR * NX2);
  const int NSEQ = 4 * ZR + (ZR + 1) / 2;
  const int nbuf = max(NSEQ, (3 * ZR + 1) / 2 + 0) * NX2;
  const int nbuf1 = max(nbuf, 3 * ZR * NXH);
  C* b1 = b0 + nbuf;
  (void)nbuf1;
  const int z0 = blockIdx.x * ZR;
  const int k0 = 2 + blockIdx.y * KC;
  const int k1 = min(k0 + KC, ny + 1);
  if (k0 > ny) return;
  for (int m = threadIdx.x; m < NX2; m += blockDim.x) tw[m] = twx[m];
  __syncthreads();
  load_plane_rows<T>(T1, g, px, tw, win, b0, b1, k0 - 1, (k0 - 1) % 3, z0, ZR);
  load_plane_rows<T>(T1, g, px, tw, win, b0, b1, k0, k0 % 3, z0, ZR);
  const T half = (T)0.5, two = (T)2.0;
  __shared__ T red[3][8];
  for (int k = k0; k < k1; ++k) {
    load_plane_rows<T>(T1, g, px, tw, win, b0, b1, k + 1, (k + 1) % 3, z0, ZR);
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
    for (int idx = threadIdx.x; idx < ZR * NX2; idx += blockDim.x) {
      const int x = idx % NX2, r = idx / NX2;
#define WIN(s, c) win[(((s) * 3 + (c)) * ZR + r) * NX2 + x]
      const T U = WIN(s0, 0), V = WIN(s0, 1), W = WIN(s0, 2);
      const T Up = WIN(sp, 0), Wp = WIN(sp, 2);
      const T Vp = (k < ny) ? WIN(sp, 1) : V;
      const T Um = WIN(sm, 0), Vm = WIN(sm, 1), Wm = WIN(sm, 2);
#undef WIN
      const T fr = has_fringe ? fringe[(size_t)(z0 + r) * NX2 + x] : (T)0;
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
      b0[(4 * r + 0) * NX2 + x] = mk<C>(xfu, dyu);
      b0[(4 * r + 1) * NX2 + x] = mk<C>(xfw, dyw);
      b0[(4 * r + 2) * NX2 + x] = mk<C>(xfv, dyv);
      b0[(4 * r + 3) * NX2 + x] = mk<C>(zfu, zfw);
      T* p4 = reinterpret_cast<T*>(b0 + (4 * ZR + r / 2) * NX2 + x);
      p4[r & 1] = zfv;
      if ((ZR & 1) && r == ZR - 1) p4[1] = 0;
      if (do_cfl) {
        ma = fmax(ma, fabs(U + Up));
        mb = fmax(mb, fabs(V));
        mc = fmax(mc, fabs(W + Wp));
      }
    }
    if (do_cfl) {
      // block max -> atomicMax on the IEEE bits (non-negative values)
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
      double md = (double)m;
      atomicMax(&cflbits[(size_t)(k - 1) * 3 + threadIdx.x],
                (unsigned long long)__double_as_longlong(md));
    }
    C* res = block_fft<T>(b0, b1, px, NSEQ, NX2, tw, -1);
    const T kxs = 0;  (void)kxs;
    for (int idx = threadIdx.x; idx < NXH * ZR; idx += blockDim.x) {
      const int r = idx % ZR, kx = idx / ZR;
      const T kxv = (T)gd.kx[kx];
      const int km = (kx == 0) ? 0 : NX2 - kx;
      const size_t base = (size_t)(k - 1) * 6;
#define OUT(e, part) T2[((base + (e) * 2 + (part)) * NXH + kx) * NZ2 + z0 + r]
      for (int e4 = 0; e4 < 4; ++e4) {
        if (e4 == 2 && !veq) continue;
        const C zk = res[(4 * r + e4) * NX2 + kx], zm = res[(4 * r + e4) * NX2 + km];
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
        const C zk = res[i * NX2 + kx], zm = res[i * NX2 + km];
        C v;
        if ((r & 1) == 0) v = mk<C>(half * (zk.x + zm.x), half * (zk.y - zm.y));
        else v = mk<C>(half * (zk.y + zm.y), -half * (zk.x - zm.x));
        OUT(1, 1) = v;
      }
#undef OUT
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------------
// k_zfwd: grid (nxh, ceil(ny1/YB)), block 256.
template <typename T>
__global__ void __launch_bounds__(256) k_zfwd(const cplx_t<T>* __restrict__ T2,
                                              cplx_t<T>* __restrict__ vel, Geom g,
                                              FftPlan pz, const cplx_t<T>* __restrict__ twz,
                                              GridDev gd, int YB) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int NZ = g.nz, NZ2 = g.nz2, NY1 = g.ny1, NXH = g.nxh, ny = g.ny;
  C* b0 = tw + NZ2;
  const int nseq = 6 * YB;
  C* b1 = b0 + nseq * NZ2;
  const int kx = blockIdx.x;
  const int j0 = 1 + blockIdx.y * YB;   // 1-based first plane
  for (int m = threadIdx.x; m < NZ2; m += blockDim.x) tw[m] = twz[m];
  for (int idx = threadIdx.x; idx < nseq * NZ2; idx += blockDim.x) {
    const int m = idx % NZ2, s = idx / NZ2;
    const int jj = s / 6, e = (s / 2) % 3, part = s & 1;
    const int j = j0 + jj;
    const bool valid = (j >= 2 && j <= ny) && !(e == 1 && j == ny) && (j <= NY1);
    b0[idx] = valid ? T2[((((size_t)(j - 1) * 3 + e) * 2 + part) * NXH + kx) * NZ2 + m] : czero<C>();
  }
  __syncthreads();
  C* res = block_fft<T>(b0, b1, pz, nseq, NZ2, tw, -1);
  const T scale = (T)(1.0 / ((double)g.nx2 * (double)g.nz2));
  const T wsc = (kx == NXH - 1) ? (T)2 * scale : scale;
  const int off = NZ2 - NZ;
  for (int idx = threadIdx.x; idx < NZ * 3 * YB; idx += blockDim.x) {
    const int jj = idx % YB, e = (idx / YB) % 3, kz = idx / (3 * YB);
    const int j = j0 + jj;
    if (j > NY1) continue;
    const bool valid = (j >= 2 && j <= ny) && !(e == 1 && j == ny);
    C out = czero<C>();
    if (valid) {
      const C* A = res + ((jj * 3 + e) * 2 + 0) * NZ2;
      const C* Z = res + ((jj * 3 + e) * 2 + 1) * NZ2;
      C fa, fz;
      if (kz < NZ / 2) { fa = A[kz]; fz = Z[kz]; }
      else if (kz == NZ / 2) {
        fa = cadd(A[NZ / 2], cconj(A[off + NZ / 2]));
        fz = cadd(Z[NZ / 2], cconj(Z[off + NZ / 2]));
      } else { fa = A[off + kz]; fz = Z[off + kz]; }
      const C tz = cscale(wsc, fz);
      out = cadd(cimul<C>((T)gd.kz[kz], tz), cscale(wsc, fa));
    }
    vel[((size_t)(kx * NZ + kz) * 3 + e) * NY1 + (j - 1)] = out;
  }
}

// --------------------------------------------------------------------------
// check_cfl + dt adaptation (PFC/pass1.f90:202-250, 106-124): one block.
template <bool LIN>
__device__ __forceinline__ void k_cfl_finalize_body(const uint3 bid, const unsigned long long* __restrict__ cflbits,
                                                    Geom g, GridDev gd, DevScalars* sc, double* cfl, double lx,
                                                    double lz, int dt_flag, double cfl_max_param, int step) {
  __shared__ double smax[256];
  const int ny = g.ny;
  const double dt = sc->dt;
  double m = 0;
  int bad = 0;
  for (int k = 2 + threadIdx.x; k <= ny; k += blockDim.x) {
    double ma = __longlong_as_double((long long)cflbits[(size_t)(k - 1) * 3 + 0]);
    double mb = __longlong_as_double((long long)cflbits[(size_t)(k - 1) * 3 + 1]);
    double mc = __longlong_as_double((long long)cflbits[(size_t)(k - 1) * 3 + 2]);
    if (LIN) {
      const double* B = gd.baseflow;
      ma = fmax(ma, fabs(B[k - 1] + B[k]));
      mb = fmax(mb, fabs(B[(ny + 1) + k - 1]));
      mc = fmax(mc, fabs(B[2 * (ny + 1) + k - 1] + B[2 * (ny + 1) + k]));
    }
    const double hmin = fmin(gd.hn[k - 1], gd.hn[k - 2]);
    const double ta = 0.5 * ma * (double)g.nx / (0.55 * lx);
    const double tb = mb / (1.73 * hmin);
    const double tc = 0.5 * mc * (double)g.nz / (0.55 * lz);
    const double cf = (ta + tb + tc) * dt;
    cfl[k - 1] = cf;
    m = fmax(m, cf);
    if (dt_flag == 1 ? (cf >= 3.0e2) : (cf >= 1.15)) bad = 1;
  }
  smax[threadIdx.x] = m;
  bad = __syncthreads_or(bad);
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double cfl_temp = smax[0];
    sc->cfl_max = cfl_temp;
    if (bad && sc->status == 0) sc->status = dt_flag == 1 ? -5 : -4;
    if (step >= 0 && dt_flag == 1) {
      const double dt_temp = dt * cfl_max_param / cfl_temp;
      const double alt = dt + (dt_temp - dt) * dt / (1.0 + dt);
      sc->dt = fmin(dt_temp, alt);
    }
  }
}

template <bool LIN>
__global__ void k_cfl_finalize(const unsigned long long* __restrict__ cflbits, Geom g, GridDev gd, DevScalars* sc,
                               double* cfl, double lx, double lz, int dt_flag, double cfl_max_param, int step) {
  k_cfl_finalize_body<LIN>(blockIdx, cflbits, g, gd, sc, cfl, lx, lz, dt_flag, cfl_max_param, step);
}

}  // namespace cfd
