// planes.cuh -- batched single-plane transforms with the reference's
// conventions, for the non-hot callers of the transforms: boundary feedback
// (PFC/read_write.f90:1465-1532), l2_norm (:1432-1462), the plane API of
// PFC/transform.f90:195-227 and the small (nx x nz) transforms :950-1142.
//
//   k_pz_inv : spectral planes (strided) -> hybrid H[p][kx][zlen]
//              (pad = 1: 3/2 padding with Nyquist split and x-Nyquist halving
//               of xz_fft_complex_to_real_parallel; pad = 0: plain copy)
//   k_px_inv : hybrid -> physical rows phys[p][z][xlen] (FFTW c2r semantics)
//   k_px_fwd : physical rows -> hybrid (r2c, kx < nxh kept)
//   k_pz_fwd : hybrid -> spectral out[p][kx][kz]
//              (fold = 1: Nyquist fold, 1/(nx2 nz2), last-kx doubling of
//               xz_fft_real_to_complex_parallel; fold = 0: 1/(nx nz) only)
#pragma once
#include "cfd_common.cuh"
#include "fft.cuh"

namespace cfd {

struct PlaneIn {   // element (p, c, kx, kz) at base + p*sp + c*sc + kx*skx + kz*skz
  size_t sp, sc, skx, skz;
  int nc;
};

template <typename T>
__global__ void k_pz_inv(const cplx_t<T>* __restrict__ in, PlaneIn L, const int* __restrict__ plist,
                         int np, cplx_t<T>* __restrict__ H, int nxh, int nzin, int zlen,
                         int pad, int halve_last_x, FftPlan pz, const cplx_t<T>* __restrict__ twz) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* b0 = tw + zlen;
  const int nseq = L.nc;
  C* b1 = b0 + nseq * zlen;
  const int kx = blockIdx.x, pi = blockIdx.y;
  const int p = plist ? plist[pi] : pi;
  for (int m = threadIdx.x; m < zlen; m += blockDim.x) tw[m] = twz[m];
  for (int i = threadIdx.x; i < nseq * zlen; i += blockDim.x) b0[i] = czero<C>();
  __syncthreads();
  const T half = (T)0.5;
  const int NZ = nzin;
  for (int idx = threadIdx.x; idx < NZ * nseq; idx += blockDim.x) {
    const int c = idx % nseq, kz = idx / nseq;
    C v = in[p * L.sp + c * L.sc + kx * L.skx + kz * L.skz];
    C* seq = b0 + c * zlen;
    if (pad && zlen > NZ) {
      if (halve_last_x && kx == nxh - 1) v = cscale(half, v);
      if (kz < NZ / 2) seq[kz] = v;
      else if (kz == NZ / 2) {
        seq[NZ / 2] = cscale(half, v);
        seq[zlen - NZ / 2] = cscale(half, cconj(v));
      } else seq[kz + zlen - NZ] = v;
    } else {
      seq[kz] = v;
    }
  }
  __syncthreads();
  C* res = block_fft<T>(b0, b1, pz, nseq, zlen, tw, +1);
  for (int idx = threadIdx.x; idx < nseq * zlen; idx += blockDim.x) {
    const int m = idx % zlen, c = idx / zlen;
    H[(((size_t)pi * nseq + c) * nxh + kx) * zlen + m] = res[idx];
  }
}

// grid (zlen/2, np): two rows per block through one complex FFT.
template <typename T>
__global__ void k_px_inv(const cplx_t<T>* __restrict__ H, T* __restrict__ phys, int nxh, int zlen,
                         int xlen, FftPlan px, const cplx_t<T>* __restrict__ twx) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* b0 = tw + xlen;
  C* b1 = b0 + xlen;
  const int z = 2 * blockIdx.x, p = blockIdx.y;
  for (int m = threadIdx.x; m < xlen; m += blockDim.x) tw[m] = twx[m];
  const int N = xlen, Nh = xlen / 2;
  const bool two = (z + 1 < zlen);
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    const int kk = (k <= Nh) ? k : N - k;
    C x1 = czero<C>(), x2 = czero<C>();
    if (kk < nxh) {
      x1 = H[((size_t)p * nxh + kk) * zlen + z];
      if (two) x2 = H[((size_t)p * nxh + kk) * zlen + z + 1];
    }
    C zz;
    if (k == 0 || k == Nh) zz = mk<C>(x1.x, x2.x);
    else if (k < Nh) zz = mk<C>(x1.x - x2.y, x1.y + x2.x);
    else zz = mk<C>(x1.x + x2.y, -x1.y + x2.x);
    b0[k] = zz;
  }
  __syncthreads();
  C* res = block_fft<T>(b0, b1, px, 1, N, tw, +1);
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    phys[((size_t)p * zlen + z) * xlen + k] = res[k].x;
    if (two) phys[((size_t)p * zlen + z + 1) * xlen + k] = res[k].y;
  }
}

// grid (zlen/2, np)
template <typename T>
__device__ __forceinline__ void k_px_fwd_body(const uint3 bid, const T* __restrict__ phys, cplx_t<T>* __restrict__ H,
                                              int nxh, int zlen, int xlen, FftPlan px,
                                              const cplx_t<T>* __restrict__ twx) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* b0 = tw + xlen;
  C* b1 = b0 + xlen;
  const int z = 2 * bid.x, p = bid.y;
  const bool two = (z + 1 < zlen);
  for (int m = threadIdx.x; m < xlen; m += blockDim.x) tw[m] = twx[m];
  for (int k = threadIdx.x; k < xlen; k += blockDim.x)
    b0[k] = mk<C>(phys[((size_t)p * zlen + z) * xlen + k], two ? phys[((size_t)p * zlen + z + 1) * xlen + k] : (T)0);
  __syncthreads();
  C* res = block_fft<T>(b0, b1, px, 1, xlen, tw, -1);
  const T half = (T)0.5;
  for (int kx = threadIdx.x; kx < nxh; kx += blockDim.x) {
    const int km = (kx == 0) ? 0 : xlen - kx;
    const C zk = res[kx], zm = res[km];
    H[((size_t)p * nxh + kx) * zlen + z] = mk<C>(half * (zk.x + zm.x), half * (zk.y - zm.y));
    if (two) H[((size_t)p * nxh + kx) * zlen + z + 1] = mk<C>(half * (zk.y + zm.y), -half * (zk.x - zm.x));
  }
}

template <typename T>
__global__ void k_px_fwd(const T* __restrict__ phys, cplx_t<T>* __restrict__ H, int nxh, int zlen, int xlen,
                         FftPlan px, const cplx_t<T>* __restrict__ twx) {
  k_px_fwd_body<T>(blockIdx, phys, H, nxh, zlen, xlen, px, twx);
}

// grid (nxh, np); out element (p, kx, kz) at out + p*osp + kx*oskx + kz*oskz
template <typename T>
__device__ __forceinline__ void k_pz_fwd_body(const uint3 bid, const cplx_t<T>* __restrict__ H,
                                              cplx_t<T>* __restrict__ out, size_t osp, size_t oskx, size_t oskz,
                                              int nxh, int zlen, int nzout, int fold, T scale, FftPlan pz,
                                              const cplx_t<T>* __restrict__ twz) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* b0 = tw + zlen;
  C* b1 = b0 + zlen;
  const int kx = bid.x, p = bid.y;
  for (int m = threadIdx.x; m < zlen; m += blockDim.x) {
    tw[m] = twz[m];
    b0[m] = H[((size_t)p * nxh + kx) * zlen + m];
  }
  __syncthreads();
  C* S = block_fft<T>(b0, b1, pz, 1, zlen, tw, -1);
  const int NZ = nzout, off = zlen - NZ;
  const T s = (fold && kx == nxh - 1) ? (T)2 * scale : scale;
  for (int kz = threadIdx.x; kz < NZ; kz += blockDim.x) {
    C v;
    if (!fold) v = S[kz];
    else if (kz < NZ / 2) v = S[kz];
    else if (kz == NZ / 2) v = cadd(S[NZ / 2], cconj(S[off + NZ / 2]));
    else v = S[off + kz];
    out[p * osp + kx * oskx + kz * oskz] = cscale(s, v);
  }
}

template <typename T>
__global__ void k_pz_fwd(const cplx_t<T>* __restrict__ H, cplx_t<T>* __restrict__ out, size_t osp, size_t oskx,
                         size_t oskz, int nxh, int zlen, int nzout, int fold, T scale, FftPlan pz,
                         const cplx_t<T>* __restrict__ twz) {
  k_pz_fwd_body<T>(blockIdx, H, out, osp, oskx, oskz, nxh, zlen, nzout, fold, scale, pz, twz);
}

// Wall-shear feedback law of boundary (PFC/read_write.f90:1483,1498,1514,1527)
// on physical planes: in[0..3] = planes 2, 3, ny, ny-1; out[0] bottom, out[1] top.
template <typename T>
__global__ void k_feedback(const T* __restrict__ in, T* __restrict__ out, size_t np, double dm11,
                           double dm21, double dm31, double dm12, double dm22, double dm32,
                           double gain, double off) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    const double u2 = in[i], u3 = in[np + i], t2 = in[2 * np + i], t3 = in[3 * np + i];
    out[i] = (T)((dm21 * u2 + dm31 * u3 - off) / (gain - dm11));
    out[np + i] = (T)(-(dm22 * t2 + dm12 * t3 + off) / (gain + dm32));
  }
}

// Sum of squares of one physical row pair per block, for l2_norm: plane p of
// component c, shifted by (1 - y^2) for u.  grid (zlen/2, nplanes*3)
template <typename T>
__global__ void k_l2_rows(const cplx_t<T>* __restrict__ H, int nxh, int zlen, int xlen,
                          FftPlan px, const cplx_t<T>* __restrict__ twx,
                          const double* __restrict__ y, int ny, double* __restrict__ acc) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* b0 = tw + xlen;
  C* b1 = b0 + xlen;
  __shared__ double red[32];
  const int z = 2 * blockIdx.x, pc = blockIdx.y;   // pc = plane*3 + comp
  const int plane = pc / 3, comp = pc % 3;
  for (int m = threadIdx.x; m < xlen; m += blockDim.x) tw[m] = twx[m];
  const int N = xlen, Nh = xlen / 2;
  const bool two = (z + 1 < zlen);
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    const int kk = (k <= Nh) ? k : N - k;
    C x1 = czero<C>(), x2 = czero<C>();
    if (kk < nxh) {
      x1 = H[((size_t)pc * nxh + kk) * zlen + z];
      if (two) x2 = H[((size_t)pc * nxh + kk) * zlen + z + 1];
    }
    C zz;
    if (k == 0 || k == Nh) zz = mk<C>(x1.x, x2.x);
    else if (k < Nh) zz = mk<C>(x1.x - x2.y, x1.y + x2.x);
    else zz = mk<C>(x1.x + x2.y, -x1.y + x2.x);
    b0[k] = zz;
  }
  __syncthreads();
  C* res = block_fft<T>(b0, b1, px, 1, N, tw, +1);
  const double sh = (comp == 0 && plane < ny) ? 1.0 - y[plane] * y[plane] : 0.0;
  double s = 0;
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    const double a = (double)res[k].x - sh;
    s += a * a;
    if (two) {
      const double b = (double)res[k].y - sh;
      s += b * b;
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(acc + plane, t);
  }
}

}  // namespace cfd
