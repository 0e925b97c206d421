// io.cuh -- device side of the restart file and the VTK snapshot
// (PFC/read_write.f90:21-292, 296-500): layout conversions between the
// device state and the file orders, so that the host only streams bytes.
//   k_restart_out : data1 -> records kx = 0..nx/2: (nz, ny+1, 3) complex FP64
//   k_restart_in  : the inverse
//   k_vtk_planes  : the velocity on the yh planes (v interpolated to yh as
//                   output_hdf_dfsd does with yskip = 1), spectral planes
//                   [c*(ny+1) + plane][kx][kz] for the small transforms
//   k_vtk_pack    : physical planes -> big-endian float32 (u,v,w) triplets,
//                   x fastest, then plane, then z
#pragma once
#include <cstdint>

#include "cfd_common.cuh"
#include "pass1.cuh"

namespace cfd {

template <typename T>
__global__ void k_restart_out(const cplx_t<T>* __restrict__ vel, const double2* __restrict__ mvel64,
                              double2* __restrict__ dst, Geom g) {
  const int n1 = g.ny1, NZ = g.nz;
  const size_t n = (size_t)g.nw * 3 * n1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(i % n1), c = (int)((i / n1) % 3);
    const size_t w = i / ((size_t)3 * n1);
    const int kx = (int)(w / NZ), kz = (int)(w % NZ);
    double2 v;
    if (mvel64 && w == 0) v = mvel64[c * n1 + j];
    else { const cplx_t<T> s = vel[i]; v = make_double2((double)s.x, (double)s.y); }
    dst[(size_t)kx * NZ * n1 * 3 + kz + (size_t)NZ * (j + (size_t)n1 * c)] = v;
  }
}

template <typename T>
__global__ void k_restart_in(const double2* __restrict__ src, cplx_t<T>* __restrict__ vel,
                             double2* __restrict__ mvel64, Geom g) {
  const int n1 = g.ny1, NZ = g.nz;
  const size_t n = (size_t)g.nw * 3 * n1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(i % n1), c = (int)((i / n1) % 3);
    const size_t w = i / ((size_t)3 * n1);
    const int kx = (int)(w / NZ), kz = (int)(w % NZ);
    const double2 v = src[(size_t)kx * NZ * n1 * 3 + kz + (size_t)NZ * (j + (size_t)n1 * c)];
    vel[i] = mk<cplx_t<T>>((T)v.x, (T)v.y);
    if (mvel64 && w == 0) mvel64[c * n1 + j] = v;
  }
}

template <typename T>
__global__ void k_vtk_planes(const cplx_t<T>* __restrict__ vel, const double2* __restrict__ mvel64,
                             cplx_t<T>* __restrict__ out, Geom g) {
  using C = cplx_t<T>;
  const int n1 = g.ny1, ny = g.ny;
  const size_t nw = (size_t)g.nw, n = nw * 3 * n1;
  auto at = [&](size_t w, int c, int j) -> double2 {
    if (mvel64 && w == 0) return mvel64[c * n1 + j];
    const C s = vel[(w * 3 + c) * n1 + j];
    return make_double2((double)s.x, (double)s.y);
  };
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t w = i % nw;
    const int p = (int)(i / nw), c = p / n1, pl = p % n1;
    double2 v;
    if (c != 1) v = at(w, c, pl);
    else if (pl == 0) v = at(w, 1, 0);
    else if (pl == ny) v = at(w, 1, ny - 1);
    else {
      const double2 a = at(w, 1, pl - 1), b = at(w, 1, pl);
      v = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
    }
    out[i] = mk<C>((T)v.x, (T)v.y);
  }
}

template <typename T>
__global__ void k_vtk_pack(const T* __restrict__ phys, uint32_t* __restrict__ out, int nx, int n1, int nz) {
  const size_t n = (size_t)nx * n1 * nz * 3;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % 3);
    const size_t q = i / 3;
    const int x = (int)(q % nx), pl = (int)((q / nx) % n1), z = (int)(q / ((size_t)nx * n1));
    const float v = (float)phys[(((size_t)c * n1 + pl) * nz + z) * nx + x];
    const uint32_t u = __float_as_uint(v);
    out[i] = __byte_perm(u, 0, 0x0123);   // big-endian
  }
}

// ---------------------------------------------------------------------------
// Post-processing on the (x, yh, z) output grid (ParaView-Code/
// DiscriminantFilter.cpd, PFC/stats.f90:120-251):
//   k_grad_spec : spectral planes of A_ij = du_i/dx_j for planes p0..p0+np-1:
//                 ikx u_i, ikz u_i, and the 3-point Lagrange y-derivative on
//                 yh (weights wy, nodes sy) -- planes [(pl*3 + i)*3 + j]
//   k_stats_vel : per plane sums of (u_i - m_i)^2,3,4 and (u_i - m_i)(v - m_v),
//                 the mean m_i being the (0,0) coefficient of the plane
//   k_derived   : vorticity, Q = -tr(A^2)/2 and the discriminant
//                 D = (6 (tr A^3)^2 - (tr A^2)^3)/8 per point (packed
//                 big-endian when `out` is given) and the per-plane central
//                 moments of the vorticity

template <typename T>
__device__ __forceinline__ double2 vel_at_yh(const cplx_t<T>* __restrict__ vel, const double2* __restrict__ mvel64,
                                             size_t w, int c, int pl, int n1, int ny) {
  auto at = [&](int cc, int j) -> double2 {
    if (mvel64 && w == 0) return mvel64[cc * n1 + j];
    const cplx_t<T> s = vel[(w * 3 + cc) * n1 + j];
    return make_double2((double)s.x, (double)s.y);
  };
  if (c != 1) return at(c, pl);
  if (pl == 0) return at(1, 0);
  if (pl == ny) return at(1, ny - 1);
  const double2 a = at(1, pl - 1), b = at(1, pl);
  return make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
}

template <typename T>
__global__ void k_grad_spec(const cplx_t<T>* __restrict__ vel, const double2* __restrict__ mvel64,
                            cplx_t<T>* __restrict__ out, Geom g, GridDev gd, const double* __restrict__ wy,
                            const int* __restrict__ sy, int p0, int np) {
  using C = cplx_t<T>;
  const int n1 = g.ny1, ny = g.ny, NZ = g.nz;
  const size_t nw = (size_t)g.nw, n = nw * 3 * np;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t w = i % nw;
    const int r = (int)(i / nw), c = r % 3, pl = p0 + r / 3;
    const double kx = gd.kx[w / NZ], kz = gd.kz[w % NZ];
    const double2 u = vel_at_yh<T>(vel, mvel64, w, c, pl, n1, ny);
    double2 dy = make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double2 v = vel_at_yh<T>(vel, mvel64, w, c, sy[3 * pl + q], n1, ny);
      dy.x += wy[3 * pl + q] * v.x;
      dy.y += wy[3 * pl + q] * v.y;
    }
    C* o = out + ((size_t)(r / 3) * 9 + c * 3) * nw + w;
    o[0] = mk<C>((T)(-kx * u.y), (T)(kx * u.x));   // d/dx
    o[nw] = mk<C>((T)dy.x, (T)dy.y);               // d/dy
    o[2 * nw] = mk<C>((T)(-kz * u.y), (T)(kz * u.x));   // d/dz
  }
}

// grid (nz, n1), block 128: plane `blockIdx.y`, row z; phys [c][plane][z][x],
// spec [c*n1 + plane][kx][kz]; acc[plane*15 + ...] += sums
template <typename T>
__global__ void k_stats_vel(const T* __restrict__ phys, const cplx_t<T>* __restrict__ spec, int nx, int nz,
                            int n1, size_t nw, double* __restrict__ acc) {
  const int z = blockIdx.x, pl = blockIdx.y;
  double m[3], s[15];
#pragma unroll
  for (int c = 0; c < 3; ++c) m[c] = (double)spec[(size_t)(c * n1 + pl) * nw].x;
#pragma unroll
  for (int k = 0; k < 15; ++k) s[k] = 0.0;
  for (int x = threadIdx.x; x < nx; x += blockDim.x) {
    double d[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) d[c] = (double)phys[(((size_t)c * n1 + pl) * nz + z) * nx + x] - m[c];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double d2 = d[c] * d[c];
      s[c] += d2;
      s[3 + c] += d2 * d[c];
      s[6 + c] += d2 * d2;
      s[9 + c] += d[c] * d[1];
    }
  }
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    double v = s[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&acc[pl * 15 + k], v);
  }
  if (threadIdx.x == 0 && z == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) atomicAdd(&acc[pl * 15 + 12 + c], m[c]);
  }
}

// grid (nz, np), block 128: phys [(pl*9 + ij)][z][x] for the chunk's planes,
// spec the matching spectral planes (for the means); out: packed fields of
// npts points (vorticity at 3*npts, Q at 6*npts, D at 7*npts), or null;
// acc[plane*15 + ...]: vorticity sums (^2, ^3, ^4) and means
template <typename T>
__global__ void k_derived(const T* __restrict__ phys, const cplx_t<T>* __restrict__ spec, int nx, int nz, int n1,
                          size_t nw, int p0, uint32_t* __restrict__ out, double* __restrict__ acc) {
  const int z = blockIdx.x, lp = blockIdx.y, pl = p0 + lp;
  const size_t npts = (size_t)nx * n1 * nz, ps = (size_t)nz * nx;
  const T* A = phys + (size_t)lp * 9 * ps + (size_t)z * nx;
  // vorticity means from the (0,0) coefficients: w_x = A21 - A12, w_y = A02 - A20, w_z = A10 - A01
  const cplx_t<T>* S = spec + (size_t)lp * 9 * nw;
  const double mw[3] = {(double)S[7 * nw].x - (double)S[5 * nw].x, (double)S[2 * nw].x - (double)S[6 * nw].x,
                        (double)S[3 * nw].x - (double)S[1 * nw].x};
  double s[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) s[k] = 0.0;
  for (int x = threadIdx.x; x < nx; x += blockDim.x) {
    double a[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = (double)A[k * ps + x];
    const double wv[3] = {a[7] - a[5], a[2] - a[6], a[3] - a[1]};
    const double tr2 = a[0] * a[0] + 2 * a[1] * a[3] + a[4] * a[4] + 2 * a[2] * a[6] + 2 * a[5] * a[7] + a[8] * a[8];
    const double tr3 = a[0] * a[0] * a[0] + a[4] * a[4] * a[4] + 3 * a[0] * (a[1] * a[3] + a[2] * a[6]) +
                       3 * a[1] * (a[3] * a[4] + a[5] * a[6]) + 3 * a[2] * a[3] * a[7] + 3 * a[4] * a[5] * a[7] +
                       3 * a[2] * a[6] * a[8] + 3 * a[5] * a[7] * a[8] + a[8] * a[8] * a[8];
    const double q = -0.5 * tr2;
    const double dsc = 0.125 * (6.0 * tr3 * tr3 - tr2 * tr2 * tr2);
    if (out) {
      const size_t p = ((size_t)z * n1 + pl) * nx + x;
#pragma unroll
      for (int c = 0; c < 3; ++c) out[3 * npts + 3 * p + c] = __byte_perm(__float_as_uint((float)wv[c]), 0, 0x0123);
      out[6 * npts + p] = __byte_perm(__float_as_uint((float)q), 0, 0x0123);
      out[7 * npts + p] = __byte_perm(__float_as_uint((float)dsc), 0, 0x0123);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double d = wv[c] - mw[c], d2 = d * d;
      s[c] += d2;
      s[3 + c] += d2 * d;
      s[6 + c] += d2 * d2;
    }
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    double v = s[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&acc[pl * 15 + k], v);
  }
  if (threadIdx.x == 0 && z == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) atomicAdd(&acc[pl * 15 + 12 + c], mw[c]);
  }
}

}  // namespace cfd
