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

}  // namespace cfd
