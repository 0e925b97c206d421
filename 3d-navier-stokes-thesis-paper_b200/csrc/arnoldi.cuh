// arnoldi.cuh -- the device side of compute_time_deriv (PFC/arnoldi.f90:485-567),
// the propagator matvec w = Phi_T v of the Arnoldi stability solver:
//   k_absmax        : max |v| over the input vector (for the eps scaling)
//   k_arnoldi_scale : per (component, plane) weight of the transformed
//                     vector, scale/sqrt(dyh or dy) going in and
//                     sqrt(dyh or dy)/scale coming out
//   k_mean_widen    : the FP64 copy of the mean column in mixed precision
//   k_arnoldi_reset : p_grad = t_total = 0 on the device
#pragma once
#include "cfd_common.cuh"
#include "pass1.cuh"

namespace cfd {

__global__ void k_absmax(const double* __restrict__ x, size_t n, unsigned long long* __restrict__ bits) {
  double m = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = fmax(m, fabs(x[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(bits, (unsigned long long)__double_as_longlong(m));
}

// vel[(w*3 + q)*n1 + j] *= s(q, j); scale = eps / max|v|
template <typename T>
__global__ void k_arnoldi_scale(cplx_t<T>* __restrict__ vel, Geom g, GridDev gd,
                                const unsigned long long* __restrict__ maxbits, double eps, int out) {
  const int n1 = g.ny1;
  const size_t n = (size_t)g.nw * 3 * n1;
  const double scale = eps / __longlong_as_double((long long)*maxbits);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(i % n1), q = (int)((i / n1) % 3);
    const double wgt = (q == 1) ? gd.dy[j] : gd.dyh[j];
    double s;
    if (!out) s = (wgt != 0.0) ? scale / sqrt(wgt) : 0.0;
    else s = sqrt(wgt) / scale;
    const cplx_t<T> v = vel[i];
    vel[i] = mk<cplx_t<T>>((T)(s * (double)v.x), (T)(s * (double)v.y));
  }
}

template <typename T>
__global__ void k_mean_widen(const cplx_t<T>* __restrict__ vel, double2* __restrict__ m64, int n1) {
  for (int i = threadIdx.x; i < 3 * n1; i += blockDim.x) {
    const cplx_t<T> v = vel[i];
    m64[i] = make_double2((double)v.x, (double)v.y);
  }
}

__global__ void k_arnoldi_reset(DevScalars* sc) {
  sc->p_grad = 0.0;
  sc->t_total = 0.0;
}

}  // namespace cfd
