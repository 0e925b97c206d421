// les.cuh -- the LES mode's subgrid stresses on the physical planes of the
// nonlinear step (the reference's subgrid = 1 runs, PFC/main_mpi.f90:74-78,
// whose model modules are not in the reference).
//
// At every interior yh plane k (2..ny) and point (z, x) of the dealiased grid:
// the resolved velocity gradient G_ij = du_i/dx_j -- x and z by central
// differences on the dealiased grid, du/dy and dw/dy by the central difference
// over yh(k-1), yh(k+1), dv/dy = dh(k) (v(k) - v(k-1)), v at yh(k) the mean of
// its two y planes -- and from it
//   model 1, eddy viscosity (Smagorinsky with van Driest damping):
//     tau = -2 nu_t S^d, nu_t = (Cs Delta (1 - exp(-y+/A+)))^2 |S|,
//     Delta = (dx dy dz)^(1/3) of the LES grid, |S| = sqrt(2 S:S),
//     y+ = (1 - |yh|) u_tau Re, u_tau^2 = mean |dU/dy| at the walls / Re;
//   model 2, the learned closure: the network's stresses from the 10
//     features (G and the wall distance 1 - |yh|, mirrored into the lower
//     half-channel: components with one y index change sign for yh > 0),
//     kept where they are realizable (non-negative diagonal, Schwarz
//     inequalities, non-negative determinant) and their backscatter -tau:S
//     is not below -beta times the eddy viscosity's dissipation; the eddy
//     viscosity elsewhere.
// Stresses are written to S[pl][6][nz2][nx2] (pl = k - 1; components 11, 22,
// 33, 12, 13, 23), which the flux kernel adds to the momentum fluxes.
#pragma once
#include "cfd_common.cuh"
#include "pass1.cuh"

namespace cfd {

struct LesDev {
  int model;                 // 1 eddy viscosity, 2 learned closure with eddy-viscosity fallback
  double cs, aplus, beta;    // Smagorinsky constant, van Driest A+, admitted backscatter fraction
  double dx, dz;             // LES grid spacing lx/nx, lz/nz
  double hx, hz;             // dealiased grid spacing lx/nx2, lz/nz2
  double re;
  float in_shift[10], in_scale[10], out_shift[6], out_scale[6];
  double in_iscale[10];      // 1 / in_scale
};

// gradient of the resolved velocity at (plane k, z, x): G[3*i + j] = du_i/dx_j
template <typename T>
__device__ __forceinline__ void les_gradient(const T* __restrict__ P, const Geom& g, const GridDev& gd,
                                             const LesDev& les, int k, int z, int x, double G[9]) {
  const int N = g.nx2, NZ2 = g.nz2;
  const size_t cs = (size_t)NZ2 * N, ps = 3 * cs;
  const T* Pm = P + (size_t)(k - 2) * ps;
  const T* P0 = Pm + ps;
  const T* Pp = P0 + ps;
  const int xm = x == 0 ? N - 1 : x - 1, xp = x == N - 1 ? 0 : x + 1;
  const int zm = z == 0 ? NZ2 - 1 : z - 1, zp = z == NZ2 - 1 ? 0 : z + 1;
  auto at = [&](const T* b, int c, int zz, int xx) { return (double)b[c * cs + (size_t)zz * N + xx]; };
  const double ihx = 0.5 / les.hx, ihz = 0.5 / les.hz;
  const double idy = 1.0 / (gd.yh[k] - gd.yh[k - 2]), dh = gd.dh[k - 1];
  auto vc = [&](int zz, int xx) { return 0.5 * (at(Pm, 1, zz, xx) + at(P0, 1, zz, xx)); };
  G[0] = (at(P0, 0, z, xp) - at(P0, 0, z, xm)) * ihx;
  G[1] = (at(Pp, 0, z, x) - at(Pm, 0, z, x)) * idy;
  G[2] = (at(P0, 0, zp, x) - at(P0, 0, zm, x)) * ihz;
  G[3] = (vc(z, xp) - vc(z, xm)) * ihx;
  G[4] = (at(P0, 1, z, x) - at(Pm, 1, z, x)) * dh;
  G[5] = (vc(zp, x) - vc(zm, x)) * ihz;
  G[6] = (at(P0, 2, z, xp) - at(P0, 2, z, xm)) * ihx;
  G[7] = (at(Pp, 2, z, x) - at(Pm, 2, z, x)) * idy;
  G[8] = (at(P0, 2, zp, x) - at(P0, 2, zm, x)) * ihz;
}

// the eddy viscosity's length of plane k, Cs Delta (1 - exp(-y+/A+)): one
// value per plane, computed once per block (the caller's threads share k)
__device__ __forceinline__ double les_nut_length(const GridDev& gd, const LesDev& les,
                                                 const double* __restrict__ d_um_dy, int ny, int k) {
  const double dy = gd.y[k - 1] - gd.y[k - 2];
  const double delta = cbrt(les.dx * dy * les.dz);
  const double utau = sqrt(0.5 * (fabs(d_um_dy[0]) + fabs(d_um_dy[ny - 1])) / les.re);
  const double yplus = (1.0 - fabs(gd.yh[k - 1])) * utau * les.re;
  return les.cs * delta * (1.0 - exp(-yplus / les.aplus));
}

// the length above shared by a block: thread 0 computes it
__device__ __forceinline__ double les_block_length(const GridDev& gd, const LesDev& les,
                                                   const double* __restrict__ d_um_dy, int ny, int k) {
  __shared__ double len;
  if (threadIdx.x == 0) len = les_nut_length(gd, les, d_um_dy, ny, k);
  __syncthreads();
  return len;
}

// trace-free strain rate (11, 22, 33, 12, 13, 23) and the eddy viscosity
// with the plane's length f
__device__ __forceinline__ double les_strain_nut(const double G[9], double f, double Sd[6]) {
  const double tr = (G[0] + G[4] + G[8]) / 3.0;
  Sd[0] = G[0] - tr;
  Sd[1] = G[4] - tr;
  Sd[2] = G[8] - tr;
  Sd[3] = 0.5 * (G[1] + G[3]);
  Sd[4] = 0.5 * (G[2] + G[6]);
  Sd[5] = 0.5 * (G[5] + G[7]);
  const double ss = Sd[0] * Sd[0] + Sd[1] * Sd[1] + Sd[2] * Sd[2] + 2.0 * (Sd[3] * Sd[3] + Sd[4] * Sd[4] + Sd[5] * Sd[5]);
  const double smag = sqrt(2.0 * ss);
  return f * f * smag;
}

// model 1 stresses into S and, for model 2, the network's input features
// F[(k - 2) * nz2 * nx2 + z * nx2 + x][10] (normalised, FP32).  Grid
// (nx2/128 rounded up, nz2, ny - 1), block 128.
template <typename T>
__global__ void __launch_bounds__(128) k_les_sgs(const T* __restrict__ P, T* __restrict__ S, float* __restrict__ F,
                                                 Geom g, GridDev gd, LesDev les, const double* __restrict__ d_um_dy) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y, k = 2 + blockIdx.z;
  const double len = les_block_length(gd, les, d_um_dy, g.ny, k);
  if (x >= g.nx2) return;
  double G[9], Sd[6];
  les_gradient<T>(P, g, gd, les, k, z, x, G);
  const double nut = les_strain_nut(G, len, Sd);
  const size_t cs = (size_t)g.nz2 * g.nx2, o = (size_t)(k - 1) * 6 * cs + (size_t)z * g.nx2 + x;
#pragma unroll
  for (int c = 0; c < 6; ++c) S[o + c * cs] = (T)(-2.0 * nut * Sd[c]);
  if (les.model == 2) {
    // mirrored into the lower half: components with one y index flip
    const double sgn = gd.yh[k - 1] > 0.0 ? -1.0 : 1.0;
    const double f[10] = {G[0], sgn * G[1], G[2], sgn * G[3], G[4], sgn * G[5], G[6], sgn * G[7], G[8],
                          1.0 - fabs(gd.yh[k - 1])};
    float* out = F + (((size_t)(k - 2) * g.nz2 + z) * g.nx2 + x) * 10;
#pragma unroll
    for (int i = 0; i < 10; ++i) out[i] = (float)((f[i] - les.in_shift[i]) * les.in_iscale[i]);
  }
}

// model 2 at one point: the network's (normalised) stresses y[6] where they
// pass the checks, the eddy viscosity's (already in S) elsewhere; f[10]: the
// point's normalised features, len: its plane's eddy-viscosity length, o:
// the point's offset in S (components cs apart).  The gradient comes back
// from the features (the normalisation and the mirroring undone), not from
// the planes.  Returns whether the point falls back.
template <typename T>
__device__ __forceinline__ bool les_blend_point(const float* f, const float* y, double len, const GridDev& gd,
                                                const LesDev& les, int k, T* __restrict__ S, size_t o, size_t cs) {
  const double sgn = gd.yh[k - 1] > 0.0 ? -1.0 : 1.0;
  double G[9], Sd[6];
#pragma unroll
  for (int i = 0; i < 9; ++i) G[i] = (double)f[i] * les.in_scale[i] + les.in_shift[i];
  G[1] *= sgn;
  G[3] *= sgn;
  G[5] *= sgn;
  G[7] *= sgn;
  const double nut = les_strain_nut(G, len, Sd);
  double t[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) t[c] = les.out_shift[c] + les.out_scale[c] * (double)y[c];
  if (gd.yh[k - 1] > 0.0) {   // back from the mirrored frame: 12 and 23 flip
    t[3] = -t[3];
    t[5] = -t[5];
  }
  bool ok = true;
#pragma unroll
  for (int c = 0; c < 6; ++c) ok = ok && isfinite(t[c]);
  // realizability of the stress tensor (positive semi-definite)
  ok = ok && t[0] >= 0.0 && t[1] >= 0.0 && t[2] >= 0.0 && t[3] * t[3] <= t[0] * t[1] &&
       t[4] * t[4] <= t[0] * t[2] && t[5] * t[5] <= t[1] * t[2];
  const double det = t[0] * (t[1] * t[2] - t[5] * t[5]) - t[3] * (t[3] * t[2] - t[5] * t[4]) +
                     t[4] * (t[3] * t[5] - t[1] * t[4]);
  ok = ok && det >= 0.0;
  // backscatter: the transfer -tau:S against the eddy viscosity's
  const double eps_nn = -(t[0] * Sd[0] + t[1] * Sd[1] + t[2] * Sd[2] + 2.0 * (t[3] * Sd[3] + t[4] * Sd[4] + t[5] * Sd[5]));
  const double eps_ev = 2.0 * nut *
                        (Sd[0] * Sd[0] + Sd[1] * Sd[1] + Sd[2] * Sd[2] + 2.0 * (Sd[3] * Sd[3] + Sd[4] * Sd[4] + Sd[5] * Sd[5]));
  ok = ok && eps_nn >= -les.beta * eps_ev;
  if (ok) {
#pragma unroll
    for (int c = 0; c < 6; ++c) S[o + c * cs] = (T)t[c];
  }
  return !ok;
}

// the eddy-viscosity length of every interior plane: len[k] for k = 2 .. ny
// (one block)
static __global__ void k_les_lengths(double* __restrict__ len, GridDev gd, LesDev les,
                                     const double* __restrict__ d_um_dy, int ny) {
  for (int k = 2 + threadIdx.x; k <= ny; k += blockDim.x) len[k] = les_nut_length(gd, les, d_um_dy, ny, k);
}

// the blend of the points of the network's outputs, run by the output layer
// of the network's forward kernel (mlp_les.h): the outputs never go to memory
template <typename T>
struct LesBlend {
  T* S;                       // S[pl][6][nz2][nx2]
  const float* F;             // features F[pt][10]
  const double* len;          // len[k], k_les_lengths
  GridDev gd;
  LesDev les;
  int nx2, nz2;
  unsigned long long* nfall;
  // point pt = (k - 2) nz2 nx2 + z nx2 + x with its network outputs y[6];
  // every lane of the warp calls it (valid false past the last point)
  __device__ __forceinline__ void operator()(long long pt, bool valid, const float* y) const {
    bool fall = false;
    if (valid) {
      const long long plane = (long long)nz2 * nx2;
      const int k = 2 + (int)(pt / plane);
      const long long rem = pt - (long long)(k - 2) * plane;
      const size_t cs = (size_t)plane, o = (size_t)(k - 1) * 6 * cs + (size_t)rem;
      float f[10];
#pragma unroll
      for (int i = 0; i < 10; ++i) f[i] = __ldg(F + pt * 10 + i);
      fall = les_blend_point<T>(f, y, len[k], gd, les, k, S, o, cs);
    }
    const unsigned m = __ballot_sync(0xffffffffu, fall);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(nfall, (unsigned long long)__popc(m));
  }
};

}  // namespace cfd
