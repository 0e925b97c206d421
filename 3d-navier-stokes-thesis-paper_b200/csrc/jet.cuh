// jet.cuh -- crossflow wall forcing cbc(:,:,2) on the device: jet_profile
// (PFC/pass2.f90:423-673) for a closed channel (bl_grid = 0).
//   k_jet_walk    : end-of-substep time and the random walk of the Freund
//                   forcing parameters (:454-477), RANDOM_NUMBER replaced by
//                   the counter RNG: draw n of call k is u01(seed, k, 0, n, 7)
//   k_jet_field   : physical planes on the nx x nz grid: the suction profile
//                   (define_suction_profile, :553-609) and the jet outflow of
//                   each forced wall (define_jet_profile, :611-656, or the
//                   Gaussian spanwise slot)
//   k_jet_combine : after the small forward transforms: filter_cosine passes
//                   (:658-671), top-wall sign, suction balance (:493-537)
#pragma once
#include <cstdint>

#include "cfd_common.cuh"
#include "pass1.cuh"
#include "pass2.cuh"

namespace cfd {

struct JetParams {
  int mode;                        // 0 off, 1 tanh jet, 2 Gaussian slot
  double xjet[2], zjet[2], jetmag[2], forcing[2], for_freq[2];
  double jet_diam, width, freq, frac_xbuff;
  int filter;
  unsigned long long seed;
};

struct JetState {
  double jf[24], inc[24];   // (3,2,4) parameters and increments
  double time, incr;        // of the current call
  long long calls;
};

__device__ __forceinline__ uint64_t jet_smix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
// the counter RNG shared with the host initial-field generator
__device__ __forceinline__ double jet_u01(uint64_t seed, long long x, int z, int j, int col) {
  const uint64_t ctr = ((((uint64_t)x * 65536u + (uint64_t)z) * 65536u + (uint64_t)j) * 8u) + (uint64_t)col;
  const uint64_t h = jet_smix(seed ^ jet_smix(ctr));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

// one warp.  use_sc: time = t_total + dt*sum(rkc(1:rk)+rkd(1:rk)),
// incr = dt*(rkc(rk)+rkd(rk)) from the device scalars (PFC/pass2.f90:37-38);
// otherwise the given time/incr.
__device__ __forceinline__ void k_jet_walk_body(const uint3 bid, JetState* __restrict__ st, JetParams jp,
                                                const DevScalars* __restrict__ sc, RkTab rkt, int rk, double time,
                                                double incr, int use_sc) {
  const int n = threadIdx.x;
  if (use_sc) {
    double s = 0.0;
    for (int r = 1; r <= rk; ++r) s += rkt.Cc(r) + rkt.D(r);
    time = sc->t_total + sc->dt * s;
    incr = sc->dt * (rkt.Cc(rk) + rkt.D(rk));
  }
  const long long k = st->calls;
  __syncwarp();
  if (n == 0) { st->time = time; st->incr = incr; st->calls = k + 1; }
  if (jp.seed == 0 || n >= 24) return;
  const double r = jet_u01(jp.seed, k, 0, n, 7);
  double inc = st->inc[n] * ((r - 0.05) >= 0.0 ? 1.0 : -1.0);   // SIGN(1, r - 0.05)
  double f = st->jf[n] + incr * inc;
  const int kk = n / 6;   // (i,j,k): n = i + 3 j + 6 k
  if (kk == 0) {
    if (f <= 0.01) { f = 0.01; inc = fabs(inc); }
    else if (f >= 0.07) { f = 0.07; inc = -fabs(inc); }
  } else if (kk == 1) {
    if (f <= 0.1) { f = 0.1; inc = fabs(inc); }
    else if (f >= 0.7) { f = 0.7; inc = -fabs(inc); }
  }
  st->jf[n] = f;
  st->inc[n] = inc;
}

__global__ void k_jet_walk(JetState* __restrict__ st, JetParams jp, const DevScalars* __restrict__ sc, RkTab rkt,
                           int rk, double time, double incr, int use_sc) {
  k_jet_walk_body(blockIdx, st, jp, sc, rkt, rk, time, incr, use_sc);
}

// |(a, b)| of a default-real complex: both parts rounded to single, the
// modulus formed in double and rounded to single
__device__ __forceinline__ double abs_cmplx_single(double a, double b) {
  const double af = (double)(float)a, bf = (double)(float)b;
  return (double)(float)sqrt(af * af + bf * bf);
}

// grid (nz, 3), block 128: planes 0 suction, 1 bottom jet, 2 top jet;
// phys[p][z][x] on the nx x nz grid
template <typename T>
__device__ __forceinline__ void k_jet_field_body(const uint3 bid, T* __restrict__ phys, JetParams jp,
                                                 const JetState* __restrict__ st, int nx, int nz, double lx,
                                                 double lz) {
  const int z = bid.x, p = bid.y;
  const double pi = 3.14159265358979323846;
  const double time = st->time;
  const double zc = (double)z * lz / (double)nz;
  for (int x = threadIdx.x; x < nx; x += blockDim.x) {
    const double xc = (double)x * lx / (double)nx;
    double v = 0.0;
    if (p == 0) {
      const double frac_suct = 0.5 * jp.frac_xbuff, suct_start = 1.0 - jp.frac_xbuff;
      const double suct_rise = 0.25 * frac_suct, suct_fall = 0.25 * frac_suct;
      const double xstart = lx * suct_start, xrise = xstart + lx * suct_rise;
      const double xfall = xstart + lx * frac_suct - lx * suct_fall, xend = xstart + lx * frac_suct;
      if (xc > xstart && xc < xend) {
        if (xc < xrise) {
          const double x2 = (xc - xstart) / (xrise - xstart);
          v = 1.0 / (1.0 + exp(1.0 / x2 + 1.0 / (x2 - 1.0)));
        } else if (xc > xfall) {
          const double x2 = (xend - xc) / (xend - xfall);
          v = 1.0 / (1.0 + exp(1.0 / x2 + 1.0 / (x2 - 1.0)));
        } else {
          v = 1.0;
        }
      }
    } else {
      const int w = p - 1;
      const double jm = jp.jetmag[w];
      if (jp.mode == 1 && jm != 0.0) {
        const double v_ampl = jm * (1.0 + jp.forcing[w] * sin(2.0 * pi * time * jp.for_freq[w] * jm / jp.jet_diam));
        const double xd1 = xc - jp.xjet[w], xd2 = xc - (lx + jp.xjet[w]);
        const double zd1 = zc - jp.zjet[w], zd2 = zc - (lz + jp.zjet[w]);
        const double r1 = abs_cmplx_single(xd1, zd1) * 2.0 / jp.jet_diam;
        const double r2 = abs_cmplx_single(xd2, zd1) * 2.0 / jp.jet_diam;
        const double r3 = abs_cmplx_single(xd1, zd2) * 2.0 / jp.jet_diam;
        const double r4 = abs_cmplx_single(xd2, zd2) * 2.0 / jp.jet_diam;
        const double r = fmin(fmin(r1, r2), fmin(r3, r4));
        if (r == 0.0) {
          v = v_ampl;
        } else {
          const double phi = atan2(zd1, xd1);
          double s = 0.0;
#pragma unroll
          for (int i = 0; i < 6; ++i) {
            const double fw = (double)(i % 3);
            s += st->jf[i] * cos(st->jf[6 + i] * jm * time / jp.jet_diam + st->jf[12 + i]) *
                 cos(fw * phi + st->jf[18 + i]);
          }
          const double bjet = 5.0 + s;
          v = v_ampl * 0.5 * (1.0 - tanh(bjet * (r - 1.0 / r)));
        }
      } else if (jp.mode == 2 && jm != 0.0) {
        const double a = jm * 0.5 * (1.0 + sin(2.0 * pi * jp.freq * time));
        double d = fabs(xc - jp.xjet[w]);
        if (lx - d < d) d = lx - d;
        v = a * exp(-(d / jp.width) * (d / jp.width));
      }
    }
    phys[((size_t)p * nz + z) * nx + x] = (T)v;
  }
}

template <typename T>
__global__ void k_jet_field(T* __restrict__ phys, JetParams jp, const JetState* __restrict__ st, int nx, int nz,
                            double lx, double lz) {
  k_jet_field_body<T>(blockIdx, phys, jp, st, nx, nz, lx, lz);
}

// spec[p][kx][kz] (p = 0 suction, 1 bottom, 2 top) -> cbc(:,:,2) of the
// forced walls, the other wall slots zeroed
template <typename T>
__device__ __forceinline__ void k_jet_combine_body(const uint3 bid, const cplx_t<T>* __restrict__ spec,
                                                   cplx_t<T>* __restrict__ cbc, JetParams jp, GridDev gd, int nx,
                                                   int nz, int nxh, double lx, double lz) {
  using C = cplx_t<T>;
  const int nw = nz * nxh;
  const int w = bid.x * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  const int kx = w / nz, kz = w % nz;
  const double pi = 3.14159265358979323846;
  const double fx = 1.0 + cos(pi * gd.kx[kx] / ((double)(nx / 2) * 2.0 * pi / lx));
  const double fz = 1.0 + cos(pi * gd.kz[kz] / ((double)(nz / 2) * 2.0 * pi / lz));
  auto filt = [&](C v) {
    double re = (double)v.x, im = (double)v.y;
    for (int n = 0; n < jp.filter; ++n) {
      re = re * 0.5 * fx * 0.5 * fz;
      im = im * 0.5 * fx * 0.5 * fz;
    }
    return mk<C>((T)re, (T)im);
  };
  // the (0,0) coefficients carry the filter factor 1
  const C cs = filt(spec[w]);
  const double sum_suction = (double)spec[0].x;
  for (int wall = 0; wall < 2; ++wall) {
    C out = czero<C>();
    if (jp.mode != 0 && jp.jetmag[wall] != 0.0) {
      const double sg = wall == 1 ? -1.0 : 1.0;
      const C cj = filt(spec[(size_t)(1 + wall) * nw + w]);
      const double sum = sg * (double)spec[(size_t)(1 + wall) * nw].x;
      const double q = sum / sum_suction;
      out = mk<C>((T)(sg * (double)cj.x - q * (double)cs.x), (T)(sg * (double)cj.y - q * (double)cs.y));
    }
    // cbc layout [bot, top][comp][kx][kz]: component 2 (v) is index 1
    cbc[((size_t)wall * 3 + 1) * nw + w] = out;
  }
}

template <typename T>
__global__ void k_jet_combine(const cplx_t<T>* __restrict__ spec, cplx_t<T>* __restrict__ cbc, JetParams jp,
                              GridDev gd, int nx, int nz, int nxh, double lx, double lz) {
  k_jet_combine_body<T>(blockIdx, spec, cbc, jp, gd, nx, nz, nxh, lx, lz);
}

// ---------------------------------------------------------------------------
// init_buffer (PFC/init_jet_buffer.f90:358-483): the fringe profile on the
// nx x nz grid.  Each direction's band rises and falls with
// 1/(1+exp(1/t + 1/(t-1))) (define_fringe_region, :453-482); where the x and
// z bands overlap the two ramps combine through sqrt(tx^2 + tz^2).
struct FringeParams {
  int xfringe, zfringe;
  double frac_xbuff, buff_xrise, buff_xfall, frac_zbuff;
};

__device__ __forceinline__ void fringe_region(double t, double ts, double tr, double tf, double te, double& f,
                                              double& f2) {
  f = 0.0;
  f2 = 0.0;
  if (t > ts) {
    if (t < tr) {
      const double t2 = (t - ts) / (tr - ts);
      f = 1.0 / (1.0 + exp(1.0 / t2 + 1.0 / (t2 - 1.0)));
      f2 = t2;
    } else if (t > tf && t < te) {
      const double t2 = (te - t) / (te - tf);
      f = 1.0 / (1.0 + exp(1.0 / t2 + 1.0 / (t2 - 1.0)));
      f2 = t2;
    } else if (t >= te) {
      f = 0.0;
    } else {
      f = 1.0;
    }
  }
}

template <typename T>
__global__ void k_fringe_profile(T* __restrict__ out, FringeParams fp, int nx, int nz, double lx, double lz) {
  const int z = blockIdx.x;
  const double tz = (double)z * lz / (double)nz;
  double fz = 0.0, fz2 = 0.0;
  if (fp.zfringe == 1) {
    double fa, fa2, fb, fb2;
    fringe_region(tz, -1.0, -1.0, 0.0, fp.frac_zbuff * lz, fa, fa2);
    fringe_region(tz, lz - fp.frac_zbuff * lz, lz, lz + 1.0, lz + 1.0, fb, fb2);
    fz = fa + fb;
    fz2 = fa2 + fb2;
  }
  for (int x = threadIdx.x; x < nx; x += blockDim.x) {
    const double tx = (double)x * lx / (double)nx;
    double fx = 0.0, fx2 = 0.0;
    if (fp.xfringe == 1) {
      const double xs = lx * (1.0 - fp.frac_xbuff);
      fringe_region(tx, xs, xs + lx * fp.buff_xrise, lx - lx * fp.buff_xfall, lx, fx, fx2);
    }
    double v;
    if (fx < 1.0 && fz < 1.0 && fx * fz > 0.0) {
      const double t = sqrt(fx2 * fx2 + fz2 * fz2);
      v = (t < 1.0) ? 1.0 / (1.0 + exp(1.0 / t + 1.0 / (t - 1.0))) : 1.0;
    } else {
      v = fmax(fx, fz);
    }
    out[(size_t)z * nx + x] = (T)v;
  }
}

template <typename T>
__global__ void k_scale_real(const T* __restrict__ in, T* __restrict__ out, size_t n, double s) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (T)(s * (double)in[i]);
}

}  // namespace cfd
