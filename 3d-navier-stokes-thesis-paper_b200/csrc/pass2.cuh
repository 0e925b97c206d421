// pass2.cuh -- per-(kx,kz) implicit RK3/Crank-Nicolson substep of
// PFC/pass2.f90:29-352 with the solvers of PFC/solve.f90 and the y-operators
// of PFC/diff_int.f90, one warp per wavenumber.
//
// The wavenumber's y-columns (u, v, w, pressure and the correction) are staged
// in shared memory; lane g owns rows [g*M, g*M+M).  Every tridiagonal system
// (three Helmholtz solves, one pressure solve) is solved by a partition
// method: each lane eliminates inside its M rows (Thomas-like sweeps), the
// 2*32 interface unknowns form a tridiagonal system solved by parallel cyclic
// reduction over warp shuffles, and each lane back-substitutes its interior.
#pragma once
#include "cfd_common.cuh"
#include "pass1.cuh"

namespace cfd {

struct RkTab {   // RK3 constants as the reference widens them (PFC/pass2.f90:14-18)
  double a[4], b[4], c[4], d[4];
  // select by substep without indexing a kernel parameter at run time (which
  // would copy the table to a local stack frame)
  __device__ __forceinline__ static double pick(const double (&v)[4], int k) {
    return k == 1 ? v[1] : (k == 2 ? v[2] : (k == 3 ? v[3] : v[0]));
  }
  __device__ __forceinline__ double A(int k) const { return pick(a, k); }
  __device__ __forceinline__ double B(int k) const { return pick(b, k); }
  __device__ __forceinline__ double Cc(int k) const { return pick(c, k); }
  __device__ __forceinline__ double D(int k) const { return pick(d, k); }
};

// Partition + PCR solve of a tridiagonal system distributed M rows per lane
// across the 32 lanes of a warp.  Row j = lane*M + i:
//   a[i] x_{j-1} + b[i] x_j + c[i] x_{j+1} = f[i].
// Rows past the end must be identity rows (a = c = 0, b = 1).  On return f
// holds the solution.  Requires M >= 2.
template <typename T, int M>
__device__ __forceinline__ void tri_partition_solve(T (&a)[M], T (&b)[M], T (&c)[M],
                                                    cplx_t<T> (&f)[M], int lane) {
  using C = cplx_t<T>;
  T ap[M], cq[M];
  // downward elimination inside the block: rows i>=1 couple to x_0 through ap
  ap[0] = 0;
  if (M > 1) ap[1] = a[1];
#pragma unroll
  for (int i = 2; i < M; ++i) {
    const T r = a[i] / b[i - 1];
    ap[i] = -r * ap[i - 1];
    b[i] = b[i] - r * c[i - 1];
    f[i] = mk<C>(f[i].x - r * f[i - 1].x, f[i].y - r * f[i - 1].y);
  }
  // upward elimination: interior rows couple to x_{M-1} through cq
#pragma unroll
  for (int i = 0; i < M; ++i) cq[i] = 0;
  if (M > 2) cq[M - 2] = c[M - 2];
#pragma unroll
  for (int i = M - 3; i >= 1; --i) {
    const T r = c[i] / b[i + 1];
    ap[i] = ap[i] - r * ap[i + 1];
    cq[i] = -r * cq[i + 1];
    f[i] = mk<C>(f[i].x - r * f[i + 1].x, f[i].y - r * f[i + 1].y);
  }
  // interface rows: slot 0 = block row 0, slot 1 = block row M-1
  T A0 = a[0], B0 = b[0], C0 = c[0];
  C F0 = f[0];
  if (M > 2) {
    const T r = c[0] / b[1];
    B0 = b[0] - r * ap[1];
    C0 = -r * cq[1];
    F0 = mk<C>(f[0].x - r * f[1].x, f[0].y - r * f[1].y);
  }
  T A1 = ap[M - 1], B1 = b[M - 1], C1 = c[M - 1];
  C F1 = f[M - 1];
  // PCR on the 64 interface rows (2*lane + slot)
  const unsigned full = 0xffffffffu;
  // stride 1
  {
    // lower neighbour of slot 0 is lane-1 slot 1; upper of slot 1 is lane+1 slot 0
    T la = __shfl_up_sync(full, A1, 1), lb = __shfl_up_sync(full, B1, 1), lc = __shfl_up_sync(full, C1, 1);
    T lfx = __shfl_up_sync(full, F1.x, 1), lfy = __shfl_up_sync(full, F1.y, 1);
    T ua = __shfl_down_sync(full, A0, 1), ub = __shfl_down_sync(full, B0, 1), uc = __shfl_down_sync(full, C0, 1);
    T ufx = __shfl_down_sync(full, F0.x, 1), ufy = __shfl_down_sync(full, F0.y, 1);
    if (lane == 0) { la = 0; lb = 1; lc = 0; lfx = 0; lfy = 0; }
    if (lane == 31) { ua = 0; ub = 1; uc = 0; ufx = 0; ufy = 0; }
    // slot 0: lower = (la..), upper = own slot 1
    const T k1a = A0 / lb, k2a = C0 / B1;
    const T nA0 = -k1a * la, nC0 = -k2a * C1;
    const T nB0 = B0 - k1a * lc - k2a * A1;
    const C nF0 = mk<C>(F0.x - k1a * lfx - k2a * F1.x, F0.y - k1a * lfy - k2a * F1.y);
    // slot 1: lower = own slot 0, upper = (ua..)
    const T k1b = A1 / B0, k2b = C1 / ub;
    const T nA1 = -k1b * A0, nC1 = -k2b * uc;
    const T nB1 = B1 - k1b * C0 - k2b * ua;
    const C nF1 = mk<C>(F1.x - k1b * F0.x - k2b * ufx, F1.y - k1b * F0.y - k2b * ufy);
    A0 = nA0; B0 = nB0; C0 = nC0; F0 = nF0;
    A1 = nA1; B1 = nB1; C1 = nC1; F1 = nF1;
  }
#pragma unroll
  for (int t = 1; t < 32; t <<= 1) {
    // stride 2t: neighbours are lane -/+ t, same slot
    const bool hasl = lane >= t, hasu = lane + t < 32;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      T& A = s ? A1 : A0;
      T& B = s ? B1 : B0;
      T& Cc = s ? C1 : C0;
      C& Fv = s ? F1 : F0;
      T la = __shfl_up_sync(full, A, t), lb = __shfl_up_sync(full, B, t), lc = __shfl_up_sync(full, Cc, t);
      T lfx = __shfl_up_sync(full, Fv.x, t), lfy = __shfl_up_sync(full, Fv.y, t);
      T ua = __shfl_down_sync(full, A, t), ub = __shfl_down_sync(full, B, t), uc = __shfl_down_sync(full, Cc, t);
      T ufx = __shfl_down_sync(full, Fv.x, t), ufy = __shfl_down_sync(full, Fv.y, t);
      if (!hasl) { la = 0; lb = 1; lc = 0; lfx = 0; lfy = 0; }
      if (!hasu) { ua = 0; ub = 1; uc = 0; ufx = 0; ufy = 0; }
      const T k1 = A / lb, k2 = Cc / ub;
      const T nB = B - k1 * lc - k2 * ua;
      const C nF = mk<C>(Fv.x - k1 * lfx - k2 * ufx, Fv.y - k1 * lfy - k2 * ufy);
      A = -k1 * la;
      Cc = -k2 * uc;
      B = nB;
      Fv = nF;
    }
  }
  const C x0 = mk<C>(F0.x / B0, F0.y / B0);
  const C xl = mk<C>(F1.x / B1, F1.y / B1);
#pragma unroll
  for (int i = 1; i < M - 1; ++i) {
    const T rb = (T)1 / b[i];
    f[i] = mk<C>((f[i].x - ap[i] * x0.x - cq[i] * xl.x) * rb, (f[i].y - ap[i] * x0.y - cq[i] * xl.y) * rb);
  }
  f[0] = x0;
  f[M - 1] = xl;
}

// shared-memory column: row j at (j / M) * LS + j % M, LS odd (bank spread)
template <int M> struct ColIdx {
  static constexpr int LS = (M % 2) ? M : M + 1;
  static constexpr int SIZE = 32 * LS;
  __device__ static __forceinline__ int at(int j) { return (j / M) * LS + (j % M); }
};

// conversion between the storage and compute complex types
template <typename C, typename SC>
__device__ __forceinline__ C cvt(SC v) { return mk<C>((decltype(C::x))v.x, (decltype(C::x))v.y); }

// Load a global y-column [0, n) into a shared column (coalesced), zero-padded.
template <typename C, int M, typename SC>
__device__ __forceinline__ void load_col(C* s, const SC* __restrict__ gsrc, int n, int lane) {
  for (int j = lane; j < 32 * M; j += 32) s[ColIdx<M>::at(j)] = (j < n) ? cvt<C>(gsrc[j]) : czero<C>();
}
template <typename C, int M, typename SC>
__device__ __forceinline__ void store_col(SC* __restrict__ gdst, const C* s, int n, int lane) {
  for (int j = lane; j < n; j += 32) gdst[j] = cvt<SC>(s[ColIdx<M>::at(j)]);
}

// Second difference d2_dy (PFC/diff_int.f90:31-46) at row j of an n-row
// column.  The end rows use their own (copied) coefficient columns applied to
// rows 1..3 and n-2..n, as the Fortran does.
template <typename T, int M>
__device__ __forceinline__ cplx_t<T> d2_row(const cplx_t<T>* s, const double* __restrict__ d,
                                            int j, int n) {
  using C = cplx_t<T>;
  int jm, j0, jp;
  if (j == 0) { jm = 0; j0 = 1; jp = 2; }
  else if (j == n - 1) { jm = n - 3; j0 = n - 2; jp = n - 1; }
  else { jm = j - 1; j0 = j; jp = j + 1; }
  const T d1 = (T)__ldg(d + 3 * j), d2 = (T)__ldg(d + 3 * j + 1), d3 = (T)__ldg(d + 3 * j + 2);
  const C fm = s[ColIdx<M>::at(jm)], f0 = s[ColIdx<M>::at(j0)], fp = s[ColIdx<M>::at(jp)];
  return mk<C>(d1 * fm.x + d2 * f0.x + d3 * fp.x, d1 * fm.y + d2 * f0.y + d3 * fp.y);
}

// Helmholtz solve (SOLVE_HELMHOLTZ, PFC/solve.f90:154-264, Dirichlet rows)
// of an n-row column in shared memory: rows 1..n-2 are
// (-diff*d2(1), alpha - diff*d2(2), -diff*d2(3)), row 0 / n-1 fix botbc/topbc.
template <typename T, int M>
__device__ __forceinline__ void helmholtz_col(cplx_t<T>* s, int n, T alpha, T diff,
                                              const double* __restrict__ d2, cplx_t<T> topbc,
                                              cplx_t<T> botbc, int lane) {
  using C = cplx_t<T>;
  T a[M], b[M], c[M];
  C f[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int j = lane * M + i;
    if (j == 0) { a[i] = 0; b[i] = 1; c[i] = 0; f[i] = botbc; }
    else if (j == n - 1) { a[i] = 0; b[i] = 1; c[i] = 0; f[i] = topbc; }
    else if (j < n - 1) {
      a[i] = -diff * (T)__ldg(d2 + 3 * j);
      b[i] = -diff * (T)__ldg(d2 + 3 * j + 1) + alpha;
      c[i] = -diff * (T)__ldg(d2 + 3 * j + 2);
      f[i] = s[ColIdx<M>::at(j)];
    } else { a[i] = 0; b[i] = 1; c[i] = 0; f[i] = czero<C>(); }
  }
  tri_partition_solve<T, M>(a, b, c, f, lane);
  __syncwarp();
#pragma unroll
  for (int i = 0; i < M; ++i) s[ColIdx<M>::at(lane * M + i)] = f[i];
  __syncwarp();
}

// SOLVE_P (PFC/solve.f90:269-338) on an (ny+1)-row column with zero Neumann
// data, including the dm re-extrapolation of rows 1 and ny+1.
template <typename T, int M>
__device__ __forceinline__ void solve_p_col(cplx_t<T>* s, int ny, T alpha, const GridDev& gd,
                                            int lane) {
  using C = cplx_t<T>;
  T a[M], b[M], c[M];
  C f[M];
  const int n = ny + 1;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int j = lane * M + i;
    if (j == 0) {
      const T dn0 = (T)gd.dn[0];
      a[i] = 0; b[i] = -dn0; c[i] = dn0; f[i] = czero<C>();
    } else if (j == n - 1) {
      const T dnl = (T)gd.dn[ny - 1];
      a[i] = -dnl; b[i] = dnl; c[i] = 0; f[i] = czero<C>();
    } else if (j < n - 1) {
      const T dh = (T)gd.dh[j], dm1 = (T)gd.dn[j - 1], dn0 = (T)gd.dn[j];
      a[i] = dh * dm1;
      b[i] = -(dh * dm1) - dh * dn0 + alpha;
      c[i] = dh * dn0;
      f[i] = s[ColIdx<M>::at(j)];
    } else { a[i] = 0; b[i] = 1; c[i] = 0; f[i] = czero<C>(); }
  }
  tri_partition_solve<T, M>(a, b, c, f, lane);
  __syncwarp();
#pragma unroll
  for (int i = 0; i < M; ++i) s[ColIdx<M>::at(lane * M + i)] = f[i];
  __syncwarp();
  if (lane == 0) {
    const T m11 = (T)gd.dm[0], m21 = (T)gd.dm[1], m31 = (T)gd.dm[2];
    const T m12 = (T)gd.dm[3], m22 = (T)gd.dm[4], m32 = (T)gd.dm[5];
    const C p1 = s[ColIdx<M>::at(1)], p2 = s[ColIdx<M>::at(2)];
    const C q1 = s[ColIdx<M>::at(ny - 2)], q2 = s[ColIdx<M>::at(ny - 1)];
    s[ColIdx<M>::at(0)] = mk<C>((-m21 * p1.x - m31 * p2.x) / m11, (-m21 * p1.y - m31 * p2.y) / m11);
    s[ColIdx<M>::at(ny)] = mk<C>((-m12 * q1.x - m22 * q2.x) / m32, (-m12 * q1.y - m22 * q2.y) / m32);
  }
  __syncwarp();
}

// subtract_pressure_gradient (PFC/solve.f90:54-77) from three shared columns,
// rows owned by this lane.
template <typename T, int M>
__device__ __forceinline__ void sub_grad(cplx_t<T>* su, cplx_t<T>* sv, cplx_t<T>* sw,
                                         const cplx_t<T>* sp, T coef, T kx, T kz, int ny,
                                         const GridDev& gd, int lane) {
  using C = cplx_t<T>;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int j = lane * M + i;
    if (j >= 1 && j <= ny - 1) {
      const C p = sp[ColIdx<M>::at(j)];
      const int q = ColIdx<M>::at(j);
      su[q] = csub(su[q], cimul<C>(coef * kx, p));
      sw[q] = csub(sw[q], cimul<C>(coef * kz, p));
      if (j <= ny - 2) {
        const C pp = sp[ColIdx<M>::at(j + 1)];
        const T dn = (T)gd.dn[j];
        sv[q] = csub(sv[q], cscale(coef * dn, csub(pp, p)));
      }
    }
  }
  __syncwarp();
}

// One (kx,kz) != (0,0) wavenumber per warp: PHASE1 (PFC/pass2.f90:184-352).
// mode 0: RK substep.  mode 1: remove_initial_divergence (strip_divergence
// with coef 1, PFC/init_vel.f90:518-536).  mode 2: solve_continuous_poisson
// (PFC/init_vel.f90:477-513): pressure from the velocity held in cru and the
// nonlinear term in vel.
// T is the arithmetic precision, S the storage precision of the state: the
// mixed path runs its low-|k| wavenumbers with T = double over S = float.
template <typename T, typename S, int M>
__global__ void __launch_bounds__(128) k_rhs(cplx_t<S>* __restrict__ vel,
                                             cplx_t<S>* __restrict__ cru,
                                             cplx_t<S>* __restrict__ prs,
                                             const cplx_t<S>* __restrict__ cbc_top,
                                             const cplx_t<S>* __restrict__ cbc_bot, Geom g,
                                             GridDev gd, const DevScalars* __restrict__ sc,
                                             RkTab rkt, int rk, double re, int mode,
                                             const int* __restrict__ wlist, int nlist) {
  using C = cplx_t<T>;
  using CI = ColIdx<M>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int widx = blockIdx.x * (blockDim.x >> 5) + warp;
  if (widx >= nlist) return;
  const int w = wlist ? wlist[widx] : widx + 1;   // skip the mean mode
  const int NZ = g.nz, ny = g.ny, n1 = g.ny1;
  const int kxi = w / NZ, kzi = w % NZ;
  const T kx = (T)gd.kx[kxi], kz = (T)gd.kz[kzi];
  const T k2 = (T)(gd.kx[kxi] * gd.kx[kxi] + gd.kz[kzi] * gd.kz[kzi]);
  C* sbase = reinterpret_cast<C*>(smem_raw) + warp * 5 * CI::SIZE;
  C* su = sbase;
  C* sv = sbase + CI::SIZE;
  C* sw = sbase + 2 * CI::SIZE;
  C* sp = sbase + 3 * CI::SIZE;
  C* sh = sbase + 4 * CI::SIZE;
  using SC = cplx_t<S>;
  SC* gvel = vel + (size_t)w * 3 * n1;
  SC* gcru = cru + (size_t)w * 3 * n1;
  SC* gprs = prs + (size_t)w * n1;
  const size_t nw = (size_t)g.nw;

  if (mode == 1) {
    // strip_divergence(data1 column, ch, 1, x, z)
    load_col<C, M>(su, gvel, n1, lane);
    load_col<C, M>(sv, gvel + n1, n1, lane);
    load_col<C, M>(sw, gvel + 2 * n1, n1, lane);
    __syncwarp();
  } else if (mode == 2) {
    // cru = -NL + (1/re)(D2 - k2) u, with u from cru (velocity copy)
    const T visc = (T)(1.0 / re);
    load_col<C, M>(sp, gcru, n1, lane);
    load_col<C, M>(sh, gcru + n1, n1, lane);
    __syncwarp();
    C r[3][M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = lane * M + i;
      if (j < n1) {
        const C u = sp[CI::at(j)], v = sh[CI::at(j)];
        const C du = d2_row<T, M>(sp, gd.d2h, j, n1);
        r[0][i] = cadd(cscale((T)-1, cvt<C>(gvel[j])), cscale(visc, csub(du, cscale(k2, u))));
        if (j < ny) {
          const C dv = d2_row<T, M>(sh, gd.d2n, j, ny);
          r[1][i] = cadd(cscale((T)-1, cvt<C>(gvel[n1 + j])), cscale(visc, csub(dv, cscale(k2, v))));
        } else r[1][i] = cscale((T)-1, cvt<C>(gvel[n1 + j]));
      } else { r[0][i] = czero<C>(); r[1][i] = czero<C>(); }
    }
    __syncwarp();
    load_col<C, M>(sp, gcru + 2 * n1, n1, lane);
    __syncwarp();
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = lane * M + i;
      if (j < n1) {
        const C ww = sp[CI::at(j)];
        const C dw = d2_row<T, M>(sp, gd.d2h, j, n1);
        r[2][i] = cadd(cscale((T)-1, cvt<C>(gvel[2 * n1 + j])), cscale(visc, csub(dw, cscale(k2, ww))));
      } else r[2][i] = czero<C>();
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int q = CI::at(lane * M + i);
      su[q] = r[0][i]; sv[q] = r[1][i]; sw[q] = r[2][i];
    }
    __syncwarp();
  } else {
    // ---- stage A: cv = cru + coef*cu (+ explicit viscous, old pressure on rk1)
    const double dt = sc->dt;
    const T coef = (T)(rkt.B(rk) * dt);
    const T vis_exp = (T)(rkt.Cc(rk) * (dt / re));
    const T rk_press = (T)((rkt.Cc(rk) + rkt.D(rk)) * dt);
    C* scol[3] = {su, sv, sw};
    for (int q = 0; q < 3; ++q) load_col<C, M>(scol[q], gcru + q * n1, n1, lane);
    __syncwarp();
    for (int q = 0; q < 3; ++q) {
      const double* d2 = (q == 1) ? gd.d2n : gd.d2h;
      const int nq = (q == 1) ? ny : n1;
      C r[M];
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const int j = lane * M + i;
        if (j < n1) {
          const C cr = scol[q][CI::at(j)];
          const C nl = cvt<C>(gvel[q * n1 + j]);
          C v = mk<C>(cr.x - coef * nl.x, cr.y - coef * nl.y);
          if (rk == 1 && j < nq) {
            const C du = d2_row<T, M>(scol[q], d2, j, nq);
            v = cadd(v, cscale(vis_exp, csub(du, cscale(k2, cr))));
          }
          r[i] = v;
        } else r[i] = czero<C>();
      }
      __syncwarp();
#pragma unroll
      for (int i = 0; i < M; ++i) scol[q][CI::at(lane * M + i)] = r[i];
      __syncwarp();
    }
    load_col<C, M>(sp, gprs, n1, lane);
    __syncwarp();
    if (rk == 1) sub_grad<T, M>(su, sv, sw, sp, rk_press, kx, kz, ny, gd, lane);
    // ---- stage B: Helmholtz solves for u, w (ny+1 rows, d2h) and v (ny rows, d2n)
    const T vis_imp = (T)(rkt.D(rk) * (dt / re));
    const T alpha = (T)1 + vis_imp * k2;
    helmholtz_col<T, M>(su, n1, alpha, vis_imp, gd.d2h, cvt<C>(cbc_top[w]), cvt<C>(cbc_bot[w]), lane);
    helmholtz_col<T, M>(sw, n1, alpha, vis_imp, gd.d2h, cvt<C>(cbc_top[2 * nw + w]), cvt<C>(cbc_bot[2 * nw + w]), lane);
    helmholtz_col<T, M>(sv, ny, alpha, vis_imp, gd.d2n, cvt<C>(cbc_top[nw + w]), cvt<C>(cbc_bot[nw + w]), lane);
    if (lane == 0) sv[CI::at(ny)] = czero<C>();
    __syncwarp();
  }

  // ---- stage C: strip_divergence (PFC/solve.f90:14-50)
  const double dt = sc->dt;
  const T rk_press = (mode == 0) ? (T)((rkt.Cc(rk) + rkt.D(rk)) * dt) : (T)1;
  {
    const T tmp = (T)1 / rk_press;
    C r[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = lane * M + i;
      if (j >= 1 && j <= ny - 1) {
        const T dh = (T)gd.dh[j];
        const C dv = cscale(dh, csub(sv[CI::at(j)], sv[CI::at(j - 1)]));
        const C s = cadd(cadd(cimul<C>(kx, su[CI::at(j)]), dv), cimul<C>(kz, sw[CI::at(j)]));
        r[i] = cscale(tmp, s);
      } else r[i] = czero<C>();
    }
    C* dst = (mode == 2) ? sp : sh;
    __syncwarp();
#pragma unroll
    for (int i = 0; i < M; ++i) dst[CI::at(lane * M + i)] = r[i];
    __syncwarp();
    solve_p_col<T, M>(dst, ny, -k2, gd, lane);
    if (mode == 2) {
      store_col<C, M>(gprs, sp, n1, lane);
      return;
    }
    sub_grad<T, M>(su, sv, sw, dst, rk_press, kx, kz, ny, gd, lane);
  }
  if (mode == 1) {
    store_col<C, M>(gvel, su, n1, lane);
    store_col<C, M>(gvel + n1, sv, n1, lane);
    store_col<C, M>(gvel + 2 * n1, sw, n1, lane);
    return;
  }
  // ---- p = p + alpha*ch - vis_imp*D2h(ch)  (Brown, Cortez & Minion)
  const T vis_imp = (T)(rkt.D(rk) * (dt / re));
  const T alpha = (T)1 + vis_imp * k2;
  {
    C r[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = lane * M + i;
      if (j < n1) {
        const C ch = sh[CI::at(j)];
        const C d2c = d2_row<T, M>(sh, gd.d2h, j, n1);
        const C p = sp[CI::at(j)];
        r[i] = mk<C>(p.x + alpha * ch.x - vis_imp * d2c.x, p.y + alpha * ch.y - vis_imp * d2c.y);
      } else r[i] = czero<C>();
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < M; ++i) sp[CI::at(lane * M + i)] = r[i];
    __syncwarp();
  }
  // ---- stage D: next-substep accumulator (PFC/pass2.f90:312-333) and stores
  C* scol[3] = {su, sv, sw};
  if (rk < 3) {
    const T coef2 = (T)(dt * rkt.A(rk + 1));
    const T vis_exp2 = (T)((dt / re) * rkt.Cc(rk + 1));
    const T rkp2 = (T)((rkt.Cc(rk + 1) + rkt.D(rk + 1)) * dt);
    for (int q = 0; q < 3; ++q) {
      const double* d2 = (q == 1) ? gd.d2n : gd.d2h;
      const int nq = (q == 1) ? ny : n1;
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const int j = lane * M + i;
        if (j >= n1) continue;
        const C cv = scol[q][CI::at(j)];
        const C nl = cvt<C>(gvel[q * n1 + j]);
        C v = mk<C>(cv.x - coef2 * nl.x, cv.y - coef2 * nl.y);
        if (j < nq) {
          const C du = d2_row<T, M>(scol[q], d2, j, nq);
          v = cadd(v, cscale(vis_exp2, csub(du, cscale(k2, cv))));
        }
        if (j >= 1 && j <= ny - 1) {
          const C p = sp[CI::at(j)];
          if (q == 0) v = csub(v, cimul<C>(rkp2 * kx, p));
          else if (q == 2) v = csub(v, cimul<C>(rkp2 * kz, p));
          else if (j <= ny - 2) {
            const C pp = sp[CI::at(j + 1)];
            v = csub(v, cscale(rkp2 * (T)gd.dn[j], csub(pp, p)));
          }
        }
        gcru[q * n1 + j] = cvt<SC>(v);
      }
    }
  } else {
    for (int q = 0; q < 3; ++q) store_col<C, M>(gcru + q * n1, scol[q], n1, lane);
  }
  __syncwarp();
  for (int q = 0; q < 3; ++q) store_col<C, M>(gvel + q * n1, scol[q], n1, lane);
  store_col<C, M>(gprs, sp, n1, lane);
}

// The kx = kz = 0 mode in FP64 (PFC/pass2.f90:217-263, compute_p_grad
// :356-375, d_um_dy update :84-89), one warp.  In mixed precision the mean
// columns of vel and cru also live in FP64 side buffers (mvel64, mcru64).
template <typename T, int M>
__global__ void __launch_bounds__(32) k_rhs_mean(cplx_t<T>* __restrict__ vel,
                                                 cplx_t<T>* __restrict__ cru,
                                                 cplx_t<T>* __restrict__ prs,
                                                 double2* __restrict__ mvel64,
                                                 double2* __restrict__ mcru64,
                                                 const cplx_t<T>* __restrict__ cbc_top,
                                                 const cplx_t<T>* __restrict__ cbc_bot, Geom g,
                                                 GridDev gd, DevScalars* __restrict__ sc,
                                                 double* __restrict__ d_um_dy, RkTab rkt,
                                                 int rk, double re, double beta,
                                                 int fix_mass, int mode) {
  using C = double2;
  using CI = ColIdx<M>;
  __shared__ C S[4 * CI::SIZE];
  const int lane = threadIdx.x;
  const int ny = g.ny, n1 = g.ny1;
  const size_t nw = (size_t)g.nw;
  C* su = S;
  C* sv = S + CI::SIZE;
  C* sw = S + 2 * CI::SIZE;
  C* st = S + 3 * CI::SIZE;
  const bool side = (mcru64 != nullptr);
  auto gv = [&](int q, int j) -> C {
    if (side) return mvel64[q * n1 + j];
    const cplx_t<T> v = vel[q * n1 + j];
    return mk<C>((double)v.x, (double)v.y);
  };
  auto gc = [&](int q, int j) -> C {
    if (side) return mcru64[q * n1 + j];
    const cplx_t<T> v = cru[q * n1 + j];
    return mk<C>((double)v.x, (double)v.y);
  };
  auto put = [&](cplx_t<T>* dst, double2* dst64, int idx, C v) {
    dst[idx] = mk<cplx_t<T>>((T)v.x, (T)v.y);
    if (side) dst64[idx] = v;
  };
  if (mode == 1) {
    // remove_initial_divergence, mean branch: v(2:ny) = v(1)
    C v0 = gv(1, 0);
    for (int j = 1 + lane; j < ny; j += 32) put(vel, mvel64, n1 + j, v0);
    __syncwarp();
    // d_um_dy initialisation (PFC/init_vel.f90:333-342) and data2 = data1
    for (int j = lane; j < n1; j += 32) {
      for (int q = 0; q < 3; ++q) {
        C v = (q == 1 && j >= 1 && j < ny) ? v0 : gv(q, j);
        if (side) mcru64[q * n1 + j] = v;
      }
    }
    __syncwarp();
    if (lane == 0) {
      const double* dm = gd.dm;
      C u0 = gv(0, 0), u1 = gv(0, 1), u2 = gv(0, 2);
      d_um_dy[0] = dm[0] * u0.x + dm[1] * u1.x + dm[2] * u2.x;
      C a = gv(0, ny - 2), b = gv(0, ny - 1), c = gv(0, ny);
      d_um_dy[ny - 1] = dm[3] * a.x + dm[4] * b.x + dm[5] * c.x;
    }
    for (int j = 1 + lane; j <= ny - 2; j += 32) d_um_dy[j] = gd.dn[j] * (gv(0, j + 1).x - gv(0, j).x);
    return;
  }
  if (mode == 2) {
    for (int j = lane; j < n1; j += 32) prs[j] = czero<cplx_t<T>>();
    return;
  }
  const double dt = sc->dt;
  const double coef = rkt.B(rk) * dt;
  const double vis_imp = rkt.D(rk) * (dt / re);
  const double rk_press = (rkt.Cc(rk) + rkt.D(rk)) * dt;
  C* scol[3] = {su, sv, sw};
  // cv = cru + coef*cu (+ explicit viscous on rk1)
  for (int q = 0; q < 3; ++q) {
    for (int j = lane; j < 32 * M; j += 32) st[CI::at(j)] = (j < n1) ? gc(q, j) : mk<C>(0, 0);
    __syncwarp();
    const double* d2 = (q == 1) ? gd.d2n : gd.d2h;
    const int nq = (q == 1) ? ny : n1;
    for (int j = lane; j < 32 * M; j += 32) {
      C v = mk<C>(0, 0);
      if (j < n1) {
        const C cr = st[CI::at(j)];
        const cplx_t<T> nl = vel[q * n1 + j];
        v = mk<C>(cr.x - coef * (double)nl.x, cr.y - coef * (double)nl.y);
        if (rk == 1 && j < nq) {
          const double vis_exp = rkt.Cc(rk) * (dt / re);
          const C du = d2_row<double, M>(st, d2, j, nq);
          v = cadd(v, cscale(vis_exp, du));
        }
      }
      scol[q][CI::at(j)] = v;
    }
    __syncwarp();
  }
  // constant mass flux pressure gradient (cu = -NL)
  double pg = sc->p_grad;
  if (fix_mass == 1) {
    double part = 0;
    for (int j = 1 + lane; j <= ny - 1; j += 32) part += gd.dyh[j] * (-(double)vel[j].x);
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    pg = -part + 0.5 * (d_um_dy[ny - 1] - d_um_dy[0]) / re;
  }
  const double cb = cos(beta) * rk_press * pg, sb = sin(beta) * rk_press * pg;
  for (int j = lane; j < n1; j += 32) {
    su[CI::at(j)].x -= cb;
    sw[CI::at(j)].x -= sb;
  }
  __syncwarp();
  auto bc = [&](const cplx_t<T>* a, size_t idx) { const cplx_t<T> v = a[idx]; return mk<C>((double)v.x, (double)v.y); };
  helmholtz_col<double, M>(su, n1, 1.0, vis_imp, gd.d2h, bc(cbc_top, 0), bc(cbc_bot, 0), lane);
  helmholtz_col<double, M>(sw, n1, 1.0, vis_imp, gd.d2h, bc(cbc_top, 2 * nw), bc(cbc_bot, 2 * nw), lane);
  const C vb = bc(cbc_bot, nw);
  for (int j = lane; j < n1; j += 32) sv[CI::at(j)] = (j < ny) ? vb : mk<C>(0, 0);
  __syncwarp();
  // next-substep accumulator and stores
  for (int q = 0; q < 3; ++q) {
    const double* d2 = (q == 1) ? gd.d2n : gd.d2h;
    const int nq = (q == 1) ? ny : n1;
    for (int j = lane; j < n1; j += 32) {
      const C cv = scol[q][CI::at(j)];
      C v = cv;
      if (rk < 3) {
        const double coef2 = dt * rkt.A(rk + 1);
        const double vis_exp2 = (dt / re) * rkt.Cc(rk + 1);
        const cplx_t<T> nl = vel[q * n1 + j];
        v = mk<C>(cv.x - coef2 * (double)nl.x, cv.y - coef2 * (double)nl.y);
        if (j < nq) v = cadd(v, cscale(vis_exp2, d2_row<double, M>(scol[q], d2, j, nq)));
      }
      put(cru, mcru64, q * n1 + j, v);
    }
  }
  __syncwarp();
  for (int q = 0; q < 3; ++q)
    for (int j = lane; j < n1; j += 32) put(vel, mvel64, q * n1 + j, scol[q][CI::at(j)]);
  for (int j = lane; j < n1; j += 32) prs[j] = czero<cplx_t<T>>();
  __syncwarp();
  if (lane == 0) {
    sc->p_grad = pg;
    const double* dm = gd.dm;
    d_um_dy[0] = dm[0] * su[CI::at(0)].x + dm[1] * su[CI::at(1)].x + dm[2] * su[CI::at(2)].x;
    d_um_dy[ny - 1] = dm[3] * su[CI::at(ny - 2)].x + dm[4] * su[CI::at(ny - 1)].x + dm[5] * su[CI::at(ny)].x;
  }
  for (int j = 1 + lane; j <= ny - 2; j += 32) d_um_dy[j] = gd.dn[j] * (su[CI::at(j + 1)].x - su[CI::at(j)].x);
}

}  // namespace cfd
