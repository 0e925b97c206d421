// pass2v2.cuh -- the RK3/Crank-Nicolson substep of PFC/pass2.f90:184-352
// (PHASE1) for the (kx,kz) != (0,0) wavenumbers, G lanes per wavenumber
// (G = 16 or 32, 32/G wavenumbers per warp).  Same arithmetic as k_rhs
// (pass2.cuh) mode 0, organised for throughput:
//   - the seven input columns (NL u,v,w; cru u,v,w; p) are copied into shared
//     memory with cp.async at the start, contiguous per column;
//   - u and w share one partition solve (same Helmholtz matrix, two right-hand
//     sides); every solve multiplies by reciprocals;
//   - the outputs are staged in shared memory and stored coalesced.
#pragma once
#include "cfd_common.cuh"
#include "pass1.cuh"
#include "pass1_reg.cuh"
#include "pass2.cuh"

namespace cfd {

// Reciprocal used by the solves: the approximate single-precision divide
// intrinsic (2 ulp) in FP32, an IEEE divide in FP64.
template <typename T> __device__ __forceinline__ T rcpv(T x);
template <> __device__ __forceinline__ float rcpv<float>(float x) { return __fdividef(1.0f, x); }
template <> __device__ __forceinline__ double rcpv<double>(double x) { return 1.0 / x; }

// One strided PCR step (stride 2t in interface rows = t lanes) of one slot.
template <typename T, int G, int NR>
__device__ __forceinline__ void pcr_step(T& A, T& B, T& Cc, cplx_t<T> (&Fv)[NR], int t, int g) {
  using C = cplx_t<T>;
  const unsigned full = 0xffffffffu;
  const bool hasl = g >= t, hasu = g + t < G;
  T la = __shfl_up_sync(full, A, t, G), lb = __shfl_up_sync(full, B, t, G), lc = __shfl_up_sync(full, Cc, t, G);
  T ua = __shfl_down_sync(full, A, t, G), ub = __shfl_down_sync(full, B, t, G), uc = __shfl_down_sync(full, Cc, t, G);
  C lf[NR], uf[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    lf[r] = mk<C>(__shfl_up_sync(full, Fv[r].x, t, G), __shfl_up_sync(full, Fv[r].y, t, G));
    uf[r] = mk<C>(__shfl_down_sync(full, Fv[r].x, t, G), __shfl_down_sync(full, Fv[r].y, t, G));
  }
  if (!hasl) {
    la = 0; lb = 1; lc = 0;
#pragma unroll
    for (int r = 0; r < NR; ++r) lf[r] = czero<C>();
  }
  if (!hasu) {
    ua = 0; ub = 1; uc = 0;
#pragma unroll
    for (int r = 0; r < NR; ++r) uf[r] = czero<C>();
  }
  const T k1 = A * rcpv(lb), k2 = Cc * rcpv(ub);
  const T nB = B - k1 * lc - k2 * ua;
#pragma unroll
  for (int r = 0; r < NR; ++r)
    Fv[r] = mk<C>(Fv[r].x - k1 * lf[r].x - k2 * uf[r].x, Fv[r].y - k1 * lf[r].y - k2 * uf[r].y);
  A = -k1 * la;
  Cc = -k2 * uc;
  B = nB;
}

// Partition + PCR solve over the G lanes of a lane group, NR right-hand sides.
// Row j = g*M + i of lane g:  a[i] x_{j-1} + b[i] x_j + c[i] x_{j+1} = f[r][i].
// Rows past the system are identity rows.  Solutions overwrite f.
// Each lane eliminates its first M-1 rows in terms of the two interface
// unknowns next to them -- x_L, the previous lane's last row, and x_E, its own
// last row: x_i = y_i - x_L v_i - x_E w_i (Thomas on the M-1 rows with the
// right-hand sides f, a_0 e_0 and c_{M-2} e_{M-2}).  The last rows then form a
// tridiagonal system of G unknowns, one per lane, solved by cyclic reduction
// across the lanes (log2 G shuffle steps); the interior rows follow.
template <typename T, int M, int G, int NR>
__device__ __forceinline__ void tri_group_solve(T (&a)[M], T (&b)[M], T (&c)[M],
                                                cplx_t<T> (&f)[NR][M], int g) {
  using C = cplx_t<T>;
  static_assert(M >= 2, "at least two rows per lane");
  T v[M], w[M], rb[M];
  // forward sweep over the first M-1 rows
  rb[0] = rcpv(b[0]);
  v[0] = a[0];
#pragma unroll
  for (int i = 1; i < M - 1; ++i) {
    const T m = a[i] * rb[i - 1];
    b[i] = b[i] - m * c[i - 1];
    rb[i] = rcpv(b[i]);
    v[i] = -m * v[i - 1];
#pragma unroll
    for (int r = 0; r < NR; ++r) f[r][i] = mk<C>(f[r][i].x - m * f[r][i - 1].x, f[r][i].y - m * f[r][i - 1].y);
  }
  // backward sweep: y (in f), v, w
  w[M - 2] = c[M - 2] * rb[M - 2];
  v[M - 2] = v[M - 2] * rb[M - 2];
#pragma unroll
  for (int r = 0; r < NR; ++r) f[r][M - 2] = mk<C>(f[r][M - 2].x * rb[M - 2], f[r][M - 2].y * rb[M - 2]);
#pragma unroll
  for (int i = M - 3; i >= 0; --i) {
    w[i] = -c[i] * w[i + 1] * rb[i];
    v[i] = (v[i] - c[i] * v[i + 1]) * rb[i];
#pragma unroll
    for (int r = 0; r < NR; ++r)
      f[r][i] = mk<C>((f[r][i].x - c[i] * f[r][i + 1].x) * rb[i], (f[r][i].y - c[i] * f[r][i + 1].y) * rb[i]);
  }
  // interface row (local row M-1) with the next lane's first row substituted
  const unsigned full = 0xffffffffu;
  T vn = __shfl_down_sync(full, v[0], 1, G), wn = __shfl_down_sync(full, w[0], 1, G);
  C yn[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) yn[r] = mk<C>(__shfl_down_sync(full, f[r][0].x, 1, G), __shfl_down_sync(full, f[r][0].y, 1, G));
  if (g == G - 1) {
    vn = 0; wn = 0;
#pragma unroll
    for (int r = 0; r < NR; ++r) yn[r] = czero<C>();
  }
  const T aE = a[M - 1], cE = c[M - 1];
  T A = -aE * v[M - 2];
  T B = b[M - 1] - aE * w[M - 2] - cE * vn;
  T Cc = -cE * wn;
  C F[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r)
    F[r] = mk<C>(f[r][M - 1].x - aE * f[r][M - 2].x - cE * yn[r].x, f[r][M - 1].y - aE * f[r][M - 2].y - cE * yn[r].y);
#pragma unroll
  for (int t = 1; t < G; t <<= 1) pcr_step<T, G, NR>(A, B, Cc, F, t, g);
  const T rB = rcpv(B);
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const C xE = mk<C>(F[r].x * rB, F[r].y * rB);
    C xL = mk<C>(__shfl_up_sync(full, xE.x, 1, G), __shfl_up_sync(full, xE.y, 1, G));
    if (g == 0) xL = czero<C>();
#pragma unroll
    for (int i = 0; i < M - 1; ++i)
      f[r][i] = mk<C>(f[r][i].x - xL.x * v[i] - xE.x * w[i], f[r][i].y - xL.y * v[i] - xE.y * w[i]);
    f[r][M - 1] = xE;
  }
}

// Grid coefficients of the RK substep in the storage precision, lane-major:
// tbl[(kind*M + i)*G + g] is coefficient `kind` of row j = g*M + i (0 past the
// end of its range), so that the G lanes of a group read consecutive words.
enum Rhs2Coef { RC_D2H = 0, RC_D2N = 3, RC_DN = 6, RC_DH = 7, RC_DNM1 = 8, RC_NUM = 9 };

template <typename T, int M, int G>
__device__ __forceinline__ T rc(const T* __restrict__ tbl, int kind, int i, int g) {
  return __ldg(tbl + (kind * M + i) * G + g);
}

// second difference of column s at row j = g*M + i of an n-row system (end
// rows copy their neighbours' stencil), coefficients d2[kind0 .. kind0+2]
template <typename T, int M, int G>
__device__ __forceinline__ cplx_t<T> d2c_t(const cplx_t<T>* s, const T* __restrict__ tbl, int kind0, int i, int g,
                                           int j, int n) {
  using C = cplx_t<T>;
  const int j0 = (j == 0) ? 1 : ((j == n - 1) ? n - 2 : j);
  const T d1 = rc<T, M, G>(tbl, kind0, i, g), d2 = rc<T, M, G>(tbl, kind0 + 1, i, g),
          d3 = rc<T, M, G>(tbl, kind0 + 2, i, g);
  const C fm = s[j0 - 1], f0 = s[j0], fp = s[j0 + 1];
  return mk<C>(d1 * fm.x + d2 * f0.x + d3 * fp.x, d1 * fm.y + d2 * f0.y + d3 * fp.y);
}

// column stride (complex elements) of the staged columns: ny+1 rounded up to
// even (16-byte aligned columns for FP32 complex)
__host__ __device__ __forceinline__ int rhs2_ld(int n1) { return (n1 + 1) & ~1; }

// Shared memory per wavenumber: eight columns
//   0-2 cru (u,v,w), overwritten by the new velocity cv;  3 pressure;
//   4 pressure correction;  5-7 nonlinear term, overwritten by the next cru.
// T is the arithmetic precision, S the storage precision of the state (the
// mixed path runs its |k| < 4 list with T = double over S = float).
template <typename T, typename S, int M, int G>
__device__ __forceinline__ void k_rhs2_body(const uint3 bid, cplx_t<S>* __restrict__ vel, cplx_t<S>* __restrict__ cru,
                                            cplx_t<S>* __restrict__ prs, const cplx_t<S>* __restrict__ cbc_top,
                                            const cplx_t<S>* __restrict__ cbc_bot, Geom g, GridDev gd,
                                            const DevScalars* __restrict__ sc, RkTab rkt, int rk, double re,
                                            const int* __restrict__ wlist, int nlist, const T* __restrict__ tbl) {
  using C = cplx_t<T>;
  using CS = cplx_t<S>;
  constexpr int GPW = 32 / G;                 // lane groups (wavenumbers) per warp
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int grp = lane / G, gl = lane % G;
  const int widx = (bid.x * (blockDim.x >> 5) + warp) * GPW + grp;
  const bool valid = widx < nlist;
  const int w = valid ? wlist[widx] : 1;
  const int NZ = g.nz, ny = g.ny, n1 = g.ny1;
  const int LD = rhs2_ld(n1);
  const size_t nw = (size_t)g.nw;
  const int kxi = w / NZ, kzi = w % NZ;
  const T kx = (T)gd.kx[kxi], kz = (T)gd.kz[kzi];
  const T k2 = valid ? (T)(gd.kx[kxi] * gd.kx[kxi] + gd.kz[kzi] * gd.kz[kzi]) : (T)1;
  C* S_ = reinterpret_cast<C*>(smem_raw) + (size_t)(warp * GPW + grp) * 8 * LD;
  C* sV = S_;             // 3 columns: cru, then the new velocity cv
  C* sP = S_ + 3 * LD;    // pressure
  C* sH = S_ + 4 * LD;    // pressure correction
  C* sN = S_ + 5 * LD;    // 3 columns: nonlinear term, then the next cru
  CS* gvel = vel + (size_t)w * 3 * n1;
  CS* gcru = cru + (size_t)w * 3 * n1;
  CS* gprs = prs + (size_t)w * n1;

  // ---- asynchronous staging of the seven input columns: cru (u,v,w), p, NL (u,v,w)
  if (valid && sizeof(S) != sizeof(T)) {
    // widening copy (mixed storage, FP64 arithmetic)
#pragma unroll
    for (int col = 0; col < 7; ++col) {
      const CS* src = (col < 3) ? gcru + col * n1 : (col == 3 ? gprs : gvel + (col - 4) * n1);
      C* dst = S_ + (col < 4 ? col : col + 1) * LD;
      for (int j = gl; j < n1; j += G) dst[j] = cvt<C>(src[j]);
    }
  } else if (valid) {
    const int cb = (int)(n1 * sizeof(C));
    const bool v16 = (cb % 16) == 0;
    const int csz = v16 ? 16 : 8, nch = cb / csz;
#pragma unroll
    for (int col = 0; col < 7; ++col) {
      const char* src = reinterpret_cast<const char*>((col < 3) ? gcru + col * n1 : (col == 3 ? gprs : gvel + (col - 4) * n1));
      char* dst = reinterpret_cast<char*>(S_ + (col < 4 ? col : col + 1) * LD);
      for (int part = gl; part < nch; part += G) {
        if (v16) cp_async16(dst + part * 16, src + part * 16);
        else cp_async8(dst + part * 8, src + part * 8);
      }
    }
  } else {
    for (int idx = gl; idx < 8 * LD; idx += G) S_[idx] = czero<C>();
  }
  cp_async_commit();
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncwarp();

  const double dt = sc->dt;
  const T coef = (T)(rkt.B(rk) * dt);
  const T vis_imp = (T)(rkt.D(rk) * (dt / re));
  const T rk_press = (T)((rkt.Cc(rk) + rkt.D(rk)) * dt);
  const T alpha = (T)1 + vis_imp * k2;
  // ---- stage A: cv = cru + coef*cu (+ explicit viscous term and old pressure gradient on rk1)
  {
    const T vis_exp = (T)(rkt.Cc(rk) * (dt / re));
    C r[3][M];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int kd = (q == 1) ? RC_D2N : RC_D2H;
      const int nq = (q == 1) ? ny : n1;
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const int j = gl * M + i;
        C v = czero<C>();
        if (j < n1) {
          const C cr = sV[q * LD + j];
          const C nl = sN[q * LD + j];
          v = mk<C>(cr.x - coef * nl.x, cr.y - coef * nl.y);
          if (rk == 1) {
            if (j < nq) {
              const C du = d2c_t<T, M, G>(sV + q * LD, tbl, kd, i, gl, j, nq);
              v = cadd(v, cscale(vis_exp, csub(du, cscale(k2, cr))));
            }
            if (j >= 1 && j <= ny - 1) {
              const C p = sP[j];
              if (q == 0) v = csub(v, cimul<C>(rk_press * kx, p));
              else if (q == 2) v = csub(v, cimul<C>(rk_press * kz, p));
              else if (j <= ny - 2)
                v = csub(v, cscale(rk_press * rc<T, M, G>(tbl, RC_DN, i, gl), csub(sP[j + 1], p)));
            }
          }
        }
        r[q][i] = v;
      }
    }
    __syncwarp();
    // ---- stage B: Helmholtz solves, u and w together (d2h), then v (d2n)
    {
      T a[M], b[M], c[M];
      C f[2][M];
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const int j = gl * M + i;
        if (j == 0) {
          a[i] = 0; b[i] = 1; c[i] = 0;
          f[0][i] = cvt<C>(cbc_bot[w]); f[1][i] = cvt<C>(cbc_bot[2 * nw + w]);
        } else if (j == n1 - 1) {
          a[i] = 0; b[i] = 1; c[i] = 0;
          f[0][i] = cvt<C>(cbc_top[w]); f[1][i] = cvt<C>(cbc_top[2 * nw + w]);
        } else if (j < n1 - 1) {
          a[i] = -vis_imp * rc<T, M, G>(tbl, RC_D2H, i, gl);
          b[i] = -vis_imp * rc<T, M, G>(tbl, RC_D2H + 1, i, gl) + alpha;
          c[i] = -vis_imp * rc<T, M, G>(tbl, RC_D2H + 2, i, gl);
          f[0][i] = r[0][i]; f[1][i] = r[2][i];
        } else {
          a[i] = 0; b[i] = 1; c[i] = 0;
          f[0][i] = czero<C>(); f[1][i] = czero<C>();
        }
      }
      tri_group_solve<T, M, G, 2>(a, b, c, f, gl);
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const int j = gl * M + i;
        if (j < LD) { sV[j] = f[0][i]; sV[2 * LD + j] = f[1][i]; }
      }
    }
    {
      T a[M], b[M], c[M];
      C f[1][M];
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const int j = gl * M + i;
        if (j == 0) { a[i] = 0; b[i] = 1; c[i] = 0; f[0][i] = cvt<C>(cbc_bot[nw + w]); }
        else if (j == ny - 1) { a[i] = 0; b[i] = 1; c[i] = 0; f[0][i] = cvt<C>(cbc_top[nw + w]); }
        else if (j < ny - 1) {
          a[i] = -vis_imp * rc<T, M, G>(tbl, RC_D2N, i, gl);
          b[i] = -vis_imp * rc<T, M, G>(tbl, RC_D2N + 1, i, gl) + alpha;
          c[i] = -vis_imp * rc<T, M, G>(tbl, RC_D2N + 2, i, gl);
          f[0][i] = r[1][i];
        } else { a[i] = 0; b[i] = 1; c[i] = 0; f[0][i] = czero<C>(); }
      }
      tri_group_solve<T, M, G, 1>(a, b, c, f, gl);
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const int j = gl * M + i;
        if (j < LD) sV[LD + j] = f[0][i];
      }
    }
    __syncwarp();
  }
  // ---- stage C: strip_divergence (PFC/solve.f90:14-50) and SOLVE_P
  {
    const T tmp = (T)1 / rk_press;
    T a[M], b[M], c[M];
    C f[1][M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = gl * M + i;
      if (j == 0) {
        const T dn0 = rc<T, M, G>(tbl, RC_DN, i, gl);
        a[i] = 0; b[i] = -dn0; c[i] = dn0; f[0][i] = czero<C>();
      } else if (j == n1 - 1) {
        const T dnl = rc<T, M, G>(tbl, RC_DNM1, i, gl);
        a[i] = -dnl; b[i] = dnl; c[i] = 0; f[0][i] = czero<C>();
      } else if (j < n1 - 1) {
        const T dh = rc<T, M, G>(tbl, RC_DH, i, gl), dm1 = rc<T, M, G>(tbl, RC_DNM1, i, gl),
                dn0 = rc<T, M, G>(tbl, RC_DN, i, gl);
        a[i] = dh * dm1;
        b[i] = -(dh * dm1) - dh * dn0 - k2;
        c[i] = dh * dn0;
        const C dv = cscale(dh, csub(sV[LD + j], sV[LD + j - 1]));
        const C s = cadd(cadd(cimul<C>(kx, sV[j]), dv), cimul<C>(kz, sV[2 * LD + j]));
        f[0][i] = cscale(tmp, s);
      } else { a[i] = 0; b[i] = 1; c[i] = 0; f[0][i] = czero<C>(); }
    }
    tri_group_solve<T, M, G, 1>(a, b, c, f, gl);
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = gl * M + i;
      if (j < LD) sH[j] = f[0][i];
    }
    __syncwarp();
    if (gl == 0) {
      const T m11 = (T)gd.dm[0], m21 = (T)gd.dm[1], m31 = (T)gd.dm[2];
      const T m12 = (T)gd.dm[3], m22 = (T)gd.dm[4], m32 = (T)gd.dm[5];
      const C p1 = sH[1], p2 = sH[2], q1 = sH[ny - 2], q2 = sH[ny - 1];
      sH[0] = mk<C>((-m21 * p1.x - m31 * p2.x) / m11, (-m21 * p1.y - m31 * p2.y) / m11);
      sH[ny] = mk<C>((-m12 * q1.x - m22 * q2.x) / m32, (-m12 * q1.y - m22 * q2.y) / m32);
    }
    __syncwarp();
    // subtract the correction gradient from cv; p += alpha*ch - vis_imp*D2h(ch)
    C pn[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = gl * M + i;
      pn[i] = czero<C>();
      if (j < n1) {
        const C ch = sH[j];
        if (j >= 1 && j <= ny - 1) {
          sV[j] = csub(sV[j], cimul<C>(rk_press * kx, ch));
          sV[2 * LD + j] = csub(sV[2 * LD + j], cimul<C>(rk_press * kz, ch));
          if (j <= ny - 2)
            sV[LD + j] = csub(sV[LD + j], cscale(rk_press * rc<T, M, G>(tbl, RC_DN, i, gl), csub(sH[j + 1], ch)));
        }
        const C d2c_ = d2c_t<T, M, G>(sH, tbl, RC_D2H, i, gl, j, n1);
        const C p = sP[j];
        pn[i] = mk<C>(p.x + alpha * ch.x - vis_imp * d2c_.x, p.y + alpha * ch.y - vis_imp * d2c_.y);
      }
    }
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = gl * M + i;
      if (j < n1) sP[j] = pn[i];
    }
    __syncwarp();
  }
  // ---- stage D: next-substep accumulator (PFC/pass2.f90:312-333) at each
  // lane's own rows into the nonlinear-term columns; then data1 <- cv,
  // data2 <- accumulator and data4 <- p, coalesced
  if (rk < 3) {
    const T coef2 = (T)(dt * rkt.A(rk + 1));
    const T vis_exp2 = (T)((dt / re) * rkt.Cc(rk + 1));
    const T rkp2 = (T)((rkt.Cc(rk + 1) + rkt.D(rk + 1)) * dt);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int kd = (q == 1) ? RC_D2N : RC_D2H;
      const int nq = (q == 1) ? ny : n1;
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const int j = gl * M + i;
        if (j >= n1) continue;
        const C cv = sV[q * LD + j];
        const C nl = sN[q * LD + j];
        C v = mk<C>(cv.x - coef2 * nl.x, cv.y - coef2 * nl.y);
        if (j < nq) {
          const C du = d2c_t<T, M, G>(sV + q * LD, tbl, kd, i, gl, j, nq);
          v = cadd(v, cscale(vis_exp2, csub(du, cscale(k2, cv))));
        }
        if (j >= 1 && j <= ny - 1) {
          const C p = sP[j];
          if (q == 0) v = csub(v, cimul<C>(rkp2 * kx, p));
          else if (q == 2) v = csub(v, cimul<C>(rkp2 * kz, p));
          else if (j <= ny - 2) v = csub(v, cscale(rkp2 * rc<T, M, G>(tbl, RC_DN, i, gl), csub(sP[j + 1], p)));
        }
        sN[q * LD + j] = v;
      }
    }
  }
  __syncwarp();
  if (valid) {
    const C* acc = (rk < 3) ? sN : sV;
    for (int q = 0; q < 3; ++q)
      for (int j = gl; j < n1; j += G) {
        gvel[q * n1 + j] = cvt<CS>(sV[q * LD + j]);
        gcru[q * n1 + j] = cvt<CS>(acc[q * LD + j]);
      }
    for (int j = gl; j < n1; j += G) gprs[j] = cvt<CS>(sP[j]);
  }
}

template <typename T, typename S, int M, int G>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 5 : 1)
k_rhs2(cplx_t<S>* __restrict__ vel, cplx_t<S>* __restrict__ cru, cplx_t<S>* __restrict__ prs,
       const cplx_t<S>* __restrict__ cbc_top, const cplx_t<S>* __restrict__ cbc_bot, Geom g, GridDev gd,
       const DevScalars* __restrict__ sc, RkTab rkt, int rk, double re, const int* __restrict__ wlist, int nlist,
       const T* __restrict__ tbl) {
  k_rhs2_body<T, S, M, G>(blockIdx, vel, cru, prs, cbc_top, cbc_bot, g, gd, sc, rkt, rk, re, wlist, nlist, tbl);
}

// Mean mode (kx = kz = 0) of the substep with the constant-mass-flux pressure
// gradient (PFC/pass2.f90:217-263, 356-375), FP64 arithmetic, one warp of 32
// lanes: the cru and NL columns are staged in shared memory, u and w share
// one solve (alpha = 1), v takes the wall value.  In mixed precision the FP64
// mean columns live in mvel64/mcru64 beside the FP32 state.
template <typename S, int M>
__device__ __forceinline__ void k_rhs_mean2_body(const uint3 bid, cplx_t<S>* __restrict__ vel,
                                                 cplx_t<S>* __restrict__ cru, cplx_t<S>* __restrict__ prs,
                                                 double2* __restrict__ mvel64, double2* __restrict__ mcru64,
                                                 const cplx_t<S>* __restrict__ cbc_top,
                                                 const cplx_t<S>* __restrict__ cbc_bot, Geom g, GridDev gd,
                                                 DevScalars* __restrict__ sc, double* __restrict__ d_um_dy, RkTab rkt,
                                                 int rk, double re, double beta, int fix_mass,
                                                 const double* __restrict__ tbl) {
  using C = double2;
  using CS = cplx_t<S>;
  constexpr int G = 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x;
  const int ny = g.ny, n1 = g.ny1, LD = rhs2_ld(n1);
  const size_t nw = (size_t)g.nw;
  C* sC = reinterpret_cast<C*>(smem_raw);   // 3 columns: cru
  C* sN = sC + 3 * LD;                      // 3 columns: nonlinear term
  C* sV = sN + 3 * LD;                      // 3 columns: new velocity
  const bool side = (mcru64 != nullptr);
  for (int q = 0; q < 3; ++q)
    for (int j = lane; j < n1; j += G) {
      sC[q * LD + j] = side ? mcru64[q * n1 + j] : cvt<C>(cru[q * n1 + j]);
      sN[q * LD + j] = cvt<C>(vel[q * n1 + j]);
    }
  __syncwarp();
  const double dt = sc->dt;
  const double coef = rkt.B(rk) * dt;
  const double vis_imp = rkt.D(rk) * (dt / re);
  const double rk_press = (rkt.Cc(rk) + rkt.D(rk)) * dt;
  const double vis_exp = rkt.Cc(rk) * (dt / re);
  // cv = cru + coef*cu (+ explicit viscous term on rk1; k = 0)
  C r[3][M];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int kd = (q == 1) ? RC_D2N : RC_D2H;
    const int nq = (q == 1) ? ny : n1;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = lane * M + i;
      C v = make_double2(0.0, 0.0);
      if (j < n1) {
        const C cr = sC[q * LD + j], nl = sN[q * LD + j];
        v = make_double2(cr.x - coef * nl.x, cr.y - coef * nl.y);
        if (rk == 1 && j < nq) v = cadd(v, cscale(vis_exp, d2c_t<double, M, G>(sC + q * LD, tbl, kd, i, lane, j, nq)));
      }
      r[q][i] = v;
    }
  }
  // constant mass flux pressure gradient (cu = -NL)
  double pg = sc->p_grad;
  if (fix_mass == 1) {
    double part = 0;
    for (int j = 1 + lane; j <= ny - 1; j += G) part += gd.dyh[j] * (-sN[j].x);
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    pg = -part + 0.5 * (d_um_dy[ny - 1] - d_um_dy[0]) / re;
  }
  const double cb = cos(beta) * rk_press * pg, sb = sin(beta) * rk_press * pg;
  {
    double a[M], b[M], c[M];
    C f[2][M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = lane * M + i;
      if (j == 0) {
        a[i] = 0; b[i] = 1; c[i] = 0;
        f[0][i] = cvt<C>(cbc_bot[0]); f[1][i] = cvt<C>(cbc_bot[2 * nw]);
      } else if (j == n1 - 1) {
        a[i] = 0; b[i] = 1; c[i] = 0;
        f[0][i] = cvt<C>(cbc_top[0]); f[1][i] = cvt<C>(cbc_top[2 * nw]);
      } else if (j < n1 - 1) {
        a[i] = -vis_imp * rc<double, M, G>(tbl, RC_D2H, i, lane);
        b[i] = -vis_imp * rc<double, M, G>(tbl, RC_D2H + 1, i, lane) + 1.0;
        c[i] = -vis_imp * rc<double, M, G>(tbl, RC_D2H + 2, i, lane);
        f[0][i] = make_double2(r[0][i].x - cb, r[0][i].y);
        f[1][i] = make_double2(r[2][i].x - sb, r[2][i].y);
      } else {
        a[i] = 0; b[i] = 1; c[i] = 0;
        f[0][i] = make_double2(0.0, 0.0); f[1][i] = make_double2(0.0, 0.0);
      }
    }
    tri_group_solve<double, M, G, 2>(a, b, c, f, lane);
    const C vb = cvt<C>(cbc_bot[nw]);
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = lane * M + i;
      if (j < n1) {
        sV[j] = f[0][i];
        sV[2 * LD + j] = f[1][i];
        sV[LD + j] = (j < ny) ? vb : make_double2(0.0, 0.0);
      }
    }
  }
  __syncwarp();
  // next-substep accumulator (PFC/pass2.f90:312-333) and the stores
  const double coef2 = (rk < 3) ? dt * rkt.A(rk + 1) : 0.0;
  const double vis_exp2 = (rk < 3) ? (dt / re) * rkt.Cc(rk + 1) : 0.0;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int kd = (q == 1) ? RC_D2N : RC_D2H;
    const int nq = (q == 1) ? ny : n1;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int j = lane * M + i;
      if (j >= n1) continue;
      const C cv = sV[q * LD + j];
      C v = cv;
      if (rk < 3) {
        const C nl = sN[q * LD + j];
        v = make_double2(cv.x - coef2 * nl.x, cv.y - coef2 * nl.y);
        if (j < nq) v = cadd(v, cscale(vis_exp2, d2c_t<double, M, G>(sV + q * LD, tbl, kd, i, lane, j, nq)));
      }
      cru[q * n1 + j] = cvt<CS>(v);
      if (side) mcru64[q * n1 + j] = v;
    }
  }
  for (int q = 0; q < 3; ++q)
    for (int j = lane; j < n1; j += G) {
      const C v = sV[q * LD + j];
      vel[q * n1 + j] = cvt<CS>(v);
      if (side) mvel64[q * n1 + j] = v;
    }
  for (int j = lane; j < n1; j += G) prs[j] = cvt<CS>(make_double2(0.0, 0.0));
  if (lane == 0) {
    sc->p_grad = pg;
    const double* dm = gd.dm;
    d_um_dy[0] = dm[0] * sV[0].x + dm[1] * sV[1].x + dm[2] * sV[2].x;
    d_um_dy[ny - 1] = dm[3] * sV[ny - 2].x + dm[4] * sV[ny - 1].x + dm[5] * sV[ny].x;
  }
  for (int j = 1 + lane; j <= ny - 2; j += G) d_um_dy[j] = gd.dn[j] * (sV[j + 1].x - sV[j].x);
}

template <typename S, int M>
__global__ void __launch_bounds__(32)
k_rhs_mean2(cplx_t<S>* __restrict__ vel, cplx_t<S>* __restrict__ cru, cplx_t<S>* __restrict__ prs,
            double2* __restrict__ mvel64, double2* __restrict__ mcru64, const cplx_t<S>* __restrict__ cbc_top,
            const cplx_t<S>* __restrict__ cbc_bot, Geom g, GridDev gd, DevScalars* __restrict__ sc,
            double* __restrict__ d_um_dy, RkTab rkt, int rk, double re, double beta, int fix_mass,
            const double* __restrict__ tbl) {
  k_rhs_mean2_body<S, M>(blockIdx, vel, cru, prs, mvel64, mcru64, cbc_top, cbc_bot, g, gd, sc, d_um_dy, rkt, rk, re,
                         beta, fix_mass, tbl);
}

template <int M> size_t rhs_mean2_smem(int n1) { return sizeof(double2) * 9 * (size_t)rhs2_ld(n1); }

template <typename T, int M, int G>
size_t rhs2_smem(int warps, int n1) {
  return sizeof(cplx_t<T>) * (size_t)warps * (32 / G) * 8 * rhs2_ld(n1);
}

// host: fills the lane-major coefficient table (RC_NUM*M*G values of T)
template <typename T>
void rhs2_fill_table(T* out, int M, int G, int ny, const double* dh, const double* dn, const double* d2h,
                     const double* d2n) {
  const int n1 = ny + 1;
  for (int kind = 0; kind < RC_NUM; ++kind)
    for (int i = 0; i < M; ++i)
      for (int gg = 0; gg < G; ++gg) {
        const int j = gg * M + i;
        double v = 0.0;
        if (kind < 3) v = (j < n1) ? d2h[3 * j + kind] : 0.0;
        else if (kind < 6) v = (j < ny) ? d2n[3 * j + kind - 3] : 0.0;
        else if (kind == RC_DN) v = (j < ny) ? dn[j] : 0.0;
        else if (kind == RC_DH) v = (j < n1) ? dh[j] : 0.0;
        else v = (j >= 1 && j - 1 < ny) ? dn[j - 1] : 0.0;
        out[(kind * M + i) * G + gg] = (T)v;
      }
}

}  // namespace cfd
