/*
 * chanflow_oracle.c -- CPU FP64 restatement of the reference channel-flow
 * solver's per-timestep hot path.  TEST INFRASTRUCTURE ONLY (the checker the
 * CUDA product is compared against); see chanflow_oracle.h for the pinning
 * story and the array layouts.  Every routine cites the Fortran it follows
 * (PFC = ParallelFortran-Code/ of the reference project).
 *
 * The plane loop of PFC/pass1.f90:65-83 is split into two parallel phases
 * (inverse transforms of every plane, then fluxes + forward transforms of
 * every plane); each flux is computed from the same operands with the same
 * expression as the sequential Fortran loop, so the values are unchanged.
 */
#include "chanflow_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* ------------------------------------------------------------------ */
/* RK3 constants: default-real (single precision) literals widened to FP64,
 * exactly as PFC/pass2.f90:14-18 initialises REAL(prec) PARAMETERs.      */
static const float rka_f[3] = {0.0f, -17.0f / 60.0f, -5.0f / 12.0f};
static const float rkb_f[3] = {8.0f / 15.0f, 5.0f / 12.0f, 3.0f / 4.0f};
static const float rkc_f[3] = {29.0f / 96.0f, -3.0f / 40.0f, 1.0f / 6.0f};
static const float rkd_f[3] = {37.0f / 160.0f, 5.0f / 24.0f, 1.0f / 6.0f};
#define RKA(i) ((double)rka_f[(i)-1])
#define RKB(i) ((double)rkb_f[(i)-1])
#define RKC(i) ((double)rkc_f[(i)-1])
#define RKD(i) ((double)rkd_f[(i)-1])

/* ------------------------------------------------------------------ */
/* Mixed-radix Stockham FFT (radix 4/2/3/5/generic).  Replaces FFTW's
 * dfftw_execute calls; sign -1 forward, +1 backward, unnormalised, the same
 * convention as FFTW (PFC/transform.f90:34-36).                          */
typedef struct {
  int n, npass;
  int radix[32];
  int ns[32];
  cplx *tw[2][32]; /* per sign: tw[s][p][r*ns+k] = exp(sign*2pi i k r/(ns*R)) */
} fft_plan;

#define MAX_PLANS 256
static fft_plan g_plans[MAX_PLANS];
static int g_nplans = 0;

static fft_plan *plan_build(int n) {
  for (int i = 0; i < g_nplans; i++)
    if (g_plans[i].n == n) return &g_plans[i];
  if (g_nplans >= MAX_PLANS) abort();   /* more distinct lengths than the cache holds */
  fft_plan *p = &g_plans[g_nplans++];
  memset(p, 0, sizeof(*p));
  p->n = n;
  int m = n, k = 0;
  while (m % 4 == 0) { p->radix[k++] = 4; m /= 4; }
  while (m % 2 == 0) { p->radix[k++] = 2; m /= 2; }
  while (m % 3 == 0) { p->radix[k++] = 3; m /= 3; }
  while (m % 5 == 0) { p->radix[k++] = 5; m /= 5; }
  for (int f = 7; m > 1; f++)
    while (m % f == 0) { p->radix[k++] = f; m /= f; }
  p->npass = k;
  int ns = 1;
  for (int q = 0; q < k; q++) {
    int R = p->radix[q];
    p->ns[q] = ns;
    for (int s = 0; s < 2; s++) {
      double sg = s == 0 ? -1.0 : 1.0;
      cplx *t = (cplx *)malloc(sizeof(cplx) * (size_t)R * ns);
      for (int r = 0; r < R; r++)
        for (int kk = 0; kk < ns; kk++) {
          double ang = sg * 2.0 * M_PI * (double)(kk * r) / (double)(ns * R);
          t[r * ns + kk] = cos(ang) + I * sin(ang);
        }
      p->tw[s][q] = t;
    }
    ns *= R;
  }
  return p;
}

static void dft_small(cplx *v, int R, double sg) {
  if (R == 2) {
    cplx a = v[0], b = v[1];
    v[0] = a + b; v[1] = a - b;
  } else if (R == 4) {
    cplx a = v[0], b = v[1], c = v[2], d = v[3];
    cplx t0 = a + c, t1 = a - c, t2 = b + d, t3 = (b - d) * (sg * I);
    v[0] = t0 + t2; v[2] = t0 - t2; v[1] = t1 + t3; v[3] = t1 - t3;
  } else if (R == 3) {
    cplx a = v[0], b = v[1], c = v[2];
    cplx t1 = b + c, t2 = a - 0.5 * t1, t3 = (sg * 0.86602540378443864676) * (b - c);
    v[0] = a + t1; v[1] = t2 + I * t3; v[2] = t2 - I * t3;
  } else {
    cplx w[64];
    for (int q = 0; q < R; q++) {
      cplx s = 0;
      for (int r = 0; r < R; r++) {
        double ang = sg * 2.0 * M_PI * (double)((q * r) % R) / (double)R;
        s += v[r] * (cos(ang) + I * sin(ang));
      }
      w[q] = s;
    }
    for (int q = 0; q < R; q++) v[q] = w[q];
  }
}

/* out may alias in; work needs 2n entries */
static void fft_exec(const fft_plan *p, int sign, const cplx *in, cplx *out,
                     cplx *work) {
  int n = p->n, s = sign < 0 ? 0 : 1;
  double sg = sign < 0 ? -1.0 : 1.0;
  cplx *a = work, *b = work + n;
  memcpy(a, in, sizeof(cplx) * n);
  for (int q = 0; q < p->npass; q++) {
    int R = p->radix[q], ns = p->ns[q], nr = n / R;
    const cplx *t = p->tw[s][q];
    for (int j = 0; j < nr; j++) {
      cplx v[64];
      int k = j % ns;
      for (int r = 0; r < R; r++) v[r] = a[j + r * nr] * t[r * ns + k];
      dft_small(v, R, sg);
      int d = (j / ns) * ns * R + k;
      for (int r = 0; r < R; r++) b[d + r * ns] = v[r];
    }
    cplx *tmp = a; a = b; b = tmp;
  }
  memcpy(out, a, sizeof(cplx) * n);
}

void orc_fft(int n, int sign, const double complex *in, double complex *out) {
  fft_plan *p;
#pragma omp critical(orc_plan)
  p = plan_build(n);
  cplx *w = (cplx *)malloc(sizeof(cplx) * 2 * n);
  fft_exec(p, sign, in, out, w);
  free(w);
}

/* real-to-half-complex of length n: X_k, k = 0..n/2 (FFTW r2c) */
static void rfft_fwd(const fft_plan *p, const double *x, cplx *X, cplx *work) {
  int n = p->n;
  cplx *buf = work + 2 * n;
  for (int i = 0; i < n; i++) buf[i] = x[i];
  fft_exec(p, -1, buf, buf, work);
  for (int k = 0; k <= n / 2; k++) X[k] = buf[k];
}

/* half-complex-to-real of length n (FFTW c2r, unnormalised): the imaginary
 * parts of the DC and Nyquist inputs do not contribute.                   */
static void rfft_inv(const fft_plan *p, const cplx *X, double *x, cplx *work) {
  int n = p->n;
  cplx *buf = work + 2 * n;
  buf[0] = creal(X[0]);
  for (int k = 1; k < n / 2; k++) {
    buf[k] = X[k];
    buf[n - k] = conj(X[k]);
  }
  if (n % 2 == 0) buf[n / 2] = creal(X[n / 2]);
  else { buf[n / 2] = X[n / 2]; buf[n - n / 2] = conj(X[n / 2]); }
  fft_exec(p, +1, buf, buf, work);
  for (int i = 0; i < n; i++) x[i] = creal(buf[i]);
}

/* ------------------------------------------------------------------ */
struct orc_ctx {
  orc_params p;
  int nxh;                       /* nx/2+1 */
  double pi;
  /* grid, PFC/gridparms.f90 (1-based in the comments, 0-based here) */
  double *y, *yh, *hh, *dh, *hn, *dn, *iu, *d2h, *d2n, *dyh, *dy;
  double dm[12], d2m[8];
  double *kx, *kz, *k2;          /* kx(nxh), kz(nz), k2(nz,nxh) */
  double *buffer, *target_inflow, *baseflow, *d_um_dy, *cfl;
  double *xcoord, *zcoord;
  /* state */
  cplx *data1, *data2, *data4, *cbc_top, *cbc_bot;
  double t_total, dt, p_grad;
  int step, rk_step, status;
  fft_plan *px2, *pz2, *pxs, *pzs;
  /* crossflow jet (PFC/pass2.f90:37-44, 423-673) */
  int crossflow;
  orc_jet jet;
  long long jet_calls;
};

#define D1(c, z, x, j, q) (c)->data1[(z) + (size_t)(c)->p.nz * ((x) + (size_t)(c)->nxh * ((j) + (size_t)((c)->p.ny + 1) * (q)))]
#define D2(c, j, q, z, x) (c)->data2[(j) + (size_t)((c)->p.ny + 1) * ((q) + 3 * ((z) + (size_t)(c)->p.nz * (x)))]
#define D4(c, j, z, x) (c)->data4[(j) + (size_t)((c)->p.ny + 1) * ((z) + (size_t)(c)->p.nz * (x))]
/* Fortran-index helpers for grid vectors: F(v,i) = v(i) */
#define F(v, i) ((v)[(i)-1])
#define DM(i, j) c->dm[((i)-1) + 3 * ((j)-1)]
#define D2H(i, j) c->d2h[((i)-1) + 3 * ((j)-1)]
#define D2N(i, j) c->d2n[((i)-1) + 3 * ((j)-1)]
#define IU(i, j) c->iu[((i)-1) + 2 * ((j)-1)]

static void *xcalloc(size_t n, size_t s) {
  void *p = calloc(n ? n : 1, s);
  return p;
}

/* DEFINE_COORDINATES, PFC/setup.f90:541-754 (channel branch) */
static void define_coordinates(orc_ctx *c) {
  int ny = c->p.ny, nx = c->p.nx, nz = c->p.nz;
  const double zero = 0.0, half = 0.5, one = 1.0, two = 2.0, three = 3.0;
  double STRETCH = c->p.stretch;
  c->xcoord = xcalloc(nx + 1, sizeof(double));
  c->zcoord = xcalloc(nz + 1, sizeof(double));
  for (int x = 1; x <= nx + 1; x++) F(c->xcoord, x) = (double)(x - 1) * c->p.lx / (double)nx;
  for (int z = 1; z <= nz + 1; z++) F(c->zcoord, z) = (double)(z - 1) * c->p.lz / (double)nz;
  for (int pl = 1; pl <= ny; pl++) {
    double xi = two * (double)(pl - 1) / (double)(ny - 1) - one;
    F(c->y, pl) = tanh(STRETCH * xi) / tanh(STRETCH);
  }
  if (c->p.uniform_grid) {           /* which_test == 6, PFC/setup.f90:608-614 */
    F(c->y, 1) = -half;
    for (int pl = 2; pl <= ny - 1; pl++) F(c->y, pl) = F(c->y, 1) + (double)(pl - 1) / (double)(ny - 1);
    F(c->y, ny) = half;
  }
  F(c->yh, 1) = F(c->y, 1);
  for (int j = 2; j <= ny; j++) F(c->yh, j) = half * (F(c->y, j - 1) + F(c->y, j));
  F(c->yh, ny + 1) = F(c->y, ny);

  F(c->hh, 1) = F(c->y, 2) - F(c->y, 1);
  for (int j = 2; j <= ny; j++) F(c->hh, j) = F(c->y, j) - F(c->y, j - 1);
  F(c->hh, ny + 1) = F(c->y, ny) - F(c->y, ny - 1);
  for (int j = 1; j <= ny + 1; j++) F(c->dh, j) = one / F(c->hh, j);
  for (int j = 1; j <= ny; j++) F(c->hn, j) = F(c->yh, j + 1) - F(c->yh, j);
  for (int j = 1; j <= ny; j++) F(c->dn, j) = one / F(c->hn, j);
  for (int j = 1; j <= ny; j++) {
    IU(1, j) = half * F(c->hh, j) / F(c->hn, j);
    IU(2, j) = half * F(c->hh, j + 1) / F(c->hn, j);
  }
  double *HN = c->hn, *DN = c->dn, *DH = c->dh, *Y = c->y, *YH = c->yh;
  DM(1, 1) = -(F(DN, 1) * (two * F(HN, 1) + F(HN, 2)) / (F(HN, 1) + F(HN, 2)));
  DM(2, 1) = F(DN, 1) * F(DN, 2) * (F(HN, 1) + F(HN, 2));
  DM(3, 1) = -(F(DN, 2) * F(HN, 1) / (F(HN, 1) + F(HN, 2)));
  DM(1, 2) = F(DN, ny - 1) * F(HN, ny) / (F(HN, ny - 1) + F(HN, ny));
  DM(2, 2) = -(F(DN, ny) * F(DN, ny - 1) * (F(HN, ny) + F(HN, ny - 1)));
  DM(3, 2) = F(DN, ny) * (two * F(HN, ny) + F(HN, ny - 1)) / (F(HN, ny) + F(HN, ny - 1));
  DM(1, 3) = (F(Y, 1) - F(Y, 2) + F(Y, 1) - F(Y, 3)) / ((F(Y, 1) - F(Y, 2)) * (F(Y, 1) - F(Y, 3)));
  DM(2, 3) = (F(Y, 1) - F(Y, 3)) / ((F(Y, 2) - F(Y, 1)) * (F(Y, 2) - F(Y, 3)));
  DM(3, 3) = (F(Y, 1) - F(Y, 2)) / ((F(Y, 3) - F(Y, 1)) * (F(Y, 3) - F(Y, 2)));
  DM(1, 4) = (F(Y, ny) - F(Y, ny - 1)) / ((F(Y, ny - 2) - F(Y, ny)) * (F(Y, ny - 2) - F(Y, ny - 1)));
  DM(2, 4) = (F(Y, ny) - F(Y, ny - 2)) / ((F(Y, ny - 1) - F(Y, ny)) * (F(Y, ny - 1) - F(Y, ny - 2)));
  DM(3, 4) = (F(Y, ny) - F(Y, ny - 1) + F(Y, ny) - F(Y, ny - 2)) / ((F(Y, ny) - F(Y, ny - 1)) * (F(Y, ny) - F(Y, ny - 2)));
  {
    double t1 = F(YH, 1) - F(YH, 2), t2 = F(YH, 1) - F(YH, 3), t3 = F(YH, 1) - F(YH, 4);
    c->d2m[0] = two * (t1 + t2 + t3) / (t1 * t2 * t3);
    c->d2m[1] = two * (t2 + t3) / ((F(YH, 2) - F(YH, 1)) * (F(YH, 2) - F(YH, 3)) * (F(YH, 2) - F(YH, 4)));
    c->d2m[2] = two * (t1 + t3) / ((F(YH, 3) - F(YH, 1)) * (F(YH, 3) - F(YH, 2)) * (F(YH, 3) - F(YH, 4)));
    c->d2m[3] = two * (t1 + t2) / ((F(YH, 4) - F(YH, 1)) * (F(YH, 4) - F(YH, 2)) * (F(YH, 4) - F(YH, 3)));
  }
  (void)three;
  for (int pl = 2; pl <= ny - 1; pl++) {
    D2N(1, pl) = F(DN, pl) * F(DH, pl);
    D2N(2, pl) = -(F(DN, pl) * F(DH, pl)) - F(DN, pl) * F(DH, pl + 1);
    D2N(3, pl) = F(DN, pl) * F(DH, pl + 1);
    D2H(1, pl) = F(DH, pl) * F(DN, pl - 1);
    D2H(2, pl) = -(F(DH, pl) * F(DN, pl - 1)) - F(DH, pl) * F(DN, pl);
    D2H(3, pl) = F(DH, pl) * F(DN, pl);
  }
  D2H(1, 2) = -(F(DH, 2) * DM(1, 1));
  D2H(2, 2) = -(F(DH, 2) * F(DN, 2)) - F(DH, 2) * DM(2, 1);
  D2H(3, 2) = F(DH, 2) * F(DN, 2) - F(DH, 2) * DM(3, 1);
  D2H(1, ny) = F(DH, ny) * F(DN, ny - 1) + F(DH, ny) * DM(1, 2);
  D2H(2, ny) = -(F(DH, ny) * F(DN, ny - 1)) + F(DH, ny) * DM(2, 2);
  D2H(3, ny) = F(DH, ny) * DM(3, 2);
  for (int i = 1; i <= 3; i++) {
    D2H(i, 1) = D2H(i, 2);
    D2N(i, 1) = D2N(i, 2);
    D2N(i, ny) = D2N(i, ny - 1);
    D2H(i, ny + 1) = D2H(i, ny);
  }
  F(c->dyh, 1) = zero;
  for (int j = 2; j <= ny; j++) F(c->dyh, j) = F(c->hh, j);
  F(c->dyh, ny + 1) = zero;
  F(c->dy, 1) = half * F(c->hh, 2);
  for (int j = 2; j <= ny - 1; j++) F(c->dy, j) = half * (F(c->hh, j) + F(c->hh, j + 1));
  F(c->dy, ny) = half * F(c->hh, ny);
  F(c->dy, ny + 1) = zero;
}

/* wavenumbers, PFC/setup.f90:1439-1466 */
static void define_wavenumbers(orc_ctx *c) {
  int nz = c->p.nz, nxh = c->nxh;
  double pi = c->pi;
  for (int x = 1; x <= nxh; x++) F(c->kx, x) = (double)(x - 1) * 2.0 * pi / c->p.lx;
  for (int z = 1; z <= nz / 2 + 1; z++) F(c->kz, z) = (double)(z - 1) * 2.0 * pi / c->p.lz;
  for (int z = nz; z >= nz / 2 + 2; z--) F(c->kz, z) = -F(c->kz, nz + 2 - z);
  for (int x = 0; x < nxh; x++)
    for (int z = 0; z < nz; z++) c->k2[z + nz * x] = c->kx[x] * c->kx[x] + c->kz[z] * c->kz[z];
}

orc_ctx *orc_create(const orc_params *p) {
  orc_ctx *c = (orc_ctx *)xcalloc(1, sizeof(orc_ctx));
  c->p = *p;
  int ny = p->ny, nz = p->nz, nx2 = p->nx2, nz2 = p->nz2;
  c->nxh = p->nx / 2 + 1;
  c->pi = atan2(0.0, -1.0);
#ifdef _OPENMP
  if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
  c->y = xcalloc(ny, 8); c->yh = xcalloc(ny + 1, 8); c->hh = xcalloc(ny + 1, 8);
  c->dh = xcalloc(ny + 1, 8); c->hn = xcalloc(ny, 8); c->dn = xcalloc(ny, 8);
  c->iu = xcalloc(2 * ny, 8); c->d2h = xcalloc(3 * (ny + 1), 8); c->d2n = xcalloc(3 * ny, 8);
  c->dyh = xcalloc(ny + 1, 8); c->dy = xcalloc(ny + 1, 8);
  c->kx = xcalloc(c->nxh, 8); c->kz = xcalloc(nz, 8); c->k2 = xcalloc((size_t)nz * c->nxh, 8);
  c->buffer = xcalloc((size_t)nx2 * nz2, 8);
  c->target_inflow = xcalloc(3 * (ny + 1), 8);
  c->baseflow = xcalloc(3 * (ny + 1), 8);
  c->d_um_dy = xcalloc(ny, 8);
  c->cfl = xcalloc(ny + 1, 8);
  size_t nf = (size_t)nz * c->nxh * (ny + 1);
  c->data1 = xcalloc(3 * nf, sizeof(cplx));
  c->data2 = xcalloc(3 * nf, sizeof(cplx));
  c->data4 = xcalloc(nf, sizeof(cplx));
  c->cbc_top = xcalloc(3 * (size_t)nz * c->nxh, sizeof(cplx));
  c->cbc_bot = xcalloc(3 * (size_t)nz * c->nxh, sizeof(cplx));
  define_coordinates(c);
  define_wavenumbers(c);
  c->dt = p->dt;
  c->p_grad = -2.0 / p->re;     /* PFC/setup.f90:1384 */
  c->t_total = 0.0;
  c->step = 0; c->rk_step = 1;
#pragma omp critical(orc_plan)
  {
    c->px2 = plan_build(nx2); c->pz2 = plan_build(nz2);
    c->pxs = plan_build(p->nx); c->pzs = plan_build(nz);
  }
  return c;
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  double *v[] = {c->y, c->yh, c->hh, c->dh, c->hn, c->dn, c->iu, c->d2h, c->d2n, c->dyh, c->dy,
                 c->kx, c->kz, c->k2, c->buffer, c->target_inflow, c->baseflow, c->d_um_dy,
                 c->cfl, c->xcoord, c->zcoord};
  for (size_t i = 0; i < sizeof(v) / sizeof(v[0]); i++) free(v[i]);
  free(c->data1); free(c->data2); free(c->data4); free(c->cbc_top); free(c->cbc_bot);
  free(c);
}

double *orc_grid(orc_ctx *c, const char *n, int *len) {
  int ny = c->p.ny;
#define G(name, ptr, l) if (!strcmp(n, name)) { *len = (l); return (ptr); }
  G("y", c->y, ny) G("yh", c->yh, ny + 1) G("hh", c->hh, ny + 1) G("dh", c->dh, ny + 1)
  G("hn", c->hn, ny) G("dn", c->dn, ny) G("iu", c->iu, 2 * ny) G("d2h", c->d2h, 3 * (ny + 1))
  G("d2n", c->d2n, 3 * ny) G("dyh", c->dyh, ny + 1) G("dy", c->dy, ny + 1) G("dm", c->dm, 12)
  G("d2m", c->d2m, 8) G("kx", c->kx, c->nxh) G("kz", c->kz, c->p.nz)
  G("k2", c->k2, c->p.nz * c->nxh) G("xcoord", c->xcoord, c->p.nx + 1) G("zcoord", c->zcoord, c->p.nz + 1)
#undef G
  *len = 0;
  return NULL;
}
double complex *orc_data1(orc_ctx *c) { return c->data1; }
double complex *orc_data2(orc_ctx *c) { return c->data2; }
double complex *orc_data4(orc_ctx *c) { return c->data4; }
double complex *orc_cbc_top(orc_ctx *c) { return c->cbc_top; }
double complex *orc_cbc_bot(orc_ctx *c) { return c->cbc_bot; }
double *orc_buffer(orc_ctx *c) { return c->buffer; }
double *orc_target_inflow(orc_ctx *c) { return c->target_inflow; }
double *orc_baseflow(orc_ctx *c) { return c->baseflow; }
double *orc_d_um_dy(orc_ctx *c) { return c->d_um_dy; }
double *orc_cfl(orc_ctx *c) { return c->cfl; }
void orc_get_scalars(orc_ctx *c, double *t, double *dt, double *pg) {
  if (t) *t = c->t_total;
  if (dt) *dt = c->dt;
  if (pg) *pg = c->p_grad;
}
void orc_set_scalars(orc_ctx *c, double t, double dt, double pg) {
  c->t_total = t; c->dt = dt; c->p_grad = pg;
}
void orc_set_step(orc_ctx *c, int step, int rk) { c->step = step; c->rk_step = rk; }
int orc_status(orc_ctx *c) { return c->status; }

/* ------------------------------------------------------------------ */
/* xz_fft_complex_to_real_parallel, PFC/transform.f90:339-409 (one rank) */
static void xz_c2r_w(orc_ctx *c, const cplx *cd, double *data, cplx *work) {
  int nz = c->p.nz, nz2 = c->p.nz2, nx = c->p.nx, nx2 = c->p.nx2, nxh = c->nxh;
  int nx2h = nx2 / 2 + 1;
  cplx *Q = work;                      /* (nz2, nxh) */
  cplx *X = Q + (size_t)nz2 * nxh;     /* nx2h */
  cplx *fw = X + nx2h;                 /* fft work 3*max(n) */
  for (int x = 0; x < nxh; x++) {
    cplx *P = Q + (size_t)nz2 * x;
    const cplx *col = cd + (size_t)nz * x;
    if (nz2 > nz) {
      for (int m = 0; m < nz / 2; m++) P[m] = col[m];
      P[nz / 2] = 0.5 * col[nz / 2];
      for (int m = nz / 2 + 1; m < nz2 - nz / 2; m++) P[m] = 0;
      P[nz2 - nz / 2] = 0.5 * conj(col[nz / 2]);
      for (int m = nz2 - nz / 2 + 1; m < nz2; m++) P[m] = col[m - (nz2 - nz)];
      if (nx2 > nx && x == nxh - 1)
        for (int m = 0; m < nz2; m++) P[m] = 0.5 * P[m];
    } else {
      for (int m = 0; m <= nz / 2; m++) P[m] = col[m];
      for (int m = nz / 2 + 1; m <= nz2 - nz / 2; m++) P[m] = 0;
      for (int m = nz2 - nz / 2 + 1; m < nz2; m++) P[m] = col[m - (nz2 - nz)];
    }
    fft_exec(c->pz2, +1, P, P, fw);
  }
  for (int z = 0; z < nz2; z++) {
    for (int k = 0; k < nx2h; k++) X[k] = k < nxh ? Q[z + (size_t)nz2 * k] : 0;
    rfft_inv(c->px2, X, data + (size_t)nx2 * z, fw);
  }
}

static size_t xz_work_len(orc_ctx *c) {
  int n = c->p.nx2 > c->p.nz2 ? c->p.nx2 : c->p.nz2;
  if (c->p.nx > n) n = c->p.nx;
  if (c->p.nz > n) n = c->p.nz;
  return (size_t)2 * c->p.nz2 * c->nxh + (size_t)c->p.nx2 + 8 * (size_t)n + 64;
}

void orc_xz_c2r(orc_ctx *c, const double complex *cd, double *data) {
  cplx *w = malloc(sizeof(cplx) * xz_work_len(c));
  xz_c2r_w(c, cd, data, w);
  free(w);
}

/* forward x r2c of every z row: R(x, z) for x < nxh, layout (nz2, nxh) by kx column */
static void x_r2c_rows(orc_ctx *c, const double *data, cplx *R, cplx *fw) {
  int nz2 = c->p.nz2, nx2 = c->p.nx2, nxh = c->nxh;
  cplx *X = fw + 3 * (size_t)(nx2 > nz2 ? nx2 : nz2) + 8;
  for (int z = 0; z < nz2; z++) {
    rfft_fwd(c->px2, data + (size_t)nx2 * z, X, fw);
    for (int k = 0; k < nxh; k++) R[z + (size_t)nz2 * k] = X[k];
  }
}

/* xz_fft_real_to_complex_parallel, PFC/transform.f90:258-335 */
static void xz_r2c_w(orc_ctx *c, const double *data, cplx *cd, cplx *work) {
  int nz = c->p.nz, nz2 = c->p.nz2, nx2 = c->p.nx2, nxh = c->nxh;
  cplx *R = work;
  cplx *fw = R + (size_t)nz2 * nxh;
  x_r2c_rows(c, data, R, fw);
  double scale = 1.0 / (double)(nx2 * nz2);
  int off = nz2 - nz;
  for (int x = 0; x < nxh; x++) {
    cplx *S = R + (size_t)nz2 * x;
    fft_exec(c->pz2, -1, S, S, fw);
    cplx *col = cd + (size_t)nz * x;
    for (int m = 0; m < nz / 2; m++) col[m] = scale * S[m];
    col[nz / 2] = scale * (S[nz / 2] + conj(S[off + nz / 2]));
    for (int m = nz / 2 + 1; m < nz; m++) col[m] = scale * S[off + m];
  }
  for (int m = 0; m < nz; m++) cd[m + (size_t)nz * (nxh - 1)] = 2.0 * cd[m + (size_t)nz * (nxh - 1)];
}

void orc_xz_r2c(orc_ctx *c, const double *data, double complex *cd) {
  cplx *w = malloc(sizeof(cplx) * xz_work_len(c) * 2);
  xz_r2c_w(c, data, cd, w);
  free(w);
}

/* parallel_divergence_of_fluxes, PFC/transform.f90:573-690 */
static void div_fluxes_w(orc_ctx *c, const double *dx, const double *dy,
                         const double *dz, cplx *cd, cplx *work) {
  int nz = c->p.nz, nz2 = c->p.nz2, nx2 = c->p.nx2, nxh = c->nxh;
  size_t wl = xz_work_len(c);
  cplx *Ry = work, *Rx = work + (size_t)nz2 * nxh;
  cplx *fw = Rx + (size_t)nz2 * nxh;
  x_r2c_rows(c, dy, Ry, fw);
  x_r2c_rows(c, dx, Rx, fw);
  for (int x = 0; x < nxh; x++) {
    cplx ikx = I * c->kx[x];
    cplx *A = Ry + (size_t)nz2 * x, *B = Rx + (size_t)nz2 * x;
    for (int m = 0; m < nz2; m++) A[m] = A[m] + ikx * B[m];
    fft_exec(c->pz2, -1, A, A, fw);
  }
  xz_r2c_w(c, dz, cd, fw + wl);
  double scale = 1.0 / (double)(nx2 * nz2);
  int off = nz2 - nz;
  for (int x = 0; x < nxh; x++) {
    double s = (x == nxh - 1) ? 2.0 * scale : scale;
    cplx *T = Ry + (size_t)nz2 * x, *col = cd + (size_t)nz * x;
    for (int m = 0; m < nz / 2; m++) col[m] = (I * c->kz[m]) * col[m] + s * T[m];
    col[nz / 2] = (I * c->kz[nz / 2]) * col[nz / 2] + s * (T[nz / 2] + conj(T[off + nz / 2]));
    for (int m = nz / 2 + 1; m < nz; m++) col[m] = (I * c->kz[m]) * col[m] + s * T[off + m];
  }
}

void orc_div_fluxes(orc_ctx *c, const double *dx, const double *dy, const double *dz,
                    double complex *cd) {
  cplx *w = malloc(sizeof(cplx) * xz_work_len(c) * 4);
  div_fluxes_w(c, dx, dy, dz, cd, w);
  free(w);
}

/* small_fft_real_to_complex / small_fft_complex_to_real,
 * PFC/transform.f90:1071-1142 and :950-1000 (nx x nz grid, no dealiasing) */
void orc_small_r2c(orc_ctx *c, const double *data, double complex *cd) {
  int nx = c->p.nx, nz = c->p.nz, nxh = c->nxh;
  int n = nx > nz ? nx : nz;
  cplx *R = malloc(sizeof(cplx) * ((size_t)nz * nxh + 8 * n + 64));
  cplx *fw = R + (size_t)nz * nxh;
  cplx *X = fw + 3 * n + 8;
  for (int z = 0; z < nz; z++) {
    rfft_fwd(c->pxs, data + (size_t)nx * z, X, fw);
    for (int k = 0; k < nxh; k++) R[z + (size_t)nz * k] = X[k];
  }
  double scale = 1.0 / (double)(nx * nz);
  for (int x = 0; x < nxh; x++) {
    cplx *S = R + (size_t)nz * x;
    fft_exec(c->pzs, -1, S, S, fw);
    for (int m = 0; m < nz; m++) cd[m + (size_t)nz * x] = scale * S[m];
  }
  free(R);
}

void orc_small_c2r(orc_ctx *c, const double complex *cd, double *data) {
  int nx = c->p.nx, nz = c->p.nz, nxh = c->nxh;
  int n = nx > nz ? nx : nz;
  cplx *Q = malloc(sizeof(cplx) * ((size_t)nz * nxh + 8 * n + 64));
  cplx *fw = Q + (size_t)nz * nxh;
  cplx *X = fw + 3 * n + 8;
  for (int x = 0; x < nxh; x++) fft_exec(c->pzs, +1, cd + (size_t)nz * x, Q + (size_t)nz * x, fw);
  for (int z = 0; z < nz; z++) {
    for (int k = 0; k < nxh; k++) X[k] = Q[z + (size_t)nz * k];
    rfft_inv(c->pxs, X, data + (size_t)nx * z, fw);
  }
  free(Q);
}

/* ------------------------------------------------------------------ */
/* nonlinear, PFC/pass1.f90:26-124 with compute_wall_parallel_flux (:128-173),
 * compute_wall_normal_flux (:175-200) and check_cfl (:202-250).
 * linearized != 0 follows nonlinear_linearized, PFC/pass1_linearized.f90:135-344
 * and its check_cfl (:456-508), with a baseflow uniform in x and z.        */
static void nonlinear_impl(orc_ctx *c, int linearized) {
  int ny = c->p.ny, nz = c->p.nz, nx2 = c->p.nx2, nz2 = c->p.nz2, nxh = c->nxh;
  size_t np = (size_t)nx2 * nz2, nfp = (size_t)nz * nxh;
  const double half = 0.5, two = 2.0;
  /* phys[q][j-1] for plane j = 1..ny+1 */
  double *phys = malloc(sizeof(double) * np * 3 * (ny + 1));
#define PH(q, j) (phys + np * ((size_t)(q) * (ny + 1) + ((j)-1)))
  size_t wl = xz_work_len(c);
#pragma omp parallel
  {
    cplx *w = malloc(sizeof(cplx) * wl);
#pragma omp for schedule(dynamic)
    for (int t = 0; t < 3 * (ny + 1); t++) {
      int q = t / (ny + 1), j = t % (ny + 1) + 1;
      if (q == 1 && j == ny + 1) continue;   /* v never transformed at ny+1 */
      xz_c2r_w(c, &D1(c, 0, 0, j - 1, q), PH(q, j), w);
    }
    free(w);
  }
  cplx *nl = malloc(sizeof(cplx) * nfp * 3 * (ny + 1));
#define NL(q, j) (nl + nfp * ((size_t)(q) * (ny + 1) + ((j)-1)))
  double *B = c->baseflow; /* (ny+1,3) */
#define BF(j, q) B[((j)-1) + (ny + 1) * (q)]
  int docfl = (c->rk_step == 1);
  double *tgt = c->target_inflow;
#define TGT(j, q) tgt[((j)-1) + (ny + 1) * (q)]
#pragma omp parallel
  {
    double *f = malloc(sizeof(double) * np * 9);
    double *fpu = f, *fpu0 = f + np, *dyu = f + 2 * np, *xf = f + 3 * np, *zf = f + 4 * np;
    double *fpw = f + 5 * np, *fpw0 = f + 6 * np, *fp = f + 7 * np, *fp0 = f + 8 * np;
    cplx *w = malloc(sizeof(cplx) * wl * 4);
#pragma omp for schedule(dynamic)
    for (int k = 2; k <= ny; k++) {
      double *U = PH(0, k), *V = PH(1, k), *W = PH(2, k);
      double *Up = PH(0, k + 1), *Wp = PH(2, k + 1);
      double *Vp = (k < ny) ? PH(1, k + 1) : V;  /* up(:,:,2) = u(:,:,2) at ny */
      double *Um = PH(0, k - 1), *Vm = PH(1, k - 1), *Wm = PH(2, k - 1);
      double dhk = F(c->dh, k);
      if (!linearized) {
        for (size_t i = 0; i < np; i++) {
          if (k == 2) { fpu0[i] = Vm[i] * Um[i]; fpw0[i] = Vm[i] * Wm[i]; }
          else { fpu0[i] = Vm[i] * half * (Um[i] + U[i]); fpw0[i] = Vm[i] * half * (Wm[i] + W[i]); }
          if (k < ny) { fpu[i] = V[i] * half * (U[i] + Up[i]); fpw[i] = V[i] * half * (W[i] + Wp[i]); }
          else { fpu[i] = V[i] * Up[i]; fpw[i] = V[i] * Wp[i]; }
        }
      } else {
        for (size_t i = 0; i < np; i++) {
          if (k == 2) {
            fpu0[i] = BF(1, 1) * Um[i] + Vm[i] * BF(1, 0);
            fpw0[i] = BF(1, 1) * Wm[i] + Vm[i] * BF(1, 2);
          } else {
            fpu0[i] = BF(k - 1, 1) * half * (Um[i] + U[i]) + Vm[i] * half * (BF(k - 1, 0) + BF(k, 0));
            fpw0[i] = BF(k - 1, 1) * half * (Wm[i] + W[i]) + Vm[i] * half * (BF(k - 1, 2) + BF(k, 2));
          }
          if (k < ny) {
            fpu[i] = BF(k, 1) * half * (U[i] + Up[i]) + V[i] * half * (BF(k, 0) + BF(k + 1, 0));
            fpw[i] = BF(k, 1) * half * (W[i] + Wp[i]) + V[i] * half * (BF(k, 2) + BF(k + 1, 2));
          } else {
            fpu[i] = BF(ny, 1) * Up[i] + V[i] * BF(ny + 1, 0);
            fpw[i] = BF(ny, 1) * Wp[i] + V[i] * BF(ny + 1, 2);
          }
        }
      }
      /* u equation */
      for (size_t i = 0; i < np; i++) {
        dyu[i] = dhk * (fpu[i] - fpu0[i]) + c->buffer[i] * (U[i] - TGT(k, 0));
        if (!linearized) { xf[i] = U[i] * U[i]; zf[i] = W[i] * U[i]; }
        else { xf[i] = two * BF(k, 0) * U[i]; zf[i] = BF(k, 2) * U[i] + W[i] * BF(k, 0); }
      }
      div_fluxes_w(c, xf, dyu, zf, NL(0, k), w);
      /* w equation */
      for (size_t i = 0; i < np; i++) {
        dyu[i] = dhk * (fpw[i] - fpw0[i]) + c->buffer[i] * (W[i] - TGT(k, 2));
        if (!linearized) { xf[i] = U[i] * W[i]; zf[i] = W[i] * W[i]; }
        else { xf[i] = BF(k, 2) * U[i] + W[i] * BF(k, 0); zf[i] = two * BF(k, 2) * W[i]; }
      }
      div_fluxes_w(c, xf, dyu, zf, NL(2, k), w);
      /* v equation (planes 2..ny-1) */
      if (k <= ny - 1) {
        double dnk = F(c->dn, k), iu1 = IU(1, k), iu2 = IU(2, k);
        for (size_t i = 0; i < np; i++) {
          if (!linearized) {
            double t0 = half * (Vm[i] + V[i]);
            double t1 = half * (V[i] + Vp[i]);
            fp0[i] = t0 * t0;
            fp[i] = t1 * t1;
          } else {
            double t0 = half * (Vm[i] + V[i]), b0 = half * (BF(k - 1, 1) + BF(k, 1));
            double t1 = half * (V[i] + Vp[i]), b1 = half * (BF(k, 1) + BF(k + 1, 1));
            fp0[i] = two * t0 * b0;
            fp[i] = two * t1 * b1;
          }
          dyu[i] = dnk * (fp[i] - fp0[i]) + c->buffer[i] * (V[i] - TGT(k, 1));
          if (!linearized) {
            xf[i] = V[i] * (iu1 * U[i] + iu2 * Up[i]);
            zf[i] = V[i] * (iu1 * W[i] + iu2 * Wp[i]);
          } else {
            xf[i] = BF(k, 1) * (iu1 * U[i] + iu2 * Up[i]) + V[i] * (iu1 * BF(k, 0) + iu2 * BF(k + 1, 0));
            zf[i] = BF(k, 1) * (iu1 * W[i] + iu2 * Wp[i]) + V[i] * (iu1 * BF(k, 2) + iu2 * BF(k + 1, 2));
          }
        }
        div_fluxes_w(c, xf, dyu, zf, NL(1, k), w);
      }
      if (docfl) {
        double ma = 0, mb = 0, mc = 0;
        for (size_t i = 0; i < np; i++) {
          double a = fabs(U[i] + Up[i]), b = fabs(V[i]), d = fabs(W[i] + Wp[i]);
          if (a > ma) ma = a;
          if (b > mb) mb = b;
          if (d > mc) mc = d;
        }
        if (linearized) {
          double ba = fabs(BF(k, 0) + BF(k + 1, 0)), bb = fabs(BF(k, 1)), bc = fabs(BF(k, 2) + BF(k + 1, 2));
          if (ba > ma) ma = ba;
          if (bb > mb) mb = bb;
          if (bc > mc) mc = bc;
        }
        double hmin = F(c->hn, k) < F(c->hn, k - 1) ? F(c->hn, k) : F(c->hn, k - 1);
        double ta = half * ma * (double)c->p.nx / (0.55 * c->p.lx);
        double tb = mb / (1.73 * hmin);
        double tc = half * mc * (double)c->p.nz / (0.55 * c->p.lz);
        c->cfl[k - 1] = (ta + tb + tc) * c->dt;
      }
    }
    free(f);
    free(w);
  }
  /* write back: NL for planes 2..ny (u,w), 2..ny-1 (v); zero the rest */
  for (int q = 0; q < 3; q++)
    for (int j = 1; j <= ny + 1; j++) {
      cplx *dst = &D1(c, 0, 0, j - 1, q);
      int valid = (j >= 2 && j <= ny) && !(q == 1 && j == ny);
      if (valid) memcpy(dst, NL(q, j), sizeof(cplx) * nfp);
      else memset(dst, 0, sizeof(cplx) * nfp);
    }
  if (docfl) {
    for (int k = 2; k <= ny; k++) {
      double cf = c->cfl[k - 1];
      if (c->p.dt_flag == 1 ? (cf >= 3.0e2) : (cf >= 1.15)) {
        c->status = c->p.dt_flag == 1 ? -2 : -1;   /* 'DT IS TOO BIG' / 'CFL IS TOO BIG' */
      }
    }
  }
  if (c->step >= 0 && c->rk_step == 1) {
    double cfl_temp = 0;
    for (int k = 2; k <= ny; k++)
      if (c->cfl[k - 1] > cfl_temp) cfl_temp = c->cfl[k - 1];
    if (c->p.dt_flag == 1) {
      double dt_temp = c->dt * c->p.cfl_max / cfl_temp;
      double alt = c->dt + (dt_temp - c->dt) * c->dt / (1.0 + c->dt);
      c->dt = dt_temp < alt ? dt_temp : alt;
    }
  }
  free(nl);
  free(phys);
#undef PH
#undef NL
#undef BF
#undef TGT
}

void orc_nonlinear(orc_ctx *c) { nonlinear_impl(c, 0); }
void orc_nonlinear_linearized(orc_ctx *c) { nonlinear_impl(c, 1); }

/* ------------------------------------------------------------------ */
/* diff_int, PFC/diff_int.f90 */
static void d_dy(orc_ctx *c, int n1, const cplx *f, int n2, cplx *df, const double *d) {
  int ny = c->p.ny;
  if (n1 == ny) {
    df[0] = d[0] * (f[1] - f[0]);
    for (int i = 1; i < n2 - 1; i++) df[i] = d[i] * (f[i] - f[i - 1]);
    df[n2 - 1] = d[n2 - 1] * (f[n1 - 1] - f[n1 - 2]);
  } else if (n1 == ny + 1) {
    for (int i = 0; i < n2; i++) df[i] = d[i] * (f[i + 1] - f[i]);
  }
}
static void d2_dy(int n, const cplx *f, cplx *df, const double *d) {
  df[0] = d[0] * f[0] + d[1] * f[1] + d[2] * f[2];
  for (int i = 1; i < n - 1; i++)
    df[i] = d[3 * i] * f[i - 1] + d[3 * i + 1] * f[i] + d[3 * i + 2] * f[i + 1];
  df[n - 1] = d[3 * (n - 1)] * f[n - 3] + d[3 * (n - 1) + 1] * f[n - 2] + d[3 * (n - 1) + 2] * f[n - 1];
}

/* solve.f90 */
static void solve_helmholtz(orc_ctx *c, int n, cplx *f, double alpha, double diff,
                            const double *d2, cplx topbc, cplx botbc) {
  /* SOLVE_HELMHOLTZ, PFC/solve.f90:154-264 with TOP/BOT_NEUMANN = 0 (bl_grid=0) */
  double A[1200], B[1200], C[1200];
  (void)c;
  A[0] = 0; B[0] = 1; C[0] = 0; f[0] = botbc;
  for (int i = 1; i < n - 1; i++) {
    A[i] = -diff * d2[3 * i];
    B[i] = -diff * d2[3 * i + 1] + alpha;
    C[i] = -diff * d2[3 * i + 2];
  }
  A[n - 1] = 0; B[n - 1] = 1; C[n - 1] = 0; f[n - 1] = topbc;
  for (int i = 1; i < n; i++) {
    B[i - 1] = 1.0 / B[i - 1];
    C[i - 1] = C[i - 1] * B[i - 1];
    f[i - 1] = f[i - 1] * B[i - 1];
    B[i] = B[i] - A[i] * C[i - 1];
    f[i] = f[i] - A[i] * f[i - 1];
  }
  B[n - 1] = 1.0 / B[n - 1];
  f[n - 1] = f[n - 1] * B[n - 1];
  for (int i = n - 2; i >= 0; i--) f[i] = f[i] - C[i] * f[i + 1];
}

static void solve_p(orc_ctx *c, cplx *P, double alpha, cplx topbc, cplx botbc) {
  /* SOLVE_P, PFC/solve.f90:269-338 */
  int ny = c->p.ny;
  double A[1200], B[1200], C[1200];
  double *DN = c->dn, *DH = c->dh;
  A[0] = 0; B[0] = -F(DN, 1); C[0] = F(DN, 1);
  A[1] = F(DH, 2) * F(DN, 1);
  B[1] = -(F(DH, 2) * F(DN, 1)) - F(DH, 2) * F(DN, 2) + alpha;
  C[1] = F(DH, 2) * F(DN, 2);
  for (int j = 3; j <= ny - 1; j++) {
    A[j - 1] = D2H(1, j); B[j - 1] = D2H(2, j) + alpha; C[j - 1] = D2H(3, j);
  }
  A[ny - 1] = F(DH, ny) * F(DN, ny - 1);
  B[ny - 1] = -(F(DH, ny) * F(DN, ny - 1)) - F(DH, ny) * F(DN, ny) + alpha;
  C[ny - 1] = F(DH, ny) * F(DN, ny);
  A[ny] = -F(DN, ny); B[ny] = F(DN, ny); C[ny] = 0;
  P[0] = botbc;
  P[ny] = topbc;
  for (int j = 2; j <= ny + 1; j++) {
    B[j - 2] = 1.0 / B[j - 2];
    C[j - 2] = C[j - 2] * B[j - 2];
    P[j - 2] = P[j - 2] * B[j - 2];
    B[j - 1] = B[j - 1] - A[j - 1] * C[j - 2];
    P[j - 1] = P[j - 1] - A[j - 1] * P[j - 2];
  }
  P[ny] = P[ny] * (1.0 / B[ny]);
  for (int j = ny; j >= 1; j--) P[j - 1] = P[j - 1] - C[j - 1] * P[j];
  P[0] = (botbc - DM(2, 1) * P[1] - DM(3, 1) * P[2]) / DM(1, 1);
  P[ny] = (topbc - DM(1, 2) * P[ny - 2] - DM(2, 2) * P[ny - 1]) / DM(3, 2);
}

/* SUBTRACT_PRESSURE_GRADIENT, PFC/solve.f90:54-77; cu is (ny+1,3) */
static void subtract_pressure_gradient(orc_ctx *c, cplx *cu, const cplx *cp, double coef,
                                       int x, int z) {
  int ny = c->p.ny, n1 = ny + 1;
  cplx dp[1200];
  d_dy(c, ny + 1, cp, ny, dp, c->dn);
  cplx ikx = I * c->kx[x], ikz = I * c->kz[z];
  for (int j = 2; j <= ny; j++) cu[j - 1] = cu[j - 1] - coef * ikx * cp[j - 1];
  for (int j = 2; j <= ny - 1; j++) cu[n1 + j - 1] = cu[n1 + j - 1] - coef * dp[j - 1];
  for (int j = 2; j <= ny; j++) cu[2 * n1 + j - 1] = cu[2 * n1 + j - 1] - coef * ikz * cp[j - 1];
}

/* strip_divergence, PFC/solve.f90:14-50 */
void orc_strip_divergence_column(orc_ctx *c, double complex *cu, double complex *cp,
                                 double coef, int x, int z) {
  int ny = c->p.ny, n1 = ny + 1;
  cplx dv[1200];
  double tmp = 1.0 / coef;
  d_dy(c, ny, cu + n1, ny + 1, dv, c->dh);
  cplx ikx = I * c->kx[x], ikz = I * c->kz[z];
  cp[0] = 0;
  for (int j = 2; j <= ny; j++)
    cp[j - 1] = tmp * (ikx * cu[j - 1] + dv[j - 1] + ikz * cu[2 * n1 + j - 1]);
  cp[ny] = 0;
  solve_p(c, cp, -c->k2[z + c->p.nz * x], 0, 0);
  subtract_pressure_gradient(c, cu, cp, coef, x, z);
}

/* PHASE1 for one wavenumber, PFC/pass2.f90:184-352.  cu (ny+1,3) holds
 * -NL on entry and the new velocity on exit; cru (ny+1,3); cp (ny+1).    */
static void phase1(orc_ctx *c, int x, int z, cplx *cu, cplx *cru, cplx *cp) {
  int ny = c->p.ny, n1 = ny + 1, rk = c->rk_step, nz = c->p.nz;
  double dt = c->dt, re = c->p.re;
  double k2 = c->k2[z + nz * x];
  double vis_imp = RKD(rk) * (dt / re);
  double rk_press = (RKC(rk) + RKD(rk)) * dt;
  double coef = RKB(rk) * dt;
  cplx cv[3 * 1200], ch[1200], du[1200];
  for (int i = 0; i < 3 * n1; i++) cv[i] = cru[i] + coef * cu[i];
  if (rk == 1) {
    double vis_exp = RKC(rk) * (dt / re);
    /* add_explicit_diffusive_terms(cv, cru) */
    d2_dy(n1, cru, du, c->d2h);
    for (int j = 0; j < n1; j++) cv[j] = cv[j] + vis_exp * (du[j] - k2 * cru[j]);
    d2_dy(ny, cru + n1, du, c->d2n);
    for (int j = 0; j < ny; j++) cv[n1 + j] = cv[n1 + j] + vis_exp * (du[j] - k2 * cru[n1 + j]);
    d2_dy(n1, cru + 2 * n1, du, c->d2h);
    for (int j = 0; j < n1; j++) cv[2 * n1 + j] = cv[2 * n1 + j] + vis_exp * (du[j] - k2 * cru[2 * n1 + j]);
    if (k2 != 0.0) subtract_pressure_gradient(c, cv, cp, rk_press, x, z);
  }
  size_t cb = (size_t)z + (size_t)nz * x, cs = (size_t)nz * c->nxh;
  if (k2 == 0.0) {
    if (c->p.fix_mass == 1) {
      /* COMPUTE_P_GRAD, PFC/pass2.f90:356-375 (cu = -NL) */
      double tmp = 0;
      for (int pl = 2; pl <= ny; pl++) tmp = tmp + F(c->dyh, pl) * creal(cu[pl - 1]);
      c->p_grad = -tmp + 0.5 * (F(c->d_um_dy, ny) - F(c->d_um_dy, 1)) / re;
    }
    for (int j = 0; j < n1; j++) cv[j] = cv[j] - cos(c->p.beta) * rk_press * c->p_grad;
    for (int j = 0; j < n1; j++) cv[2 * n1 + j] = cv[2 * n1 + j] - sin(c->p.beta) * rk_press * c->p_grad;
    solve_helmholtz(c, n1, cv, 1.0, vis_imp, c->d2h, c->cbc_top[cb], c->cbc_bot[cb]);
    solve_helmholtz(c, n1, cv + 2 * n1, 1.0, vis_imp, c->d2h, c->cbc_top[cb + 2 * cs], c->cbc_bot[cb + 2 * cs]);
    for (int j = 0; j < n1; j++) cp[j] = 0;
    cv[n1] = c->cbc_bot[cb + cs];
    for (int j = 2; j <= ny; j++) cv[n1 + j - 1] = cv[n1];
    cv[n1 + ny] = 0;
  } else {
    double alpha = 1.0 + vis_imp * k2;
    solve_helmholtz(c, n1, cv, alpha, vis_imp, c->d2h, c->cbc_top[cb], c->cbc_bot[cb]);
    solve_helmholtz(c, n1, cv + 2 * n1, alpha, vis_imp, c->d2h, c->cbc_top[cb + 2 * cs], c->cbc_bot[cb + 2 * cs]);
    solve_helmholtz(c, ny, cv + n1, alpha, vis_imp, c->d2n, c->cbc_top[cb + cs], c->cbc_bot[cb + cs]);
    cv[n1 + ny] = 0;
    orc_strip_divergence_column(c, cv, ch, rk_press, x, z);
    d2_dy(n1, ch, du, c->d2h);
    for (int j = 0; j < n1; j++) cp[j] = cp[j] + alpha * ch[j] - vis_imp * du[j];
  }
  if (rk < 3) {
    double coef2 = dt * RKA(rk + 1);
    for (int i = 0; i < 3 * n1; i++) cru[i] = cv[i] + coef2 * cu[i];
    double vis_exp = (dt / re) * RKC(rk + 1);
    d2_dy(n1, cv, du, c->d2h);
    for (int j = 0; j < n1; j++) cru[j] = cru[j] + vis_exp * (du[j] - k2 * cv[j]);
    d2_dy(ny, cv + n1, du, c->d2n);
    for (int j = 0; j < ny; j++) cru[n1 + j] = cru[n1 + j] + vis_exp * (du[j] - k2 * cv[n1 + j]);
    d2_dy(n1, cv + 2 * n1, du, c->d2h);
    for (int j = 0; j < n1; j++) cru[2 * n1 + j] = cru[2 * n1 + j] + vis_exp * (du[j] - k2 * cv[2 * n1 + j]);
    if (k2 != 0.0) {
      double rkp2 = (RKC(rk + 1) + RKD(rk + 1)) * dt;
      subtract_pressure_gradient(c, cru, cp, rkp2, x, z);
    }
  } else {
    for (int i = 0; i < 3 * n1; i++) cru[i] = cv[i];
  }
  for (int i = 0; i < 3 * n1; i++) cu[i] = cv[i];
}

/* rhs_solve, PFC/pass2.f90:29-180 (crossflow jet handled by orc_jet_profile) */
static void rhs_one(orc_ctx *c, int x, int z) {
  int ny = c->p.ny, n1 = ny + 1;
  cplx cu[3 * 1200], cru[3 * 1200], cp[1200];
  for (int q = 0; q < 3; q++)
    for (int j = 0; j < n1; j++) {
      cu[q * n1 + j] = -D1(c, z, x, j, q);
      cru[q * n1 + j] = D2(c, j, q, z, x);
    }
  for (int j = 0; j < n1; j++) cp[j] = D4(c, j, z, x);
  phase1(c, x, z, cu, cru, cp);
  for (int q = 0; q < 3; q++)
    for (int j = 0; j < n1; j++) {
      D1(c, z, x, j, q) = cu[q * n1 + j];
      D2(c, j, q, z, x) = cru[q * n1 + j];
    }
  for (int j = 0; j < n1; j++) D4(c, j, z, x) = cp[j];
  if (c->k2[z + c->p.nz * x] == 0.0) {
    /* PFC/pass2.f90:84-89 */
    double *d = c->d_um_dy;
    d[0] = creal(DM(1, 1) * cu[0] + DM(2, 1) * cu[1] + DM(3, 1) * cu[2]);
    for (int j = 2; j <= ny - 1; j++) d[j - 1] = creal(F(c->dn, j) * (cu[j] - cu[j - 1]));
    d[ny - 1] = creal(DM(1, 2) * cu[ny - 2] + DM(2, 2) * cu[ny - 1] + DM(3, 2) * cu[ny]);
  }
}

void orc_rhs_solve(orc_ctx *c) {
  int nz = c->p.nz, nxh = c->nxh;
  if (c->crossflow) {
    /* end-of-substep time and increment, PFC/pass2.f90:37-38 */
    double s = 0.0;
    for (int r = 1; r <= c->rk_step; r++) s += RKC(r) + RKD(r);
    orc_jet_profile(c, c->t_total + c->dt * s, c->dt * (RKC(c->rk_step) + RKD(c->rk_step)));
  }
  rhs_one(c, 0, 0); /* mean mode first: it updates p_grad and d_um_dy */
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 1; t < nz * nxh; t++) rhs_one(c, t / nz, t % nz);
}

/* ------------------------------------------------------------------ */
/* boundary, PFC/read_write.f90:1465-1532 */
void orc_boundary(orc_ctx *c) {
  int nz = c->p.nz, nxh = c->nxh, ny = c->p.ny;
  size_t np = (size_t)c->p.nx2 * c->p.nz2, cs = (size_t)nz * nxh;
  memset(c->cbc_top, 0, sizeof(cplx) * 3 * cs);
  memset(c->cbc_bot, 0, sizeof(cplx) * 3 * cs);
  double *u2 = malloc(sizeof(double) * np * 3), *u3 = u2 + np, *ub = u3 + np;
  for (int q = 0; q < 3; q += 2) {
    double g = q == 0 ? c->p.ctrlu : c->p.ctrlw;
    if (g == 0.0) continue;
    double off = q == 0 ? 2.0 : 0.0;
    orc_xz_c2r(c, &D1(c, 0, 0, 1, q), u2);
    orc_xz_c2r(c, &D1(c, 0, 0, 2, q), u3);
    for (size_t i = 0; i < np; i++) ub[i] = (DM(2, 1) * u2[i] + DM(3, 1) * u3[i] - off) / (g - DM(1, 1));
    orc_xz_r2c(c, ub, c->cbc_bot + q * cs);
    orc_xz_c2r(c, &D1(c, 0, 0, ny - 1, q), u2);
    orc_xz_c2r(c, &D1(c, 0, 0, ny - 2, q), u3);
    for (size_t i = 0; i < np; i++) ub[i] = -(DM(2, 2) * u2[i] + DM(1, 2) * u3[i] + off) / (g + DM(3, 2));
    orc_xz_r2c(c, ub, c->cbc_top + q * cs);
  }
  free(u2);
}

/* l2_norm, PFC/read_write.f90:1432-1462.  Plane ny+1 carries dy(ny+1)=0, so
 * its term is zero (the Fortran reads y(ny+1) beyond y's bounds there).    */
void orc_l2_norm(orc_ctx *c, double *l2out, double *drag) {
  int ny = c->p.ny;
  size_t np = (size_t)c->p.nx2 * c->p.nz2;
  double l2 = 0.0;
  double *u = malloc(sizeof(double) * np);
  for (int pl = 1; pl <= ny; pl++)
    for (int q = 0; q < 3; q++) {
      orc_xz_c2r(c, &D1(c, 0, 0, pl - 1, q), u);
      if (q == 0) {
        double yy = F(c->y, pl);
        for (size_t i = 0; i < np; i++) u[i] = u[i] - (1.0 - yy * yy);
      }
      double s = 0;
      for (size_t i = 0; i < np; i++) s += u[i] * u[i];
      l2 = l2 + s * F(c->dy, pl);
    }
  free(u);
  l2 = sqrt(l2 / (double)c->p.nx2 / (double)c->p.nz2 / 2.0);
  if (l2out) *l2out = l2;
  if (drag) *drag = F(c->d_um_dy, 1) - F(c->d_um_dy, ny);
}

/* ------------------------------------------------------------------ */
/* seeded counter-based generator standing in for RANDOM_NUMBER: SplitMix64
 * of (seed, kx index, kz index, row, column) -> uniform [0,1).            */
static uint64_t smix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
static double rng_u01(uint64_t seed, int x, int z, int j, int col) {
  uint64_t ctr = ((((uint64_t)x * 65536u + (uint64_t)z) * 65536u + (uint64_t)j) * 8u) + (uint64_t)col;
  uint64_t h = smix(seed ^ smix(ctr));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

/* random_divfree_vector(filter=0), PFC/init_vel.f90:357-432 */
static void random_divfree_vector(orc_ctx *c, uint64_t seed, int p, int q, double ampl, cplx *cu) {
  int ny = c->p.ny, n1 = ny + 1, nz = c->p.nz;
  double temp[4][1200];
  for (int col = 0; col < 4; col++)
    for (int j = 0; j < n1; j++) temp[col][j] = rng_u01(seed, p, q, j, col);
  for (int i = 0; i < 3 * n1; i++) cu[i] = 0;
  double k2 = c->k2[q + nz * p];
  if (k2 != 0.0) {
    for (int col = 0; col < 4; col++)
      for (int j = 0; j < n1; j++) temp[col][j] = 2.0 * (temp[col][j] - 0.5);
    for (int j = 0; j < n1; j++) cu[j] = temp[0][j] + I * temp[1][j];
    for (int j = 0; j < ny; j++) cu[n1 + j] = temp[2][j] + I * temp[3][j];
    cu[n1 + ny] = 0;
    cplx ikx = I * c->kx[p], ikz = I * c->kz[q];
    cplx u_old[1200];
    for (int j = 0; j < n1; j++) u_old[j] = cu[j];
    cu[2 * n1] = 0;
    for (int j = 2; j <= ny; j++)
      cu[2 * n1 + j - 1] = (ikx * u_old[j - 1] + ikz * F(c->dh, j) * (cu[n1 + j - 1] - cu[n1 + j - 2])) / k2;
    cu[2 * n1 + ny] = 0;
    cu[0] = 0;
    for (int j = 2; j <= ny; j++)
      cu[j - 1] = (-ikz * u_old[j - 1] + ikx * F(c->dh, j) * (cu[n1 + j - 1] - cu[n1 + j - 2])) / k2;
    cu[ny] = 0;
    double tmp = 0;
    for (int j = 2; j <= ny; j++)
      tmp += F(c->dyh, j) * (cabs(cu[j - 1]) + cabs(cu[2 * n1 + j - 1]) + 0.5 * cabs(cu[n1 + j - 2]) + 0.5 * cabs(cu[n1 + j - 1]));
    if (tmp > 0.0)
      for (int i = 0; i < 3 * n1; i++) cu[i] = ampl * cu[i] / tmp;
  } else {
    for (int j = 0; j < n1; j++) { cu[j] = temp[0][j]; cu[2 * n1 + j] = temp[1][j]; }
  }
}

/* remove_initial_divergence, PFC/init_vel.f90:518-536 */
void orc_remove_initial_divergence(orc_ctx *c) {
  int ny = c->p.ny, n1 = ny + 1, nz = c->p.nz, nxh = c->nxh;
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < nz * nxh; t++) {
    int x = t / nz, z = t % nz;
    if (c->k2[z + nz * x] == 0.0) {
      for (int j = 2; j <= ny; j++) D1(c, z, x, j - 1, 1) = D1(c, z, x, 0, 1);
    } else {
      cplx cu[3 * 1200], ch[1200];
      for (int q = 0; q < 3; q++)
        for (int j = 0; j < n1; j++) cu[q * n1 + j] = D1(c, z, x, j, q);
      orc_strip_divergence_column(c, cu, ch, 1.0, x, z);
      for (int q = 0; q < 3; q++)
        for (int j = 0; j < n1; j++) D1(c, z, x, j, q) = cu[q * n1 + j];
    }
  }
}

/* PFC/init_vel.f90:333-342 */
void orc_compute_d_um_dy(orc_ctx *c) {
  int ny = c->p.ny;
  double *d = c->d_um_dy;
  d[0] = creal(DM(1, 1) * D1(c, 0, 0, 0, 0) + DM(2, 1) * D1(c, 0, 0, 1, 0) + DM(3, 1) * D1(c, 0, 0, 2, 0));
  for (int j = 2; j <= ny - 1; j++) d[j - 1] = creal(F(c->dn, j) * (D1(c, 0, 0, j, 0) - D1(c, 0, 0, j - 1, 0)));
  d[ny - 1] = creal(DM(1, 2) * D1(c, 0, 0, ny - 2, 0) + DM(2, 2) * D1(c, 0, 0, ny - 1, 0) + DM(3, 2) * D1(c, 0, 0, ny, 0));
}

static void copy_data1_to_data2(orc_ctx *c) {
  int ny = c->p.ny, nz = c->p.nz, nxh = c->nxh;
  for (int x = 0; x < nxh; x++)
    for (int z = 0; z < nz; z++)
      for (int q = 0; q < 3; q++)
        for (int j = 0; j <= ny; j++) D2(c, j, q, z, x) = D1(c, z, x, j, q);
}
static void copy_data2_to_data1(orc_ctx *c) {
  int ny = c->p.ny, nz = c->p.nz, nxh = c->nxh;
  for (int x = 0; x < nxh; x++)
    for (int z = 0; z < nz; z++)
      for (int q = 0; q < 3; q++)
        for (int j = 0; j <= ny; j++) D1(c, z, x, j, q) = D2(c, j, q, z, x);
}

/* COMPUTE_INITIAL_PRESSURE + solve_continuous_poisson, PFC/init_vel.f90:437-514 */
void orc_compute_initial_pressure(orc_ctx *c, int linearized) {
  int ny = c->p.ny, n1 = ny + 1, nz = c->p.nz, nxh = c->nxh;
  int save_step = c->step, save_rk = c->rk_step;
  c->step = -1;
  c->rk_step = 3;
  nonlinear_impl(c, linearized);
  double visc = 1.0 / c->p.re;
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < nz * nxh; t++) {
    int x = t / nz, z = t % nz;
    cplx cu[3 * 1200], cru[3 * 1200], du[1200], cp[1200];
    double k2 = c->k2[z + nz * x];
    for (int q = 0; q < 3; q++)
      for (int j = 0; j < n1; j++) {
        cu[q * n1 + j] = D2(c, j, q, z, x);
        cru[q * n1 + j] = -D1(c, z, x, j, q);
      }
    d2_dy(n1, cu, du, c->d2h);
    for (int j = 0; j < n1; j++) cru[j] = cru[j] + visc * (du[j] - k2 * cu[j]);
    d2_dy(ny, cu + n1, du, c->d2n);
    for (int j = 0; j < ny; j++) cru[n1 + j] = cru[n1 + j] + visc * (du[j] - k2 * cu[n1 + j]);
    d2_dy(n1, cu + 2 * n1, du, c->d2h);
    for (int j = 0; j < n1; j++) cru[2 * n1 + j] = cru[2 * n1 + j] + visc * (du[j] - k2 * cu[2 * n1 + j]);
    if (k2 == 0.0) {
      for (int j = 0; j < n1; j++) D4(c, j, z, x) = 0;
    } else {
      orc_strip_divergence_column(c, cru, cp, 1.0, x, z);
      for (int j = 0; j < n1; j++) D4(c, j, z, x) = cp[j];
    }
  }
  copy_data2_to_data1(c);
  c->step = save_step;
  c->rk_step = save_rk;
}

/* DEFINE_INITIAL_FIELD, PFC/init_vel.f90:25-353, for the channel presets
 * which_test 1, 4, 6 and the laminar + k^-2 noise preset 10.               */
double orc_rng_u01(unsigned long long seed, int x, int z, int j, int col) {
  return rng_u01(seed, x, z, j, col);
}

void orc_init_field(orc_ctx *c, int which_test, unsigned long long seed, double ampl) {
  orc_initial_velocity(c, which_test, seed, ampl);
  orc_remove_initial_divergence(c);
  orc_compute_d_um_dy(c);
  copy_data1_to_data2(c);
  orc_compute_initial_pressure(c, 0);
}

/* define_initial_field after its which_test branch (PFC/init_vel.f90:325-351)
 * for a velocity the caller wrote into data1 (the Orr-Sommerfeld modes of
 * which_test 2, 5, 8): t = 0, data2 and data4 cleared, divergence removed,
 * d_um_dy, data2 = data1, initial pressure. */
void orc_init_from_velocity(orc_ctx *c) {
  size_t nf = (size_t)c->p.nz * c->nxh * (c->p.ny + 1);
  c->t_total = 0;
  memset(c->data2, 0, sizeof(cplx) * 3 * nf);
  memset(c->data4, 0, sizeof(cplx) * nf);
  orc_remove_initial_divergence(c);
  orc_compute_d_um_dy(c);
  copy_data1_to_data2(c);
  orc_compute_initial_pressure(c, 0);
}

/* the which_test velocity before divergence removal, PFC/init_vel.f90:88-244 */
void orc_initial_velocity(orc_ctx *c, int which_test, unsigned long long seed, double ampl) {
  int ny = c->p.ny, n1 = ny + 1, nz = c->p.nz, nxh = c->nxh;
  size_t nf = (size_t)nz * nxh * n1;
  c->t_total = 0;
  memset(c->data1, 0, sizeof(cplx) * 3 * nf);
  memset(c->data2, 0, sizeof(cplx) * 3 * nf);
  memset(c->data4, 0, sizeof(cplx) * nf);
  double beta = c->p.beta;
  if (which_test == 1 || which_test == 10) {
    for (int j = 0; j < n1; j++) {
      double yh = c->yh[j];
      D1(c, 0, 0, j, 0) = (1.0 - yh * yh) * cos(beta);
      D1(c, 0, 0, j, 2) = (1.0 - yh * yh) * sin(beta);
    }
  } else if (which_test == 4) {
    for (int j = 0; j < n1; j++) D1(c, 0, 0, j, 0) = 0.75 * (1.0 - pow(c->yh[j], 8));
  } else if (which_test == 6) {
    c->p_grad = 0;
    c->p.fix_mass = 0;
    for (int j = 0; j < n1; j++) D1(c, 0, 1, j, 0) = -0.5 * sin(c->pi * c->yh[j]);
    for (int j = 0; j < ny; j++) D1(c, 0, 1, j, 1) = I * (-0.5 * cos(c->pi * c->y[j]));
  }
  if (which_test == 4 || which_test == 10) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int t = 0; t < nz * nxh; t++) {
      int x = t / nz, z = t % nz;
      double k2 = c->k2[z + nz * x];
      if (k2 == 0.0) continue;
      cplx cu[3 * 1200];
      random_divfree_vector(c, seed, x, z, ampl, cu);
      double f = 1.0 / k2 < 1.0 ? 1.0 / k2 : 1.0;
      for (int q = 0; q < 3; q++)
        for (int j = 0; j < n1; j++) D1(c, z, x, j, q) = cu[q * n1 + j] * f;
    }
  }
}

/* timestep loop body, PFC/main_mpi.f90:70-86 */
void orc_timestep(orc_ctx *c, int nsteps, int linearized) {
  for (int s = 0; s < nsteps; s++) {
    c->step = c->step < 0 ? 1 : c->step + 1;
    orc_boundary(c);
    for (int rk = 1; rk <= 3; rk++) {
      c->rk_step = rk;
      nonlinear_impl(c, linearized);
      orc_rhs_solve(c);
    }
    c->t_total = c->t_total + c->dt;
  }
}

double orc_bulk_flux(orc_ctx *c) {
  double s = 0;
  for (int j = 0; j <= c->p.ny; j++) s += c->dyh[j] * creal(D1(c, 0, 0, j, 0));
  return s;
}

/* max |divergence| over all wavenumbers, CHECK_DIVERGENCE PFC/pass2.f90:380-419 */
double orc_max_divergence(orc_ctx *c) {
  int ny = c->p.ny, nz = c->p.nz, nxh = c->nxh, n1 = ny + 1;
  double m = 0;
  for (int x = 0; x < nxh; x++)
    for (int z = 0; z < nz; z++) {
      cplx v[1200], dv[1200];
      for (int j = 0; j < n1; j++) v[j] = D1(c, z, x, j, 1);
      d_dy(c, ny, v, ny + 1, dv, c->dh);
      for (int j = 2; j <= ny; j++) {
        cplx t = I * c->kx[x] * D1(c, z, x, j - 1, 0) + dv[j - 1] + I * c->kz[z] * D1(c, z, x, j - 1, 2);
        if (cabs(t) > m) m = cabs(t);
      }
    }
  return m;
}

/* ------------------------------------------------------------------ */
/* jet_profile, PFC/pass2.f90:423-673, with bl_grid = 0 (closed channel:
 * the suction profile balances the jet's mass flux).  Mode 2 is the Gaussian
 * slot generator writing the same cbc(:,:,2) slot. */
static void filter_cosine(orc_ctx *c, cplx *cu) {
  int nz = c->p.nz, nxh = c->nxh;
  for (int x = 0; x < nxh; x++)
    for (int z = 0; z < nz; z++)
      cu[z + (size_t)nz * x] = cu[z + (size_t)nz * x] * 0.5 *
          (1.0 + cos(c->pi * c->kx[x] / ((double)(c->p.nx / 2) * 2.0 * c->pi / c->p.lx))) * 0.5 *
          (1.0 + cos(c->pi * c->kz[z] / ((double)(nz / 2) * 2.0 * c->pi / c->p.lz)));
}

void orc_set_jet(orc_ctx *c, const orc_jet *j) {
  if (j) c->jet = *j;
  c->crossflow = j != NULL && j->mode != 0;
  c->jet_calls = 0;
}

void orc_get_jet_forcing(orc_ctx *c, double *jf, double *incr) {
  if (jf) memcpy(jf, c->jet.jet_forcing, sizeof(double) * 24);
  if (incr) memcpy(incr, c->jet.jet_forcing_incr, sizeof(double) * 24);
}

/* random walk of the Freund forcing parameters, PFC/pass2.f90:454-477 */
static void jet_walk(orc_ctx *c, double time_incr) {
  orc_jet *jt = &c->jet;
  double *jf = jt->jet_forcing, *inc = jt->jet_forcing_incr;
  for (int n = 0; n < 24; n++) {
    double r = rng_u01(jt->seed, (int)c->jet_calls, 0, n, 7);
    /* SIGN(1, r - 0.05) */
    inc[n] = inc[n] * ((r - 0.05) >= 0.0 ? 1.0 : -1.0);
  }
  for (int n = 0; n < 24; n++) jf[n] = jf[n] + time_incr * inc[n];
  for (int j = 0; j < 2; j++)
    for (int i = 0; i < 3; i++) {
      int a = i + 3 * j, b = i + 3 * j + 6;   /* (i,j,1), (i,j,2) */
      if (jf[a] <= 0.01) { jf[a] = 0.01; inc[a] = fabs(inc[a]); }
      else if (jf[a] >= 0.07) { jf[a] = 0.07; inc[a] = -fabs(inc[a]); }
      if (jf[b] <= 0.1) { jf[b] = 0.1; inc[b] = fabs(inc[b]); }
      else if (jf[b] >= 0.7) { jf[b] = 0.7; inc[b] = -fabs(inc[b]); }
    }
}

void orc_jet_profile(orc_ctx *c, double time, double time_incr) {
  const orc_jet *jt = &c->jet;
  int nx = c->p.nx, nz = c->p.nz, nxh = c->nxh;
  size_t cs = (size_t)nz * nxh, ns = (size_t)nx * nz;
  double lx = c->p.lx, lz = c->p.lz, pi = c->pi;
  if (jt->seed != 0) jet_walk(c, time_incr);
  c->jet_calls++;
  double *f = malloc(sizeof(double) * ns * 2), *vj = f + ns;
  cplx *cs_ = malloc(sizeof(cplx) * cs * 2), *cj = cs_ + cs;
  /* define_suction_profile, PFC/pass2.f90:553-609 */
  double frac_suct = 0.5 * jt->frac_xbuff, suct_start = 1.0 - jt->frac_xbuff;
  double suct_rise = 0.25 * frac_suct, suct_fall = 0.25 * frac_suct;
  double xstart = lx * suct_start, xrise = xstart + lx * suct_rise;
  double xfall = xstart + lx * frac_suct - lx * suct_fall, xend = xstart + lx * frac_suct;
  if (xend > lx) c->status = -3;   /* 'Suction must end inside box.' */
  for (int x = 1; x <= nx; x++) {
    double xc = F(c->xcoord, x), fx = 0.0;
    if (xc > xstart && xc < xend) {
      if (xc < xrise) { double x2 = (xc - xstart) / (xrise - xstart); fx = 1.0 / (1.0 + exp(1.0 / x2 + 1.0 / (x2 - 1.0))); }
      else if (xc > xfall) { double x2 = (xend - xc) / (xend - xfall); fx = 1.0 / (1.0 + exp(1.0 / x2 + 1.0 / (x2 - 1.0))); }
      else fx = 1.0;
    }
    for (int z = 0; z < nz; z++) f[(x - 1) + (size_t)nx * z] = fx;
  }
  orc_small_r2c(c, f, cs_);
  for (int n = 0; n < jt->filter_jet_profile; n++) filter_cosine(c, cs_);
  double sum_suction = creal(cs_[0]);
  for (int wall = 0; wall < 2; wall++) {
    cplx *dst = (wall == 0 ? c->cbc_bot : c->cbc_top) + cs;
    if (jt->jetmag[wall] == 0.0 || jt->mode == 0) { memset(dst, 0, sizeof(cplx) * cs); continue; }
    double jm = jt->jetmag[wall];
    if (jt->mode == 1) {
      /* define_jet_profile, PFC/pass2.f90:611-656 */
      const double fw[6] = {0, 1, 2, 0, 1, 2};
      double v_ampl = jm * (1.0 + jt->forcing[wall] * sin(2.0 * pi * time * jt->for_freq[wall] * jm / jt->jet_diam));
      for (int z = 1; z <= nz; z++)
        for (int x = 1; x <= nx; x++) {
          double xd1 = F(c->xcoord, x) - jt->xjet[wall], xd2 = F(c->xcoord, x) - (lx + jt->xjet[wall]);
          double zd1 = F(c->zcoord, z) - jt->zjet[wall], zd2 = F(c->zcoord, z) - (lz + jt->zjet[wall]);
          /* ABS(CMPLX(a,b)) without KIND is a default-real (single) complex */
          double r1 = (double)hypotf((float)xd1, (float)zd1) * 2.0 / jt->jet_diam;
          double r2 = (double)hypotf((float)xd2, (float)zd1) * 2.0 / jt->jet_diam;
          double r3 = (double)hypotf((float)xd1, (float)zd2) * 2.0 / jt->jet_diam;
          double r4 = (double)hypotf((float)xd2, (float)zd2) * 2.0 / jt->jet_diam;
          double r = fmin(fmin(r1, r2), fmin(r3, r4));
          double v;
          if (r == 0.0) v = v_ampl;
          else {
            double phi = atan2(zd1, xd1), s = 0;
            for (int i = 0; i < 6; i++)
              s += jt->jet_forcing[i] * cos(jt->jet_forcing[6 + i] * jm * time / jt->jet_diam + jt->jet_forcing[12 + i]) *
                   cos(fw[i] * phi + jt->jet_forcing[18 + i]);
            double bjet = 5.0 + s;
            v = v_ampl * 0.5 * (1.0 - tanh(bjet * (r - 1.0 / r)));
          }
          vj[(x - 1) + (size_t)nx * (z - 1)] = v;
        }
    } else {
      /* Gaussian spanwise slot at x = xjet */
      double a = jm * 0.5 * (1.0 + sin(2.0 * pi * jt->freq * time));
      for (int z = 0; z < nz; z++)
        for (int x = 1; x <= nx; x++) {
          double d = fabs(F(c->xcoord, x) - jt->xjet[wall]);
          if (lx - d < d) d = lx - d;
          vj[(x - 1) + (size_t)nx * z] = a * exp(-(d / jt->width) * (d / jt->width));
        }
    }
    orc_small_r2c(c, vj, cj);
    if (wall == 1) for (size_t i = 0; i < cs; i++) cj[i] = -cj[i];
    for (int n = 0; n < jt->filter_jet_profile; n++) filter_cosine(c, cj);
    double sum = creal(cj[0]);
    for (size_t i = 0; i < cs; i++) dst[i] = cj[i] - (sum / sum_suction) * cs_[i];
  }
  free(f);
  free(cs_);
}

/* ------------------------------------------------------------------ */
/* compute_time_deriv, PFC/arnoldi.f90:485-567: w = Phi_T v with the
 * linearized operator.  p_grad and d_um_dy start from zero on every call.   */
void orc_arnoldi_matvec(orc_ctx *c, int tend, const double *v, double *w) {
  int nx = c->p.nx, nz = c->p.nz, ny = c->p.ny, nxh = c->nxh;
  size_t ns = (size_t)nx * nz, cs = (size_t)nz * nxh, nf = cs * (ny + 1);
  const double eps = 1.0e-8;
  memset(c->data1, 0, sizeof(cplx) * 3 * nf);
  memset(c->data2, 0, sizeof(cplx) * 3 * nf);
  double mx = 0;
  for (size_t i = 0; i < ns * (ny + 1) * 3; i++) if (fabs(v[i]) > mx) mx = fabs(v[i]);
  double scale = eps / mx;
  for (int q = 0; q < 3; q++)
    for (int j = 1; j <= ny + 1; j++) {
      cplx *dst = &D1(c, 0, 0, j - 1, q);
      orc_small_r2c(c, v + ns * ((size_t)(j - 1) + (size_t)(ny + 1) * q), dst);
      double wgt = q == 1 ? F(c->dy, j) : F(c->dyh, j);
      if (wgt != 0.0) { double s = scale / sqrt(wgt); for (size_t i = 0; i < cs; i++) dst[i] = s * dst[i]; }
      else memset(dst, 0, sizeof(cplx) * cs);
    }
  copy_data1_to_data2(c);
  c->p_grad = 0;
  memset(c->d_um_dy, 0, sizeof(double) * ny);
  orc_compute_initial_pressure(c, 1);
  c->t_total = 0;
  for (int s = 1; s <= tend; s++) {
    c->step = s;
    for (int rk = 1; rk <= 3; rk++) {
      c->rk_step = rk;
      nonlinear_impl(c, 1);
      orc_rhs_solve(c);
    }
    c->t_total = c->t_total + c->dt;
  }
  for (int q = 0; q < 3; q++)
    for (int j = 1; j <= ny + 1; j++) {
      cplx *src = &D1(c, 0, 0, j - 1, q);
      double wgt = q == 1 ? F(c->dy, j) : F(c->dyh, j);
      double s = sqrt(wgt) / scale;
      for (size_t i = 0; i < cs; i++) src[i] = s * src[i];
      orc_small_c2r(c, src, w + ns * ((size_t)(j - 1) + (size_t)(ny + 1) * q));
    }
}
