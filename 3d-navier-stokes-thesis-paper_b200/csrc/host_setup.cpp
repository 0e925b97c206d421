// host_setup.cpp -- host-side setup for callers without the Fortran host:
// flow.dat reader (PFC/setup.f90:45-201), define_coordinates (:541-754),
// wavenumbers (:1439-1466) and the seeded initial field (PFC/init_vel.f90).
#include <cctype>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "chanflow.h"
#include "chanflow_host.h"

typedef std::complex<double> cd;

extern "C" {

void cfh_run_defaults(cfh_run* r) {
  memset(r, 0, sizeof(*r));
  r->re = 2500.0;
  r->lx = 4.0 * M_PI;
  r->lz = 2.0 * M_PI;
  r->nx = 32; r->ny = 33; r->nz = 32; r->nx2 = 48; r->nz2 = 48;
  r->tend = 100; r->output_step = 100; r->save_step = 100; r->l2_step = 20;
  r->which_test = 10;
  r->disturb_ampl = 1e-3;
  r->fix_mass = 1;
  r->stretch = 2.75;
  r->dt = -1.0;
  r->seed = 1;
  r->precision = CFG_FP64;
  r->jet_diam = 1.0;
  r->frac_xbuff = 0.25;
}

// first list-directed value of a line (Fortran d exponents accepted)
static bool first_value(const std::string& line, double* v) {
  size_t i = 0;
  while (i < line.size() && (isspace((unsigned char)line[i]) || line[i] == ',')) ++i;
  size_t j = i;
  while (j < line.size() && !isspace((unsigned char)line[j]) && line[j] != ',' && line[j] != '/') ++j;
  if (j == i) return false;
  std::string tok = line.substr(i, j - i);
  for (char& ch : tok)
    if (ch == 'd' || ch == 'D') ch = 'e';
  char* end = nullptr;
  *v = strtod(tok.c_str(), &end);
  return end && *end == '\0';
}

int cfh_read_flow_dat(const char* path, cfh_run* r, char* err, int errlen) {
  auto seterr = [&](const char* m) {
    if (err && errlen > 0) snprintf(err, errlen, "%s", m);
    return -1;
  };
  cfh_run_defaults(r);
  FILE* f = fopen(path, "r");
  if (!f) return seterr("cannot open flow.dat");
  std::vector<std::string> lines;
  char buf[4096];
  while (fgets(buf, sizeof(buf), f)) lines.push_back(buf);
  fclose(f);
  size_t ln = 0;
  bool ok = true;
  auto rd = [&](double* v) {
    if (ln >= lines.size()) { ok = false; return; }
    if (!first_value(lines[ln], v)) ok = false;
    ++ln;
  };
  auto rdi = [&](int* v) { double d = 0; rd(&d); *v = (int)d; };
  auto skip = [&](int n) { ln += n; if (ln > lines.size()) ok = false; };
  double tmp, aspect;
  int scale_by_pi, itmp, nscalar;
  rd(&r->re); skip(3);
  rd(&r->ctrlu); rd(&r->ctrlw); rd(&r->lx); rd(&aspect); rdi(&scale_by_pi);
  rdi(&r->nx); rdi(&r->ny); rdi(&r->nz); rdi(&r->nx2); rdi(&r->nz2);
  rdi(&nscalar); skip(2);
  rdi(&itmp); rdi(&itmp); rdi(&itmp); rdi(&itmp); rdi(&itmp);   // split_scalar .. dynamic_scalar
  rdi(&r->tend); rdi(&r->output_step); rdi(&r->save_step); rdi(&r->l2_step);
  rdi(&r->read_vel); rdi(&r->save_vel); rdi(&r->vel_out); skip(1); rdi(&itmp); skip(1);
  rdi(&r->which_test); rd(&r->disturb_ampl); skip(10);
  rdi(&itmp); rdi(&r->fix_mass); rdi(&r->dt_flag); rdi(&r->divg_check); rd(&r->beta);
  skip(2); skip(1); rdi(&itmp); rdi(&itmp); rdi(&itmp); rdi(&itmp);
  skip(1); rdi(&r->bl_grid); rd(&tmp); rd(&tmp); rd(&tmp); rdi(&itmp);
  skip(1); rdi(&r->crossflow); rdi(&r->filter_jet_profile); skip(1); rd(&r->jet_diam); rd(&tmp);
  skip(2); rd(&r->xjet_top); rd(&r->zjet_top); rd(&r->jetmag_top); rd(&r->forcing_top); rd(&r->for_freq_top); rd(&tmp);
  skip(1); rd(&r->xjet_bot); rd(&r->zjet_bot); rd(&r->jetmag_bot); rd(&r->forcing_bot); rd(&r->for_freq_bot); rd(&tmp);
  skip(1); rd(&r->fringe_gain); skip(1); rdi(&r->xfringe); rd(&r->frac_xbuff); rd(&r->buff_xrise);
  rd(&r->buff_xfall);
  skip(1); rdi(&r->zfringe); rd(&r->frac_zbuff); rd(&r->buff_zrise); rd(&r->buff_zfall);
  if (!ok) return seterr("flow.dat: missing or malformed value before line 96");
  const double pi = atan2(0.0, -1.0);
  r->beta = r->beta * asin(1.0);
  if (scale_by_pi == 1) r->lx = r->lx * pi;
  r->lz = r->lx / aspect;
  // extension block (lines after 95, "value  name"); the Fortran reader ignores it
  for (size_t i = ln; i < lines.size(); ++i) {
    double v;
    if (!first_value(lines[i], &v)) continue;
    char name[64] = {0};
    if (sscanf(lines[i].c_str(), "%*s %63s", name) != 1) continue;
    std::string n(name);
    if (n == "stretch") r->stretch = v;
    else if (n == "dt") r->dt = v;
    else if (n == "seed") r->seed = (unsigned long long)v;
    else if (n == "precision") r->precision = (int)v;
    else if (n == "uniform_grid") r->uniform_grid = (int)v;
    else if (n == "jet_mode") r->jet_mode = (int)v;
    else if (n == "jet_width") r->jet_width = v;
    else if (n == "jet_peak") r->jet_peak = v;
    else if (n == "jet_freq") r->jet_freq = v;
    else if (n == "which_test") r->which_test = (int)v;
    else if (n == "disturb_ampl") r->disturb_ampl = v;
  }
  // which_test presets, PFC/setup.f90:163-201 (after the extension block,
  // which may set which_test)
  if (r->read_vel == 0) {
    if (r->which_test == 2) { r->re = 7500; r->lx = 2 * pi; r->beta = 0; r->fix_mass = 0; r->crossflow = 0; r->bl_grid = 0; r->xfringe = r->zfringe = 0; }
    else if (r->which_test == 5) { r->re = 7500; r->lz = 2 * pi; r->beta = pi / 2; r->fix_mass = 0; r->crossflow = 0; r->bl_grid = 0; r->xfringe = r->zfringe = 0; }
    else if (r->which_test == 8) { r->re = 7500; r->lx = 2 * sqrt(2.0) * pi; r->lz = r->lx; r->beta = pi / 4; r->fix_mass = 0; r->crossflow = 0; r->bl_grid = 0; r->xfringe = r->zfringe = 0; }
    else if (r->which_test == 6) { r->re = 10; r->lx = 2; r->fix_mass = 0; r->crossflow = 0; r->bl_grid = 0; r->xfringe = r->zfringe = 0; r->uniform_grid = 1; }
  }
  if (r->dt <= 0) {   // define_parameters, PFC/setup.f90:1377,1386-1393
    r->dt = 0.25 * r->lx / (double)r->nx;
    // the Orr-Sommerfeld runs: two periods of the mode in tend steps
    if (r->read_vel == 0 && r->which_test % 3 == 2 && r->tend >= 40)
      r->dt = 2.0 * (2.0 * pi / 0.24989154) / (double)r->tend;
    if (r->read_vel == 0 && r->which_test == 6) {
      r->dt = 0.5 / (double)r->ny;
      r->tend = (int)(1.0 / r->dt);
    }
  }
  if (r->nx < 4 || r->ny < 5 || r->nz < 4 || r->nx2 < r->nx || r->nz2 < r->nz) return seterr("flow.dat: bad grid size");
  return 0;
}

cfh_grid* cfh_grid_alloc(int nx, int ny, int nz, int nx2, int nz2) {
  cfh_grid* g = (cfh_grid*)calloc(1, sizeof(cfh_grid));
  g->nx = nx; g->ny = ny; g->nz = nz; g->nx2 = nx2; g->nz2 = nz2;
  const int nxh = nx / 2 + 1;
  auto A = [](size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); };
  g->y = A(ny); g->yh = A(ny + 1); g->hh = A(ny + 1); g->hn = A(ny); g->dh = A(ny + 1); g->dn = A(ny);
  g->iu = A(2 * ny); g->dm = A(12); g->d2h = A(3 * (ny + 1)); g->d2n = A(3 * ny); g->dyh = A(ny + 1);
  g->dy = A(ny + 1); g->kx = A(nxh); g->kz = A(nz); g->buffer = A((size_t)nx2 * nz2);
  g->target_inflow = A(3 * (ny + 1)); g->xcoord = A(nx + 1); g->zcoord = A(nz + 1);
  return g;
}

void cfh_grid_free(cfh_grid* g) {
  if (!g) return;
  double* v[] = {g->y, g->yh, g->hh, g->hn, g->dh, g->dn, g->iu, g->dm, g->d2h, g->d2n, g->dyh, g->dy,
                 g->kx, g->kz, g->buffer, g->target_inflow, g->xcoord, g->zcoord};
  for (double* p : v) free(p);
  free(g);
}

int cfh_define_grid(cfh_grid* g, double lx, double lz, double STRETCH, int uniform) {
  const int ny = g->ny, nx = g->nx, nz = g->nz, nxh = nx / 2 + 1;
  if (ny < 5) return -1;
  const double zero = 0.0, half = 0.5, one = 1.0, two = 2.0;
  const double pi = atan2(0.0, -1.0);
#define Y(i) g->y[(i)-1]
#define YH(i) g->yh[(i)-1]
#define HH(i) g->hh[(i)-1]
#define HN(i) g->hn[(i)-1]
#define DH(i) g->dh[(i)-1]
#define DN(i) g->dn[(i)-1]
#define DM(i, j) g->dm[((i)-1) + 3 * ((j)-1)]
#define D2H(i, j) g->d2h[((i)-1) + 3 * ((j)-1)]
#define D2N(i, j) g->d2n[((i)-1) + 3 * ((j)-1)]
  for (int x = 1; x <= nx + 1; ++x) g->xcoord[x - 1] = (double)(x - 1) * lx / (double)nx;
  for (int z = 1; z <= nz + 1; ++z) g->zcoord[z - 1] = (double)(z - 1) * lz / (double)nz;
  for (int p = 1; p <= ny; ++p) {
    const double xi = two * (double)(p - 1) / (double)(ny - 1) - one;
    Y(p) = tanh(STRETCH * xi) / tanh(STRETCH);
  }
  if (uniform) {
    Y(1) = -half;
    for (int p = 2; p <= ny - 1; ++p) Y(p) = Y(1) + (double)(p - 1) / (double)(ny - 1);
    Y(ny) = half;
  }
  YH(1) = Y(1);
  for (int j = 2; j <= ny; ++j) YH(j) = half * (Y(j - 1) + Y(j));
  YH(ny + 1) = Y(ny);
  HH(1) = Y(2) - Y(1);
  for (int j = 2; j <= ny; ++j) HH(j) = Y(j) - Y(j - 1);
  HH(ny + 1) = Y(ny) - Y(ny - 1);
  for (int j = 1; j <= ny + 1; ++j) DH(j) = one / HH(j);
  for (int j = 1; j <= ny; ++j) HN(j) = YH(j + 1) - YH(j);
  for (int j = 1; j <= ny; ++j) DN(j) = one / HN(j);
  for (int j = 1; j <= ny; ++j) {
    g->iu[2 * (j - 1)] = half * HH(j) / HN(j);
    g->iu[2 * (j - 1) + 1] = half * HH(j + 1) / HN(j);
  }
  DM(1, 1) = -(DN(1) * (two * HN(1) + HN(2)) / (HN(1) + HN(2)));
  DM(2, 1) = DN(1) * DN(2) * (HN(1) + HN(2));
  DM(3, 1) = -(DN(2) * HN(1) / (HN(1) + HN(2)));
  DM(1, 2) = DN(ny - 1) * HN(ny) / (HN(ny - 1) + HN(ny));
  DM(2, 2) = -(DN(ny) * DN(ny - 1) * (HN(ny) + HN(ny - 1)));
  DM(3, 2) = DN(ny) * (two * HN(ny) + HN(ny - 1)) / (HN(ny) + HN(ny - 1));
  DM(1, 3) = (Y(1) - Y(2) + Y(1) - Y(3)) / ((Y(1) - Y(2)) * (Y(1) - Y(3)));
  DM(2, 3) = (Y(1) - Y(3)) / ((Y(2) - Y(1)) * (Y(2) - Y(3)));
  DM(3, 3) = (Y(1) - Y(2)) / ((Y(3) - Y(1)) * (Y(3) - Y(2)));
  DM(1, 4) = (Y(ny) - Y(ny - 1)) / ((Y(ny - 2) - Y(ny)) * (Y(ny - 2) - Y(ny - 1)));
  DM(2, 4) = (Y(ny) - Y(ny - 2)) / ((Y(ny - 1) - Y(ny)) * (Y(ny - 1) - Y(ny - 2)));
  DM(3, 4) = (Y(ny) - Y(ny - 1) + Y(ny) - Y(ny - 2)) / ((Y(ny) - Y(ny - 1)) * (Y(ny) - Y(ny - 2)));
  for (int p = 2; p <= ny - 1; ++p) {
    D2N(1, p) = DN(p) * DH(p);
    D2N(2, p) = -(DN(p) * DH(p)) - DN(p) * DH(p + 1);
    D2N(3, p) = DN(p) * DH(p + 1);
    D2H(1, p) = DH(p) * DN(p - 1);
    D2H(2, p) = -(DH(p) * DN(p - 1)) - DH(p) * DN(p);
    D2H(3, p) = DH(p) * DN(p);
  }
  D2H(1, 2) = -(DH(2) * DM(1, 1));
  D2H(2, 2) = -(DH(2) * DN(2)) - DH(2) * DM(2, 1);
  D2H(3, 2) = DH(2) * DN(2) - DH(2) * DM(3, 1);
  D2H(1, ny) = DH(ny) * DN(ny - 1) + DH(ny) * DM(1, 2);
  D2H(2, ny) = -(DH(ny) * DN(ny - 1)) + DH(ny) * DM(2, 2);
  D2H(3, ny) = DH(ny) * DM(3, 2);
  for (int i = 1; i <= 3; ++i) {
    D2H(i, 1) = D2H(i, 2);
    D2N(i, 1) = D2N(i, 2);
    D2N(i, ny) = D2N(i, ny - 1);
    D2H(i, ny + 1) = D2H(i, ny);
  }
  g->dyh[0] = zero;
  for (int j = 2; j <= ny; ++j) g->dyh[j - 1] = HH(j);
  g->dyh[ny] = zero;
  g->dy[0] = half * HH(2);
  for (int j = 2; j <= ny - 1; ++j) g->dy[j - 1] = half * (HH(j) + HH(j + 1));
  g->dy[ny - 1] = half * HH(ny);
  g->dy[ny] = zero;
  for (int x = 1; x <= nxh; ++x) g->kx[x - 1] = (double)(x - 1) * 2.0 * pi / lx;
  for (int z = 1; z <= nz / 2 + 1; ++z) g->kz[z - 1] = (double)(z - 1) * 2.0 * pi / lz;
  for (int z = nz; z >= nz / 2 + 2; --z) g->kz[z - 1] = -g->kz[nz + 2 - z - 1];
#undef Y
#undef YH
#undef HH
#undef HN
#undef DH
#undef DN
#undef DM
#undef D2H
#undef D2N
  return 0;
}

static uint64_t smix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

double cfh_rng_u01(unsigned long long seed, int x, int z, int j, int col) {
  const uint64_t ctr = ((((uint64_t)x * 65536u + (uint64_t)z) * 65536u + (uint64_t)j) * 8u) + (uint64_t)col;
  const uint64_t h = smix((uint64_t)seed ^ smix(ctr));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

int cfh_initial_field(const cfh_grid* g, int which_test, unsigned long long seed, double ampl, double beta,
                      double* data1) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, nxh = nx / 2 + 1, n1 = ny + 1;
  const double pi = atan2(0.0, -1.0);
  cd* d1 = reinterpret_cast<cd*>(data1);
  const size_t nf = (size_t)nz * nxh * n1;
  for (size_t i = 0; i < 3 * nf; ++i) d1[i] = 0.0;
  auto D1 = [&](int z, int x, int j, int c) -> cd& { return d1[z + (size_t)nz * (x + (size_t)nxh * (j + (size_t)n1 * c))]; };
  if (which_test == 1 || which_test == 10) {
    for (int j = 0; j < n1; ++j) {
      const double yh = g->yh[j];
      D1(0, 0, j, 0) = (1.0 - yh * yh) * cos(beta);
      D1(0, 0, j, 2) = (1.0 - yh * yh) * sin(beta);
    }
  } else if (which_test == 4) {
    for (int j = 0; j < n1; ++j) D1(0, 0, j, 0) = 0.75 * (1.0 - pow(g->yh[j], 8));
  } else if (which_test == 6) {
    for (int j = 0; j < n1; ++j) D1(0, 1, j, 0) = -0.5 * sin(pi * g->yh[j]);
    for (int j = 0; j < ny; ++j) D1(0, 1, j, 1) = cd(0.0, -0.5 * cos(pi * g->y[j]));
  } else if (which_test != 0) {
    return -1;
  }
  if (which_test == 4 || which_test == 10) {
    // random_divfree_vector(filter=0) * min(1, 1/k^2), PFC/init_vel.f90:217-225,357-432
    std::vector<cd> cu(3 * (size_t)n1), uo(n1);
    for (int x = 0; x < nxh; ++x)
      for (int z = 0; z < nz; ++z) {
        const double k2 = g->kx[x] * g->kx[x] + g->kz[z] * g->kz[z];
        if (k2 == 0.0) continue;
        double temp[4][1200];
        for (int col = 0; col < 4; ++col)
          for (int j = 0; j < n1; ++j) temp[col][j] = 2.0 * (cfh_rng_u01(seed, x, z, j, col) - 0.5);
        for (int j = 0; j < n1; ++j) cu[j] = cd(temp[0][j], temp[1][j]);
        for (int j = 0; j < ny; ++j) cu[n1 + j] = cd(temp[2][j], temp[3][j]);
        cu[n1 + ny] = 0.0;
        const cd ikx(0.0, g->kx[x]), ikz(0.0, g->kz[z]);
        for (int j = 0; j < n1; ++j) uo[j] = cu[j];
        cu[2 * n1] = 0.0;
        for (int j = 2; j <= ny; ++j)
          cu[2 * n1 + j - 1] = (ikx * uo[j - 1] + ikz * g->dh[j - 1] * (cu[n1 + j - 1] - cu[n1 + j - 2])) / k2;
        cu[2 * n1 + ny] = 0.0;
        cu[0] = 0.0;
        for (int j = 2; j <= ny; ++j)
          cu[j - 1] = (-ikz * uo[j - 1] + ikx * g->dh[j - 1] * (cu[n1 + j - 1] - cu[n1 + j - 2])) / k2;
        cu[ny] = 0.0;
        double tmp = 0;
        for (int j = 2; j <= ny; ++j)
          tmp += g->dyh[j - 1] * (std::abs(cu[j - 1]) + std::abs(cu[2 * n1 + j - 1]) + 0.5 * std::abs(cu[n1 + j - 2]) +
                                  0.5 * std::abs(cu[n1 + j - 1]));
        if (tmp > 0.0)
          for (auto& v : cu) v = ampl * v / tmp;
        const double f = 1.0 / k2 < 1.0 ? 1.0 / k2 : 1.0;
        for (int c = 0; c < 3; ++c)
          for (int j = 0; j < n1; ++j) D1(z, x, j, c) = cu[c * n1 + j] * f;
      }
  }
  return 0;
}

int cfh_read_efn(const char* path, double* uin) {
  FILE* f = fopen(path, "r");
  if (!f) return -1;
  char tok[128];
  int n = 0;
  while (n < 4 * 65 && fscanf(f, "%127s", tok) == 1) {
    for (char* p = tok; *p; ++p)
      if (*p == 'D' || *p == 'd') *p = 'e';   // Fortran double-precision exponent
    char* end = nullptr;
    const double v = strtod(tok, &end);
    if (end == tok || *end != '\0') break;
    uin[n++] = v;
  }
  fclose(f);
  return n == 4 * 65 ? 0 : -2;
}

int cfh_interp_eigenfunction(const cfh_grid* g, const double* uin, double* u, double* v) {
  constexpr int nc = 65;
  const int ny = g->ny, n1 = ny + 1;
  const double nn = nc - 1, pi = atan2(0.0, -1.0);
  // Chebyshev coefficients: T(i,j) = (2/N) cos(pi (i-1)(j-1) / N), halved on
  // the first and last row and column
  double ucheb[nc][4] = {};
  for (int i = 0; i < nc; ++i)
    for (int j = 0; j < nc; ++j) {
      double t = (2.0 / nn) * cos(pi * (double)(i * j) / nn);
      if (i == 0 || i == nc - 1) t *= 0.5;
      if (j == 0 || j == nc - 1) t *= 0.5;
      for (int k = 0; k < 4; ++k) ucheb[i][k] += t * uin[j + nc * k];
    }
  auto series = [&](double y, int k) {
    const double th = acos(y < -1.0 ? -1.0 : y > 1.0 ? 1.0 : y);
    double s = 0.0;
    for (int j = 0; j < nc; ++j) s += cos((double)j * th) * ucheb[j][k];
    return s;
  };
  for (int p = 0; p < 2 * n1; ++p) u[p] = v[p] = 0.0;
  for (int p = 1; p < ny; ++p) {   // yh(2..ny)
    u[2 * p] = series(g->yh[p], 0);
    u[2 * p + 1] = series(g->yh[p], 1);
  }
  for (int p = 0; p < ny; ++p) {   // y(1..ny)
    v[2 * p] = series(g->y[p], 2);
    v[2 * p + 1] = series(g->y[p], 3);
  }
  return 0;
}

int cfh_initial_field_mode(const cfh_grid* g, int which_test, double ampl, double beta, const double* u,
                           const double* v, double* data1) {
  if (which_test != 2 && which_test != 5 && which_test != 8) return -1;
  const int nx = g->nx, ny = g->ny, nz = g->nz, nxh = nx / 2 + 1, n1 = ny + 1;
  if (nxh < 2 || nz < 2) return -1;
  cd* d1 = reinterpret_cast<cd*>(data1);
  const cd* uu = reinterpret_cast<const cd*>(u);
  const cd* vv = reinterpret_cast<const cd*>(v);
  const size_t nf = (size_t)nz * nxh * n1;
  for (size_t i = 0; i < 3 * nf; ++i) d1[i] = 0.0;
  auto D1 = [&](int z, int x, int j, int c) -> cd& { return d1[z + (size_t)nz * (x + (size_t)nxh * (j + (size_t)n1 * c))]; };
  for (int j = 0; j < n1; ++j) {
    const double lam = 1.0 - g->yh[j] * g->yh[j];
    if (which_test == 2) D1(0, 0, j, 0) = lam;
    else if (which_test == 5) D1(0, 0, j, 2) = lam;
    else { D1(0, 0, j, 0) = lam * cos(beta); D1(0, 0, j, 2) = lam * sin(beta); }
  }
  if (which_test == 2) {          // (z 1, x 2)
    for (int j = 0; j < n1; ++j) D1(0, 1, j, 0) = ampl * uu[j];
    for (int j = 0; j < ny; ++j) D1(0, 1, j, 1) = ampl * vv[j];
  } else if (which_test == 5) {   // (z 2, x 1) and its conjugate (z nz, x 1)
    for (int j = 0; j < n1; ++j) {
      D1(1, 0, j, 2) = ampl * uu[j];
      D1(nz - 1, 0, j, 2) = ampl * std::conj(uu[j]);
    }
    for (int j = 0; j < ny; ++j) {
      D1(1, 0, j, 1) = ampl * vv[j];
      D1(nz - 1, 0, j, 1) = ampl * std::conj(vv[j]);
    }
  } else {                        // (z 2, x 2), rotated by beta
    for (int j = 0; j < n1; ++j) {
      D1(1, 1, j, 0) = ampl * uu[j] * cos(beta);
      D1(1, 1, j, 2) = ampl * uu[j] * sin(beta);
    }
    for (int j = 0; j < ny; ++j) D1(1, 1, j, 1) = ampl * vv[j];
  }
  return 0;
}

}  // extern "C"
