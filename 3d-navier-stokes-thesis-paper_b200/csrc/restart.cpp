// restart.cpp -- the restart file of read_write::save_velocity /
// read_velocity (PFC/read_write.f90:21-292) and the VTK velocity snapshot of
// output_hdf_dfsd (PFC/read_write.f90:296-500), host side.
//
// Restart file: Fortran unformatted sequential records, each framed by a
// 4-byte record length before and after (the gfortran/ifort default), native
// byte order:
//   record 1      NX, NY, NZ (int32), LX, LZ, RE, DT, T_TOTAL (float64)
//   records 2..   one per kx = 1..nx/2+1: slice(nz, ny+1, 3) complex(8),
//                 i.e. data1(1:nz, kx, 1:ny+1, 1:3)
//   last record   lagr_avg, ndynscalar (int32) = 0, 0 (no dynamic SGS data)
// There are no scalar records (nscalar = 0).
//
// VTK snapshot ("t_###.vtk"): legacy VTK, rectilinear grid, BINARY, big-endian
// float32: the header lines, nx x coordinates, ny+1 yh coordinates, nz z
// coordinates, then POINT_DATA nx*(ny+1)*nz with VECTORS flowvec float
// ordered (u, v, w) fastest, then x, then the plane, then z.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "chanflow.h"
#include "chanflow_host.h"
#include "restart.h"

namespace {

void set_err(char* err, int errlen, const std::string& m) {
  if (err && errlen > 0) {
    std::snprintf(err, (size_t)errlen, "%s", m.c_str());
  }
}

bool put_record(FILE* f, const void* p, size_t n) {
  if (n > 0x7fffffffULL) return false;
  const int32_t m = (int32_t)n;
  return std::fwrite(&m, 4, 1, f) == 1 && (n == 0 || std::fwrite(p, 1, n, f) == n) && std::fwrite(&m, 4, 1, f) == 1;
}

// reads one record of exactly n bytes
bool get_record(FILE* f, void* p, size_t n, std::string& why) {
  int32_t m0 = 0, m1 = 0;
  if (std::fread(&m0, 4, 1, f) != 1) {
    why = "unexpected end of file";
    return false;
  }
  if (m0 < 0 || (size_t)m0 != n) {
    why = "record of " + std::to_string(m0) + " bytes where " + std::to_string(n) + " were expected";
    return false;
  }
  if (std::fread(p, 1, n, f) != n || std::fread(&m1, 4, 1, f) != 1 || m1 != m0) {
    why = "truncated or malformed record";
    return false;
  }
  return true;
}

struct Header {
  int32_t nx, ny, nz;
  double lx, lz, re, dt, t_total;
};

bool put_header(FILE* f, const Header& h) {
  unsigned char b[52];
  std::memcpy(b, &h.nx, 4);
  std::memcpy(b + 4, &h.ny, 4);
  std::memcpy(b + 8, &h.nz, 4);
  std::memcpy(b + 12, &h.lx, 8);
  std::memcpy(b + 20, &h.lz, 8);
  std::memcpy(b + 28, &h.re, 8);
  std::memcpy(b + 36, &h.dt, 8);
  std::memcpy(b + 44, &h.t_total, 8);
  return put_record(f, b, sizeof(b));
}

bool get_header(FILE* f, Header& h, std::string& why) {
  unsigned char b[52];
  if (!get_record(f, b, sizeof(b), why)) return false;
  std::memcpy(&h.nx, b, 4);
  std::memcpy(&h.ny, b + 4, 4);
  std::memcpy(&h.nz, b + 8, 4);
  std::memcpy(&h.lx, b + 12, 8);
  std::memcpy(&h.lz, b + 20, 8);
  std::memcpy(&h.re, b + 28, 8);
  std::memcpy(&h.dt, b + 36, 8);
  std::memcpy(&h.t_total, b + 44, 8);
  return true;
}

// the consistency checks of read_velocity (PFC/read_write.f90:41-55)
bool check_header(const Header& h, int nx, int ny, int nz, double lx, double lz, std::string& why) {
  const double eps = 2.220446049250313e-16;   // EPSILON(1.0d0)
  auto bad_int = [&](const char* n, int t, int v) {
    why = std::string("INCONSISTENT PARAMETERS: ") + n + " HAS BEEN CHANGED FROM " + std::to_string(t) + " TO " +
          std::to_string(v);
  };
  if (h.nx != nx) { bad_int("NX", h.nx, nx); return false; }
  if (h.ny != ny) { bad_int("NY", h.ny, ny); return false; }
  if (h.nz != nz) { bad_int("NZ", h.nz, nz); return false; }
  char buf[160];
  if (std::fabs(lx - h.lx) > lx * eps) {
    std::snprintf(buf, sizeof(buf), "INCONSISTENT PARAMETERS: LX HAS BEEN CHANGED FROM %10.5f TO %10.5f", h.lx, lx);
    why = buf;
    return false;
  }
  if (std::fabs(lz - h.lz) > lz * eps) {
    std::snprintf(buf, sizeof(buf), "INCONSISTENT PARAMETERS: LZ HAS BEEN CHANGED FROM %10.5f TO %10.5f", h.lz, lz);
    why = buf;
    return false;
  }
  return true;
}

void be32(unsigned char* d, float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  d[0] = (unsigned char)(u >> 24);
  d[1] = (unsigned char)(u >> 16);
  d[2] = (unsigned char)(u >> 8);
  d[3] = (unsigned char)u;
}

}  // namespace

namespace cfd_io {

int write_restart_slabs(const char* path, int nx, int ny, int nz, double lx, double lz, double re, double dt,
                        double t_total, const double* slabs, std::string& why) {
  const int nxh = nx / 2 + 1;
  const size_t slab = (size_t)nz * (ny + 1) * 3 * 16;
  if (slab > 0x7fffffffULL) {
    why = "a kx slice exceeds the 2 GiB record limit of the file layout";
    return CFG_E_ARG;
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    why = std::string("cannot open ") + path + ": " + std::strerror(errno);
    return CFG_E_ARG;
  }
  Header h{nx, ny, nz, lx, lz, re, dt, t_total};
  bool ok = put_header(f, h);
  for (int x = 0; ok && x < nxh; ++x) ok = put_record(f, reinterpret_cast<const char*>(slabs) + slab * x, slab);
  const int32_t tail[2] = {0, 0};
  ok = ok && put_record(f, tail, sizeof(tail));
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    why = std::string("write error on ") + path;
    return CFG_E_ARG;
  }
  return CFG_OK;
}

int read_restart_slabs(const char* path, int nx, int ny, int nz, double lx, double lz, double re, double* dt,
                       double* t_total, double* slabs, std::string& why) {
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    why = std::string("cannot open ") + path + ": " + std::strerror(errno);
    return CFG_E_ARG;
  }
  Header h{};
  bool ok = get_header(f, h, why) && check_header(h, nx, ny, nz, lx, lz, why);
  if (ok && std::fabs(re - h.re) > re * 2.220446049250313e-16)
    std::fprintf(stderr, "REYNOLDS NUMBER CHANGED TO%12.4f  FROM %12.4f\n", re, h.re);
  const int nxh = nx / 2 + 1;
  const size_t slab = (size_t)nz * (ny + 1) * 3 * 16;
  for (int x = 0; ok && x < nxh; ++x) ok = get_record(f, reinterpret_cast<char*>(slabs) + slab * x, slab, why);
  std::fclose(f);
  if (!ok) {
    if (why.empty()) why = "malformed restart file";
    why = std::string(path) + ": " + why;
    return CFG_E_ARG;
  }
  if (dt) *dt = h.dt;
  if (t_total) *t_total = h.t_total;
  return CFG_OK;
}

int write_vtk(const char* path, int nx, int ny, int nz, double lx, double lz, const double* yh,
              const unsigned char* vec_be, int derived, std::string& why) {
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    why = std::string("cannot open ") + path + ": " + std::strerror(errno);
    return CFG_E_ARG;
  }
  const int n1 = ny + 1;
  // CHARACTER(LEN=30) lines as the reference writes them: the literal, the
  // number written into its columns, blank padding to 30, then a line feed
  auto line30 = [](const char* lit, int col, const char* num) {
    std::string l(30, ' ');
    for (size_t i = 0; lit[i] && i < 30; ++i) l[i] = lit[i];
    for (size_t i = 0; num[i] && col - 1 + i < 30; ++i) l[col - 1 + i] = num[i];
    return l + "\n";
  };
  std::string head = "# vtk DataFile Version 2.0\n(This is header line) vtk rectilinear grid with binary data\n"
                     "BINARY\nDATASET RECTILINEAR_GRID\n";
  char num[32];
  std::snprintf(num, sizeof(num), "%5d%5d%5d", nx, n1, nz);
  head += line30("DIMENSIONS", 12, num);
  bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
  auto coords = [&](const char* lit, int n, auto value) {
    char k[16];
    std::snprintf(k, sizeof(k), "%3d", n);
    const std::string l = line30(lit, 15, k);
    std::vector<unsigned char> b((size_t)n * 4 + 1);
    for (int i = 0; i < n; ++i) be32(&b[(size_t)i * 4], (float)value(i));
    b[(size_t)n * 4] = '\n';
    ok = ok && std::fwrite(l.data(), 1, l.size(), f) == l.size() && std::fwrite(b.data(), 1, b.size(), f) == b.size();
  };
  coords("X_COORDINATES     float", nx, [&](int x) { return lx * (double)x / (double)nx; });
  coords("Y_COORDINATES     float", n1, [&](int j) { return yh[j]; });
  coords("Z_COORDINATES     float", nz, [&](int z) { return lz * (double)z / (double)nz; });
  const size_t npts = (size_t)nx * n1 * nz;
  std::snprintf(num, sizeof(num), "%9zu", npts);
  const std::string pd = line30("POINT_DATA", 12, num);
  const char* vec = "VECTORS flowvec float\n";
  ok = ok && std::fwrite(pd.data(), 1, pd.size(), f) == pd.size() &&
       std::fwrite(vec, 1, std::strlen(vec), f) == std::strlen(vec) &&
       std::fwrite(vec_be, 1, npts * 12, f) == npts * 12 && std::fputc('\n', f) != EOF;
  if (derived) {
    // vorticity, Q-criterion and discriminant behind the velocity, same
    // point order (the reference snapshot stops after flowvec)
    const unsigned char* d = vec_be + npts * 12;
    const char* vor = "VECTORS vorticity float\n";
    const char* qh = "SCALARS Q float 1\nLOOKUP_TABLE default\n";
    const char* dh = "SCALARS D float 1\nLOOKUP_TABLE default\n";
    ok = ok && std::fwrite(vor, 1, std::strlen(vor), f) == std::strlen(vor) &&
         std::fwrite(d, 1, npts * 12, f) == npts * 12 && std::fputc('\n', f) != EOF &&
         std::fwrite(qh, 1, std::strlen(qh), f) == std::strlen(qh) &&
         std::fwrite(d + npts * 12, 1, npts * 4, f) == npts * 4 && std::fputc('\n', f) != EOF &&
         std::fwrite(dh, 1, std::strlen(dh), f) == std::strlen(dh) &&
         std::fwrite(d + npts * 16, 1, npts * 4, f) == npts * 4 && std::fputc('\n', f) != EOF;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    why = std::string("write error on ") + path;
    return CFG_E_ARG;
  }
  return CFG_OK;
}

}  // namespace cfd_io

// host arrays in data1 layout (nz, nx/2+1, ny+1, 3)
extern "C" int cfh_save_velocity(const char* path, int nx, int ny, int nz, double lx, double lz, double re,
                                 double dt, double t_total, const double* data1, char* err, int errlen) {
  if (!path || !data1 || nx < 2 || ny < 2 || nz < 2) return CFG_E_ARG;
  const int nxh = nx / 2 + 1, n1 = ny + 1;
  std::vector<double> slabs((size_t)nz * n1 * 3 * nxh * 2);
  for (int c = 0; c < 3; ++c)
    for (int j = 0; j < n1; ++j)
      for (int x = 0; x < nxh; ++x)
        for (int z = 0; z < nz; ++z) {
          const size_t src = z + (size_t)nz * (x + (size_t)nxh * (j + (size_t)n1 * c));
          const size_t dst = (size_t)x * nz * n1 * 3 + z + (size_t)nz * (j + (size_t)n1 * c);
          slabs[2 * dst] = data1[2 * src];
          slabs[2 * dst + 1] = data1[2 * src + 1];
        }
  std::string why;
  const int r = cfd_io::write_restart_slabs(path, nx, ny, nz, lx, lz, re, dt, t_total, slabs.data(), why);
  if (r) set_err(err, errlen, why);
  return r;
}

extern "C" int cfh_read_velocity(const char* path, int nx, int ny, int nz, double lx, double lz, double re,
                                 double* dt, double* t_total, double* data1, char* err, int errlen) {
  if (!path || !data1 || nx < 2 || ny < 2 || nz < 2) return CFG_E_ARG;
  const int nxh = nx / 2 + 1, n1 = ny + 1;
  std::vector<double> slabs((size_t)nz * n1 * 3 * nxh * 2);
  std::string why;
  const int r = cfd_io::read_restart_slabs(path, nx, ny, nz, lx, lz, re, dt, t_total, slabs.data(), why);
  if (r) {
    set_err(err, errlen, why);
    return r;
  }
  for (int c = 0; c < 3; ++c)
    for (int j = 0; j < n1; ++j)
      for (int x = 0; x < nxh; ++x)
        for (int z = 0; z < nz; ++z) {
          const size_t dst = z + (size_t)nz * (x + (size_t)nxh * (j + (size_t)n1 * c));
          const size_t src = (size_t)x * nz * n1 * 3 + z + (size_t)nz * (j + (size_t)n1 * c);
          data1[2 * dst] = slabs[2 * src];
          data1[2 * dst + 1] = slabs[2 * src + 1];
        }
  return CFG_OK;
}
