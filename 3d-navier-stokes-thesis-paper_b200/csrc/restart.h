// restart.h -- host-side writers/readers of the restart file and the VTK
// snapshot (restart.cpp), shared by the C ABI (capi.cu) and chanflow_host.h.
#pragma once
#include <string>

namespace cfd_io {

// slabs: nx/2+1 consecutive records of (nz, ny+1, 3) complex doubles
int write_restart_slabs(const char* path, int nx, int ny, int nz, double lx, double lz, double re, double dt,
                        double t_total, const double* slabs, std::string& why);
int read_restart_slabs(const char* path, int nx, int ny, int nz, double lx, double lz, double re, double* dt,
                       double* t_total, double* slabs, std::string& why);
// vec_be: nx*(ny+1)*nz*3 big-endian float32 values, (u,v,w) fastest, then x,
// the plane, z; with `derived`, followed by the vorticity (3 per point), Q
// and D (1 per point) in the same order
int write_vtk(const char* path, int nx, int ny, int nz, double lx, double lz, const double* yh,
              const unsigned char* vec_be, int derived, std::string& why);

}  // namespace cfd_io
