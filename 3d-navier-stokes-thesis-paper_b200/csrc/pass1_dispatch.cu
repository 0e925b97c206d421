// pass1_dispatch.cu -- selects the per-length translation unit.
#include "pass1_fast.h"

namespace cfd {
int p1_fast_launch_24(int which, bool f32, const P1Launch& a, const P1Launch* tab, int nmem);
size_t p1_fast_smem_24(int which, bool f32, int param, int nxh, int nz);
int p1_fast_launch_48(int which, bool f32, const P1Launch& a, const P1Launch* tab, int nmem);
size_t p1_fast_smem_48(int which, bool f32, int param, int nxh, int nz);
int p1_fast_launch_72(int which, bool f32, const P1Launch& a, const P1Launch* tab, int nmem);
size_t p1_fast_smem_72(int which, bool f32, int param, int nxh, int nz);
int p1_fast_launch_96(int which, bool f32, const P1Launch& a, const P1Launch* tab, int nmem);
size_t p1_fast_smem_96(int which, bool f32, int param, int nxh, int nz);
int p1_fast_launch_144(int which, bool f32, const P1Launch& a, const P1Launch* tab, int nmem);
size_t p1_fast_smem_144(int which, bool f32, int param, int nxh, int nz);
int p1_fast_launch_192(int which, bool f32, const P1Launch& a, const P1Launch* tab, int nmem);
size_t p1_fast_smem_192(int which, bool f32, int param, int nxh, int nz);
int p1_fast_launch_288(int which, bool f32, const P1Launch& a, const P1Launch* tab, int nmem);
size_t p1_fast_smem_288(int which, bool f32, int param, int nxh, int nz);
int p1_fast_launch_384(int which, bool f32, const P1Launch& a, const P1Launch* tab, int nmem);
size_t p1_fast_smem_384(int which, bool f32, int param, int nxh, int nz);
int p1_fast_launch_576(int which, bool f32, const P1Launch& a, const P1Launch* tab, int nmem);
size_t p1_fast_smem_576(int which, bool f32, int param, int nxh, int nz);

int p1_fast_launch(int which, int n, bool f32, const P1Launch& a) {
  return p1_fast_launch_batch(which, n, f32, a, nullptr, 0);
}

int p1_fast_launch_batch(int which, int n, bool f32, const P1Launch& a, const P1Launch* tab, int nmem) {
  switch (n) {
    case 24: return p1_fast_launch_24(which, f32, a, tab, nmem);
    case 48: return p1_fast_launch_48(which, f32, a, tab, nmem);
    case 72: return p1_fast_launch_72(which, f32, a, tab, nmem);
    case 96: return p1_fast_launch_96(which, f32, a, tab, nmem);
    case 144: return p1_fast_launch_144(which, f32, a, tab, nmem);
    case 192: return p1_fast_launch_192(which, f32, a, tab, nmem);
    case 288: return p1_fast_launch_288(which, f32, a, tab, nmem);
    case 384: return p1_fast_launch_384(which, f32, a, tab, nmem);
    case 576: return p1_fast_launch_576(which, f32, a, tab, nmem);
    default: return -1;
  }
}

size_t p1_fast_smem(int which, int n, bool f32, int param, int nxh, int nz) {
  switch (n) {
    case 24: return p1_fast_smem_24(which, f32, param, nxh, nz);
    case 48: return p1_fast_smem_48(which, f32, param, nxh, nz);
    case 72: return p1_fast_smem_72(which, f32, param, nxh, nz);
    case 96: return p1_fast_smem_96(which, f32, param, nxh, nz);
    case 144: return p1_fast_smem_144(which, f32, param, nxh, nz);
    case 192: return p1_fast_smem_192(which, f32, param, nxh, nz);
    case 288: return p1_fast_smem_288(which, f32, param, nxh, nz);
    case 384: return p1_fast_smem_384(which, f32, param, nxh, nz);
    case 576: return p1_fast_smem_576(which, f32, param, nxh, nz);
    default: return 0;
  }
}

}  // namespace cfd
