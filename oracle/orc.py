"""ctypes wrapper of the CPU oracle (oracle/_build/liborc.so).

TEST INFRASTRUCTURE ONLY: the FP64 restatement of the reference solver that the
CUDA product is checked against.  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use it.  Arrays are exposed as numpy views in the
reference's Fortran layouts (order='F').
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liborc.so")


class OrcParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nx2", C.c_int), ("nz2", C.c_int),
        ("re", C.c_double), ("lx", C.c_double), ("lz", C.c_double), ("beta", C.c_double),
        ("dt", C.c_double), ("cfl_max", C.c_double),
        ("fix_mass", C.c_int), ("dt_flag", C.c_int),
        ("ctrlu", C.c_double), ("ctrlw", C.c_double),
        ("stretch", C.c_double),
        ("uniform_grid", C.c_int), ("nthreads", C.c_int),
    ]


class OrcJet(C.Structure):
    """orc_jet: index 0 of the per-wall pairs is the bottom wall, 1 the top."""
    _fields_ = [
        ("mode", C.c_int),
        ("xjet", C.c_double * 2), ("zjet", C.c_double * 2),
        ("jetmag", C.c_double * 2), ("forcing", C.c_double * 2), ("for_freq", C.c_double * 2),
        ("jet_diam", C.c_double),
        ("width", C.c_double), ("freq", C.c_double),
        ("frac_xbuff", C.c_double),
        ("filter_jet_profile", C.c_int),
        ("jet_forcing", C.c_double * 24),
        ("jet_forcing_incr", C.c_double * 24),
        ("seed", C.c_ulonglong),
    ]


def build():
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [vp]
        L.orc_grid.restype = dp
        L.orc_grid.argtypes = [vp, C.c_char_p, ip]
        for n in ("orc_data1", "orc_data2", "orc_data4", "orc_cbc_top", "orc_cbc_bot",
                  "orc_buffer", "orc_target_inflow", "orc_baseflow", "orc_d_um_dy", "orc_cfl"):
            getattr(L, n).restype = dp
            getattr(L, n).argtypes = [vp]
        L.orc_get_scalars.argtypes = [vp, dp, dp, dp]
        L.orc_set_scalars.argtypes = [vp, C.c_double, C.c_double, C.c_double]
        L.orc_set_step.argtypes = [vp, C.c_int, C.c_int]
        L.orc_status.argtypes = [vp]
        L.orc_status.restype = C.c_int
        L.orc_fft.argtypes = [C.c_int, C.c_int, vp, vp]
        for n in ("orc_xz_c2r", "orc_xz_r2c", "orc_small_r2c", "orc_small_c2r"):
            getattr(L, n).argtypes = [vp, vp, vp]
        L.orc_div_fluxes.argtypes = [vp, vp, vp, vp, vp]
        for n in ("orc_nonlinear", "orc_nonlinear_linearized", "orc_rhs_solve", "orc_boundary",
                  "orc_remove_initial_divergence", "orc_compute_d_um_dy", "orc_init_from_velocity"):
            getattr(L, n).argtypes = [vp]
        L.orc_l2_norm.argtypes = [vp, dp, dp]
        L.orc_init_field.argtypes = [vp, C.c_int, C.c_ulonglong, C.c_double]
        L.orc_initial_velocity.argtypes = [vp, C.c_int, C.c_ulonglong, C.c_double]
        L.orc_rng_u01.argtypes = [C.c_ulonglong, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_rng_u01.restype = C.c_double
        L.orc_compute_initial_pressure.argtypes = [vp, C.c_int]
        L.orc_timestep.argtypes = [vp, C.c_int, C.c_int]
        L.orc_bulk_flux.argtypes = [vp]
        L.orc_bulk_flux.restype = C.c_double
        L.orc_max_divergence.argtypes = [vp]
        L.orc_max_divergence.restype = C.c_double
        L.orc_set_jet.argtypes = [vp, C.POINTER(OrcJet)]
        L.orc_jet_profile.argtypes = [vp, C.c_double, C.c_double]
        L.orc_get_jet_forcing.argtypes = [vp, vp, vp]
        L.orc_arnoldi_matvec.argtypes = [vp, C.c_int, vp, vp]
        _lib = L
    return _lib


def fft(x, sign):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    lib().orc_fft(len(x), sign, x.ctypes.data, out.ctypes.data)
    return out


def _view(ptr, shape, dtype):
    n = int(np.prod(shape))
    if dtype == np.complex128:
        a = np.ctypeslib.as_array(ptr, shape=(2 * n,)).view(np.complex128)
    else:
        a = np.ctypeslib.as_array(ptr, shape=(n,))
    return a.reshape(shape, order="F")


class Oracle:
    """One oracle context: grid, state and the reference's hot-path routines."""

    def __init__(self, nx, ny, nz, nx2=None, nz2=None, re=2500.0, lx=4 * np.pi,
                 lz=2 * np.pi, beta=0.0, dt=0.005, cfl_max=0.95, fix_mass=1, dt_flag=0,
                 ctrlu=0.0, ctrlw=0.0, stretch=1.5, uniform_grid=0, nthreads=0):
        nx2 = nx2 or 3 * nx // 2
        nz2 = nz2 or 3 * nz // 2
        self.p = OrcParams(nx, ny, nz, nx2, nz2, re, lx, lz, beta, dt, cfl_max, fix_mass,
                           dt_flag, ctrlu, ctrlw, stretch, uniform_grid, nthreads)
        self.L = lib()
        self.h = self.L.orc_create(C.byref(self.p))
        self.nx, self.ny, self.nz, self.nx2, self.nz2 = nx, ny, nz, nx2, nz2
        self.nxh = nx // 2 + 1

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- accessors
    def grid(self, name):
        n = C.c_int(0)
        p = self.L.orc_grid(self.h, name.encode(), C.byref(n))
        a = np.ctypeslib.as_array(p, shape=(n.value,)).copy()
        if name in ("d2h", "d2n", "dm", "iu", "d2m"):
            rows = {"d2h": 3, "d2n": 3, "dm": 3, "iu": 2, "d2m": 4}[name]
            a = a.reshape((rows, -1), order="F")
        if name == "k2":
            a = a.reshape((self.nz, self.nxh), order="F")
        return a

    @property
    def data1(self):
        return _view(self.L.orc_data1(self.h), (self.nz, self.nxh, self.ny + 1, 3), np.complex128)

    @property
    def data2(self):
        return _view(self.L.orc_data2(self.h), (self.ny + 1, 3, self.nz, self.nxh), np.complex128)

    @property
    def data4(self):
        return _view(self.L.orc_data4(self.h), (self.ny + 1, self.nz, self.nxh), np.complex128)

    @property
    def cbc_top(self):
        return _view(self.L.orc_cbc_top(self.h), (self.nz, self.nxh, 3), np.complex128)

    @property
    def cbc_bot(self):
        return _view(self.L.orc_cbc_bot(self.h), (self.nz, self.nxh, 3), np.complex128)

    @property
    def buffer(self):
        return _view(self.L.orc_buffer(self.h), (self.nx2, self.nz2), np.float64)

    @property
    def target_inflow(self):
        return _view(self.L.orc_target_inflow(self.h), (self.ny + 1, 3), np.float64)

    @property
    def baseflow(self):
        return _view(self.L.orc_baseflow(self.h), (self.ny + 1, 3), np.float64)

    @property
    def d_um_dy(self):
        return _view(self.L.orc_d_um_dy(self.h), (self.ny,), np.float64)

    @property
    def cfl(self):
        return _view(self.L.orc_cfl(self.h), (self.ny + 1,), np.float64)

    def scalars(self):
        t, dt, pg = C.c_double(), C.c_double(), C.c_double()
        self.L.orc_get_scalars(self.h, C.byref(t), C.byref(dt), C.byref(pg))
        return t.value, dt.value, pg.value

    def set_scalars(self, t, dt, pg):
        self.L.orc_set_scalars(self.h, t, dt, pg)

    def set_step(self, step, rk):
        self.L.orc_set_step(self.h, step, rk)

    def status(self):
        return self.L.orc_status(self.h)

    # --- transforms
    def xz_c2r(self, cdata):
        cd = np.asfortranarray(cdata, dtype=np.complex128)
        out = np.zeros((self.nx2, self.nz2), order="F")
        self.L.orc_xz_c2r(self.h, cd.ctypes.data, out.ctypes.data)
        return out

    def xz_r2c(self, data):
        d = np.asfortranarray(data, dtype=np.float64)
        out = np.zeros((self.nz, self.nxh), dtype=np.complex128, order="F")
        self.L.orc_xz_r2c(self.h, d.ctypes.data, out.ctypes.data)
        return out

    def div_fluxes(self, dx, dy, dz):
        a = [np.asfortranarray(v, dtype=np.float64) for v in (dx, dy, dz)]
        out = np.zeros((self.nz, self.nxh), dtype=np.complex128, order="F")
        self.L.orc_div_fluxes(self.h, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data,
                              out.ctypes.data)
        return out

    def small_r2c(self, data):
        d = np.asfortranarray(data, dtype=np.float64)
        out = np.zeros((self.nz, self.nxh), dtype=np.complex128, order="F")
        self.L.orc_small_r2c(self.h, d.ctypes.data, out.ctypes.data)
        return out

    def small_c2r(self, cdata):
        cd = np.asfortranarray(cdata, dtype=np.complex128)
        out = np.zeros((self.nx, self.nz), order="F")
        self.L.orc_small_c2r(self.h, cd.ctypes.data, out.ctypes.data)
        return out

    # --- hot path
    def nonlinear(self):
        self.L.orc_nonlinear(self.h)

    def nonlinear_linearized(self):
        self.L.orc_nonlinear_linearized(self.h)

    def rhs_solve(self):
        self.L.orc_rhs_solve(self.h)

    def boundary(self):
        self.L.orc_boundary(self.h)

    def l2_norm(self):
        l2, drag = C.c_double(), C.c_double()
        self.L.orc_l2_norm(self.h, C.byref(l2), C.byref(drag))
        return l2.value, drag.value

    def init_field(self, which_test, seed=1, ampl=1e-3):
        self.L.orc_init_field(self.h, which_test, seed, ampl)

    def initial_velocity(self, which_test, seed=1, ampl=1e-3):
        self.L.orc_initial_velocity(self.h, which_test, seed, ampl)

    def init_from_velocity(self, data1):
        """define_initial_field's common tail for a given velocity (data1
        layout): divergence removal, d_um_dy, data2 = data1, pressure."""
        self.data1[...] = data1
        self.L.orc_init_from_velocity(self.h)

    def remove_initial_divergence(self):
        self.L.orc_remove_initial_divergence(self.h)

    def compute_d_um_dy(self):
        self.L.orc_compute_d_um_dy(self.h)

    def compute_initial_pressure(self, linearized=0):
        self.L.orc_compute_initial_pressure(self.h, linearized)

    def timestep(self, nsteps=1, linearized=0):
        self.L.orc_timestep(self.h, nsteps, linearized)

    def bulk_flux(self):
        return self.L.orc_bulk_flux(self.h)

    def max_divergence(self):
        return self.L.orc_max_divergence(self.h)

    def set_jet(self, jet):
        """Crossflow on (jet an OrcJet) or off (None)."""
        self.L.orc_set_jet(self.h, C.byref(jet) if jet is not None else None)

    def jet_profile(self, time, time_incr):
        self.L.orc_jet_profile(self.h, time, time_incr)

    def jet_forcing(self):
        jf = np.zeros(24)
        inc = np.zeros(24)
        self.L.orc_get_jet_forcing(self.h, jf.ctypes.data, inc.ctypes.data)
        return jf, inc

    def arnoldi_matvec(self, v, tend):
        v = np.asfortranarray(v, dtype=np.float64)
        w = np.zeros_like(v, order="F")
        self.L.orc_arnoldi_matvec(self.h, tend, v.ctypes.data, w.ctypes.data)
        return w
