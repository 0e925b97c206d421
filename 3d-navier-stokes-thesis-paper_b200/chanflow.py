"""Python mirror of the reference solver's hot-path module interfaces over the
C ABI of include/chanflow.h (libchanflow_b200.so, built in-tree for sm_100a).

The method names follow the Fortran module procedures they replace
(PFC = ParallelFortran-Code/ of the reference):

    ChannelFlow.nonlinear            pass1::nonlinear          PFC/pass1.f90:26
    ChannelFlow.nonlinear_linearized pass1_linearized          PFC/pass1_linearized.f90:135
    ChannelFlow.rhs_solve            pass2::rhs_solve          PFC/pass2.f90:29
    ChannelFlow.boundary             read_write::boundary      PFC/read_write.f90:1465
    ChannelFlow.l2_norm              read_write::l2_norm       PFC/read_write.f90:1432
    ChannelFlow.xz_fft_complex_to_real / xz_fft_real_to_complex
                                     transform module          PFC/transform.f90:195-227
    ChannelFlow.timestep             main_mpi timestep loop    PFC/main_mpi.f90:70-86

Arrays cross the boundary in the reference's Fortran layouts (numpy arrays
with order='F').  There is no CPU fallback: constructing a ChannelFlow without
the CUDA library or without a GPU raises.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libchanflow_b200.so")

FP64 = 0
MIXED = 1

ERRORS = {
    -1: "invalid argument", -2: "CUDA error", -3: "out of device memory",
    -4: "CFL IS TOO BIG", -5: "DT IS TOO BIG", -6: "call out of sequence",
    -7: "size beyond the fixed scratch capacity",
}


class CfgParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nx2", C.c_int), ("nz2", C.c_int),
        ("re", C.c_double), ("lx", C.c_double), ("lz", C.c_double), ("beta", C.c_double),
        ("dt", C.c_double), ("cfl_max", C.c_double),
        ("fix_mass", C.c_int), ("dt_flag", C.c_int),
        ("ctrlu", C.c_double), ("ctrlw", C.c_double),
        ("precision", C.c_int), ("device", C.c_int),
    ]


_DP = C.POINTER(C.c_double)


class CfgGrid(C.Structure):
    _fields_ = [(n, _DP) for n in ("y", "yh", "hn", "dh", "dn", "iu", "dm", "d2h", "d2n", "dyh",
                                   "dy", "kx", "kz", "buffer", "target_inflow")]


class CfgJet(C.Structure):
    """cfg_jet (include/chanflow.h): index 0 of each pair is the bottom wall."""
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


class CfgFringe(C.Structure):
    """cfg_fringe (include/chanflow.h): init_buffer's parameters."""
    _fields_ = [
        ("fringe_gain", C.c_double), ("xfringe", C.c_int), ("zfringe", C.c_int),
        ("frac_xbuff", C.c_double), ("buff_xrise", C.c_double), ("buff_xfall", C.c_double),
        ("frac_zbuff", C.c_double),
    ]


class CfgLes(C.Structure):
    """cfg_les (include/chanflow.h): the LES mode's subgrid model."""
    _fields_ = [
        ("model", C.c_int), ("cs", C.c_double), ("aplus", C.c_double), ("beta", C.c_double),
        ("mlp", C.c_void_p),
        ("in_shift", C.c_float * 10), ("in_scale", C.c_float * 10),
        ("out_shift", C.c_float * 6), ("out_scale", C.c_float * 6),
    ]


class CfhRun(C.Structure):
    _fields_ = [
        ("re", C.c_double), ("ctrlu", C.c_double), ("ctrlw", C.c_double), ("lx", C.c_double),
        ("lz", C.c_double), ("beta", C.c_double), ("disturb_ampl", C.c_double),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nx2", C.c_int), ("nz2", C.c_int),
        ("tend", C.c_int), ("output_step", C.c_int), ("save_step", C.c_int), ("l2_step", C.c_int),
        ("read_vel", C.c_int), ("save_vel", C.c_int), ("vel_out", C.c_int), ("which_test", C.c_int),
        ("fix_mass", C.c_int), ("dt_flag", C.c_int), ("divg_check", C.c_int),
        ("bl_grid", C.c_int), ("crossflow", C.c_int), ("filter_jet_profile", C.c_int),
        ("jet_diam", C.c_double), ("xjet_top", C.c_double), ("zjet_top", C.c_double),
        ("jetmag_top", C.c_double), ("forcing_top", C.c_double), ("for_freq_top", C.c_double),
        ("xjet_bot", C.c_double), ("zjet_bot", C.c_double), ("jetmag_bot", C.c_double),
        ("forcing_bot", C.c_double), ("for_freq_bot", C.c_double),
        ("xfringe", C.c_int), ("zfringe", C.c_int), ("frac_xbuff", C.c_double),
        ("stretch", C.c_double), ("dt", C.c_double), ("seed", C.c_ulonglong),
        ("precision", C.c_int), ("uniform_grid", C.c_int), ("jet_mode", C.c_int),
        ("jet_width", C.c_double), ("jet_peak", C.c_double), ("jet_freq", C.c_double),
        ("fringe_gain", C.c_double), ("buff_xrise", C.c_double), ("buff_xfall", C.c_double),
        ("frac_zbuff", C.c_double), ("buff_zrise", C.c_double), ("buff_zfall", C.c_double),
    ]


class CfhGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nx2", C.c_int), ("nz2", C.c_int)] + \
        [(n, _DP) for n in ("y", "yh", "hh", "hn", "dh", "dn", "iu", "dm", "d2h", "d2n", "dyh", "dy",
                            "kx", "kz", "buffer", "target_inflow", "xcoord", "zcoord")]


# exported symbols: name -> (restype, argtypes)
_VP = C.c_void_p
SYMBOLS = {
    "cfg_create": (C.c_int, [C.POINTER(CfgParams), C.POINTER(CfgGrid), C.POINTER(_VP)]),
    "cfg_destroy": (None, [_VP]),
    "cfg_last_error": (C.c_char_p, [_VP]),
    "cfg_upload_state": (C.c_int, [_VP, _VP, _VP, _VP]),
    "cfg_download_state": (C.c_int, [_VP, _VP, _VP, _VP]),
    "cfg_set_scalars": (C.c_int, [_VP, C.c_double, C.c_double, C.c_double, _VP]),
    "cfg_get_scalars": (C.c_int, [_VP, _DP, _DP, _DP, _VP, _DP]),
    "cfg_set_wall_bc": (C.c_int, [_VP, _VP, _VP]),
    "cfg_get_wall_bc": (C.c_int, [_VP, _VP, _VP]),
    "cfg_boundary": (C.c_int, [_VP]),
    "cfg_nonlinear": (C.c_int, [_VP, C.c_int, C.c_int]),
    "cfg_nonlinear_linearized": (C.c_int, [_VP, C.c_int, C.c_int]),
    "cfg_set_baseflow": (C.c_int, [_VP, _VP]),
    "cfg_rhs_solve": (C.c_int, [_VP, C.c_int, C.c_int]),
    "cfg_timestep": (C.c_int, [_VP, C.c_int]),
    "cfg_timestep_linearized": (C.c_int, [_VP, C.c_int]),
    "cfg_xz_c2r": (C.c_int, [_VP, _VP, _VP]),
    "cfg_xz_r2c": (C.c_int, [_VP, _VP, _VP]),
    "cfg_small_r2c": (C.c_int, [_VP, _VP, _VP, C.c_int]),
    "cfg_small_c2r": (C.c_int, [_VP, _VP, _VP, C.c_int]),
    "cfg_l2_norm": (C.c_int, [_VP, _DP, _DP]),
    "cfg_arnoldi_matvec": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "cfg_save_velocity": (C.c_int, [_VP, C.c_char_p]),
    "cfg_read_velocity": (C.c_int, [_VP, C.c_char_p]),
    "cfg_write_vtk": (C.c_int, [_VP, C.c_char_p]),
    "cfg_wait_io": (C.c_int, [_VP]),
    "cfg_init_buffer": (C.c_int, [_VP, C.POINTER(CfgFringe)]),
    "cfg_get_buffer": (C.c_int, [_VP, _VP, _VP]),
    "cfg_write_vtk_derived": (C.c_int, [_VP, C.c_char_p]),
    "cfg_plane_statistics": (C.c_int, [_VP, _VP]),
    "cfg_set_jet": (C.c_int, [_VP, C.POINTER(CfgJet)]),
    "cfg_jet_profile": (C.c_int, [_VP, C.c_double, C.c_double]),
    "cfg_get_jet_forcing": (C.c_int, [_VP, _VP, _VP]),
    "cfg_remove_initial_divergence": (C.c_int, [_VP]),
    "cfg_compute_initial_pressure": (C.c_int, [_VP, C.c_int]),
    "cfg_diagnostics": (C.c_int, [_VP, _DP, _DP]),
    "cfg_status": (C.c_int, [_VP]),
    "cfg_synchronize": (C.c_int, [_VP]),
    "cfg_launch_count": (C.c_longlong, [_VP]),
    "cfg_stream": (_VP, [_VP]),
    "cfg_xz_c2r_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _VP, _VP, _VP]),
    "cfg_set_les": (C.c_int, [_VP, C.c_void_p]),
    "cfg_les_features": (C.c_int, [_VP, _VP]),
    "cfg_les_stresses": (C.c_int, [_VP, _VP]),
    "cfg_les_fallbacks": (C.c_int, [_VP, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]),
    "cfg_mlp_nparams": (C.c_int, []),
    "cfg_mlp_create": (C.c_int, [C.c_int, C.POINTER(_VP)]),
    "cfg_mlp_destroy": (None, [_VP]),
    "cfg_mlp_set_params": (C.c_int, [_VP, _VP]),
    "cfg_mlp_get_params": (C.c_int, [_VP, _VP]),
    "cfg_mlp_forward": (C.c_int, [_VP, _VP, _VP, C.c_longlong, _VP]),
    "cfg_mlp_accumulate_grad": (C.c_int, [_VP, _VP, _VP, _VP, C.c_int, _VP]),
    "cfg_mlp_get_grads": (C.c_int, [_VP, _VP, _VP]),
    "cfg_mlp_zero_grads": (C.c_int, [_VP, _VP]),
    "cfg_mlp_adam_step": (C.c_int, [_VP, C.c_float, C.c_float, C.c_float, C.c_float, _VP]),
    "cfg_mlp_status": (C.c_int, [_VP]),
    "cfg_profile_enable": (C.c_int, [_VP, C.c_int]),
    "cfg_profile_read": (C.c_int, [_VP, C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_int), _DP]),
    "cfg_partition": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _VP, _VP, _VP, _VP, _VP, _VP]),
    "cfg_group_create": (C.c_int, [C.POINTER(CfgParams), C.POINTER(CfgGrid), C.c_int, _VP, C.POINTER(_VP)]),
    "cfg_group_size": (C.c_int, [_VP]),
    "cfg_group_rank": (_VP, [_VP, C.c_int]),
    "cfg_group_timestep": (C.c_int, [_VP, C.c_int]),
    "cfg_group_synchronize": (C.c_int, [_VP]),
    "cfg_group_destroy": (None, [_VP]),
    "cfg_autotune": (C.c_int, [_VP, C.c_int, _VP]),
    "cfg_set_tiles": (C.c_int, [_VP, _VP]),
    "cfg_get_tiles": (C.c_int, [_VP, _VP]),
    "cfg_ensemble_create": (C.c_int, [C.c_int, _VP, C.c_int, C.POINTER(_VP)]),
    "cfg_ensemble_timestep": (C.c_int, [_VP, C.c_int]),
    "cfg_ensemble_synchronize": (C.c_int, [_VP]),
    "cfg_ensemble_stream": (_VP, [_VP]),
    "cfg_ensemble_set_batched": (C.c_int, [_VP, C.c_int]),
    "cfg_ensemble_batched": (C.c_int, [_VP]),
    "cfg_ensemble_destroy": (None, [_VP]),
    "cfg_rank_record_size": (C.c_size_t, []),
    "cfg_rank_create": (C.c_int, [C.POINTER(CfgParams), C.POINTER(CfgGrid), C.c_int, C.c_int, C.POINTER(_VP)]),
    "cfg_rank_export": (C.c_int, [_VP, _VP]),
    "cfg_rank_connect": (C.c_int, [_VP, _VP]),
    "cfg_rank_timestep": (C.c_int, [_VP, C.c_int, C.c_void_p, _VP]),
    "cfg_rank_timestep_ordered": (C.c_int, [_VP, C.c_int, C.c_void_p, _VP]),
    "cfh_run_defaults": (None, [C.POINTER(CfhRun)]),
    "cfh_read_flow_dat": (C.c_int, [C.c_char_p, C.POINTER(CfhRun), C.c_char_p, C.c_int]),
    "cfh_grid_alloc": (C.POINTER(CfhGrid), [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "cfh_grid_free": (None, [C.POINTER(CfhGrid)]),
    "cfh_define_grid": (C.c_int, [C.POINTER(CfhGrid), C.c_double, C.c_double, C.c_double, C.c_int]),
    "cfh_initial_field": (C.c_int, [C.POINTER(CfhGrid), C.c_int, C.c_ulonglong, C.c_double,
                                    C.c_double, _VP]),
    "cfh_read_efn": (C.c_int, [C.c_char_p, _VP]),
    "cfh_interp_eigenfunction": (C.c_int, [C.POINTER(CfhGrid), _VP, _VP, _VP]),
    "cfh_initial_field_mode": (C.c_int, [C.POINTER(CfhGrid), C.c_int, C.c_double, C.c_double, _VP, _VP, _VP]),
    "cfh_rng_u01": (C.c_double, [C.c_ulonglong, C.c_int, C.c_int, C.c_int, C.c_int]),
    "cfh_save_velocity": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, _VP, C.c_char_p, C.c_int]),
    "cfh_read_velocity": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                    _DP, _DP, _VP, C.c_char_p, C.c_int]),
}

_lib = None


def load_library(path=LIB_PATH):
    """Load libchanflow_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(f"CUDA extension missing: {path} (run __graft_entry__.build())")
        L = C.CDLL(path)
        for name, (res, args) in SYMBOLS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class ChanflowError(RuntimeError):
    pass


def _p(a):
    return None if a is None else a.ctypes.data


class Grid:
    """Host-side grid operators: define_coordinates + wavenumbers (C++ setup)."""

    NAMES = {"y": "ny", "yh": "ny1", "hh": "ny1", "hn": "ny", "dh": "ny1", "dn": "ny",
             "iu": (2, "ny"), "dm": (3, 4), "d2h": (3, "ny1"), "d2n": (3, "ny"), "dyh": "ny1",
             "dy": "ny1", "kx": "nxh", "kz": "nz", "buffer": ("nx2", "nz2"),
             "target_inflow": ("ny1", 3), "xcoord": "nx1", "zcoord": "nz1"}

    def __init__(self, nx, ny, nz, nx2=None, nz2=None, lx=4 * np.pi, lz=2 * np.pi, stretch=2.75,
                 uniform=0):
        L = load_library()
        nx2 = nx2 or 3 * nx // 2
        nz2 = nz2 or 3 * nz // 2
        self.nx, self.ny, self.nz, self.nx2, self.nz2 = nx, ny, nz, nx2, nz2
        self.lx, self.lz = lx, lz
        h = L.cfh_grid_alloc(nx, ny, nz, nx2, nz2)
        if L.cfh_define_grid(h, lx, lz, stretch, uniform) != 0:
            L.cfh_grid_free(h)
            raise ChanflowError("define_grid failed")
        dims = {"ny": ny, "ny1": ny + 1, "nxh": nx // 2 + 1, "nz": nz, "nx2": nx2, "nz2": nz2,
                "nx1": nx + 1, "nz1": nz + 1}
        for name, shp in self.NAMES.items():
            shp = shp if isinstance(shp, tuple) else (shp,)
            shp = tuple(dims[s] if isinstance(s, str) else s for s in shp)
            n = int(np.prod(shp))
            arr = np.ctypeslib.as_array(getattr(h.contents, name), shape=(n,)).copy()
            setattr(self, name, np.asfortranarray(arr.reshape(shp, order="F")))
        L.cfh_grid_free(h)

    def cfg_grid(self):
        keep = []

        def ptr(a):
            a = np.asfortranarray(a, dtype=np.float64)
            keep.append(a)
            return a.ctypes.data_as(_DP)

        g = CfgGrid(*[ptr(getattr(self, n)) for n in ("y", "yh", "hn", "dh", "dn", "iu", "dm", "d2h",
                                                       "d2n", "dyh", "dy", "kx", "kz", "buffer",
                                                       "target_inflow")])
        return g, keep


def initial_field(grid, which_test, seed=1, ampl=1e-3, beta=0.0, efn=None):
    """Seeded which_test initial velocity in data1 layout (before the device
    divergence removal and initial pressure).  which_test 2, 5 and 8 (the
    Orr-Sommerfeld mode, PFC/init_vel.f90:95-159) take the eigenfunction as
    efn: the (65, 4) array of efn.m (Re u, Im u, Re v, Im v at the Chebyshev
    points) or the path of such a file."""
    L = load_library()
    nxh = grid.nx // 2 + 1
    d1 = np.zeros((grid.nz, nxh, grid.ny + 1, 3), dtype=np.complex128, order="F")
    h = L.cfh_grid_alloc(grid.nx, grid.ny, grid.nz, grid.nx2, grid.nz2)
    try:
        for name in ("y", "yh", "dh", "dyh", "kx", "kz"):
            src = np.ascontiguousarray(getattr(grid, name).ravel(order="F"))
            C.memmove(getattr(h.contents, name), src.ctypes.data, src.nbytes)
        if which_test in (2, 5, 8):
            if efn is None:
                raise ChanflowError(f"which_test {which_test} needs the eigenfunction (efn)")
            if isinstance(efn, (str, bytes, os.PathLike)):
                uin = np.zeros((65, 4), order="F")
                r = L.cfh_read_efn(os.fsencode(efn), uin.ctypes.data)
                if r != 0:
                    raise ChanflowError(f"cannot read the eigenfunction file {efn!r} ({r})")
            else:
                uin = np.asfortranarray(efn, dtype=np.float64)
                if uin.shape != (65, 4):
                    raise ChanflowError(f"efn must be (65, 4), got {uin.shape}")
            u = np.zeros(grid.ny + 1, np.complex128)
            v = np.zeros(grid.ny + 1, np.complex128)
            L.cfh_interp_eigenfunction(h, uin.ctypes.data, u.ctypes.data, v.ctypes.data)
            r = L.cfh_initial_field_mode(h, which_test, ampl, beta, u.ctypes.data, v.ctypes.data, d1.ctypes.data)
        else:
            r = L.cfh_initial_field(h, which_test, seed, ampl, beta, d1.ctypes.data)
    finally:
        L.cfh_grid_free(h)
    if r != 0:
        raise ChanflowError(f"unsupported which_test {which_test}")
    return d1


def read_flow_dat(path):
    L = load_library()
    run = CfhRun()
    err = C.create_string_buffer(256)
    r = L.cfh_read_flow_dat(path.encode(), C.byref(run), err, 256)
    if r != 0:
        raise ChanflowError(err.value.decode())
    return run


def save_velocity_file(path, data1, lx, lz, re, dt, t_total):
    """Write a host data1 (nz, nx/2+1, ny+1, 3) as the reference's restart
    file (read_write::save_velocity, PFC/read_write.f90:211-292)."""
    L = load_library()
    d = np.asfortranarray(data1, dtype=np.complex128)
    nz, nxh, n1, _ = d.shape
    err = C.create_string_buffer(256)
    r = L.cfh_save_velocity(os.fsencode(path), 2 * (nxh - 1), n1 - 1, nz, lx, lz, re, dt, t_total,
                            d.ctypes.data, err, 256)
    if r != 0:
        raise ChanflowError(err.value.decode())


def read_velocity_file(path, nx, ny, nz, lx, lz, re):
    """Read a restart file with read_velocity's checks; returns
    (data1, dt, t_total)."""
    L = load_library()
    d = np.zeros((nz, nx // 2 + 1, ny + 1, 3), np.complex128, order="F")
    dt, t = C.c_double(), C.c_double()
    err = C.create_string_buffer(256)
    r = L.cfh_read_velocity(os.fsencode(path), nx, ny, nz, lx, lz, re, C.byref(dt), C.byref(t), d.ctypes.data,
                            err, 256)
    if r != 0:
        raise ChanflowError(err.value.decode())
    return d, dt.value, t.value


class ChannelFlow:
    """One device context: state, plans and the hot-path routines."""

    def __init__(self, grid, re=2500.0, dt=0.005, beta=0.0, cfl_max=0.95, fix_mass=1, dt_flag=0,
                 ctrlu=0.0, ctrlw=0.0, precision=FP64, device=0):
        self.L = load_library()
        self.grid = grid
        self.nx, self.ny, self.nz = grid.nx, grid.ny, grid.nz
        self.nx2, self.nz2 = grid.nx2, grid.nz2
        self.nxh = grid.nx // 2 + 1
        self.precision = precision
        self.params = CfgParams(grid.nx, grid.ny, grid.nz, grid.nx2, grid.nz2, re, grid.lx, grid.lz,
                                beta, dt, cfl_max, fix_mass, dt_flag, ctrlu, ctrlw, precision, device)
        g, keep = grid.cfg_grid()
        h = C.c_void_p()
        r = self.L.cfg_create(C.byref(self.params), C.byref(g), C.byref(h))
        if r != 0:
            raise ChanflowError(f"cfg_create failed ({ERRORS.get(r, r)})")
        self.h = h
        self.step = 0

    def _chk(self, r):
        if r != 0:
            msg = self.L.cfg_last_error(self.h)
            raise ChanflowError(f"{ERRORS.get(r, r)}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                self.L.cfg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state
    def shapes(self):
        n1 = self.ny + 1
        return ((self.nz, self.nxh, n1, 3), (n1, 3, self.nz, self.nxh), (n1, self.nz, self.nxh))

    def upload_state(self, data1=None, data2=None, data4=None):
        a = [None if d is None else np.asfortranarray(d, dtype=np.complex128) for d in (data1, data2, data4)]
        self._chk(self.L.cfg_upload_state(self.h, _p(a[0]), _p(a[1]), _p(a[2])))

    def download_state(self):
        s1, s2, s4 = self.shapes()
        d1 = np.zeros(s1, np.complex128, order="F")
        d2 = np.zeros(s2, np.complex128, order="F")
        d4 = np.zeros(s4, np.complex128, order="F")
        self._chk(self.L.cfg_download_state(self.h, _p(d1), _p(d2), _p(d4)))
        return d1, d2, d4

    def set_scalars(self, t_total, dt, p_grad, d_um_dy=None):
        d = None if d_um_dy is None else np.ascontiguousarray(d_um_dy, dtype=np.float64)
        self._chk(self.L.cfg_set_scalars(self.h, t_total, dt, p_grad, _p(d)))

    def scalars(self):
        t, dt, pg, cm = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        dud = np.zeros(self.ny)
        self._chk(self.L.cfg_get_scalars(self.h, C.byref(t), C.byref(dt), C.byref(pg), _p(dud),
                                         C.byref(cm)))
        return {"t_total": t.value, "dt": dt.value, "p_grad": pg.value, "d_um_dy": dud,
                "cfl_max": cm.value}

    def set_wall_bc(self, cbc_top=None, cbc_bot=None):
        a = [None if d is None else np.asfortranarray(d, dtype=np.complex128) for d in (cbc_top, cbc_bot)]
        self._chk(self.L.cfg_set_wall_bc(self.h, _p(a[0]), _p(a[1])))

    def wall_bc(self):
        top = np.zeros((self.nz, self.nxh, 3), np.complex128, order="F")
        bot = np.zeros_like(top)
        self._chk(self.L.cfg_get_wall_bc(self.h, _p(top), _p(bot)))
        return top, bot

    def set_baseflow(self, profile):
        p = np.asfortranarray(profile, dtype=np.float64)
        self._chk(self.L.cfg_set_baseflow(self.h, _p(p)))

    # ---- hot path (reference module procedures)
    def boundary(self):
        self._chk(self.L.cfg_boundary(self.h))

    def nonlinear(self, step, rk_step):
        self._chk(self.L.cfg_nonlinear(self.h, step, rk_step))

    def nonlinear_linearized(self, step, rk_step):
        self._chk(self.L.cfg_nonlinear_linearized(self.h, step, rk_step))

    def rhs_solve(self, step, rk_step):
        self._chk(self.L.cfg_rhs_solve(self.h, step, rk_step))

    def timestep(self, nsteps=1):
        self._chk(self.L.cfg_timestep(self.h, nsteps))

    def timestep_linearized(self, nsteps=1):
        self._chk(self.L.cfg_timestep_linearized(self.h, nsteps))

    def xz_fft_complex_to_real(self, cdata):
        cd = np.asfortranarray(cdata, dtype=np.complex128)
        out = np.zeros((self.nx2, self.nz2), order="F")
        self._chk(self.L.cfg_xz_c2r(self.h, _p(cd), _p(out)))
        return out

    def xz_fft_real_to_complex(self, data):
        d = np.asfortranarray(data, dtype=np.float64)
        out = np.zeros((self.nz, self.nxh), np.complex128, order="F")
        self._chk(self.L.cfg_xz_r2c(self.h, _p(d), _p(out)))
        return out

    def small_fft_real_to_complex(self, data):
        """small_fft_real_to_complex (PFC/transform.f90:950-1142): data
        (nx, nz[, nplanes]) real -> (nz, nx/2+1[, nplanes]) complex, 1/(nx nz)."""
        d = np.asfortranarray(data, dtype=np.float64)
        npl = 1 if d.ndim == 2 else d.shape[2]
        out = np.zeros((self.nz, self.nxh, npl), np.complex128, order="F")
        self._chk(self.L.cfg_small_r2c(self.h, _p(d), _p(out), npl))
        return out[:, :, 0] if d.ndim == 2 else out

    def small_fft_complex_to_real(self, cdata):
        cd = np.asfortranarray(cdata, dtype=np.complex128)
        npl = 1 if cd.ndim == 2 else cd.shape[2]
        out = np.zeros((self.nx, self.nz, npl), order="F")
        self._chk(self.L.cfg_small_c2r(self.h, _p(cd), _p(out), npl))
        return out[:, :, 0] if cd.ndim == 2 else out

    def arnoldi_matvec(self, v, tend):
        """compute_time_deriv (PFC/arnoldi.f90:485-567): w = Phi_T v for a
        real vector of shape (nx, nz, ny+1, 3) (or its flat Fortran-order
        ravel).  Overwrites the state."""
        shape = (self.nx, self.nz, self.ny + 1, 3)
        vv = np.asfortranarray(np.reshape(v, shape, order="F"), dtype=np.float64)
        w = np.zeros(shape, order="F")
        self._chk(self.L.cfg_arnoldi_matvec(self.h, int(tend), _p(vv), _p(w)))
        return w if np.ndim(v) == 4 else w.ravel(order="F")

    def save_velocity(self, path, wait=False):
        """read_write::save_velocity: the restart file of the current data1,
        written in the background (wait_io() or the next output waits)."""
        self._chk(self.L.cfg_save_velocity(self.h, os.fsencode(path)))
        if wait:
            self.wait_io()

    def read_velocity(self, path):
        """read_write::read_velocity: data1, t_total (and dt if dt_flag)."""
        self._chk(self.L.cfg_read_velocity(self.h, os.fsencode(path)))

    def write_vtk(self, path, wait=False):
        """The VTK velocity snapshot of output_hdf_dfsd (background write)."""
        self._chk(self.L.cfg_write_vtk(self.h, os.fsencode(path)))
        if wait:
            self.wait_io()

    def write_vtk_derived(self, path, wait=False):
        """The snapshot plus vorticity, Q-criterion and discriminant."""
        self._chk(self.L.cfg_write_vtk_derived(self.h, os.fsencode(path)))
        if wait:
            self.wait_io()

    def plane_statistics(self):
        """(ny+1, 27) per-plane moments of velocity and vorticity (see
        include/chanflow.h, cfg_plane_statistics)."""
        out = np.zeros((self.ny + 1, 27), order="F")
        self._chk(self.L.cfg_plane_statistics(self.h, _p(out)))
        return out

    def init_buffer(self, fringe_gain, xfringe=1, zfringe=0, frac_xbuff=0.1, buff_xrise=0.03,
                    buff_xfall=0.02, frac_zbuff=0.1):
        """init_buffer (PFC/init_jet_buffer.f90:358-483) on the device."""
        f = CfgFringe(fringe_gain, xfringe, zfringe, frac_xbuff, buff_xrise, buff_xfall, frac_zbuff)
        self._chk(self.L.cfg_init_buffer(self.h, C.byref(f)))

    def buffer(self):
        """(buffer (nx2, nz2), target_inflow (ny+1, 3)) on the device."""
        b = np.zeros((self.nx2, self.nz2), order="F")
        t = np.zeros((self.ny + 1, 3), order="F")
        self._chk(self.L.cfg_get_buffer(self.h, _p(b), _p(t)))
        return b, t

    def wait_io(self):
        self._chk(self.L.cfg_wait_io(self.h))

    def set_les(self, model, cs=0.1, aplus=25.0, beta=0.0, mlp=None, in_shift=None, in_scale=None,
                out_shift=None, out_scale=None):
        """LES mode: model 0 off, 1 eddy viscosity (Smagorinsky cs, van
        Driest aplus), 2 the learned closure (an Mlp) with the eddy
        viscosity as its per-point fallback (beta: admitted backscatter as a
        fraction of the eddy viscosity's dissipation).  The shifts and scales
        normalise the 10 features and map the 6 outputs back."""
        l = CfgLes()
        l.model, l.cs, l.aplus, l.beta = int(model), cs, aplus, beta
        l.mlp = mlp.h.value if mlp is not None else None
        for name, n, default in (("in_shift", 10, 0.0), ("in_scale", 10, 1.0), ("out_shift", 6, 0.0),
                                 ("out_scale", 6, 1.0)):
            v = locals()[name]
            arr = getattr(l, name)
            for i in range(n):
                arr[i] = float(default if v is None else v[i])
        self._les_mlp = mlp          # keep the network alive while the context uses it
        self._chk(self.L.cfg_set_les(self.h, C.byref(l)))

    def les_features(self, ptr):
        """The closure's features of the current state into a device buffer
        of (ny-1)*nz2*nx2*10 floats (model 2 must be set)."""
        self._chk(self.L.cfg_les_features(self.h, ptr))

    def les_stresses(self):
        """The last subgrid stresses, (ny+1, 6, nz2, nx2) FP64."""
        S = np.zeros((self.ny + 1, 6, self.grid.nz2, self.grid.nx2))
        self._chk(self.L.cfg_les_stresses(self.h, S.ctypes.data))
        return S

    def les_fallbacks(self):
        f, n = C.c_ulonglong(), C.c_ulonglong()
        self._chk(self.L.cfg_les_fallbacks(self.h, C.byref(f), C.byref(n)))
        return f.value, n.value

    def set_jet(self, jet):
        """crossflow = 1 with a CfgJet (jet_profile every substep), or None."""
        self._chk(self.L.cfg_set_jet(self.h, C.byref(jet) if jet is not None else None))

    def jet_profile(self, time, time_incr):
        """pass2::jet_profile(time, time_incr, cbc_top(:,:,2), cbc_bot(:,:,2))."""
        self._chk(self.L.cfg_jet_profile(self.h, time, time_incr))

    def jet_forcing(self):
        jf, inc = np.zeros(24), np.zeros(24)
        self._chk(self.L.cfg_get_jet_forcing(self.h, _p(jf), _p(inc)))
        return jf, inc

    def l2_norm(self):
        l2, drag = C.c_double(), C.c_double()
        self._chk(self.L.cfg_l2_norm(self.h, C.byref(l2), C.byref(drag)))
        return l2.value, drag.value

    def remove_initial_divergence(self):
        self._chk(self.L.cfg_remove_initial_divergence(self.h))

    def compute_initial_pressure(self, linearized=0):
        self._chk(self.L.cfg_compute_initial_pressure(self.h, linearized))

    def diagnostics(self):
        q, d = C.c_double(), C.c_double()
        self._chk(self.L.cfg_diagnostics(self.h, C.byref(q), C.byref(d)))
        return q.value, d.value

    def status(self):
        return self.L.cfg_status(self.h)

    def autotune(self, trial_steps=3):
        """Tune the kernels' tiles on this grid (cfg_autotune); the state is
        restored.  Returns (rhs warps, flux rows, zinv planes, zfwd planes)."""
        t = np.zeros(4, np.int32)
        self._chk(self.L.cfg_autotune(self.h, trial_steps, _p(t)))
        return tuple(int(v) for v in t)

    def set_tiles(self, tiles):
        t = np.ascontiguousarray(tiles, dtype=np.int32)
        self._chk(self.L.cfg_set_tiles(self.h, _p(t)))

    def tiles(self):
        """(warps per rhs block, z rows per flux block, planes per inverse and
        forward z-transform block)."""
        t = np.zeros(4, dtype=np.int32)
        self._chk(self.L.cfg_get_tiles(self.h, _p(t)))
        return [int(v) for v in t]

    def synchronize(self):
        self._chk(self.L.cfg_synchronize(self.h))

    def launch_count(self):
        return self.L.cfg_launch_count(self.h)

    def stream_ptr(self):
        """The cudaStream_t this context issues its kernels on."""
        return self.L.cfg_stream(self.h)

    def profile_enable(self, on=True):
        self._chk(self.L.cfg_profile_enable(self.h, 1 if on else 0))

    def profile_read(self):
        """{kernel name: (launches, total device ms)} since profile_enable."""
        n = self.L.cfg_profile_read(self.h, -1, None, 0, None, None)
        if n < 0:
            self._chk(n)
        out = {}
        for i in range(n):
            name = C.create_string_buffer(64)
            cnt, ms = C.c_int(), C.c_double()
            self._chk(self.L.cfg_profile_read(self.h, i, name, 64, C.byref(cnt), C.byref(ms)))
            out[name.value.decode()] = (cnt.value, ms.value)
        return out

    # ---- define_initial_field (PFC/init_vel.f90:25-353) on the device
    def define_initial_field(self, which_test, seed=1, ampl=1e-3, beta=0.0, efn=None):
        """define_initial_field (PFC/init_vel.f90:24-352): the which_test
        velocity (efn: the eigenfunction of which_test 2, 5, 8), its
        divergence removed and the initial pressure computed, t = 0."""
        d1 = initial_field(self.grid, which_test, seed, ampl, beta, efn)
        self.upload_state(d1, None, np.zeros(self.shapes()[2], np.complex128, order="F"))
        if which_test == 6:
            sc = self.scalars()
            self.set_scalars(0.0, sc["dt"], 0.0)
        else:
            sc = self.scalars()
            self.set_scalars(0.0, sc["dt"], sc["p_grad"])
        self.remove_initial_divergence()
        self.compute_initial_pressure(0)


def arnoldi_eigs(flow, tend, nev=12, ncv=25, tol=1e-8, maxiter=None, v0=None):
    """Host driver of the Arnoldi stability solver (PFC/arnoldi.f90:150-330):
    the largest-magnitude eigenvalues mu of the propagator Phi_T, T = tend*dt
    (fixed dt), by implicitly restarted Arnoldi (ARPACK through
    scipy.sparse.linalg.eigs, in place of the reference's PARPACK
    pdnaupd/pdneupd) with ChannelFlow.arnoldi_matvec as the operator, and the
    linearized eigenvalues cr = log(|mu| + eps)/T, ci = atan2(Im mu, Re mu)/T
    (:803-806).  Returns (mu, cr + i*ci, eigenvectors (n, nev))."""
    from scipy.sparse.linalg import LinearOperator, eigs
    n = flow.nx * flow.nz * (flow.ny + 1) * 3
    op = LinearOperator((n, n), matvec=lambda x: flow.arnoldi_matvec(np.real(np.ravel(x)), tend), dtype=np.float64)
    mu, vec = eigs(op, k=nev, ncv=ncv, which="LM", tol=tol, maxiter=maxiter, v0=v0)
    T = tend * flow.scalars()["dt"]
    lam = (np.log(np.abs(mu) + np.finfo(np.float64).eps) + 1j * np.arctan2(mu.imag, mu.real)) / T
    order = np.argsort(-np.abs(mu))
    return mu[order], lam[order], vec[:, order]


def stability_columns(nx, nz):
    """The Fourier columns (kx index a, kz index b) of a real nx x nz field
    that carry a free complex amplitude: 1 <= a < nx/2 with every kz but the
    Nyquist one, and a = 0 with 1 <= b < nz/2 (its kz < 0 partners are the
    conjugates).  Mean and Nyquist columns are left out."""
    cols = [(a, b) for a in range(1, nx // 2) for b in range(nz) if b != nz // 2]
    cols += [(0, b) for b in range(1, nz // 2)]
    return np.array(cols, dtype=np.int64)


def arnoldi_columns(flow, tend, ncv=60, nev=10, seed=3, restarts=4, keep=None, tol=1e-9):
    """Leading eigenvalues of the propagator Phi_T (T = tend*dt) about a
    parallel baseflow U(y), by Arnoldi run on every Fourier column at once.

    The linearized operator about a profile U(y) (PFC/pass1_linearized.f90,
    PFC/arnoldi.f90:485-567) does not couple Fourier columns, so its spectrum
    is the union of the columns' spectra.  Each column (stability_columns)
    gets its own Krylov basis of up to ncv vectors of (ny+1)*3 complex
    amplitudes, Gram-Schmidt orthogonalised twice in FP64 on the host; one
    GPU matvec (cfg_arnoldi_matvec) on the physical field that superposes all
    columns' current vectors advances every column's iteration.  Between
    cycles each column keeps its `keep` (default ncv/2) leading Schur vectors
    (a Krylov-Schur restart, Stewart 2001), `restarts` cycles in all.
    Returns (mu, lam, residual, column) for the nev eigenvalues of largest
    modulus among the Ritz values whose Arnoldi residual estimate is below
    tol |mu|: mu the propagator eigenvalue, lam = (log|mu| + i arg mu)/T,
    residual the explicit ||Phi x - mu x|| / ||x|| of its Ritz vector (one
    more matvec per Ritz rank), column its (kx index, kz index)."""
    import scipy.linalg as sl
    nx, nz, n1 = flow.nx, flow.nz, flow.ny + 1
    cols = stability_columns(nx, nz)
    ncol, n = len(cols), n1 * 3
    ncv = min(ncv, n)
    keep = keep or ncv // 2
    a, b = cols[:, 0], cols[:, 1]
    rng = np.random.default_rng(seed)

    def embed(V):
        """(ncol, n) column vectors -> real physical field (nx, nz, ny+1, 3)."""
        Ch = np.zeros((nz, nx // 2 + 1, n), complex)
        Ch[b, a] = V
        k0 = a == 0
        Ch[(-b[k0]) % nz, 0] = np.conj(V[k0])
        X = np.fft.irfft2(Ch, s=(nz, nx), axes=(0, 1))       # (nz, nx, n)
        return np.asfortranarray(X.transpose(1, 0, 2).reshape(nx, nz, n1, 3, order="C"))

    def extract(X):
        Xz = np.ascontiguousarray(np.asarray(X).reshape(nx, nz, n, order="C").transpose(1, 0, 2))
        return np.fft.rfft2(Xz, axes=(0, 1))[b, a]

    def apply(V):
        return extract(flow.arnoldi_matvec(embed(V), tend))

    T = tend * flow.scalars()["dt"]
    Vb = np.zeros((ncol, ncv + 1, n), complex)
    H = np.zeros((ncol, ncv + 1, ncv), complex)
    v = rng.standard_normal((ncol, n)) + 1j * rng.standard_normal((ncol, n))
    Vb[:, 0] = v / np.linalg.norm(v, axis=1, keepdims=True)
    j0 = 0
    for cycle in range(max(1, restarts)):
        for j in range(j0, ncv):
            w = apply(Vb[:, j])
            for _ in range(2):
                h = np.einsum("cjn,cn->cj", Vb[:, :j + 1].conj(), w)
                w = w - np.einsum("cjn,cj->cn", Vb[:, :j + 1], h)
                H[:, :j + 1, j] += h
            nrm = np.linalg.norm(w, axis=1)
            H[:, j + 1, j] = nrm
            Vb[:, j + 1] = w / np.maximum(nrm, 1e-300)[:, None]
        if cycle == restarts - 1:
            break
        # Krylov-Schur restart: the keep leading Schur vectors of each column
        Hn = np.zeros_like(H)
        Vn = np.zeros_like(Vb)
        for c in range(ncol):
            ev = np.linalg.eigvals(H[c, :ncv, :ncv])
            thr = np.sort(np.abs(ev))[::-1][keep - 1]
            S, Q, _ = sl.schur(H[c, :ncv, :ncv], output="complex", sort=lambda z, t=thr: abs(z) >= t * (1 - 1e-12))
            Vn[c, :keep] = Q[:, :keep].T @ Vb[c, :ncv]
            Hn[c, :keep, :keep] = S[:keep, :keep]
            Hn[c, keep, :keep] = H[c, ncv, ncv - 1] * Q[ncv - 1, :keep]
            Vn[c, keep] = Vb[c, ncv]
        Vb, H, j0 = Vn, Hn, keep
    theta, Y = np.linalg.eig(H[:, :ncv, :ncv])
    # the nev largest over all columns' converged Ritz values (Arnoldi
    # residual estimate |h_{m+1,m} y_m| below tol relative to |theta|)
    est = np.abs(H[:, ncv, ncv - 1])[:, None] * np.abs(Y[:, ncv - 1, :])
    mag = np.where(est <= tol * np.abs(theta), np.abs(theta), -1.0)
    flat = np.argsort(-mag, axis=None)[:nev]
    ci, ri = np.unravel_index(flat, theta.shape)
    mu = theta[ci, ri]
    X = np.einsum("kjn,kj->kn", Vb[ci, :ncv], Y[ci, :, ri])
    res = np.zeros(nev)
    # explicit residuals, one matvec per set of distinct columns
    todo = list(range(nev))
    while todo:
        batch, seen = [], set()
        for k in todo:
            if ci[k] not in seen:
                seen.add(ci[k])
                batch.append(k)
        V = np.zeros((ncol, n), complex)
        for k in batch:
            V[ci[k]] = X[k]
        W = apply(V)
        for k in batch:
            res[k] = np.linalg.norm(W[ci[k]] - mu[k] * X[k]) / np.linalg.norm(X[k])
        todo = [k for k in todo if k not in batch]
    lam = (np.log(np.abs(mu)) + 1j * np.angle(mu)) / T
    return mu, lam, res, cols[ci]


PARTITION_KEYS = ("nx_proc", "x_start", "nz_proc", "z_start", "nz_small_proc", "z_small_start")


def partition(nx, nz, nz2, nproc):
    """distribute_data (PFC/setup.f90:298-437): the split of the nx/2+1
    Fourier columns, the nz2 physical z rows and the nz undealiased z rows
    among nproc ranks, as a dict of int arrays (keys PARTITION_KEYS)."""
    L = load_library()
    arrs = [np.zeros(nproc, np.int32) for _ in PARTITION_KEYS]
    r = L.cfg_partition(nx, nz, nz2, nproc, *[_p(a) for a in arrs])
    if r != 0:
        raise ChanflowError(f"cfg_partition failed ({ERRORS.get(r, r)})")
    return dict(zip(PARTITION_KEYS, arrs))


class Group:
    """cfg_group: nranks contexts that advance one field together, rank i
    holding the Fourier columns [x_start[i], x_start[i] + nx_proc[i]) of the
    state and the z2 rows [z_start[i], ...) of the physical planes -- the
    reference's MPI decomposition (PFC/setup.f90:298-437) with the transposes
    of the x-z transforms as stores into the owning rank's buffers.
    devices: one GPU per rank (default: all ranks on `device`)."""

    def __init__(self, grid, nranks, devices=None, re=2500.0, dt=0.005, beta=0.0, cfl_max=0.95, fix_mass=1,
                 dt_flag=0, precision=FP64, device=0):
        self.L = load_library()
        self.grid = grid
        self.nranks = nranks
        self.params = CfgParams(grid.nx, grid.ny, grid.nz, grid.nx2, grid.nz2, re, grid.lx, grid.lz,
                                beta, dt, cfl_max, fix_mass, dt_flag, 0.0, 0.0, precision, device)
        g, keep = grid.cfg_grid()
        devs = None if devices is None else np.ascontiguousarray(devices, dtype=np.int32)
        h = C.c_void_p()
        r = self.L.cfg_group_create(C.byref(self.params), C.byref(g), nranks, _p(devs), C.byref(h))
        if r != 0:
            raise ChanflowError(f"cfg_group_create failed ({ERRORS.get(r, r)})")
        self.h = h
        self.part = partition(grid.nx, grid.nz, grid.nz2, nranks)
        self.ranks = []
        for i in range(nranks):
            f = ChannelFlow.__new__(ChannelFlow)
            f.L, f.grid, f.precision, f.params = self.L, grid, precision, self.params
            f.nx, f.ny, f.nz, f.nx2, f.nz2 = grid.nx, grid.ny, grid.nz, grid.nx2, grid.nz2
            f.nxh = int(self.part["nx_proc"][i])
            f.h = C.c_void_p(self.L.cfg_group_rank(self.h, i))
            f._owned = False
            f.step = 0
            self.ranks.append(f)

    def _chk(self, r, rank=0):
        if r != 0:
            msg = self.L.cfg_last_error(self.ranks[rank].h)
            raise ChanflowError(f"{ERRORS.get(r, r)}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "h", None):
            for f in self.ranks:
                f.h = None
            self.L.cfg_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _slab(self, i):
        x0 = int(self.part["x_start"][i])
        return slice(x0, x0 + int(self.part["nx_proc"][i]))

    def upload_state(self, data1=None, data2=None, data4=None):
        """Whole-field arrays in the reference's layouts, split by kx slab."""
        for i, f in enumerate(self.ranks):
            sl = self._slab(i)
            f.upload_state(None if data1 is None else data1[:, sl],
                           None if data2 is None else data2[..., sl],
                           None if data4 is None else data4[..., sl])

    def download_state(self):
        parts = [f.download_state() for f in self.ranks]
        d1 = np.concatenate([p[0] for p in parts], axis=1)
        d2 = np.concatenate([p[1] for p in parts], axis=3)
        d4 = np.concatenate([p[2] for p in parts], axis=2)
        return np.asfortranarray(d1), np.asfortranarray(d2), np.asfortranarray(d4)

    def set_scalars(self, t_total, dt, p_grad, d_um_dy=None):
        for f in self.ranks:
            f.set_scalars(t_total, dt, p_grad, d_um_dy)

    def scalars(self, rank=0):
        return self.ranks[rank].scalars()

    def timestep(self, n=1):
        self._chk(self.L.cfg_group_timestep(self.h, n))

    def synchronize(self):
        self._chk(self.L.cfg_group_synchronize(self.h))

    def status(self):
        return [f.status() for f in self.ranks]


_BARRIER = C.CFUNCTYPE(C.c_int, C.c_void_p)


class Rank(ChannelFlow):
    """One rank of a multi-process run (cfg_rank_*, one process per GPU as
    under mpirun): this process's slabs of one field (distribute_data,
    PFC/setup.f90:298-437); the other ranks' transpose targets are reached
    through CUDA IPC mappings.  After record()s have been all-gathered and
    passed to connect(), timestep() advances the field; `barrier` (default
    torch.distributed.barrier) runs between the phases of every substep and
    must return once all ranks have called it.  Arrays passed to
    upload_state are this rank's local slabs, data1(nz, nx_proc, ny+1, 3)."""

    def __init__(self, grid, rank, nranks, re=2500.0, dt=0.005, beta=0.0, cfl_max=0.95, fix_mass=1,
                 dt_flag=0, precision=FP64, device=0):
        self.L = load_library()
        self.grid = grid
        self.nx, self.ny, self.nz = grid.nx, grid.ny, grid.nz
        self.nx2, self.nz2 = grid.nx2, grid.nz2
        self.precision = precision
        self.rank, self.nranks = rank, nranks
        self.part = partition(grid.nx, grid.nz, grid.nz2, nranks)
        self.nxh = int(self.part["nx_proc"][rank])
        self.x_start = int(self.part["x_start"][rank])
        self.params = CfgParams(grid.nx, grid.ny, grid.nz, grid.nx2, grid.nz2, re, grid.lx, grid.lz,
                                beta, dt, cfl_max, fix_mass, dt_flag, 0.0, 0.0, precision, device)
        g, keep = grid.cfg_grid()
        h = C.c_void_p()
        r = self.L.cfg_rank_create(C.byref(self.params), C.byref(g), rank, nranks, C.byref(h))
        if r != 0:
            raise ChanflowError(f"cfg_rank_create failed ({ERRORS.get(r, r)})")
        self.h = h
        self.step = 0

    def slab(self):
        """Slice of the global kx index held by this rank."""
        return slice(self.x_start, self.x_start + self.nxh)

    def record(self):
        b = C.create_string_buffer(self.L.cfg_rank_record_size())
        self._chk(self.L.cfg_rank_export(self.h, b))
        return b.raw

    def nccl_barrier(self):
        """A stream-ordered barrier for timestep(ordered=True): an all-reduce
        of one word on this rank's stream (torch.distributed with NCCL, one
        GPU per rank)."""
        import torch
        import torch.distributed as dist
        dev = torch.device("cuda", self.params.device)
        word = torch.zeros(1, device=dev)
        stream = torch.cuda.ExternalStream(self.stream_ptr(), device=dev)

        def barrier():
            with torch.cuda.stream(stream):
                dist.all_reduce(word)

        return barrier

    def connect(self, records):
        blob = b"".join(records)
        assert len(blob) == self.nranks * self.L.cfg_rank_record_size()
        buf = C.create_string_buffer(blob, len(blob))
        self._chk(self.L.cfg_rank_connect(self.h, buf))

    def timestep(self, nsteps=1, barrier=None, ordered=False):
        """ordered=False: `barrier` is a host barrier (the rank's stream is
        synchronised before it).  ordered=True: `barrier` must enqueue a
        stream-ordered barrier on stream_ptr() (nccl_barrier() does, with an
        NCCL all-reduce of one word), and the host never waits."""
        if barrier is None:
            import torch.distributed as dist
            barrier = self.nccl_barrier() if ordered else dist.barrier
        err = []

        def cb(_user):
            try:
                barrier()
                return 0
            except Exception as e:  # reported after the C call returns
                err.append(e)
                return -1

        fn = _BARRIER(cb)
        step = self.L.cfg_rank_timestep_ordered if ordered else self.L.cfg_rank_timestep
        r = step(self.h, nsteps, C.cast(fn, C.c_void_p), None)
        if err:
            raise err[0]
        self._chk(r)


class Mlp:
    """The learned subgrid-stress closure network on the tensor cores
    (cfg_mlp_*): 10 -> 64 -> 64 -> 64 -> 6, GELU, BF16 operands, FP32
    accumulation.  Data arguments are device pointers (e.g. torch tensors'
    data_ptr()); stream is a cudaStream_t value (None: the default stream)."""

    def __init__(self, device=0, params=None):
        self.L = load_library()
        self.nparams = self.L.cfg_mlp_nparams()
        h = _VP()
        r = self.L.cfg_mlp_create(device, C.byref(h))
        if r != 0:
            raise ChanflowError(f"cfg_mlp_create failed ({r})")
        self.h = h
        if params is not None:
            self.set_params(params)

    def _chk(self, r):
        if r != 0:
            raise ChanflowError(f"cfg_mlp call failed ({r})")

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.nparams:
            raise ChanflowError(f"expected {self.nparams} parameters, got {p.size}")
        self._chk(self.L.cfg_mlp_set_params(self.h, p.ctypes.data))

    def get_params(self):
        p = np.zeros(self.nparams, np.float32)
        self._chk(self.L.cfg_mlp_get_params(self.h, p.ctypes.data))
        return p

    def forward(self, x_ptr, y_ptr, n, stream=None):
        self._chk(self.L.cfg_mlp_forward(self.h, x_ptr, y_ptr, int(n), stream))

    def accumulate_grad(self, x_ptr, t_ptr, idx_ptr, batch, stream=None):
        self._chk(self.L.cfg_mlp_accumulate_grad(self.h, x_ptr, t_ptr, idx_ptr, int(batch), stream))

    def grads(self):
        g = np.zeros(self.nparams, np.float32)
        loss = C.c_float()
        self._chk(self.L.cfg_mlp_get_grads(self.h, g.ctypes.data, C.byref(loss)))
        return g, loss.value

    def zero_grads(self, stream=None):
        self._chk(self.L.cfg_mlp_zero_grads(self.h, stream))

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self._chk(self.L.cfg_mlp_adam_step(self.h, lr, beta1, beta2, eps, stream))

    def status(self):
        return self.L.cfg_mlp_status(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.L.cfg_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ensemble:
    """cfg_ensemble: independent ChannelFlow members on one GPU advanced
    together, one CUDA graph launch per step after the first (configuration
    C5: many grids, Reynolds numbers, seeds and forcings).  autotune tunes the
    tiles once per distinct grid.  batched: None keeps the library's default
    (batched when every member allows it), True requires the batched layout
    (one launch per kernel per class of equal grids, over a member table),
    False one graph branch per member.  Call synchronize() before reading a
    member."""

    def __init__(self, members, autotune=True, batched=None):
        self.L = load_library()
        self.members = list(members)
        hs = (C.c_void_p * len(self.members))(*[m.h.value for m in self.members])
        h = C.c_void_p()
        r = self.L.cfg_ensemble_create(len(self.members), C.cast(hs, C.c_void_p), 1 if autotune else 0,
                                       C.byref(h))
        if r != 0:
            msg = self.L.cfg_last_error(self.members[0].h)
            raise ChanflowError(f"cfg_ensemble_create failed ({ERRORS.get(r, r)}): {msg.decode() if msg else ''}")
        self.h = h
        if batched is not None:
            r = self.L.cfg_ensemble_set_batched(self.h, 1 if batched else 0)
            if r != 0:
                self.close()
                raise ChanflowError(f"cfg_ensemble_set_batched failed ({ERRORS.get(r, r)})")

    @property
    def batched(self):
        return bool(self.L.cfg_ensemble_batched(self.h))

    def timestep(self, nsteps=1):
        r = self.L.cfg_ensemble_timestep(self.h, nsteps)
        if r != 0:
            raise ChanflowError(f"cfg_ensemble_timestep failed ({ERRORS.get(r, r)})")

    def synchronize(self):
        if self.L.cfg_ensemble_synchronize(self.h) != 0:
            raise ChanflowError("cfg_ensemble_synchronize failed")

    def stream_ptr(self):
        return self.L.cfg_ensemble_stream(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.L.cfg_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

