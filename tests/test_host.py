"""Host-side logic of the product, no GPU needed: the C-ABI library loads and
exports every symbol its headers declare; the C++ setup (flow.dat reader,
define_coordinates, wavenumbers, seeded initial field) matches the oracle."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("chanflow.h", "chanflow_host.h")]


def declared_functions():
    names = []
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(cf[gh]_[a-z0-9_]+)\s*\(", txt):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_all_declared_symbols(cf):
    L = cf.load_library()
    decl = declared_functions()
    assert len(decl) >= 30
    for n in decl:
        assert hasattr(L, n), n
        assert n in cf.SYMBOLS, n


def test_missing_library_fails_loudly(cf, tmp_path):
    import importlib
    mod = importlib.import_module("chanflow_b200.chanflow")
    saved = mod._lib
    mod._lib = None
    try:
        with pytest.raises(RuntimeError):
            mod.load_library(str(tmp_path / "nope.so"))
    finally:
        mod._lib = saved


@pytest.mark.parametrize("ny,stretch,uniform", [(33, 1.5, 0), (200, 2.75, 0), (17, 2.75, 1)])
def test_grid_matches_oracle(cf, orc, ny, stretch, uniform):
    g = cf.Grid(32, ny, 16, lx=4 * np.pi, lz=2 * np.pi, stretch=stretch, uniform=uniform)
    o = orc.Oracle(32, ny, 16, lx=4 * np.pi, lz=2 * np.pi, stretch=stretch, uniform_grid=uniform)
    for name in ("y", "yh", "hh", "hn", "dh", "dn", "dyh", "dy", "kx", "kz", "xcoord", "zcoord"):
        assert np.array_equal(getattr(g, name).ravel(order="F"), o.grid(name).ravel(order="F")), name
    for name in ("iu", "dm", "d2h", "d2n"):
        assert np.array_equal(getattr(g, name), o.grid(name)), name


def test_rng_matches_oracle(cf, orc):
    L = cf.load_library()
    O = orc.lib()
    for args in [(1, 0, 1, 0, 0), (7, 3, 5, 100, 3), (2 ** 40 + 5, 64, 127, 193, 2)]:
        assert L.cfh_rng_u01(*args) == O.orc_rng_u01(*args)


@pytest.mark.parametrize("which", [1, 4, 6, 10])
def test_initial_field_matches_oracle(cf, orc, which):
    g = cf.Grid(16, 17, 12, lx=4 * np.pi, lz=2 * np.pi, stretch=1.5)
    d1 = cf.initial_field(g, which, seed=11, ampl=1e-2)
    o = orc.Oracle(16, 17, 12, lx=4 * np.pi, lz=2 * np.pi, stretch=1.5)
    o.initial_velocity(which, seed=11, ampl=1e-2)
    np.testing.assert_allclose(d1, o.data1, rtol=0, atol=1e-15)


FLOW_C1 = os.path.join(os.path.dirname(__file__), "golden", "flow_c1.dat")


def test_flow_dat_reader(cf):
    run = cf.read_flow_dat(FLOW_C1)
    assert (run.nx, run.ny, run.nz, run.nx2, run.nz2) == (32, 33, 32, 48, 48)
    assert run.re == 2500.0
    assert abs(run.lx - 4 * np.pi) < 1e-15 and abs(run.lz - 2 * np.pi) < 1e-15
    assert run.fix_mass == 1 and run.dt_flag == 0 and run.tend == 100
    assert run.which_test == 10 and run.stretch == 1.5 and run.dt == 0.005
    assert run.seed == 1 and abs(run.disturb_ampl - 1e-3) < 1e-18


def test_flow_dat_reader_rejects_truncated(cf, tmp_path):
    lines = open(FLOW_C1).read().splitlines()[:40]
    p = tmp_path / "flow.dat"
    p.write_text("\n".join(lines) + "\n")
    with pytest.raises(cf.ChanflowError):
        cf.read_flow_dat(str(p))


def test_flow_dat_reader_on_reference_file(cf):
    """The reference's own flow.dat (tests/golden/flow_ref.dat, copied from
    ParallelFortran-Code/flow.dat by tests/golden/make_fixtures.py)."""
    run = cf.read_flow_dat(os.path.join(ROOT, "tests", "golden", "flow_ref.dat"))
    assert (run.nx, run.ny, run.nz, run.nx2, run.nz2) == (128, 200, 64, 192, 96)
    assert run.re == 7500.0 and run.which_test == 9 and run.l2_step == 20
    assert abs(run.lx - 6 * np.pi) < 1e-14 and abs(run.lz - 2 * np.pi) < 1e-14


def test_arnoldi_driver_eigenvalues(cf):
    """arnoldi_eigs on an operator of known spectrum: Phi_T = exp(L T) with
    L diagonal; the driver must return mu = exp(lambda T) ordered by |mu| and
    recover lambda = log|mu|/T + i atan2(Im mu, Re mu)/T (PFC/arnoldi.f90:803-806)."""
    import numpy as np

    class FakeFlow:
        nx, ny, nz = 4, 3, 4

        def __init__(self):
            n = self.nx * self.nz * (self.ny + 1) * 3
            rng = np.random.default_rng(0)
            self.T = 0.5
            lam = -rng.uniform(0.5, 4.0, n)
            lam[:3] = [-0.01, -0.2, -0.35]
            self.mu = np.exp(lam * self.T)
            self.lam = lam
            self.calls = 0

        def arnoldi_matvec(self, v, tend):
            assert tend == 10
            self.calls += 1
            return self.mu * v

        def scalars(self):
            return {"dt": 0.05}

    f = FakeFlow()
    mu, lam, vec = cf.chanflow.arnoldi_eigs(f, 10, nev=3, ncv=12, tol=1e-12,
                                            v0=np.ones(f.mu.size))
    np.testing.assert_allclose(mu.real, np.exp(np.array([-0.01, -0.2, -0.35]) * f.T), rtol=1e-10)
    np.testing.assert_allclose(lam.real, [-0.01, -0.2, -0.35], rtol=1e-8)
    assert np.abs(lam.imag).max() < 1e-12
    assert vec.shape == (f.mu.size, 3)


def test_partition_matches_reference_table(cf):
    """cfg_partition against the distribute_data table the reference printed
    for Nx=128, Nz=64 (Nz2=96) on 24 ranks (PFC/diagnostics.txt:17-43)."""
    import json
    gold = json.load(open(os.path.join(ROOT, "tests", "golden", "partition_nproc24.json")))
    part = cf.partition(gold["nx"], gold["nz"], gold["nz2"], gold["nproc"])
    for k in cf.PARTITION_KEYS:
        assert list(part[k]) == gold[k], k
    nxh = gold["nx"] // 2 + 1
    assert gold["xleft_zleft_zsmallleft"] == [nxh % 24, gold["nz2"] % 24, gold["nz"] % 24]


@pytest.mark.parametrize("nx,nz,nproc", [(256, 256, 8), (32, 32, 5), (6, 4, 4), (384, 384, 7)])
def test_partition_covers_grid(cf, nx, nz, nproc):
    nz2 = 3 * nz // 2
    p = cf.partition(nx, nz, nz2, nproc)
    for cnt, start, total in (("nx_proc", "x_start", nx // 2 + 1), ("nz_proc", "z_start", nz2),
                              ("nz_small_proc", "z_small_start", nz)):
        c, s = p[cnt], p[start]
        assert c.sum() == total and s[0] == 0
        assert np.all(s[1:] == np.cumsum(c)[:-1])
        assert c.max() - c.min() <= 1 and np.all(np.diff(c) <= 0)


def test_group_rejects_partition_without_whole_tiles(cf):
    # 48 z2 rows on 4 ranks: 12 rows each, not a multiple of 8 (refused on
    # the host before any device work)
    grid = cf.Grid(32, 33, 32, stretch=1.5)
    with pytest.raises(cf.ChanflowError):
        cf.Group(grid, 4)


def test_headers_compile_as_c99(tmp_path):
    """The C ABI headers are plain C (what a Fortran ISO_C_BINDING or any
    other FFI binds against): they compile as C99 with -pedantic."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    src = tmp_path / "h.c"
    src.write_text('#include "chanflow.h"\n#include "chanflow_host.h"\n'
                   "int main(void) { return (int)cfg_rank_record_size(); }\n")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                        "-I" + os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


RUN_BIN = os.path.join(ROOT, "3d-navier-stokes-thesis-paper_b200", "lib", "chanflow_run")
GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.mark.skipif(not os.path.exists(RUN_BIN), reason="chanflow_run not built")
def test_run_program_arguments(tmp_path):
    """chanflow_run (the DNS program over the C ABI): usage, a missing
    argument and an unreadable flow.dat are refused before any device work."""
    import subprocess
    r = subprocess.run([RUN_BIN, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage: chanflow_run" in r.stdout
    assert subprocess.run([RUN_BIN], capture_output=True).returncode == 2
    r = subprocess.run([RUN_BIN, str(tmp_path / "missing.dat")], capture_output=True, text=True)
    assert r.returncode == 1 and "cannot open" in r.stderr
    # --restart with read_vel = 0 in flow.dat is refused (the file would be ignored)
    r = subprocess.run([RUN_BIN, os.path.join(GOLD, "flow_c1.dat"), "--restart", str(tmp_path / "x.out")],
                       capture_output=True, text=True)
    assert r.returncode == 2 and "read_vel = 0" in r.stderr


def test_group_splits_and_gathers_kx_slabs(cf):
    """chanflow.Group's host side: whole-field arrays in the reference layouts
    go to the ranks as their kx slabs (data1 axis 1, data2 and data4 the last
    axis) and come back concatenated in rank order."""
    nx, ny, nz, n = 32, 9, 16, 3
    part = cf.partition(nx, nz, 3 * nz // 2, n)

    class FakeRank:
        def __init__(self, i):
            self.i = i
            self.got = None

        def upload_state(self, d1, d2, d4):
            self.got = (np.array(d1), np.array(d2), np.array(d4))

        def download_state(self):
            return self.got

    g = cf.Group.__new__(cf.Group)
    g.part = part
    g.ranks = [FakeRank(i) for i in range(n)]
    nxh = nx // 2 + 1
    rng = np.random.default_rng(0)
    d1 = rng.standard_normal((nz, nxh, ny + 1, 3)) + 0j
    d2 = rng.standard_normal((ny + 1, 3, nz, nxh)) + 0j
    d4 = rng.standard_normal((ny + 1, nz, nxh)) + 0j
    g.upload_state(d1, d2, d4)
    for i, r in enumerate(g.ranks):
        x0, nl = int(part["x_start"][i]), int(part["nx_proc"][i])
        np.testing.assert_array_equal(r.got[0], d1[:, x0:x0 + nl])
        np.testing.assert_array_equal(r.got[1], d2[..., x0:x0 + nl])
        np.testing.assert_array_equal(r.got[2], d4[..., x0:x0 + nl])
    b1, b2, b4 = g.download_state()
    np.testing.assert_array_equal(b1, d1)
    np.testing.assert_array_equal(b2, d2)
    np.testing.assert_array_equal(b4, d4)
    g.h = None   # nothing to destroy
