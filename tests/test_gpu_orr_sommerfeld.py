"""The Orr-Sommerfeld known-answer test on the GPU (the reference's
which_test 2: PFC/init_vel.f90:95-114, PFC/setup.f90:163-171,1386-1388,
growth output PFC/pass2.f90:126-133).

Laminar Poiseuille flow at Re 7500 plus 1e-4 times the least-stable
two-dimensional mode (alpha = 1, lx = 2 pi), fix_mass 0, the reference's
stretch 2.75, dt = 2 (2 pi / 0.24989154) / tend.  The mode's energy grows
as exp(2 alpha c_i t), c = 0.24989154 + 0.00223497 i.

- FP64: the mode energy every 10 steps equals the oracle's to 1e-9
  (relative), and the growth rate over the second period is within 1 % of
  2 alpha c_i at ny = 193, its error falling more than 3x from ny = 97 (the
  second-order y differences; the DNS mean also drifts slowly from 1 - yh^2
  toward the discrete steady profile, so the DNS rate is not the discrete
  eigenvalue exactly).
- Mixed precision: the growth rate within 2e-3 (relative) of FP64's.
- The Arnoldi path (the linearized matvec about 1 - yh^2, T = 10, on vectors
  of the kx = 1, kz = 0 column): the FP64 propagator's leading eigenvalue
  equals the oracle's to 1e-8, mixed equals FP64 to 1e-5, and the discrete
  phase speeds at ny = 97 and 193, Richardson-extrapolated, match
  c = 0.24989154 + 0.00223497 i (c_r to 1e-5, c_i to 0.2 %).
- chanflow_run with a which_test 2 flow.dat and an efn.m written by
  orr_sommerfeld.write_efn takes the reference's dt and writes the mode's
  energy to fort.80 as the reference does; it equals the oracle's to 1e-9.
"""
import importlib
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

C_OS = 0.24989154 + 0.00223497j
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN_BIN = os.path.join(ROOT, "3d-navier-stokes-thesis-paper_b200", "lib", "chanflow_run")
NX, NZ, STRETCH = 16, 8, 2.75


@pytest.fixture(scope="module")
def osm(cf):
    return importlib.import_module("chanflow_b200.orr_sommerfeld")


@pytest.fixture(scope="module")
def efn(osm):
    c, u, v, _ = osm.least_stable()
    return osm.efn_columns(u, v)


def os_dt(tend):
    return 2 * (2 * np.pi / 0.24989154) / tend


def growth(e, t):
    h = len(e) // 2
    return 0.5 * np.log(e[-1] / e[h]) / (t[-1] - t[h])


def run_gpu(cf, osm, efn, ny, prec, tend=500):
    grid = cf.Grid(NX, ny, NZ, lx=2 * np.pi, lz=2 * np.pi, stretch=STRETCH)
    f = cf.ChannelFlow(grid, re=7500.0, dt=os_dt(tend), fix_mass=0, precision=prec)
    f.define_initial_field(2, ampl=1e-4, efn=efn)
    e, t = [], []
    for _ in range(tend // 10):
        f.timestep(10)
        e.append(osm.mode_energy(f.download_state()[0], grid.dyh))
        t.append(f.scalars()["t_total"])
    assert f.status() == 0
    f.close()
    return np.array(e), np.array(t)


def run_oracle(cf, orc, osm, efn, ny, tend=500):
    grid = cf.Grid(NX, ny, NZ, lx=2 * np.pi, lz=2 * np.pi, stretch=STRETCH)
    o = orc.Oracle(NX, ny, NZ, re=7500.0, dt=os_dt(tend), stretch=STRETCH, fix_mass=0, lx=2 * np.pi,
                   lz=2 * np.pi)
    o.init_from_velocity(cf.initial_field(grid, 2, ampl=1e-4, efn=efn))
    dyh = o.grid("dyh")
    e, t = [], []
    for _ in range(tend // 10):
        o.timestep(10)
        e.append(osm.mode_energy(o.data1, dyh))
        t.append(o.scalars()[0])
    o.close()
    return np.array(e), np.array(t)


@pytest.fixture(scope="module")
def fp64_runs(cf, orc, osm, efn):
    return {ny: (run_gpu(cf, osm, efn, ny, cf.FP64), run_oracle(cf, orc, osm, efn, ny)) for ny in (97, 193)}


def test_os_growth_fp64_matches_oracle_and_theory(fp64_runs):
    ci = C_OS.imag
    g = {}
    for ny, ((e, t), (eo, to)) in fp64_runs.items():
        assert np.abs(t - to).max() < 1e-10
        assert np.abs(e / eo - 1).max() < 1e-9, (ny, np.abs(e / eo - 1).max())
        g[ny] = growth(e, t)
    # within the y discretization error (the oracle: 0.51 % at ny = 193),
    # which falls with the grid
    assert abs(g[193] - ci) < 0.01 * ci, g
    assert abs(g[193] - ci) < abs(g[97] - ci) / 3, g


def test_os_growth_mixed_matches_fp64(cf, osm, efn, fp64_runs):
    (e64, t64), _ = fp64_runs[193]
    e, t = run_gpu(cf, osm, efn, 193, cf.MIXED)
    g64, g = growth(e64, t64), growth(e, t)
    print(f"os growth fp64 {g64:.9e} mixed {g:.9e} rel {abs(g - g64) / g64:.3e}")
    assert abs(g - g64) < 2e-3 * g64, (g, g64)


def column_vector(ny, col):
    """A real Arnoldi vector (nx, nz, ny+1, 3) holding only the kx = 1, kz = 0
    Fourier column col (ny+1, 3) complex: 2 Re(col exp(i x))."""
    x = 2 * np.pi * np.arange(NX) / NX
    ph = np.exp(1j * x)
    v = 2 * np.real(ph[:, None, None, None] * col[None, None, :, :]) * np.ones((1, NZ, 1, 1))
    return np.asfortranarray(v).ravel(order="F")


def arnoldi_leading(cf, orc, ny, prec, tend_T=100, dt=0.1):
    """Leading eigenvalue mu of the T = tend_T*dt propagator about Poiseuille
    flow on vectors of the kx = 1, kz = 0 column (the linearized operator
    about a profile U(y) does not couple columns, so the Krylov space stays
    in it); prec None runs the oracle's matvec."""
    from scipy.sparse.linalg import LinearOperator, eigs
    grid = cf.Grid(NX, ny, NZ, lx=2 * np.pi, lz=2 * np.pi, stretch=STRETCH)
    base = np.zeros((ny + 1, 3), order="F")
    base[:, 0] = 1 - grid.yh ** 2
    rng = np.random.default_rng(11)
    v0 = column_vector(ny, rng.standard_normal((ny + 1, 3)) + 1j * rng.standard_normal((ny + 1, 3)))
    n = v0.size
    if prec is None:
        o = orc.Oracle(NX, ny, NZ, re=7500.0, dt=dt, stretch=STRETCH, fix_mass=0, lx=2 * np.pi, lz=2 * np.pi)
        o.baseflow[:, :] = base
        mv = lambda x: o.arnoldi_matvec(np.real(np.ravel(x)).reshape((NX, NZ, ny + 1, 3), order="F"),
                                        tend_T).ravel(order="F")
    else:
        f = cf.ChannelFlow(grid, re=7500.0, dt=dt, fix_mass=0, precision=prec)
        f.set_baseflow(base)
        mv = lambda x: f.arnoldi_matvec(np.real(np.ravel(x)), tend_T)
    # FP32 transforms leave ~1e-7 noise in the mixed matvec: its tolerance is
    # looser (an unreachable one would run ARPACK to its iteration limit)
    tol = 1e-7 if prec == cf.MIXED else 1e-12
    mu = eigs(LinearOperator((n, n), matvec=mv, dtype=np.float64), k=2, ncv=16, which="LM", tol=tol,
              v0=v0, maxiter=60, return_eigenvectors=False)
    (o if prec is None else f).close()
    mu = mu[np.argmax(np.abs(mu))]
    lam = np.log(mu) / (tend_T * dt)          # = -i alpha c, or its conjugate
    return mu, abs(lam.imag) + 1j * lam.real


def test_os_mode_from_arnoldi(cf, orc):
    """The Arnoldi path finds the Orr-Sommerfeld mode: the FP64 GPU
    propagator's leading eigenvalue equals the oracle's to 1e-8 (ny = 97),
    mixed precision's equals FP64's to 1e-5, and the discrete phase speeds
    at ny = 97 and 193, Richardson-extrapolated, give c_r within 1e-5 of the
    reference's 0.24989154 and c_i within 0.2 % of 0.00223497 (measured on
    the oracle: c = 0.248604 + 0.0021716 i and 0.249569 + 0.0022199 i,
    extrapolated 0.249891 + 0.0022360 i)."""
    mu64, c97 = arnoldi_leading(cf, orc, 97, cf.FP64)
    muo, _ = arnoldi_leading(cf, orc, 97, None)
    mum, _ = arnoldi_leading(cf, orc, 97, cf.MIXED)
    _, c193 = arnoldi_leading(cf, orc, 193, cf.FP64)
    print(f"arnoldi c(97) {c97:.8f} c(193) {c193:.8f} fp64-oracle {abs(mu64 - muo):.2e} "
          f"mixed-fp64 {abs(mum - mu64):.2e}")
    assert abs(mu64 - muo) < 1e-8 * abs(muo), (mu64, muo)
    assert abs(mum - mu64) < 1e-5 * abs(mu64), (mum, mu64)
    cx = c193 + (c193 - c97) / 3
    assert abs(cx.real - C_OS.real) < 1e-5, cx
    assert abs(cx.imag - C_OS.imag) < 0.002 * C_OS.imag, cx


FLOW_OS = """0.d0	re	(which_test 2 sets Re 7500)
		Orr-Sommerfeld test: which_test 2


0.d+0	ctrlu
0.d+0	ctrlw
2.d0	lx
1.0d0	lx/lz
1	scale lengths by pi
16	nx
97	ny
8	nz
24	nx2
12	nz2
0	nscalar
0.7d0	pr
0.4d0	pr_t
0	split_scalar
0	subgrid
3	filter_dim
0	lagr_avg
0	dynamic_scalar
{tend}	tend
10	output_step
100	save_step
100	l2_step
0	read_vel
0	save_vel
0	vel_out

0	snap_out

2	which_test
1.d-4	disturb_ampl










0	test_run
1	fix_mass
0	dt_flag
0	divg_check
0.0d0	beta


OUTPUT FILE PARAMETERS
1	xskip
1	yskip
1	zskip
0	filter_output
GRID PARAMETERS
0	bl_grid
1.d0	ly
0.5d0	ly_half
0.33d0	delta_bl
5	nbl
JET PARAMETERS
0	crossflow
0	filter_jet_profile

1.d0	jet_diam
0.d0	forcing_phase

TOP WALL JET
0.125d0	xjet_top
0.5d0	zjet_top
0.d0	jetmag_top
0.0d0	forcing_top
0.2d0	for_freq_top
0.0d0	swirl_top
BOTTOM WALL JET
0.125d0	xjet_bot
0.5d0	zjet_bot
0.d0	jetmag_bot
0.0d0	forcing_bot
0.19d0	for_freq_bot
0.0d0	swirl_bot
FRINGE
10.d0	fringe_gain

0	xfringe
0.25d0	frac_xbuff
0.10d0	buff_xrise
0.05d0	buff_xfall

0	zfringe
0.10d0	frac_zbuff
0.05d0	buff_zrise
0.05d0	buff_zfall
B200 EXTENSION BLOCK (ignored by the Fortran reader)
2.75d0	stretch
0	precision
"""


@pytest.mark.skipif(not os.path.exists(RUN_BIN), reason="chanflow_run not built (build())")
def test_run_program_orr_sommerfeld(cf, orc, osm, efn, tmp_path):
    """The program's fort.80 record of the mode energy (every output_step =
    10 steps) equals the oracle's to 1e-9; dt is the reference's."""
    tend = 500
    (tmp_path / "flow.dat").write_text(FLOW_OS.format(tend=tend))
    osm.write_efn(str(tmp_path / "efn.m"))
    r = subprocess.run([RUN_BIN, "flow.dat"], capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr + r.stdout
    dt = float(re.search(r"INITIAL DT = (\S+)", r.stdout).group(1))
    assert abs(dt - os_dt(tend)) < 1e-15
    rec = np.array([[float(v) for v in ln.split()] for ln in (tmp_path / "fort.80").read_text().splitlines()])
    assert rec.shape == (tend // 10, 4)
    eo, to = run_oracle(cf, orc, osm, efn, 97, tend)
    assert np.abs(rec[:, 1] / eo - 1).max() < 1e-9
    assert abs(growth(rec[:, 1], to) - C_OS.imag) < 0.025 * C_OS.imag
