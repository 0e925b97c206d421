"""GPU parity: the sm_100a kernels behind the C ABI against the FP64 CPU oracle
on the same seeded inputs.

Tolerances (relative L2 over the whole array unless stated):
  all-FP64 path: 1e-12 per routine, 1e-10 after 100 steps (config C1);
  mixed FP32/FP64 path: 1e-5 per routine and after 100 steps (config C1).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RKC = np.array([29 / 96, -3 / 40, 1 / 6], dtype=np.float32).astype(np.float64)
RKD = np.array([37 / 160, 5 / 24, 1 / 6], dtype=np.float32).astype(np.float64)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def make(cf, orc, nx=16, ny=17, nz=16, prec=0, re=2500.0, dt=0.005, stretch=1.5, fix_mass=1,
         ctrlu=0.0, ctrlw=0.0, dt_flag=0, uniform=0, lx=4 * np.pi, lz=2 * np.pi):
    grid = cf.Grid(nx, ny, nz, lx=lx, lz=lz, stretch=stretch, uniform=uniform)
    flow = cf.ChannelFlow(grid, re=re, dt=dt, fix_mass=fix_mass, ctrlu=ctrlu, ctrlw=ctrlw,
                          dt_flag=dt_flag, precision=prec)
    o = orc.Oracle(nx, ny, nz, re=re, dt=dt, stretch=stretch, fix_mass=fix_mass, ctrlu=ctrlu,
                   ctrlw=ctrlw, dt_flag=dt_flag, uniform_grid=uniform, lx=lx, lz=lz)
    return grid, flow, o


TOL = {0: 1e-12, 1: 1e-5}


@pytest.mark.parametrize("prec", [0, 1])
def test_xz_transforms(cf, orc, prec):
    grid, flow, o = make(cf, orc, 24, 9, 16, prec=prec)
    rng = np.random.default_rng(5)
    c = rng.standard_normal((16, 13)) + 1j * rng.standard_normal((16, 13))
    np.testing.assert_array_less(rel(flow.xz_fft_complex_to_real(c), o.xz_c2r(c)), TOL[prec])
    d = rng.standard_normal((36, 24))
    np.testing.assert_array_less(rel(flow.xz_fft_real_to_complex(d), o.xz_r2c(d)), TOL[prec])


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("rk", [1, 2])
def test_nonlinear(cf, orc, prec, rk):
    grid, flow, o = make(cf, orc, 32, 33, 16, prec=prec)
    o.init_field(10, seed=5, ampl=5e-2)
    flow.upload_state(o.data1.copy(), o.data2.copy(), o.data4.copy())
    o.set_step(1, rk)
    o.nonlinear()
    flow.nonlinear(1, rk)
    d1, _, _ = flow.download_state()
    assert rel(d1, o.data1) < TOL[prec]
    if rk == 1:
        sc = flow.scalars()
        assert abs(sc["cfl_max"] - o.cfl[1:33].max()) < 1e-6 * o.cfl[1:33].max()


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("rk", [1, 2, 3])
def test_rhs_solve(cf, orc, prec, rk):
    grid, flow, o = make(cf, orc, 32, 33, 16, prec=prec)
    o.init_field(10, seed=6, ampl=5e-2)
    o.set_step(1, rk)
    o.nonlinear()
    dud = o.d_um_dy.copy()
    t, dt, pg = o.scalars()
    flow.upload_state(o.data1.copy(), o.data2.copy(), o.data4.copy())
    flow.set_scalars(t, dt, pg, dud)
    o.rhs_solve()
    flow.rhs_solve(1, rk)
    d1, d2, d4 = flow.download_state()
    tol = TOL[prec]
    assert rel(d1, o.data1) < tol
    assert rel(d2, o.data2) < tol
    assert rel(d4, o.data4) < 10 * tol
    sc = flow.scalars()
    assert abs(sc["p_grad"] - o.scalars()[2]) < (1e-10 if prec == 0 else 1e-6) * abs(o.scalars()[2])
    assert rel(sc["d_um_dy"], o.d_um_dy) < (1e-12 if prec == 0 else 1e-9)


@pytest.mark.parametrize("prec", [0, 1])
def test_initial_field(cf, orc, prec):
    grid, flow, o = make(cf, orc, 32, 33, 32, prec=prec)
    o.init_field(10, seed=1, ampl=1e-3)
    flow.define_initial_field(10, seed=1, ampl=1e-3)
    d1, d2, d4 = flow.download_state()
    assert rel(d1, o.data1) < TOL[prec]
    assert rel(d2, o.data2) < TOL[prec]
    assert rel(d4, o.data4) < 10 * TOL[prec]
    assert rel(flow.scalars()["d_um_dy"], o.d_um_dy) < 1e-12


@pytest.mark.parametrize("prec,tol,ptol", [(0, 1e-10, 1e-10), (1, 1e-5, 3e-5)])
def test_config_c1_100_steps(cf, orc, prec, tol, ptol):
    """Config C1: 32x33x32, Re 2500, stretch 1.5, laminar + 1e-3 k^-2 noise,
    constant flux, dt 0.005, 100 steps.  The perturbation (every Fourier
    column but the mean) is gated on its own: FP64 1e-10 (measured on a B200
    2.6e-14), mixed 3e-5 (measured 5.6e-6 with the whole velocity in the FP32
    transforms; the mean split keeps it lower, see
    test_gpu_metric_config.py)."""
    grid, flow, o = make(cf, orc, 32, 33, 32, prec=prec)
    o.init_field(10, seed=1, ampl=1e-3)
    flow.define_initial_field(10, seed=1, ampl=1e-3)
    o.timestep(100)
    flow.timestep(100)
    d1, d2, d4 = flow.download_state()
    e = rel(d1, o.data1)
    assert e < tol, e
    # the perturbation (non-mean part) is also checked on its own
    pert = d1.copy(); pert[0, 0] = 0
    opert = o.data1.copy(); opert[0, 0] = 0
    assert rel(pert, opert) < ptol, rel(pert, opert)
    sc = flow.scalars()
    t, dt, pg = o.scalars()
    assert abs(sc["t_total"] - t) < 1e-12
    assert abs(sc["p_grad"] - pg) < 1e3 * tol * abs(pg)
    q, div = flow.diagnostics()
    assert abs(q - o.bulk_flux()) < 1e-9
    assert div < (1e-12 if prec == 0 else 1e-6)
    assert flow.status() == 0


@pytest.mark.parametrize("prec", [0, 1])
def test_boundary_feedback(cf, orc, prec):
    grid, flow, o = make(cf, orc, 32, 33, 16, prec=prec, ctrlu=0.5, ctrlw=0.3)
    o.init_field(10, seed=9, ampl=5e-2)
    flow.upload_state(o.data1.copy(), o.data2.copy(), o.data4.copy())
    t, dt, pg = o.scalars()
    flow.set_scalars(t, dt, pg, o.d_um_dy.copy())
    o.boundary()
    flow.boundary()
    top, bot = flow.wall_bc()
    assert rel(top, o.cbc_top) < TOL[prec]
    assert rel(bot, o.cbc_bot) < TOL[prec]
    # and two full steps with the feedback law active
    o.timestep(2)
    flow.timestep(2)
    d1, _, _ = flow.download_state()
    assert rel(d1, o.data1) < (1e-11 if prec == 0 else 1e-5)


@pytest.mark.parametrize("prec", [0, 1])
def test_l2_norm(cf, orc, prec):
    grid, flow, o = make(cf, orc, 32, 33, 16, prec=prec)
    o.init_field(10, seed=2, ampl=1e-2)
    flow.define_initial_field(10, seed=2, ampl=1e-2)
    l2, drag = flow.l2_norm()
    ol2, odrag = o.l2_norm()
    assert abs(l2 - ol2) < (1e-10 if prec == 0 else 1e-5) * ol2
    assert abs(drag - odrag) < 1e-9 * abs(odrag)


def test_which_test6_on_gpu(cf, orc):
    """The analytic decaying-vortex solution (PFC/main_mpi.f90:121-161) run on the
    GPU, substep by substep with the analytic wall values in cbc."""
    ny, nx, nz, re = 33, 8, 4, 10.0
    dt = 0.5 / ny
    grid, flow, o = make(cf, orc, nx, ny, nz, re=re, dt=dt, fix_mass=0, uniform=1, lx=2.0, lz=2.0,
                         stretch=2.75)
    flow.define_initial_field(6)
    pi = np.pi
    t = 0.0
    top = np.zeros((nz, nx // 2 + 1, 3), np.complex128, order="F")
    bot = np.zeros_like(top)
    for step in range(1, int(1 / dt) + 1):
        for rk in range(1, 4):
            tt = t + dt * np.sum(RKC[:rk] + RKD[:rk])
            top[0, 1, 0] = -0.5 * np.exp(-2 * pi ** 2 * tt / re)
            bot[0, 1, 0] = 0.5 * np.exp(-2 * pi ** 2 * tt / re)
            flow.set_wall_bc(top, bot)
            flow.nonlinear(step, rk)
            flow.rhs_solve(step, rk)
        t += dt
        flow.set_scalars(t, dt, 0.0)
    d1, _, _ = flow.download_state()
    xs = np.arange(grid.nx2)
    eu = max(np.abs(flow.xz_fft_complex_to_real(d1[:, :, j, 0]) + np.cos(2 * pi * xs / grid.nx2)[:, None]
                    * np.sin(pi * grid.yh[j]) * np.exp(-2 * pi ** 2 * t / re)).max() for j in range(ny + 1))
    assert eu < 6e-5   # 4.5e-5 at ny=33 (2nd order, see test_oracle)


@pytest.mark.parametrize("prec", [0, 1])
def test_linearized(cf, orc, prec):
    grid, flow, o = make(cf, orc, 32, 33, 16, prec=prec, fix_mass=0)
    base = np.zeros((34, 3), order="F")
    base[:, 0] = 1 - grid.yh ** 2
    o.baseflow[:, :] = base
    flow.set_baseflow(base)
    o.init_field(10, seed=4, ampl=1e-3)
    o.data1[0, 0] = 0
    flow.upload_state(o.data1.copy(), o.data2.copy(), o.data4.copy())
    o.set_step(1, 1)
    o.nonlinear_linearized()
    flow.nonlinear_linearized(1, 1)
    d1, _, _ = flow.download_state()
    assert rel(d1, o.data1) < TOL[prec]
    assert abs(flow.scalars()["cfl_max"] - o.cfl[1:33].max()) < 1e-6 * o.cfl[1:33].max()


def test_cfl_abort_is_a_status(cf, orc):
    grid, flow, o = make(cf, orc, 16, 17, 16, dt=2.0)
    flow.define_initial_field(10, seed=3, ampl=1e-2)
    flow.timestep(1)
    assert flow.status() == -4


@pytest.mark.parametrize("prec", [0, 1])
def test_adaptive_dt_against_oracle(cf, orc, prec):
    """dt_flag = 1 (PFC/pass1.f90:107-124): after each step's first substep
    dt moves toward cfl_max/cfl (dt_temp = dt*cfl_max/cfl, dt = min(dt_temp,
    dt + (dt_temp - dt)*dt/(1 + dt))).  From 0.005 the rule raises dt to ~0.1
    in 20 steps at 32x33x32; the dt sequence and the state follow the oracle:
    FP64 dt to 1e-12, state 1e-10 (measured 1.4e-15, 1.1e-15); mixed dt to
    1e-6, state 1e-5 whole and 1e-4 perturbation (measured 4.5e-8, 4.2e-8,
    2.9e-5)."""
    grid, flow, o = make(cf, orc, 32, 33, 32, prec=prec, dt_flag=1)
    o.init_field(10, seed=1, ampl=1e-3)
    flow.define_initial_field(10, seed=1, ampl=1e-3)
    gd, od = [], []
    for _ in range(20):
        o.timestep(1)
        flow.timestep(1)
        od.append(o.scalars()[1])
        gd.append(flow.scalars()["dt"])
    od, gd = np.array(od), np.array(gd)
    assert od[-1] > 10 * od[0]          # the rule did adapt dt
    assert np.abs(gd / od - 1).max() < (1e-12 if prec == 0 else 1e-6)
    d1, _, _ = flow.download_state()
    assert rel(d1, o.data1) < (1e-10 if prec == 0 else 1e-5)
    p1, po = d1.copy(), o.data1.copy()
    p1[0, 0] = 0
    po[0, 0] = 0
    assert rel(p1, po) < (1e-10 if prec == 0 else 1e-4)
    # t_total sums the dt sequence: FP64 to round-off, mixed to its dt bar
    assert abs(flow.scalars()["t_total"] - o.scalars()[0]) < (1e-12 if prec == 0 else 1e-6) * o.scalars()[0]
    assert flow.status() == 0
