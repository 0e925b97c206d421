"""The CPU oracle pinned against the reference's own known-answer data.

- PFC/makegrid.m: y/yh at ny=200, stretch 2.75 (golden fixture)
- which_test=6 analytic decaying vortices (PFC/main_mpi.f90:121-161): the
  velocity error converges at 2nd order; the walls carry the analytic
  time-dependent values the reference supplies through cbc in its
  which_test=6 branch (PFC/pass2.f90:274-277)
- constant bulk flux under fix_mass, round-off divergence
"""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
RKC = np.array([29 / 96, -3 / 40, 1 / 6], dtype=np.float32).astype(np.float64)
RKD = np.array([37 / 160, 5 / 24, 1 / 6], dtype=np.float32).astype(np.float64)


def test_fft_matches_numpy(orc):
    rng = np.random.default_rng(0)
    for n in (6, 12, 48, 72, 96, 144, 192, 288, 384, 576):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert np.abs(orc.fft(x, -1) - np.fft.fft(x)).max() < 1e-12 * n
        assert np.abs(orc.fft(x, +1) - np.fft.ifft(x) * n).max() < 1e-12 * n


def test_makegrid_golden(orc):
    g = json.load(open(os.path.join(GOLD, "makegrid_ny200.json")))
    o = orc.Oracle(128, 200, 64, re=7500, stretch=2.75, lx=6 * np.pi, lz=2 * np.pi)
    assert np.abs(o.grid("y") - np.array(g["y"])).max() <= 0.5e-8 + 1e-15
    assert np.abs(o.grid("yh") - np.array(g["yh"])).max() <= 0.5e-8 + 1e-15


def test_xz_round_trip(orc):
    """xz_fft_real_to_complex inverts xz_fft_complex_to_real on resolved modes."""
    o = orc.Oracle(16, 9, 8)
    rng = np.random.default_rng(1)
    c = rng.standard_normal((8, 9)) + 1j * rng.standard_normal((8, 9))
    c[:, 0] = c[:, 0].real          # real DC column in x
    c[4, :] = 0                     # no kz Nyquist (split convention)
    c[:, 8] = 0                     # no kx Nyquist
    # hermitian kx=0 column
    for kz in range(1, 4):
        c[8 - kz, 0] = np.conj(c[kz, 0])
    c[0, 0] = c[0, 0].real
    back = o.xz_r2c(o.xz_c2r(c))
    assert np.abs(back - c).max() < 1e-13


def _kat6(orc, ny, nx=8, nz=4):
    dt = 0.5 / ny
    tend = int(1.0 / dt)
    re = 10.0
    pi = np.pi
    o = orc.Oracle(nx, ny, nz, re=re, lx=2.0, lz=2.0, dt=dt, fix_mass=0, dt_flag=0, uniform_grid=1)
    o.init_field(6)
    t = 0.0
    for step in range(1, tend + 1):
        for rk in range(1, 4):
            o.set_step(step, rk)
            tt = t + dt * np.sum(RKC[:rk] + RKD[:rk])
            o.cbc_top[0, 1, 0] = -0.5 * np.exp(-2 * pi ** 2 * tt / re)
            o.cbc_bot[0, 1, 0] = 0.5 * np.exp(-2 * pi ** 2 * tt / re)
            o.nonlinear()
            o.rhs_solve()
        t = t + dt
        o.set_scalars(t, dt, 0.0)
    xs = np.arange(o.nx2)
    y, yh = o.grid("y"), o.grid("yh")
    eu = max(np.abs(o.xz_c2r(o.data1[:, :, j, 0]) + np.cos(2 * pi * xs / o.nx2)[:, None]
                    * np.sin(pi * yh[j]) * np.exp(-2 * pi ** 2 * t / re)).max() for j in range(ny + 1))
    ev = max(np.abs(o.xz_c2r(o.data1[:, :, j, 1]) - np.sin(2 * pi * xs / o.nx2)[:, None]
                    * np.cos(pi * y[j]) * np.exp(-2 * pi ** 2 * t / re)).max() for j in range(ny))
    # pressure: the reference holds the mean (kx=kz=0) pressure at zero, so
    # compare the non-mean part -cos(2 pi x)/4 exp(-4 pi^2 t/Re)
    ep = 0.0
    for j in range(1, ny):
        p = o.xz_c2r(o.data4[j, :, :])
        ex = -0.25 * np.cos(4 * pi * xs / o.nx2)[:, None] * np.exp(-4 * pi ** 2 * t / re)
        ep = max(ep, np.abs((p - p.mean()) - ex).max())
    return eu, ev, ep, o.max_divergence()


def test_which_test6_second_order(orc):
    e17 = _kat6(orc, 17)
    e33 = _kat6(orc, 33)
    e65 = _kat6(orc, 65)
    for i in (0, 1):
        assert e33[i] < 2e-4
        r1, r2 = e17[i] / e33[i], e33[i] / e65[i]
        assert 3.6 < r1 < 4.4 and 3.8 < r2 < 4.2, (i, r1, r2)
    assert e65[2] < 5e-4
    assert e65[3] < 1e-13


def test_bulk_flux_and_divergence(orc):
    o = orc.Oracle(16, 17, 16, re=2500.0, dt=0.005, fix_mass=1)
    o.init_field(10, seed=3, ampl=1e-2)
    q0 = o.bulk_flux()
    assert abs(q0 - 4.0 / 3.0) < 2e-2
    o.timestep(10)
    assert abs(o.bulk_flux() - q0) < 1e-8
    assert o.max_divergence() < 1e-13
    assert o.status() == 0
    t, dt, pg = o.scalars()
    assert abs(t - 0.05) < 1e-14
    assert abs(pg + 2.0 / 2500.0) < 2e-5


def test_cfl_abort_flag(orc):
    """check_cfl STOP 'CFL IS TOO BIG' (PFC/pass1.f90:235-244) becomes a status."""
    o = orc.Oracle(16, 17, 16, re=2500.0, dt=2.0, fix_mass=1)
    o.init_field(10, seed=3, ampl=1e-2)
    o.timestep(1)
    assert o.status() == -1
    assert o.cfl[1:17].max() >= 1.15


def test_jet_gaussian_slot_profile(orc):
    """Mode 2 with no filter: the wall value transformed back to physical
    space is the Gaussian slot minus the suction profile scaled to cancel its
    mass flux (PFC/pass2.f90:493-537)."""
    nx, nz = 32, 16
    o = orc.Oracle(nx, 9, nz)
    lx = 4 * np.pi
    j = orc.OrcJet()
    j.mode = 2
    j.jetmag[0] = 0.1
    j.xjet[0] = 0.3 * lx
    j.width, j.freq, j.frac_xbuff = 0.2 * lx, 0.5, 0.2
    o.set_jet(j)
    t = 0.3
    o.jet_profile(t, 0.1)
    v = o.small_c2r(np.asfortranarray(o.cbc_bot[:, :, 1]))
    x = np.arange(nx) * lx / nx
    d = np.abs(x - j.xjet[0])
    d = np.minimum(d, lx - d)
    slot = 0.1 * 0.5 * (1 + np.sin(2 * np.pi * 0.5 * t)) * np.exp(-(d / j.width) ** 2)
    # suction band: x in (0.8 lx, 0.9 lx), smooth rise/fall over 0.025 lx
    xs, xe = 0.8 * lx, 0.9 * lx
    xr, xf = xs + 0.025 * lx, xe - 0.025 * lx
    f = np.zeros(nx)
    for i, xc in enumerate(x):
        if xs < xc < xe:
            if xc < xr:
                x2 = (xc - xs) / (xr - xs)
                f[i] = 1 / (1 + np.exp(1 / x2 + 1 / (x2 - 1)))
            elif xc > xf:
                x2 = (xe - xc) / (xe - xf)
                f[i] = 1 / (1 + np.exp(1 / x2 + 1 / (x2 - 1)))
            else:
                f[i] = 1.0
    expect = slot - slot.mean() / f.mean() * f
    np.testing.assert_allclose(v, np.repeat(expect[:, None], nz, axis=1), atol=1e-13)
    # the top wall is not forced (jetmag 0)
    assert np.abs(o.cbc_top[:, :, 1]).max() == 0.0


def test_jet_random_walk_bounds(orc):
    o = orc.Oracle(16, 9, 16)
    j = orc.OrcJet()
    j.mode, j.jetmag[0], j.jet_diam = 1, 0.1, 0.5
    j.frac_xbuff, j.seed = 0.2, 99
    for i in range(24):
        j.jet_forcing[i] = [0.04, 0.4, 1.0, 1.0][i // 6]
        j.jet_forcing_incr[i] = 0.3
    o.set_jet(j)
    flips = 0
    prev = np.full(24, 0.3)
    for k in range(400):
        o.jet_profile(0.01 * k, 0.05)
        jf, inc = o.jet_forcing()
        assert jf[0:6].min() >= 0.01 and jf[0:6].max() <= 0.07
        assert jf[6:12].min() >= 0.1 and jf[6:12].max() <= 0.7
        flips += int(np.sum(np.sign(inc[12:]) != np.sign(prev[12:])))
        prev = inc
    # phases are not clamped: their increments flip with probability 0.05
    assert 0.02 < flips / (400 * 12) < 0.09
