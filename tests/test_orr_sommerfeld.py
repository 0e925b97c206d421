"""The Orr-Sommerfeld known-answer test (the reference's which_test 2,
PFC/init_vel.f90:95-114) on the CPU: the eigenmode generator, the efn.m
reader and interpolation (READ_EIGENFUNCTION, PFC/init_vel.f90:540-640), and
the oracle's growth of the mode.

Pins:
- the least-stable mode of plane Poiseuille flow at Re 7500, alpha 1 has the
  phase speed the reference hard-codes, 0.24989154 (PFC/setup.f90:1387), and
  the growth c_i = 0.00223497 of the published eigenvalue
  c = 0.24989154 + 0.00223497 i;
- the oracle DNS started from that mode (laminar + 1e-4 mode, fix_mass 0,
  the reference's stretch 2.75, dt = 2 (2 pi / 0.24989154) / tend as
  PFC/setup.f90:1386-1388 sets it) grows the mode's energy (ke of
  PFC/pass2.f90:113-117) at 2 alpha c_i to the accuracy of its second-order
  y differences: within 0.6 % at ny = 193 and, Richardson-extrapolated from
  ny = 97 and 193, within 0.1 % (measured 0.51 % and 0.04 %; the DNS mean
  also drifts slowly, by ~2e-5 over the run, from 1 - yh^2 toward the
  discrete steady profile, which moves the rate by a fraction of that
  error).
"""
import importlib

import numpy as np
import pytest

C_RE7500 = 0.24989154 + 0.00223497j


@pytest.fixture(scope="module")
def osm(cf):
    return importlib.import_module("chanflow_b200.orr_sommerfeld")


def test_least_stable_mode_matches_reference_phase_speed(osm):
    c, u, v, x = osm.least_stable(7500.0, 1.0)
    assert abs(c.real - osm.PHASE_SPEED_RE7500) < 5e-9, c
    assert abs(c.imag - C_RE7500.imag) < 1e-8, c   # the published digits
    # resolved: a finer collocation gives the same eigenvalue
    c2 = osm.least_stable(7500.0, 1.0, n=80)[0]
    assert abs(c2 - c) < 1e-8
    # boundary conditions of the eigenfunction: v = v' = 0 (u = 0) at the walls
    assert abs(v[0]) < 1e-12 and abs(v[-1]) < 1e-12
    assert abs(u[0]) < 1e-8 and abs(u[-1]) < 1e-8
    assert abs(np.abs(u).max() - 1.0) < 1e-14


def test_efn_file_round_trip_and_interpolation(cf, osm, tmp_path):
    """write_efn -> cfh_read_efn -> cfh_interp_eigenfunction equals the
    degree-64 Chebyshev interpolant of the collocation values evaluated with
    numpy on the solver's yh (u) and y (v) points."""
    path = tmp_path / "efn.m"
    osm.write_efn(str(path))
    c, u, v, x = osm.least_stable()
    lines = path.read_text().split()
    assert len(lines) == 260
    # Fortran D exponents are read too
    path_d = tmp_path / "efn_d.m"
    path_d.write_text("\n".join(s.replace("e", "D") for s in lines) + "\n")
    grid = cf.Grid(16, 97, 8, lx=2 * np.pi, lz=2 * np.pi, stretch=2.75)
    for p in (path, path_d):
        d1 = cf.initial_field(grid, 2, ampl=1.0, efn=str(p))
        ch = np.polynomial.chebyshev.Chebyshev
        ui = ch.fit(x, u.real, 64)(grid.yh) + 1j * ch.fit(x, u.imag, 64)(grid.yh)
        vi = ch.fit(x, v.real, 64)(grid.y) + 1j * ch.fit(x, v.imag, 64)(grid.y)
        col = d1[0, 1]
        assert np.abs(col[1:97, 0] - ui[1:97]).max() < 1e-10
        assert col[0, 0] == 0 and col[97, 0] == 0
        assert np.abs(col[:97, 1] - vi).max() < 1e-10
        assert np.abs(d1[0, 0, :, 0] - (1 - grid.yh ** 2)).max() < 1e-15
    with pytest.raises(cf.ChanflowError):
        short = tmp_path / "short.m"
        short.write_text("1.0\n2.0\n")
        cf.initial_field(grid, 2, efn=str(short))


def os_growth_oracle(cf, orc, osm, ny, tend=500, ampl=1e-4):
    nx, nz, stretch = 16, 8, 2.75
    c, u, v, _ = osm.least_stable()
    grid = cf.Grid(nx, ny, nz, lx=2 * np.pi, lz=2 * np.pi, stretch=stretch)
    d1 = cf.initial_field(grid, 2, ampl=ampl, efn=osm.efn_columns(u, v))
    dt = 2 * (2 * np.pi / 0.24989154) / tend
    o = orc.Oracle(nx, ny, nz, re=7500.0, dt=dt, stretch=stretch, fix_mass=0, lx=2 * np.pi, lz=2 * np.pi)
    o.init_from_velocity(d1)
    dyh = o.grid("dyh")
    e, t = [], []
    for _ in range(tend // 10):
        o.timestep(10)
        e.append(osm.mode_energy(o.data1, dyh))
        t.append(o.scalars()[0])
    o.close()
    h = len(e) // 2
    return 0.5 * np.log(e[-1] / e[h]) / (t[-1] - t[h])


def test_oracle_orr_sommerfeld_growth(cf, orc, osm):
    g97 = os_growth_oracle(cf, orc, osm, 97)
    g193 = os_growth_oracle(cf, orc, osm, 193)
    ci = C_RE7500.imag
    assert abs(g193 - ci) < 0.006 * ci, g193
    # second order in the y spacing: the error falls ~4x from 97 to 193 planes
    assert 3.0 < (g97 - ci) / (g193 - ci) < 5.5, (g97, g193)
    assert abs(g193 + (g193 - g97) / 3 - ci) < 0.001 * ci, (g97, g193)
