"""Configuration C2 at its full size on the GPU: DNS at Re 2800 on
128x129x128, seeded 1e-2 noise on the laminar profile, the Gaussian wall-jet
slot (width 0.2, peak 0.1 U_c, frequency 0.5) and the linear wall-shear
feedback law (ctrlu = 0.5), dt 0.0025.  The FP64 path is pinned to the
oracle routine by routine and over 100 steps at smaller sizes
(test_gpu_parity.py, test_gpu_forcing.py); here the mixed path must stay
within 1e-5 relative L2 of the FP64 path over 100 steps at the full size,
its perturbation (all but the mean column) within 1e-5 and 1e-4 of that
perturbation's change over the run,
both paths must agree on the bulk flux and p_grad, and the divergence must
stay at round-off."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def c2_flow(cf, grid, prec):
    f = cf.ChannelFlow(grid, re=2800.0, dt=0.0025, fix_mass=1, ctrlu=0.5, ctrlw=0.0, precision=prec)
    f.define_initial_field(10, seed=2, ampl=1e-2)
    j = cf.CfgJet()
    j.mode = 2
    j.xjet[0], j.zjet[0] = 0.3 * grid.lx, 0.5 * grid.lz
    j.jetmag[0] = 0.1
    j.width, j.freq = 0.2, 0.5
    j.frac_xbuff = 0.2
    j.seed = 2
    f.set_jet(j)
    return f


def test_config_c2_mixed_matches_fp64_100_steps(cf):
    grid = cf.Grid(128, 129, 128, stretch=1.5)
    a = c2_flow(cf, grid, cf.FP64)
    b = c2_flow(cf, grid, cf.MIXED)
    d0 = a.download_state()[0]
    a.timestep(100)
    b.timestep(100)
    da, db = a.download_state()[0], b.download_state()[0]
    err = np.linalg.norm(db - da) / np.linalg.norm(da)
    # the perturbation (all Fourier columns but the mean) on its own, and
    # its change over the run: measured on a B200, err 2.4e-8, perturbation
    # error 1.6e-6, perturbation change 0.98
    pa, pb, p0 = da.copy(), db.copy(), d0.copy()
    for p in (pa, pb, p0):
        p[0, 0] = 0
    perr = np.linalg.norm(pb - pa) / np.linalg.norm(pa)
    chg = np.linalg.norm(pa - p0) / np.linalg.norm(pa)
    assert err < 1e-5, (err, perr, chg)
    assert chg > 0.1, chg                  # the run moved the perturbation
    assert perr < 1e-5 and perr < 1e-4 * chg, (perr, chg)
    assert a.status() == 0 and b.status() == 0
    # with wall slip from the feedback law the flux is held only up to the
    # wall terms (the reference's compute_p_grad); both paths agree on it
    qa, diva = a.diagnostics()
    qb, divb = b.diagnostics()
    assert abs(qa - 4.0 / 3.0) < 1e-3 and abs(qb - qa) < 1e-6 * qa, (qa, qb)
    assert diva < 1e-8 and divb < 1e-6, (diva, divb)
    sa, sb = a.scalars(), b.scalars()
    assert abs(sa["t_total"] - 0.25) < 1e-12 and abs(sb["t_total"] - 0.25) < 1e-12
    assert abs(sa["p_grad"] - sb["p_grad"]) < 1e-5 * abs(sa["p_grad"])


def test_largest_grid_mixed_matches_fp64(cf):
    """The largest supported transform length (nx2 = nz2 = 576, the
    384x193x384 DNS grid of configuration C4) in both precisions: 4 steps
    from the seeded initial field agree to 1e-5 relative L2, and the
    divergence stays at round-off and the bulk flux is held."""
    grid = cf.Grid(384, 193, 384, stretch=1.5)
    runs = []
    for prec in (cf.FP64, cf.MIXED):
        f = cf.ChannelFlow(grid, re=2500.0, dt=0.0025, fix_mass=1, precision=prec)
        f.define_initial_field(10, seed=4, ampl=1e-2)
        q0, _ = f.diagnostics()
        f.timestep(4)
        runs.append(f.download_state()[0])
        q, div = f.diagnostics()
        # constant flux: the discrete flux of the initial field is held (it
        # is 4/3 up to the quadrature of the stretched grid)
        assert f.status() == 0 and abs(q - q0) < 1e-7 and div < 1e-6, (q0, q, div)
        f.close()
    a, b = runs
    assert np.linalg.norm(b - a) / np.linalg.norm(a) < 1e-5
