"""GPU parity of the wall-forcing and small-grid routines against the oracle:
small_fft_real_to_complex / small_fft_complex_to_real (PFC/transform.f90:950-1142),
jet_profile with its random walk (PFC/pass2.f90:423-673) and time steps with
crossflow on.

Tolerances (relative L2): FP64 1e-12 per routine, 1e-10 after 20 steps;
mixed 1e-5 (the wall values and small transforms are FP32 there).
"""
import numpy as np
import pytest

from test_gpu_parity import make, rel

pytestmark = pytest.mark.gpu

TOL = {0: 1e-12, 1: 1e-5}


@pytest.mark.parametrize("prec", [0, 1])
def test_small_transforms(cf, orc, prec):
    grid, flow, o = make(cf, orc, 24, 9, 16, prec=prec)
    rng = np.random.default_rng(11)
    d = rng.standard_normal((24, 16))
    assert rel(flow.small_fft_real_to_complex(d), o.small_r2c(d)) < TOL[prec]
    c = o.small_r2c(rng.standard_normal((24, 16)))
    assert rel(flow.small_fft_complex_to_real(c), o.small_c2r(c)) < TOL[prec]
    # several planes per call
    ds = rng.standard_normal((24, 16, 5))
    cs = flow.small_fft_real_to_complex(ds)
    for p in range(5):
        assert rel(cs[:, :, p], o.small_r2c(ds[:, :, p])) < TOL[prec]
    back = flow.small_fft_complex_to_real(cs)
    assert rel(back, ds) < TOL[prec]


def jet_params(cf, orc, mode, lx, lz, seed=7):
    rng = np.random.default_rng(seed)
    jf = np.zeros(24)
    jf[0:6] = rng.uniform(0.02, 0.06, 6)      # A
    jf[6:12] = rng.uniform(0.2, 0.6, 6)       # St
    jf[12:24] = rng.uniform(0.0, 2 * np.pi, 12)
    inc = rng.uniform(-0.5, 0.5, 24)
    out = []
    for S in (cf.CfgJet, orc.OrcJet):
        j = S()
        j.mode = mode
        j.xjet[0], j.xjet[1] = 0.3 * lx, 0.55 * lx
        j.zjet[0], j.zjet[1] = 0.5 * lz, 0.25 * lz
        j.jetmag[0], j.jetmag[1] = 0.1, (0.07 if mode == 1 else 0.0)
        j.forcing[0], j.forcing[1] = 0.2, 0.1
        j.for_freq[0], j.for_freq[1] = 0.3, 0.4
        j.jet_diam = 0.6
        j.width, j.freq = 0.2 * lx, 0.5
        j.frac_xbuff = 0.2
        j.filter_jet_profile = 2
        for i in range(24):
            j.jet_forcing[i] = jf[i]
            j.jet_forcing_incr[i] = inc[i]
        j.seed = seed
        out.append(j)
    return out


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("mode", [1, 2])
def test_jet_profile(cf, orc, prec, mode):
    grid, flow, o = make(cf, orc, 32, 17, 32, prec=prec)
    jg, jo = jet_params(cf, orc, mode, grid.lx, grid.lz)
    flow.set_jet(jg)
    o.set_jet(jo)
    for k, t in enumerate([0.0, 0.37, 1.1, 2.05]):
        flow.jet_profile(t, 0.8)
        o.jet_profile(t, 0.8)
        top, bot = flow.wall_bc()
        assert rel(bot[:, :, 1], o.cbc_bot[:, :, 1]) < TOL[prec], k
        if mode == 1:
            assert rel(top[:, :, 1], o.cbc_top[:, :, 1]) < TOL[prec], k
        else:
            assert np.abs(top[:, :, 1]).max() == 0.0
        jf, inc = flow.jet_forcing()
        ojf, oinc = o.jet_forcing()
        np.testing.assert_allclose(jf, ojf, rtol=1e-14, atol=1e-15)
        np.testing.assert_array_equal(inc, oinc)
    # the walk keeps amplitude and Strouhal number in their bands
    assert jf[0:6].min() >= 0.01 and jf[0:6].max() <= 0.07
    assert jf[6:12].min() >= 0.1 and jf[6:12].max() <= 0.7
    # the suction balances the jet: no net mass flux through either wall
    assert abs(bot[0, 0, 1]) < 1e-6 * np.abs(bot[:, :, 1]).max()


def test_jet_rejects_suction_outside_box(cf, orc):
    grid, flow, o = make(cf, orc, 16, 9, 16)
    jg, _ = jet_params(cf, orc, 2, grid.lx, grid.lz)
    jg.frac_xbuff = 0.0
    with pytest.raises(cf.ChanflowError):
        flow.set_jet(jg)
    # no jet set: jet_profile is out of sequence
    with pytest.raises(cf.ChanflowError):
        flow.jet_profile(0.0, 0.1)


@pytest.mark.parametrize("prec,tol", [(0, 1e-10), (1, 1e-5)])
@pytest.mark.parametrize("mode", [1, 2])
def test_timestep_with_crossflow(cf, orc, prec, tol, mode):
    """20 steps with the jet on (jet_profile every substep from the
    device-resident time) and wall-shear feedback ctrlu = 0.5."""
    grid, flow, o = make(cf, orc, 32, 33, 32, prec=prec, ctrlu=0.5)
    jg, jo = jet_params(cf, orc, mode, grid.lx, grid.lz, seed=3)
    o.init_field(10, seed=2, ampl=1e-2)
    flow.upload_state(o.data1.copy(), o.data2.copy(), o.data4.copy())
    flow.set_scalars(*o.scalars(), d_um_dy=o.d_um_dy.copy())
    flow.set_jet(jg)
    o.set_jet(jo)
    o.timestep(20)
    flow.timestep(20)
    d1, d2, d4 = flow.download_state()
    assert rel(d1, o.data1) < tol
    top, bot = flow.wall_bc()
    assert rel(bot[:, :, 1], o.cbc_bot[:, :, 1]) < 10 * tol
    jf, _ = flow.jet_forcing()
    np.testing.assert_allclose(jf, o.jet_forcing()[0], rtol=1e-12, atol=1e-14)
    assert flow.status() == 0
