"""GPU parity of the fringe region: init_buffer (PFC/init_jet_buffer.f90:
358-483) computed on the device against the oracle's numpy restatement
(oracle/forcing.py), and time steps with the fringe term buffer*(u - target)
of the nonlinear step (PFC/pass1.f90) against the oracle given the same
buffer.

Tolerances: buffer FP64 1e-12 (relative L2), mixed 1e-6; 10 steps FP64 1e-10,
mixed 1e-5."""
import numpy as np
import pytest

import forcing
from test_gpu_parity import make, rel

pytestmark = pytest.mark.gpu

PARAMS = dict(fringe_gain=4.0, xfringe=1, zfringe=1, frac_xbuff=0.2, buff_xrise=0.06, buff_xfall=0.03,
              frac_zbuff=0.15)


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-6)])
def test_init_buffer(cf, orc, prec, tol):
    grid, flow, o = make(cf, orc, 32, 17, 16, prec=prec)
    flow.init_buffer(**PARAMS)
    b, t = flow.buffer()
    eb, et = forcing.init_buffer(o, 32, 16, grid.lx, grid.lz, grid.yh, 0.0, **PARAMS)
    assert rel(b, eb) < tol
    np.testing.assert_allclose(t, et, rtol=1e-15, atol=1e-15)


@pytest.mark.parametrize("prec,tol", [(0, 1e-10), (1, 1e-5)])
def test_steps_with_fringe(cf, orc, prec, tol):
    grid, flow, o = make(cf, orc, 32, 33, 16, prec=prec)
    flow.init_buffer(**PARAMS)
    eb, et = forcing.init_buffer(o, 32, 16, grid.lx, grid.lz, grid.yh, 0.0, **PARAMS)
    o.buffer[:, :] = eb
    o.target_inflow[:, :] = et
    o.init_field(10, seed=12, ampl=1e-2)
    flow.upload_state(o.data1.copy(), o.data2.copy(), o.data4.copy())
    flow.set_scalars(*o.scalars(), d_um_dy=o.d_um_dy.copy())
    o.timestep(10)
    flow.timestep(10)
    d1, _, _ = flow.download_state()
    assert rel(d1, o.data1) < tol
    assert flow.status() == 0
