"""The alternative kernel paths a context can be switched to at creation
(environment switches read by cfg_create; the defaults are the fast paths):
CHANFLOW_GENERIC_FFT (shared-memory Stockham FFTs in every transform),
CHANFLOW_FUSED_XFLUX (inverse x, fluxes and forward x in one kernel),
CHANFLOW_FLUX_ZR=2 and =8 (two or, FP32 only, eight z rows per flux
block), CHANFLOW_XINV_ROWS=24 and =8 (z rows per inverse-x block; 24 FP32
only), CHANFLOW_RHS_V1 (the first
per-wavenumber solver) and CHANFLOW_RHS2_LANES=32 and =16 (one and two
wavenumbers per warp; the default at this grid's 34 rows in FP32 is 8
lanes, four wavenumbers per warp).
Each must give the default path's state after three steps to 1e-12 in FP64
and 1e-5 in mixed precision (different summation orders).  The alternative
paths keep the whole velocity in their FP32 transforms, so in mixed precision
the default they are compared with does too (CHANFLOW_NO_MEAN_SPLIT=1); the
mean split itself is checked against the oracle at the benchmark's size
(test_gpu_metric_config.py)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SWITCHES = [("CHANFLOW_GENERIC_FFT", "1"), ("CHANFLOW_FUSED_XFLUX", "1"), ("CHANFLOW_FLUX_ZR", "2"),
            ("CHANFLOW_FLUX_ZR", "8"), ("CHANFLOW_XINV_ROWS", "24"), ("CHANFLOW_XINV_ROWS", "8"),
            ("CHANFLOW_RHS_V1", "1"), ("CHANFLOW_RHS2_LANES", "32"), ("CHANFLOW_RHS2_LANES", "16")]


def run(cf, grid, env, prec):
    keys = [k for k, _ in SWITCHES] + ["CHANFLOW_NO_MEAN_SPLIT"]
    saved = {k: os.environ.get(k) for k in keys}
    try:
        for k in keys:
            os.environ.pop(k, None)
        os.environ.update(env)
        f = cf.ChannelFlow(grid, re=2500.0, dt=0.004, precision=prec, dt_flag=1)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    f.define_initial_field(10, seed=13, ampl=5e-2)
    f.timestep(3)
    out = f.download_state()
    assert f.status() == 0
    f.close()
    return out


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-5)])
@pytest.mark.parametrize("name,value", SWITCHES)
def test_switch_matches_default_path(cf, name, value, prec, tol):
    grid = cf.Grid(32, 33, 32, stretch=1.5)
    base = {"CHANFLOW_NO_MEAN_SPLIT": "1"} if prec == 1 else {}
    ref = run(cf, grid, base, prec)
    got = run(cf, grid, dict(base, **{name: value}), prec)
    for a, b in zip(ref, got):
        assert np.linalg.norm(b - a) / np.linalg.norm(a) < tol
