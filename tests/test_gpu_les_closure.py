"""Configuration C4's pipeline end to end at a small size: DNS 96x49x96 at Re
3000 from the turbulent-profile field with strong seeded noise, 6 snapshots
box-filtered by 3 onto the LES grid 32x17x32, the closure trained on five of
them with the tensor-core kernels, judged on the sixth, and LES runs with
each closure.

What the trained network gains over the method without it (the eddy
viscosity): a priori, on the held-out snapshot, its deviatoric stresses are
closer to the filtered DNS's than the eddy viscosity's, and its tau_12
correlates better.  The LES with the learned closure runs stably with its
fallback active where needed.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_c4_pipeline_small(cf):
    lc = importlib.import_module("chanflow_b200.les_closure")
    out = lc.run_c4(nx=96, ny=49, nz=96, factor=3, re=3000.0, ampl=0.5, spinup=6.0, nsnap=6, snap_dt=0.5,
                    train_iters=800, batch=2048, lr=3e-3, les_spin=3.0, les_avg=3.0)
    print({k: v for k, v in out.items() if k != "filtered_dns"})
    assert out["dns"]["status"] == 0 and out["dns"]["status_end"] == 0
    ap = out["a_priori"]
    assert ap["nn_deviatoric_rel_err"] < ap["ev_deviatoric_rel_err"], ap
    assert ap["nn_corr_12"] > ap["ev_corr_12"], ap
    losses = [l for _, l in out["training"]["losses"]]
    assert losses[-1] < losses[0]
    for name, r in out["les"].items():
        assert r["status"] == 0, (name, r)
        assert np.isfinite(r["mean_profile_rel_l2"]), (name, r)
    assert 0.0 <= out["les"]["learned"]["fallback_fraction"] < 1.0
