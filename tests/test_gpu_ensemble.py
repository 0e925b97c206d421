"""Ensembles (configuration C5) on one GPU: members of different grids,
Reynolds numbers, noise seeds, jet forcing and precisions, tuned once per
grid and advanced by one CUDA graph launch per step, must reproduce each
member run alone with the default tiles bit for bit (the tiles change the
schedule, never the arithmetic) -- in both step layouts: one graph branch
per member, and batched (one launch per kernel for each class of equal
grids, every member's arguments from a table in device memory)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MEMBERS = [  # (nx, ny, nz, Re, seed, jet, precision: 1 mixed, 0 FP64)
    (48, 49, 48, 2000.0, 1001, True, 1),
    (48, 49, 48, 2600.0, 1002, False, 1),
    (64, 65, 64, 2300.0, 1003, True, 1),
    (96, 97, 96, 2900.0, 1004, False, 1),
    (48, 49, 48, 2400.0, 1005, True, 0),
]


def member(cf, nx, ny, nz, re, seed, jet, prec=1):
    grid = cf.Grid(nx, ny, nz, stretch=1.5)
    f = cf.ChannelFlow(grid, re=re, dt=0.0025, precision=prec)
    f.define_initial_field(10, seed=seed, ampl=1e-2)
    if jet:
        j = cf.CfgJet()
        j.mode = 2
        j.xjet[0], j.zjet[0] = 0.3 * grid.lx, 0.5 * grid.lz
        j.jetmag[0] = 0.1
        j.width, j.freq = 0.2, 0.5
        j.frac_xbuff = 0.2
        j.seed = seed
        f.set_jet(j)
    return f


def test_ensemble_graph_matches_members_alone(cf):
    steps = 6
    alone = [member(cf, *m) for m in MEMBERS]
    for f in alone:
        f.timestep(steps)
    ref = [f.download_state() for f in alone]
    ref_launch = [f.launch_count() for f in alone]

    ens_members = [member(cf, *m) for m in MEMBERS]
    ens = cf.Ensemble(ens_members, autotune=True)
    # an FP64 member: the batched layout is not available
    assert not ens.batched
    with pytest.raises(cf.ChanflowError):
        cf.Ensemble([member(cf, *m) for m in MEMBERS[-2:]], autotune=False, batched=True)
    ens.timestep(steps)
    ens.synchronize()
    for k, f in enumerate(ens_members):
        got = f.download_state()
        for a, b in zip(ref[k], got):
            np.testing.assert_array_equal(a, b)
        assert f.status() == 0
        assert f.launch_count() == ref_launch[k]
        assert f.scalars()["t_total"] == alone[k].scalars()["t_total"]
    ens.close()


def test_autotune_restores_state(cf):
    f = member(cf, 64, 65, 64, 2300.0, 7, True, 1)
    g = member(cf, 64, 65, 64, 2300.0, 7, True, 1)
    tiles = f.autotune(2)
    assert len(tiles) == 4
    f.timestep(3)
    g.timestep(3)
    for a, b in zip(f.download_state(), g.download_state()):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(f.jet_forcing()[0], g.jet_forcing()[0])


# mixed precision only: three classes (48, 64 and 96 points), jets and plain
# members in the same class, different Reynolds numbers within a class
BATCH_MEMBERS = [
    (48, 49, 48, 2000.0, 1001, True, 1),
    (48, 49, 48, 2600.0, 1002, False, 1),
    (48, 49, 48, 2100.0, 1006, True, 1),
    (64, 65, 64, 2300.0, 1003, True, 1),
    (64, 65, 64, 2800.0, 1007, False, 1),
    (96, 97, 96, 2900.0, 1004, False, 1),
    (96, 97, 96, 2200.0, 1008, True, 1),
]


@pytest.mark.parametrize("autotune", [False, True])
def test_batched_ensemble_matches_members_alone(cf, autotune):
    steps = 6
    alone = [member(cf, *m) for m in BATCH_MEMBERS]
    for f in alone:
        f.timestep(steps)
    ref = [f.download_state() for f in alone]

    ens_members = [member(cf, *m) for m in BATCH_MEMBERS]
    ens = cf.Ensemble(ens_members, autotune=autotune)
    assert ens.batched
    ens.timestep(steps)
    ens.synchronize()
    for k, f in enumerate(ens_members):
        got = f.download_state()
        for a, b in zip(ref[k], got):
            np.testing.assert_array_equal(a, b)
        assert f.status() == 0
        sa, sb = f.scalars(), alone[k].scalars()
        for key in ("t_total", "dt", "p_grad", "cfl_max"):
            assert sa[key] == sb[key], key
        np.testing.assert_array_equal(sa["d_um_dy"], sb["d_um_dy"])
        if BATCH_MEMBERS[k][5]:
            np.testing.assert_array_equal(f.jet_forcing()[0], alone[k].jet_forcing()[0])
    # the layout switch: the next steps in branches continue bit for bit
    ens.L.cfg_ensemble_set_batched(ens.h, 0)
    assert not ens.batched
    ens.timestep(2)
    ens.synchronize()
    for f in alone:
        f.timestep(2)
    for k, f in enumerate(ens_members):
        for a, b in zip(alone[k].download_state(), f.download_state()):
            np.testing.assert_array_equal(a, b)
    ens.close()
