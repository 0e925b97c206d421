"""Multi-rank runs (cfg_group) on one GPU: P ranks with the reference's slab
decomposition (distribute_data, PFC/setup.f90:298-437) advance one field
and must reproduce the single-context run bit for bit -- every wavenumber,
row and plane goes through the same kernels with the same arithmetic; only
the storage is split and the two transposes go through the scatter stores.
Ranks on one GPU share it through their own streams and event barriers (no
kernel waits on another), so this covers the index arithmetic of the slabs,
the scatter tables, the CFL fold across ranks and the mean mode on rank 0.
"""
import numpy as np
import pytest

from conftest import whole_velocity_transforms

pytestmark = pytest.mark.gpu


def prepared(cf, grid, prec, dt_flag, seed):
    """A divergence-free state with its initial pressure, made on a single
    context (which_test 10: laminar profile plus seeded noise)."""
    d1 = cf.initial_field(grid, 10, seed=seed, ampl=5e-2)
    f = cf.ChannelFlow(grid, re=2500.0, dt=0.004, precision=prec, dt_flag=dt_flag)
    f.upload_state(d1, d1.transpose(2, 3, 0, 1).copy(), None)
    f.remove_initial_divergence()
    f.compute_initial_pressure()
    st = f.download_state()
    sc = f.scalars()
    f.close()
    return st, sc


@pytest.mark.parametrize("prec,nranks,dt_flag,fringe", [
    (0, 2, 0, False), (0, 3, 1, True), (1, 2, 1, False), (1, 6, 0, True), (1, 1, 0, False)])
def test_group_matches_single_context(cf, prec, nranks, dt_flag, fringe):
    grid = cf.Grid(32, 33, 32, stretch=1.5)
    if fringe:
        x = np.arange(grid.nx2)[:, None] / grid.nx2
        z = np.arange(grid.nz2)[None, :] / grid.nz2
        grid.buffer = np.asfortranarray(0.5 * np.exp(-((x - 0.9) / 0.05) ** 2) * (1 + 0.3 * np.cos(2 * np.pi * z)))
    st, sc = prepared(cf, grid, prec, dt_flag, seed=7 + nranks)
    # ranks of a multi-rank run keep the whole velocity in the FP32 transforms
    # (the mean column lives on rank 0 only): so does the reference context
    with whole_velocity_transforms(nranks > 1):
        one = cf.ChannelFlow(grid, re=2500.0, dt=0.004, precision=prec, dt_flag=dt_flag)
    grp = cf.Group(grid, nranks, re=2500.0, dt=0.004, precision=prec, dt_flag=dt_flag)
    for f in (one, grp):
        f.upload_state(*st)
        f.set_scalars(sc["t_total"], sc["dt"], sc["p_grad"], sc["d_um_dy"])
    one.timestep(4)
    grp.timestep(4)
    grp.synchronize()
    a, b = one.download_state(), grp.download_state()
    for x, y in zip(a, b):
        assert x.shape == y.shape
        np.testing.assert_array_equal(x, y)
    s1 = one.scalars()
    for r in range(nranks):
        s2 = grp.scalars(r)
        assert s2["dt"] == s1["dt"] and s2["t_total"] == s1["t_total"]
    s0 = grp.scalars(0)
    assert s0["p_grad"] == s1["p_grad"]
    np.testing.assert_array_equal(s0["d_um_dy"], s1["d_um_dy"])
    if dt_flag:
        assert s1["dt"] != 0.004   # the CFL fold did change dt
    assert one.status() == 0 and grp.status() == [0] * nranks
    # the partition is the reference's
    part = cf.partition(grid.nx, grid.nz, grid.nz2, nranks)
    assert [f.nxh for f in grp.ranks] == list(part["nx_proc"])
    grp.close()
    one.close()


def test_group_rank_refuses_whole_plane_calls(cf):
    grid = cf.Grid(32, 33, 32, stretch=1.5)
    grp = cf.Group(grid, 2, precision=1)
    with pytest.raises(cf.ChanflowError, match="multi-rank"):
        grp.ranks[1].nonlinear(1, 1)
    with pytest.raises(cf.ChanflowError, match="multi-rank"):
        grp.ranks[0].l2_norm()
    grp.close()
