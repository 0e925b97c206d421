"""GPU side of the output routines: the restart file written from the device
state (save_velocity), read back into a context (read_velocity), written in
the background while steps continue, and the VTK velocity snapshot of
output_hdf_dfsd (PFC/read_write.f90:296-500) against the oracle's small
inverse transforms of the same data1.

Tolerances: the restart data are the device state, bit for bit; the VTK
values are float32 (relative 1e-6 of the field's maximum in FP64, 1e-5 mixed).
"""
import numpy as np
import pytest

from fortran_records import parse_restart, parse_vtk
from test_gpu_parity import make

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1])
def test_save_and_read_velocity(cf, orc, prec, tmp_path):
    grid, flow, o = make(cf, orc, 32, 17, 16, prec=prec)
    flow.define_initial_field(10, seed=4, ampl=1e-2)
    flow.timestep(3)
    d1, _, _ = flow.download_state()
    sc = flow.scalars()
    p = tmp_path / "newvel.out"
    flow.save_velocity(p, wait=True)
    head, got, tail = parse_restart(p, 32, 17, 16)
    np.testing.assert_array_equal(got, d1)
    assert head["t_total"] == sc["t_total"] and head["dt"] == sc["dt"]
    assert (head["nx"], head["ny"], head["nz"]) == (32, 17, 16)
    np.testing.assert_array_equal(tail, [0, 0])
    # into a fresh context: data1 and t_total come back
    _, flow2, _ = make(cf, orc, 32, 17, 16, prec=prec)
    flow2.read_velocity(p)
    e1, _, _ = flow2.download_state()
    np.testing.assert_array_equal(e1, d1)
    assert flow2.scalars()["t_total"] == sc["t_total"]
    # a different grid is refused with the reference's message
    _, flow3, _ = make(cf, orc, 32, 17, 32, prec=prec)
    with pytest.raises(cf.ChanflowError, match="NZ HAS BEEN CHANGED"):
        flow3.read_velocity(p)


def test_save_is_a_snapshot_while_steps_continue(cf, orc, tmp_path):
    grid, flow, o = make(cf, orc, 32, 17, 16)
    flow.define_initial_field(10, seed=5, ampl=1e-2)
    flow.timestep(2)
    d1, _, _ = flow.download_state()
    t = flow.scalars()["t_total"]
    p = tmp_path / "snap.out"
    flow.save_velocity(p)
    flow.timestep(4)          # issued while the copy and the write may be in flight
    flow.wait_io()
    head, got, _ = parse_restart(p, 32, 17, 16)
    np.testing.assert_array_equal(got, d1)
    assert head["t_total"] == t
    assert flow.scalars()["t_total"] > t


@pytest.mark.parametrize("prec,tol", [(0, 1e-6), (1, 1e-5)])
def test_vtk_snapshot(cf, orc, prec, tol, tmp_path):
    nx, ny, nz = 32, 17, 16
    grid, flow, o = make(cf, orc, nx, ny, nz, prec=prec)
    flow.define_initial_field(10, seed=6, ampl=5e-2)
    flow.timestep(2)
    d1, _, _ = flow.download_state()
    p = tmp_path / "t_001.vtk"
    flow.write_vtk(p, wait=True)
    v = parse_vtk(p)
    assert v["lines"][:4] == ["# vtk DataFile Version 2.0",
                              "(This is header line) vtk rectilinear grid with binary data",
                              "BINARY", "DATASET RECTILINEAR_GRID"]
    assert v["lines"][4] == "DIMENSIONS " + "%5d%5d%5d" % (nx, ny + 1, nz) + " " * 4
    assert v["lines"][5] == "X_COORDINATES  32 float" + " " * 7
    assert v["lines"][-1] == "VECTORS flowvec float"
    np.testing.assert_array_equal(v["x"], (grid.lx * np.arange(nx) / nx).astype(np.float32))
    np.testing.assert_array_equal(v["y"], grid.yh.astype(np.float32))
    np.testing.assert_array_equal(v["z"], (grid.lz * np.arange(nz) / nz).astype(np.float32))
    # expected: u, w at yh; v averaged onto yh (first/last plane copied)
    exp = np.zeros((nx, ny + 1, nz, 3))
    for pl in range(ny + 1):
        for c in range(3):
            if c != 1:
                cu = d1[:, :, pl, c]
            elif pl == 0:
                cu = d1[:, :, 0, 1]
            elif pl == ny:
                cu = d1[:, :, ny - 1, 1]
            else:
                cu = 0.5 * (d1[:, :, pl - 1, 1] + d1[:, :, pl, 1])
            exp[:, pl, :, c] = o.small_c2r(np.asfortranarray(cu))
    err = np.abs(v["vel"] - exp).max() / np.abs(exp).max()
    assert err < tol, err
