"""Host side of the restart file (read_write::save_velocity / read_velocity,
PFC/read_write.f90:21-292): the record layout, the round trip and
read_velocity's consistency checks, on the CPU."""
import numpy as np
import pytest

from fortran_records import parse_restart


def field(nx, ny, nz, seed=0):
    rng = np.random.default_rng(seed)
    sh = (nz, nx // 2 + 1, ny + 1, 3)
    return np.asfortranarray(rng.standard_normal(sh) + 1j * rng.standard_normal(sh))


def test_restart_layout_and_round_trip(cf, tmp_path):
    nx, ny, nz = 8, 5, 6
    d1 = field(nx, ny, nz)
    p = tmp_path / "newvel.out"
    cf.save_velocity_file(p, d1, 4 * np.pi, 2 * np.pi, 2500.0, 0.005, 1.25)
    head, got, tail = parse_restart(p, nx, ny, nz)
    assert (head["nx"], head["ny"], head["nz"]) == (nx, ny, nz)
    assert head["lx"] == 4 * np.pi and head["lz"] == 2 * np.pi
    assert head["re"] == 2500.0 and head["dt"] == 0.005 and head["t_total"] == 1.25
    np.testing.assert_array_equal(got, d1)
    np.testing.assert_array_equal(tail, [0, 0])
    back, dt, t = cf.read_velocity_file(p, nx, ny, nz, 4 * np.pi, 2 * np.pi, 2800.0)
    np.testing.assert_array_equal(back, d1)
    assert dt == 0.005 and t == 1.25


@pytest.mark.parametrize("what", ["nx", "ny", "nz", "lx", "lz"])
def test_read_velocity_rejects_changed_parameters(cf, tmp_path, what):
    nx, ny, nz = 8, 5, 6
    p = tmp_path / "savevel.out"
    cf.save_velocity_file(p, field(nx, ny, nz), 4 * np.pi, 2 * np.pi, 2500.0, 0.005, 0.0)
    args = dict(nx=nx, ny=ny, nz=nz, lx=4 * np.pi, lz=2 * np.pi, re=2500.0)
    args[what] = args[what] * 2 if what in ("nx", "ny", "nz") else args[what] * (1 + 1e-12)
    with pytest.raises(cf.ChanflowError, match=what.upper() + " HAS BEEN CHANGED"):
        cf.read_velocity_file(p, **args)


def test_read_velocity_rejects_truncated_file(cf, tmp_path):
    nx, ny, nz = 8, 5, 6
    p = tmp_path / "savevel.out"
    cf.save_velocity_file(p, field(nx, ny, nz), 1.0, 1.0, 100.0, 0.01, 0.0)
    b = p.read_bytes()
    p.write_bytes(b[:len(b) // 2])
    with pytest.raises(cf.ChanflowError):
        cf.read_velocity_file(p, nx, ny, nz, 1.0, 1.0, 100.0)
