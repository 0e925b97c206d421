"""GPU parity of the post-processing kernels against the oracle's numpy
restatement (oracle/postproc.py): the velocity-gradient tensor, vorticity,
Q-criterion and discriminant (ParaView-Code/DiscriminantFilter.cpd:17) on the
snapshot grid, and the per-plane moments of PFC/stats.f90:423-456.

Tolerances: FP64 -- moments 1e-9 relative per column (absolute 1e-12 where a
column vanishes), VTK fields at float32 resolution (1e-6 of each field's
maximum); mixed -- 1e-4 and 1e-4."""
import numpy as np
import pytest

import postproc
from fortran_records import parse_vtk
from test_gpu_parity import make

pytestmark = pytest.mark.gpu


def reference(o, flow, grid):
    d1, _, _ = flow.download_state()
    u, A = postproc.velocity_and_gradient(o, d1, grid.yh, o.grid("kx"), o.grid("kz"))
    vort, Q, D = postproc.invariants(A)
    return u, vort, Q, D


@pytest.mark.parametrize("prec,tol", [(0, 1e-9), (1, 1e-4)])
def test_plane_statistics(cf, orc, prec, tol):
    grid, flow, o = make(cf, orc, 32, 17, 16, prec=prec)
    flow.define_initial_field(10, seed=8, ampl=5e-2)
    flow.timestep(3)
    u, vort, Q, D = reference(o, flow, grid)
    exp = postproc.plane_moments(u, vort)
    got = flow.plane_statistics()
    for k in range(27):
        scale = np.abs(exp[:, k]).max()
        err = np.abs(got[:, k] - exp[:, k]).max()
        assert err <= tol * scale + 1e-12 * (1 if prec == 0 else 1e4), (k, err, scale)


@pytest.mark.parametrize("prec,tol", [(0, 1e-6), (1, 1e-4)])
def test_vtk_derived(cf, orc, prec, tol, tmp_path):
    grid, flow, o = make(cf, orc, 32, 17, 16, prec=prec)
    flow.define_initial_field(10, seed=9, ampl=5e-2)
    flow.timestep(2)
    u, vort, Q, D = reference(o, flow, grid)
    p = tmp_path / "t_002.vtk"
    flow.write_vtk_derived(p, wait=True)
    v = parse_vtk(p)
    for name, exp in (("vel", u), ("vorticity", vort), ("Q", Q), ("D", D)):
        err = np.abs(v[name] - exp).max() / np.abs(exp).max()
        assert err < tol, (name, err)
