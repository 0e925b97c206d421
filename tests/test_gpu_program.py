"""chanflow_run, the reference's DNS program (PFC/main_mpi.f90) over the C
ABI without Python: the configuration C1 flow.dat for 20 steps must end at
t = 20 dt with the same l2 norm as the same run through the Python API."""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN_BIN = os.path.join(ROOT, "3d-navier-stokes-thesis-paper_b200", "lib", "chanflow_run")
FLOW = os.path.join(ROOT, "tests", "golden", "flow_c1.dat")


@pytest.mark.skipif(not os.path.exists(RUN_BIN), reason="chanflow_run not built (build())")
def test_run_program_matches_python_api(cf, tmp_path):
    r = subprocess.run([RUN_BIN, FLOW, "--steps", "20", "--outdir", str(tmp_path)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    m = re.search(r"step 20\s+l2 = (\S+)\s+drag = (\S+)", r.stdout)
    fin = re.search(r"FINAL TIME = (\S+)", r.stdout)
    assert m and fin, r.stdout
    run = cf.read_flow_dat(FLOW)
    grid = cf.Grid(run.nx, run.ny, run.nz, lx=run.lx, lz=run.lz, stretch=run.stretch)
    f = cf.ChannelFlow(grid, re=run.re, dt=run.dt, fix_mass=run.fix_mass, dt_flag=run.dt_flag,
                       precision=run.precision)
    f.define_initial_field(run.which_test, seed=run.seed, ampl=run.disturb_ampl)
    f.timestep(20)
    l2, drag = f.l2_norm()
    assert abs(float(m.group(1)) - l2) <= 1e-9 * abs(l2)
    assert abs(float(fin.group(1)) - 20 * run.dt) < 1e-12
    f.close()
