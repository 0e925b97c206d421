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


def flow_variant(tmp_path, name, **repl):
    """flow_c1.dat with the values of the named lines replaced."""
    out = []
    for ln in open(FLOW).read().splitlines():
        parts = ln.split()
        if len(parts) >= 2 and parts[1] in repl:
            ln = f"{repl[parts[1]]}\t{parts[1]}"
        out.append(ln)
    p = tmp_path / name
    p.write_text("\n".join(out) + "\n")
    return str(p)


def run_prog(args, cwd=None):
    r = subprocess.run([RUN_BIN] + args, capture_output=True, text=True, timeout=300, cwd=cwd)
    return r


@pytest.mark.skipif(not os.path.exists(RUN_BIN), reason="chanflow_run not built (build())")
def test_run_program_fringe_against_oracle(cf, orc, tmp_path):
    """An x fringe run (xfringe = 1, fix_mass = 0): the program starts from
    p_grad = 0 as define_parameters sets it (PFC/setup.f90:1384-1385) and
    its l2 norm after 10 steps equals the oracle's with the same fringe."""
    import forcing
    fp = dict(fringe_gain=4.0, xfringe=1, zfringe=0, frac_xbuff=0.2, buff_xrise=0.06, buff_xfall=0.03)
    path = flow_variant(tmp_path, "flow_fringe.dat", tend=10, l2_step=10, fix_mass=0, **fp)
    r = run_prog([path, "--outdir", str(tmp_path)])
    assert r.returncode == 0, r.stderr
    l2 = float(re.search(r"step 10\s+l2 = (\S+)", r.stdout).group(1))
    pg = float(re.search(r"P_GRAD = (\S+)", r.stdout).group(1))
    assert pg == 0.0
    run = cf.read_flow_dat(path)
    o = orc.Oracle(run.nx, run.ny, run.nz, re=run.re, dt=run.dt, stretch=run.stretch, fix_mass=0)
    grid = cf.Grid(run.nx, run.ny, run.nz, lx=run.lx, lz=run.lz, stretch=run.stretch)
    eb, et = forcing.init_buffer(o, run.nx, run.nz, grid.lx, grid.lz, grid.yh, 0.0, frac_zbuff=0.1, **fp)
    o.buffer[:, :] = eb
    o.target_inflow[:, :] = et
    o.set_scalars(0.0, run.dt, 0.0)
    o.init_field(run.which_test, seed=run.seed, ampl=run.disturb_ampl)
    o.timestep(10)
    assert abs(o.scalars()[2]) == 0.0
    ol2, _ = o.l2_norm()
    assert abs(l2 - ol2) < 1e-9 * ol2, (l2, ol2)


@pytest.mark.skipif(not os.path.exists(RUN_BIN), reason="chanflow_run not built (build())")
def test_run_program_restart_round_trip(cf, tmp_path):
    """save_vel = 1 writes newvel.out after the loop (PFC/main_mpi.f90:46);
    read_vel = 1 reads it back (read_velocity) and continues from its time:
    the restarted program ends where the same restart through the Python API
    ends, bit for bit; a missing restart file is an error."""
    a = flow_variant(tmp_path, "flow_a.dat", tend=10, l2_step=10, save_vel=1, save_step=1000)
    r = run_prog([a, "--outdir", str(tmp_path)])
    assert r.returncode == 0, r.stderr
    rst = tmp_path / "newvel.out"
    assert rst.exists()
    b = flow_variant(tmp_path, "flow_b.dat", tend=10, l2_step=10, read_vel=1)
    r = run_prog([b, "--restart", str(rst)])
    assert r.returncode == 0, r.stderr
    l2 = float(re.search(r"step 10\s+l2 = (\S+)", r.stdout).group(1))
    t_fin = float(re.search(r"FINAL TIME = (\S+)", r.stdout).group(1))
    run = cf.read_flow_dat(b)
    assert abs(t_fin - 20 * run.dt) < 1e-12
    grid = cf.Grid(run.nx, run.ny, run.nz, lx=run.lx, lz=run.lz, stretch=run.stretch)
    f = cf.ChannelFlow(grid, re=run.re, dt=run.dt, fix_mass=run.fix_mass, precision=run.precision)
    f.read_velocity(str(rst))
    f.remove_initial_divergence()
    f.compute_initial_pressure(0)
    f.timestep(10)
    fl2, _ = f.l2_norm()
    f.close()
    assert l2 == float(f"{fl2:.10e}"), (l2, fl2)
    # the default restart file savevel.out must exist in the working directory
    r = run_prog([b], cwd=str(tmp_path))
    assert r.returncode != 0 and "savevel.out" in r.stderr
