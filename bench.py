"""Benchmark of the channel-flow DNS time step on B200.

Workload: one time step (3 RK3/Crank-Nicolson substeps: nonlinear term with
dealiased x-z transforms, per-wavenumber implicit y-solves) of the channel at
256x193x256 (dealiased 384x384), Re 2500, tanh stretch 1.5, laminar 1-y^2
plus seeded 1e-3 k^-2 divergence-free noise, constant bulk flux, dt 0.005.
Metric: Mpts*steps/s with Mpts = nx*ny*nz = 12.648.

  python bench.py [--gpus N] [--steps K] [--warmup W]        our arm
  python bench.py --impl reference [--steps K] [--warmup W]  the CPU arm

With N > 1 (torchrun, one process per GPU) every rank advances its own
independent domain (replicas, weak scaling); the timed region is bracketed by a
barrier and the maximum device time over ranks is used.

  python bench.py --slab P [--steps K] [--warmup W]

runs ONE field split into P slab ranks (cfg_group, one process, ranks placed
round robin on the visible GPUs; several ranks may share a GPU): strong
scaling of a single domain, timed with an event pair on every rank's stream,
maximum over ranks.

  python bench.py --ensemble M [--steps K] [--warmup W]

runs configuration C5 on one GPU: M members with grids from {48x49x48,
64x65x64, 96x97x96}, Re uniform in [2000, 3000], noise seeds 1000+m
(amplitude 1e-2), the Gaussian wall jet on odd members, mixed precision,
tiles autotuned per grid, one CUDA graph launch per step; the same members
stepped one call per member per step are timed beside it.

  python bench.py --arnoldi [--arnoldi-maxiter R]

runs configuration C3: the Arnoldi stability solver about laminar Poiseuille
flow at Re 2900 on 64x65x64, T = 1 (100 linearized steps of dt 0.01 per
matvec), Krylov dimension 60, 10 leading eigenvalues, a seeded FP64 start
vector; FP64 and mixed matvecs through the host ARPACK driver, with their
matvec counts, times and the agreement of the leading eigenvalues.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, NZ = 256, 193, 256
RE, DT, STRETCH, AMPL, SEED = 2500.0, 0.005, 1.5, 1e-3, 1
METRIC = "Mpts·steps/s/GPU at 256×193×256, mixed vs FP64; NN-LES speedup at equal U+ error"
UNIT = "Mpts·steps/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def mpts(nx, ny, nz):
    return nx * ny * nz / 1e6


def workload_config(nx, ny, nz, precision):
    return {
        "workload": f"channel-flow DNS time step (3 RK3/CN substeps) at {nx}x{ny}x{nz} "
                    f"(dealiased {3 * nx // 2}x{3 * nz // 2}), Re {RE:g}, stretch {STRETCH}, "
                    f"laminar + {AMPL:g} k^-2 noise, constant flux, dt {DT}",
        "grid": [nx, ny, nz], "dealiased": [3 * nx // 2, 3 * nz // 2],
        "precision": precision, "mpts": round(mpts(nx, ny, nz), 4),
        "cache": "no L2 flush: the per-step state (>= 1 GB) is larger than the 126 MB L2",
        "parallelism": "replicas (one independent domain per GPU)",
    }


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# --------------------------------------------------------------------------
# CPU arm: the oracle (FP64 C restatement of the reference, OpenMP)
def time_oracle(nx, ny, nz, steps, warmup, budget_s=150.0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    nthreads = os.cpu_count() or 1
    o = orc.Oracle(nx, ny, nz, re=RE, dt=DT, stretch=STRETCH, nthreads=nthreads)
    o.init_field(10, seed=SEED, ampl=AMPL)
    t0 = time.perf_counter()
    o.timestep(1)
    t_step = time.perf_counter() - t0
    sample_ny = ny
    total = (steps + warmup) * t_step
    if total > budget_s:
        # bounded sample: the same x-z grid on fewer y planes
        frac = budget_s / total
        sample_ny = max(9, int(ny * frac))
        o.close()
        o = orc.Oracle(nx, sample_ny, nz, re=RE, dt=DT, stretch=STRETCH, nthreads=nthreads)
        o.init_field(10, seed=SEED, ampl=AMPL)
    for _ in range(max(0, warmup - 1)):
        o.timestep(1)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.timestep(1)
    el = time.perf_counter() - t0
    o.close()
    value = mpts(nx, sample_ny, nz) * steps / el
    sample = (f"{steps} full time steps of the oracle at {nx}x{sample_ny}x{nz}"
              + ("" if sample_ny == ny else f" (bounded sample: {sample_ny} of {ny} y-planes)"))
    return value, el / steps * 1e3, nthreads, sample


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    value, ms, cores, sample = time_oracle(args.nx, args.ny, args.nz, args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": workload_config(args.nx, args.ny, args.nz, "fp64"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample + "; reference Fortran binary unbuildable here "
                                            "(no Fortran compiler, MPI or FFTW)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
class Ranks:
    """One process per GPU (torchrun env): barrier and max/sum over ranks of
    host scalars.  Replicas only -- the step itself has no collective."""

    def __init__(self, world, rank, local, backend):
        import torch
        self.world, self.rank, self.local, self.backend = world, rank, local, backend
        self.device = "cpu"
        if world > 1:
            import datetime
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(local)
                self.device = torch.device("cuda", local)
                kw["device_id"] = self.device
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
        elif backend == "nccl":
            torch.cuda.set_device(0)

    @classmethod
    def from_env(cls, backend):
        return cls(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                   int(os.environ.get("LOCAL_RANK", "0")), backend)

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def _reduce(self, x, op):
        if self.world == 1:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        import torch.distributed as dist
        return self._reduce(x, dist.ReduceOp.MAX)

    def sum(self, x):
        import torch.distributed as dist
        return self._reduce(x, dist.ReduceOp.SUM)

    def close(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


def throughput(world, units_per_rank, steps, ms_max):
    """Whole-job Mpts*steps/s: every rank advanced its own domain `steps`
    times; the job took the slowest rank's device time."""
    return world * units_per_rank * steps / (ms_max / 1e3)


# --------------------------------------------------------------------------
class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed
    region, every 20 ms so that a timed region of a few tens of ms still has
    samples of its own."""

    PERIOD_MS = 20

    def __init__(self, device):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-i", str(device), "-lms", str(self.PERIOD_MS)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self, t0=None, t1=None):
        """Samples whose timestamps fall in [t0, t1] (host wall clock), or all."""
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        for ln in open(self.f.name):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if t0 is not None and rows:
            import datetime
            inside = []
            for r in rows:
                try:
                    ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except ValueError:
                    continue
                if t0 <= ts <= t1:
                    inside.append(r)
            rows = inside
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows),
                "period_ms": self.PERIOD_MS}


def make_flow(cf, nx, ny, nz, precision, device):
    grid = cf.Grid(nx, ny, nz, lx=4 * np.pi, lz=2 * np.pi, stretch=STRETCH)
    flow = cf.ChannelFlow(grid, re=RE, dt=DT, fix_mass=1, precision=precision, device=device)
    flow.define_initial_field(10, seed=SEED, ampl=AMPL)
    return flow


def timed_steps(torch, flow, steps, profile=False):
    stream = torch.cuda.ExternalStream(flow.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    flow.synchronize()
    if profile:
        flow.profile_enable(True)
    n0 = flow.launch_count()
    e0.record(stream)
    flow.timestep(steps)
    e1.record(stream)
    e1.synchronize()
    n1 = flow.launch_count()
    prof = flow.profile_read() if profile else None
    if profile:
        flow.profile_enable(False)
    return e0.elapsed_time(e1), n1 - n0, prof


def run_slab(args):
    import torch
    import __graft_entry__
    cf = __graft_entry__.load_package()
    nx, ny, nz, K, W, P = args.nx, args.ny, args.nz, args.steps, args.warmup, args.slab
    ndev = max(1, torch.cuda.device_count())
    devs = [i % ndev for i in range(P)]
    # the initial state (divergence removal and initial pressure need whole
    # planes) is made on one context and split among the ranks
    one = make_flow(cf, nx, ny, nz, cf.MIXED, 0)
    st, sc = one.download_state(), one.scalars()
    grid = one.grid
    one.close()
    grp = cf.Group(grid, P, devices=devs, re=RE, dt=DT, fix_mass=1, precision=cf.MIXED)
    grp.upload_state(*st)
    grp.set_scalars(sc["t_total"], sc["dt"], sc["p_grad"], sc["d_um_dy"])
    grp.timestep(W)
    grp.synchronize()
    ev = []
    for i, f in enumerate(grp.ranks):
        with torch.cuda.device(devs[i]):
            s_ = torch.cuda.ExternalStream(f.stream_ptr())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev.append((s_, e0, e1))
    for s_, e0, _ in ev:
        e0.record(s_)
    grp.timestep(K)
    for s_, _, e1 in ev:
        e1.record(s_)
    grp.synchronize()
    ms = max(e0.elapsed_time(e1) for _, e0, e1 in ev)
    status = grp.status()
    grp.close()
    cfg = workload_config(nx, ny, nz, "mixed")
    cfg["parallelism"] = f"slab x{P}: one field, {P} ranks on {len(set(devs))} GPU(s), one process"
    line = {"metric": METRIC, "value": mpts(nx, ny, nz) * K / (ms / 1e3), "unit": UNIT,
            "n_gpus": len(set(devs)), "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": cfg, "status": status}
    print(json.dumps(line), flush=True)
    return 0


def ensemble_members(cf, M):
    grids = [(48, 49, 48), (64, 65, 64), (96, 97, 96)]
    rng = np.random.default_rng(5)
    out = []
    for m in range(M):
        nx, ny, nz = grids[m % 3]
        grid = cf.Grid(nx, ny, nz, lx=4 * np.pi, lz=2 * np.pi, stretch=STRETCH)
        f = cf.ChannelFlow(grid, re=float(rng.uniform(2000.0, 3000.0)), dt=0.0025, fix_mass=1, precision=cf.MIXED)
        f.define_initial_field(10, seed=1000 + m, ampl=1e-2)
        if m % 2 == 1:
            j = cf.CfgJet()
            j.mode = 2
            j.xjet[0], j.zjet[0] = 0.3 * grid.lx, 0.5 * grid.lz
            j.jetmag[0] = 0.1
            j.width, j.freq = 0.2, 0.5
            j.frac_xbuff = 0.2
            j.seed = 1000 + m
            f.set_jet(j)
        out.append(f)
    return out


def run_ensemble(args):
    """Configuration C5: M members of three grids stepped together, timed in
    both step layouts (batched: one launch per kernel per class of equal
    grids; branches: one graph branch per member) and without a graph, with
    the 256x193x256 step's per-point rate measured in the same process as the
    yardstick."""
    import torch
    import __graft_entry__
    cf = __graft_entry__.load_package()
    M, K, W = args.ensemble, args.steps, args.warmup

    tiles = {}

    def graph_run(batched):
        mem = ensemble_members(cf, M)
        t0 = time.perf_counter()
        ens = cf.Ensemble(mem, autotune=True, batched=batched)
        tune_s = time.perf_counter() - t0
        ens.timestep(W)
        ens.synchronize()
        s_ = torch.cuda.ExternalStream(ens.stream_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("ensemble_timed")   # lets a profiler select the timed steps
        e0.record(s_)
        ens.timestep(K)
        e1.record(s_)
        e1.synchronize()
        torch.cuda.nvtx.range_pop()
        ms = e0.elapsed_time(e1) / K
        status = [f.status() for f in mem]
        launches = sum(f.launch_count() for f in mem)
        tiles.update({f"{f.nx}x{f.ny}x{f.nz}" + ("" if batched else " (branches)"): f.tiles() for f in mem})
        ens.close()
        for f in mem:
            f.close()
        return ms, tune_s, status, launches

    mem = ensemble_members(cf, M)
    pts = sum(mpts(f.nx, f.ny, f.nz) for f in mem)
    for f in mem:
        f.close()
    ms_b, tune_s, status, _ = graph_run(True)
    if args.ensemble_only:
        # the batched layout alone (for profiling its kernels)
        print(json.dumps({"metric": "ensemble member-steps/s (C5)", "value": M / (ms_b / 1e3),
                          "unit": "member·steps/s", "ms_per_step": ms_b, "mpts_steps_per_s": pts / (ms_b / 1e3),
                          "status": status}), flush=True)
        return 0
    ms_g, _, status_g, _ = graph_run(False)
    # one call per member per step (no graph), same members, default tiles
    mem = ensemble_members(cf, M)
    for f in mem:
        f.timestep(W)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(K):
        for f in mem:
            f.timestep(1)
    torch.cuda.synchronize()
    ms_eager = (time.perf_counter() - t0) * 1e3 / K
    for f in mem:
        f.close()
    # the yardstick: the 256x193x256 mixed step's rate per grid point
    big = make_flow(cf, NX, NY, NZ, cf.MIXED, 0)
    big.autotune(3)   # as the headline run does
    big.timestep(3)
    ms_big = timed_steps(torch, big, 50)[0] / 50
    big.close()
    big_rate = mpts(NX, NY, NZ) / (ms_big / 1e3)
    rate = pts / (ms_b / 1e3)
    cfg = {"workload": f"ensemble of {M} channel-flow members (C5): grids 48x49x48 / 64x65x64 / 96x97x96, "
                       "Re U[2000,3000], seeds 1000+m, jet on odd members, mixed precision, dt 0.0025",
           "members": M, "mpts_total": round(pts, 4),
           "parallelism": "one GPU, one CUDA graph per step, batched (one launch per kernel per grid class)",
           "autotune_s": round(tune_s, 2), "tiles": tiles}
    line = {"metric": "ensemble member-steps/s (C5)", "value": M / (ms_b / 1e3), "unit": "member·steps/s",
            "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms_b, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "config": cfg,
            "mpts_steps_per_s": rate,
            "vs_metric_grid_rate": {"ratio": rate / big_rate, "metric_grid_mpts_steps_per_s": big_rate,
                                    "metric_grid_ms_per_step": ms_big},
            "branches": {"ms_per_step": ms_g, "value": M / (ms_g / 1e3), "mpts_steps_per_s": pts / (ms_g / 1e3),
                         "layout": "one graph branch per member"},
            "no_graph": {"ms_per_step": ms_eager, "value": M / (ms_eager / 1e3),
                         "timing": "host wall clock around the enqueue loop, synchronised"},
            "status": status, "status_branches": status_g}
    print(json.dumps(line), flush=True)
    return 0


def run_arnoldi(args):
    """Configuration C3: 10 leading eigenvalues of the T = 1 propagator about
    laminar Poiseuille flow at Re 2900 on 64x65x64, Krylov dimension 60 per
    Fourier column (chanflow.arnoldi_columns: the linearized operator does
    not couple columns; one GPU matvec advances every column's Arnoldi),
    FP64 and mixed precision, with explicit residuals and their agreement."""
    import __graft_entry__
    cf = __graft_entry__.load_package()
    from chanflow_b200.chanflow import arnoldi_columns
    nx, ny, nz, tend = 64, 65, 64, 100
    grid = cf.Grid(nx, ny, nz, lx=4 * np.pi, lz=2 * np.pi, stretch=STRETCH)
    out = {}
    for name, prec, tol in (("fp64", cf.FP64, 1e-9), ("mixed", cf.MIXED, 1e-5)):
        f = cf.ChannelFlow(grid, re=2900.0, dt=0.01, fix_mass=0, precision=prec)
        base = np.zeros((ny + 1, 3), order="F")
        base[:, 0] = 1 - grid.yh ** 2
        f.set_baseflow(base)
        calls = [0]
        mv = f.arnoldi_matvec

        def counted(x, t, mv=mv):
            calls[0] += 1
            return mv(x, t)

        f.arnoldi_matvec = counted
        t0 = time.perf_counter()
        mu, lam, res, cols = arnoldi_columns(f, tend, ncv=60, nev=10, restarts=args.arnoldi_maxiter, tol=tol)
        out[name] = {"matvecs": calls[0], "s": time.perf_counter() - t0,
                     "mu": [[float(z.real), float(z.imag)] for z in mu],
                     "lambda": [[float(z.real), float(z.imag)] for z in lam],
                     "residual": [float(r) for r in res], "column_kx_kz": cols.tolist()}
        f.close()
    a = np.array([complex(*z) for z in out["fp64"]["mu"]])
    b = np.array([complex(*z) for z in out["mixed"]["mu"]])
    out["max_rel_diff_mixed_fp64"] = float(max(np.abs(b - m).min() / abs(m) for m in a))
    out["fp64_max_residual"] = float(max(out["fp64"]["residual"]))
    line = {"metric": "Arnoldi eigenvalues (C3)", "config": {"workload": "linearized channel about Poiseuille, "
            "Re 2900, 64x65x64, T = 1 (100 steps of dt 0.01), Krylov 60 per Fourier column, nev 10, "
            "seeded start vectors; mean and Nyquist columns excluded"},
            "n_gpus": 1, "data": "synthetic (seeded)", "result": out}
    print(json.dumps(line), flush=True)
    return 0


def run_mlp(args):
    """The closure network's tensor-core kernels alone: forward over n points
    and one training batch (forward + backward + gradient accumulation),
    timed with CUDA events; achieved FLOP/s against the measured bf16 peak
    (algorithmic: 2 x 9216 multiply-adds per point forward, 3x that to train)."""
    import importlib
    import torch
    import __graft_entry__
    cf = __graft_entry__.load_package()
    lc = importlib.import_module("chanflow_b200.les_closure")
    n, B, reps = args.mlp_points, args.mlp_batch, max(3, args.steps)
    net = cf.Mlp(0, lc.init_params(1))
    x = torch.randn(n, 10, device="cuda")
    y = torch.empty(n, 6, device="cuda")
    t = torch.randn(n, 6, device="cuda")
    idx = torch.randint(0, n, (B,), device="cuda", dtype=torch.int32)
    for _ in range(args.warmup):
        net.forward(x.data_ptr(), y.data_ptr(), n)
        net.accumulate_grad(x.data_ptr(), t.data_ptr(), idx.data_ptr(), B)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    for _ in range(reps):
        net.forward(x.data_ptr(), y.data_ptr(), n)
    e[1].record()
    for _ in range(reps):
        net.accumulate_grad(x.data_ptr(), t.data_ptr(), idx.data_ptr(), B)
    e[2].record()
    e[2].synchronize()
    fwd_ms, trn_ms = e[0].elapsed_time(e[1]) / reps, e[1].elapsed_time(e[2]) / reps
    macs = 10 * 64 + 64 * 64 * 2 + 64 * 6
    pk, kind = peaks()
    peak = float(pk.get("bf16_tflops", PEAKS_FALLBACK["bf16_tflops"]))
    fwd = 2 * macs * n / (fwd_ms / 1e3) / 1e12
    trn = 6 * macs * B / (trn_ms / 1e3) / 1e12
    line = {"metric": "closure network TFLOP/s (tensor cores)", "value": fwd, "unit": "TFLOP/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "bf16 (f32 accumulation)", "data": "synthetic (random inputs)",
            "config": {"workload": f"MLP 10-64-64-64-6 GELU forward over {n} points, training batch {B}"},
            "roofline": {"bound": "tensor", "achieved": fwd, "peak": peak, "unit": "TFLOP/s", "frac": fwd / peak,
                         "peak_kind": kind, "kernel": "k_mlp_fwd"},
            "forward_ms": fwd_ms, "train_batch_ms": trn_ms, "train_tflops": trn, "status": net.status()}
    print(json.dumps(line), flush=True)
    net.close()
    return 0


def run_les_step(args):
    """One LES step at configuration C4's LES grid (128x65x128) with the
    learned closure (random weights: every point runs the network and the
    checks) against the same grid with the eddy viscosity and without a
    model; CUDA-event times per step and per kernel."""
    import importlib
    import torch
    import __graft_entry__
    cf = __graft_entry__.load_package()
    lc = importlib.import_module("chanflow_b200.les_closure")
    grid = cf.Grid(128, 65, 128, lx=4 * np.pi, lz=2 * np.pi, stretch=STRETCH)
    out = {}
    for name, model in (("none", 0), ("eddy_viscosity", 1), ("learned", 2)):
        f = cf.ChannelFlow(grid, re=args.les_re, dt=0.005, precision=cf.MIXED)
        f.define_initial_field(4, seed=4, ampl=0.3)
        net = None
        if model:
            net = cf.Mlp(0, lc.init_params(2)) if model == 2 else None
            f.set_les(model, cs=0.1, mlp=net, in_shift=np.zeros(10), in_scale=np.ones(10), out_shift=np.zeros(6),
                      out_scale=np.full(6, 1e-3))
        f.timestep(args.warmup)
        ms, _, _ = timed_steps(torch, f, args.steps)
        _, _, prof = timed_steps(torch, f, 2, profile=True)
        out[name] = {"ms_per_step": ms / args.steps, "status": f.status(),
                     "kernels_ms": {k: v[1] / max(v[0], 1) for k, v in (prof or {}).items()}}
        f.close()
        if net is not None:
            net.close()
    line = {"metric": "LES step time at 128x65x128 (C4 LES grid)", "value": out["learned"]["ms_per_step"],
            "unit": "ms/step", "higher_is_better": False, "n_gpus": 1, "dtype": "f32 (bf16 network)",
            "data": "synthetic (seeded field, random network)", "config": {"workload": "LES 128x65x128, Re "
                                                                           f"{args.les_re:g}"}, "result": out}
    print(json.dumps(line), flush=True)
    return 0


def run_les(args):
    """Configuration C4: the learned-closure LES against plain GPU DNS."""
    import importlib
    import __graft_entry__
    __graft_entry__.load_package()
    lc = importlib.import_module("chanflow_b200.les_closure")
    t0 = time.time()
    out = lc.run_c4(nx=args.les_nx, ny=args.les_ny, nz=args.les_nx, re=args.les_re, spinup=args.les_spinup,
                    nsnap=args.les_nsnap, train_iters=args.les_train_iters, les_spin=args.les_time / 2,
                    les_avg=args.les_time / 2, beta=args.les_beta, artifact=args.les_artifact,
                    log=lambda m: print(m, file=sys.stderr, flush=True))
    learned = out["les"]["learned"]
    line = {"metric": "NN-LES speedup at equal U+ error (C4)",
            "value": out["speedup_per_time_unit"]["learned"], "unit": "x (DNS ms per time unit / LES ms per time unit)",
            "higher_is_better": True, "n_gpus": 1, "dtype": "f32 solver, bf16 network (f32 accumulation)",
            "data": "synthetic: this solver's DNS from seeded noise, box-filtered", "vs_baseline": None,
            "config": {"workload": f"LES {args.les_nx // 3}x{(args.les_ny - 1) // 3 + 1}x{args.les_nx // 3} with the "
                                   f"learned closure vs DNS {args.les_nx}x{args.les_ny}x{args.les_nx}, Re {args.les_re:g}, "
                                   "filter 3x in x, z"},
            "mean_profile_max_rel_err": learned.get("mean_profile_max_rel_err"), "result": out,
            "wall_s": time.time() - t0}
    print(json.dumps(line), flush=True)
    return 0


def pinned_state(torch, flow):
    """Pinned host copies of the flow's data1, data2, data4 (reference
    layouts, interleaved complex FP64) filled with its current state."""
    s1, s2, s4 = flow.shapes()
    pin = [torch.empty(int(np.prod(s)) * 2, dtype=torch.float64, pin_memory=True) for s in (s1, s2, s4)]
    d1, d2, d4 = flow.download_state()
    for t, a in zip(pin, (d1, d2, d4)):
        t.numpy()[:] = np.asfortranarray(a).ravel(order="F").view(np.float64)
    return pin


def host_round_trip_steps(flow, ptr, n, uploaded=None, start=None):
    """n steps of a host-owned state through the C ABI: upload data1, data2,
    data4 from pinned host memory, one time step, download them again.
    uploaded (a threading.Event) is set after the first upload; start, if
    given, is waited for before the first one."""
    L = flow.L
    if start is not None:
        start.wait()
    for i in range(n):
        flow._chk(L.cfg_upload_state(flow.h, ptr[0], ptr[1], ptr[2]))
        if i == 0 and uploaded is not None:
            uploaded.set()
        flow.timestep(1)
        flow._chk(L.cfg_download_state(flow.h, ptr[0], ptr[1], ptr[2]))


def e2e_overlapped(torch, cf, nx, ny, nz, dev, n):
    """Two independent domains, each driven by its own host thread through
    the same host round trip per step as the serial e2e (the C calls release
    the interpreter lock).  The second domain starts once the first has
    uploaded, half a cycle behind it, so that one domain's uploads run while
    the other downloads (the host link carries both directions at once) and
    each domain's step runs under the other's copies.  Device time from
    events on both streams, first start to last end."""
    import threading
    flows = [make_flow(cf, nx, ny, nz, cf.MIXED, dev) for _ in range(2)]
    pins = [pinned_state(torch, f) for f in flows]
    streams = [torch.cuda.ExternalStream(f.stream_ptr()) for f in flows]
    for f in flows:
        host_round_trip_steps(f, [t.data_ptr() for t in pins[flows.index(f)]], 1)   # warm-up
        f.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in flows]
    for (e0, _), st in zip(ev, streams):
        e0.record(st)
    first_up = threading.Event()
    th = [threading.Thread(target=host_round_trip_steps, args=(flows[0], [t.data_ptr() for t in pins[0]], n),
                           kwargs={"uploaded": first_up}),
          threading.Thread(target=host_round_trip_steps, args=(flows[1], [t.data_ptr() for t in pins[1]], n),
                           kwargs={"start": first_up})]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for (_, e1), st in zip(ev, streams):
        e1.record(st)
    for _, e1 in ev:
        e1.synchronize()
    ms = max(ev[0][0].elapsed_time(e1) for _, e1 in ev)
    nbytes = sum(t.numel() * 8 for t in pins[0])
    for f in flows:
        f.close()
    return ms, nbytes


def error_vs_fp64(cf, nx, ny, nz, dev, steps):
    """Relative L2 difference of the mixed-precision velocity (data1) from
    the FP64 path's after `steps` steps from the same seeded initial field:
    over the whole field and over its perturbation (every Fourier column
    except the kx = kz = 0 mean), with the change of the FP64 field over the
    run beside them."""
    a = make_flow(cf, nx, ny, nz, cf.FP64, dev)
    b = make_flow(cf, nx, ny, nz, cf.MIXED, dev)
    d0 = a.download_state()[0]
    a.timestep(steps)
    b.timestep(steps)
    da, db = a.download_state()[0], b.download_state()[0]
    st = (a.status(), b.status())
    a.close()
    b.close()

    def rel(x, y):
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))

    pa, pb, p0 = da.copy(), db.copy(), d0.copy()
    for arr in (pa, pb, p0):
        arr[0, 0] = 0
    return {"steps": steps, "whole_field": rel(db, da), "perturbation": rel(pb, pa),
            "fp64_change_whole": rel(da, d0), "fp64_change_perturbation": rel(pa, p0), "status": list(st),
            "field": "data1 (u, v, w), relative L2; perturbation = all columns but kx = kz = 0"}


def run_ours(args):
    import torch
    import __graft_entry__
    cf = __graft_entry__.load_package()

    rk = Ranks.from_env("nccl")
    world, rank = rk.world, rk.rank
    dev = torch.cuda.current_device()
    barrier, max_over_ranks, sum_over_ranks = rk.barrier, rk.max, rk.sum

    nx, ny, nz, K, W = args.nx, args.ny, args.nz, args.steps, args.warmup
    units = mpts(nx, ny, nz)
    results = {}
    for prec_name, prec in (("mixed", cf.MIXED), ("fp64", cf.FP64)):
        if prec_name == "fp64" and args.no_fp64:
            continue
        flow = make_flow(cf, nx, ny, nz, prec, dev)
        # launch tiles tuned on this grid (outside the timed region; the
        # state is restored, results do not depend on the tiles)
        tiles = flow.autotune(3) if not args.no_autotune else None
        clocks = Clocks(dev) if prec_name == "mixed" else None
        flow.timestep(W)
        flow.synchronize()
        barrier()
        t_host0 = time.time()
        ms, nlaunch, _ = timed_steps(torch, flow, K)
        t_host1 = time.time()
        cl = clocks.stop(t_host0, t_host1) if clocks else None
        barrier()
        ms_max = max_over_ranks(ms)
        st = flow.status()
        q, div = flow.diagnostics()
        # per-kernel breakdown: a separate, shorter run with an event pair
        # around every launch (not part of the timed number)
        kp = max(1, min(K, 10))
        _, _, prof = timed_steps(torch, flow, kp, profile=True)
        results[prec_name] = {"ms_total": ms_max, "launches": sum_over_ranks(nlaunch), "prof": prof, "tiles": tiles,
                              "prof_steps": kp, "clocks": cl, "status": st, "div": div, "q": q}
        if prec_name == "mixed" and not args.no_e2e:
            # end to end through the public API with host buffers: every step
            # uploads data1/data2/data4 from pinned host memory, advances one
            # step and downloads data1/data2/data4 (a host-owned state).
            ke = max(1, min(K, args.e2e_steps))
            pin = pinned_state(torch, flow)
            ptr = [t.data_ptr() for t in pin]
            stream = torch.cuda.ExternalStream(flow.stream_ptr())
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            host_round_trip_steps(flow, ptr, ke)
            e1.record(stream)
            e1.synchronize()
            e2e_ms = max_over_ranks(e0.elapsed_time(e1))
            nbytes = sum(t.numel() * 8 for t in pin)
            results["e2e"] = {"value": throughput(world, units, ke, e2e_ms), "unit": UNIT,
                              "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                              "how": "serial: every step uploads data1/data2/data4 from pinned host memory, "
                                     "steps once and downloads them (a host-owned state)"}
            del pin
        flow.close()
        torch.cuda.synchronize()

    # the same e2e with two domains whose host round trips overlap (two host
    # threads); every rank does the same
    ke = max(1, min(K, args.e2e_steps))
    ms_ov, nb_ov = e2e_overlapped(torch, cf, nx, ny, nz, dev, ke) if not args.no_e2e else (float("nan"), 0)
    ms_ov = max_over_ranks(ms_ov)
    results["e2e_overlapped"] = None if args.no_e2e else {
        "value": throughput(world, 2 * units, ke, ms_ov), "unit": UNIT,
        "h2d_bytes_per_step": nb_ov, "d2h_bytes_per_step": nb_ov,
        "how": "two independent domains per GPU, one host thread each, every domain step uploads, steps and "
               "downloads its state as in the serial e2e; the second starts half a cycle behind, so one "
               "domain's uploads run during the other's downloads and steps"}
    # mixed against FP64 on the workload (outside every timed region)
    err = error_vs_fp64(cf, nx, ny, nz, dev, args.error_steps) if args.error_steps > 0 else None

    # CPU baseline on rank 0 at N = 1
    cpu = None
    if world == 1 and not args.no_cpu:
        v, ms, cores, sample = time_oracle(nx, ny, nz, steps=1, warmup=1, budget_s=30.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        mix = results["mixed"]
        ms_step = mix["ms_total"] / K
        value = throughput(world, units, K, mix["ms_total"])
        pk, pk_kind = peaks()
        hbm = float(pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
        nxh, n1, nx2, nz2 = nx // 2 + 1, ny + 1, 3 * nx // 2, 3 * nz // 2
        nf = nz * nxh * n1
        sc, sr = 8, 4  # FP32 complex / real bytes
        # algorithmic bytes per launch: what each kernel must read and write
        # given its inputs and outputs (one substep)
        t1 = 3 * n1 * nxh * nz2 * sc                 # hybrid planes
        pp = 3 * n1 * nz2 * nx2 * sr                 # physical planes
        t2 = 6 * (ny - 1) * nxh * nz2 * sc           # x-transformed fluxes
        per_kernel_bytes = {
            "k_zinv": 3 * nf * sc + t1, "k_xinv": t1 + pp, "k_flux": pp + t2,
            "k_zfwd": t2 + 3 * nf * sc, "k_xflux": t1 + t2,
            "k_rhs": 14 * nf * sc,   # all wavenumbers (the ~50 FP64 ones run beside it)
        }
        prof = dict(mix["prof"] or {})
        if "k_zfwd_low" in prof and "k_zfwd" in prof:
            # the z transform runs as two launches (low kx columns first)
            lo, hi = prof.pop("k_zfwd_low"), prof["k_zfwd"]
            prof["k_zfwd"] = (hi[0], hi[1] + lo[1])
        kp = mix["prof_steps"]
        tot_prof = sum(v[1] for k, v in prof.items() if k not in ("k_rhs_fp64", "k_rhs_mean")) or 1.0
        kernels = {}
        for k, v in prof.items():
            ent = {"launches": v[0], "ms_per_launch": v[1] / max(v[0], 1)}
            if k in ("k_rhs_fp64", "k_rhs_mean"):
                ent["note"] = "side stream, overlaps k_rhs: wall time from its fork, not a serial share"
            else:
                ent["share"] = v[1] / tot_prof
            if k in per_kernel_bytes:
                ent["algorithmic_bytes"] = per_kernel_bytes[k]
                ent["achieved_gbs"] = per_kernel_bytes[k] / (ent["ms_per_launch"] / 1e3) / 1e9
                ent["frac"] = ent["achieved_gbs"] / hbm
            kernels[k] = ent
        traffic = {}
        tp = os.path.join(ROOT, "profiles", "traffic_per_launch.json")
        if os.path.exists(tp):
            traffic = json.load(open(tp)).get("bytes", {})
        # the dominant kernel: largest total device time on the main stream
        dom = max((k for k in kernels if "share" in kernels[k] and k in per_kernel_bytes),
                  key=lambda k: kernels[k]["share"], default=None)
        best = None
        if dom is not None:
            kd = kernels[dom]
            best = {"bound": "hbm", "kernel": dom, "achieved": kd["achieved_gbs"], "peak": hbm, "unit": "GB/s",
                    "frac": kd["frac"], "traffic": traffic.get(dom), "algorithmic_bytes": kd["algorithmic_bytes"],
                    "ms_per_launch": kd["ms_per_launch"],
                    "peak_kind": "measured (MEASURED_PEAKS.json hbm_gbs)" if pk_kind == "measured"
                    else "fallback"}
        step_bytes = 3 * 20 * nf * sc
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (f64 mean mode and |k|<4 solves)", "data": "synthetic (seeded initial field)",
            "config": dict(workload_config(nx, ny, nz, "mixed"),
                           tiles={k: list(v["tiles"]) for k, v in results.items() if v and v.get("tiles")}),
            "roofline": best,
            "roofline_step": {"bound": "hbm", "achieved": step_bytes / (ms_step / 1e3) / 1e9, "peak": hbm,
                              "unit": "GB/s", "frac": step_bytes / (ms_step / 1e3) / 1e9 / hbm,
                              "algorithmic_bytes": step_bytes},
            "kernels": kernels,
            "e2e": results.get("e2e"),
            "e2e_overlapped": results.get("e2e_overlapped"),
            "error_vs_fp64": err,
            "gpu_launches": int(mix["launches"]),
            "clocks": mix["clocks"],
            "cpu_baseline": cpu,
            "checks": {"status": mix["status"], "max_divergence": mix["div"], "bulk_flux": mix["q"]},
        }
        if "fp64" in results:
            f = results["fp64"]
            line["value_fp64"] = throughput(world, units, K, f["ms_total"])
            line["ms_per_step_fp64"] = f["ms_total"] / K
            line["fp64_roofline_step"] = {
                "achieved": 3 * 20 * nf * 16 / (f["ms_total"] / K / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": 3 * 20 * nf * 16 / (f["ms_total"] / K / 1e3) / 1e9 / hbm}
        print(json.dumps(line), flush=True)
    rk.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--ny", type=int, default=NY)
    ap.add_argument("--nz", type=int, default=NZ)
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--error-steps", type=int, default=100,
                    help="steps of the mixed-vs-FP64 error check outside the timed region (0: skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--slab", type=int, default=0, help="one field in P slab ranks (one process)")
    ap.add_argument("--ensemble", type=int, default=0, help="configuration C5 with M members (one GPU)")
    ap.add_argument("--ensemble-only", action="store_true", help="time the batched ensemble layout only")
    ap.add_argument("--arnoldi", action="store_true", help="configuration C3 (Arnoldi eigenvalues)")
    ap.add_argument("--arnoldi-maxiter", type=int, default=6, help="Krylov-Schur cycles of the C3 run")
    ap.add_argument("--les", action="store_true", help="configuration C4 (learned-closure LES vs DNS)")
    ap.add_argument("--mlp", action="store_true", help="the closure network's tensor-core kernels alone")
    ap.add_argument("--mlp-points", type=int, default=2400000)
    ap.add_argument("--mlp-batch", type=int, default=65536)
    ap.add_argument("--les-step", action="store_true", help="LES step times at the C4 LES grid")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end legs (profiling runs)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default tiles (profiling runs)")
    ap.add_argument("--les-nx", type=int, default=384)
    ap.add_argument("--les-ny", type=int, default=193)
    ap.add_argument("--les-re", type=float, default=10350.0)
    ap.add_argument("--les-spinup", type=float, default=60.0)
    ap.add_argument("--les-nsnap", type=int, default=40)
    ap.add_argument("--les-train-iters", type=int, default=3000)
    ap.add_argument("--les-time", type=float, default=40.0)
    ap.add_argument("--les-beta", type=float, default=0.0, help="admitted backscatter of the learned closure")
    ap.add_argument("--les-artifact", default=None, help="save the a-posteriori inputs (.npz) here")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.slab > 0:
        return run_slab(args)
    if args.ensemble > 0:
        return run_ensemble(args)
    if args.arnoldi:
        return run_arnoldi(args)
    if args.les:
        return run_les(args)
    if args.mlp:
        return run_mlp(args)
    if args.les_step:
        return run_les_step(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
