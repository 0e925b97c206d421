"""The multi-process (replica) plumbing of bench.py, on the CPU with gloo at
world size 2: barrier, max/sum over ranks, the whole-job throughput taken on
the slowest rank, and the reference arm's non-zero ranks exiting without
work.  The step itself has no collective (each rank advances its own
domain), so nothing else crosses ranks."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    rk = bench.Ranks.from_env("gloo")
    ms = 10.0 + rank          # rank 1 is the slower one
    mx = rk.max(ms)
    sm = rk.sum(1.0 + rank)
    rk.barrier()
    v = bench.throughput(rk.world, 12.648, 5, mx)
    rk.close()
    q.put((rank, mx, sm, v))


def test_ranks_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, sm, v in out:
        assert mx == 11.0
        assert sm == 3.0
        assert v == pytest.approx(2 * 12.648 * 5 / 11e-3)


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1"], cwd=ROOT, env=env,
                       capture_output=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == b""
