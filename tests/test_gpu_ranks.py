"""Multi-process runs (cfg_rank_*): two processes, each one rank of the slab
decomposition, exchange CUDA IPC handles through torch.distributed (gloo on
127.0.0.1) and advance one field with a host barrier between the phases.
Both processes share the one GPU of this run; no kernel or stream waits on
the other process (each rank completes its own stores before the host
barrier).  The gathered state must equal the single-context run bit for bit.
"""
import datetime
import os
import socket

import numpy as np
import pytest

from conftest import whole_velocity_transforms

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, nranks, port, prec, dt_flag, inp, outp, ordered):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks, timeout=datetime.timedelta(seconds=120))
    import __graft_entry__
    cf = __graft_entry__.load_package()
    z = np.load(inp)
    grid = cf.Grid(32, 33, 32, stretch=1.5)
    me = cf.Rank(grid, rank, nranks, re=2500.0, dt=0.004, precision=prec, dt_flag=dt_flag)
    recs = [None] * nranks
    dist.all_gather_object(recs, me.record())
    me.connect(recs)
    sl = me.slab()
    me.upload_state(z["d1"][:, sl], z["d2"][..., sl], z["d4"][..., sl])
    me.set_scalars(float(z["t"]), float(z["dt"]), float(z["pg"]), z["dud"])
    if ordered:
        # the stream-ordered entry point; NCCL cannot put two ranks on one
        # GPU, so the barrier here waits for this rank's stream on the host,
        # then meets the others (a valid, stronger stream-ordered barrier)
        def barrier():
            me.synchronize()
            dist.barrier()
        me.timestep(4, barrier=barrier, ordered=True)
    else:
        me.timestep(4, barrier=dist.barrier)
    d1, d2, d4 = me.download_state()
    sc = me.scalars()
    np.savez(outp % rank, d1=d1, d2=d2, d4=d4, dt=sc["dt"], pg=sc["p_grad"], dud=sc["d_um_dy"],
             status=me.status())
    dist.barrier()   # no rank unmaps while another still writes into it
    me.close()
    dist.destroy_process_group()


@pytest.mark.parametrize("prec,dt_flag,ordered", [(0, 1, False), (1, 0, False), (1, 1, True)])
def test_two_processes_match_single_context(cf, tmp_path, prec, dt_flag, ordered):
    import multiprocessing as mp
    grid = cf.Grid(32, 33, 32, stretch=1.5)
    d1 = cf.initial_field(grid, 10, seed=11, ampl=5e-2)
    with whole_velocity_transforms():   # as the ranks of a multi-rank run
        f = cf.ChannelFlow(grid, re=2500.0, dt=0.004, precision=prec, dt_flag=dt_flag)
    f.upload_state(d1, d1.transpose(2, 3, 0, 1).copy(), None)
    f.remove_initial_divergence()
    f.compute_initial_pressure()
    st, sc = f.download_state(), f.scalars()
    inp = str(tmp_path / "in.npz")
    np.savez(inp, d1=st[0], d2=st[1], d4=st[2], t=sc["t_total"], dt=sc["dt"], pg=sc["p_grad"], dud=sc["d_um_dy"])
    f.upload_state(*st)
    f.timestep(4)
    ref, rsc = f.download_state(), f.scalars()
    f.close()

    nranks = 2
    outp = str(tmp_path / "out%d.npz")
    ctx = mp.get_context("spawn")
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, nranks, port, prec, dt_flag, inp, outp, ordered))
          for r in range(nranks)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=300)
    codes = [p.exitcode for p in ps]
    for p in ps:
        if p.is_alive():
            p.kill()
    assert codes == [0] * nranks, codes
    outs = [np.load(outp % r) for r in range(nranks)]
    got = (np.concatenate([o["d1"] for o in outs], axis=1), np.concatenate([o["d2"] for o in outs], axis=3),
           np.concatenate([o["d4"] for o in outs], axis=2))
    for a, b in zip(ref, got):
        np.testing.assert_array_equal(a, b)
    for o in outs:
        assert float(o["dt"]) == rsc["dt"] and int(o["status"]) == 0
    assert float(outs[0]["pg"]) == rsc["p_grad"]
    np.testing.assert_array_equal(outs[0]["dud"], rsc["d_um_dy"])
