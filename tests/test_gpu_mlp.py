"""The closure network's tensor-core kernels (cfg_mlp_*, csrc/mlp.cu) against
the CPU restatement (oracle/mlp_oracle.py, BF16 operands emulated):

- forward on 1000 points (a partial last tile): relative L2 <= 2e-3 (BF16
  activations: a rounding of a hidden value that falls the other way moves
  an output by ~1 BF16 ulp);
- the gradient of one batch of 700 rows picked by an index list: relative
  L2 <= 1e-2 per weight and bias tensor, the loss to 1e-4;
- the Adam update from the GPU's own gradient: parameters to 1e-6;
- training: a student network fitted to a fixed teacher network's outputs
  lowers its loss more than 10x in 300 Adam steps;
- reproducibility: two trainings from the same start on the same batches
  (one of them larger than the per-tile gradient slices held from creation)
  end with the same parameters and losses, bit for bit.
"""
import numpy as np
import pytest

import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def params(seed):
    rng = np.random.default_rng(seed)
    p = mo.init_params(seed).astype(np.float64)
    d = mo.unpack(p)
    for l in range(4):
        d[f"b{l}"] = 0.1 * rng.standard_normal(d[f"b{l}"].shape)
    return mo.pack(d).astype(np.float32)


def test_forward_matches_oracle(cf):
    import torch
    m = cf.Mlp(0, params(1))
    rng = np.random.default_rng(2)
    x = rng.standard_normal((1000, 10)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    yd = torch.full((1000, 6), float("nan"), device="cuda")
    m.forward(xd.data_ptr(), yd.data_ptr(), 1000)
    torch.cuda.synchronize()
    assert m.status() == 0
    y = yd.cpu().numpy()
    yo, _ = mo.forward(m.get_params().astype(np.float64), x.astype(np.float64))
    e = rel(y, yo)
    print(f"mlp forward rel L2 {e:.3e}")
    assert np.isfinite(y).all() and e < 2e-3, e
    m.close()


def test_gradient_matches_oracle(cf):
    import torch
    p = params(3)
    m = cf.Mlp(0, p)
    rng = np.random.default_rng(4)
    x = rng.standard_normal((1000, 10)).astype(np.float32)
    t = rng.standard_normal((1000, 6)).astype(np.float32)
    idx = rng.choice(1000, 700, replace=False).astype(np.int32)
    xd, td, idd = (torch.from_numpy(a).cuda() for a in (x, t, idx))
    m.accumulate_grad(xd.data_ptr(), td.data_ptr(), idd.data_ptr(), 700)
    g, loss = m.grads()
    assert m.status() == 0
    lo, go = mo.loss_and_grad(p.astype(np.float64), x[idx].astype(np.float64), t[idx].astype(np.float64))
    assert abs(loss - lo) < 1e-4 * lo, (loss, lo)
    gd, god = mo.unpack(g), mo.unpack(go)
    for name, _ in mo.SHAPES:
        e = rel(gd[name], god[name])
        print(f"grad {name} rel L2 {e:.3e}")
        assert e < 1e-2, (name, e)
    # the Adam update from this gradient
    m.adam_step(1e-3)
    p1 = m.get_params()
    po, _, _ = mo.adam(p.astype(np.float64), g.astype(np.float64), np.zeros(p.size), np.zeros(p.size), 1, 1e-3)
    assert np.abs(p1 - po).max() < 1e-6
    g2, loss2 = m.grads()
    assert not g2.any() and loss2 == 0.0          # the step cleared the accumulators
    m.close()


def test_training_fits_a_teacher(cf):
    import torch
    rng = np.random.default_rng(5)
    teacher = params(6).astype(np.float64)
    x = rng.standard_normal((8192, 10)).astype(np.float32)
    t, _ = mo.forward(teacher, x.astype(np.float64), emulate=False)
    t = t.astype(np.float32)
    m = cf.Mlp(0, mo.init_params(7))
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(8)
    losses = []
    for it in range(300):
        idx = torch.randint(0, 8192, (1024,), device="cuda", dtype=torch.int32, generator=gen)
        m.accumulate_grad(xd.data_ptr(), td.data_ptr(), idx.data_ptr(), 1024)
        if it % 50 == 0 or it == 299:
            losses.append(m.grads()[1])
        m.adam_step(3e-3)
    torch.cuda.synchronize()
    assert m.status() == 0
    print("mlp training losses", losses)
    assert losses[-1] < 0.1 * losses[0], losses
    m.close()


def test_training_is_reproducible(cf):
    import torch
    rng = np.random.default_rng(9)
    x = rng.standard_normal((8192, 10)).astype(np.float32)
    t = rng.standard_normal((8192, 6)).astype(np.float32)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()

    def run():
        m = cf.Mlp(0, params(10))
        gen = torch.Generator(device="cuda")
        gen.manual_seed(11)
        losses = []
        for it in range(20):
            for b in (1000, 70000 if it == 5 else 3000):
                idx = torch.randint(0, 8192, (b,), device="cuda", dtype=torch.int32, generator=gen)
                m.accumulate_grad(xd.data_ptr(), td.data_ptr(), idx.data_ptr(), b)
            losses.append(m.grads()[1])
            m.adam_step(1e-3)
        torch.cuda.synchronize()
        assert m.status() == 0
        p = m.get_params()
        m.close()
        return p, losses

    p1, l1 = run()
    p2, l2 = run()
    assert l1 == l2, (l1, l2)
    assert np.array_equal(p1.view(np.uint32), p2.view(np.uint32))
