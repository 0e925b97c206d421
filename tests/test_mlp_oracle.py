"""The CPU restatement of the closure network (oracle/mlp_oracle.py), the
checker of the tensor-core kernels: its BF16 rounding equals torch's, and its
backward pass equals finite differences of its forward pass (FP64)."""
import numpy as np

import mlp_oracle as mo


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(0)
    a = np.concatenate([rng.standard_normal(4000) * 10.0 ** rng.integers(-6, 6, 4000),
                        np.array([1.0, 1.00390625, 1.005859375, -2.5, 0.0])])
    ref = torch.from_numpy(a.astype(np.float32)).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(mo.bf16(a), ref)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = mo.init_params(3).astype(np.float64)
    p += 0.05 * rng.standard_normal(p.size)            # non-zero biases too
    x = rng.standard_normal((37, 10))
    t = rng.standard_normal((37, 6))
    loss, g = mo.loss_and_grad(p, x, t, emulate=False)
    idx = rng.choice(p.size, 60, replace=False)
    for i in idx:
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (mo.loss_and_grad(p + e, x, t, False)[0] - mo.loss_and_grad(p - e, x, t, False)[0]) / 2e-6
        assert abs(fd - g[i]) < 1e-6 * max(1.0, abs(g[i])) + 1e-8, (i, fd, g[i])
    assert loss > 0


def test_adam_first_step_moves_by_lr():
    p = np.zeros(5)
    g = np.array([1.0, -2.0, 3.0, 0.5, -0.1])
    ph, m, v = mo.adam(p, g, np.zeros(5), np.zeros(5), 1, lr=1e-3)
    # the bias-corrected first step is lr * sign(g) (up to eps)
    assert np.allclose(ph, -1e-3 * np.sign(g), rtol=1e-6)
