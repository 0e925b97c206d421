"""CPU restatement of the learned subgrid-stress closure network -- TEST
INFRASTRUCTURE ONLY: the checker of the tensor-core kernels of
3d-navier-stokes-thesis-paper_b200/csrc/mlp.cu (forward, backward, Adam).

The network: 10 -> 64 -> 64 -> 64 -> 6, GELU (tanh form) on the hidden
layers, y = W x + b per layer; parameters as one flat FP32 vector
W0[64][10] b0[64] W1[64][64] b1[64] W2[64][64] b2[64] W3[6][64] b3[6].
Loss: the mean over the batch and the 6 outputs of (y - t)^2.

The reference has no learned closure (its subgrid modules are missing, see
PFC/main_mpi.f90:10-13), so parity is against this restatement.  With
emulate=True the arithmetic follows the kernels' precisions: every operand
of a product (inputs, weights, activations, backward gradients) is rounded
to BF16 (round to nearest even, through FP32), products and sums are exact
(FP64 here, FP32 accumulation on the GPU), bias gradients sum the unrounded
gradients.  emulate=False is plain FP64 (checked by finite differences).
"""
import math

import numpy as np

IN, H, OUT = 10, 64, 6
SHAPES = [("W0", (H, IN)), ("b0", (H,)), ("W1", (H, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
          ("W3", (OUT, H)), ("b3", (OUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, o = {}, 0
    for name, s in SHAPES:
        n = int(np.prod(s))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(s)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def bf16(a):
    """Round to BF16 (nearest even) through FP32, returned as float64."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


C_GELU, A_GELU = math.sqrt(2.0 / math.pi), 0.044715


def gelu(z):
    """GELU in its tanh form (Hendrycks & Gimpel 2016), exact tanh."""
    return 0.5 * z * (1.0 + np.tanh(C_GELU * (z + A_GELU * z ** 3)))


def gelu_d(z):
    t = np.tanh(C_GELU * (z + A_GELU * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * A_GELU * z * z)


def init_params(seed=0):
    """He-normal weights (scaled by sqrt(2/fan_in)) and zero biases, FP32."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, s in SHAPES:
        d[name] = rng.standard_normal(s) * math.sqrt(2.0 / s[1]) if name[0] == "W" else np.zeros(s)
    return pack(d).astype(np.float32)


def forward(p, x, emulate=True):
    """Outputs y (n, 6) and the cache of the backward pass."""
    P = unpack(p)
    r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    xs, zs = [r(x)], []
    for l in range(4):
        z = xs[-1] @ r(P[f"W{l}"]).T + P[f"b{l}"]
        zs.append(z)
        if l < 3:
            xs.append(r(gelu(z)))
    return zs[3], (xs, zs)


def loss_and_grad(p, x, t, emulate=True):
    """Mean-square loss over batch x 6 outputs and its gradient (flat)."""
    P = unpack(p)
    r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    y, (xs, zs) = forward(p, x, emulate)
    b = x.shape[0]
    d = y - t
    loss = float(np.sum(d * d) / (6.0 * b))
    dz = 2.0 * d / (6.0 * b)
    g = {}
    for l in range(3, -1, -1):
        g[f"b{l}"] = dz.sum(axis=0)
        dzr = r(dz)
        g[f"W{l}"] = dzr.T @ xs[l]
        if l > 0:
            dx = dzr @ r(P[f"W{l}"])
            dz = dx * gelu_d(zs[l - 1])
    return loss, pack(g)


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (bias corrected); returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    ph = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return ph, m, v
