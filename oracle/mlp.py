"""CPU ORACLE — test infrastructure only. The learned warm start's network in numpy float64: forward, backward and
Adam, with the same roundings to BF16 the GPU kernels make (weights, inputs, hidden activations and the
back-propagated deltas are BF16 operands of the tensor-core products; every product accumulates in FP32 or better).

The network has no reference counterpart: it is the 16 -> 64 -> 64 -> 2 multilayer perceptron with SiLU activations
that predicts a contact's starting normal and friction impulse. Used only by tests/ to check the CUDA kernels'
outputs and gradients.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 16, 64, 2


def bf16(a) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32)
    out = np.where(np.isnan(f), f, out)
    return out.astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def init(seed: int = 0) -> dict:
    """He-style initial weights (FP32 masters)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return {
        "w1": (rng.standard_normal((IN, HID)) * np.sqrt(2.0 / IN)).astype(np.float32),
        "b1": np.zeros(HID, np.float32),
        "w2": (rng.standard_normal((HID, HID)) * np.sqrt(2.0 / HID)).astype(np.float32),
        "b2": np.zeros(HID, np.float32),
        "w3": (rng.standard_normal((HID, OUT)) * np.sqrt(1.0 / HID)).astype(np.float32),
        "b3": np.zeros(OUT, np.float32),
    }


def _rounding(exact: bool):
    return (lambda a: np.asarray(a, dtype=np.float64)) if exact else bf16


def forward(p: dict, x, exact: bool = False):
    """y, and what the backward pass needs. x: (B, 16). exact: no rounding to BF16 (float64 throughout)."""
    r = _rounding(exact)
    xb = r(x)
    z1 = xb @ r(p["w1"]) + np.asarray(p["b1"], np.float64)
    h1 = r(silu(z1))
    z2 = h1 @ r(p["w2"]) + np.asarray(p["b2"], np.float64)
    h2 = r(silu(z2))
    y = h2 @ r(p["w3"]) + np.asarray(p["b3"], np.float64)
    return y, (xb, z1, h1, z2, h2)


def gradients(p: dict, x, t, exact: bool = False):
    """Gradients of the loss sum over the batch of |y - t|^2 / B (mean squared error over rows, summed over the two
    outputs), the deltas rounded to BF16 where the kernels feed them to the tensor cores (the bias gradients are
    sums of the rounded deltas: the kernels form them as a product with a row of ones)."""
    b = x.shape[0]
    r = _rounding(exact)
    y, (xb, z1, h1, z2, h2) = forward(p, x, exact)
    d3 = 2.0 * (y - t) / b
    d3b = r(d3)
    g = {"w3": h2.T @ d3b, "b3": d3b.sum(0)}
    dh2 = d3b @ r(p["w3"]).T
    d2 = dh2 * silu_grad(z2)
    d2b = r(d2)
    g["w2"] = h1.T @ d2b
    g["b2"] = d2b.sum(0)
    dh1 = d2b @ r(p["w2"]).T
    d1 = dh1 * silu_grad(z1)
    d1b = r(d1)
    g["w1"] = xb.T @ d1b
    g["b1"] = d1b.sum(0)
    loss = float(np.sum((y - t) ** 2) / b)
    return g, loss


def adam(p: dict, g: dict, m: dict, v: dict, step: int, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8) -> None:
    """One Adam step on the FP32 masters, in place (step counts from 1)."""
    for k in p:
        m[k] = beta1 * m[k] + (1 - beta1) * g[k]
        v[k] = beta2 * v[k] + (1 - beta2) * g[k] * g[k]
        mh = m[k] / (1 - beta1 ** step)
        vh = v[k] / (1 - beta2 ** step)
        p[k] = (p[k] - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32)
