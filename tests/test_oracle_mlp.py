"""Pins the network oracle (oracle/mlp.py): its exact backward pass equals finite differences of its exact forward,
its BF16 rounding is round-to-nearest-even, and its Adam step is the published update (Kingma and Ba, 2015)."""
import numpy as np

from oracle import mlp as M


def loss_of(p, x, t):
    y, _ = M.forward(p, x, exact=True)
    return float(np.sum((y - t) ** 2) / x.shape[0])


def test_oracle_backward_equals_finite_differences():
    rng = np.random.default_rng(0)
    p = {k: v.astype(np.float64) for k, v in M.init(1).items()}
    for k in ("b1", "b2", "b3"):
        p[k] = rng.standard_normal(p[k].shape) * 0.1
    x = rng.standard_normal((40, 16))
    t = rng.standard_normal((40, 2))
    g, _ = M.gradients(p, x, t, exact=True)
    eps = 1e-6
    for k in p:
        flat = p[k].reshape(-1)
        for i in rng.choice(flat.size, size=min(12, flat.size), replace=False):
            keep = flat[i]
            flat[i] = keep + eps
            up = loss_of(p, x, t)
            flat[i] = keep - eps
            down = loss_of(p, x, t)
            flat[i] = keep
            numeric = (up - down) / (2 * eps)
            assert abs(numeric - g[k].reshape(-1)[i]) < 1e-6 + 1e-5 * abs(numeric), (k, i)


def test_oracle_bf16_rounds_to_nearest_even():
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties go to the even one (1); just above goes up
    assert M.bf16(np.float32(1.0 + 2.0 ** -8)) == 1.0
    assert M.bf16(np.float32(1.0 + 2.0 ** -8 + 2.0 ** -20)) == 1.0 + 2.0 ** -7
    assert M.bf16(np.float32(1.0 + 3 * 2.0 ** -8)) == 1.0 + 2.0 ** -6  # tie to even upward
    assert M.bf16(np.float32(-2.5)) == -2.5


def test_oracle_adam_step():
    p = {"w": np.array([1.0], np.float32)}
    g = {"w": np.array([0.5])}
    m = {"w": np.zeros(1)}
    v = {"w": np.zeros(1)}
    M.adam(p, g, m, v, 1, lr=1e-3)
    # the first step moves each weight by lr against the gradient's sign
    assert abs(float(p["w"][0]) - (1.0 - 1e-3)) < 1e-7
