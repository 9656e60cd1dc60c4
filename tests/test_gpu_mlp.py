"""The learned warm start's network on the tensor cores: forward outputs and gradients against the float64 oracle
(oracle/mlp.py, which rounds to BF16 where the kernels do), and training that lowers the loss."""
import numpy as np
import pytest

from oracle import mlp as M

pytestmark = pytest.mark.gpu

# BF16 operands carry 8 significant bits; the products accumulate in FP32 on the GPU and in float64 in the oracle.
OUT_TOL = 2e-2   # forward: relative to the outputs' scale
GRAD_TOL = 3e-2  # gradients: relative to each gradient block's scale


def net(seed=0):
    from vxr.learned import Mlp
    return Mlp(seed=seed)


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-12))


def test_gpu_mlp_forward_matches_the_oracle():
    """1,000 rows (a ragged last tile) through the GPU's weights: the same outputs as the oracle's forward."""
    rng = np.random.default_rng(1)
    n = net(3)
    x = rng.standard_normal((1000, 16)).astype(np.float32)
    y = n.forward(x)
    p, mean, inv = n.get()
    want, _ = M.forward(p, (x - mean) * inv)
    assert rel_err(y, want) < OUT_TOL
    n.close()


def test_gpu_mlp_gradients_match_the_oracle():
    """Gradients of the mean squared error over 300 rows (three tiles, the last ragged), every block of weights and
    biases, against the oracle's."""
    rng = np.random.default_rng(2)
    n = net(5)
    x = rng.standard_normal((300, 16)).astype(np.float32)
    t = rng.standard_normal((300, 2)).astype(np.float32)
    g, loss = n.gradients(x, t)
    p, _, _ = n.get()
    want, want_loss = M.gradients(p, x, t)
    for k in want:
        assert rel_err(g[k], want[k]) < GRAD_TOL, k
    assert abs(loss - want_loss) / want_loss < 1e-2
    n.close()


def test_gpu_mlp_two_calls_agree_and_set_get_round_trip():
    rng = np.random.default_rng(3)
    n = net(7)
    p, _, _ = n.get()
    p["b3"][:] = [0.5, -0.25]
    n.set(p, np.zeros(16, np.float32), np.ones(16, np.float32))
    q, _, _ = n.get()
    assert np.array_equal(q["b3"], p["b3"])
    x = rng.standard_normal((257, 16)).astype(np.float32)
    assert np.array_equal(n.forward(x), n.forward(x))
    n.close()


def test_gpu_mlp_training_fits_a_smooth_function():
    """Adam over a smooth two-output function of the 16 inputs: the loss falls by an order of magnitude, and the
    trained network's outputs still match the oracle's forward with the trained weights."""
    rng = np.random.default_rng(4)
    x = rng.standard_normal((20000, 16)).astype(np.float32)
    t = np.stack([np.tanh(x[:, 0] + 0.5 * x[:, 1]) + 0.1 * x[:, 2], np.maximum(x[:, 3], 0.0) - 0.3 * x[:, 4]], 1)
    t = t.astype(np.float32)
    n = net(11)
    before = float(np.mean(np.sum((n.forward(x) - t) ** 2, 1)))
    losses = n.train(x, t, epochs=8, batch=1024, lr=1e-3, seed=1)
    after = float(np.mean(np.sum((n.forward(x) - t) ** 2, 1)))
    assert losses[-1] < losses[0]
    assert after < 0.1 * before, (before, after, losses)
    p, mean, inv = n.get()
    want, _ = M.forward(p, (x[:2000] - mean) * inv)
    assert rel_err(n.forward(x[:2000]), want) < OUT_TOL
    n.close()
