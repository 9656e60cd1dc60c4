"""The learned warm start's network on the tensor cores: forward outputs and gradients against the float64 oracle
(oracle/mlp.py, which rounds to BF16 where the kernels do), and training that lowers the loss."""
import numpy as np
import pytest

from oracle import mlp as M

pytestmark = pytest.mark.gpu

# The oracle rounds to BF16 exactly where the kernels do (weights, inputs, hidden activations, deltas), so the two
# differ only by FP32 against float64 accumulation and by the SiLU's exponential (expf against exp). Either can move
# an activation across a BF16 rounding boundary, which changes it by one BF16 step (2^-8 relative) and its
# descendants by less. So the largest difference is held to 0.5% of a block's scale, and the typical one (the
# median) to 1e-4 of it: a product laid out wrong (a K-chunk or a row block misplaced) moves most elements, and
# fails the median however small its effect on the largest.
OUT_TOL = 5e-3     # forward, largest difference: relative to the outputs' scale
GRAD_TOL = 5e-3    # gradients, largest difference: relative to each gradient block's scale
TYPICAL_TOL = 1e-4  # median difference, relative to the scale


def net(seed=0):
    from vxr.learned import Mlp
    return Mlp(seed=seed)


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-12))


def typical_err(a, b):
    return float(np.median(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-12))


def test_gpu_mlp_forward_matches_the_oracle():
    """1,000 rows (a ragged last tile) through the GPU's weights: the same outputs as the oracle's forward."""
    rng = np.random.default_rng(1)
    n = net(3)
    x = rng.standard_normal((1000, 16)).astype(np.float32)
    y = n.forward(x)
    p, mean, inv = n.get()
    want, _ = M.forward(p, (x - mean) * inv)
    assert rel_err(y, want) < OUT_TOL, rel_err(y, want)
    assert typical_err(y, want) < TYPICAL_TOL, typical_err(y, want)
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
        assert rel_err(g[k], want[k]) < GRAD_TOL, (k, rel_err(g[k], want[k]))
        assert typical_err(g[k], want[k]) < TYPICAL_TOL, (k, typical_err(g[k], want[k]))
    assert abs(loss - want_loss) / want_loss < 1e-3
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
    got = n.forward(x[:2000])
    assert rel_err(got, want) < OUT_TOL, rel_err(got, want)
    assert typical_err(got, want) < TYPICAL_TOL, typical_err(got, want)
    n.close()
