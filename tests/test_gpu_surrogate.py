"""The surrogate MLP's tensor-core kernels (include/cbm_surrogate.h): forward
pass and gradients against the CPU oracle (oracle/mlp_oracle.py, float64
with the same BF16 roundings), and training on the GPU that fits a smooth
map the untrained network does not."""
import os
import sys

import numpy as np
import pytest

import cbmtest

sys.path.insert(0, os.path.join(cbmtest.ROOT, "oracle"))
import mlp_oracle  # noqa: E402

pytestmark = pytest.mark.gpu

# tolerance of a GPU result against the oracle, norm-relative: one BF16 ulp
# (2^-8).  The oracle applies the same BF16 roundings at the same points, so
# what remains is FP32 accumulation in another order than float64 and the
# few roundings that this pushes across a BF16 tie; emulating that with
# float32 products in numpy gives at most 1.6e-4 (W1's gradient), 20 x below
# the bound.  A wrong tile, a dropped K chunk or a transposed operand is far
# above it.
REL_TOL = 2.0 ** -8


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _padded_x(x, I):
    out = np.zeros((x.shape[0], I), dtype=np.float32)
    out[:, :x.shape[1]] = x
    return out


@pytest.mark.parametrize("batch", [256, 200])
def test_forward_and_gradients_match_oracle(batch):
    from cerebellum_simulation_b200.surrogate import MLP
    rng = np.random.Generator(np.random.PCG64(3))
    net = MLP(64, 256, 256, 50, max_batch=256, seed=5)
    p = net.get_params()
    # non-zero biases exercise the bias paths
    W1, b1, W2, b2, W3, b3 = net.unpack(p)
    b1[:256] = rng.normal(0, 0.1, 256); b2[:256] = rng.normal(0, 0.1, 256); b3[:50] = rng.normal(0, 0.1, 50)
    net.set_params(p)
    x = rng.normal(0, 1, (batch, 64)).astype(np.float32)
    t = rng.normal(0, 1, (batch, 50)).astype(np.float32)
    params = net.unpack(net.get_params())
    I, H1, H2, O = net.padded
    _, _, _, y_ref = mlp_oracle.forward(params, _padded_x(x, I))
    y = net.forward(x)
    assert _rel(y, y_ref[:, :50]) < REL_TOL
    g, loss = net.gradients(x, t)
    t_pad = np.zeros((batch, O)); t_pad[:, :50] = t
    g_ref, loss_ref = mlp_oracle.gradients(params, _padded_x(x, I), t_pad, 50)
    assert abs(loss - loss_ref) / loss_ref < REL_TOL
    for name, a, b in zip(["W1", "b1", "W2", "b2", "W3", "b3"], net.unpack(g), g_ref):
        assert _rel(a, b) < REL_TOL, name
    # padding stays zero
    gW3 = net.unpack(g)[4]
    assert not gW3[50:].any()


def test_training_fits_a_smooth_map():
    """The trained network predicts a held-out smooth map of its input far
    better than the untrained one and than predicting the mean."""
    from cerebellum_simulation_b200.surrogate import MLP
    rng = np.random.Generator(np.random.PCG64(8))
    n = 4096
    x = rng.uniform(-1, 1, (n, 16)).astype(np.float32)
    proj = rng.normal(0, 1, (16, 50)) / 4
    t = np.tanh(x @ proj).astype(np.float32) + 0.5 * np.sin(3 * x[:, :1]).astype(np.float32)
    net = MLP(16, 128, 128, 50, max_batch=256, seed=1)
    x_tr, t_tr, x_te, t_te = x[:3584], t[:3584], x[3584:], t[3584:]
    before = float(np.mean((net.forward(x_te) - t_te) ** 2))
    net.train(x_tr, t_tr, batch=256, epochs=60, lr=2e-3, seed=2)
    after = float(np.mean((net.forward(x_te) - t_te) ** 2))
    mean_only = float(np.mean((t_tr.mean(0) - t_te) ** 2))
    assert after < 0.2 * mean_only and after < 0.1 * before, (before, after, mean_only)
