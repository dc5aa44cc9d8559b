"""Test infrastructure: CPU oracle of the surrogate MLP's forward pass and
gradients (include/cbm_surrogate.h), in float64 with the BF16 roundings the
GPU kernels apply at the same points: the weights and the input before the
products, every hidden activation after its ReLU, and the output gradient
before the weight-gradient products.  Only tests import it."""
import numpy as np


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (r.astype(np.uint32)).view(np.float32).astype(np.float64)


def forward(params, x):
    """params: (W1, b1, W2, b2, W3, b3) padded; x: [B, I] padded input."""
    W1, b1, W2, b2, W3, b3 = [np.asarray(p, dtype=np.float64) for p in params]
    xb = bf16(x)
    h1 = bf16(np.maximum(xb @ bf16(W1).T + b1, 0.0))
    h2 = bf16(np.maximum(h1 @ bf16(W2).T + b2, 0.0))
    y = h2 @ bf16(W3).T + b3
    return xb, h1, h2, y


def gradients(params, x, t, n_out):
    """Gradients of mean((y - t)^2) over the first n_out output columns."""
    W1, b1, W2, b2, W3, b3 = [np.asarray(p, dtype=np.float64) for p in params]
    xb, h1, h2, y = forward(params, x)
    B, O = y.shape
    mask = np.zeros(O)
    mask[:n_out] = 1.0
    dy = 2.0 * (y - t) * mask / (B * n_out)
    loss = float(np.sum(((y - t) * mask) ** 2) / (B * n_out))
    dyb = bf16(dy)
    gW3 = dyb.T @ h2
    gb3 = dy.sum(0)
    dh2 = (dyb @ bf16(W3)) * (h2 > 0)
    dh2b = bf16(dh2)
    gW2 = dh2b.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2b @ bf16(W2)) * (h1 > 0)
    dh1b = bf16(dh1)
    gW1 = dh1b.T @ xb
    gb1 = dh1.sum(0)
    return (gW1, gb1, gW2, gb2, gW3, gb3), loss
