"""TEST INFRASTRUCTURE ONLY: FP64 restatement of the learned PPE warm start
network (fluidized_bed_master_b200/csrc/mlp_tcgen05.cuh) for gradient checks.

16 -> 64 -> 64 -> 1 MLP with ReLU.  The tensor-core kernels read BF16
operands, so this oracle rounds to BF16 (round to nearest even) at exactly
the points where the kernels do:
  * X, W1, W2, w3 (inputs / weights of the MMAs and of the last dot);
  * H1 = relu(X W1^T + b1) before the second MMA and the dW2 MMA;
  * delta2 before the D3 = delta2 W2 and the [dW2 | db2] MMAs;
  * delta1 before the [dW1 | db1] MMA.
Everything else (biases, masks, y, dL/dy, the w3 and b3 gradients) is FP32
in the kernels and FP64 here.  The network has no counterpart in the
reference (its PPE is one Jacobi sweep, functions_PPE2.cuh:542-698).
"""
import numpy as np

N_IN, N_H = 16, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_H * N_IN
OFF_W2 = OFF_B1 + N_H
OFF_B2 = OFF_W2 + N_H * N_H
OFF_W3 = OFF_B2 + N_H
OFF_B3 = OFF_W3 + N_H
N_PARAM = OFF_B3 + 1


def bf16(a):
    """Round to BF16 (nearest even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def bf16_bits(a):
    """BF16 bit patterns (uint16) of float values, nearest even."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    W1 = p[OFF_W1:OFF_B1].reshape(N_H, N_IN)
    b1 = p[OFF_B1:OFF_W2]
    W2 = p[OFF_W2:OFF_B2].reshape(N_H, N_H)
    b2 = p[OFF_B2:OFF_W3]
    w3 = p[OFF_W3:OFF_B3]
    b3 = p[OFF_B3]
    return W1, b1, W2, b2, w3, b3


def init_params(seed=0):
    """He-style initialisation used by the engine (same formula)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAM)
    p[OFF_W1:OFF_B1] = rng.standard_normal(N_H * N_IN) * np.sqrt(2.0 / N_IN)
    p[OFF_W2:OFF_B2] = rng.standard_normal(N_H * N_H) * np.sqrt(2.0 / N_H)
    p[OFF_W3:OFF_B3] = rng.standard_normal(N_H) * np.sqrt(1.0 / N_H)
    return p


def _ident(a):
    return np.asarray(a, dtype=np.float64)


def forward(params, x, rounding=True):
    """x: (n, 16) feature values (already BF16).  Returns y and the cache.
    rounding=False drops every BF16 rounding (pure FP64 network)."""
    r = bf16 if rounding else _ident
    W1, b1, W2, b2, w3, b3 = unpack(params)
    W1b, W2b, w3b = r(W1), r(W2), r(w3)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ W1b.T + b1
    h1 = r(np.maximum(z1, 0.0))
    z2 = h1 @ W2b.T + b2
    h2 = np.maximum(z2, 0.0)
    y = h2 @ w3b + b3
    return y, (x, z1, h1, z2, h2, W2b, w3b)


def grad(params, x, target, weight, weight_sum, rounding=True):
    """Gradient of L = sum w (y - t)^2 / weight_sum, flattened like the
    parameters, plus (sum w e^2, sum w)."""
    r = bf16 if rounding else _ident
    y, (x, z1, h1, z2, h2, W2b, w3b) = forward(params, x, rounding)
    w = np.asarray(weight, dtype=np.float64)
    e = y - np.asarray(target, dtype=np.float64)
    g3 = 2.0 * w * e / weight_sum
    d2 = np.where(h2 > 0, g3[:, None] * w3b[None, :], 0.0)
    d2b = r(d2)
    d3 = d2b @ W2b
    d1b = r(np.where(z1 > 0, d3, 0.0))
    g = np.zeros(N_PARAM)
    g[OFF_W1:OFF_B1] = (d1b.T @ x).ravel()
    g[OFF_B1:OFF_W2] = d1b.sum(0)
    g[OFF_W2:OFF_B2] = (d2b.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2b.sum(0)
    g[OFF_W3:OFF_B3] = (g3[:, None] * h2).sum(0)
    g[OFF_B3] = g3.sum()
    return g, float((w * e * e).sum()), float(w.sum())
