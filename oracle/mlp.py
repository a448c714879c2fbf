"""FP64 numpy restatement of the learned-budget MLP (test infrastructure only).

The budget model has no counterpart in the reference (it is an addition of this
library), so this oracle is pinned by central finite differences of its own FP64
loss (tests/test_oracle_pin.py) rather than by reference outputs.

Model: input normalisation x -> (x - mean) * inv (FP32, as the device computes
it), then 256 -> 256 -> 256 -> 2 with exact GELU (x * Phi(x)); parameters
W1 b1 W2 b2 W3 b3 mean inv (W row-major [out, in]).  Loss: binary cross-entropy
with logits on both outputs, summed over the outputs and averaged over the batch.

With ``bf16_ops=True`` every GEMM operand is first rounded to float32 and then to
bfloat16 (round to nearest even), the way the device kernels stage their tiles;
biases and the elementwise steps stay unrounded.  Products and sums are FP64
here, FP32 on the device.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

SHAPES = [(256, 256), (256,), (256, 256), (256,), (2, 256), (2,), (256,), (256,)]


def bf16(x) -> np.ndarray:
    """float -> float32 -> bfloat16 (round to nearest even) -> float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def init_params(seed: int = 0):
    """Random weights and biases, and a non-trivial normalisation (test values)."""
    g = np.random.default_rng(seed)
    out = []
    for s in SHAPES[:6]:
        if len(s) == 2:
            out.append(g.uniform(-1, 1, s) / np.sqrt(s[1]))
        else:
            out.append(g.uniform(-0.1, 0.1, s))
    out.append(g.normal(0, 0.5, 256))
    out.append(g.uniform(0.5, 2.0, 256))
    return [np.asarray(p, np.float32) for p in out]


def normalize(X, mean, inv) -> np.ndarray:
    """(x - mean) * inv in IEEE FP32, one rounding per operation."""
    X = np.asarray(X, np.float32)
    return ((X - np.asarray(mean, np.float32)) * np.asarray(inv, np.float32)).astype(np.float32)


def _r(x, on):
    return bf16(x) if on else np.asarray(x, np.float64)


def forward(params, X, bf16_ops: bool = True):
    W1, b1, W2, b2, W3, b3 = [np.asarray(p, np.float64) for p in params[:6]]
    X = normalize(X, params[6], params[7]).astype(np.float64)
    z1 = _r(X, bf16_ops) @ _r(W1, bf16_ops).T + b1
    a1 = gelu(z1)
    z2 = _r(a1, bf16_ops) @ _r(W2, bf16_ops).T + b2
    a2 = gelu(z2)
    z3 = _r(a2, bf16_ops) @ _r(W3, bf16_ops).T + b3
    return z1, a1, z2, a2, z3


def loss_of(z3, Y):
    t = np.asarray(Y, np.float64)
    B = z3.shape[0]
    return float(np.sum(np.maximum(z3, 0) - z3 * t + np.log1p(np.exp(-np.abs(z3)))) / B)


def loss_and_grads(params, X, Y, bf16_ops: bool = True):
    """Mean BCE and its gradients (list in SHAPES order), mirroring the device backward."""
    W1, b1, W2, b2, W3, b3 = [np.asarray(p, np.float64) for p in params[:6]]
    z1, a1, z2, a2, z3 = forward(params, X, bf16_ops)
    X = normalize(X, params[6], params[7]).astype(np.float64)
    B = X.shape[0]
    t = np.asarray(Y, np.float64)
    g3 = (1.0 / (1.0 + np.exp(-z3)) - t) / B
    r = lambda x: _r(x, bf16_ops)  # noqa: E731
    dW3 = r(g3).T @ r(a2)
    db3 = g3.sum(0)
    g2 = (r(g3) @ r(W3)) * gelu_d(z2)
    dW2 = r(g2).T @ r(a1)
    db2 = g2.sum(0)
    g1 = (r(g2) @ r(W2)) * gelu_d(z1)
    dW1 = r(g1).T @ r(X)
    db1 = g1.sum(0)
    return loss_of(z3, Y), [dW1, db1, dW2, db2, dW3, db3]
