"""CPU oracle of the proposal network (test infrastructure only).

The reference has no learned component, so this oracle follows the
library's own definition of the network: a 44 -> 256 -> 256 -> 44 ReLU
perceptron trained on masked binary cross-entropy with logits, whose GEMM
operands are bf16 (round to nearest even) with wide accumulation.  The
forward and backward passes here round at exactly the points the device
kernels round (inputs, weights, hidden activations, and the gradients that
feed GEMMs) and accumulate in float64, so the device results must agree up
to fp32 accumulation order and the occasional one-ulp bf16 rounding flip.
`skip` is the weight of the parameter-free residual path (logit += skip *
input of the same index).  `exact=True` turns every rounding off (plain float64 backpropagation),
which the tests check against finite differences.

Only tests import this module; the product path never does.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 44, 256, 44


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even); returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(x) -> np.ndarray:
    """bfloat16 bit patterns (uint16) of float values, nearest-even."""
    a = np.ascontiguousarray(bf16(x).astype(np.float32))
    return (a.view(np.uint32) >> 16).astype(np.uint16)


def _r(x, exact):
    return np.asarray(x, dtype=np.float64) if exact else bf16(x)


def forward(p: dict, x, exact: bool = False, skip: float = 0.0):
    """Logits (network output + skip * x) and the cached activations."""
    X = _r(x, exact)
    W1, W2, W3 = (_r(p[k], exact) for k in ("W1", "W2", "W3"))
    Z1 = X @ W1.T + p["b1"]
    H1 = _r(np.maximum(Z1, 0), exact)
    Z2 = H1 @ W2.T + p["b2"]
    H2 = _r(np.maximum(Z2, 0), exact)
    Z3 = H2 @ W3.T + p["b3"] + skip * np.asarray(x, dtype=np.float64)
    return Z3, dict(X=X, H1=H1, H2=H2, W2=W2, W3=W3)


def loss_and_grads(p: dict, x, t, mask, exact: bool = False, skip: float = 0.0):
    """Mean masked BCE-with-logits and its gradients (same keys as p)."""
    t = np.asarray(t, dtype=np.float64)
    m = np.asarray(mask, dtype=np.float64)
    cnt = m.sum()
    inv = 1.0 / cnt if cnt > 0 else 0.0
    Z3, c = forward(p, x, exact, skip)
    loss = float((m * (np.maximum(Z3, 0) - Z3 * t + np.log1p(np.exp(-np.abs(Z3))))).sum() * inv)
    s = 1.0 / (1.0 + np.exp(-Z3))
    dZ3 = _r((s - t) * m * inv, exact)
    g = {"W3": dZ3.T @ c["H2"], "b3": dZ3.sum(0)}
    dH2 = dZ3 @ c["W3"]
    dZ2 = _r(dH2 * (c["H2"] > 0), exact)
    g["W2"] = dZ2.T @ c["H1"]
    g["b2"] = dZ2.sum(0)
    dH1 = dZ2 @ c["W2"]
    dZ1 = _r(dH1 * (c["H1"] > 0), exact)
    g["W1"] = dZ1.T @ c["X"]
    g["b1"] = dZ1.sum(0)
    return loss, g


def init_params(seed: int = 0) -> dict:
    rng = np.random.default_rng(seed)

    def u(rows, cols):
        lim = np.sqrt(6.0 / cols)
        return rng.uniform(-lim, lim, (rows, cols)).astype(np.float32)

    return {"W1": u(HID, IN), "b1": rng.normal(0, 0.05, HID).astype(np.float32),
            "W2": u(HID, HID), "b2": rng.normal(0, 0.05, HID).astype(np.float32),
            "W3": u(OUT, HID), "b3": rng.normal(0, 0.05, OUT).astype(np.float32)}
