"""CPU oracle of the closure MLP (NumPy, FP64 accumulation with the GPU's bf16 roundings).

TEST INFRASTRUCTURE ONLY: ``tests/`` import it to check the forward and backward kernels of
``vlasov1d2v_b200`` (``vl_mlp_forward`` / ``vl_mlp_backward``); the product never imports it.

Network: x (96) -> 128 -> 128 -> 128 -> 48, GELU (erf form) on the three hidden layers.
The GPU rounds every matrix operand to bf16 (inputs, hidden activations, backpropagated
pre-activation gradients and the weights) and accumulates in FP32; this oracle applies the same
bf16 roundings and accumulates in FP64.  Weight matrices are [in][out], biases FP32.
"""
from __future__ import annotations

import math

import numpy as np

IN, HID, OUT = 96, 128, 48
DIMS = [(IN, HID), (HID, HID), (HID, HID), (HID, OUT)]


def bf16(x):
    """Round to bfloat16 (round to nearest, ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def forward(X, W, b, round_bf16=True):
    """Y and the saved (H_l, Z_l) of the network; W[l] [in][out] (already bf16 values)."""
    r = bf16 if round_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    H = [r(X)]
    Z = []
    h = H[0]
    for l in range(3):
        z = h @ W[l] + b[l]
        Z.append(z)
        h = r(gelu(z))
        H.append(h)
    Y = h @ W[3] + b[3]
    return Y, H, Z


def backward(Y, T, W, H, Z, nout, round_bf16=True):
    """Gradients (dW[l] [in][out], db[l]) of L = sum_{rows, c < nout} (Y - T)^2 / (rows nout)."""
    r = bf16 if round_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    n = Y.shape[0]
    dY = np.zeros_like(Y)
    dY[:, :nout] = 2.0 * (Y[:, :nout] - T[:, :nout]) / (n * nout)
    dz = r(dY.astype(np.float32))
    dW = [None] * 4
    db = [None] * 4
    for l in range(3, -1, -1):
        dW[l] = H[l].T @ dz
        db[l] = dz.sum(axis=0)
        if l > 0:
            dh = dz @ W[l].T
            dz = r((dh * gelu_d(Z[l - 1])).astype(np.float32))
    return dW, db


def loss(Y, T, nout):
    return float(np.mean((Y[:, :nout] - T[:, :nout]) ** 2))
