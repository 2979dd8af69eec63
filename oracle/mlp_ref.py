"""CPU reference of the term-priority network (FP64 numpy) — TEST INFRASTRUCTURE ONLY.

The network of ppvm_b200/csrc/mlp.cuh and learned.cu: y = w3 . gelu(W2 gelu(W1 x + b1) + b2)
+ b3 with the erf form of GELU; loss = mean((y - t)^2).  ``bf16`` rounds like the device
(round to nearest even on the top 16 bits of an IEEE float) so the tests can feed the
reference the same weights and inputs the tensor cores see.
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf

IN, H = 8, 64
SIZES = [("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("w3", (H,)), ("b3", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], dtype=np.float64).reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).reshape(-1) for name, _ in SIZES])


def bf16(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward(p, X, tc=False):
    """tc: round weights, inputs and the layer-1 activations to BF16 as the device does."""
    q = unpack(p)
    W1, W2 = (bf16(q["W1"]), bf16(q["W2"])) if tc else (q["W1"], q["W2"])
    X = bf16(X) if tc else np.asarray(X, dtype=np.float64)
    Z1 = X @ W1.T + q["b1"]
    H1 = gelu(Z1)
    Z2 = (bf16(H1) if tc else H1) @ W2.T + q["b2"]
    H2 = gelu(Z2)
    return H2 @ q["w3"] + q["b3"][0], (X, Z1, H1, Z2, H2)


def loss_and_grad(p, X, t, tc=False):
    q = unpack(p)
    y, (Xr, Z1, H1, Z2, H2) = forward(p, X, tc)
    n = len(t)
    e = y - np.asarray(t, dtype=np.float64)
    dy = 2.0 * e / n
    g = {"w3": H2.T @ dy, "b3": np.array([dy.sum()])}
    dZ2 = np.outer(dy, q["w3"]) * gelu_grad(Z2)
    W2 = bf16(q["W2"]) if tc else q["W2"]
    g["W2"] = dZ2.T @ H1
    g["b2"] = dZ2.sum(0)
    dZ1 = (dZ2 @ W2) * gelu_grad(Z1)
    g["W1"] = dZ1.T @ Xr
    g["b1"] = dZ1.sum(0)
    return float(np.mean(e * e)), pack(g)
