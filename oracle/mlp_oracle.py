"""CPU oracle of the closure network (test infrastructure only).

Float64 restatement of the 16 -> 64 -> 64 -> 4 SiLU network that
ultraballpit_b200/csrc/sph_mlp.cu trains, rounding to bfloat16 (nearest
even) at the same points as the tensor-core kernels: inputs, weights,
hidden activations, dL/dy and dL/dz before they enter a matrix product.
Used to check the device forward pass and gradients.
"""
from __future__ import annotations

import numpy as np

SHAPES = (("W1", (64, 16)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)), ("W3", (4, 64)), ("b3", (4,)))
N_PARAMS = 5508


def bf16(a) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + n], np.float64).reshape(shp)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p: np.ndarray, x: np.ndarray):
    w = unpack(p)
    xb = bf16(x)
    z1 = xb @ bf16(w["W1"]).T + w["b1"]
    h1 = bf16(silu(z1))
    z2 = h1 @ bf16(w["W2"]).T + w["b2"]
    h2 = bf16(silu(z2))
    y = h2 @ bf16(w["W3"]).T + w["b3"]
    return y, (xb, z1, h1, z2, h2)


def loss_grad(p: np.ndarray, x: np.ndarray, t: np.ndarray):
    """Mean squared error over n x 4 outputs and its gradient."""
    w = unpack(p)
    y, (xb, z1, h1, z2, h2) = forward(p, x)
    n = x.shape[0]
    err = y - t
    loss = float(np.mean(err * err))
    dy = bf16(2.0 * err / (n * 4))
    g = {}
    g["W3"] = dy.T @ h2
    g["b3"] = dy.sum(0)
    d2 = (dy @ bf16(w["W3"])) * silu_grad(z2)
    g["b2"] = d2.sum(0)
    d2b = bf16(d2)
    g["W2"] = d2b.T @ h1
    d1 = (d2b @ bf16(w["W2"])) * silu_grad(z1)
    g["b1"] = d1.sum(0)
    g["W1"] = bf16(d1).T @ xb
    return loss, pack(g)
