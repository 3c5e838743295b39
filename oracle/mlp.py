"""Numpy oracle of the learned-guess network -- TEST INFRASTRUCTURE ONLY.

Forward and backward of 64 -> 128 -> 128 -> 128 (ReLU) -> 1 in float64 with
the GPU kernels' rounding points: inputs, weights and the first two hidden
activations rounded to bfloat16 (round to nearest even), the third hidden
layer kept unrounded for the output dot product.  Loss: mean squared error.
Parameter order matches the flat vector of memphys_b200/csrc/mp_mlp.cuh.
"""
from __future__ import annotations

import numpy as np

IN, H = 64, 128
SIZES = [("W1", (IN, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
         ("b3", (H,)), ("w4", (H,)), ("b4", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(theta):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def forward(theta, X, rounding=True):
    p = unpack(theta)
    q = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    x = q(X)
    W1, W2, W3 = q(p["W1"]), q(p["W2"]), q(p["W3"])
    h1 = q(np.maximum(x @ W1 + p["b1"], 0.0))
    h2 = q(np.maximum(h1 @ W2 + p["b2"], 0.0))
    h3 = np.maximum(h2 @ W3 + p["b3"], 0.0)
    y = h3 @ p["w4"] + p["b4"][0]
    return y, (x, h1, h2, h3, W1, W2, W3)


def loss_grad(theta, X, t, rounding=True):
    """Mean squared error and its gradient w.r.t. the flat parameter vector (the
    gradient w.r.t. the rounded weights, as the GPU's straight-through update uses)."""
    p = unpack(theta)
    y, (x, h1, h2, h3, W1, W2, W3) = forward(theta, X, rounding)
    B = X.shape[0]
    dy = 2.0 * (y - t) / B
    g = {"w4": h3.T @ dy, "b4": np.array([dy.sum()])}
    d3 = np.outer(dy, p["w4"]) * (h3 > 0)
    g["W3"], g["b3"] = h2.T @ d3, d3.sum(0)
    d2 = (d3 @ W3.T) * (h2 > 0)
    g["W2"], g["b2"] = h1.T @ d2, d2.sum(0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    g["W1"], g["b1"] = x.T @ d1, d1.sum(0)
    flat = np.concatenate([g[name].ravel() for name, _ in SIZES])
    return float(np.mean((y - t) ** 2)), flat
