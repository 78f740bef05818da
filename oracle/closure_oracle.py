"""ORACLE (test infrastructure, not product): numpy restatement of the learned
far-field closure's network math, the checker for the GPU kernels in
polesitter_b200/csrc/k_closure.cu.

The closure has no counterpart in the reference, so this restates the
library's own definition (include/polesitter_b200.h, "learned far-field
closure"):

* features of a particle from its leaf's raw order-1 quantities (the C
  oracle's ``feat`` output of ``pso_set_closure``): s = |L| + h |G|_F and
  x = (L / s, G h / s, (x_i - c) / h, depth / 10, 0, 0, 0), scale m s / 100;
* the network 16 -> 64 -> 64 -> 64 -> 8 with GELU (tanh form), weights and
  hidden activations rounded to BF16 (round to nearest even) where the GPU
  rounds them, everything else in float64;
* the training loss (mean squared error over outputs 0..2) and its exact
  gradient by backpropagation.

Only tests/ import this module.
"""

from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 16, 64, 8
OUT_USED = 3
OUT_SCALE = 0.01

_SHAPES = [("W1", (N_IN, N_HID)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
           ("W3", (N_HID, N_HID)), ("b3", (N_HID,)), ("W4", (N_HID, N_OUT)), ("b4", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in _SHAPES)


def unpack(params):
    out, o = {}, 0
    for name, shape in _SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(params[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def pack(parts) -> np.ndarray:
    return np.concatenate([np.asarray(parts[name], np.float64).ravel() for name, _ in _SHAPES])


def bf16(a):
    """float32 -> bfloat16 -> float, round to nearest even (finite inputs)."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    u = np.sqrt(2.0 / np.pi) * (z + 0.044715 * z ** 3)
    return 0.5 * z * (1.0 + np.tanh(u))


def gelu_grad(z):
    u = np.sqrt(2.0 / np.pi) * (z + 0.044715 * z ** 3)
    th = np.tanh(u)
    return 0.5 * (1.0 + th) + 0.5 * z * (1.0 - th * th) * np.sqrt(2.0 / np.pi) * (
        1.0 + 3.0 * 0.044715 * z * z)


def features_from_raw(raw):
    """raw (n x 16): L(3), G(6: xx yy zz xy xz yz), x - c (3), h, depth, m, 0."""
    r = np.asarray(raw, np.float64)
    L, G, u = r[:, 0:3], r[:, 3:9], r[:, 9:12]
    h, depth, m = r[:, 12:13], r[:, 13:14], r[:, 14:15]
    gn = np.sqrt((G[:, :3] ** 2).sum(1) + 2.0 * (G[:, 3:] ** 2).sum(1))[:, None]
    s = np.linalg.norm(L, axis=1, keepdims=True) + h * gn + 1e-30
    x = np.zeros((r.shape[0], N_IN))
    x[:, 0:3] = L / s
    x[:, 3:9] = G * h / s
    x[:, 9:12] = u / h
    x[:, 12] = 0.1 * depth[:, 0]
    return x, (m * s * OUT_SCALE)[:, 0]


def forward(params, x):
    """Network outputs (n x 8) and the cache the backward pass needs."""
    P = unpack(params)
    h0 = bf16(x)
    z1 = h0 @ bf16(P["W1"]) + P["b1"]
    h1 = bf16(gelu(z1))
    z2 = h1 @ bf16(P["W2"]) + P["b2"]
    h2 = bf16(gelu(z2))
    z3 = h2 @ bf16(P["W3"]) + P["b3"]
    h3 = bf16(gelu(z3))
    y = h3 @ bf16(P["W4"]) + P["b4"]
    return y, (h0, z1, h1, z2, h2, z3, h3)


def loss_and_grad(params, x, t):
    """Mean squared error over outputs 0..2 and its gradient (parameter
    layout), as one training step on one batch computes them."""
    P = unpack(params)
    y, (h0, z1, h1, z2, h2, z3, h3) = forward(params, x)
    n = x.shape[0]
    e = y[:, :OUT_USED] - np.asarray(t, np.float64)
    loss = float((e * e).sum() / (OUT_USED * n))
    dy = np.zeros_like(y)
    dy[:, :OUT_USED] = 2.0 * e / (OUT_USED * n)
    g = {"W4": h3.T @ dy, "b4": dy.sum(0)}
    d3 = (dy @ bf16(P["W4"]).T) * gelu_grad(z3)
    g["W3"], g["b3"] = h2.T @ d3, d3.sum(0)
    d2 = (d3 @ bf16(P["W3"]).T) * gelu_grad(z2)
    g["W2"], g["b2"] = h1.T @ d2, d2.sum(0)
    d1 = (d2 @ bf16(P["W2"]).T) * gelu_grad(z1)
    g["W1"], g["b1"] = h0.T @ d1, d1.sum(0)
    return loss, pack(g)
