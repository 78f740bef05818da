"""The learned far-field closure: training data, training and weights.

The closure (no counterpart in the reference) runs inside the tick: with
``Context.set_closure(2)`` every tick evaluates the order-1 local expansion,
then an MLP correction per particle, then the sampled FP64 judge that keeps
the correction only when it lowers the median relative force error.  This
module produces the network's weights the way the method itself defines
them: residuals between FP64 direct sums and the order-1 FMM on generated
snapshots (``workloads.clumpy_plummer``), fitted on the GPU by the library's
own training kernels (``ps_b200_closure_train``).
"""

from __future__ import annotations

import os

import numpy as np

from . import workloads as W

N_PARAMS = 9928
OUT_SCALE = 0.01           # dF = m s OUT_SCALE y
TARGET_CLIP = 20.0         # |target| bound in units of OUT_SCALE * m * s
HERE = os.path.dirname(os.path.abspath(__file__))

_SHAPES = [("W1", (16, 64)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)),
           ("W3", (64, 64)), ("b3", (64,)), ("W4", (64, 8)), ("b4", (8,))]


def init_params(seed: int = 0) -> np.ndarray:
    """Glorot-uniform weights over the used inputs (13) and outputs (3), the
    last layer scaled by 0.1; padding rows/columns and biases zero."""
    rng = np.random.Generator(np.random.PCG64(seed))
    parts = []
    for name, shape in _SHAPES:
        a = np.zeros(shape, np.float32)
        if name.startswith("W"):
            fan_in = 13 if name == "W1" else 64
            fan_out = 3 if name == "W4" else 64
            lim = np.sqrt(6.0 / (fan_in + fan_out)) * (0.1 if name == "W4" else 1.0)
            a[:fan_in, :fan_out] = rng.uniform(-lim, lim, size=(fan_in, fan_out))
        parts.append(a.ravel())
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == N_PARAMS
    return p


def snapshot_dataset(ctx, n_snapshots: int, n: int, theta: float, samples: int, seed: int,
                     n_clumps: int = 32, clump_fraction: float = 0.3):
    """Training pairs from ``n_snapshots`` clumpy Plummer snapshots of ``n``
    particles: for ``samples`` particles of each, the network input x (16)
    and the target (F_fp64 - F_order1) / (m s OUT_SCALE) (3), clipped to
    +-TARGET_CLIP.  ``ctx`` must hold at least ``n`` particles; it is left in
    closure mode 1 at ``theta``."""
    from . import OPT_THETA
    ctx.set_option(OPT_THETA, theta)
    ctx.set_closure(1)
    xs, ts = [], []
    codes = np.zeros(n, np.uint32)
    for k in range(n_snapshots):
        p = W.clumpy_plummer(n, seed + k, n_clumps=n_clumps, clump_fraction=clump_fraction)
        ctx.tick(p, codes)
        rng = np.random.Generator(np.random.PCG64(seed + k + 7_000_003))
        idx = np.sort(rng.choice(n, size=min(samples, n), replace=False)).astype(np.uint32)
        x, scale = ctx.closure_features(idx)
        f64 = ctx.direct_f64(p, idx)
        fb = np.stack([p.fx, p.fy, p.fz], 1)[idx].astype(np.float64)
        t = (f64 - fb) / np.maximum(scale.astype(np.float64), 1e-37)[:, None]
        xs.append(x)
        ts.append(np.clip(t, -TARGET_CLIP, TARGET_CLIP).astype(np.float32))
    return np.concatenate(xs), np.concatenate(ts)


def train(ctx, x, t, params=None, epochs: int = 30, batch: int = 4096, lr: float = 2e-3,
          seed: int = 0):
    """Adam on the GPU (ps_b200_closure_train); returns (params, losses)."""
    p0 = init_params(seed) if params is None else np.asarray(params, np.float32)
    return ctx.closure_train(x, t, p0, epochs, batch, lr, seed)


def save(path: str, params, **meta) -> None:
    np.savez_compressed(path, params=np.asarray(params, np.float32),
                        **{k: np.asarray(v) for k, v in meta.items()})


def load(path: str):
    d = np.load(path)
    meta = {k: d[k].item() if d[k].ndim == 0 else d[k] for k in d.files if k != "params"}
    return d["params"].astype(np.float32), meta


def default_weights_path() -> str:
    """The shipped weights, trained by ``python -m polesitter_b200.train_closure``."""
    return os.path.join(HERE, "closure_weights.npz")
