"""Train the learned far-field closure and write its weights.

    python -m polesitter_b200.train_closure --theta 6.5 --leaf-cap 16 \
        --out polesitter_b200/closure_weights.npz

Steps (all on the GPU through the library's C API):
  1. snapshots: ``--snapshots`` clumpy Plummer spheres of ``--n`` particles
     (workloads.clumpy_plummer: Plummer host + 32 sub-clumps holding 30% of
     the mass), each ticked once in closure mode 1 (order-1 local expansion)
     on a tree of leaf capacity ``--leaf-cap``;
  2. targets: for ``--samples`` particles per snapshot, the FP64 direct-sum
     force minus the order-1 force, in units of the correction's scale;
  3. Adam on the BF16 network with the library's training kernels;
  4. held-out check: ``--eval`` fresh snapshots ticked in mode 2; the median
     relative force error (FP64 judge sample) with and without the learned
     correction.
"""

from __future__ import annotations

import argparse
import time

import numpy as np

from . import Context, closure


def evaluate(ctx, params, n: int, theta: float, count: int, seed: int):
    from . import OPT_THETA
    from . import workloads as W
    ctx.closure_set_weights(params)
    ctx.set_option(OPT_THETA, theta)
    ctx.set_closure(2)
    base, mlp, used = [], [], 0
    codes = np.zeros(n, np.uint32)
    for k in range(count):
        p = W.clumpy_plummer(n, seed + k)
        ctx.tick(p, codes)
        j = ctx.closure_last()
        base.append(j["median_base"])
        mlp.append(j["median_mlp"])
        used += int(j["used"])
    return float(np.mean(base)), float(np.mean(mlp)), used


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--theta", type=float, default=6.5)
    ap.add_argument("--leaf-cap", type=int, default=1)
    ap.add_argument("--n", type=int, default=65536)
    ap.add_argument("--snapshots", type=int, default=2048)
    ap.add_argument("--samples", type=int, default=4096)
    ap.add_argument("--epochs", type=int, default=100)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--eval", type=int, default=16)
    ap.add_argument("--out", default=closure.default_weights_path())
    a = ap.parse_args(argv)
    with Context(a.n, theta=a.theta) as ctx:
        from . import OPT_LEAF_CAP
        ctx.set_option(OPT_LEAF_CAP, a.leaf_cap)
        t0 = time.time()
        x, t = closure.snapshot_dataset(ctx, a.snapshots, a.n, a.theta, a.samples, a.seed)
        t1 = time.time()
        print(f"dataset: {x.shape[0]} samples from {a.snapshots} snapshots in {t1 - t0:.1f} s",
              flush=True)
        params, losses = closure.train(ctx, x, t, epochs=a.epochs, batch=a.batch, lr=a.lr,
                                       seed=a.seed)
        t2 = time.time()
        print(f"training: {a.epochs} epochs in {t2 - t1:.1f} s, loss {losses[0]:.4f} -> "
              f"{losses[-1]:.4f}", flush=True)
        base, mlp, used = evaluate(ctx, params, a.n, a.theta, a.eval, 10_000_000 + a.seed)
        print(f"held-out ({a.eval} snapshots): median relative error {base:.3e} without, "
              f"{mlp:.3e} with the correction (applied on {used}/{a.eval})", flush=True)
    closure.save(a.out, params, theta=a.theta, leaf_cap=a.leaf_cap, n=a.n, snapshots=a.snapshots,
                 samples=a.samples, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed,
                 losses=losses, eval_median_base=base, eval_median_mlp=mlp)
    print(f"wrote {a.out}")


if __name__ == "__main__":
    main()
