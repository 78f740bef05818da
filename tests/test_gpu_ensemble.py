"""The batched ensemble (ps_b200_ensemble_*), through the C ABI.

Many independent systems advanced together (every phase one launch over all
systems, replayed CUDA graphs) must give exactly what each system gives on
its own: the same sorted positions, ids, forces and velocities as
ps_b200_run_ticks per system with the same theta, leaf capacity and
expansion order, bit for bit.  The autotuner must leave the state
untouched and choose, per size class, a theta and leaf capacity whose error
meets its target."""

from __future__ import annotations

import numpy as np
import pytest

import polesitter_b200 as P
from polesitter_b200 import workloads as W

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "z", "mass", "fx", "fy", "fz")


class _D:
    pass


def _device(torch, p):
    d = _D()
    for k in KEYS:
        setattr(d, k, torch.from_numpy(getattr(p, k).copy()).cuda())
    d.id = torch.from_numpy(p.id.view(np.int32).copy()).cuda()
    return d


def _part(p, a, b):
    q = W.Particles(p.x[a:b].copy(), p.y[a:b].copy(), p.z[a:b].copy(), p.mass[a:b].copy(),
                    p.id[a:b].copy())
    return q


@pytest.mark.parametrize("caps,order", [(None, 0), ([1, 16, 32, 1, 64, 8, 2, 16, 16], 0),
                                        ([1, 16, 32, 1, 64, 8, 2, 16, 16], 1)],
                         ids=["leaf1", "mixed_leaf_caps", "mixed_leaf_caps_order1"])
def test_ensemble_equals_each_system_alone(caps, order):
    torch = pytest.importorskip("torch")
    counts, p, vx, vy, vz = W.ensemble(7, 3, n_min=64, n_max=40000)
    counts = np.concatenate([counts, [1, 2]])  # tiny systems too
    extra = W.uniform_cube(3, 77)
    p = W.Particles(np.concatenate([p.x, extra.x]), np.concatenate([p.y, extra.y]),
                    np.concatenate([p.z, extra.z]), np.concatenate([p.mass, extra.mass]),
                    np.concatenate([p.id, np.array([0, 0, 1], np.uint32)]))
    vx, vy, vz = (np.concatenate([v, np.zeros(3, np.float32)]) for v in (vx, vy, vz))
    theta = np.array([2.0, 1.0, 3.0, 2.0, 4.0, 1.5, 2.0, 2.0, 2.0], np.float32)
    offs = np.concatenate([[0], np.cumsum(counts)])
    d = _device(torch, p)
    v = [torch.from_numpy(a.copy()).cuda() for a in (vx, vy, vz)]
    codes = torch.zeros(p.n, dtype=torch.int32, device="cuda")
    with P.Ensemble(counts, theta) as ens:
        if caps is not None:
            ens.set_leaf_caps(caps)
            assert np.array_equal(ens.leaf_caps(), caps)
        ens.set_order(order)
        assert ens.order() == order
        ens.run(d, codes, *v, 1e-3, 3)
    torch.cuda.synchronize()
    for k in range(len(counts)):
        a, b = offs[k], offs[k + 1]
        q = _part(p, a, b)
        vk = [vx[a:b].copy(), vy[a:b].copy(), vz[a:b].copy()]
        with P.Context(int(b - a), theta=float(theta[k])) as ctx:
            if caps is not None:
                ctx.set_option(P.OPT_LEAF_CAP, caps[k])
            if order:
                ctx.set_closure(order)
            ctx.run_ticks(q, np.zeros(b - a, np.uint32), *vk, 1e-3, 3)
        for key in KEYS:
            assert np.array_equal(getattr(d, key)[a:b].cpu().numpy(), getattr(q, key)), (k, key)
        assert np.array_equal(d.id[a:b].cpu().numpy().view(np.uint32), q.id), k
        for c in range(3):
            assert np.array_equal(v[c][a:b].cpu().numpy(), vk[c]), (k, c)


def test_autotune_meets_target_and_leaves_state():
    torch = pytest.importorskip("torch")
    counts, p, vx, vy, vz = W.ensemble(6, 5, n_min=2048, n_max=30000)
    d = _device(torch, p)
    before = {k: getattr(d, k).clone() for k in ("x", "y", "z", "mass")}
    codes = torch.zeros(p.n, dtype=torch.int32, device="cuda")
    target = 3e-2
    with P.Ensemble(counts) as ens:
        theta, scale = ens.autotune(d, codes, target)
        caps = ens.leaf_caps()
        order = ens.order()
        assert order in (0, 1)
        assert set(caps.tolist()) <= {1, 16, 32, 64}
        assert np.array_equal(ens.theta(), theta)
        for k, v in before.items():
            assert torch.equal(getattr(d, k), v), k
        assert scale in (1.0, 0.5, 0.25)
        assert set(theta.tolist()) <= {1.0, 1.5, 2.0, 3.0, 4.0, 6.0, 8.0}
        v = [torch.from_numpy(a.copy()).cuda() for a in (vx, vy, vz)]
        ens.run(d, codes, *v, 1e-3, 1)
    torch.cuda.synchronize()
    # each tuned system meets the target on its first tick (FP64 check)
    offs = np.concatenate([[0], np.cumsum(counts)])
    for k in range(len(counts)):
        a, b = offs[k], offs[k + 1]
        q = _part(p, a, b)
        with P.Context(int(b - a), theta=float(theta[k])) as ctx:
            ctx.set_option(P.OPT_LEAF_CAP, int(caps[k]))
            if order:
                ctx.set_closure(order)
            ctx.tick(q, np.zeros(b - a, np.uint32))
            tg = np.arange(0, b - a, max(1, (b - a) // 512), dtype=np.uint32)
            f64 = ctx.direct_f64(q, tg)
        F = np.stack([q.fx, q.fy, q.fz], 1)[tg].astype(np.float64)
        err = np.median(np.linalg.norm(F - f64, axis=1) / np.linalg.norm(f64, axis=1))
        assert err <= 1.5 * target or theta[k] == 8.0, (k, theta[k], err)


def test_autotune_leaf_ladder_of_one_keeps_the_reference_tree():
    torch = pytest.importorskip("torch")
    counts, p, vx, vy, vz = W.ensemble(3, 6, n_min=2048, n_max=8000)
    d = _device(torch, p)
    codes = torch.zeros(p.n, dtype=torch.int32, device="cuda")
    with P.Ensemble(counts) as ens:
        ens.set_leaf_ladder([1])
        ens.autotune(d, codes, 3e-2)
        assert np.all(ens.leaf_caps() == 1)
        with pytest.raises(P.PolesitterError):
            ens.set_leaf_ladder([0])
        with pytest.raises(P.PolesitterError):
            ens.set_leaf_caps([16])  # one per system


def test_ensemble_rejects_host_arrays_and_wrong_sizes():
    counts, p, vx, vy, vz = W.ensemble(2, 9, n_min=100, n_max=200)
    with P.Ensemble(counts) as ens:
        with pytest.raises(P.PolesitterError) as e:
            ens.run(p, np.zeros(p.n, np.uint32), vx, vy, vz, 1e-3, 1)
        assert e.value.code == P.PS_EINVAL
    with pytest.raises(P.PolesitterError):
        P.Ensemble(np.array([10, 0]))
