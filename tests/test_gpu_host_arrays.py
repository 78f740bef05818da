"""Host arrays through the C ABI give the same tick as device arrays.

With pinned host buffers, ps_calc_forces copies the sorted positions,
masses, ids and codes back on a stream of their own while the traversal
runs, and only the forces at the end; pageable buffers are copied back at
the end.  Either way the caller's arrays must hold exactly what device
arrays hold after the same tick."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import polesitter_b200 as P
from polesitter_b200 import closure as CL
from polesitter_b200 import workloads as W

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "mass", "fx", "fy", "fz")


class Arrays:
    pass


def _arrays(p, kind):
    a = Arrays()
    if kind == "device":
        dev = torch.device("cuda", 0)
        for k in FIELDS:
            setattr(a, k, torch.from_numpy(getattr(p, k).copy()).to(dev))
        a.id = torch.from_numpy(p.id.view(np.int32).copy()).to(dev)
        codes = torch.zeros(p.n, dtype=torch.int32, device=dev)
    elif kind == "pinned":
        for k in FIELDS:
            t = torch.empty(p.n, dtype=torch.float32, pin_memory=True)
            t.numpy()[:] = getattr(p, k)
            setattr(a, k, t.numpy())
        t = torch.empty(p.n, dtype=torch.int32, pin_memory=True)
        t.numpy()[:] = p.id.view(np.int32)
        a.id = t.numpy().view(np.uint32)
        codes = torch.zeros(p.n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    else:
        for k in FIELDS:
            setattr(a, k, getattr(p, k).copy())
        a.id = p.id.copy()
        codes = np.zeros(p.n, np.uint32)
    return a, codes


def _host(v):
    if isinstance(v, torch.Tensor):
        return v.cpu().numpy().view(np.uint32 if v.dtype == torch.int32 else np.float32)
    return np.asarray(v).view(np.uint32 if v.dtype in (np.int32, np.uint32) else np.float32)


def _tick(p, kind, theta, closure):
    a, codes = _arrays(p, kind)
    with P.Context(p.n, theta=theta) as ctx:
        if closure:
            ctx.set_option(P.OPT_LEAF_CAP, 16)
            ctx.closure_set_weights(CL.load(CL.default_weights_path())[0])
            ctx.set_closure(2)
        for _ in range(2):  # two ticks in a row: the second starts from sorted input
            ctx.tick(a, codes)
    out = {k: _host(getattr(a, k)) for k in FIELDS}
    out["id"] = _host(a.id)
    out["codes"] = _host(codes)
    return out


@pytest.mark.parametrize("closure", [False, True], ids=["plain", "closure"])
def test_pinned_and_pageable_host_arrays_equal_device_arrays(closure):
    p = W.clumpy_plummer(200_000, 31) if closure else W.plummer(200_000, 30)
    theta = 6.25 if closure else 2.0
    ref = _tick(p, "device", theta, closure)
    for kind in ("pinned", "pageable"):
        got = _tick(p, kind, theta, closure)
        for k in ref:
            assert np.array_equal(got[k], ref[k]), (kind, k)
