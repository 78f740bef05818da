"""Seeded workload generators: determinism and the shapes they promise."""

from __future__ import annotations

import numpy as np

from polesitter_b200 import workloads as W


def test_seeded_and_deterministic():
    a, b = W.plummer(5000, 7), W.plummer(5000, 7)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.mass, b.mass)
    assert not np.array_equal(a.x, W.plummer(5000, 8).x)


def test_plummer_shape():
    p = W.plummer(200000, 1, a=1.0, rmax=10.0)
    r = np.sqrt(p.x.astype(np.float64) ** 2 + p.y ** 2 + p.z ** 2)
    assert r.max() <= 10.0 + 1e-4
    # half-mass radius of a Plummer sphere ~1.305 a (slightly less when truncated)
    assert 1.2 < np.median(r) < 1.32
    assert np.allclose(p.mass, 1.0 / p.n)
    assert p.x.dtype == np.float32


def test_uniform_cube_bounds():
    p = W.uniform_cube(10000, 2)
    for v in (p.x, p.y, p.z):
        assert v.min() >= -1.0 and v.max() <= 1.0
    assert p.mass.min() >= 0.5 and p.mass.max() <= 1.5


def test_lcg_matches_reference_recurrence():
    # tests/accuracy.c:33-40 with state 7331 (fill_uniform, :111-122)
    s = 7331
    vals = []
    for _ in range(4):
        s = (s * 1664525 + 1013904223) & 0xFFFFFFFF
        vals.append(np.float32(s >> 8) / np.float32(16777215.0))
    p = W.lcg_uniform(1)
    assert p.x[0] == vals[0] * np.float32(100.0) - np.float32(50.0)
    assert p.mass[0] == np.float32(0.5) + vals[3] * np.float32(1.5)


def test_two_plummer_velocities():
    p, vx, vy, vz = W.two_plummer(40000, 3)
    assert p.n == 40000 and vx.shape == (40000,)
    n1 = 30000
    # the heavier sphere sits left, moving right; the lighter one the reverse
    assert p.x[:n1].mean() < 0 < p.x[n1:].mean()
    assert vx[:n1].mean() > 0 > vx[n1:].mean()
    # centre-of-mass momentum ~ 0
    assert abs(vx.mean()) < 0.01
