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


def test_clumpy_plummer_family():
    p = W.clumpy_plummer(20000, 5)
    assert p.n == 20000 and np.allclose(p.mass, 1.0 / p.n)
    q = W.clumpy_plummer(20000, 5)
    assert np.array_equal(p.x, q.x)
    r = np.sqrt(p.x.astype(np.float64) ** 2 + p.y ** 2 + p.z ** 2)
    assert r.max() < 16.0
    # 30% of the particles sit in 32 small clumps: far denser cores than the host
    H, _ = np.histogramdd(np.stack([p.x, p.y, p.z], 1), bins=64, range=[(-4, 4)] * 3)
    assert H.max() > 20 * np.percentile(H[H > 0], 90)


def test_ensemble_family():
    counts, p, vx, vy, vz = W.ensemble(40, 3)
    assert len(counts) == 40 and p.n == counts.sum() == vx.size
    assert counts.min() >= 1024 and counts.max() <= 262144
    offs = np.concatenate([[0], np.cumsum(counts)])
    for k in range(40):
        a, b = offs[k], offs[k + 1]
        assert np.array_equal(p.id[a:b], np.arange(b - a, dtype=np.uint32))
        if k % 2 == 0:  # uniform cubes at rest
            assert np.all(np.abs(p.x[a:b]) <= 1.0) and not vx[a:b].any()
        else:           # Plummer spheres with velocities, mass 1/N
            assert np.allclose(p.mass[a:b], 1.0 / (b - a)) and vx[a:b].any()
    c2, p2, *_ = W.ensemble(40, 3)
    assert np.array_equal(c2, counts) and np.array_equal(p2.x, p.x)
