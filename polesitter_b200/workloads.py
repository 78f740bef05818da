"""Seeded synthetic particle sets for the FMM tick.

The reference publishes no datasets; its own tests and benchmark draw
particles from seeded generators (tests/accuracy.c:33-40 LCG,
tests/benchmark.c:158-165 ``srand(7331)``).  These generators produce the
shapes the workloads are quoted on:

* ``uniform_cube``   - i.i.d. uniform positions in a cube, uniform masses
                       (N=1024 in [-1,1]^3, masses in [0.5,1.5]).
* ``plummer``        - an equal-mass Plummer sphere (scale radius ``a``,
                       radii truncated at ``rmax``), N=1,048,576 at scale.
* ``two_plummer``    - two Plummer spheres on a collision course with
                       velocities from the isotropic Plummer distribution
                       function (multi-tick workload).
* ``lcg_uniform`` / ``lcg_two_clusters`` - bit-exact restatements of the
                       reference accuracy test's LCG fills
                       (tests/accuracy.c:33-40, :111-137).

All arrays are float32 structure-of-arrays, matching ``ps_particle_arrs_t``
(polesitter.h:312-322).
"""

from __future__ import annotations

import numpy as np

__all__ = [
    "Particles",
    "uniform_cube",
    "plummer",
    "plummer_velocities",
    "two_plummer",
    "lcg_uniform",
    "lcg_two_clusters",
    "benchmark_cube",
]


class Particles:
    """Caller-owned SoA arrays (x, y, z, mass, fx, fy, fz, id)."""

    def __init__(self, x, y, z, mass, ids=None):
        n = len(x)
        self.x = np.ascontiguousarray(x, dtype=np.float32)
        self.y = np.ascontiguousarray(y, dtype=np.float32)
        self.z = np.ascontiguousarray(z, dtype=np.float32)
        self.mass = np.ascontiguousarray(mass, dtype=np.float32)
        self.fx = np.zeros(n, np.float32)
        self.fy = np.zeros(n, np.float32)
        self.fz = np.zeros(n, np.float32)
        self.id = (np.arange(n, dtype=np.uint32) if ids is None
                   else np.ascontiguousarray(ids, dtype=np.uint32))

    @property
    def n(self) -> int:
        return len(self.x)

    def copy(self) -> "Particles":
        p = Particles(self.x.copy(), self.y.copy(), self.z.copy(),
                      self.mass.copy(), self.id.copy())
        p.fx[:] = self.fx
        p.fy[:] = self.fy
        p.fz[:] = self.fz
        return p


def uniform_cube(n: int, seed: int, lo: float = -1.0, hi: float = 1.0,
                 mass_lo: float = 0.5, mass_hi: float = 1.5) -> Particles:
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = rng.uniform(lo, hi, size=(3, n)).astype(np.float32)
    m = rng.uniform(mass_lo, mass_hi, size=n).astype(np.float32)
    return Particles(pos[0], pos[1], pos[2], m)


def _plummer_radii(rng, n: int, a: float, rmax: float) -> np.ndarray:
    out = np.empty(0, np.float64)
    while out.size < n:
        u = rng.uniform(0.0, 1.0, size=max(1024, int((n - out.size) * 1.05)))
        u = u[u > 0.0]
        r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        out = np.concatenate([out, r[r <= rmax * a]])
    return out[:n]


def _isotropic(rng, n: int) -> np.ndarray:
    cz = rng.uniform(-1.0, 1.0, size=n)
    phi = rng.uniform(0.0, 2.0 * np.pi, size=n)
    s = np.sqrt(np.maximum(0.0, 1.0 - cz * cz))
    return np.stack([s * np.cos(phi), s * np.sin(phi), cz])


def plummer(n: int, seed: int, a: float = 1.0, rmax: float = 10.0,
            total_mass: float = 1.0, center=(0.0, 0.0, 0.0)) -> Particles:
    """Equal-mass Plummer sphere: r = a / sqrt(u^(-2/3) - 1), r <= rmax*a,
    isotropic directions, mass total_mass/n each."""
    rng = np.random.Generator(np.random.PCG64(seed))
    r = _plummer_radii(rng, n, a, rmax)
    d = _isotropic(rng, n)
    pos = d * r[None, :] + np.asarray(center, np.float64)[:, None]
    m = np.full(n, total_mass / n, np.float32)
    return Particles(pos[0].astype(np.float32), pos[1].astype(np.float32),
                     pos[2].astype(np.float32), m)


def plummer_velocities(rng, r: np.ndarray, a: float = 1.0,
                       total_mass: float = 1.0, g: float = 1.0) -> np.ndarray:
    """Isotropic Plummer distribution-function velocities (Aarseth, Henon and
    Wielen 1974 rejection: q in [0,1] with density q^2 (1-q^2)^3.5, speed
    v = q * v_esc(r))."""
    n = r.size
    q = np.empty(n, np.float64)
    filled = 0
    while filled < n:
        m = max(1024, (n - filled) * 12)
        x1 = rng.uniform(0.0, 1.0, size=m)
        x2 = rng.uniform(0.0, 0.1, size=m)
        ok = x2 < x1 * x1 * (1.0 - x1 * x1) ** 3.5
        take = x1[ok][: n - filled]
        q[filled: filled + take.size] = take
        filled += take.size
    vesc = np.sqrt(2.0 * g * total_mass) * (r * r + a * a) ** -0.25
    return _isotropic(rng, n) * (q * vesc)[None, :]


def two_plummer(n_total: int, seed: int, mass_ratio: float = 3.0,
                a: float = 1.0, rmax: float = 10.0, separation: float = 20.0,
                rel_velocity: float = 0.3):
    """Two Plummer spheres (particle counts proportional to mass, equal
    particle masses) with centres ``separation`` apart on the x axis and a
    relative velocity ``rel_velocity`` along x.  Returns (Particles, vx, vy, vz)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n1 = int(round(n_total * mass_ratio / (1.0 + mass_ratio)))
    n2 = n_total - n1
    m1, m2 = mass_ratio / (1.0 + mass_ratio), 1.0 / (1.0 + mass_ratio)
    xs, vs = [], []
    for cnt, mass, cx, vx in ((n1, m1, -separation * m2, rel_velocity * m2),
                              (n2, m2, separation * m1, -rel_velocity * m1)):
        r = _plummer_radii(rng, cnt, a, rmax)
        pos = _isotropic(rng, cnt) * r[None, :]
        vel = plummer_velocities(rng, r, a, mass)
        pos[0] += cx
        vel[0] += vx
        xs.append(pos)
        vs.append(vel)
    pos = np.concatenate(xs, axis=1).astype(np.float32)
    vel = np.concatenate(vs, axis=1).astype(np.float32)
    m = np.full(n_total, 1.0 / n_total, np.float32)
    return Particles(pos[0], pos[1], pos[2], m), vel[0].copy(), vel[1].copy(), vel[2].copy()


def clumpy_plummer(n: int, seed: int, n_clumps: int = 32, clump_fraction: float = 0.3,
                   a: float = 1.0, rmax: float = 10.0, clump_a=(0.02, 0.1)) -> Particles:
    """The learned closure's snapshot family: an equal-mass Plummer sphere
    (scale ``a``, radii truncated at ``rmax * a``) holding a fraction
    1 - ``clump_fraction`` of the particles, plus ``n_clumps`` small Plummer
    sub-clumps that share the rest equally.  Clump centres are drawn from the
    host sphere (within 5a), clump scale radii log-uniform in ``clump_a``
    (truncated at 10 clump radii).  Particle masses are all 1/n."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n_clumped = int(round(n * clump_fraction)) if n_clumps > 0 else 0
    per = np.full(n_clumps, n_clumped // max(n_clumps, 1), np.int64)
    per[: n_clumped - int(per.sum())] += 1
    n_host = n - int(per.sum())
    r = _plummer_radii(rng, n_host, a, rmax)
    parts = [_isotropic(rng, n_host) * r[None, :]]
    centres = _isotropic(rng, n_clumps) * _plummer_radii(rng, n_clumps, a, 5.0)[None, :]
    scales = np.exp(rng.uniform(np.log(clump_a[0]), np.log(clump_a[1]), size=n_clumps))
    for k in range(n_clumps):
        if per[k] == 0:
            continue
        rc = _plummer_radii(rng, int(per[k]), scales[k], 10.0)
        parts.append(_isotropic(rng, int(per[k])) * rc[None, :] + centres[:, k:k + 1])
    pos = np.concatenate(parts, axis=1).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    return Particles(pos[0], pos[1], pos[2], m)


def ensemble(n_systems: int, seed: int, n_min: int = 1024, n_max: int = 262144):
    """The batched-ensemble workload: ``n_systems`` independent systems with
    N drawn log-uniform in [n_min, n_max]; even-numbered ones uniform cubes
    ([-1, 1]^3, masses U[0.5, 1.5] / N, at rest), odd-numbered ones Plummer
    spheres with a in [0.5, 2] (masses 1/N, isotropic Plummer velocities).
    Returns (counts, Particles of all systems concatenated, vx, vy, vz)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=n_systems)).astype(np.int64)
    xs, vs, ms = [], [], []
    for k, n in enumerate(counts):
        sub = int(rng.integers(0, 2**31))
        if k % 2 == 0:
            p = uniform_cube(int(n), sub)
            pos = np.stack([p.x, p.y, p.z])
            m = (p.mass / np.float32(n)).astype(np.float32)
            vel = np.zeros((3, n), np.float64)
        else:
            r2 = np.random.Generator(np.random.PCG64(sub))
            a = r2.uniform(0.5, 2.0)
            r = _plummer_radii(r2, int(n), a, 10.0)
            pos = _isotropic(r2, int(n)) * r[None, :]
            vel = plummer_velocities(r2, r, a, 1.0)
            m = np.full(int(n), 1.0 / n, np.float32)
        xs.append(pos.astype(np.float32))
        vs.append(vel.astype(np.float32))
        ms.append(m)
    pos = np.concatenate(xs, axis=1)
    vel = np.concatenate(vs, axis=1)
    p = Particles(pos[0], pos[1], pos[2], np.concatenate(ms))
    p.id[:] = np.concatenate([np.arange(n, dtype=np.uint32) for n in counts])
    return counts, p, vel[0].copy(), vel[1].copy(), vel[2].copy()


def _lcg_stream(state: int, count: int) -> tuple[np.ndarray, int]:
    """``state = state*1664525 + 1013904223 (mod 2^32)`` (tests/accuracy.c:33-36),
    returned as float32 ``(state >> 8) / 16777215`` (accuracy.c:38-40)."""
    out = np.empty(count, np.float32)
    s = state
    for i in range(count):
        s = (s * 1664525 + 1013904223) & 0xFFFFFFFF
        out[i] = np.float32(s >> 8) / np.float32(16777215.0)
    return out, s


def lcg_uniform(n: int) -> Particles:
    """tests/accuracy.c:111-122: 100-wide cube centred on 0, mass in [0.5,2)."""
    u, _ = _lcg_stream(7331, 4 * n)
    u = u.reshape(n, 4)
    f = np.float32
    x = u[:, 0] * f(100.0) - f(50.0)
    y = u[:, 1] * f(100.0) - f(50.0)
    z = u[:, 2] * f(100.0) - f(50.0)
    m = f(0.5) + u[:, 3] * f(1.5)
    return Particles(x, y, z, m)


def lcg_two_clusters(n: int) -> Particles:
    """tests/accuracy.c:124-137: two 2-wide clusters at x = -12.75 / +12.75."""
    u, _ = _lcg_stream(20260803, 4 * n)
    u = u.reshape(n, 4)
    f = np.float32
    half = n // 2
    idx = np.arange(n)
    center = np.where(idx < half, f(-12.0), f(12.0)).astype(np.float32)
    skew = np.where(idx < half, f(-0.75), f(0.75)).astype(np.float32)
    x = (center + skew) + (u[:, 0] - f(0.5)) * f(2.0)
    y = (u[:, 1] - f(0.5)) * f(2.0)
    z = (u[:, 2] - f(0.5)) * f(2.0)
    m = f(0.5) + u[:, 3] * f(2.0)
    return Particles(x.astype(np.float32), y.astype(np.float32),
                     z.astype(np.float32), m.astype(np.float32))


def benchmark_cube(n: int, seed: int = 7331) -> Particles:
    """The reference benchmark's workload shape (tests/benchmark.c:158-165):
    uniform cube [0,100]^3, unit masses.  Seeded PCG64 stands in for libc
    ``rand()``."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = rng.uniform(0.0, 100.0, size=(3, n)).astype(np.float32)
    return Particles(pos[0], pos[1], pos[2], np.ones(n, np.float32))
