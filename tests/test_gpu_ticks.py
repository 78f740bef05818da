"""ps_b200_run_ticks: the caller's tick loop (README.md:65-111) on the device.

Checked through the C ABI: (1) one iteration equals ps_prepare_particles +
ps_calc_forces followed by the oracle's C update (velocity permutation
through ids, semi-implicit Euler) applied to the same forces, bit for bit;
(2) several iterations track the oracle's own loop (ids identical, positions
and velocities within the forces' rounding); (3) host and device arrays give
identical results; (4) massless particles keep their position."""

from __future__ import annotations

import numpy as np
import pytest

import polesitter_b200 as P
from polesitter_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _state(n, seed):
    p, vx, vy, vz = W.two_plummer(n, seed)
    return p, vx.astype(np.float32), vy.astype(np.float32), vz.astype(np.float32)


def test_one_iteration_is_calc_plus_the_c_update(oracle):
    p, vx, vy, vz = _state(30000, 5)
    dt = np.float32(1e-3)
    a = p.copy()
    va = [vx.copy(), vy.copy(), vz.copy()]
    with P.Context(p.n, theta=2.0) as ctx:
        codes = np.zeros(p.n, np.uint32)
        ctx.run_ticks(a, codes, *va, float(dt), 1)
        b = p.copy()
        b.id[:] = np.arange(p.n, dtype=np.uint32)
        codes_b = np.zeros(p.n, np.uint32)
        ctx.tick(b, codes_b)
    vb = [vx.copy(), vy.copy(), vz.copy()]
    oracle.euler_step(b, *vb, float(dt))
    assert np.array_equal(codes, codes_b)
    assert np.array_equal(a.id, b.id)
    for k in ("x", "y", "z", "mass", "fx", "fy", "fz"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    for u, w in zip(va, vb):
        assert np.array_equal(u, w)


def test_several_iterations_track_the_oracle_loop(oracle):
    p, vx, vy, vz = _state(20000, 7)
    a, b = p.copy(), p.copy()
    va = [vx.copy(), vy.copy(), vz.copy()]
    vb = [vx.copy(), vy.copy(), vz.copy()]
    with P.Context(p.n, theta=2.0) as ctx:
        codes = np.zeros(p.n, np.uint32)
        ctx.run_ticks(a, codes, *va, 1e-3, 5)
    oracle.run_ticks(b, *vb, 1e-3, 5, theta=2.0)
    assert np.array_equal(a.id, b.id)
    pos_a = np.stack([a.x, a.y, a.z], 1).astype(np.float64)
    pos_b = np.stack([b.x, b.y, b.z], 1).astype(np.float64)
    assert np.abs(pos_a - pos_b).max() <= 1e-6 * np.abs(pos_b).max()
    vel_a = np.stack(va, 1).astype(np.float64)
    vel_b = np.stack(vb, 1).astype(np.float64)
    assert np.linalg.norm(vel_a - vel_b) <= 1e-5 * np.linalg.norm(vel_b)


def test_host_and_device_arrays_agree():
    torch = pytest.importorskip("torch")
    p, vx, vy, vz = _state(12345, 9)
    host = p.copy()
    vh = [vx.copy(), vy.copy(), vz.copy()]
    with P.Context(p.n, theta=2.0) as ctx:
        ctx.run_ticks(host, np.zeros(p.n, np.uint32), *vh, 2e-3, 3)

        class D:
            pass
        d = D()
        for k in ("x", "y", "z", "mass", "fx", "fy", "fz"):
            setattr(d, k, torch.from_numpy(getattr(p, k).copy()).cuda())
        d.id = torch.from_numpy(p.id.view(np.int32).copy()).cuda()
        vd = [torch.from_numpy(v.copy()).cuda() for v in (vx, vy, vz)]
        codes = torch.zeros(p.n, dtype=torch.int32, device="cuda")
        ctx.run_ticks(d, codes, *vd, 2e-3, 3)
        torch.cuda.synchronize()
    for k in ("x", "y", "z", "mass", "fx", "fy", "fz"):
        assert np.array_equal(getattr(d, k).cpu().numpy(), getattr(host, k)), k
    assert np.array_equal(d.id.cpu().numpy().view(np.uint32), host.id)
    for u, w in zip(vd, vh):
        assert np.array_equal(u.cpu().numpy(), w)


def test_massless_particles_stay_and_zero_ticks_is_a_no_op():
    p, vx, vy, vz = _state(4096, 11)
    p.mass[::7] = 0.0
    start = p.copy()
    v0 = [vx.copy(), vy.copy(), vz.copy()]
    with P.Context(p.n, theta=2.0) as ctx:
        codes = np.zeros(p.n, np.uint32)
        ctx.run_ticks(p, codes, vx, vy, vz, 1e-2, 0)
        assert np.array_equal(p.x, start.x) and np.array_equal(vx, v0[0])
        ctx.run_ticks(p, codes, vx, vy, vz, 1e-2, 1)
    # ids map sorted slots to the original indices: massless ones did not move
    zero = p.mass == 0.0
    assert zero.any()
    orig = p.id[zero]
    assert np.array_equal(p.x[zero], start.x[orig])
    assert np.array_equal(vx[zero], v0[0][orig])
