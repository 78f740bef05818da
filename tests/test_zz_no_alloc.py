"""ps_b200_prepare_particles_noalloc, the allocation-free ps_prepare_particles.

It serves callers that cannot allocate device memory: engines that reserve
their memory up front and forbid allocation inside their frame loop, so that
no frame stalls on the allocator or fails for want of memory.  Its scratch is
one static device array shared by every call.  This file is collected last so
that a failure here leaves all other tests already run.

Checked through the C ABI against the regular entry point on two calls in a
row (the second smaller than the first, so leftovers of the first call in the
shared scratch would show), for each of the three Morton quantisation
variants, and once at exactly the largest count the scratch serves: Morton
codes are integer outputs and must match bit for bit, and so must the
bounding box."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import polesitter_b200 as P
from polesitter_b200 import workloads as W

pytestmark = pytest.mark.gpu


class _Dev:
    pass


def _device_arrays(torch, p):
    d = _Dev()
    for k in ("x", "y", "z", "mass", "fx", "fy", "fz"):
        setattr(d, k, torch.from_numpy(getattr(p, k).copy()).cuda())
    d.id = torch.from_numpy(p.id.view(np.int32).copy()).cuda()
    return d


def _noalloc(d, n, codes):
    arrs = P.arrs_of(d, n)
    mn, mx, rg = C.c_float(), C.c_float(), C.c_float()
    r = P.lib().ps_b200_prepare_particles_noalloc(C.byref(arrs), codes.data_ptr(), C.byref(mn),
                                                  C.byref(mx), C.byref(rg))
    return r, (mn.value, mx.value, rg.value)


def _check_same(torch, p):
    n = p.n
    d = _device_arrays(torch, p)
    want_codes = torch.zeros(n, dtype=torch.int32, device="cuda")
    want_box = P.prepare_particles(d, want_codes)
    got_codes = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    r, got_box = _noalloc(d, n, got_codes)
    torch.cuda.synchronize()
    assert r == P.PS_OK, P.lib().ps_b200_last_error()
    assert got_box == want_box
    assert torch.equal(got_codes, want_codes)


@pytest.mark.parametrize("variant", [P.MORTON_AVX2, P.MORTON_NEON, P.MORTON_SCALAR])
def test_noalloc_prepare_matches_regular_on_two_calls(variant):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    P.set_morton_variant(variant)
    try:
        for n, seed in ((1 << 20, 42), (5003, 7)):
            _check_same(torch, W.plummer(n, seed))
    finally:
        P.set_morton_variant(P.MORTON_AVX2)


def test_noalloc_prepare_at_its_largest_count():
    # 4,194,304 particles: every per-block slot of the scratch is used, and
    # the last one sits next to the final box
    torch = pytest.importorskip("torch")
    _check_same(torch, W.uniform_cube(4 * 1024 * 1024, 11))
    _check_same(torch, W.plummer(3000, 12))


def test_noalloc_rejects_what_it_cannot_serve():
    torch = pytest.importorskip("torch")
    n = 4 * 1024 * 1024 + 1
    d = _Dev()
    for k in ("x", "y", "z"):
        setattr(d, k, torch.zeros(n, dtype=torch.float32, device="cuda"))
    for k in ("mass", "fx", "fy", "fz", "id"):
        setattr(d, k, None)
    codes = torch.zeros(n, dtype=torch.int32, device="cuda")
    r, _ = _noalloc(d, n, codes)
    assert r == P.PS_EINVAL
    assert b"exceed" in P.lib().ps_b200_last_error()
    # host arrays would need device mirrors, i.e. an allocation
    p = W.uniform_cube(64, 1)
    host_codes = np.zeros(64, np.uint32)
    arrs = P.arrs_of(p)
    f = C.c_float()
    r = P.lib().ps_b200_prepare_particles_noalloc(C.byref(arrs), host_codes.ctypes.data,
                                                  C.byref(f), C.byref(f), C.byref(f))
    assert r == P.PS_EINVAL
