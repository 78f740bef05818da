"""The tick's failure paths, driven without a GPU fault.

* Bounded wait.  The radix sort's decoupled look-back polls a predecessor's
  flag a bounded number of times and raises PSG_ERR_SORT_SPIN instead of
  waiting for good.  PS_B200_OPT_SORT_SPIN lowers the limit to a few polls
  while the first tile of the first pass publishes ~200 us late, so the wait
  runs out: ps_calc_forces must return PS_EDEVICE (not hang), and the same
  context must then tick correctly with the normal limit.
* Capacity regrow.  The traversal's stores (near lists, P2P chunks, full-leaf
  records) raise a status bit when they run out; the host grows them and
  reruns the traversal in the same tick.  PS_B200_OPT_SHRINK_STORES shrinks
  them to their minimum so the next tick must take that path: it needs more
  than one traversal run, and its results equal those of a context whose
  stores were large from the start, bit for bit.

The reference has neither: it swallows an out-of-memory in the middle of its
tree build (polesitter.h:931-933)."""

from __future__ import annotations

import re

import numpy as np
import pytest

import polesitter_b200 as P
from polesitter_b200 import workloads as W
from test_gpu_parity import assert_forces_close, forces

pytestmark = pytest.mark.gpu


def test_sort_wait_runs_out_and_context_recovers(oracle):
    p0 = W.plummer(65536, 21)
    with P.Context(p0.n, theta=2.0) as ctx:
        ctx.set_option(P.OPT_SORT_SPIN, 4)
        p = p0.copy()
        with pytest.raises(P.PolesitterError) as e:
            ctx.tick(p, np.zeros(p.n, np.uint32))
        assert e.value.code == P.PS_EDEVICE
        m = re.search(r"device status error 0x([0-9a-f]+)", str(e.value))
        assert m and int(m.group(1), 16) & 0x1, str(e.value)  # PSG_ERR_SORT_SPIN
        ctx.set_option(P.OPT_SORT_SPIN, 0)
        a, b = p0.copy(), p0.copy()
        oracle.tick(a, theta=2.0)
        ctx.tick(b, np.zeros(b.n, np.uint32))
    assert np.array_equal(a.id, b.id)
    assert_forces_close(forces(b), forces(a))


@pytest.mark.parametrize("name,gen,theta,cap", [
    ("plummer65536", lambda: W.plummer(65536, 3), 2.0, 1),
    ("clumpy20000", lambda: W.clumpy_plummer(20000, 3), 2.0, 1),
    ("clumpy65536_b16", lambda: W.clumpy_plummer(65536, 6), 6.0, 16),
])
def test_stores_regrow_and_rerun_bit_equal(name, gen, theta, cap):
    p0 = gen()
    out = []
    for shrink in (False, True):
        with P.Context(p0.n, theta=theta) as ctx:
            if cap != 1:
                ctx.set_option(P.OPT_LEAF_CAP, cap)
            p = p0.copy()
            ctx.tick(p, np.zeros(p.n, np.uint32))  # grows the stores as needed
            if shrink:
                ctx.set_option(P.OPT_SHRINK_STORES, 1)
            p = p0.copy()
            ctx.tick(p, np.zeros(p.n, np.uint32))
            st = ctx.stats()
            out.append((p, st))
    (pa, sa), (pb, sb) = out
    assert sa["traversal_runs"] == 1
    assert sb["traversal_runs"] > 1
    assert sb["near_levels"] == 10 and sb["streamed"] == 0
    assert np.array_equal(pa.id, pb.id)
    for k in ("fx", "fy", "fz"):
        assert np.array_equal(getattr(pa, k), getattr(pb, k)), k
