"""Every theta the reference runs, through the C ABI.

The reference's pair recursion (polesitter.h:1050-1146, :1258-1494) needs no
storage that grows with theta.  The GPU tick keeps, per level, the near list
of every internal node (the sources it was not separated from), and spills
each leaf group's P2P source list; both grow roughly as theta^3.  When they
would not fit, the library stores near lists only down to a depth K and lets
each leaf group below walk its ancestor chain from K, summing its P2P as the
sources are found ("streamed").  The interaction set does not change.

The bar on small systems is the parity bar of test_gpu_parity.py: codes,
order, tree and multipoles bit-exact, every leaf's M2L and P2P pair counts
equal to the oracle's, forces within 1e-5 relative L2 and 1e-4 per particle.
The M2L pairs of internal nodes deeper than K are summed by each chain that
passes through them and are not stored per node, so their counts and local
fields are left out.  On the 1M clumpy snapshot the reference's tick takes
hours at theta 48, so there the bar is size-independent: every theta in
{16, 24, 32, 40, 48} returns PS_OK, its error against an FP64 direct sum falls
as theta grows, and at theta 12 the chain + stream tick equals the stored-list
tick (same P2P pair count, forces within 1e-5)."""

from __future__ import annotations

import numpy as np
import pytest

import polesitter_b200 as P
from conftest import rel_l2
from polesitter_b200 import workloads as W
from test_gpu_parity import FORCE_REL_L2, FORCE_REL_MAX, TOPO, assert_forces_close, forces

pytestmark = pytest.mark.gpu


def _tick(p, theta, near_levels=None, stream=False, leaf_cap=1, debug=True):
    with P.Context(p.n, theta=theta) as ctx:
        if debug:
            ctx.set_option(P.OPT_DEBUG, 1)
        if leaf_cap != 1:
            ctx.set_option(P.OPT_LEAF_CAP, leaf_cap)
        if near_levels is not None:
            ctx.set_option(P.OPT_NEAR_LEVELS, near_levels)
        if stream:
            ctx.set_option(P.OPT_STREAM, 1)
        codes = np.zeros(p.n, np.uint32)
        ctx.tick(p, codes)
        return {"codes": codes, "tree": ctx.tree() if debug else None, "stats": ctx.stats()}


# (name, particles, theta, near-list depth K (None: all), stream, leaf capacity)
CASES = [
    ("uniform4096_K4", lambda: W.uniform_cube(4096, 1), 2.0, 4, True, 1),
    ("plummer20000_t8_K5", lambda: W.plummer(20000, 4), 8.0, 5, True, 1),
    ("plummer20000_t8_stream", lambda: W.plummer(20000, 4), 8.0, None, True, 1),
    ("plummer65536_stream", lambda: W.plummer(65536, 3), 2.0, None, True, 1),
    # depth-10 leaves of hundreds of particles: the full-leaf variant streams
    ("clumpy20000_K6", lambda: W.clumpy_plummer(20000, 3), 2.0, 6, True, 1),
    ("clumpy20000_b16_t6_K5", lambda: W.clumpy_plummer(20000, 4), 6.0, 5, True, 16),
    ("clumpy20000_b64_t4_stream", lambda: W.clumpy_plummer(20000, 5), 4.0, None, True, 64),
    ("uniform3000_t24_K4", lambda: W.uniform_cube(3000, 8), 24.0, 4, True, 1),
    ("clumpy6000_t48_K5", lambda: W.clumpy_plummer(6000, 9), 48.0, 5, True, 1),
]


@pytest.mark.parametrize("name,gen,theta,K,stream,cap", CASES, ids=[c[0] for c in CASES])
def test_chain_and_stream_vs_oracle(oracle, name, gen, theta, K, stream, cap):
    p = gen()
    a, b = p.copy(), p.copy()
    ro = oracle.tick(a, theta=theta, leaf_cap=cap)
    rg = _tick(b, theta, near_levels=K, stream=stream, leaf_cap=cap)
    st = rg["stats"]
    assert st["streamed"] == (1 if stream else 0)
    kk = 10 if K is None else K
    # the shallow-leaf walk reads the lists of depths < its depth: K stays >= it - 1
    assert st["near_levels"] >= kk
    assert np.array_equal(rg["codes"], ro["codes"])
    assert np.array_equal(b.id, a.id)
    t, o = rg["tree"], ro["tree"]
    for k in TOPO + ("first_child", "parent"):
        assert np.array_equal(t[k], o[k]), k
    assert np.array_equal(t["geo"], o["geo"])
    assert np.array_equal(t["mp"], o["mp"])
    kept = (t["nchild"] == 0) | (t["depth"] <= st["near_levels"])
    assert np.array_equal(t["m2l_cnt"][kept], o["m2l_cnt"][kept])
    assert np.array_equal(t["p2p_cnt"], o["p2p_cnt"])
    assert st["p2p_pairs"] == ro["stats"]["p2p_pairs"]
    assert rel_l2(t["local_exp"][kept], o["l_tot"][kept]) < FORCE_REL_L2
    # leaf capacity > 1: a particle's P2P sum runs over thousands of sources,
    # summed in another order (the bar of test_leaf_capacity_vs_oracle)
    assert_forces_close(forces(b), forces(a), mx=FORCE_REL_MAX if cap == 1 else 1e-3)


def _median_error(ctx, p, k=1024, seed=5):
    rng = np.random.default_rng(seed)
    tg = np.sort(rng.choice(p.n, size=k, replace=False)).astype(np.uint32)
    ref = ctx.direct_f64(p, tg)
    got = forces(p)[tg]
    rel = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    return float(np.median(rel))


def test_clumpy_1m_every_theta():
    # the reference's own tree (leaf capacity 1) and far field; theta 16 and
    # up need more near-list entries than 32-bit offsets reach
    p0 = W.clumpy_plummer(1 << 20, 424242)
    errs = []
    with P.Context(p0.n, theta=16.0) as ctx:
        for theta in (16.0, 24.0, 32.0, 40.0, 48.0):
            ctx.set_option(P.OPT_THETA, theta)
            p = p0.copy()
            ctx.tick(p, np.zeros(p.n, np.uint32))  # raises unless PS_OK
            F = forces(p)
            assert np.isfinite(F).all()
            errs.append(_median_error(ctx, p))
            st = ctx.stats()
            print(f"theta {theta}: median rel error {errs[-1]:.3e}, near lists to depth "
                  f"{st['near_levels']}, streamed {st['streamed']}, runs {st['traversal_runs']}")
    assert errs[0] < 1e-2
    assert all(e1 < e0 for e0, e1 in zip(errs, errs[1:])), errs


def test_clumpy_1m_chain_equals_stored_lists():
    # theta 12 fits with every level's near lists: the chain + stream tick
    # must give the same interaction set and forces
    p0 = W.clumpy_plummer(1 << 20, 424242)
    a, b = p0.copy(), p0.copy()
    ra = _tick(a, 12.0, debug=True)
    rb = _tick(b, 12.0, near_levels=5, stream=True, debug=True)
    assert ra["stats"]["near_levels"] == 10 and ra["stats"]["streamed"] == 0
    assert rb["stats"]["near_levels"] == 5 and rb["stats"]["streamed"] == 1
    assert ra["stats"]["p2p_pairs"] == rb["stats"]["p2p_pairs"]
    assert ra["stats"]["p2p_interactions"] == rb["stats"]["p2p_interactions"]
    assert np.array_equal(a.id, b.id)
    assert_forces_close(forces(b), forces(a))
