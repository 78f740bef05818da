"""The oracle (oracle/ps_oracle.c) against the reference's own known answers,
the golden fixtures made by the reference, and -- where the checker's build of
the reference exists -- the reference itself, live.

Known answers restated from the reference's tests (tests/main.c:50-476,
tests/accuracy.c:74-109, :427-568)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_names, golden_particles, load_golden, rel_l2
from polesitter_b200 import workloads as W

THETA_SQRT12 = 3.4641  # tests/main.c:11


# ---- known answers of tests/main.c ------------------------------------------

def test_morton_bit_positions(oracle):
    # tests/main.c:50-72
    assert oracle.morton_encode(1, 0, 0) == 1
    assert oracle.morton_encode(0, 1, 0) == 2
    assert oracle.morton_encode(0, 0, 1) == 4
    assert oracle.morton_encode(3, 0, 0) == 9
    assert oracle.morton_encode(1023, 1023, 1023) == (1 << 30) - 1


def test_radix_sort_co_sorts(oracle):
    # tests/main.c:192-233
    p = W.Particles([9, 1, 5, 4], [9, 1, 5, 4], [9, 1, 5, 4], [9, 1, 5, 4])
    codes = np.array([999, 10, 500, 42], np.uint32)
    oracle.sort(p, codes)
    assert codes.tolist() == [10, 42, 500, 999]
    assert p.mass.tolist() == [1.0, 4.0, 5.0, 9.0]
    assert p.id.tolist() == [1, 3, 2, 0]


def test_octree_two_corner_particles(oracle):
    # tests/main.c:125-190: codes of (0,0,0) and (1023,1023,1023) end in the
    # leaves down child 0 and child 7, one particle each
    lo, hi = oracle.morton_encode(0, 0, 0), oracle.morton_encode(1023, 1023, 1023)
    p = W.Particles([0, 1], [0, 1], [0, 1], [1, 1])
    r = oracle.calc(p, np.array([lo, hi], np.uint32), 0.0, 0.0, 0.0, 10.0, THETA_SQRT12)
    t = r["tree"]
    assert t["nchild"][0] == 2 and t["leaf"][0] == 0
    kids = t["first_child"][0] + np.arange(2)
    assert t["octant"][kids].tolist() == [0, 7]
    assert t["leaf"][kids].tolist() == [1, 1]
    assert t["count"][kids].tolist() == [1, 1]
    assert t["start"][kids].tolist() == [0, 1]


def test_p2m(oracle):
    # tests/main.c:235-280
    mp = oracle.p2m([2.0, -1.0], [3.0, -2.0], [4.0, -3.0], [2.0, 3.0])
    np.testing.assert_allclose(mp, [5.0, 1.0, 0.0, -1.0], atol=1e-4)


def test_m2l_field(oracle):
    # tests/main.c:282-323: unit mass at (10,10,10) from the target
    hit, loc = oracle.m2l_pair([-5, -5, -5, 1], [5, 5, 5, 1], [1, 0, 0, 0], THETA_SQRT12)
    assert hit
    np.testing.assert_allclose(loc[1:], [0.00192354] * 3, atol=1e-6)


def test_m2l_dipole_orientation(oracle):
    # tests/accuracy.c:74-109
    hit, loc = oracle.m2l_pair([0, 0, 0, 1], [100, 0, 0, 1], [1, 1, 0, 0], 2.0)
    assert hit
    assert abs(float(loc[1]) - 0.00009799856) <= 5e-9


def test_mac_not_separated_is_not_applied(oracle):
    hit, loc = oracle.m2l_pair([0, 0, 0, 1], [3, 0, 0, 1], [1, 0, 0, 0], 2.0)
    assert not hit and not loc.any()


def test_p2p_pair_force(oracle):
    # tests/main.c:427-476: two particles one unit apart
    p = W.Particles([0.0, 1.0], [0.0, 0.0], [0.0, 0.0], [2.0, 3.0])
    oracle.p2p_pair(p, 0, 2, 0, 2)
    expected = (2.0 * 3.0) * 1.1 ** -1.5
    assert abs(p.fx[0] - expected) < 1e-4 and abs(p.fx[1] + expected) < 1e-4
    assert abs(p.fy).max() < 1e-6 and abs(p.fz).max() < 1e-6


@pytest.mark.parametrize("fill,name", [(W.lcg_uniform, "uniform-512"),
                                       (W.lcg_two_clusters, "two-clusters-512")])
def test_accuracy_gate(oracle, fill, name):
    # tests/accuracy.c:427-568: RMS relative error vs the FP64 direct sum < 0.10
    p = fill(512)
    ref_in = p.copy()
    oracle.tick(p, theta=2.0)
    f64 = oracle.direct_f64(ref_in)
    got = np.zeros_like(f64)
    got[p.id] = np.stack([p.fx, p.fy, p.fz], axis=1)
    d = got - f64
    rms = np.sqrt((d * d).sum() / (f64 * f64).sum())
    assert rms < 0.10, (name, rms)


# ---- golden fixtures made by the reference ----------------------------------

@pytest.mark.parametrize("name", golden_names())
def test_matches_golden(oracle, name):
    g = load_golden(name)
    p = golden_particles(g)
    r = oracle.tick(p, theta=float(g["theta"]))
    assert np.array_equal(r["codes"], g["codes"])
    assert np.array_equal(np.array([r["min"], r["max"], r["range"]], np.float32), g["bbox"])
    assert np.array_equal(p.id, g["id"])
    for k in ("x", "y", "z", "mass"):
        assert np.array_equal(getattr(p, k), g[k])
    t = r["tree"]
    for k in ("depth", "start", "count", "leaf", "nchild", "octant"):
        assert np.array_equal(t[k], g["t_" + k]), k
    assert np.array_equal(t["geo"], g["t_geo"])
    # the fixtures come from the reference's fast-math build: sums may be
    # reassociated, so values agree to rounding, not bit for bit
    assert rel_l2(t["mp"], g["t_mp"]) < 1e-6
    assert rel_l2(t["l_tot"], g["t_loc"]) < 1e-5
    F = np.stack([p.fx, p.fy, p.fz])
    G = np.stack([g["fx"], g["fy"], g["fz"]])
    assert rel_l2(F, G) < 2e-6


# ---- the reference itself, where its checker build exists ------------------

def _ref_or_skip(variant):
    from oracle import refbind
    if not refbind.available(variant):
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    return refbind.RefLib(variant)


@pytest.mark.parametrize("n,seed,theta", [(1500, 3, 2.0), (777, 4, 1.0), (2048, 5, 3.4641)])
def test_bit_exact_vs_strict_reference(oracle, n, seed, theta):
    ref = _ref_or_skip("_strict")
    p = W.plummer(n, seed)
    a, b = p.copy(), p.copy()
    ro = oracle.tick(a, theta=theta)
    rr = ref.tick(b, theta=theta, thrd_cnt=4, dump_tree=True)
    assert np.array_equal(ro["codes"], rr["codes"])
    assert np.array_equal(a.id, b.id)
    t = rr["tree"]
    for k in ("depth", "start", "count", "leaf", "nchild", "octant"):
        assert np.array_equal(ro["tree"][k], t[k])
    for k_o, k_r in (("geo", "geo"), ("mp", "mp"), ("l_tot", "loc")):
        assert np.array_equal(ro["tree"][k_o], t[k_r]), k_o
    for k in ("fx", "fy", "fz"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


@pytest.mark.parametrize("variant", [1, 2])
def test_other_morton_variants_vs_formula(oracle, variant):
    # NEON truncation (:2101-2113) and the scalar formula (:2133-2153)
    p = W.uniform_cube(1001, 8)
    rc, codes, mn, mx, rg = oracle.prepare(p, variant)
    f = np.float32
    lanes = 4 if variant == 1 else 0
    vec_end = (p.n // lanes) * lanes if lanes else 0
    scale = f(1023.0) / f(rg)
    want = []
    for i in range(p.n):
        q = []
        for v in (p.x[i], p.y[i], p.z[i]):
            if i < vec_end:
                t = (f(v) - f(mn)) * scale
                t = t if t < f(1023) else f(1023)
                t = f(0) if f(0) > t else t
                q.append(int(t))
            else:
                t = int(((f(v) - f(mn)) / f(rg)) * f(1023.0))
                q.append(min(max(t, 0), 1023))
        want.append(oracle.morton_encode(*q))
    assert codes.tolist() == want


def test_euler_step_follows_the_readme_loop(oracle):
    # README.md:82-111: v_new[i] = v[ids[i]]; massive particles get
    # v += (f / m) * dt and x += v * dt, rounded as written
    f = np.float32
    rng = np.random.default_rng(3)
    n = 257
    p = W.uniform_cube(n, 4)
    p.id[:] = rng.permutation(n).astype(np.uint32)
    p.mass[::5] = 0.0
    for k in ("fx", "fy", "fz"):
        getattr(p, k)[:] = rng.normal(size=n).astype(np.float32)
    v = [rng.normal(size=n).astype(np.float32) for _ in range(3)]
    dt = f(0.016)
    want_v = [vv[p.id].copy() for vv in v]
    want_x = [p.x.copy(), p.y.copy(), p.z.copy()]
    for i in range(n):
        if p.mass[i] <= 0:
            continue
        for c, fc in enumerate((p.fx, p.fy, p.fz)):
            want_v[c][i] = f(want_v[c][i] + f(f(fc[i] / p.mass[i]) * dt))
            want_x[c][i] = f(want_x[c][i] + f(want_v[c][i] * dt))
    oracle.euler_step(p, *v, float(dt))
    for c in range(3):
        assert np.array_equal(v[c], want_v[c])
    assert np.array_equal(p.x, want_x[0]) and np.array_equal(p.z, want_x[2])


def test_closure_order1_beats_order0(oracle):
    # the closure's order-1 local expansion (no counterpart in the reference)
    # is a strictly better far field than the reference's order-0 one
    n = 4096
    p0 = W.clumpy_plummer(n, 12)
    tg = np.arange(0, n, 4, dtype=np.uint32)
    errs = []
    for order in (0, 1):
        p = p0.copy()
        oracle.tick(p, theta=4.0, order=order, want_tree=False)
        f64 = oracle.direct_f64(p, tg)
        F = np.stack([p.fx, p.fy, p.fz], 1)[tg].astype(np.float64)
        errs.append(np.median(np.linalg.norm(F - f64, axis=1) / np.linalg.norm(f64, axis=1)))
    assert errs[1] < 0.5 * errs[0], errs


def test_closure_features_are_normalised(oracle):
    from oracle import closure_oracle as CO
    n = 4096
    p = W.clumpy_plummer(n, 13)
    raw = np.zeros((n, 16), np.float32)
    oracle.tick(p, theta=6.0, order=1, feat=raw, want_tree=False)
    x, scale = CO.features_from_raw(raw)
    assert np.all(np.linalg.norm(x[:, 0:3], axis=1) <= 1.0 + 1e-6)
    # rounded (not truncated) Morton quantisation (polesitter.h:2015-2073) lets
    # a particle sit up to ~1.5 half widths from its depth-10 cell's centre
    assert np.all(np.abs(x[:, 9:12]) <= 2.0)
    assert np.all(x[:, 13:] == 0) and np.all(scale > 0)
    assert set(np.round(x[:, 12] * 10).astype(int)) <= set(range(1, 11))


def test_closure_network_oracle_gradient_by_finite_differences(monkeypatch):
    # the numpy backward pass against central differences (BF16 rounding
    # switched off so that the loss is smooth)
    from oracle import closure_oracle as CO
    monkeypatch.setattr(CO, "bf16", lambda a: np.asarray(a, np.float64))
    rng = np.random.default_rng(1)
    p = rng.normal(0.0, 0.2, CO.N_PARAMS)
    x = rng.normal(0.0, 1.0, (40, 16))
    t = rng.normal(0.0, 1.0, (40, 3))
    _, g = CO.loss_and_grad(p, x, t)
    idx = rng.choice(CO.N_PARAMS, 30, replace=False)
    eps = 1e-6
    num = []
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = CO.loss_and_grad(q, x, t)
        q[i] -= 2 * eps
        lm, _ = CO.loss_and_grad(q, x, t)
        num.append((lp - lm) / (2 * eps))
    assert np.abs(np.array(num) - g[idx]).max() <= 1e-6 * np.abs(g).max()


def test_bf16_rounding_is_round_to_nearest_even():
    from oracle import closure_oracle as CO
    one = np.float32(1.0)
    ulp = np.float32(2.0 ** -7)  # bf16 spacing at 1
    vals = np.array([one, one + ulp / 2, one + ulp / 2 + ulp / 8, one + 1.5 * ulp], np.float32)
    got = CO.bf16(vals)
    assert got.tolist() == [1.0, 1.0, float(one + ulp), float(one + 2 * ulp)]


def _starts_by_window_rule(codes, cap):
    """Node starts per depth from sorted codes by the flag rule the GPU tree
    build uses: a depth-d node starts at i iff a depth-d run starts there
    and d - 1 <= W(i) = max over j in [i-cap, i] of cpl2(codes[j], codes[j+cap]),
    with W >= 0 (the root is split) once n >= 2."""
    c = codes.astype(np.int64) & 0x3FFFFFFF
    n = len(c)

    def cpl2(a, b):
        x = a ^ b
        out = np.full(x.shape, 10, np.int64)
        nz = x != 0
        out[nz] = (29 - np.floor(np.log2(x[nz])).astype(np.int64)) // 3
        return out

    cpl = np.full(n, -1, np.int64)
    cpl[1:] = cpl2(c[:-1], c[1:])
    w = np.full(n, 0 if n >= 2 else -1, np.int64)
    if n > cap:
        wj = cpl2(c[: n - cap], c[cap:])  # window starting at j
        for i in range(n):
            lo, hi = max(0, i - cap), min(i, n - 1 - cap)
            if lo <= hi:
                w[i] = max(w[i], wj[lo:hi + 1].max())
    out = {}
    for d in range(1, 11):
        start = (cpl < d)
        start[0] = True
        out[d] = np.nonzero(start & (w >= d - 1))[0]
    return out


@pytest.mark.parametrize("cap", [1, 2, 5, 16, 64])
def test_leaf_capacity_start_rule_matches_the_split_recursion(oracle, cap):
    # the GPU's one-pass flag rule against the oracle's recursive splitting
    p = W.clumpy_plummer(3000, 11)
    r = oracle.tick(p, theta=2.0, leaf_cap=cap)
    t = r["tree"]
    rule = _starts_by_window_rule(r["codes"], cap)
    for d in range(1, 11):
        got = np.sort(t["start"][t["depth"] == d])
        assert np.array_equal(got, rule[d]), d


def test_leaf_capacity_tree_shape(oracle):
    p = W.plummer(4000, 12)
    base = oracle.tick(p.copy(), theta=2.0)
    one = oracle.tick(p.copy(), theta=2.0, leaf_cap=1)
    assert np.array_equal(base["tree"]["start"], one["tree"]["start"])
    for cap in (8, 32):
        t = oracle.tick(p.copy(), theta=2.0, leaf_cap=cap)["tree"]
        leaf = t["nchild"] == 0
        below = t["depth"] > 0
        assert t["count"][leaf & below & (t["depth"] < 10)].max() <= cap
        assert t["count"][~leaf & below].min() > cap
        assert t["nchild"][0] > 0
    # a root holding fewer than cap particles is split all the same
    q = W.uniform_cube(5, 1)
    t = oracle.tick(q, theta=2.0, leaf_cap=16)["tree"]
    assert t["nchild"][0] > 0 and np.all(t["nchild"][1:] == 0)
