"""ctypes binding of the oracle restatement (oracle/ps_oracle.c).

Test infrastructure only.  ``Oracle.tick`` mirrors the reference's
``ps_prepare_particles`` + ``ps_calc_forces`` (polesitter.h:1911-2170,
:1840-1909) on a ``workloads.Particles`` set, mutating it in place the way the
reference mutates the caller's arrays, and returns the canonical tree table and
interaction statistics the GPU path is checked against.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpsoracle.so")

MORTON_AVX2, MORTON_NEON, MORTON_SCALAR = 0, 1, 2


def _ptr(a):
    return None if a is None else a.ctypes.data


def ensure_built() -> str:
    if not os.path.exists(LIB_PATH) or (
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "ps_oracle.c"))):
        subprocess.check_call(["sh", os.path.join(HERE, "build_oracle.sh")])
    return LIB_PATH


class Oracle:
    def __init__(self):
        lib = C.CDLL(ensure_built())
        vp, sz, f32 = C.c_void_p, C.c_size_t, C.c_float
        lib.pso_morton_encode.restype = C.c_uint32
        lib.pso_morton_encode.argtypes = [C.c_uint32] * 3
        lib.pso_prepare.restype = C.c_int
        lib.pso_prepare.argtypes = [sz, vp, vp, vp, vp, vp, vp, vp, C.c_int]
        lib.pso_sort.argtypes = [sz] + [vp] * 6
        lib.pso_new.restype = vp
        lib.pso_free.argtypes = [vp]
        lib.pso_calc.restype = C.c_int
        lib.pso_calc.argtypes = [vp, sz] + [vp] * 8 + [f32] * 5 + [C.c_int, C.c_int]
        lib.pso_num_nodes.restype = sz
        lib.pso_num_nodes.argtypes = [vp]
        lib.pso_num_p2p.restype = sz
        lib.pso_num_p2p.argtypes = [vp]
        lib.pso_stats.argtypes = [vp, vp]
        lib.pso_level_starts.argtypes = [vp, vp]
        lib.pso_tree.argtypes = [vp] + [vp] * 14
        lib.pso_p2p_list.argtypes = [vp, vp, vp]
        lib.pso_direct_f64.argtypes = [sz, vp, vp, vp, vp, vp, sz, vp, vp, vp]
        lib.pso_p2m.argtypes = [sz, vp, vp, vp, vp, f32, f32, f32, vp]
        lib.pso_m2l_pair.restype = C.c_int
        lib.pso_m2l_pair.argtypes = [vp, vp, vp, f32, vp]
        lib.pso_p2p_pair.argtypes = [vp] * 7 + [C.c_uint32] * 4
        lib.pso_euler_step.argtypes = [sz] + [vp] * 11 + [f32, vp]
        lib.pso_set_closure.argtypes = [vp, C.c_int, vp]
        lib.pso_set_leaf_cap.argtypes = [vp, C.c_uint32]
        self.lib = lib

    def morton_encode(self, x, y, z) -> int:
        return self.lib.pso_morton_encode(x, y, z)

    def prepare(self, p, variant: int = MORTON_AVX2):
        codes = np.zeros(p.n, np.uint32)
        mn, mx, rg = (np.zeros(1, np.float32) for _ in range(3))
        rc = self.lib.pso_prepare(p.n, _ptr(p.x), _ptr(p.y), _ptr(p.z), _ptr(codes),
                                  _ptr(mn), _ptr(mx), _ptr(rg), variant)
        return rc, codes, float(mn[0]), float(mx[0]), float(rg[0])

    def sort(self, p, codes):
        self.lib.pso_sort(p.n, _ptr(codes), _ptr(p.id), _ptr(p.x), _ptr(p.y),
                          _ptr(p.z), _ptr(p.mass))

    def calc(self, p, codes, cx, cy, cz, hw, theta=2.0, mt=True, accum_mode=0,
             want_tree=True, want_p2p=False, order=0, feat=None, leaf_cap=1):
        """ps_calc_forces on arrays that are already sorted (``sort``).
        ``order`` 1 selects the closure's order-1 local expansion; ``feat``
        (n x 16 float32) then receives the raw per-particle closure features.
        ``leaf_cap`` > 1 splits only nodes holding more particles than that
        (the reference splits every node holding two or more)."""
        h = self.lib.pso_new()
        try:
            if leaf_cap != 1:
                self.lib.pso_set_leaf_cap(h, int(leaf_cap))
            if order or feat is not None:
                assert feat is None or (feat.dtype == np.float32 and feat.shape == (p.n, 16))
                self.lib.pso_set_closure(h, order, None if feat is None else _ptr(feat))
            rc = self.lib.pso_calc(h, p.n, _ptr(codes), _ptr(p.x), _ptr(p.y), _ptr(p.z),
                                   _ptr(p.mass), _ptr(p.fx), _ptr(p.fy), _ptr(p.fz),
                                   cx, cy, cz, hw, theta, int(mt), accum_mode)
            assert rc == 0
            st = np.zeros(4, np.uint64)
            self.lib.pso_stats(h, _ptr(st))
            lv = np.zeros(12, np.uint32)
            self.lib.pso_level_starts(h, _ptr(lv))
            out = {"stats": {"mac_tests": int(st[0]), "m2l_pairs": int(st[1]),
                             "p2p_pairs": int(st[2]), "p2p_interactions": int(st[3])},
                   "level_start": lv}
            if want_tree:
                n = self.lib.pso_num_nodes(h)
                t = {k: np.zeros(n, dt) for k, dt in (
                    ("depth", np.int32), ("start", np.uint32), ("count", np.uint32),
                    ("leaf", np.uint32), ("nchild", np.uint32), ("octant", np.int32),
                    ("first_child", np.uint32), ("parent", np.uint32),
                    ("m2l_cnt", np.uint32), ("p2p_cnt", np.uint32))}
                for k in ("geo", "mp", "l_m2l", "l_tot"):
                    t[k] = np.zeros((n, 4), np.float32)
                self.lib.pso_tree(h, _ptr(t["depth"]), _ptr(t["start"]), _ptr(t["count"]),
                                  _ptr(t["leaf"]), _ptr(t["nchild"]), _ptr(t["octant"]),
                                  _ptr(t["first_child"]), _ptr(t["parent"]), _ptr(t["geo"]),
                                  _ptr(t["mp"]), _ptr(t["l_m2l"]), _ptr(t["l_tot"]),
                                  _ptr(t["m2l_cnt"]), _ptr(t["p2p_cnt"]))
                out["tree"] = t
            if want_p2p:
                n = self.lib.pso_num_p2p(h)
                pt, ps = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
                self.lib.pso_p2p_list(h, _ptr(pt), _ptr(ps))
                out["p2p"] = (pt, ps)
            return out
        finally:
            self.lib.pso_free(h)

    def tick(self, p, theta=2.0, variant=MORTON_AVX2, mt=True, accum_mode=0,
             want_tree=True, want_p2p=False, order=0, feat=None, leaf_cap=1):
        """prepare + calc on ``p`` in place (arrays end sorted, forces set)."""
        rc, codes, mn, mx, rg = self.prepare(p, variant)
        assert rc == 0
        f32 = np.float32
        c = f32(mn) + f32(rg) / f32(2.0)
        hw = f32(rg) / f32(2.0)
        self.sort(p, codes)
        out = self.calc(p, codes, float(c), float(c), float(c), float(hw), theta, mt,
                        accum_mode, want_tree, want_p2p, order, feat, leaf_cap)
        out.update(codes=codes, min=mn, max=mx, range=rg, root_c=float(c), root_hw=float(hw))
        return out

    def euler_step(self, p, vx, vy, vz, dt):
        """The caller's update after a tick (README.md:82-111): permute the
        velocities through ``p.id``, then semi-implicit Euler, in place."""
        tmp = np.zeros(3 * p.n, np.float32)
        self.lib.pso_euler_step(p.n, _ptr(p.id), _ptr(vx), _ptr(vy), _ptr(vz), _ptr(p.x),
                                _ptr(p.y), _ptr(p.z), _ptr(p.mass), _ptr(p.fx), _ptr(p.fy),
                                _ptr(p.fz), dt, _ptr(tmp))

    def run_ticks(self, p, vx, vy, vz, dt, ticks, theta=2.0, leaf_cap=1):
        """``ticks`` iterations of README.md:65-111: ids reset, prepare +
        calc, velocity permutation, Euler.  Returns the last tick's codes."""
        codes = None
        for _ in range(ticks):
            p.id[:] = np.arange(p.n, dtype=np.uint32)
            codes = self.tick(p, theta=theta, want_tree=False, leaf_cap=leaf_cap)["codes"]
            self.euler_step(p, vx, vy, vz, dt)
        return codes

    def p2m(self, x, y, z, m, centre=(0.0, 0.0, 0.0)):
        a = [np.ascontiguousarray(v, np.float32) for v in (x, y, z, m)]
        out = np.zeros(4, np.float32)
        self.lib.pso_p2m(len(a[0]), *(_ptr(v) for v in a), *centre, _ptr(out))
        return out

    def m2l_pair(self, tgt_geo, src_geo, src_mp, theta):
        tg = np.asarray(tgt_geo, np.float32)
        sg = np.asarray(src_geo, np.float32)
        sm = np.asarray(src_mp, np.float32)
        out = np.zeros(4, np.float32)
        hit = self.lib.pso_m2l_pair(_ptr(tg), _ptr(sg), _ptr(sm), theta, _ptr(out))
        return bool(hit), out

    def p2p_pair(self, p, t0, tn, s0, sn):
        self.lib.pso_p2p_pair(_ptr(p.x), _ptr(p.y), _ptr(p.z), _ptr(p.mass), _ptr(p.fx),
                              _ptr(p.fy), _ptr(p.fz), t0, tn, s0, sn)

    def direct_f64(self, p, targets=None):
        """FP64 direct-sum forces (tests/accuracy.c:42-72) for ``targets``
        (indices into the current arrays; all particles if None)."""
        tg = None if targets is None else np.ascontiguousarray(targets, np.uint32)
        nt = p.n if tg is None else len(tg)
        fx, fy, fz = (np.zeros(nt, np.float64) for _ in range(3))
        self.lib.pso_direct_f64(p.n, _ptr(p.x), _ptr(p.y), _ptr(p.z), _ptr(p.mass),
                                _ptr(tg), nt, _ptr(fx), _ptr(fy), _ptr(fz))
        return np.stack([fx, fy, fz], axis=1)


def rel_errors(f32_forces: np.ndarray, f64_ref: np.ndarray):
    """Per-particle relative force error |F - F_ref| / |F_ref| and the RMS
    relative error sqrt(sum|dF|^2 / sum|F_ref|^2) (tests/accuracy.c:505-531)."""
    d = np.asarray(f32_forces, np.float64) - f64_ref
    e2 = (d * d).sum(1)
    r2 = (f64_ref * f64_ref).sum(1)
    ok = r2 > 1e-24
    rel = np.sqrt(e2[ok] / r2[ok])
    rms = float(np.sqrt(e2.sum() / r2.sum())) if r2.sum() > 0 else 0.0
    return {"median": float(np.median(rel)) if rel.size else 0.0, "rms": rms,
            "max": float(rel.max()) if rel.size else 0.0}
