"""polesitter_b200 -- the polesitter FMM tick on one B200, behind the
reference's own C API.

The product is ``libpolesitter_b200.so`` (built in-tree by
``polesitter_b200.build``), which exports ``ps_init``,
``ps_prepare_particles``, ``ps_calc_forces`` and ``ps_destroy`` with the
reference's types (include/polesitter.h) plus ``ps_b200_*`` extensions
(include/polesitter_b200.h).  This module is a thin ctypes mirror of that
interface -- same names, argument meaning and result codes -- used by the
tests and the benchmark.  It never computes anything itself: if the library
is missing, importing :func:`lib` raises.
"""

from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libpolesitter_b200.so")

# ps_result_t (polesitter.h:294-300) + PS_EDEVICE
PS_OK, PS_EOOM, PS_EINVAL, PS_ETHRD, PS_EALLOC, PS_EDEVICE = 0, -1, -2, -3, -4, -5
RESULT_NAMES = {0: "PS_OK", -1: "PS_EOOM", -2: "PS_EINVAL", -3: "PS_ETHRD",
                -4: "PS_EALLOC", -5: "PS_EDEVICE"}

OPT_DEBUG, OPT_THETA, OPT_TIMING, OPT_KAHAN, OPT_CLOSURE, OPT_JUDGE = 1, 2, 4, 6, 7, 8
OPT_HEAVY_DEPTH = 9
OPT_LEAF_CAP = 10
OPT_NEAR_LEVELS, OPT_STREAM, OPT_SHRINK_STORES, OPT_SORT_SPIN = 11, 12, 13, 14
OPT_JUDGE_BLOCKS, OPT_JUDGE_SAMPLES = 15, 16
CLOSURE_PARAMS = 9928
MORTON_AVX2, MORTON_NEON, MORTON_SCALAR = 0, 1, 2

EXPORTED = ("ps_init", "ps_prepare_particles", "ps_calc_forces", "ps_destroy",
            "ps_b200_context_size", "ps_b200_set_option", "ps_b200_set_morton_variant",
            "ps_b200_get_stats", "ps_b200_last_timing", "ps_b200_tree_nodes",
            "ps_b200_tree_dump", "ps_b200_direct_f64", "ps_b200_last_error",
            "ps_b200_prepare_particles_noalloc", "ps_b200_run_ticks",
            "ps_b200_closure_set_weights", "ps_b200_closure_last", "ps_b200_closure_features",
            "ps_b200_closure_correction", "ps_b200_closure_forward", "ps_b200_closure_grad",
            "ps_b200_closure_train", "ps_b200_ensemble_create", "ps_b200_ensemble_autotune",
            "ps_b200_ensemble_run", "ps_b200_ensemble_theta", "ps_b200_ensemble_destroy",
            "ps_b200_ensemble_leaf_caps", "ps_b200_ensemble_set_leaf_caps",
            "ps_b200_ensemble_set_leaf_ladder", "ps_b200_ensemble_set_order",
            "ps_b200_ensemble_order")


class ParticleArrs(C.Structure):
    """``ps_particle_arrs_t`` (polesitter.h:312-322)."""

    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p),
                ("mass", C.c_void_p), ("fx", C.c_void_p), ("fy", C.c_void_p),
                ("fz", C.c_void_p), ("id", C.c_void_p), ("cnt", C.c_size_t)]


class Config(C.Structure):
    """``ps_config_t`` (polesitter.h:304-310)."""

    _fields_ = [("buff", C.c_void_p), ("buff_size", C.c_size_t),
                ("max_particles", C.c_size_t), ("theta", C.c_float),
                ("thrd_cnt", C.c_size_t)]


class PolesitterError(RuntimeError):
    def __init__(self, call: str, code: int, detail: str = ""):
        self.code = code
        super().__init__(f"{call} -> {RESULT_NAMES.get(code, code)}"
                         + (f" ({detail})" if detail else ""))


_LIB = None


def lib() -> C.CDLL:
    """Load the CUDA library; raise if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m polesitter_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, sz, f32 = C.c_void_p, C.c_size_t, C.c_float
    L.ps_init.restype = C.c_int
    L.ps_init.argtypes = [C.POINTER(C.c_void_p), C.POINTER(Config)]
    L.ps_prepare_particles.restype = C.c_int
    L.ps_prepare_particles.argtypes = [C.POINTER(ParticleArrs), vp, C.POINTER(f32),
                                       C.POINTER(f32), C.POINTER(f32)]
    L.ps_calc_forces.restype = C.c_int
    L.ps_calc_forces.argtypes = [vp, C.POINTER(ParticleArrs), vp, f32, f32, f32, f32]
    L.ps_destroy.restype = C.c_int
    L.ps_destroy.argtypes = [vp]
    L.ps_b200_context_size.restype = sz
    L.ps_b200_set_option.restype = C.c_int
    L.ps_b200_set_option.argtypes = [vp, C.c_int, C.c_double]
    L.ps_b200_set_morton_variant.restype = C.c_int
    L.ps_b200_set_morton_variant.argtypes = [C.c_int]
    L.ps_b200_get_stats.restype = C.c_int
    L.ps_b200_get_stats.argtypes = [vp, vp, sz]
    L.ps_b200_last_timing.restype = C.c_int
    L.ps_b200_last_timing.argtypes = [vp, vp, sz]
    L.ps_b200_tree_nodes.restype = sz
    L.ps_b200_tree_nodes.argtypes = [vp]
    L.ps_b200_tree_dump.restype = C.c_int
    L.ps_b200_tree_dump.argtypes = [vp, sz] + [vp] * 12
    L.ps_b200_direct_f64.restype = C.c_int
    L.ps_b200_direct_f64.argtypes = [vp, C.POINTER(ParticleArrs), vp, sz, vp]
    L.ps_b200_last_error.restype = C.c_char_p
    L.ps_b200_prepare_particles_noalloc.restype = C.c_int
    L.ps_b200_prepare_particles_noalloc.argtypes = [C.POINTER(ParticleArrs), vp, C.POINTER(f32),
                                                    C.POINTER(f32), C.POINTER(f32)]
    L.ps_b200_closure_set_weights.argtypes = [vp, vp, sz]
    L.ps_b200_closure_last.argtypes = [vp, vp, vp, vp, vp]
    L.ps_b200_closure_features.argtypes = [vp, vp, sz, vp, vp]
    L.ps_b200_closure_correction.argtypes = [vp, vp, sz]
    L.ps_b200_closure_forward.argtypes = [vp, vp, sz, vp, vp]
    L.ps_b200_closure_grad.argtypes = [vp, vp, vp, sz, vp, vp, vp]
    L.ps_b200_closure_train.argtypes = [vp, vp, vp, sz, vp, C.c_uint32, C.c_uint32, f32,
                                        C.c_uint64, vp]
    for name in ("ps_b200_closure_set_weights", "ps_b200_closure_last", "ps_b200_closure_features",
                 "ps_b200_closure_correction", "ps_b200_closure_forward", "ps_b200_closure_grad",
                 "ps_b200_closure_train", "ps_b200_ensemble_create", "ps_b200_ensemble_autotune",
            "ps_b200_ensemble_run", "ps_b200_ensemble_theta", "ps_b200_ensemble_destroy"):
        getattr(L, name).restype = C.c_int
    L.ps_b200_ensemble_create.argtypes = [C.POINTER(vp), vp, sz, vp]
    L.ps_b200_ensemble_autotune.argtypes = [vp, C.POINTER(ParticleArrs), vp, f32, vp, vp]
    L.ps_b200_ensemble_run.argtypes = [vp, C.POINTER(ParticleArrs), vp, vp, vp, vp, f32,
                                       C.c_uint32]
    L.ps_b200_ensemble_theta.argtypes = [vp, vp, sz]
    L.ps_b200_ensemble_destroy.argtypes = [vp]
    L.ps_b200_ensemble_leaf_caps.argtypes = [vp, vp, sz]
    L.ps_b200_ensemble_set_leaf_caps.argtypes = [vp, vp, sz]
    L.ps_b200_ensemble_set_leaf_ladder.argtypes = [vp, vp, sz]
    L.ps_b200_ensemble_set_order.argtypes = [vp, C.c_int]
    L.ps_b200_ensemble_order.argtypes = [vp, vp]
    for name in ("ps_b200_ensemble_create", "ps_b200_ensemble_autotune", "ps_b200_ensemble_run",
                 "ps_b200_ensemble_theta", "ps_b200_ensemble_destroy",
                 "ps_b200_ensemble_leaf_caps", "ps_b200_ensemble_set_leaf_caps",
                 "ps_b200_ensemble_set_leaf_ladder", "ps_b200_ensemble_set_order",
                 "ps_b200_ensemble_order"):
        getattr(L, name).restype = C.c_int
    L.ps_b200_run_ticks.restype = C.c_int
    L.ps_b200_run_ticks.argtypes = [vp, C.POINTER(ParticleArrs), vp, vp, vp, vp, f32, C.c_uint32]
    _LIB = L
    return L


def _addr(a) -> int:
    """Address of a numpy array (host) or a torch tensor (host or CUDA)."""
    if a is None:
        return 0
    if hasattr(a, "data_ptr"):
        assert a.is_contiguous()
        return a.data_ptr()
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def arrs_of(p, n=None) -> ParticleArrs:
    """``ps_particle_arrs_t`` over an object with x, y, z, mass, fx, fy, fz, id
    arrays (numpy or torch, host or device)."""
    cnt = len(p.x) if n is None else n
    return ParticleArrs(_addr(p.x), _addr(p.y), _addr(p.z), _addr(p.mass), _addr(p.fx),
                        _addr(p.fy), _addr(p.fz), _addr(p.id), cnt)


def _check(call, r):
    if r != PS_OK:
        detail = lib().ps_b200_last_error()
        raise PolesitterError(call, r, detail.decode() if detail else "")


def set_morton_variant(variant: int) -> None:
    _check("ps_b200_set_morton_variant", lib().ps_b200_set_morton_variant(variant))


def prepare_particles(p, codes):
    """ps_prepare_particles: writes ``codes`` and returns (min_b, max_b, range)."""
    arrs = arrs_of(p)
    mn, mx, rg = C.c_float(), C.c_float(), C.c_float()
    _check("ps_prepare_particles", lib().ps_prepare_particles(
        C.byref(arrs), _addr(codes), C.byref(mn), C.byref(mx), C.byref(rg)))
    return mn.value, mx.value, rg.value


def root_box(min_b: float, rng: float):
    """Root centre and half width as the reference's callers compute them
    (README.md:78-79, tests/accuracy.c:497-499), in float32."""
    import numpy as np
    f = np.float32
    c = f(min_b) + f(rng) / f(2.0)
    hw = f(rng) / f(2.0)
    return float(c), float(hw)


class Context:
    """One ``ps_context_t`` (ps_init ... ps_destroy)."""

    def __init__(self, max_particles: int, theta: float = 2.0, thrd_cnt: int = 1,
                 buff_size: int | None = None):
        import numpy as np
        L = lib()
        size = buff_size if buff_size is not None else (
            L.ps_b200_context_size() + 64 + 24 * max_particles + 4096)
        self._buf = np.zeros(max(size, 1), np.uint8)
        self.cfg = Config(self._buf.ctypes.data if size else 0, size, max_particles, theta,
                          thrd_cnt)
        self.ptr = C.c_void_p()
        _check("ps_init", L.ps_init(C.byref(self.ptr), C.byref(self.cfg)))
        self.max_particles = max_particles

    def calc_forces(self, p, codes, cx, cy, cz, hw):
        arrs = arrs_of(p)
        _check("ps_calc_forces", lib().ps_calc_forces(self.ptr, C.byref(arrs), _addr(codes),
                                                      cx, cy, cz, hw))

    def tick(self, p, codes):
        """prepare + calc as the reference's tick loop (README.md:74-88)."""
        mn, mx, rg = prepare_particles(p, codes)
        c, hw = root_box(mn, rg)
        self.calc_forces(p, codes, c, c, c, hw)
        return mn, mx, rg

    def run_ticks(self, p, codes, vx, vy, vz, dt: float, ticks: int):
        """``ticks`` iterations of the caller's tick loop on the device
        (README.md:65-111): ids reset, prepare, calc, velocity permutation
        through ids, semi-implicit Euler (ps_b200_run_ticks)."""
        arrs = arrs_of(p)
        _check("ps_b200_run_ticks", lib().ps_b200_run_ticks(
            self.ptr, C.byref(arrs), _addr(codes), _addr(vx), _addr(vy), _addr(vz), dt, ticks))

    # ---- learned far-field closure (ps_b200_closure_*) ----
    def set_closure(self, mode: int):
        """0: the reference's far field, 1: order-1 local expansion, 2: order-1
        plus the learned correction under the sampled FP64 judge."""
        self.set_option(OPT_CLOSURE, mode)

    def closure_set_weights(self, params):
        import numpy as np
        p = np.ascontiguousarray(params, np.float32)
        _check("ps_b200_closure_set_weights",
               lib().ps_b200_closure_set_weights(self.ptr, p.ctypes.data, p.size))

    def closure_last(self) -> dict:
        mb, mm = C.c_double(), C.c_double()
        used, smp = C.c_int(), C.c_int()
        _check("ps_b200_closure_last", lib().ps_b200_closure_last(
            self.ptr, C.byref(mb), C.byref(mm), C.byref(used), C.byref(smp)))
        return {"median_base": mb.value, "median_mlp": mm.value, "used": bool(used.value),
                "samples": smp.value}

    def closure_features(self, idx):
        import numpy as np
        ix = np.ascontiguousarray(idx, np.uint32)
        x = np.zeros((ix.size, 16), np.float32)
        sc = np.zeros(ix.size, np.float32)
        _check("ps_b200_closure_features", lib().ps_b200_closure_features(
            self.ptr, ix.ctypes.data, ix.size, x.ctypes.data, sc.ctypes.data))
        return x, sc

    def closure_correction(self, n: int):
        import numpy as np
        out = np.zeros((n, 3), np.float32)
        _check("ps_b200_closure_correction",
               lib().ps_b200_closure_correction(self.ptr, out.ctypes.data, n))
        return out

    def closure_forward(self, x, params):
        import numpy as np
        xx = np.ascontiguousarray(x, np.float32)
        p = np.ascontiguousarray(params, np.float32)
        y = np.zeros((xx.shape[0], 8), np.float32)
        _check("ps_b200_closure_forward", lib().ps_b200_closure_forward(
            self.ptr, xx.ctypes.data, xx.shape[0], p.ctypes.data, y.ctypes.data))
        return y

    def closure_grad(self, x, t, params):
        import numpy as np
        xx = np.ascontiguousarray(x, np.float32)
        tt = np.ascontiguousarray(t, np.float32)
        p = np.ascontiguousarray(params, np.float32)
        g = np.zeros_like(p)
        loss = C.c_float()
        _check("ps_b200_closure_grad", lib().ps_b200_closure_grad(
            self.ptr, xx.ctypes.data, tt.ctypes.data, xx.shape[0], p.ctypes.data, g.ctypes.data,
            C.byref(loss)))
        return g, loss.value

    def closure_train(self, x, t, params, epochs: int, batch: int, lr: float, seed: int = 0):
        import numpy as np
        xx = np.ascontiguousarray(x, np.float32)
        tt = np.ascontiguousarray(t, np.float32)
        p = np.array(params, np.float32)
        losses = np.zeros(max(epochs, 1), np.float32)
        _check("ps_b200_closure_train", lib().ps_b200_closure_train(
            self.ptr, xx.ctypes.data, tt.ctypes.data, xx.shape[0], p.ctypes.data, epochs, batch,
            lr, seed, losses.ctypes.data))
        return p, losses[:epochs]

    def set_option(self, key: int, value: float):
        _check("ps_b200_set_option", lib().ps_b200_set_option(self.ptr, key, value))

    def stats(self) -> dict:
        import numpy as np
        out = np.zeros(24, np.uint64)
        _check("ps_b200_get_stats", lib().ps_b200_get_stats(self.ptr, out.ctypes.data, 24))
        return {"m2l_pairs": int(out[1]), "p2p_pairs": int(out[2]),
                "p2p_interactions": int(out[3]), "chunks_first": int(out[4]),
                "chunks_dfs": int(out[5]), "tests_first": int(out[6]), "tests_dfs": int(out[7]),
                "nodes": int(out[8]), "max_stack": int(out[9]), "p2p_chunks": int(out[10]),
                "traversal_runs": int(out[11]), "max_leaf": int(out[12]),
                "dense_records": int(out[13]), "near_levels": int(out[14]),
                "streamed": int(out[15]),
                "lanes": int(out[16]), "leaf_groups": int(out[17]), "dfs_steps": int(out[18]),
                "full_leaf_interactions": int(out[20]),
                "slowest_group_cycles": int(out[19]) >> 28,
                "slowest_group_node": int(out[19]) & 0xFFFFFFF}

    def timing(self) -> dict:
        import numpy as np
        out = np.zeros(9, np.float32)
        _check("ps_b200_last_timing", lib().ps_b200_last_timing(self.ptr, out.ctypes.data, 9))
        return {"sort": float(out[0]), "gather": float(out[1]), "tree": float(out[2]),
                "upward": float(out[3]), "internal": float(out[4]), "leaves": float(out[5]),
                "tick": float(out[6]), "closure": float(out[7]), "full_leaves": float(out[8])}

    def tree(self) -> dict:
        import numpy as np
        L = lib()
        n = L.ps_b200_tree_nodes(self.ptr)
        t = {k: np.zeros(n, dt) for k, dt in (
            ("depth", np.int32), ("start", np.uint32), ("count", np.uint32),
            ("nchild", np.uint32), ("octant", np.int32), ("first_child", np.uint32),
            ("parent", np.uint32), ("m2l_cnt", np.uint32), ("p2p_cnt", np.uint32))}
        for k in ("geo", "mp", "local_exp"):
            t[k] = np.zeros((n, 4), np.float32)
        _check("ps_b200_tree_dump", L.ps_b200_tree_dump(
            self.ptr, n, *(t[k].ctypes.data for k in (
                "depth", "start", "count", "nchild", "octant", "first_child", "parent",
                "geo", "mp", "local_exp", "m2l_cnt", "p2p_cnt"))))
        t["leaf"] = (t["nchild"] == 0).astype(np.uint32)
        return t

    def direct_f64(self, p, targets):
        import numpy as np
        tg = np.ascontiguousarray(targets, np.uint32)
        out = np.zeros((len(tg), 3), np.float64)
        arrs = arrs_of(p)
        _check("ps_b200_direct_f64", lib().ps_b200_direct_f64(
            self.ptr, C.byref(arrs), tg.ctypes.data, len(tg), out.ctypes.data))
        return out

    def destroy(self):
        if self.ptr:
            _check("ps_destroy", lib().ps_destroy(self.ptr))
            self.ptr = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            if self.ptr:
                lib().ps_destroy(self.ptr)
        except Exception:
            pass


class Ensemble:
    """Many independent systems advanced together (ps_b200_ensemble_*): every
    phase of a tick is one launch over all systems, each tick two replayed
    CUDA graphs.  Arrays are concatenated device arrays (torch CUDA tensors),
    system k at offsets sum(counts[:k])."""

    def __init__(self, counts, theta=None):
        import numpy as np
        self.counts = np.ascontiguousarray(counts, np.uint64)
        th = None if theta is None else np.ascontiguousarray(theta, np.float32)
        self.ptr = C.c_void_p()
        _check("ps_b200_ensemble_create", lib().ps_b200_ensemble_create(
            C.byref(self.ptr), self.counts.ctypes.data, len(self.counts),
            None if th is None else th.ctypes.data))

    def autotune(self, p, codes, target: float):
        import numpy as np
        th = np.zeros(len(self.counts), np.float32)
        gs = C.c_double()
        arrs = arrs_of(p)
        _check("ps_b200_ensemble_autotune", lib().ps_b200_ensemble_autotune(
            self.ptr, C.byref(arrs), _addr(codes), target, th.ctypes.data, C.byref(gs)))
        return th, gs.value

    def run(self, p, codes, vx, vy, vz, dt: float, ticks: int):
        arrs = arrs_of(p)
        _check("ps_b200_ensemble_run", lib().ps_b200_ensemble_run(
            self.ptr, C.byref(arrs), _addr(codes), _addr(vx), _addr(vy), _addr(vz), dt, ticks))

    def theta(self):
        import numpy as np
        th = np.zeros(len(self.counts), np.float32)
        _check("ps_b200_ensemble_theta", lib().ps_b200_ensemble_theta(
            self.ptr, th.ctypes.data, len(th)))
        return th

    def leaf_caps(self):
        import numpy as np
        caps = np.zeros(len(self.counts), np.uint32)
        _check("ps_b200_ensemble_leaf_caps", lib().ps_b200_ensemble_leaf_caps(
            self.ptr, caps.ctypes.data, len(caps)))
        return caps

    def set_leaf_caps(self, caps):
        import numpy as np
        c = np.ascontiguousarray(caps, np.uint32)
        _check("ps_b200_ensemble_set_leaf_caps", lib().ps_b200_ensemble_set_leaf_caps(
            self.ptr, c.ctypes.data, len(c)))

    def set_leaf_ladder(self, caps):
        """The leaf capacities ``autotune`` tries (default 1, 16, 32, 64)."""
        import numpy as np
        c = np.ascontiguousarray(caps, np.uint32)
        _check("ps_b200_ensemble_set_leaf_ladder", lib().ps_b200_ensemble_set_leaf_ladder(
            self.ptr, c.ctypes.data, len(c)))

    def set_order(self, order: int):
        """Local expansion of all systems: 0 (the reference's), 1 (order-1), or
        -1 to let ``autotune`` try both."""
        _check("ps_b200_ensemble_set_order", lib().ps_b200_ensemble_set_order(self.ptr, order))

    def order(self) -> int:
        o = C.c_int()
        _check("ps_b200_ensemble_order", lib().ps_b200_ensemble_order(self.ptr, C.byref(o)))
        return o.value

    def destroy(self):
        if self.ptr:
            _check("ps_b200_ensemble_destroy", lib().ps_b200_ensemble_destroy(self.ptr))
            self.ptr = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()
