"""ctypes binding of the checker's build of the reference (oracle/_ref).

Test infrastructure only: loads ``oracle/_ref/libpsref.so`` (the unmodified
polesitter header compiled with its own flags by ``oracle/build_ref.sh``) and
exposes the reference's public tick plus the white-box tree view exported by
``oracle/ref_wrap.c``.  Nothing in the product imports this module.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


class ParticleArrs(C.Structure):
    """Layout of ``ps_particle_arrs_t`` (polesitter.h:312-322)."""

    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p),
                ("mass", C.c_void_p), ("fx", C.c_void_p), ("fy", C.c_void_p),
                ("fz", C.c_void_p), ("id", C.c_void_p), ("cnt", C.c_size_t)]


class Config(C.Structure):
    """Layout of ``ps_config_t`` (polesitter.h:304-310)."""

    _fields_ = [("buff", C.c_void_p), ("buff_size", C.c_size_t),
                ("max_particles", C.c_size_t), ("theta", C.c_float),
                ("thrd_cnt", C.c_size_t)]


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def arrs_of(p) -> ParticleArrs:
    return ParticleArrs(_ptr(p.x), _ptr(p.y), _ptr(p.z), _ptr(p.mass),
                        _ptr(p.fx), _ptr(p.fy), _ptr(p.fz), _ptr(p.id), p.n)


def available(variant: str = "") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libpsref{variant}.so"))


class RefLib:
    """The reference's compiled tick (variant "" = its own flags,
    "_strict" = strict IEEE build of the same source)."""

    def __init__(self, variant: str = ""):
        path = os.path.join(REF_DIR, f"libpsref{variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} missing: run oracle/build_ref.sh where the reference "
                "checkout is present")
        lib = C.CDLL(path)
        lib.psref_ctx_size.restype = C.c_size_t
        lib.psref_init.argtypes = [C.POINTER(C.c_void_p), C.POINTER(Config)]
        lib.psref_prepare.argtypes = [C.POINTER(ParticleArrs), C.c_void_p,
                                      C.POINTER(C.c_float), C.POINTER(C.c_float),
                                      C.POINTER(C.c_float)]
        lib.psref_calc.argtypes = [C.c_void_p, C.POINTER(ParticleArrs), C.c_void_p,
                                   C.c_float, C.c_float, C.c_float, C.c_float]
        lib.psref_destroy.argtypes = [C.c_void_p]
        lib.psref_morton_encode.restype = C.c_uint32
        lib.psref_morton_encode.argtypes = [C.c_uint32] * 3
        lib.psref_tree_nodes.restype = C.c_size_t
        lib.psref_tree_nodes.argtypes = [C.c_void_p]
        lib.psref_tree_dump.restype = C.c_size_t
        lib.psref_tree_dump.argtypes = [C.c_void_p, C.c_size_t] + [C.c_void_p] * 9
        lib.psref_m2l_pair.restype = C.c_int
        lib.psref_m2l_pair.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_float, C.c_void_p]
        lib.psref_p2p_pair.argtypes = [C.POINTER(ParticleArrs)] + [C.c_uint32] * 4
        self.lib = lib
        self.ctx_size = lib.psref_ctx_size()

    # -- public API -------------------------------------------------------
    def buffer_size(self, max_particles: int, n_nodes_hint: int | None = None) -> int:
        """Caller buffer that fits ctx + radix temps + node arena + locals +
        the scatter buffers (polesitter.h:1716-1752, :1632-1634)."""
        nodes = n_nodes_hint if n_nodes_hint is not None else 4 * max_particles + 4096
        return (self.ctx_size + 64 + 24 * max_particles + 80 * nodes
                + 40 * 98560 + (1 << 20))

    def prepare(self, p):
        arrs = arrs_of(p)
        codes = np.zeros(p.n, np.uint32)
        mn, mx, rg = C.c_float(), C.c_float(), C.c_float()
        rc = self.lib.psref_prepare(C.byref(arrs), _ptr(codes), C.byref(mn),
                                    C.byref(mx), C.byref(rg))
        return rc, codes, mn.value, mx.value, rg.value

    def tick(self, p, theta: float = 2.0, thrd_cnt: int = 4, dump_tree: bool = False,
             buff_size: int | None = None):
        """One ``ps_prepare_particles`` + ``ps_calc_forces`` on ``p`` (mutated in
        place, exactly as the reference mutates the caller's arrays).  Returns
        a dict with codes, bbox and (optionally) the canonical tree table."""
        size = buff_size or self.buffer_size(p.n)
        buf = np.zeros(size, np.uint8)
        cfg = Config(_ptr(buf), size, p.n, theta, thrd_cnt)
        ctx = C.c_void_p()
        rc = self.lib.psref_init(C.byref(ctx), C.byref(cfg))
        if rc != 0:
            raise RuntimeError(f"ps_init failed: {rc}")
        try:
            rc, codes, mn, mx, rg = self.prepare(p)
            if rc != 0:
                raise RuntimeError(f"ps_prepare_particles failed: {rc}")
            f32 = np.float32
            rc_ = f32(mn) + f32(rg) / f32(2.0)
            hw = f32(rg) / f32(2.0)
            arrs = arrs_of(p)
            rc2 = self.lib.psref_calc(ctx, C.byref(arrs), _ptr(codes), rc_, rc_, rc_, hw)
            if rc2 != 0:
                raise RuntimeError(f"ps_calc_forces failed: {rc2}")
            out = {"codes": codes, "min": mn, "max": mx, "range": rg,
                   "root_c": float(rc_), "root_hw": float(hw)}
            if dump_tree:
                out["tree"] = self.tree(ctx)
            return out
        finally:
            self.lib.psref_destroy(ctx)
            del buf

    def tree(self, ctx) -> dict:
        n = self.lib.psref_tree_nodes(ctx)
        t = {k: np.zeros(n, dt) for k, dt in (
            ("depth", np.int32), ("start", np.uint32), ("count", np.uint32),
            ("leaf", np.uint32), ("nchild", np.uint32), ("octant", np.int32))}
        geo = np.zeros((n, 4), np.float32)
        mp = np.zeros((n, 4), np.float32)
        loc = np.zeros((n, 4), np.float32)
        got = self.lib.psref_tree_dump(ctx, n, _ptr(t["depth"]), _ptr(t["start"]),
                                       _ptr(t["count"]), _ptr(t["leaf"]),
                                       _ptr(t["nchild"]), _ptr(t["octant"]),
                                       _ptr(geo), _ptr(mp), _ptr(loc))
        assert got == n
        t.update(geo=geo, mp=mp, loc=loc)
        return t

    def m2l_pair(self, tgt_geo, src_geo, src_mp, theta):
        tg = np.asarray(tgt_geo, np.float32)
        sg = np.asarray(src_geo, np.float32)
        sm = np.asarray(src_mp, np.float32)
        out = np.zeros(4, np.float32)
        hit = self.lib.psref_m2l_pair(_ptr(tg), _ptr(sg), _ptr(sm), theta, _ptr(out))
        return bool(hit), out
