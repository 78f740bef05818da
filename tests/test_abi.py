"""The drop-in boundary without a GPU: the library builds and loads, exports
every function its headers declare, keeps the reference's struct layouts and
result codes, and rejects bad arguments on the host exactly where the
reference does (polesitter.h:1700, :1843, :1914, :2173)."""

from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import polesitter_b200 as P
from conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")


def _declared_functions():
    names = set()
    for h in ("polesitter.h", "polesitter_b200.h"):
        src = open(os.path.join(INCLUDE, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"\b(ps_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_builds_and_exports_every_declared_symbol():
    from polesitter_b200.build import build
    build()
    lib = P.lib()
    declared = _declared_functions()
    assert {"ps_init", "ps_prepare_particles", "ps_calc_forces", "ps_destroy"} <= set(declared)
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", P.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (ps_[a-z0-9_]+)", out))
    assert set(declared) == exported


LAYOUT_PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "polesitter.h"
int main(void) {
    printf("%zu %zu %zu %zu %zu %zu\n", sizeof(ps_config_t), offsetof(ps_config_t, theta),
           offsetof(ps_config_t, thrd_cnt), sizeof(ps_particle_arrs_t),
           offsetof(ps_particle_arrs_t, id), offsetof(ps_particle_arrs_t, cnt));
    printf("%d %d %d %d %d\n", PS_OK, PS_EOOM, PS_EINVAL, PS_ETHRD, PS_EALLOC);
    return 0;
}
"""


def _probe_layout(include_dir):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write(LAYOUT_PROBE)
        subprocess.run(["gcc", "-std=c99", "-I" + include_dir, src, "-o", exe], check=True)
        return subprocess.run([exe], capture_output=True, text=True, check=True).stdout


def test_struct_layout_and_result_codes_match_reference():
    ours = _probe_layout(INCLUDE)
    ref_root = os.environ.get("PS_REFERENCE_ROOT",
                              os.path.join(os.path.dirname(ROOT), "reference"))
    ref_dir = os.path.join(ref_root, "src")
    if not os.path.exists(os.path.join(ref_dir, "polesitter.h")):
        # the reference's layout, restated: ps_config_t (polesitter.h:304-310)
        # and ps_particle_arrs_t (:312-322) on LP64, enum values (:294-300)
        assert ours.split() == "40 24 32 72 56 64 0 -1 -2 -3 -4".split()
        return
    assert ours == _probe_layout(ref_dir)


def test_ctypes_mirror_layout():
    assert C.sizeof(P.Config) == 40 and C.sizeof(P.ParticleArrs) == 72


def _arrs(n=4):
    class A:
        pass
    a = A()
    for k in ("x", "y", "z", "mass", "fx", "fy", "fz"):
        setattr(a, k, np.zeros(n, np.float32))
    a.id = np.arange(n, dtype=np.uint32)
    return a


def test_init_argument_checks():
    L = P.lib()
    ctx = C.c_void_p()
    assert L.ps_init(None, None) == P.PS_EINVAL
    assert L.ps_init(C.byref(ctx), None) == P.PS_EINVAL
    cfg = P.Config(None, 1 << 20, 16, 2.0, 1)
    assert L.ps_init(C.byref(ctx), C.byref(cfg)) == P.PS_EINVAL  # no buffer
    buf = np.zeros(64, np.uint8)
    cfg = P.Config(buf.ctypes.data, 64, 16, 2.0, 1)
    assert L.ps_init(C.byref(ctx), C.byref(cfg)) == P.PS_EINVAL  # smaller than the context
    # the reference's sizing rule for its radix temporaries (:1716-1723)
    size = L.ps_b200_context_size() + 64
    buf = np.zeros(size, np.uint8)
    cfg = P.Config(buf.ctypes.data, size, 1000, 2.0, 1)
    assert L.ps_init(C.byref(ctx), C.byref(cfg)) == P.PS_EOOM


def test_prepare_calc_destroy_argument_checks():
    L = P.lib()
    a = _arrs()
    arrs = P.arrs_of(a)
    codes = np.zeros(4, np.uint32)
    f = C.c_float()
    assert L.ps_prepare_particles(None, codes.ctypes.data, C.byref(f), C.byref(f),
                                  C.byref(f)) == P.PS_EINVAL
    assert L.ps_prepare_particles(C.byref(arrs), None, C.byref(f), C.byref(f),
                                  C.byref(f)) == P.PS_EINVAL
    empty = P.arrs_of(a, n=0)
    assert L.ps_prepare_particles(C.byref(empty), codes.ctypes.data, C.byref(f), C.byref(f),
                                  C.byref(f)) == P.PS_EINVAL
    assert L.ps_calc_forces(None, C.byref(arrs), codes.ctypes.data, 0, 0, 0, 1) == P.PS_EINVAL
    fake_ctx = np.zeros(4096, np.uint8)  # not an initialised context
    assert L.ps_calc_forces(fake_ctx.ctypes.data, C.byref(arrs), codes.ctypes.data,
                            0, 0, 0, 1) == P.PS_EINVAL
    assert L.ps_destroy(None) == P.PS_EINVAL
    assert L.ps_destroy(fake_ctx.ctypes.data) == P.PS_EINVAL
    assert L.ps_b200_set_morton_variant(7) == P.PS_EINVAL
    assert L.ps_b200_set_morton_variant(0) == P.PS_OK


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure path")
def test_init_without_gpu_reports_device_error():
    with pytest.raises(P.PolesitterError) as e:
        P.Context(1024)
    assert e.value.code in (P.PS_EDEVICE, P.PS_EALLOC)


def test_product_does_not_load_the_oracle():
    # the product library links nothing from oracle/
    out = subprocess.run(["ldd", P.LIB_PATH], capture_output=True, text=True).stdout
    assert "psoracle" not in out and "psref" not in out
    for src in os.listdir(os.path.join(ROOT, "polesitter_b200")):
        if src.endswith(".py"):
            text = open(os.path.join(ROOT, "polesitter_b200", src)).read()
            assert "import oracle" not in text and "from oracle" not in text, src
