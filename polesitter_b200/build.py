"""Build libpolesitter_b200.so in-tree for sm_100a.

    python -m polesitter_b200.build [--force] [--verbose]

Every CUDA source is compiled by nvcc for ``-gencode
arch=compute_100a,code=sm_100a`` with ``-lineinfo``; the C99 host layer by
gcc; both are linked into ``polesitter_b200/libpolesitter_b200.so`` (static
cudart), which exports the reference's four functions (include/polesitter.h)
and the ps_b200_* extensions (include/polesitter_b200.h).  Objects go to
``polesitter_b200/_build`` and are rebuilt only when a source or header is
newer.
"""

from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libpolesitter_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
                     "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
CC_FLAGS = ["-std=c99", "-O2", "-fPIC", "-Wall", "-Wextra", "-I" + os.path.join(ROOT, "include")]


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"command failed: {' '.join(cmd[:3])} ... (exit {r.returncode})")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return r


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    hdr_time = _newest(headers)
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(
                os.path.getmtime(src), hdr_time):
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            r = _run([NVCC] + NVCC_FLAGS + extra + ["-c", src, "-o", obj], verbose)
            if ptxas_info:
                print(r.stderr, flush=True)
    for src in sorted(glob.glob(os.path.join(HOST, "*.c"))):
        obj = os.path.join(BUILD, "host_" + os.path.basename(src)[:-2] + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(
                os.path.getmtime(src), hdr_time):
            _run(["gcc"] + CC_FLAGS + ["-c", src, "-o", obj], verbose)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs +
             ["-lpthread"], verbose)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print -Xptxas -v (forces rebuild)")
    a = ap.parse_args(argv)
    print(build(force=a.force or a.ptxas_info, verbose=a.verbose, ptxas_info=a.ptxas_info))


if __name__ == "__main__":
    main()
