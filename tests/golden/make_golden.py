"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the unmodified polesitter tick (the reference header compiled with its
own flags into oracle/_ref/libpsref.so by oracle/build_ref.sh) on small
seeded workloads and stores inputs and outputs:

    inputs : x, y, z, mass (float32), theta
    outputs: Morton codes, min/max/range, sorted x/y/z/mass, ids,
             forces fx/fy/fz (sorted order) and the canonical tree table
             (level-major, Morton order per level: depth, start, count,
             leaf, nchild, octant, centre + half width, multipole, local_exp)

Usage (needs the reference checkout, i.e. only where oracle/_ref exists):
    python tests/golden/make_golden.py
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.refbind import RefLib  # noqa: E402
from polesitter_b200 import workloads as W  # noqa: E402

CASES = {
    "uniform1024_t2": (lambda: W.uniform_cube(1024, 1), 2.0),
    "uniform1024_t1": (lambda: W.uniform_cube(1024, 1), 1.0),
    "lcg_uniform512_t2": (lambda: W.lcg_uniform(512), 2.0),
    "lcg_clusters512_t2": (lambda: W.lcg_two_clusters(512), 2.0),
    "ragged1003_t2": (lambda: W.uniform_cube(1003, 5), 2.0),
    "tiny7_t2": (lambda: W.uniform_cube(7, 9), 2.0),
    "pair2_t2": (lambda: W.uniform_cube(2, 9), 2.0),
    "plummer4097_t2": (lambda: W.plummer(4097, 11), 2.0),
    "bench_cube3000_t1": (lambda: W.benchmark_cube(3000), 1.0),
    "sqrt12_1024": (lambda: W.uniform_cube(1024, 3), 3.4641),
}


def main():
    ref = RefLib("")
    for name, (gen, theta) in CASES.items():
        p = gen()
        inp = p.copy()
        r = ref.tick(p, theta=theta, thrd_cnt=4, dump_tree=True)
        t = r["tree"]
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            theta=np.float32(theta), x_in=inp.x, y_in=inp.y, z_in=inp.z, mass_in=inp.mass,
            codes=r["codes"], bbox=np.array([r["min"], r["max"], r["range"]], np.float32),
            x=p.x, y=p.y, z=p.z, mass=p.mass, id=p.id, fx=p.fx, fy=p.fy, fz=p.fz,
            t_depth=t["depth"], t_start=t["start"], t_count=t["count"], t_leaf=t["leaf"],
            t_nchild=t["nchild"], t_octant=t["octant"], t_geo=t["geo"], t_mp=t["mp"],
            t_loc=t["loc"])
        print(f"{name}: n={p.n} nodes={len(t['depth'])}")


if __name__ == "__main__":
    main()
