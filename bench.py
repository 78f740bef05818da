#!/usr/bin/env python
"""Benchmark of the polesitter FMM tick on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

A step is one tick exactly as the reference's callers run it
(tests/benchmark.c:175-184, README.md:74-88): ps_prepare_particles +
ps_calc_forces on N = 1,048,576 equal-mass Plummer particles (a = 1, radii
truncated at 10a, seeded), theta = 2 -- the single-GPU configuration the
headline metric is quoted on.  Each step starts from the same unsorted
particle order (the tick sorts the caller's arrays in place) and with L2
flushed (the 20 MB of inputs fit in the 126 MB L2); both happen outside the
timed step.

Reported (one JSON line on rank 0):
  value      ticks/s of the whole job, device-resident arrays (all ranks)
  e2e        ticks/s through the same C ABI with pinned HOST arrays, the
             host<->device copies inside each step
  roofline   the dominant kernel (the leaf pass of the interaction kernel:
             MAC + M2L + L2L + P2P + L2P), FP32-bound, from its CUDA-event
             time and the algorithmic flop count of the step
  accuracy   relative force error against an FP64 direct sum on the GPU
             for 4096 sampled particles
  cpu_baseline  the reference's own threaded CPU tick (oracle/_ref) on the
             same workload, timed on this host's cores
With --gpus N > 1 every rank runs an independent replica (the path has no
exchange step on one system): weak scaling, value = N x ticks / max time.

--impl reference times the reference's CPU implementation of the same tick
(the unmodified header compiled by oracle/build_ref.sh) with all host threads.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ticks/s at N=1M, learned-closure vs plain GPU FMM at equal 1e-3 force error"
UNIT = "ticks/s"
N_DEFAULT = 1 << 20
THETA = 2.0
SEED = 42
WORKLOAD = ("plain FMM tick (ps_prepare_particles + ps_calc_forces), Plummer sphere "
            "N=1,048,576, a=1, r<=10a, equal mass 1/N, theta=2, float32 SoA")
KERNELS_PER_TICK = 35  # 2 prepare + 6 sort + gather + write-back + 4 tree + 11 upward + 10 traversal
# DRAM bytes (read + write) of one leaf-pass launch at this workload, from the
# ncu capture summarised in profiles/traversal_leaf_plummer1m.md
LEAF_PASS_DRAM_BYTES = 254.3e6
FLOP_M2L = 35   # per M2L pair: polesitter.h:1065-1092
FLOP_P2P = 20   # per particle pair: polesitter.h:1424-1444


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--theta", type=float, default=THETA)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def plummer(n):
    from polesitter_b200 import workloads as W
    return W.plummer(n, SEED)


def cpu_reference_ticks(p0, ticks, warmup, theta):
    """Time the reference's own tick (oracle/_ref, all host threads);
    fall back to the oracle port, single-threaded, if that build is absent."""
    cores = os.cpu_count() or 1
    from oracle import refbind
    if refbind.available(""):
        ref = refbind.RefLib("")
        run = lambda p: ref.tick(p, theta=theta, thrd_cnt=cores)  # noqa: E731
        kind, used = "reference", cores
    else:
        from oracle.oracle import Oracle
        o = Oracle()
        run = lambda p: o.tick(p, theta=theta, want_tree=False)  # noqa: E731
        kind, used = "port", 1
    for _ in range(warmup):
        run(p0.copy())
    times = []
    for _ in range(ticks):
        p = p0.copy()
        t0 = time.perf_counter()
        run(p)
        times.append(time.perf_counter() - t0)
    return {"value": len(times) / sum(times), "unit": UNIT, "cores": used, "kind": kind,
            "sample": f"{len(times)} full ticks of the benchmark workload (N={p0.n}) after "
                      f"{warmup} warm-up, thrd_cnt={used}; median {statistics.median(times):.3f} s/tick"}


def run_reference(args):
    rank, _, world = dist_info()
    if rank != 0:
        return 0
    p0 = plummer(args.n)
    base = cpu_reference_ticks(p0, args.steps, args.warmup, args.theta)
    line = {"metric": METRIC, "value": base["value"], "unit": UNIT, "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 / base["value"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Plummer sphere)",
            "config": {"workload": WORKLOAD, "n": args.n, "theta": args.theta},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args):
    import torch
    import polesitter_b200 as P

    rank, local_rank, world = dist_info()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    n = args.n
    p0 = plummer(n)
    dev = torch.device("cuda", local_rank)

    class Arrays:
        pass

    def device_arrays():
        a = Arrays()
        for k in ("x", "y", "z", "mass", "fx", "fy", "fz"):
            setattr(a, k, torch.from_numpy(getattr(p0, k).copy()).to(dev))
        a.id = torch.from_numpy(p0.id.view(np.int32).copy()).to(dev)
        return a

    d = device_arrays()
    pristine = device_arrays()
    codes = torch.zeros(n, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def reset():
        for k in ("x", "y", "z", "mass", "id"):
            getattr(d, k).copy_(getattr(pristine, k))
        flush.fill_(1)
        torch.cuda.synchronize()

    ctx = P.Context(n, theta=args.theta)
    # one untimed tick with per-node interaction counters on: the algorithmic
    # work of this workload (it is identical in every timed step)
    ctx.set_option(P.OPT_DEBUG, 1)
    reset()
    ctx.tick(d, codes)
    st = ctx.stats()
    tree = ctx.tree()
    leaf = tree["nchild"] == 0
    m2l_leaf = int(tree["m2l_cnt"][leaf].sum())
    m2l_all = int(st["m2l_pairs"])
    p2p_inter = int(st["p2p_interactions"])
    ctx.set_option(P.OPT_DEBUG, 0)
    ctx.set_option(P.OPT_TIMING, 1)

    for _ in range(args.warmup):
        reset()
        ctx.tick(d, codes)

    step_s, leaf_ms, internal_ms, calc_ms = [], [], [], []
    gpu_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local_rank)).split(",")[0]) \
        if os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0].isdigit() else local_rank
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(gpu_index) as clocks:
        time.sleep(0.5)  # let nvidia-smi start sampling before the timed steps
        for _ in range(args.steps):
            reset()
            t0 = time.perf_counter()
            ctx.tick(d, codes)  # synchronous: returns after the forces are written
            step_s.append(time.perf_counter() - t0)
            tm = ctx.timing()
            leaf_ms.append(tm["leaves"])
            internal_ms.append(tm["internal"])
            calc_ms.append(tm["tick"])
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    from polesitter_b200.replicas import job_time
    total = job_time(sum(step_s), dev)
    value = world * args.steps / total

    # accuracy of the last tick against an FP64 direct sum (GPU) on 4096
    # sampled particles
    rng = np.random.default_rng(7)
    sample = np.sort(rng.choice(n, size=min(4096, n), replace=False)).astype(np.uint32)
    host = Arrays()
    for k in ("x", "y", "z", "mass", "fx", "fy", "fz"):
        setattr(host, k, getattr(d, k).cpu().numpy())
    host.id = d.id.cpu().numpy().view(np.uint32)
    f64 = ctx.direct_f64(host, sample)
    f32 = np.stack([host.fx[sample], host.fy[sample], host.fz[sample]], axis=1).astype(np.float64)
    rel = np.linalg.norm(f32 - f64, axis=1) / np.linalg.norm(f64, axis=1)
    accuracy = {"vs": "FP64 direct sum on the GPU, 4096 sampled particles",
                "median_rel": float(np.median(rel)),
                "rms_rel": float(np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum())),
                "max_rel": float(rel.max())}

    # e2e: the same tick through the public API with pinned host buffers
    e2e_steps = max(1, min(args.e2e_steps, args.steps))
    pin = {k: torch.empty(n, dtype=torch.float32 if k != "id" else torch.int32,
                          pin_memory=True).numpy() for k in
           ("x", "y", "z", "mass", "fx", "fy", "fz", "id")}
    pin_codes = torch.empty(n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    hp = Arrays()
    for k, v in pin.items():
        setattr(hp, k, v.view(np.uint32) if k == "id" else v)

    def reset_host():
        for k in ("x", "y", "z", "mass"):
            getattr(hp, k)[:] = getattr(p0, k)
        hp.id[:] = p0.id
        flush.fill_(1)
        torch.cuda.synchronize()

    reset_host()
    ctx.tick(hp, pin_codes)  # allocates the host-path mirrors
    e2e_s = []
    for _ in range(e2e_steps):
        reset_host()
        t0 = time.perf_counter()
        ctx.tick(hp, pin_codes)
        e2e_s.append(time.perf_counter() - t0)
    e2e_total = job_time(sum(e2e_s), dev)
    e2e = {"value": world * e2e_steps / e2e_total, "unit": UNIT,
           # prepare: x,y,z in / codes out; calc: x,y,z,mass,id,codes in /
           # x,y,z,mass,id,codes,fx,fy,fz out -- 4 bytes per particle each
           "h2d_bytes_per_step": 4 * n * (3 + 6), "d2h_bytes_per_step": 4 * n * (1 + 9),
           "steps": e2e_steps, "ms_per_step": 1000.0 * e2e_total / e2e_steps}

    peaks, peak_src = measured_peaks()
    props = torch.cuda.get_device_properties(dev)
    fp32_peak = props.multi_processor_count * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
    leaf_s = statistics.mean(leaf_ms) / 1e3
    flops_leaf = FLOP_M2L * m2l_leaf + FLOP_P2P * p2p_inter
    achieved = flops_leaf / leaf_s / 1e12
    roofline = {"kernel": "k_trav<MODE_LEAF> (leaf pass: MAC+M2L+L2L+P2P+L2P)",
                "bound": "fp32", "achieved": achieved, "peak": fp32_peak / 1e12,
                "unit": "TFLOP/s", "frac": achieved * 1e12 / fp32_peak,
                "peak_source": f"computed: {props.multi_processor_count} SMs x 128 FP32 lanes x 2 x "
                               f"{peaks.get('sm_max_mhz', 1965.0)} MHz (sm_max_mhz, {peak_src}); "
                               "no measured FP32 peak exists",
                "traffic": LEAF_PASS_DRAM_BYTES,
                "traffic_note": "dram read+write bytes per launch, ncu capture of this workload",
                "algorithmic_flop": flops_leaf,
                "counts": {"m2l_pairs_leaf_targets": m2l_leaf, "p2p_particle_pairs": p2p_inter},
                "launch_ms": leaf_s * 1e3}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Plummer sphere)",
            "config": {"workload": WORKLOAD, "n": n, "theta": args.theta,
                       "per_gpu": "independent replica of the workload",
                       "l2": "flushed (256 MB write) and inputs reset before every step, untimed",
                       "timing": "wall clock around the synchronous API call, max over ranks"},
            "device_ms": {"calc_forces": statistics.mean(calc_ms),
                          "internal_levels": statistics.mean(internal_ms),
                          "leaf_pass": statistics.mean(leaf_ms)},
            "interactions": {"m2l_pairs": m2l_all, "p2p_particle_pairs": p2p_inter},
            "accuracy": accuracy, "e2e": e2e, "roofline": roofline,
            "clocks": clocks.summary(), "gpu_launches": KERNELS_PER_TICK * args.steps}

    ctx.destroy()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference_ticks(p0, ticks=3, warmup=1, theta=args.theta)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
