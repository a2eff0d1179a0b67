#!/usr/bin/env python
"""Throughput of SIMP's per-step SPH hot path on B200: particle-steps/s.

Workload (one GPU): the plain FP64 drop-in configuration, a 256 km basin of
262,144 particles (512 x 512 lattice, dx = 500 m, seeded jitter +/-0.05 dx),
cubic-spline kernel, Hibler VP rheology, wind 10 m/s along +x, wall on +x,
fixed dt = 1 s.  One timed step is one predictor-corrector step (two
right-hand-side evaluations) of the whole basin, state resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun): every rank advances its own replica basin (independent
basins, no exchange: weak scaling); the job value is all ranks' particle-steps
over the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time
from datetime import timedelta

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "cfg2 plain FP64: 262,144 particles (512x512 lattice, dx=500 m, 256 km basin), 1 predictor-corrector step per timed step"
METRIC = "particle-steps/s"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="target CPU time of the oracle baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world, backend):
    if world <= 1:
        return None
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return dist


def job_time_ms(dist, local_ms: float, device: str = "cuda") -> float:
    """Slowest rank's device time (every rank takes the same collective)."""
    if dist is None:
        return float(local_ms)
    import torch
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world: int, particles: int, steps: int, job_ms: float) -> float:
    """Whole-job particle-steps/s: all ranks' work over the slowest rank."""
    return world * particles * steps / (job_ms / 1e3)


# --- clocks sampled during the timed region --------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(gpu_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


# --- CPU oracle (the reference's algorithm, restated; no Fortran here) -----

def oracle_rate(basin, target_s: float, max_steps: int, warmup: int = 0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    o = O.Oracle.from_basin(basin)
    if warmup:
        o.step(warmup)
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        o.step(1)
        steps += 1
        if time.perf_counter() - t0 >= target_s:
            break
    el = time.perf_counter() - t0
    o.close()
    return basin.n * steps / el, threads, steps, el


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    from simp_b200 import basins
    b = basins.cfg2()
    # each timed step is one predictor-corrector step of the full basin on
    # the host cores; the run stops early if it would exceed ~3 minutes
    v, threads, steps, el = oracle_rate(b, target_s=180.0, max_steps=args.steps, warmup=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": WORKLOAD, "particles": b.n},
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{steps} predictor-corrector steps of the full 262,144-particle "
                                   f"basin after {args.warmup} warm-up steps, OpenMP threads={threads}; "
                                   "C++ FP64 restatement of the Fortran reference (no Fortran compiler on the box)"},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --- our path -------------------------------------------------------------------

def run_ours(args):
    import numpy as np
    import torch
    world, rank, local = dist_env()
    dist = init_dist(world, "nccl")
    torch.cuda.set_device(local)
    from simp_b200 import basins, roofline
    from simp_b200.simp import Simp
    lib = None

    b = basins.cfg2()
    sim = Simp.from_basin(b)
    lib = sim.lib
    stream = torch.cuda.ExternalStream(lib.simp_gpu_stream(sim.h))
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    sim.time_integration(args.warmup)
    lib.simp_gpu_profile(sim.h, 1)
    launches0 = lib.simp_gpu_kernel_launches(sim.h)
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    time.sleep(0.3)
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()                      # evict L2 between timed steps
        ev0[k].record(stream)
        sim.time_integration(1)
        ev1[k].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    launches = lib.simp_gpu_kernel_launches(sim.h) - launches0
    kms = (ctypes.c_double * 5)()
    nst = ctypes.c_int64()
    lib.simp_gpu_kernel_times(sim.h, kms, 5, ctypes.byref(nst))
    lib.simp_gpu_profile(sim.h, 0)
    kernel_ms = list(kms)
    # device time of the K steps: sum of in-graph kernel times per step
    dev_ms = sum(kernel_ms)
    outer_ms = sum(a.elapsed_time(z) for a, z in zip(ev0, ev1))
    dev_ms_max = job_time_ms(dist, dev_ms)
    value = job_value(world, b.n, args.steps, dev_ms_max)

    # roofline of the dominant kernel
    peak, peak_src = roofline.hbm_peak(ROOT)
    names = roofline.KERNELS
    top = max(range(5), key=lambda k: kernel_ms[k])
    avg_ms = kernel_ms[top] / max(1, nst.value)
    alg = roofline.BYTES_PER_PARTICLE[names[top]] * b.n
    achieved = alg / (avg_ms / 1e3) / 1e9
    traffic = profile_traffic(names[top])

    # end to end through the C ABI with host buffers: upload the state from
    # pinned host memory, one step, download the state
    e2e = run_e2e(sim, b, stream, min(args.e2e_steps, args.steps), dist)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, threads, steps, el = oracle_rate(b, target_s=args.cpu_seconds, max_steps=1000)
        cpu = {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
               "sample": f"first {steps} predictor-corrector steps of the same 262,144-particle basin "
                         f"({el:.1f} s), C++ FP64 restatement of the reference, OpenMP threads={threads}"}
    sim.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles": b.n, "wall_particles": b.nb,
                       "precision": "fp64", "l2": "flushed between timed steps (256 MiB write)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single basin",
                       "outer_event_ms_per_step": outer_ms / args.steps},
            "roofline": {"bound": "hbm", "kernel": names[top], "achieved": achieved, "peak": peak,
                         "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured" else "fallback",
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "alg_bytes_per_launch": alg, "avg_launch_ms": avg_ms,
                         "step_alg_bytes_per_particle": roofline.STEP_BYTES_PER_PARTICLE,
                         "kernel_ms_per_step": {n: kernel_ms[k] / max(1, nst.value) for k, n in enumerate(names)}},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def profile_traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic_cfg2.txt")
    try:
        with open(p) as f:
            v = json.load(f).get(kernel)
        return None if v is None else float(v)
    except Exception:
        return None


def run_e2e(sim, b, stream, nsteps, dist):
    import numpy as np
    import torch
    n, nb = b.n, b.nb

    def pinned(shape):
        return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()

    host = {k: pinned((n, 2)) for k in ("x", "vx")}
    for k in ("mass", "rho", "hsml", "A", "h"):
        host[k] = pinned((n,))
    st = sim.get_state()
    for k in host:
        host[k][...] = st[k]
    xb, massb = pinned((nb, 2)), pinned((nb,))
    xb[...] = b.xb
    massb[...] = b.massb
    dt = b.params.dt
    t_now = st["current_time"]
    lib = sim.lib
    from simp_b200 import _lib as L
    P = L.dptr
    dtc, tc = ctypes.c_double(), ctypes.c_double()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(nsteps):
        rc = lib.simp_gpu_set_state(sim.h, n, P(host["x"]), P(host["vx"]), P(host["mass"]), P(host["rho"]),
                                    P(host["hsml"]), P(host["A"]), P(host["h"]), nb, P(xb), P(massb),
                                    float(dt), float(t_now))
        assert rc == 0, lib.simp_gpu_last_error(sim.h)
        rc = lib.simp_gpu_step(sim.h, 1, ctypes.byref(tc), ctypes.byref(dtc))
        assert rc == 0, lib.simp_gpu_last_error(sim.h)
        rc = lib.simp_gpu_get_state(sim.h, P(host["x"]), P(host["vx"]), P(host["mass"]), P(host["rho"]),
                                    P(host["hsml"]), P(host["A"]), P(host["h"]), ctypes.byref(dtc),
                                    ctypes.byref(tc))
        assert rc == 0, lib.simp_gpu_last_error(sim.h)
        t_now, dt = tc.value, dtc.value
    e1.record(stream)
    torch.cuda.synchronize()
    ms = job_time_ms(dist, e0.elapsed_time(e1))
    world = dist.get_world_size() if dist else 1
    h2d = n * (2 * 16 + 5 * 8) + nb * 24
    d2h = n * (2 * 16 + 5 * 8) + 16
    return {"value": world * n * nsteps / (ms / 1e3), "unit": METRIC, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": nsteps,
            "path": "simp_gpu_set_state (pinned host) + simp_gpu_step(1) + simp_gpu_get_state (pinned host)"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
