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
    ap.add_argument("--e2e-steps", type=int, default=32)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="target CPU time of the oracle baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--forms", default="mixed,batched,served",
                    help="comma list of the other forms to measure on rank 0 ('' for none)")
    # enough requests, arriving fast enough, that the 150 GB budget binds
    # (about 97M resident particles of this size distribution)
    ap.add_argument("--served-requests", type=int, default=700)
    ap.add_argument("--served-rate", type=float, default=1000.0, help="Poisson arrival rate of the served stream (1/s)")
    ap.add_argument("--served-steps-scale", type=float, default=1.0,
                    help="factor on the requests' step counts U(100, 2000) (1: as the served workload states)")
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
    launches0 = lib.simp_gpu_kernel_launches(sim.h)
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    time.sleep(0.3)
    # the timed region: K back-to-back simp_gpu_step(1) calls as a host
    # makes them (each replays the step graph and returns time and dt), the
    # L2 flush enqueued between them outside the event pairs
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
    dev_ms = sum(a.elapsed_time(z) for a, z in zip(ev0, ev1))
    dev_ms_max = job_time_ms(dist, dev_ms)
    value = job_value(world, b.n, args.steps, dev_ms_max)

    # per-kernel split: the same K steps once more, with CUDA events
    # recorded inside the step graph around each kernel (this mode waits for
    # every step, so it is kept out of the timed region above)
    lib.simp_gpu_profile(sim.h, 1)
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        sim.time_integration(1)
    torch.cuda.synchronize()
    kms = (ctypes.c_double * 6)()
    nst = ctypes.c_int64()
    lib.simp_gpu_kernel_times(sim.h, kms, 6, ctypes.byref(nst))
    lib.simp_gpu_profile(sim.h, 0)
    kernel_ms = list(kms)[:5]
    sort_ms = kms[5]
    profiled_ms = (sum(kernel_ms) + sort_ms) / max(1, nst.value)

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
    lk = e2e["link"]
    # the serial floor: the step's copies at the link's plain rates around
    # the device-timed step, one after the other (get_state reads the fields
    # no step writes, here mass and hsml, while the step runs, so the
    # measured loop can come above it)
    floor_ms = lk["h2d_ms"] + lk["d2h_ms"] + dev_ms_max / args.steps
    lk["serial_floor_value"] = world * b.n / (floor_ms / 1e3)
    lk["e2e_frac_of_serial_floor"] = e2e["value"] / lk["serial_floor_value"]
    lk["d2h_bytes_during_step"] = b.n * 16

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, threads, steps, el = oracle_rate(b, target_s=args.cpu_seconds, max_steps=1000)
        cpu = {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
               "sample": f"first {steps} predictor-corrector steps of the same 262,144-particle basin "
                         f"({el:.1f} s), C++ FP64 restatement of the reference, OpenMP threads={threads}"}
    sim.close()
    forms = None
    # (the other forms are one-GPU measurements of rank 0; under torchrun the
    # other ranks would wait for them at the closing barrier, so they run
    # only at N = 1)
    if rank == 0 and world == 1 and args.forms:
        forms = run_forms(args, [f for f in args.forms.split(",") if f])
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles": b.n},
            "setup": {"wall_particles": b.nb, "precision": "fp64",
                      "l2": "flushed between timed steps (256 MiB write, outside the timed spans)",
                      "timing": "CUDA events on the context stream around each of K simp_gpu_step(1) calls",
                      "parallelism": f"replicas x{world}" if world > 1 else "single basin",
                      "profiled_kernel_sum_ms_per_step": profiled_ms},
            "roofline": {"bound": "hbm", "kernel": names[top], "achieved": achieved, "peak": peak,
                         "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured" else "fallback",
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "fp64_pipe_frac": profile_traffic(names[top], "fp64_pipe_frac"),
                         "fp64_pipe_source": "ncu sm__pipe_fp64_cycles_active of the pass (secondary roof), "
                                             "profiles/pair_passes_cfg2_fp64.md",
                         "alg_bytes_per_launch": alg, "avg_launch_ms": avg_ms,
                         "step_alg_bytes_per_particle": roofline.STEP_BYTES_PER_PARTICLE,
                         "kernel_ms_per_step": {**{n: kernel_ms[k] / max(1, nst.value) for k, n in enumerate(names)},
                                                "sort": sort_ms / max(1, nst.value)},
                         "kernel_timing": "in-graph CUDA events, a second pass of the same K steps"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clk,
            "forms": forms,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# --- the other forms: mixed single instance, batched ensemble, served stream -

def _device_steps(sim_step, stream, nsteps):
    """Device time (ms) of nsteps steps issued by sim_step(k) in one call."""
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    sim_step(nsteps)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def run_forms(args, which):
    import numpy as np
    import torch
    from simp_b200 import basins, serve
    from simp_b200.params import PREC_FP64, PREC_MIXED
    from simp_b200.simp import Batch, Simp
    out = {}
    if "mixed" in which:
        # 1,048,576-particle vortex basin, mixed precision, against FP64 on
        # the same seed: one right-hand side and a 3-step trajectory
        b = basins.cfg3()
        b.vx = basins.smooth_velocity(b.x, b.L, amp=0.3, seed=14)   # not at rest: the rheology is live
        p64 = b.params.copy()
        p64.precision = PREC_FP64
        g32 = Simp.from_basin(b)
        g64 = Simp.from_basin(b, p64)
        r32, r64 = g32.single_step(600.0), g64.single_step(600.0)
        rel = lambda a, c: float(np.linalg.norm(a - c) / max(np.linalg.norm(c), 1e-300))
        err_rhs = {k: rel(r32[k], r64[k]) for k in ("dvxdt", "dhdt")}
        res = {}
        for name, g in (("mixed", g32), ("fp64", g64)):
            g.set_state(b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h, b.xb, b.massb, b.params.dt, 0.0)
            g.time_integration(args.warmup)
            st = torch.cuda.ExternalStream(g.lib.simp_gpu_stream(g.h))
            ms = _device_steps(g.time_integration, st, args.steps)
            res[name] = {"value": b.n * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps}
        g32.set_state(b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h, b.xb, b.massb, b.params.dt, 0.0)
        g64.set_state(b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h, b.xb, b.massb, b.params.dt, 0.0)
        # the workload's own length: 2,000 steps of both forms on the same
        # seed, errors recorded along the way
        traj = {}
        done = 0
        for mark in (50, 500, 2000):
            g32.time_integration(mark - done)
            g64.time_integration(mark - done)
            done = mark
            s32, s64 = g32.get_state(), g64.get_state()
            traj[str(mark)] = {k: rel(s32[k], s64[k]) for k in ("vx", "h", "A")}
        g32.close()
        g64.close()
        out["mixed_single_instance"] = {
            "workload": "1,048,576 particles (1024x1024, dx=250 m), 4 walls, vortex 15 m/s, smoothed h/A, dt=1e-5 s",
            "metric": METRIC, "value": res["mixed"]["value"], "ms_per_step": res["mixed"]["ms_per_step"],
            "fp64_same_basin": res["fp64"], "steps": args.steps,
            "l2": "not flushed: one call of K steps; per-step working set > 126 MB L2",
            "err_vs_fp64": {"rhs_rel_l2": err_rhs,
                            "traj_rel_l2_by_step": traj,
                            "bound": "1e-4 relative L2 (velocity, thickness) against FP64 on the same seed",
                            "dt_s": b.params.dt, "vp_dt_bound_s": basins.vp_dt_bound(b.dx),
                            "note": "dt under the reference's viscous-plastic bound (time_step.f90:155); above "
                                    "it any rounding difference, a reordered FP64 sum included, grows every step"}}
    if "batched" in which:
        # 64 uneven basins (log-uniform 4,096..262,144 particles), mixed
        bs = basins.cfg4(64, steps=500)
        ntot = sum(x.n for x in bs)
        with Batch(bs[0].params, ntot, sum(x.nb for x in bs), 64) as bt:
            for x in bs:
                bt.add(x)
            bt.step(args.warmup)
            st = torch.cuda.ExternalStream(bt.lib.simp_gpu_stream(bt.h))
            l0 = bt.kernel_launches()
            ms = _device_steps(bt.step, st, args.steps)
            launches = bt.kernel_launches() - l0
            # the kernels' own time of the same number of steps (in-graph
            # events): what separates it from the step time is the launch
            # gaps, the most a single persistent launch per sub-step could save
            bt.lib.simp_gpu_profile(bt.h, 1)
            bt.step(args.steps)
            kms = (ctypes.c_double * 6)()
            nst = ctypes.c_int64()
            bt.lib.simp_gpu_kernel_times(bt.h, kms, 6, ctypes.byref(nst))
            bt.lib.simp_gpu_profile(bt.h, 0)
            kernel_ms = sum(kms) / max(1, nst.value)
        out["batched_ensemble"] = {
            "workload": f"64 basins, {ntot} particles (log-uniform 4,096..262,144), dx=1 km, mixed, dt=1e-4 s",
            "metric": METRIC, "value": ntot * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
            "steps": args.steps, "launches_per_step": launches / args.steps,
            "kernel_ms_per_step": kernel_ms,
            "launch_gap_frac": max(0.0, 1.0 - kernel_ms / (ms / args.steps)),
            "l2": "not flushed: one call of K steps; working set > 126 MB L2"}
    if "served" in which:
        # offered load well above either arm's capacity (arrivals within a
        # fraction of a second), so the makespan measures capacity
        reqs = serve.sample_stream(args.served_requests, seed=5, rate_hz=args.served_rate,
                                   steps_scale=args.served_steps_scale)
        big = max(r.basin.n for r in reqs)
        with serve.Server(reqs[0].basin.params, 150e9, max_instances=1024, max_request_particles=big,
                          quantum_steps=32, spot_every=8) as srv:
            ids = [srv.submit(r) for r in reqs]
            srv.run()
            sst = srv.stats()
            per = [srv.request(i) for i in ids]
        lat = [q["completed_s"] - q["arrival_s"] for q in per]
        spots = [{"n": q["ntotal"], "steps": q["steps"], "err_v": q["err_v"], "err_h": q["err_h"]}
                 for q in per if q["spot_checked"]]
        ser = serve.serial_fp64(reqs)
        served_value = sst["particle_steps"] / sst["makespan_s"]
        out["served_stream"] = {
            "workload": (f"{len(reqs)} requests, Poisson {args.served_rate:g}/s, particles log-uniform 1,024..1,048,576, "
                         "steps U(100, 2000)" + (f" x {args.served_steps_scale}" if args.served_steps_scale != 1.0 else "") +
                         ", dx=1 km, dt=1e-4 s, mixed, HBM budget 150 GB, FP64 replica of every 8th request"),
            "budget_capacity_particles": sst["capacity_particles"],
            "peak_resident_frac_of_capacity": sst["peak_resident_particles"] / max(1.0, sst["capacity_particles"]),
            "metric": METRIC, "value": served_value, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "makespan_s": sst["makespan_s"],
            "particle_steps": sst["particle_steps"], "peak_resident_requests": sst["peak_resident_requests"],
            "peak_resident_particles": sst["peak_resident_particles"],
            "serial_fp64": ser, "speedup_vs_serial_fp64": served_value / ser["value"],
            "time_split_s": {k: sst[k] for k in ("admit_s", "step_s", "retire_s") if k in sst},
            "spot_checks": spots}
    return out


def profile_traffic(kernel: str, key: str | None = None):
    """DRAM bytes per launch (or, with key, another per-pass figure) from
    the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic_cfg2.txt")
    try:
        with open(p) as f:
            d = json.load(f)
        v = (d.get(key) or {}).get(kernel) if key else d.get(kernel)
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
    # the host arrays' pointers, taken once (a Fortran or C host passes them as they are)
    state_ptrs = [P(host[k]) for k in ("x", "vx", "mass", "rho", "hsml", "A", "h")]
    wall_ptrs = [P(xb), P(massb)]
    ptc, pdtc = ctypes.byref(tc), ctypes.byref(dtc)
    calls = {"set_state": [], "step": [], "get_state": []}
    clock = time.perf_counter
    for _ in range(nsteps):
        c0 = clock()
        rc = lib.simp_gpu_set_state(sim.h, n, *state_ptrs, nb, *wall_ptrs, float(dt), float(t_now))
        assert rc == 0, lib.simp_gpu_last_error(sim.h)
        c1 = clock()
        # (no outputs: the step is enqueued and get_state, which returns
        # time and dt, reads its status in the same wait)
        rc = lib.simp_gpu_step(sim.h, 1, None, None)
        assert rc == 0, lib.simp_gpu_last_error(sim.h)
        c2 = clock()
        rc = lib.simp_gpu_get_state(sim.h, *state_ptrs, pdtc, ptc)
        assert rc == 0, lib.simp_gpu_last_error(sim.h)
        c3 = clock()
        t_now, dt = tc.value, dtc.value
        for k, v in zip(calls, (c1 - c0, c2 - c1, c3 - c2)):
            calls[k].append(v)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = job_time_ms(dist, e0.elapsed_time(e1))
    world = dist.get_world_size() if dist else 1
    h2d = n * (2 * 16 + 5 * 8) + nb * 24
    d2h = n * (2 * 16 + 5 * 8) + 16
    return {"value": world * n * nsteps / (ms / 1e3), "unit": METRIC, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": nsteps,
            "path": "simp_gpu_set_state (pinned host) + simp_gpu_step(1, no outputs) + simp_gpu_get_state (pinned host, with time and dt)",
            "call_ms": {k: 1e3 * float(np.median(v)) for k, v in calls.items()},
            "call_timing": "host clock around each call, median over the steps",
            "link": link_copy_rates(stream, n * (2 * 16 + 5 * 8))}


def link_copy_rates(stream, nbytes, reps=20):
    """Plain pinned-host <-> device copies of one step's state bytes, as one
    buffer each way: the host link's rate, the floor under the end-to-end
    step (copies in, the step, copies out)."""
    import torch
    hb = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
    db = torch.empty(nbytes // 8, dtype=torch.float64, device="cuda")
    out = {"bytes": nbytes}
    with torch.cuda.stream(stream):
        for name, f in (("h2d", lambda: db.copy_(hb, non_blocking=True)),
                        ("d2h", lambda: hb.copy_(db, non_blocking=True))):
            for _ in range(3):
                f()
            stream.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                f()
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / reps
            out[name + "_ms"] = ms
            out[name + "_gbs"] = nbytes / ms / 1e6
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
