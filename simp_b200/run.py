"""Run a synthetic basin through the GPU hot path and print a summary.

    python -m simp_b200.run --workload cfg2 --steps 100

Workloads: cfg1 (2,500 particles), cfg2 (262,144), cfg3 (1,048,576, vortex,
mixed), cfg2x4 (the cfg2 physics on a 1024 x 1024 lattice, 1,048,576
particles, FP64).  The role of the
reference's `make all` + simp.out run (Makefile:56-60), without CSV output.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import basins
from .simp import Simp


def workload(name: str):
    if name == "cfg1":
        return basins.cfg1()
    if name == "cfg2":
        return basins.cfg2()
    if name == "cfg3":
        return basins.cfg3()
    if name == "cfg2x4":
        return basins.make_basin(1024, 250.0, 2, name="cfg2x4_1048576", walls="+x", wind=(10.0, 0.0))
    raise SystemExit(f"unknown workload {name}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="cfg2")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--chunk", type=int, default=0, help="steps per call (0: all in one call)")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default=None,
                    help="override the workload's precision")
    ap.add_argument("--passes", choices=("gather", "tiled", "gather_one", "gather_two"), default="gather",
                    help="pair-pass implementation")
    ap.add_argument("--moving", action="store_true",
                    help="start from a smooth non-zero velocity field instead of rest")
    args = ap.parse_args()
    b = workload(args.workload)
    if args.moving:
        b.vx = basins.smooth_velocity(b.x, b.L, amp=0.3, seed=22)
    prm = b.params.copy()
    if args.precision:
        prm.precision = 1 if args.precision == "mixed" else 0
    sim = Simp.from_basin(b, prm)
    sim.set_passes({"gather": 0, "tiled": 1, "gather_one": 2, "gather_two": 3}[args.passes])
    t0 = time.perf_counter()
    done = 0
    chunk = args.chunk or args.steps
    t = dt = 0.0
    while done < args.steps:
        k = min(chunk, args.steps - done)
        t, dt = sim.time_integration(k)
        done += k
    el = time.perf_counter() - t0
    st = sim.get_state()
    v = np.hypot(st["vx"][:, 0], st["vx"][:, 1])
    print(json.dumps({"workload": b.name, "particles": b.n, "steps": done, "current_time": t, "dt": dt,
                      "wall_s": el, "particle_steps_per_s_wall": b.n * done / el,
                      "vmax": float(v.max()), "vmean": float(v.mean()),
                      "h_range": [float(st["h"].min()), float(st["h"].max())],
                      "kernel_launches": int(sim.lib.simp_gpu_kernel_launches(sim.h))}))
    sim.close()


if __name__ == "__main__":
    main()
