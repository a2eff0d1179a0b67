"""Algorithmic HBM bytes of each kernel of one predictor-corrector step.

Counted per particle, FP64 state, each array read or written once (the
minimum any implementation of the step must move; neighbour gathers of the
same arrays are served on chip and are not counted again):

kinematic pass (run at S0 and at S1), per particle:
    reads  x, y, vx, vy, hsml, m, m/rho, h, A, rho   10 x 8 B = 80 B
           cell id                                    4 B
    writes tau11, tau12, tau22 (= sigma / rho^2), div  4 x 8 B = 32 B
    total 116 B
stress pass, predictor epilogue (RHS at S0, writes S1):
    reads  x, y, hsml, m, tau11, tau12, tau22, rho, h, A, vx, vy, div
                                                     13 x 8 B = 104 B
           cell id 4 B, rebuild positions xr, yr 16 B
    writes x, y, vx, vy, h, A, rho, m/rho             8 x 8 B = 64 B
    total 188 B
stress pass, corrector epilogue (RHS at S1, base S0, writes S0):
    reads  S1: x, y, tau11, tau12, tau22, rho, h, A, vx, vy, div 11 x 8 B
           shared hsml, m 2 x 8 B, cell id 4 B, xr, yr 16 B,
           S0: x, y, vx, vy, h, A 6 x 8 B                 = 172 B
    writes x, y, vx, vy, h, A, rho, m/rho             8 x 8 B = 64 B
    total 236 B
step finish: a handful of scalars, 0 B per particle.

One step = 2 x 116 + 188 + 236 = 656 B per particle-step.
"""
from __future__ import annotations

import json
import os

KERNELS = ("kinematic_s0", "stress_predict", "kinematic_s1", "stress_correct", "step_finish")
BYTES_PER_PARTICLE = {
    "kinematic_s0": 116,
    "stress_predict": 188,
    "kinematic_s1": 116,
    "stress_correct": 236,
    "step_finish": 0,
}
STEP_BYTES_PER_PARTICLE = sum(BYTES_PER_PARTICLE.values())

FALLBACK_HBM_GBS = 6650.0


def hbm_peak(root: str):
    """(GB/s, source) from MEASURED_PEAKS.json, else the pool's fallback."""
    p = os.path.join(root, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"
