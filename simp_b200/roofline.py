"""Algorithmic HBM bytes of each kernel of one predictor-corrector step.

The per-particle-step figure is B_alg = 704 B (FP64 state), itemised per
right-hand-side evaluation (two per step), each array read or written once:

    neighbour search: cell key and index write, one sort read + write  24 B
    kinematic pass: read x, y, vx, vy, m, rho, hsml (56 B);
                    write eps11, eps12, eps22, div (32 B)               88 B
    stress pass with the rheology in its prologue: read x, y, vx, vy, m,
                    rho, hsml, h, A, eps x 3, div (104 B);
                    write dvx, dvy, dh, dA (32 B)                      136 B
    half-step update: write x, y, vx, vy, h, A, rho (56 B);
                    save or reload the step-start state (48 B)         104 B
                                                                  = 352 B

The launches fuse these: the kinematic kernel keeps the cell list exact
(the search) and computes the strain rates and stress (24 + 88 = 112 B per
particle); the stress kernel applies the pair forces and the update
(136 + 104 = 240 B per particle).  One step = 2 x (112 + 240) = 704 B.
The same B_alg is used for the mixed form, so fractions compare.
"""
from __future__ import annotations

import json
import os

KERNELS = ("kinematic_s0", "stress_predict", "kinematic_s1", "stress_correct", "step_finish")
BYTES_PER_PARTICLE = {
    "kinematic_s0": 112,
    "stress_predict": 240,
    "kinematic_s1": 112,
    "stress_correct": 240,
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
