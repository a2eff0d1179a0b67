"""Shared checks for the parity tests."""
from __future__ import annotations

import numpy as np


def canonical_pairs(res: dict):
    """Unordered pair set of an NNPS result, sorted by (min, max) index."""
    a = np.minimum(res["p_i"], res["p_j"]).astype(np.int64)
    b = np.maximum(res["p_i"], res["p_j"]).astype(np.int64)
    order = np.lexsort((b, a))
    return a[order], b[order], np.asarray(res["r_ij"])[order], np.asarray(res["hsml_ij"])[order]


def canonical_wall_pairs(res: dict):
    a = np.asarray(res["bp_i"]).astype(np.int64)
    b = np.asarray(res["bp_j"]).astype(np.int64)
    order = np.lexsort((b, a))
    return a[order], b[order], np.asarray(res["br_ij"])[order]


def bits(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def assert_same_pairs(gpu: dict, ref: dict):
    """Bit-exact equality of the pair sets and of r_ij / hsml_ij / br_ij."""
    assert gpu["nip"] == ref["nip"], (gpu["nip"], ref["nip"])
    ga, gb, gr, gh = canonical_pairs(gpu)
    ra, rb, rr, rh = canonical_pairs(ref)
    assert np.array_equal(ga, ra) and np.array_equal(gb, rb), "pair index sets differ"
    assert np.array_equal(bits(gr), bits(rr)), "r_ij not bit-exact"
    assert np.array_equal(bits(gh), bits(rh)), "hsml_ij not bit-exact"
    assert gpu["bnip"] == ref["bnip"], (gpu["bnip"], ref["bnip"])
    wa, wb, wr = canonical_wall_pairs(gpu)
    va, vb, vr = canonical_wall_pairs(ref)
    assert np.array_equal(wa, va) and np.array_equal(wb, vb), "wall pair sets differ"
    assert np.array_equal(bits(wr), bits(vr)), "br_ij not bit-exact"


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    if den == 0.0:
        return float(np.linalg.norm(a - b))
    return float(np.linalg.norm(a - b) / den)


def smooth_velocity(x: np.ndarray, L: float, amp: float = 0.3, seed: int = 0) -> np.ndarray:
    """A smooth, non-trivial velocity field (shear + divergence + rotation)."""
    from simp_b200.basins import smooth_velocity as sv
    return sv(x, L, amp=amp, seed=seed)
