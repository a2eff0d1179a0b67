"""The two implementations of the pair passes give the same bits.

SIMP_PASSES_TILED (chunks of a cell row staged in shared memory with their
halo) visits every particle's pairs in the same increasing-index order as
SIMP_PASSES_GATHER (per-particle gathers over Verlet lists), with the same
arithmetic, so states, rates and pair lists must agree bitwise, for every
tile shape, including shapes whose halo does not fit and falls back to HBM.
"""
import numpy as np
import pytest

from helpers import assert_same_pairs, smooth_velocity
from simp_b200 import basins
from simp_b200.params import PREC_FP64, PREC_MIXED
from simp_b200.simp import Simp

pytestmark = pytest.mark.gpu

GATHER, TILED = 0, 1
SHAPES = [(TILED, 256, 1024), (TILED, 128, 512), (TILED, 64, 384), (TILED, 128, 64)]


def _run(b, prm, impl, threads, cap, steps):
    g = Simp.from_basin(b, prm)
    g.set_passes(impl, threads, cap)
    r = g.single_step(600.0)
    g.time_integration(steps)
    return g, r, g.get_state()


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_tiled_equals_gather_cfg1(gpu_lib, precision):
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=0.5, seed=21)
    prm = b.params.copy()
    prm.precision = precision
    g0, r0, s0 = _run(b, prm, GATHER, 256, 1024, 40)
    for shape in SHAPES:
        g, r, s = _run(b, prm, *shape, 40)
        for k in r0:
            assert np.array_equal(r[k], r0[k]), (shape, k)
        for k in ("x", "vx", "h", "A", "rho"):
            assert np.array_equal(s[k], s0[k]), (shape, k)
        assert_same_pairs(g.nnps(), g0.nnps())
        g.close()


def test_tiled_equals_gather_at_scale(gpu_lib):
    b = basins.cfg2()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=22)
    _, r0, s0 = _run(b, b.params, GATHER, 256, 1024, 20)
    _, r1, s1 = _run(b, b.params, TILED, 256, 1024, 20)
    for k in r0:
        assert np.array_equal(r1[k], r0[k]), k
    for k in ("x", "vx", "h", "A"):
        assert np.array_equal(s1[k], s0[k]), k


def test_autotune_keeps_state(gpu_lib):
    b = basins.instance(1, 20000)
    g = Simp.from_basin(b)
    g.time_integration(3)
    before = g.get_state()
    ms = g.autotune(2)
    assert ms > 0
    impl, threads, cap = g.get_passes()
    assert impl in (GATHER, TILED)
    after = g.get_state()
    for k in ("x", "vx", "h", "A"):
        assert np.array_equal(after[k], before[k])
    g.time_integration(2)
