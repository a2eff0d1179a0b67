"""The implementations of the pair passes give the same bits.

SIMP_PASSES_TILED (chunks of a cell row staged in shared memory with their
halo) visits every particle's pairs in the same increasing-index order as
the gather forms (per-particle gathers over Verlet lists), with the same
arithmetic, so states, rates and pair lists must agree bitwise, for every
tile shape, including shapes whose halo does not fit and falls back to HBM.
The gather forms' kinematic pass as one kernel (SIMP_PASSES_GATHER_ONE) or
as pair finding plus pair sums over the stored list (SIMP_PASSES_GATHER_TWO)
sums the same pairs in the same order.
"""
import numpy as np
import pytest

from helpers import assert_same_pairs, smooth_velocity
from simp_b200 import basins
from simp_b200.params import (PASSES_GATHER as GATHER, PASSES_GATHER_ONE as ONE, PASSES_GATHER_TWO as TWO,
                               PASSES_TILED as TILED, PREC_FP64, PREC_MIXED)
from simp_b200.simp import Simp

pytestmark = pytest.mark.gpu

SHAPES = [(ONE, 256, 1024), (TWO, 256, 1024), (TILED, 256, 1024), (TILED, 128, 512), (TILED, 64, 384),
          (TILED, 128, 64)]


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
    for impl in (TILED, ONE, TWO):
        g, r1, s1 = _run(b, b.params, impl, 256, 1024, 20)
        for k in r0:
            assert np.array_equal(r1[k], r0[k]), (impl, k)
        for k in ("x", "vx", "h", "A"):
            assert np.array_equal(s1[k], s0[k]), (impl, k)
        g.close()


def test_gather_forms_agree_on_a_large_basin(gpu_lib):
    """Above 400,000 particles the default gather form runs the kinematic
    pass as one kernel; both forms stay bitwise equal there, fast wall
    particles and list rebuilds included."""
    b = basins.make_basin(640, 500.0, 7, name="sq640", walls="+x", wind=(10.0, 0.0), steps=1000)
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=23)
    g1, r1, s1 = _run(b, b.params, ONE, 256, 1024, 12)
    g2, r2, s2 = _run(b, b.params, TWO, 256, 1024, 12)
    for k in r1:
        assert np.array_equal(r2[k], r1[k]), k
    for k in ("x", "vx", "h", "A", "rho"):
        assert np.array_equal(s2[k], s1[k]), k
    assert_same_pairs(g2.nnps(), g1.nnps())
    g1.close()
    g2.close()


def test_autotune_keeps_state(gpu_lib):
    b = basins.instance(1, 20000)
    g = Simp.from_basin(b)
    g.time_integration(3)
    before = g.get_state()
    ms = g.autotune(2)
    assert ms > 0
    impl, threads, cap = g.get_passes()
    assert impl in (TILED, ONE, TWO)
    after = g.get_state()
    for k in ("x", "vx", "h", "A"):
        assert np.array_equal(after[k], before[k])
    g.time_integration(2)
