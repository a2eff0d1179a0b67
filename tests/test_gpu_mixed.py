"""Mixed-precision form (FP32 kernel evaluations and Kahan-compensated pair
sums; FP64 positions, integrator and reductions) against the FP64 oracle.

Tolerances: one right-hand side on identical inputs within 2e-6 relative L2
(FP32 rounding of the kernel gradient and of the pair terms, compensated
sums); velocity and thickness within 1e-4 relative L2 after 20 steps.
"""
import numpy as np
import pytest

from helpers import assert_same_pairs, rel_l2, smooth_velocity
from simp_b200 import basins
from simp_b200.params import PREC_MIXED, SKF_WENDLAND_C6
from simp_b200.simp import Simp

pytestmark = pytest.mark.gpu

TOL_MIXED_RHS = 2e-6
TOL_MIXED_TRAJ = 1e-4


def _mixed(b, skf=None):
    prm = b.params.copy()
    prm.precision = PREC_MIXED
    if skf is not None:
        prm.skf = skf
    return prm


@pytest.mark.parametrize("skf", [9, SKF_WENDLAND_C6])
def test_mixed_single_step(gpu_lib, oracle_mod, skf):
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, seed=11)
    prm = _mixed(b, skf)
    g = Simp.from_basin(b, prm)
    ref = prm.copy()
    ref.precision = 0
    o = oracle_mod.Oracle.from_basin(b, ref)
    rg, ro = g.single_step(600.0), o.single_step(600.0)
    for k in ("dvxdt", "dhdt", "dAdt"):
        e = rel_l2(rg[k], ro[k])
        assert e < TOL_MIXED_RHS, (k, e)
    dg, do = g.get_diag(), o.get_diag()
    for k in ("eps11", "eps12", "eps22", "sig11", "sig12", "sig22"):
        e = rel_l2(dg[k], do[k])
        assert e < TOL_MIXED_RHS, (k, e)


def test_mixed_pair_lists_bit_exact(gpu_lib, oracle_mod):
    b = basins.cfg1()
    g = Simp.from_basin(b, _mixed(b))
    o = oracle_mod.Oracle.from_basin(b)
    assert_same_pairs(g.nnps(), o.nnps())


def test_mixed_trajectory_error(gpu_lib, oracle_mod):
    """Velocity and thickness after 20 steps within 1e-4 relative L2 of the
    FP64 oracle, for the cfg1 basin in motion."""
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=0.5, seed=12)
    g = Simp.from_basin(b, _mixed(b))
    o = oracle_mod.Oracle.from_basin(b)
    g.time_integration(20)
    o.step(20)
    sg, so = g.get_state(), o.get_state()
    for k in ("vx", "h", "A"):
        e = rel_l2(sg[k], so[k])
        assert e < TOL_MIXED_TRAJ, (k, e)


def _rhs_errors(b, prm_mixed, t=600.0):
    prm64 = prm_mixed.copy()
    prm64.precision = 0
    p64 = Simp.from_basin(b, prm64)
    p32 = Simp.from_basin(b, prm_mixed)
    r64, r32 = p64.single_step(t), p32.single_step(t)
    return {k: rel_l2(r32[k], r64[k]) for k in ("dvxdt", "dhdt", "dAdt")}


def test_mixed_rhs_at_scale(gpu_lib):
    """262,144-particle basin: one mixed right-hand side against the plain
    FP64 GPU path (itself pinned to the oracle at 1e-11)."""
    b = basins.cfg2()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=13)
    for k, e in _rhs_errors(b, _mixed(b)).items():
        assert e < TOL_MIXED_RHS, (k, e)


def test_mixed_rhs_vortex_basin(gpu_lib):
    """The 1,048,576-particle vortex basin with smoothed h and A, four walls,
    one mixed right-hand side against FP64."""
    b = basins.cfg3()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=14)
    assert b.params.precision == PREC_MIXED
    for k, e in _rhs_errors(b, b.params.copy(), t=600.0).items():
        assert e < TOL_MIXED_RHS, (k, e)


def test_mixed_short_trajectory_at_scale(gpu_lib):
    """262,144 particles, 3 steps at dt = 1 s: mixed against FP64.

    At dt = 1 s these basins are far above the viscous-plastic stability
    limit (about 1e-4 s at 500 m spacing): perturbations grow about twofold
    per step whatever their source, so a trajectory comparison of any two
    implementations only means something over a few steps; longer horizons
    are compared per right-hand side (above) and on the 2,500-particle basin
    (test_mixed_trajectory_error)."""
    b = basins.cfg2()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=13)
    p64 = Simp.from_basin(b)
    p32 = Simp.from_basin(b, _mixed(b))
    assert b.params.precision == 0
    p64.time_integration(3)
    p32.time_integration(3)
    s64, s32 = p64.get_state(), p32.get_state()
    for k in ("vx", "h"):
        e = rel_l2(s32[k], s64[k])
        assert e < TOL_MIXED_TRAJ, (k, e)
    assert np.array_equal(s32["mass"], s64["mass"])
