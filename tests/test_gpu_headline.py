"""Parity at the sizes the throughput is quoted on: the 262,144-particle
basin (512 x 512 lattice, dx = 500 m, wall on +x, wind 10 m/s, cubic spline,
dt = 1 s) and the 1,048,576-particle vortex basin (1024 x 1024, dx = 250 m,
four walls) in FP64, against the FP64 oracle.

Bars, as for the small basins (test_gpu_parity.py): pair sets bit-exact with
r_ij, hsml_ij and br_ij bit-exact; one right-hand side within 1e-11
relative L2 (only the summation order differs: the GPU gathers each pair
from both sides); predictor-corrector trajectories within 1e-8 after 3
steps.  The reference's own NNPS (nnps.f90:155-517) and single_step
(single_step.f90:5-109) are what the oracle restates.
"""
import numpy as np
import pytest

from helpers import assert_same_pairs, rel_l2, smooth_velocity
from simp_b200 import basins
from simp_b200.simp import Simp

pytestmark = pytest.mark.gpu

TOL_RHS = 1e-11
TOL_TRAJ_3 = 1e-8
FIELDS = ("dxdt", "dvxdt", "dhdt", "dAdt")


def _fp64(b):
    prm = b.params.copy()
    prm.precision = 0
    return prm


def _hand_over(o, st, b, dt):
    """The GPU's state as the oracle's input (same bits on both sides)."""
    o.set_state(st["x"], st["vx"], st["mass"], st["rho"], st["hsml"], st["A"], st["h"],
                b.xb, b.massb, dt, st["current_time"])


@pytest.fixture(scope="module")
def cfg2_basin():
    return basins.cfg2()


def test_cfg2_single_step_fields(gpu_lib, oracle_mod):
    """One right-hand side of the 262,144-particle basin with a live
    velocity field (shear, divergence, rotation) and the drag on: every rate
    and every diagnostic field (strain rates, viscosities, pressure,
    stress) against the oracle."""
    b = basins.cfg2()
    b.vx = smooth_velocity(b.x, b.L, seed=21)
    prm = _fp64(b)
    g = Simp.from_basin(b, prm)
    o = oracle_mod.Oracle.from_basin(b, prm)
    rg, ro = g.single_step(3600.0), o.single_step(3600.0)
    for k in FIELDS:
        e = rel_l2(rg[k], ro[k])
        assert e < TOL_RHS, (k, e)
    dg, do = g.get_diag(), o.get_diag()
    for k in dg:
        e = rel_l2(dg[k], do[k])
        assert e < TOL_RHS, (k, e)
    assert_same_pairs(g.nnps(), o.nnps())
    assert g.interaction_stats() == o.interaction_stats()
    g.close()


def test_cfg2_three_steps(gpu_lib, oracle_mod, cfg2_basin):
    """Three predictor-corrector steps of the basin as it is benchmarked
    (at rest, wind 10 m/s, the wall pushing back): state within 1e-8 and the
    integrator's clock equal."""
    b = cfg2_basin
    prm = _fp64(b)
    g = Simp.from_basin(b, prm)
    o = oracle_mod.Oracle.from_basin(b, prm)
    tg, dtg = g.time_integration(3)
    to, dto = o.step(3)
    assert tg == to and dtg == dto
    sg, so = g.get_state(), o.get_state()
    for k in ("x", "vx", "h", "A", "rho"):
        ref = b.x if k == "x" else 0.0
        e = rel_l2(sg[k] - ref, so[k] - ref)
        assert e < TOL_TRAJ_3, (k, e)
    g.close()


@pytest.mark.parametrize("steps", [1, 100])
def test_cfg2_pairs_on_gpu_trajectory(gpu_lib, oracle_mod, cfg2_basin, steps):
    """Pair sets after 1 and 100 steps of the GPU's own trajectory (re-sorts
    every 16 steps, Verlet lists rebuilt as particles near the wall speed
    up), with that state handed to the oracle: bit-exact, and one right-hand
    side on it within 1e-11."""
    b = cfg2_basin
    prm = _fp64(b)
    g = Simp.from_basin(b, prm)
    g.time_integration(steps)
    st = g.get_state()
    assert np.all(np.isfinite(st["x"])) and np.all(np.isfinite(st["vx"]))
    o = oracle_mod.Oracle.from_basin(b, prm)
    _hand_over(o, st, b, prm.dt)
    assert_same_pairs(g.nnps(), o.nnps())
    t = st["current_time"]
    rg, ro = g.single_step(t), o.single_step(t)
    for k in ("dvxdt", "dhdt", "dAdt"):
        e = rel_l2(rg[k], ro[k])
        assert e < TOL_RHS, (k, e)
    g.close()


def test_cfg2_pairs_on_oracle_trajectory(gpu_lib, oracle_mod, cfg2_basin):
    """The oracle's own trajectory (10 steps), handed to a fresh GPU
    context: the GPU finds bit-exactly the oracle's pairs."""
    b = cfg2_basin
    prm = _fp64(b)
    o = oracle_mod.Oracle.from_basin(b, prm)
    o.step(10)
    so = o.get_state()
    g = Simp(prm, b.n, b.nb)
    g.set_state(so["x"], so["vx"], so["mass"], so["rho"], so["hsml"], so["A"], so["h"], b.xb, b.massb,
                prm.dt, so["current_time"])
    assert_same_pairs(g.nnps(), o.nnps())
    g.close()


def test_cfg3_fp64_single_step(gpu_lib, oracle_mod):
    """One FP64 right-hand side of the 1,048,576-particle vortex basin (four
    walls, smoothed h and A) at t > 0: rates and stress against the oracle,
    pair sets bit-exact."""
    b = basins.cfg3()
    b.vx = smooth_velocity(b.x, b.L, amp=0.2, seed=31)
    prm = _fp64(b)
    g = Simp.from_basin(b, prm)
    o = oracle_mod.Oracle.from_basin(b, prm)
    rg, ro = g.single_step(600.0), o.single_step(600.0)
    for k in FIELDS:
        e = rel_l2(rg[k], ro[k])
        assert e < TOL_RHS, (k, e)
    dg, do = g.get_diag(), o.get_diag()
    for k in ("eps11", "eps12", "eps22", "zeta", "sig11", "sig12", "sig22"):
        e = rel_l2(dg[k], do[k])
        assert e < TOL_RHS, (k, e)
    assert_same_pairs(g.nnps(), o.nnps())
    g.close()
