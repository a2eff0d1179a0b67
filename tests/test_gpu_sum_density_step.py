"""Summation density inside the step (den_alg = 1, density.f90:41-100) on the
GPU against the oracle, under each integrator and with the hsml, mass and
time-step switches that read the new density.

The reference calls density after each update (time_integration.f90:128,
218, 242, 262, 344, 372) over the last right-hand side's pairs and kernel
values, with the masses and densities current at the call; the predictor-
corrector calls it twice in a row at the end, the second call reading the
first one's densities.  Its self term takes the kernel_zero array that each
right-hand side's pair loop sets for the p_i of every pair (kernel.f90:503)
and that a particle which is p_i of no pair keeps from before (0 at the
start): the GPU keeps it per particle and finds p_i from the particles'
indices and reference buckets (tests/test_oracle_sum_density_step.py checks
that rule on the oracle's pair lists).  Jittered lattices under both
searches make the rule matter for many particles.  Bar: 10 steps within
1e-9 in FP64, as for the other switch variants.
"""
import numpy as np
import pytest

from helpers import rel_l2, smooth_velocity
from simp_b200 import basins
from simp_b200.params import ART_VISC_HK, PASSES_TILED, PREC_MIXED
from simp_b200.simp import Batch, Simp

pytestmark = pytest.mark.gpu

TOL_STEPS = 1e-9
TOL_MIXED = 1e-5

CASES = {
    "predictor_corrector": dict(den_alg=1),
    "euler": dict(den_alg=1, int_algorithm=1),
    "leapfrog": dict(den_alg=1, int_algorithm=3),
    # masses from the lattice area (mass_evolution.f90:66-69): the sums
    # read the masses of the call, before the update's own mass evolution
    "mass_from_area": dict(den_alg=1, mass_from_area=1),
    "mass_from_area_leapfrog": dict(den_alg=1, mass_from_area=1, int_algorithm=3),
    # Marquis hsml from the summed density (smoothing_length.f90:136-142)
    "marquis": dict(den_alg=1, sle=2),
    "marquis_euler_vp_dt": dict(den_alg=1, sle=2, int_algorithm=1, tse=2),
    "marquis_leapfrog": dict(den_alg=1, sle=2, int_algorithm=3),
    # Benz hsml: its own drhodt sum, accumulated over the steps
    "benz": dict(den_alg=1, sle=1),
    "benz_mass_from_area": dict(den_alg=1, sle=1, mass_from_area=1),
    # Monaghan time step with the artificial-viscosity CFL criterion: the
    # divergence divides by the summed density
    "monaghan_dt_hk": dict(den_alg=1, tse=1, artificial_visc=1, art_visc_alg=ART_VISC_HK),
    # jittered lattice: which particle of a pair is p_i varies, under the
    # direct and the bucket search, with fixed and with Marquis hsml
    "jitter_direct": dict(den_alg=1, nnps_algorithm=1, jitter=0.35),
    "jitter_bucket": dict(den_alg=1, jitter=0.35),
    "jitter_bucket_marquis": dict(den_alg=1, sle=2, jitter=0.35),
    "jitter_direct_marquis_leapfrog": dict(den_alg=1, sle=2, int_algorithm=3, nnps_algorithm=1, jitter=0.35),
}


def _basin(jitter=0.0):
    b = basins.cfg1()
    if jitter:
        rng = np.random.default_rng(7)
        b.x = b.x + jitter * b.dx * rng.uniform(-1.0, 1.0, b.x.shape)
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=41)
    b.h = b.h * np.linspace(0.9, 1.1, b.n)
    b.rho = b.h * 900.0
    return b


def _prm(b, **kw):
    p = b.params.copy()
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _oracle(oracle_mod, b, prm):
    o = oracle_mod.Oracle.from_basin(b, prm)
    o.set_regularization_form(False)
    return o


@pytest.mark.parametrize("name", sorted(CASES))
def test_sum_density_step_against_oracle(gpu_lib, oracle_mod, name):
    kw = dict(CASES[name])
    b = _basin(kw.pop("jitter", 0.0))
    prm = _prm(b, **kw)
    g = Simp.from_basin(b, prm)
    o = _oracle(oracle_mod, b, prm)
    tg, dtg = g.time_integration(10)
    to, dto = o.step(10)
    assert tg == pytest.approx(to, rel=1e-9) and dtg == pytest.approx(dto, rel=1e-9)
    sg, so = g.get_state(), o.get_state()
    for k in ("x", "vx", "h", "A", "rho", "mass", "hsml"):
        ref = b.x if k == "x" else 0.0
        e = rel_l2(sg[k] - ref, so[k] - ref)
        assert e < TOL_STEPS, (k, e)
    # the switch is live: the density is neither the start's nor h rho_ice
    assert rel_l2(sg["rho"], b.rho) > 1e-6
    assert rel_l2(sg["rho"], 900.0 * sg["h"]) > 1e-6
    g.close()


def test_sum_density_tiled_equals_gather(gpu_lib):
    """The tiled pair passes leave the same pair lists: bitwise the same
    trajectory."""
    b = _basin()
    prm = _prm(b, **CASES["marquis"])
    out = []
    for tiled in (False, True):
        g = Simp.from_basin(b, prm)
        if tiled:
            g.set_passes(PASSES_TILED, 128, 1024)
        g.time_integration(6)
        out.append(g.get_state())
        g.close()
    for k in ("x", "vx", "rho", "hsml"):
        assert np.array_equal(out[0][k], out[1][k]), k


def test_sum_density_batch_of_one_equals_single_context(gpu_lib):
    b = _basin()
    prm = _prm(b, **CASES["predictor_corrector"])
    with Batch(prm, b.n + 16, max(b.nb, 1) + 16, 2) as bt:
        s = bt.add(b)
        bt.step(8)
        gb = bt.get_state(s)
    g = Simp.from_basin(b, prm)
    g.time_integration(8)
    gs = g.get_state()
    g.close()
    for k in ("x", "vx", "rho", "h"):
        assert np.array_equal(gb[k], gs[k]), k


def test_sum_density_mixed_form(gpu_lib, oracle_mod):
    """Mixed precision: the density sums stay FP64 over the FP32 pass's
    pairs; 10 steps within the mixed form's bar."""
    b = _basin()
    prm = _prm(b, **CASES["marquis"])
    pm = prm.copy()
    pm.precision = PREC_MIXED
    g = Simp.from_basin(b, pm)
    o = _oracle(oracle_mod, b, prm)
    g.time_integration(10)
    o.step(10)
    sg, so = g.get_state(), o.get_state()
    for k in ("vx", "rho", "hsml"):
        e = rel_l2(sg[k], so[k])
        assert e < TOL_MIXED, (k, e)
    g.close()


def test_kept_kernel_zero_through_resorts(gpu_lib, oracle_mod):
    """40 steps (the particles are re-sorted at steps 16 and 32 and the
    kept kernel_zero moves with them) of a jittered basin with Marquis hsml,
    with a standalone right-hand side first, which sets kernel_zero too."""
    b = _basin(0.35)
    prm = _prm(b, den_alg=1, sle=2)
    g = Simp.from_basin(b, prm)
    o = _oracle(oracle_mod, b, prm)
    g.single_step(0.0)
    o.single_step(0.0)
    g.time_integration(40)
    o.step(40)
    sg, so = g.get_state(), o.get_state()
    for k in ("vx", "rho", "hsml"):
        e = rel_l2(sg[k], so[k])
        assert e < 1e-8, (k, e)
    g.close()


def test_sum_density_step_at_headline_size(gpu_lib, oracle_mod):
    """The headline basin (262,144 particles) with the summation density in
    the step: 3 predictor-corrector steps against the oracle.  A particle
    that is p_i of no pair (the corner farthest up and right, for one) has
    no self term, as in the reference."""
    b = basins.cfg2()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=43)
    # (a thickness gradient: the sum of a uniform density returns it exactly)
    b.h = b.h * np.linspace(0.9, 1.1, b.n)
    b.rho = b.h * 900.0
    prm = _prm(b, den_alg=1)
    g = Simp.from_basin(b, prm)
    o = _oracle(oracle_mod, b, prm)
    g.time_integration(3)
    o.step(3)
    sg, so = g.get_state(), o.get_state()
    for k in ("x", "vx", "h", "rho"):
        ref = b.x if k == "x" else 0.0
        e = rel_l2(sg[k] - ref, so[k] - ref)
        assert e < TOL_STEPS, (k, e)
    assert rel_l2(sg["rho"], b.rho) > 1e-6
    g.close()
