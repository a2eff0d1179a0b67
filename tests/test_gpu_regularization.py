"""Regularisation (regularization.f90: XSPH, Hernquist-Katz and Monaghan
artificial viscosity) on the GPU against the oracle's per-pair form.

The reference's own loops run serially over its pair list and carry pi_ij
from one pair into the next pair outside the viscosity criterion, and add
the XSPH term with the same sign to both particles of a pair
(regularization.f90:82-89, 193-196, 285-291); the gather form evaluates every
pair on its own, which the oracle restates as its per-pair form
(tests/test_oracle_regularization.py pins both forms).  Bars as for the
other switch variants: one right-hand side within 1e-11 (2e-6 in the mixed
form), 10 steps within 1e-9.
"""
import numpy as np
import pytest

from helpers import rel_l2, smooth_velocity
from simp_b200 import basins
from simp_b200.params import ART_VISC_HK, ART_VISC_MON, PASSES_TILED, PREC_MIXED
from simp_b200.simp import Simp

pytestmark = pytest.mark.gpu

TOL_RHS = 1e-11
TOL_STEPS = 1e-9
TOL_MIXED_RHS = 2e-6

CASES = {
    "xsph": dict(xsph_regularization=1, art_visc_alg=0),
    "hk": dict(artificial_visc=1, art_visc_alg=ART_VISC_HK),
    "monaghan": dict(artificial_visc=1, art_visc_alg=ART_VISC_MON),
    "xsph_hk": dict(xsph_regularization=1, artificial_visc=1, art_visc_alg=ART_VISC_HK),
    # regularization is called for XSPH alone and then runs art_visc_alg's
    # viscosity too, with the sound speed never refreshed (c = 0)
    "xsph_then_hk": dict(xsph_regularization=1, art_visc_alg=ART_VISC_HK),
    "xsph_mon_euler": dict(xsph_regularization=1, artificial_visc=1, art_visc_alg=ART_VISC_MON,
                           int_algorithm=1),
    "xsph_hk_leapfrog": dict(xsph_regularization=1, artificial_visc=1, art_visc_alg=ART_VISC_HK,
                             int_algorithm=3),
    # Monaghan time step with the artificial-viscosity CFL criterion
    "hk_monaghan_dt": dict(artificial_visc=1, art_visc_alg=ART_VISC_HK, tse=1),
    "mon_monaghan_dt_benz": dict(artificial_visc=1, art_visc_alg=ART_VISC_MON, tse=1, sle=1),
}


def _basin():
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=0.5, seed=50)
    return b


def _prm(b, **kw):
    p = b.params.copy()
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _pair(b, oracle_mod, prm):
    g = Simp.from_basin(b, prm)
    o = oracle_mod.Oracle.from_basin(b, prm)
    o.set_regularization_form(False)
    return g, o


@pytest.mark.parametrize("name", sorted(CASES))
def test_regularization_against_oracle(gpu_lib, oracle_mod, name):
    b = _basin()
    prm = _prm(b, **CASES[name])
    g, o = _pair(b, oracle_mod, prm)
    rg, ro = g.single_step(3600.0), o.single_step(3600.0)
    for k in ("dxdt", "dvxdt", "dhdt", "dAdt"):
        e = rel_l2(rg[k], ro[k])
        assert e < TOL_RHS, (k, e)
    # the regularisation is live: the rates differ from the plain ones
    plain = Simp.from_basin(b, b.params).single_step(3600.0)
    key = "dxdt" if prm.xsph_regularization else "dvxdt"
    assert rel_l2(rg[key], plain[key]) > 1e-9
    g.close()
    g2, o2 = _pair(b, oracle_mod, prm)
    tg, dtg = g2.time_integration(10)
    to, dto = o2.step(10)
    assert tg == pytest.approx(to, rel=1e-9) and dtg == pytest.approx(dto, rel=1e-9)
    sg, so = g2.get_state(), o2.get_state()
    for k in ("x", "vx", "h", "A", "rho", "hsml"):
        ref = b.x if k == "x" else 0.0
        e = rel_l2(sg[k] - ref, so[k] - ref)
        assert e < TOL_STEPS, (k, e)
    g2.close()


def test_regularization_tiled_equals_gather(gpu_lib):
    """The tiled pair passes feed the same pair lists to the regularisation
    pass: bitwise the same rates and trajectory."""
    b = _basin()
    prm = _prm(b, **CASES["xsph_hk"])
    out = []
    for tiled in (False, True):
        g = Simp.from_basin(b, prm)
        if tiled:
            g.set_passes(PASSES_TILED, 128, 1024)
        r = g.single_step(3600.0)
        g.time_integration(5)
        out.append((r, g.get_state()))
        g.close()
    (ra, sa), (rb, sb) = out
    for k in ("dxdt", "dvxdt"):
        assert np.array_equal(ra[k], rb[k]), k
    for k in ("x", "vx"):
        assert np.array_equal(sa[k], sb[k]), k


@pytest.mark.parametrize("name", ["xsph_hk", "monaghan"])
def test_regularization_mixed_form(gpu_lib, oracle_mod, name):
    """Mixed precision: the regularisation pass runs in FP64 over the FP32
    pass's pairs; one right-hand side within the mixed form's bar."""
    b = _basin()
    prm = _prm(b, **CASES[name])
    pm = prm.copy()
    pm.precision = PREC_MIXED
    g = Simp.from_basin(b, pm)
    o = oracle_mod.Oracle.from_basin(b, prm)
    o.set_regularization_form(False)
    rg, ro = g.single_step(3600.0), o.single_step(3600.0)
    for k in ("dxdt", "dvxdt", "dhdt"):
        e = rel_l2(rg[k], ro[k])
        assert e < TOL_MIXED_RHS, (k, e)
    g.close()
