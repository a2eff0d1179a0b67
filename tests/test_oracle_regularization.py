"""Known-answer tests of the oracle's regularisation (regularization.f90),
both of its forms: the reference's serial pair loops taken literally, and
the per-pair form the library implements.  No GPU.

- Rigid translation: every pair has v_i - v_j = 0, so XSPH and both
  artificial viscosities add nothing (the rates equal the unregularised ones).
- Uniform compression (v = -a x): every pair satisfies the viscosity
  criterion (v_i - v_j) . (x_i - x_j) < 0, so the literal and per-pair
  artificial viscosities agree to round-off.
- Momentum: the artificial viscosity adds +-m pi grad W to the two particles
  of a pair, so sum_i m_i a_i(visc) = 0 in both forms; the per-pair XSPH is
  antisymmetric, sum_i m_i xs_i = 0, which the literal form's same-signed
  term breaks.
- Mixed flow: a pair outside the criterion keeps the last pi_ij in the
  literal form, so the two forms differ there.
"""
import numpy as np
import pytest

from helpers import rel_l2, smooth_velocity
from simp_b200 import basins
from simp_b200.params import ART_VISC_HK, ART_VISC_MON


def _basin(nside=20):
    b = basins.make_basin(nside, 2000.0, 41, walls="")
    b.params.wind_force = 0
    b.params.water_force = 0
    return b


def _prm(b, xsph=0, art=0, alg=ART_VISC_HK):
    p = b.params.copy()
    p.xsph_regularization = xsph
    p.artificial_visc = art
    p.art_visc_alg = alg
    return p


def _rhs(oracle_mod, b, prm, literal, t=600.0):
    o = oracle_mod.Oracle.from_basin(b, prm)
    o.set_regularization_form(literal)
    return o.single_step(t)


@pytest.mark.parametrize("alg", [ART_VISC_HK, ART_VISC_MON])
@pytest.mark.parametrize("literal", [False, True])
def test_rigid_translation_adds_nothing(oracle_mod, alg, literal):
    b = _basin()
    b.vx[:] = (0.7, -0.2)
    base = _rhs(oracle_mod, b, _prm(b), literal)
    reg = _rhs(oracle_mod, b, _prm(b, xsph=1, art=1, alg=alg), literal)
    assert np.array_equal(reg["dxdt"], base["dxdt"])
    assert np.array_equal(reg["dvxdt"], base["dvxdt"])


@pytest.mark.parametrize("alg", [ART_VISC_HK, ART_VISC_MON])
def test_uniform_compression_literal_equals_per_pair(oracle_mod, alg):
    b = _basin()
    c = b.x.mean(axis=0)
    b.vx = -1e-5 * (b.x - c)
    prm = _prm(b, art=1, alg=alg)
    lit, per = _rhs(oracle_mod, b, prm, True), _rhs(oracle_mod, b, prm, False)
    base = _rhs(oracle_mod, b, _prm(b), False)
    # the viscosity acts (the rates change) and both forms agree
    assert rel_l2(per["dvxdt"], base["dvxdt"]) > 1e-6
    assert np.array_equal(lit["dvxdt"], per["dvxdt"])


@pytest.mark.parametrize("alg", [ART_VISC_HK, ART_VISC_MON])
@pytest.mark.parametrize("literal", [False, True])
def test_artificial_viscosity_conserves_momentum(oracle_mod, alg, literal):
    b = _basin()
    b.vx = smooth_velocity(b.x, b.L, amp=0.5, seed=3)
    base = _rhs(oracle_mod, b, _prm(b), literal)
    reg = _rhs(oracle_mod, b, _prm(b, art=1, alg=alg), literal)
    av = reg["dvxdt"] - base["dvxdt"]
    assert np.abs(av).max() > 0.0
    p = (b.mass[:, None] * av).sum(axis=0)
    scale = (b.mass[:, None] * np.abs(av)).sum(axis=0)
    assert np.all(np.abs(p) <= 1e-12 * scale), (p, scale)


def test_xsph_momentum_per_pair_and_literal(oracle_mod):
    b = _basin()
    b.vx = smooth_velocity(b.x, b.L, amp=0.5, seed=4)
    out = {}
    for lit in (False, True):
        r = _rhs(oracle_mod, b, _prm(b, xsph=1), lit)
        out[lit] = (r["dxdt"] - b.vx)           # -chi xs
    m = b.mass[:, None]
    scale = (m * np.abs(out[False])).sum(axis=0)
    assert np.all(np.abs((m * out[False]).sum(axis=0)) <= 1e-12 * scale)
    # the literal form's same-signed term does not cancel
    assert np.any(np.abs((m * out[True]).sum(axis=0)) > 1e-3 * scale)


@pytest.mark.parametrize("alg", [ART_VISC_HK, ART_VISC_MON])
def test_mixed_flow_forms_differ(oracle_mod, alg):
    """Pairs on both sides of the criterion: the literal loop carries pi_ij
    into the pairs outside it, the per-pair form gives them none."""
    b = _basin()
    b.vx = smooth_velocity(b.x, b.L, amp=0.5, seed=5)
    prm = _prm(b, art=1, alg=alg)
    lit, per = _rhs(oracle_mod, b, prm, True), _rhs(oracle_mod, b, prm, False)
    assert not np.array_equal(lit["dvxdt"], per["dvxdt"])


def test_xsph_alone_still_runs_the_viscosity(oracle_mod):
    """regularization.f90:23-35: with xsph_regularization on and
    artificial_visc off the routine still applies art_visc_alg's viscosity
    (with c = 0, never refreshed by sound_speed)."""
    b = _basin()
    b.vx = smooth_velocity(b.x, b.L, amp=0.5, seed=6)
    base = _rhs(oracle_mod, b, _prm(b), False)
    xs_hk = _rhs(oracle_mod, b, _prm(b, xsph=1, alg=ART_VISC_HK), False)
    xs_none = _rhs(oracle_mod, b, _prm(b, xsph=1, alg=0), False)
    assert np.array_equal(xs_none["dvxdt"], base["dvxdt"])
    assert not np.array_equal(xs_hk["dvxdt"], base["dvxdt"])
