"""Known-answer tests pinning the CPU oracle (no GPU).

The reference has no tests or golden vectors and cannot be compiled here, so
the oracle is pinned to closed-form values (tests/golden/, generated by
tests/golden/make_golden.py from the formulas) and to exact invariants of
the reference's algorithm.
"""
import json
import os

import numpy as np
import pytest

from helpers import canonical_pairs, smooth_velocity
from simp_b200 import basins
from simp_b200.params import (KERNELS, SKF_CUBIC, SKF_WENDLAND_C6, basin_params,
                              reference_default)

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def _params(skf):
    p = basin_params(1000.0, skf=skf)
    return p


@pytest.mark.parametrize("skf", sorted(KERNELS))
def test_kernel_matches_closed_form(oracle_mod, skf):
    g = _load("kat_kernels.json")
    key = KERNELS[skf][0]
    p = _params(skf)
    for e in g[key]:
        w, gx, gy, _ = oracle_mod.kernel(p, e["r"], g["hsml_ij"], e["r"], 0.0)
        assert w == pytest.approx(e["w"], rel=1e-11, abs=1e-30), (key, e["q"])
        assert gx == pytest.approx(e["dwdr"], rel=1e-10, abs=1e-30), (key, e["q"])
        assert gy == 0.0


# The reference's Wendland C2 factor 3/(2 pi) gives an integral of 3/14, and
# its Marquis2 factor, which leaves out scale_h^2 = 9, gives 1/9; the others
# integrate to 1.
@pytest.mark.parametrize("skf,want,tol", [(SKF_WENDLAND_C6, 1.0, 2e-6), (SKF_CUBIC, 1.0, 2e-6), (1, 1.0, 2e-6),
                                          (2, 1.0, 2e-4), (3, 1.0, 2e-6), (4, 3.0 / 14.0, 2e-6),
                                          (5, 1.0, 2e-6), (7, 1.0, 2e-3), (8, 1.0 / 9.0, 2e-4)])
def test_kernel_normalisation(oracle_mod, skf, want, tol):
    """integral of W over its support (cubic: to its single-precision
    literals, ~3e-8; Gaussian: 1 - exp(-9) on its support q <= 3)."""
    p = _params(skf)
    hij = 1000.0
    support = hij  # SIMP hsml is the support radius of every kernel
    r = np.linspace(0.0, support, 20001)[1:]
    w = np.array([oracle_mod.kernel(p, ri, hij, ri, 0.0)[0] for ri in r])
    integral = np.trapezoid(2 * np.pi * r * w, r)
    assert integral == pytest.approx(want, abs=tol)


@pytest.mark.parametrize("skf", sorted(KERNELS))
def test_gradient_is_odd(oracle_mod, skf):
    p = _params(skf)
    rng = np.random.default_rng(0)
    for _ in range(50):
        dx, dy = rng.uniform(-600, 600, size=2)
        r = float(np.hypot(dx, dy))
        a = oracle_mod.kernel(p, r, 1000.0, dx, dy)
        b = oracle_mod.kernel(p, r, 1000.0, -dx, -dy)
        assert a[1] == -b[1] and a[2] == -b[2]


@pytest.mark.parametrize("ratio", ["2.4", "3.0"])
def test_lattice_neighbour_counts(oracle_mod, ratio):
    want = _load("kat_lattice.json")["support_over_dx"][ratio]
    b = basins.make_basin(30, 1000.0, 1, jitter=0.0, walls="")
    b.hsml[:] = float(ratio) * 1000.0
    for alg in (1, 2):
        p = b.params.copy()
        p.nnps_algorithm = alg
        o = oracle_mod.Oracle.from_basin(b, p)
        o.nnps()
        assert o.interaction_stats()["maxip"] == want


def test_bucket_search_equals_direct_find(oracle_mod):
    b = basins.cfg1()
    res = []
    for alg in (1, 2):
        p = b.params.copy()
        p.nnps_algorithm = alg
        res.append(oracle_mod.Oracle.from_basin(b, p).nnps())
    a, d = (canonical_pairs(r) for r in res)
    assert res[0]["nip"] == res[1]["nip"]
    for u, v in zip(a, d):
        assert np.array_equal(u, v)


def test_bucket_rule_drops_pairs_when_hsml_varies(oracle_mod):
    """With max(hsml) > 2 min(hsml) the 3x3 bucket stencil of side
    2 min(hsml) misses pairs that direct find keeps (nnps.f90:211, 259-407)."""
    b = basins.cfg1()
    rng = np.random.default_rng(7)
    b.hsml = b.hsml * rng.uniform(0.9, 1.05, size=b.n)
    b.hsml[rng.choice(b.n, 5, replace=False)] *= 0.3
    p1, p2 = b.params.copy(), b.params.copy()
    p1.nnps_algorithm = 1
    d = oracle_mod.Oracle.from_basin(b, p1).nnps()
    k = oracle_mod.Oracle.from_basin(b, p2).nnps()
    assert k["nip"] < d["nip"]
    dset = set(zip(*canonical_pairs(d)[:2]))
    kset = set(zip(*canonical_pairs(k)[:2]))
    assert kset < dset


def test_rigid_translation_has_zero_strain_and_stress(oracle_mod):
    b = basins.make_basin(30, 2000.0, 5, walls="")
    b.vx[:] = (0.3, -0.1)
    o = oracle_mod.Oracle.from_basin(b)
    r = o.single_step(0.0)
    d = o.get_diag()
    for k in ("eps11", "eps12", "eps22", "sig11", "sig12", "sig22", "p"):
        assert np.all(d[k] == 0.0), k
    assert np.all(r["dvxdt"] == 0.0) and np.all(r["dhdt"] == 0.0)


def test_internal_stress_conserves_momentum(oracle_mod):
    """stress_1 with rho = rho_ice h adds m_j (c_i + c_j) to i and the
    negative to j: sum_i m_i a_i = 0 to round-off."""
    b = basins.make_basin(40, 2000.0, 6, walls="")
    b.vx = smooth_velocity(b.x, b.L, seed=3)
    o = oracle_mod.Oracle.from_basin(b)
    a = o.single_step(0.0)["dvxdt"]
    mom = (b.mass[:, None] * a).sum(axis=0)
    scale = np.abs(b.mass[:, None] * a).sum(axis=0)
    assert np.all(np.abs(mom) <= 1e-12 * scale)
    assert np.all(scale > 0)


def test_free_drift_speed(oracle_mod):
    """Uniform ice, uniform wind, no walls: strain stays exactly zero and the
    ice reaches the drag balance rho_a c_a (U-u)^2 = rho_w c_w u^2."""
    phys = _load("kat_physics.json")
    b = basins.make_basin(6, 2000.0, 2, walls="", wind=(phys["wind"], 0.0), dt=30.0)
    o = oracle_mod.Oracle.from_basin(b)
    o.step(1000)
    st = o.get_state()
    assert np.allclose(st["vx"][:, 0], phys["free_drift_speed"], rtol=1e-6, atol=0)
    assert np.all(np.abs(st["vx"][:, 1]) < 1e-12)


def test_mass_is_conserved(oracle_mod):
    p = reference_default()
    b = basins.cfg1()
    p.wind_u, p.wind_v, p.b_length = 10.0, 0.0, 8000.0
    b.hsml[:] = 3.0 * b.dx
    p.dt = p.rho_ice * (3.0 * b.dx) ** 2 * p.delta_min / p.P_star
    o = oracle_mod.Oracle.from_basin(b, p)
    o.step(5)
    assert np.array_equal(o.get_state()["mass"], b.mass)


@pytest.mark.parametrize("skf", sorted(KERNELS))
def test_boundary_kernel_gradient_is_derivative(oracle_mod, skf):
    """bdwdx of each boundary kernel is the derivative of its bw
    (boundary_kernel.f90): factor dW/dq against a central difference."""
    p = _params(skf)
    sh = KERNELS[skf][1]
    bl = p.b_length
    # (8 points: none on the piecewise kernels' knots q = 1, 2, where the
    # single-precision literals of the cubic leave a 1e-8 step in bw)
    for br in np.linspace(0.07, 0.93, 8) * bl:
        e = 1e-6 * bl
        num = (oracle_mod.boundary_w(p, br + e) - oracle_mod.boundary_w(p, br - e)) / (2 * e) * bl / sh
        got = oracle_mod.boundary_fdwdq(p, br)
        assert got == pytest.approx(num, rel=1e-5, abs=1e-7 * abs(oracle_mod.boundary_w(p, 0.0))), (skf, br)


def _stepped(oracle_mod, b, nsteps=1, **kw):
    p = b.params.copy()
    for k, v in kw.items():
        setattr(p, k, v)
    o = oracle_mod.Oracle.from_basin(b, p)
    o.step(nsteps)
    return o.get_state()


@pytest.mark.parametrize("int_algorithm", [1, 2, 3])
def test_con_density_keeps_density_under_translation(oracle_mod, int_algorithm):
    """con_density: a uniform velocity gives drho/dt = 0 exactly, whatever
    the integrator (density.f90:107-165)."""
    b = basins.make_basin(30, 2000.0, 5, walls="")
    b.vx[:] = (0.3, -0.1)
    st = _stepped(oracle_mod, b, 2, den_alg=2, int_algorithm=int_algorithm)
    assert np.array_equal(st["rho"], b.rho)
    assert not np.array_equal(st["x"], b.x)


def _dilating(eps):
    b = basins.make_basin(40, 2000.0, 9, walls="")
    c = 0.5 * b.L
    b.vx = np.ascontiguousarray(eps * (b.x - c))
    inner = np.all(np.abs(b.x - c) < 0.3 * b.L, axis=1)
    return b, inner


@pytest.mark.parametrize("int_algorithm", [1, 2, 3])
def test_con_density_uniform_dilatation(oracle_mod, int_algorithm):
    """v = eps (x - c) has div v = 2 eps: away from the free edges the SPH
    continuity equation gives drho/dt = -2 eps rho to the kernel's
    discretisation error (a jittered lattice, cubic spline)."""
    eps, dt = 1.0e-4, 1.0e-6
    b, inner = _dilating(eps)
    st = _stepped(oracle_mod, b, 1, den_alg=2, int_algorithm=int_algorithm, dt=dt)
    ratio = ((st["rho"] - b.rho) / dt / (-2.0 * eps * b.rho))[inner]
    assert np.all(np.abs(ratio - 1.0) < 0.05)          # (a 5% jitter of the lattice)
    assert abs(np.mean(ratio) - 1.0) < 0.015


def test_benz_hsml_follows_density(oracle_mod):
    """Benz_hsml with con_density: dh/dt = -hsml drho/dt / (2 rho) = eps hsml
    for the dilatation (smoothing_length.f90:82-94)."""
    eps, dt = 1.0e-4, 1.0e-6
    b, inner = _dilating(eps)
    st = _stepped(oracle_mod, b, 1, den_alg=2, sle=1, int_algorithm=1, dt=dt)
    ratio = ((st["hsml"] - b.hsml) / dt / (eps * b.hsml))[inner]
    assert np.all(np.abs(ratio - 1.0) < 0.05)
    assert abs(np.mean(ratio) - 1.0) < 0.015


def test_benz_hsml_accumulates_without_con_density(oracle_mod):
    """Without con_density, Benz_hsml adds each step's pair sum to drhodt,
    which nothing clears (smoothing_length.f90:62-80): in a steady
    dilatation the second step changes hsml about twice as much as the
    first.  With con_density the two changes are about equal."""
    eps, dt = 1.0e-4, 1.0e-6
    b, inner = _dilating(eps)
    for den_alg, ratio in ((3, 2.0), (2, 1.0)):
        s1 = _stepped(oracle_mod, b, 1, den_alg=den_alg, sle=1, int_algorithm=1, dt=dt)
        s2 = _stepped(oracle_mod, b, 2, den_alg=den_alg, sle=1, int_algorithm=1, dt=dt)
        d1 = (s1["hsml"] - b.hsml)[inner]
        d2 = (s2["hsml"] - s1["hsml"])[inner]
        assert np.allclose(d2 / d1, ratio, rtol=0.01), den_alg


def test_monaghan_time_step_is_cfl_at_rest(oracle_mod):
    """With no acceleration the force criterion is infinite and the time
    step is min(hsml / c), c = (Y (1 - nu) / (rho (1 + nu) (1 - 2 nu)))^0.5
    (time_step.f90:40-103, sound_speed.f90:54-55)."""
    b = basins.make_basin(20, 2000.0, 3, walls="", wind=(0.0, 0.0))
    p = b.params.copy()
    p.tse = 1
    o = oracle_mod.Oracle.from_basin(b, p)
    o.step(1)
    Y, nu = p.Y, p.nu
    c = np.sqrt(Y * (1 - nu) / (b.rho * (1 + nu) * (1 - 2 * nu)))
    assert o.get_state()["dt"] == pytest.approx(np.min(b.hsml / c), rel=1e-12)


def test_reference_default_literals():
    """Default-real literals of data_variables.f90 keep single precision."""
    p = reference_default()
    assert p.rho_air == np.float32(1.3)
    assert p.rho_air != 1.3
    assert p.e == 2.0 and p.k_t == 0.0 and p.P_star == 27500.0
