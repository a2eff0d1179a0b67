"""Parity of the CUDA path (through the C ABI) with the FP64 CPU oracle.

Bars: neighbour lists bit-exact as sorted index sets, with r_ij, hsml_ij and
br_ij bit-exact; FP64 fields within a relative L2 tolerance stated per test
(the GPU gathers each pair from both sides, so only the summation order
differs from the reference's scatter loop).
"""
import numpy as np
import pytest

from helpers import assert_same_pairs, rel_l2, smooth_velocity
from simp_b200 import basins
from simp_b200.params import SKF_WENDLAND_C6
from simp_b200.simp import (SIMP_ERR_BADARG, SIMP_ERR_IND_INT, SIMP_ERR_MAXN, SIMP_ERR_PAIR_CAP,
                            SIMP_ERR_STATE, Simp, SimpError)

pytestmark = pytest.mark.gpu

# FP64, one right-hand side on identical inputs: summation order only.
TOL_RHS = 1e-11
# FP64 trajectories: order-of-summation differences amplified by the
# non-smooth VP rheology over the stated number of steps.
TOL_TRAJ_20 = 1e-8


def _pair(b, oracle_mod, params=None):
    prm = b.params if params is None else params
    g = Simp.from_basin(b, prm)
    o = oracle_mod.Oracle.from_basin(b, prm)
    return g, o


def test_library_version(gpu_lib):
    from simp_b200.simp import version
    assert "sm_100a" in version()


@pytest.mark.parametrize("cfg", ["cfg1", "cfg1_c6", "cfg1_direct"])
def test_nnps_bit_exact_cfg1(gpu_lib, oracle_mod, cfg):
    b = basins.cfg1()
    prm = b.params.copy()
    if cfg == "cfg1_c6":
        prm.skf = SKF_WENDLAND_C6
    if cfg == "cfg1_direct":
        prm.nnps_algorithm = 1   # direct_find (nnps.f90:41-148): same pair set
    g, o = _pair(b, oracle_mod, prm)
    assert_same_pairs(g.nnps(), o.nnps())
    assert g.interaction_stats() == o.interaction_stats()


def test_nnps_bit_exact_cfg2(gpu_lib, oracle_mod):
    b = basins.cfg2()
    g, o = _pair(b, oracle_mod)
    assert_same_pairs(g.nnps(), o.nnps())


def test_nnps_after_motion(gpu_lib, oracle_mod):
    """Pair sets stay exact after particles moved (cell list not re-sorted)."""
    b = basins.cfg1()
    g, o = _pair(b, oracle_mod)
    g.time_integration(30)
    st = g.get_state()
    o.set_state(st["x"], st["vx"], st["mass"], st["rho"], st["hsml"], st["A"], st["h"],
                b.xb, b.massb, b.params.dt, st["current_time"])
    assert_same_pairs(g.nnps(), o.nnps())


def test_nnps_variable_hsml_bucket_rule(gpu_lib, oracle_mod):
    """max(hsml) > 2 min(hsml): the reference's bucket stencil drops pairs."""
    b = basins.cfg1()
    rng = np.random.default_rng(7)
    b.hsml = b.hsml * rng.uniform(0.9, 1.05, size=b.n)
    b.hsml[rng.choice(b.n, 5, replace=False)] *= 0.3   # bucket side 2 min(hsml) << max(hsml)
    g, o = _pair(b, oracle_mod)
    rg, ro = g.nnps(), o.nnps()
    assert_same_pairs(rg, ro)
    # the rule is active: brute force finds more pairs than the bucket search
    prm = b.params.copy()
    prm.nnps_algorithm = 1
    o2 = oracle_mod.Oracle.from_basin(b, prm)
    assert o2.nnps()["nip"] > ro["nip"]


def test_nnps_ties_and_half_buckets(gpu_lib, oracle_mod):
    """Unjittered lattice: pairs at exactly d == mhsml are kept (<=), and
    positions sit exactly on bucket half-boundaries (NINT ties)."""
    b = basins.make_basin(24, 1000.0, 3, jitter=0.0, walls="+x-x+y-y")
    b.hsml[:] = 2000.0          # mhsml = 2 dx = exact lattice distance
    b.x += 500.0                # x / (2 min hsml) = k / 4: every other column is a NINT tie
    b.xb += 500.0
    g, o = _pair(b, oracle_mod)
    rg, ro = g.nnps(), o.nnps()
    assert_same_pairs(rg, ro)
    # every interior particle has the 12 lattice neighbours within 2 dx
    assert ro["nip"] > 0


def test_nnps_pair_capacity(gpu_lib, oracle_mod):
    b = basins.cfg1()
    g = Simp.from_basin(b)
    with pytest.raises(SimpError) as e:
        g.nnps(cap=100)
    assert e.value.code == SIMP_ERR_PAIR_CAP


def test_maxn_error(gpu_lib):
    b = basins.cfg1()
    g = Simp(b.params, b.n - 1, b.nb)
    with pytest.raises(SimpError) as e:
        g.set_state(b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h, b.xb, b.massb, 1.0)
    assert e.value.code == SIMP_ERR_MAXN


def test_max_ind_int_error(gpu_lib):
    b = basins.cfg1()
    prm = b.params.copy()
    prm.max_ind_int = 10
    g = Simp.from_basin(b, prm)
    with pytest.raises(SimpError) as e:
        g.time_integration(1)
    assert e.value.code == SIMP_ERR_IND_INT


@pytest.mark.parametrize("skf", [9, 6, 1, 2, 3, 4, 5, 7, 8])
def test_single_step_fields(gpu_lib, oracle_mod, skf):
    """One RHS (single_step.f90) on a sheared, drifting state with drag on."""
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, seed=skf)
    prm = b.params.copy()
    prm.skf = skf
    g, o = _pair(b, oracle_mod, prm)
    rg, ro = g.single_step(3600.0), o.single_step(3600.0)
    for k in ("dxdt", "dvxdt", "dhdt", "dAdt"):
        assert rel_l2(rg[k], ro[k]) < TOL_RHS, (k, rel_l2(rg[k], ro[k]))
    dg, do = g.get_diag(), o.get_diag()
    for k in dg:
        assert rel_l2(dg[k], do[k]) < TOL_RHS, (k, rel_l2(dg[k], do[k]))


def test_single_step_at_rest_no_drag(gpu_lib, oracle_mod):
    """t = 0, v = 0: strain, stress and drag vanish; only walls act."""
    b = basins.cfg1()
    g, o = _pair(b, oracle_mod)
    rg, ro = g.single_step(0.0), o.single_step(0.0)
    assert rel_l2(rg["dvxdt"], ro["dvxdt"]) < TOL_RHS
    assert np.all(rg["dhdt"] == 0.0) and np.all(ro["dhdt"] == 0.0)
    d = g.get_diag()
    assert np.all(d["sig11"] == 0.0) and np.all(d["eps12"] == 0.0)


@pytest.mark.parametrize("skf", [1, 2, 3, 4, 5, 7, 8])
def test_other_kernels_density_and_steps(gpu_lib, oracle_mod, skf):
    """Every reference kernel (kernel.f90, boundary_kernel.f90): summation
    density and 5 steps against the oracle."""
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=30 + skf)
    prm = b.params.copy()
    prm.skf = skf
    g, o = _pair(b, oracle_mod, prm)
    assert rel_l2(g.sum_density(), o.sum_density()) < TOL_RHS
    g.time_integration(5)
    o.step(5)
    sg, so = g.get_state(), o.get_state()
    for k in ("x", "vx", "h", "A", "rho"):
        assert rel_l2(sg[k], so[k]) < 1e-9, (k, rel_l2(sg[k], so[k]))


def test_sum_density(gpu_lib, oracle_mod):
    b = basins.cfg1()
    for prm_skf in (9, 6):
        prm = b.params.copy()
        prm.skf = prm_skf
        g, o = _pair(b, oracle_mod, prm)
        assert rel_l2(g.sum_density(), o.sum_density(k0_mode=1)) < TOL_RHS


def test_trajectory_cfg1_20_steps(gpu_lib, oracle_mod):
    b = basins.cfg1()
    g, o = _pair(b, oracle_mod)
    tg, dtg = g.time_integration(20)
    to, dto = o.step(20)
    assert tg == to and dtg == dto
    sg, so = g.get_state(), o.get_state()
    for k in ("x", "vx", "h", "A", "rho"):
        assert rel_l2(sg[k] - (b.x if k == "x" else 0), so[k] - (b.x if k == "x" else 0)) < TOL_TRAJ_20, k


def test_single_step_after_motion_filters_lists_exactly(gpu_lib, oracle_mod):
    """After steps in which the Verlet lists stay valid, one RHS on the moved
    state equals the oracle's (which searches pairs from scratch)."""
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=2.0, seed=4)
    g = Simp.from_basin(b)
    g.time_integration(12)
    st = g.get_state()
    o = oracle_mod.Oracle.from_basin(b)
    o.set_state(st["x"], st["vx"], st["mass"], st["rho"], st["hsml"], st["A"], st["h"],
                b.xb, b.massb, b.params.dt, st["current_time"])
    rg, ro = g.single_step(st["current_time"]), o.single_step(st["current_time"])
    for k in ("dvxdt", "dhdt", "dAdt"):
        assert rel_l2(rg[k], ro[k]) < TOL_RHS, (k, rel_l2(rg[k], ro[k]))


def test_trajectory_fast_motion_rebuilds(gpu_lib, oracle_mod):
    """Displacements of tens of metres per step: the Verlet lists (skin
    480 m) are rebuilt every few steps and the cell list is re-sorted; the
    trajectory still follows the oracle's."""
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=8.0, seed=5)
    prm = b.params.copy()
    prm.dt = 5.0
    g, o = _pair(b, oracle_mod, prm)
    for _ in range(4):
        g.time_integration(5)
        o.step(5)
        sg, so = g.get_state(), o.get_state()
        for k in ("vx", "h"):
            assert rel_l2(sg[k], so[k]) < TOL_TRAJ_20, (k, rel_l2(sg[k], so[k]))
        # same inputs for both from here on: pair lists bit-exact
        o.set_state(sg["x"], sg["vx"], sg["mass"], sg["rho"], sg["hsml"], sg["A"], sg["h"],
                    b.xb, b.massb, prm.dt, sg["current_time"])
        assert_same_pairs(g.nnps(), o.nnps())


def test_few_fast_particles_cross_the_lists(gpu_lib, oracle_mod):
    """Nine particles at 30 m/s through a basin at rest: they leave the
    Verlet skin (480 m) within a few steps while every other particle stays
    put; the lists are rebuilt in time and every pair is still found."""
    b = basins.cfg1()
    b.vx = np.zeros_like(b.vx)
    c = np.argsort(np.hypot(b.x[:, 0] - 0.5 * b.L, b.x[:, 1] - 0.5 * b.L))[:9]
    b.vx[c] = (30.0, 12.0)
    prm = b.params.copy()
    prm.dt = 5.0
    g, o = _pair(b, oracle_mod, prm)
    for _ in range(3):
        g.time_integration(4)
        o.step(4)
        sg, so = g.get_state(), o.get_state()
        for k in ("x", "vx", "h"):
            ref = b.x if k == "x" else 0.0
            assert rel_l2(sg[k] - ref, so[k] - ref) < TOL_TRAJ_20, (k, rel_l2(sg[k] - ref, so[k] - ref))
        o.set_state(sg["x"], sg["vx"], sg["mass"], sg["rho"], sg["hsml"], sg["A"], sg["h"],
                    b.xb, b.massb, prm.dt, sg["current_time"])
        assert_same_pairs(g.nnps(), o.nnps())
    assert np.max(np.hypot(*(sg["x"][c] - b.x[c]).T)) > 480.0      # past the skin


def test_trajectory_vp_timestep_and_marquis_hsml(gpu_lib, oracle_mod):
    """Reference default switches: sle = 2 (Marquis hsml), tse = 2 (VP dt),
    Wendland C6, mass from the lattice."""
    from simp_b200.params import reference_default
    b = basins.cfg1()
    prm = reference_default()
    prm.wind_u, prm.wind_v = 10.0, 0.0
    prm.b_length = 4.0 * b.dx
    b.hsml[:] = 3.0 * b.dx   # hsml_multiplicity * dx (initialize.f90:190)
    # initialize.f90:199 calls time_step before the loop: the VP dt
    prm.dt = prm.rho_ice * (3.0 * b.dx) ** 2 * prm.delta_min / (prm.P_star * (1.0 + prm.k_t))
    g, o = _pair(b, oracle_mod, prm)
    tg, dtg = g.time_integration(10)
    to, dto = o.step(10)
    assert abs(tg - to) <= 1e-12 * abs(to) and dtg == dto
    sg, so = g.get_state(), o.get_state()
    for k in ("vx", "h", "hsml"):
        assert rel_l2(sg[k], so[k]) < TOL_TRAJ_20, k


# --- switch variants of the path -------------------------------------------

def _variant(b, **kw):
    prm = b.params.copy()
    for k, v in kw.items():
        setattr(prm, k, v)
    return prm


VARIANTS = {
    # (Mohr-Coulomb viscosities up to these caps make the explicit step at
    # dt = 1 s amplify rounding differences; 1e-3 s is under the VP bound)
    "mohr_coulomb": dict(rheology=2, zeta_max=2.5e8, eta_max=1.0e8, dt=1e-3),
    "gutfraind_eos": dict(eos_alg=2),
    "hibler_eos": dict(eos_alg=1),
    "stress_2": dict(pa_sph=2),
    "euler": dict(int_algorithm=1),
    "leapfrog": dict(int_algorithm=3),
    # continuity density (density.f90:107-165) under each integrator
    "con_density": dict(den_alg=2),
    "con_density_euler": dict(den_alg=2, int_algorithm=1),
    "con_density_leapfrog": dict(den_alg=2, int_algorithm=3),
    # Benz hsml (smoothing_length.f90:40-111): with the diagnostic density
    # its drhodt accumulates over the steps; with con_density it does not
    "benz_hsml": dict(sle=1),
    "benz_hsml_euler": dict(sle=1, int_algorithm=1),
    "benz_hsml_leapfrog": dict(sle=1, int_algorithm=3, tse=2),
    "benz_con_density": dict(sle=1, den_alg=2, tse=2),
    "benz_con_density_euler": dict(sle=1, den_alg=2, int_algorithm=1),
    "benz_mass_from_area": dict(sle=1, mass_from_area=1),
    # Monaghan time step (time_step.f90:40-103): force and CFL criteria
    "monaghan_dt": dict(tse=1),
    "monaghan_dt_benz_euler": dict(tse=1, sle=1, int_algorithm=1),
    # Marquis hsml from the continuity density (after the density pass)
    "marquis_con_density": dict(sle=2, den_alg=2),
    "marquis_con_density_leapfrog": dict(sle=2, den_alg=2, int_algorithm=3),
}


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_switch_variants_against_oracle(gpu_lib, oracle_mod, name):
    """Rheology (bulk_viscosity.f90, shear_viscosity.f90), equation of state
    (eos.f90), stress form (internal_stress.f90) and integrator
    (time_integration.f90) switches: one right-hand side and 10 steps."""
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=40)
    b.h = b.h * np.linspace(0.9, 1.1, b.n)      # thickness varies: the Gutfraind pressure is live
    b.rho = b.h * 900.0
    prm = _variant(b, **VARIANTS[name])
    g, o = _pair(b, oracle_mod, prm)
    rg, ro = g.single_step(3600.0), o.single_step(3600.0)
    for k in ("dvxdt", "dhdt", "dAdt"):
        assert rel_l2(rg[k], ro[k]) < TOL_RHS, (k, rel_l2(rg[k], ro[k]))
    g2, o2 = _pair(b, oracle_mod, prm)
    g2.time_integration(10)
    o2.step(10)
    sg, so = g2.get_state(), o2.get_state()
    for k in ("x", "vx", "h", "A", "rho", "hsml"):
        assert rel_l2(sg[k], so[k]) < 1e-9, (k, rel_l2(sg[k], so[k]))
    assert sg["current_time"] == pytest.approx(so["current_time"])
    if prm.sle != 0 or prm.den_alg == 2:
        # the variant is live: hsml or rho moved away from their start
        moved = sg["hsml"] if prm.sle != 0 else sg["rho"]
        start = b.hsml if prm.sle != 0 else b.rho
        assert not np.array_equal(moved, start)


# Boundary force variants (boundary_force.f90): basin walled on four sides,
# moving into its walls.  The Wang force adds m_i v / dt per wall pair to an
# acceleration, as the reference does, so its trajectories run away: it is
# checked on one right-hand side.
BOUNDARY = {
    "monaghan_friction": (dict(boundary_friction=1), 10),
    "monaghan_friction_c6": (dict(boundary_friction=1, skf=6), 10),
    "wang": (dict(bfa=2), 0),
    "wang_friction": (dict(bfa=2, boundary_friction=1), 0),
    "marquis_pressure": (dict(bfa=3), 10),
    # (its friction decelerates by up to 1/s per wall pair: explicit steps of
    # 1 s overshoot, as they would in the reference)
    "marquis_friction": (dict(bfa=3, boundary_pressure=0, boundary_friction=1, dt=1e-2), 10),
}


def _walled_basin():
    b = basins.make_basin(50, 2000.0, 11, walls="+x-x+y-y")
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=41)
    b.h = b.h * np.linspace(0.9, 1.1, b.n)
    b.rho = b.h * 900.0
    return b


@pytest.mark.parametrize("name", sorted(BOUNDARY))
def test_boundary_force_variants_against_oracle(gpu_lib, oracle_mod, name):
    b = _walled_basin()
    kw, nsteps = BOUNDARY[name]
    prm = _variant(b, **kw)
    g, o = _pair(b, oracle_mod, prm)
    rg, ro = g.single_step(3600.0), o.single_step(3600.0)
    for k in ("dvxdt", "dhdt", "dAdt"):
        assert rel_l2(rg[k], ro[k]) < TOL_RHS, (k, rel_l2(rg[k], ro[k]))
    if prm.bfa == 3 and prm.boundary_pressure:
        # bf_Marquis with the pressure switch on returns at once: no wall force
        q = _variant(b, **dict(kw, boundary_pressure=0))
        r0 = Simp.from_basin(b, q).single_step(3600.0)
        assert np.array_equal(rg["dvxdt"], r0["dvxdt"])
    if nsteps:
        g2, o2 = _pair(b, oracle_mod, prm)
        g2.time_integration(nsteps)
        o2.step(nsteps)
        sg, so = g2.get_state(), o2.get_state()
        for k in ("x", "vx", "h", "A", "rho"):
            assert rel_l2(sg[k], so[k]) < 1e-9, (k, rel_l2(sg[k], so[k]))


def test_wang_force_needs_wall_normals(gpu_lib):
    b = _walled_basin()
    prm = _variant(b, bfa=2)
    g = Simp(prm, b.n, b.nb)
    g.set_state(b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h, b.xb, b.massb, prm.dt, 0.0)
    with pytest.raises(SimpError) as ex:
        g.time_integration(1)
    assert ex.value.code == SIMP_ERR_STATE
    with pytest.raises(SimpError) as ex:
        g.set_wall_normals(b.bn[:-1])
    assert ex.value.code == SIMP_ERR_BADARG
    g.set_wall_normals(b.bn)
    g.single_step(3600.0)


def _map_basin(bfa):
    from simp_b200 import domain
    m = np.zeros((16, 12), dtype=np.int32)
    m[1:15, 1:11] = 1
    m[8:15, 1:6] = 0                             # a land notch: an L-shaped basin
    prm = basins.basin_params(1000.0, dt=1.0, wind=(8.0, 3.0))
    prm.bfa = bfa
    b = domain.basin_from_map(m, 4000.0, 1000.0, 10000.0, 150000.0, prm)
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=44)
    return b


def test_map_domain_basin_against_oracle(gpu_lib, oracle_mod):
    """An L-shaped map domain (particle_placing, boundary_placing_1): walls
    on every land/ice edge, including the re-entrant corner; 10 steps."""
    b = _map_basin(1)
    g, o = _pair(b, oracle_mod)
    rg, ro = g.single_step(3600.0), o.single_step(3600.0)
    for k in ("dvxdt", "dhdt", "dAdt"):
        assert rel_l2(rg[k], ro[k]) < TOL_RHS, (k, rel_l2(rg[k], ro[k]))
    g2, o2 = _pair(b, oracle_mod)
    g2.time_integration(10)
    o2.step(10)
    sg, so = g2.get_state(), o2.get_state()
    for k in ("vx", "h", "A"):
        assert rel_l2(sg[k], so[k]) < 1e-9, (k, rel_l2(sg[k], so[k]))


def test_map_domain_wang_force_with_refitted_normals(gpu_lib, oracle_mod):
    """bfa = 2 on the map domain, normals refitted by boundary_normal
    (diagonal at the corners): one right-hand side."""
    b = _map_basin(2)
    assert np.any(np.all(np.abs(b.bn) > 0.1, axis=1))           # some diagonal normals
    g, o = _pair(b, oracle_mod)
    rg, ro = g.single_step(3600.0), o.single_step(3600.0)
    for k in ("dvxdt", "dhdt", "dAdt"):
        assert rel_l2(rg[k], ro[k]) < TOL_RHS, (k, rel_l2(rg[k], ro[k]))


def test_map_domain_multilayer_walls_against_oracle(gpu_lib, oracle_mod):
    """The same map with three-line walls (boundary_placing_2): more wall
    pairs per particle; one right-hand side and 5 steps."""
    from simp_b200 import domain
    m = np.zeros((16, 12), dtype=np.int32)
    m[1:15, 1:11] = 1
    m[8:15, 1:6] = 0
    prm = basins.basin_params(1000.0, dt=1.0, wind=(8.0, 3.0))
    b = domain.basin_from_map(m, 4000.0, 1000.0, 10000.0, 150000.0, prm, b_setup=2)
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=45)
    g, o = _pair(b, oracle_mod)
    rg, ro = g.single_step(3600.0), o.single_step(3600.0)
    for k in ("dvxdt", "dhdt", "dAdt"):
        assert rel_l2(rg[k], ro[k]) < TOL_RHS, (k, rel_l2(rg[k], ro[k]))
    g2, o2 = _pair(b, oracle_mod)
    g2.time_integration(5)
    o2.step(5)
    sg, so = g2.get_state(), o2.get_state()
    for k in ("vx", "h"):
        assert rel_l2(sg[k], so[k]) < 1e-9, (k, rel_l2(sg[k], so[k]))


def test_benz_drhodt_follows_particles_through_resorts(gpu_lib, oracle_mod):
    """Benz hsml with the diagnostic density keeps the reference's
    never-cleared drhodt per particle; 20 steps cross the re-sort at step 16,
    which moves that array with the particles."""
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=46)
    prm = _variant(b, sle=1)
    g, o = _pair(b, oracle_mod, prm)
    g.time_integration(20)
    o.step(20)
    sg, so = g.get_state(), o.get_state()
    for k in ("hsml", "vx", "h"):
        assert rel_l2(sg[k], so[k]) < TOL_TRAJ_20, (k, rel_l2(sg[k], so[k]))
    assert not np.array_equal(sg["hsml"], b.hsml)


def test_con_density_mixed_precision(gpu_lib):
    """The continuity density in the mixed form against the plain form:
    its density-rate pass is FP64 in both."""
    from simp_b200.params import PREC_MIXED
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=47)
    p64 = _variant(b, den_alg=2, dt=1e-3)
    p32 = _variant(b, den_alg=2, dt=1e-3, precision=PREC_MIXED)
    g64, g32 = Simp.from_basin(b, p64), Simp.from_basin(b, p32)
    g64.time_integration(10)
    g32.time_integration(10)
    s64, s32 = g64.get_state(), g32.get_state()
    for k in ("rho", "vx", "h"):
        assert rel_l2(s32[k], s64[k]) < 1e-6, (k, rel_l2(s32[k], s64[k]))
    assert not np.array_equal(s64["rho"], b.rho)


@pytest.mark.parametrize("n", [1, 2, 3])
@pytest.mark.parametrize("walls", ["", "+x"])
def test_tiny_basins(gpu_lib, oracle_mod, n, walls):
    """Ragged smallest inputs: one, two or three particles (no pair, one
    pair, a chain), with and without a wall line: pairs, one right-hand side
    and five steps against the oracle."""
    b = basins.make_basin(3, 2000.0, 60 + n, walls=walls)
    keep = np.arange(n)
    for k in ("mass", "rho", "hsml", "A", "h"):
        setattr(b, k, getattr(b, k)[keep].copy())
    b.x = b.x[keep].copy()
    b.vx = np.tile([0.2, -0.1], (n, 1)) * (1.0 + np.arange(n))[:, None]
    g, o = _pair(b, oracle_mod)
    assert_same_pairs(g.nnps(), o.nnps())
    rg, ro = g.single_step(600.0), o.single_step(600.0)
    for k in ("dxdt", "dvxdt", "dhdt", "dAdt"):
        assert rel_l2(rg[k], ro[k]) < TOL_RHS, (k, rel_l2(rg[k], ro[k]))
    g.time_integration(5)
    o.step(5)
    sg, so = g.get_state(), o.get_state()
    for k in ("x", "vx", "h", "A"):
        assert rel_l2(sg[k], so[k]) < 1e-9, (k, rel_l2(sg[k], so[k]))
