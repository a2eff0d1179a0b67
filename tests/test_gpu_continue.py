"""set_state of a state that continues the resident basin.

A host that owns the state and calls set_state before every step (the
drop-in shim of single_step) hands back the state it just read, or that
state changed a little.  Then the library writes it into the particles'
current places and keeps the sort, the cell lists and the Verlet lists:
- handing back the state unchanged gives bitwise the device-resident run;
- a changed state gives the pairs of the oracle exactly and the rates of a
  fresh set_state within FP64 rounding (the summation order differs);
- anything else (other walls, other hsml, particles moved farther than a
  cell) is set up from scratch, bitwise as in a new context.
Whether a call continued is read from the kernel count: a continued
set_state launches six kernels (one per part of the upload, which run
while the next part is copied, and the bounds), a fresh one many more.
"""
import numpy as np
import pytest

from helpers import assert_same_pairs, rel_l2, smooth_velocity
from simp_b200 import basins
from simp_b200.params import PREC_MIXED
from simp_b200.simp import Simp

pytestmark = pytest.mark.gpu

KEYS = ("x", "vx", "mass", "rho", "hsml", "A", "h")
CONTINUED = 6   # kernels of a continued set_state


def _launches(g):
    return int(g.lib.simp_gpu_kernel_launches(g.h))


def _set(g, b, st, **changes):
    """set_state of st (with changes) and the kernels it launched."""
    v = {k: np.array(st[k], copy=True) for k in KEYS}
    v.update(changes)
    l0 = _launches(g)
    g.set_state(v["x"], v["vx"], v["mass"], v["rho"], v["hsml"], v["A"], v["h"], b.xb, b.massb,
                st["dt"], st["current_time"])
    return _launches(g) - l0, v


def _moving_cfg1(amp=0.5, seed=31):
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=amp, seed=seed)
    return b


@pytest.mark.parametrize("switches", ["cfg1", "reference_defaults", "mixed"])
def test_handing_back_the_state_is_the_device_resident_run(gpu_lib, switches):
    b = _moving_cfg1()
    prm = b.params.copy()
    if switches == "mixed":
        prm.precision = PREC_MIXED
    if switches == "reference_defaults":
        # Marquis hsml (sle 2) and the VP time step (tse 2): hsml and dt
        # change every step, and the lists are rebuilt every step
        prm.sle, prm.tse = 2, 2
        prm.max_hsml = 3.0 * float(np.max(b.hsml))
    resident = Simp.from_basin(b, prm)
    resident.time_integration(24)
    host = Simp.from_basin(b, prm)
    for _ in range(24):
        st = host.get_state()
        launched, _ = _set(host, b, st)
        assert launched == CONTINUED
        host.time_integration(1)
    a, c = resident.get_state(), host.get_state()
    for k in KEYS + ("dt", "current_time"):
        assert np.array_equal(np.asarray(c[k]), np.asarray(a[k])), k
    assert_same_pairs(host.nnps(), resident.nnps())
    resident.close()
    host.close()


def test_changed_state_matches_oracle_pairs_and_fresh_rates(gpu_lib, oracle_mod):
    b = _moving_cfg1(amp=1.0, seed=32)
    g = Simp.from_basin(b)
    g.time_integration(6)
    st = g.get_state()
    rng = np.random.default_rng(33)
    x = st["x"] + rng.uniform(-40.0, 40.0, st["x"].shape)       # far less than a cell (~6 km)
    vx = 1.1 * st["vx"] + rng.normal(0.0, 0.05, st["vx"].shape)
    h = st["h"] * rng.uniform(0.99, 1.01, st["h"].shape)
    launched, v = _set(g, b, st, x=x, vx=vx, h=h, rho=900.0 * h)
    assert launched == CONTINUED
    fresh = Simp(b.params, b.n, b.nb)
    fresh.set_state(v["x"], v["vx"], v["mass"], v["rho"], v["hsml"], v["A"], v["h"], b.xb, b.massb,
                    st["dt"], st["current_time"])
    o = oracle_mod.Oracle.from_basin(b)
    o.set_state(v["x"], v["vx"], v["mass"], v["rho"], v["hsml"], v["A"], v["h"], b.xb, b.massb,
                st["dt"], st["current_time"])
    assert_same_pairs(g.nnps(), o.nnps())
    assert_same_pairs(fresh.nnps(), o.nnps())
    rg, rf = g.single_step(st["current_time"]), fresh.single_step(st["current_time"])
    for k in rg:
        assert rel_l2(rg[k], rf[k]) < 1e-11, (k, rel_l2(rg[k], rf[k]))
    g.time_integration(8)
    fresh.time_integration(8)
    a, c = fresh.get_state(), g.get_state()
    for k in ("x", "vx", "h", "A"):
        ref = b.x if k == "x" else 0.0
        assert rel_l2(c[k] - ref, a[k] - ref) < 1e-8, (k, rel_l2(c[k] - ref, a[k] - ref))
    g.close()
    fresh.close()


@pytest.mark.parametrize("change", ["far_motion", "hsml", "walls"])
def test_other_states_start_fresh(gpu_lib, change):
    b = _moving_cfg1(seed=34)
    g = Simp.from_basin(b)
    g.time_integration(5)
    st = g.get_state()
    v = {k: np.array(st[k], copy=True) for k in KEYS}
    xb, massb = b.xb.copy(), b.massb.copy()
    if change == "far_motion":
        v["x"][7] += (9000.0, 0.0)          # one particle more than a cell (~6 km) away
    elif change == "hsml":
        v["hsml"][11] *= 1.001
    else:
        xb[0, 1] += 1.0
    l0 = _launches(g)
    g.set_state(v["x"], v["vx"], v["mass"], v["rho"], v["hsml"], v["A"], v["h"], xb, massb,
                st["dt"], st["current_time"])
    assert _launches(g) - l0 > 2
    fresh = Simp(b.params, b.n, b.nb)
    fresh.set_state(v["x"], v["vx"], v["mass"], v["rho"], v["hsml"], v["A"], v["h"], xb, massb,
                    st["dt"], st["current_time"])
    g.time_integration(4)
    fresh.time_integration(4)
    a, c = fresh.get_state(), g.get_state()
    for k in KEYS + ("dt", "current_time"):
        assert np.array_equal(np.asarray(c[k]), np.asarray(a[k])), k
    g.close()
    fresh.close()


def test_invalid_state_is_refused_as_before(gpu_lib):
    b = _moving_cfg1(seed=35)
    g = Simp.from_basin(b)
    g.time_integration(2)
    st = g.get_state()
    rho = st["rho"].copy()
    rho[3] = -1.0
    from simp_b200.simp import SimpError
    with pytest.raises(SimpError):
        _set(g, b, st, rho=rho)
    g.close()


def test_host_integrator_over_gpu_single_step(gpu_lib):
    """The pattern of the single_step shim: the reference's predictor-
    corrector (time_integration.f90:196-266) on the host, each right-hand
    side from set_state + single_step.  Every set_state continues in place
    (the half-step states included), and the trajectory follows the GPU's
    own time_integration to FP64 rounding."""
    b = _moving_cfg1(seed=36)
    rho_ice = b.params.rho_ice
    g = Simp.from_basin(b)
    st = g.get_state()
    dt, t = st["dt"], st["current_time"]
    x0, v0, h0, A0 = st["x"].copy(), st["vx"].copy(), st["h"].copy(), st["A"].copy()

    def rates(x, v, h, A):
        launched, _ = _set(g, b, dict(st, x=x, vx=v, h=h, A=A, rho=rho_ice * h, dt=dt, current_time=t))
        assert launched == CONTINUED
        return g.single_step(t)

    for _ in range(10):
        r = rates(x0, v0, h0, A0)
        x1, v1 = x0 + r["dxdt"] * dt / 2, v0 + r["dvxdt"] * dt / 2
        h1, A1 = h0 + r["dhdt"] * dt / 2, np.minimum(A0 + r["dAdt"] * dt / 2, 1.0)
        r = rates(x1, v1, h1, A1)
        x12, v12 = x0 + r["dxdt"] * dt / 2, v0 + r["dvxdt"] * dt / 2
        h12, A12 = h0 + r["dhdt"] * dt / 2, A0 + r["dAdt"] * dt / 2
        x0, v0, h0, A0 = 2 * x12 - x0, 2 * v12 - v0, 2 * h12 - h0, np.minimum(2 * A12 - A0, 1.0)
        t += dt
    ref = Simp.from_basin(b)
    ref.time_integration(10)
    a = ref.get_state()
    assert a["current_time"] == pytest.approx(t, rel=1e-14)
    for k, c in (("x", x0), ("vx", v0), ("h", h0), ("A", A0)):
        base = b.x if k == "x" else 0.0
        assert rel_l2(c - base, a[k] - base) < 1e-8, (k, rel_l2(c - base, a[k] - base))
    g.close()
    ref.close()
