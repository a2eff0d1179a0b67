"""simp_gpu_step without outputs: enqueued, not waited for.

The per-step pattern of a host that uploads, steps and reads back
(set_state, step, get_state) needs no wait between the step and the read:
the step's status comes back with the state.  The same bits and the same
time and dt as the waiting form; an error of the enqueued step surfaces at
the next get_state, or at the next step before it runs; a new state drops it.
"""
import numpy as np
import pytest

from helpers import smooth_velocity
from simp_b200 import basins
from simp_b200.simp import SIMP_ERR_IND_INT, Simp, SimpError

pytestmark = pytest.mark.gpu


def _basin():
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=12)
    return b


@pytest.mark.parametrize("switches", [{}, {"mass_from_area": 1}, {"sle": 2}, {"sle": 1, "int_algorithm": 1}])
def test_enqueued_steps_same_bits_as_waited(gpu_lib, switches):
    """With fixed hsml and mass, get_state reads those two fields while the
    step runs, from after its re-sort (every 16 steps); with either evolving
    it reads them after the step."""
    b = _basin()
    prm = b.params.copy()
    for k, v in switches.items():
        setattr(prm, k, v)
    a, e = Simp.from_basin(b, prm), Simp.from_basin(b, prm)
    for _ in range(20):                      # (a re-sort comes at step 16)
        t, dt = a.time_integration(1)
        e.step_enqueue(1)
        sa, se = a.get_state(), e.get_state()
        assert se["current_time"] == t and se["dt"] == dt
    for k in ("x", "vx", "rho", "h", "A", "hsml", "mass"):
        assert np.array_equal(sa[k], se[k]), k
    a.close()
    e.close()


def test_upload_step_download_loop(gpu_lib):
    """The end-to-end pattern: the state handed back each step continues the
    resident basin, bitwise as the resident run."""
    b = _basin()
    ref = Simp.from_basin(b)
    ref.time_integration(12)
    want = ref.get_state()
    g = Simp.from_basin(b)
    s = g.get_state()
    for _ in range(12):
        g.set_state(s["x"], s["vx"], s["mass"], s["rho"], s["hsml"], s["A"], s["h"], b.xb, b.massb,
                    s["dt"], s["current_time"])
        g.step_enqueue(1)
        s = g.get_state()
    for k in ("x", "vx", "rho", "h", "A"):
        assert np.array_equal(s[k], want[k]), k
    assert s["current_time"] == want["current_time"]


def _crowded():
    b = basins.cfg1()
    prm = b.params.copy()
    prm.max_ind_int = 10                     # fewer than the lattice's interactions
    return b, prm


def test_enqueued_error_at_get_state(gpu_lib):
    b, prm = _crowded()
    g = Simp.from_basin(b, prm)
    g.step_enqueue(1)                        # returns at once
    with pytest.raises(SimpError) as ex:
        g.get_state()
    assert ex.value.code == SIMP_ERR_IND_INT
    g.get_state()                            # reported once


def test_enqueued_error_at_next_step(gpu_lib):
    b, prm = _crowded()
    g = Simp.from_basin(b, prm)
    g.step_enqueue(1)
    with pytest.raises(SimpError) as ex:
        g.step_enqueue(1)                    # waits for the first, reports its status
    assert ex.value.code == SIMP_ERR_IND_INT


def test_new_state_drops_enqueued_status(gpu_lib):
    b, prm = _crowded()
    g = Simp.from_basin(b, prm)
    g.step_enqueue(1)
    g.set_state(b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h, b.xb, b.massb, prm.dt, 0.0)
    s = g.get_state()
    assert np.array_equal(s["x"], b.x) and s["current_time"] == 0.0


@pytest.mark.parametrize("fields", [("x",), ("h",), ("mass", "A"), ("vx", "hsml", "rho")])
def test_get_state_some_fields(gpu_lib, fields):
    """get_state with only some outputs (the others NULL), after an enqueued
    step and after a waited one: the requested fields as a full read gives
    them, the caller's other arrays untouched."""
    from simp_b200 import _lib
    b = _basin()
    g, ref = Simp.from_basin(b), Simp.from_basin(b)
    names = ("x", "vx", "mass", "rho", "hsml", "A", "h")
    for enqueued in (True, False):
        if enqueued:
            g.step_enqueue(3)
        else:
            g.time_integration(3)
        ref.time_integration(3)
        want = ref.get_state()
        out = {k: np.full_like(want[k], -7.0) for k in names}
        ptrs = [_lib.dptr(out[k]) if k in fields else None for k in names]
        assert g.lib.simp_gpu_get_state(g.h, *ptrs, None, None) == 0
        for k in names:
            if k in fields:
                assert np.array_equal(out[k], want[k]), k
            else:
                assert np.all(out[k] == -7.0), k
