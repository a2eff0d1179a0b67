"""Empty, null and over-capacity inputs at the C ABI: each is refused with its
code before anything is uploaded, and the context stays usable.

The reference's own checks are the capacity STOPs (initialize.f90:156-163
for particles, boundaries.f90:296-303 for wall particles), mirrored as
SIMP_ERR_MAXN; a basin with no particles, or a missing array, is
SIMP_ERR_BADARG.
"""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2
from simp_b200 import _lib, basins
from simp_b200.params import SimpForcing
from simp_b200.simp import SIMP_ERR_BADARG, SIMP_ERR_MAXN, Batch, Simp

pytestmark = pytest.mark.gpu

P = _lib.dptr


def _arrays(b):
    x = np.ascontiguousarray(b.x, np.float64)
    vx = np.ascontiguousarray(b.vx, np.float64)
    rest = [np.ascontiguousarray(a, np.float64) for a in (b.mass, b.rho, b.hsml, b.A, b.h)]
    xb = np.ascontiguousarray(b.xb, np.float64)
    mb = np.ascontiguousarray(b.massb, np.float64)
    return x, vx, rest, xb, mb


def _set(g, n, ptrs, nb, wall_ptrs, dt):
    return g.lib.simp_gpu_set_state(g.h, n, *ptrs, nb, *wall_ptrs, float(dt), 0.0)


def test_set_state_refusals_leave_the_context_usable(gpu_lib):
    b = basins.cfg1()
    g = Simp(b.params, b.n, b.nb)
    x, vx, rest, xb, mb = _arrays(b)
    ptrs = [P(x), P(vx)] + [P(a) for a in rest]
    walls = [P(xb), P(mb)]
    dt = b.params.dt
    assert _set(g, 0, ptrs, b.nb, walls, dt) == SIMP_ERR_BADARG                    # no particles
    assert _set(g, -3, ptrs, b.nb, walls, dt) == SIMP_ERR_BADARG
    assert _set(g, b.n, [None] + ptrs[1:], b.nb, walls, dt) == SIMP_ERR_BADARG    # a missing array
    assert _set(g, b.n, ptrs[:6] + [None], b.nb, walls, dt) == SIMP_ERR_BADARG
    assert _set(g, b.n, ptrs, b.nb, [None, None], dt) == SIMP_ERR_BADARG          # walls named, not given
    assert _set(g, b.n, ptrs, -1, walls, dt) == SIMP_ERR_BADARG
    assert _set(g, b.n + 1, ptrs, b.nb, walls, dt) == SIMP_ERR_MAXN               # initialize.f90:156-163
    assert _set(g, b.n, ptrs, b.nb + 1, walls, dt) == SIMP_ERR_MAXN               # boundaries.f90:296-303
    # then a valid state at exactly the capacity, and steps
    assert _set(g, b.n, ptrs, b.nb, walls, dt) == 0
    g.ntotal, g.ntotalb = b.n, b.nb    # (the wrapper sizes what it reads back by these)
    g.time_integration(3)
    ref = Simp.from_basin(b)
    ref.time_integration(3)
    a, r = g.get_state(), ref.get_state()
    for k in ("x", "vx", "h"):
        assert np.array_equal(a[k], r[k]), k


def test_a_basin_without_walls(gpu_lib, oracle_mod):
    """nb = 0 with null wall arrays is a basin without walls."""
    b = basins.cfg1()
    g = Simp(b.params, b.n, 1)
    x, vx, rest, _, _ = _arrays(b)
    ptrs = [P(x), P(vx)] + [P(a) for a in rest]
    assert _set(g, b.n, ptrs, 0, [None, None], b.params.dt) == 0
    g.ntotal, g.ntotalb = b.n, 0
    g.time_integration(2)
    o = oracle_mod.Oracle(b.params, b.n, 1)
    o.set_state(b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h, np.zeros((0, 2)), np.zeros(0), b.params.dt, 0.0)
    o.step(2)
    sg, so = g.get_state(), o.get_state()
    assert rel_l2(sg["vx"], so["vx"]) < 1e-9


def test_batch_add_refusals_leave_the_batch_usable(gpu_lib):
    b = basins.instance(0, 900)
    c = basins.instance(1, 400)
    with Batch(b.params, b.n + c.n, b.nb + c.nb, 4) as bt:
        s0 = bt.add(b)
        x, vx, rest, xb, mb = _arrays(c)
        ptrs = [P(x), P(vx)] + [P(a) for a in rest]
        fc = SimpForcing.of(c.params)
        slot = ctypes.c_int32()
        add = bt.lib.simp_gpu_batch_add
        assert add(bt.h, ctypes.byref(fc), 0, *ptrs, c.nb, P(xb), P(mb), ctypes.byref(slot)) == SIMP_ERR_BADARG
        assert add(bt.h, ctypes.byref(fc), c.n, None, *ptrs[1:], c.nb, P(xb), P(mb),
                   ctypes.byref(slot)) == SIMP_ERR_BADARG
        assert add(bt.h, ctypes.byref(fc), c.n + 1, *ptrs, c.nb, P(xb), P(mb),
                   ctypes.byref(slot)) == SIMP_ERR_MAXN
        bt.step(2)
        s1 = bt.add(c)                                  # the room is still there
        bt.step(2)
        assert bt.info(s0)["steps"] == 4 and bt.info(s1)["steps"] == 2


def test_a_refused_set_state_keeps_the_resident_state(gpu_lib):
    b = basins.cfg1()
    g = Simp.from_basin(b)
    g.time_integration(2)
    before = g.get_state()
    x, vx, rest, xb, mb = _arrays(b)
    ptrs = [P(x), P(vx)] + [P(a) for a in rest]
    assert _set(g, b.n, ptrs[:2] + [None] + ptrs[3:], b.nb, [P(xb), P(mb)], 1.0) == SIMP_ERR_BADARG
    assert _set(g, b.n, ptrs, -1, [P(xb), P(mb)], 1.0) == SIMP_ERR_BADARG
    after = g.get_state()
    for k in ("x", "vx", "h", "rho"):
        assert np.array_equal(before[k], after[k]), k
    assert after["current_time"] == before["current_time"]
    g.time_integration(1)                    # and it steps on
