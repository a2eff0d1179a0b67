"""Batched ensemble of uneven basins (one launch per kernel per sub-step for
the whole batch, per-basin grids, forcing, clocks and re-sort schedules).

- a basin's trajectory is bitwise the same alone, in a mix, after other
  basins joined or left, and as a single-basin context;
- every basin of a batch matches the FP64 oracle run on it alone;
- admission and removal bookkeeping and their error paths.
"""
import numpy as np
import pytest

from helpers import rel_l2, smooth_velocity
from simp_b200 import basins
from simp_b200.params import PREC_FP64, PREC_MIXED
from simp_b200.simp import (SIMP_ERR_BADARG, SIMP_ERR_MAXN, Batch, Simp,
                            SimpError)

pytestmark = pytest.mark.gpu

KEYS = ("x", "vx", "mass", "rho", "hsml", "A", "h")


def _inst(k, n, precision=PREC_FP64, amp=0.4):
    b = basins.instance(k, n, precision=precision)
    b.vx = smooth_velocity(b.x, b.L, amp=amp, seed=100 + k)
    return b


def _assert_bitwise(a, b, what):
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), (what, k, float(np.max(np.abs(a[k] - b[k]))))
    assert a["current_time"] == b["current_time"], what


def _batch(prm, maxn=40000, maxnb=4000, slots=8):
    return Batch(prm, maxn, maxnb, slots)


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_alone_equals_in_mix(gpu_lib, precision):
    """40 steps of basin A (re-sorted at its steps 16 and 32) alone, and with
    other basins joining before and after it and one leaving mid-run."""
    A = _inst(0, 900, precision)
    B = _inst(1, 2500, precision)
    C = _inst(2, 400, precision)
    D = _inst(3, 1600, precision)
    prm = A.params
    with _batch(prm) as alone:
        sa = alone.add(A)
        alone.step(40)
        ref = alone.get_state(sa)
        assert alone.info(sa)["steps"] == 40
    with _batch(prm) as mix:
        sb = mix.add(B)
        mix.step(5)
        sa = mix.add(A)
        mix.step(7)
        sc = mix.add(C)
        mix.step(13)
        mix.remove(sb)             # B leaves (ranges of the others shift)
        sd = mix.add(D)            # D takes the free slot below A's
        assert sd == sb
        mix.step(20)
        got = mix.get_state(sa)
        assert mix.info(sa)["steps"] == 40
        assert mix.info(sc)["steps"] == 33
    _assert_bitwise(got, ref, "alone vs mix")


def test_batch_of_one_equals_single_context(gpu_lib):
    """A batch holding one basin and the single-basin API give the same bits."""
    A = _inst(4, 1225)
    with _batch(A.params) as bt:
        s = bt.add(A)
        bt.step(25)
        gb = bt.get_state(s)
    g = Simp.from_basin(A)
    g.time_integration(25)
    gs = g.get_state()
    _assert_bitwise(gb, gs, "batch of one vs single context")


def test_batch_matches_oracle(gpu_lib, oracle_mod):
    """Three uneven basins with different winds stepped together, each
    against the FP64 oracle run alone, after 6 steps."""
    bs = [_inst(5, 625), _inst(6, 1444), _inst(7, 324)]
    with _batch(bs[0].params) as bt:
        slots = [bt.add(b) for b in bs]
        bt.step(6)
        for b, s in zip(bs, slots):
            got = bt.get_state(s)
            o = oracle_mod.Oracle.from_basin(b)
            o.step(6)
            so = o.get_state()
            for k in ("x", "vx", "h", "A", "rho"):
                e = rel_l2(got[k], so[k])
                assert e < 1e-9, (b.name, k, e)
            assert got["current_time"] == pytest.approx(6 * b.params.dt)


def test_uneven_ensemble_mixed_against_fp64(gpu_lib):
    """Twelve basins of 100 to 20,000 particles, mixed precision, 3 steps,
    each against the same basin stepped alone in FP64."""
    sizes = [100, 20000, 400, 6400, 2500, 900, 12100, 196, 3600, 8100, 1600, 625]
    bs = [_inst(10 + k, n, PREC_MIXED) for k, n in enumerate(sizes)]
    with Batch(bs[0].params, sum(b.n for b in bs), sum(b.nb for b in bs), 16) as bt:
        slots = [bt.add(b) for b in bs]
        bt.step(3)
        got = [bt.get_state(s) for s in slots]
    for b, gs in zip(bs, got):
        prm = b.params.copy()
        prm.precision = PREC_FP64
        g = Simp.from_basin(b, prm)
        g.time_integration(3)
        s64 = g.get_state()
        for k in ("vx", "h"):
            e = rel_l2(gs[k], s64[k])
            assert e < 1e-4, (b.name, k, e)


def test_admission_errors(gpu_lib):
    A = _inst(20, 900)
    B = _inst(21, 900)
    with Batch(A.params, A.n + B.n - 1, 4000, 2) as bt:
        bt.add(A)
        with pytest.raises(SimpError) as ex:
            bt.add(B)                       # particle capacity
        assert ex.value.code == SIMP_ERR_MAXN
        bt.step(2)                          # the batch is still usable
        assert bt.info(0)["steps"] == 2
    with Batch(A.params, 10 * A.n, 4000, 1) as bt:
        bt.add(A)
        with pytest.raises(SimpError) as ex:
            bt.add(B)                       # no free slot
        assert ex.value.code == SIMP_ERR_MAXN
        with pytest.raises(SimpError) as ex:
            bt.remove(3)
        assert ex.value.code == SIMP_ERR_BADARG
        bt.remove(0)
        assert bt.info(0)["ntotal"] == 0
        rc = bt.lib.simp_gpu_batch_get_state(bt.h, 0, *([None] * 8))
        assert rc == SIMP_ERR_BADARG        # the slot is free
        s = bt.add(B)                        # the slot is free again
        assert s == 0
        bt.step(1)
        assert bt.info(0)["steps"] == 1


def test_batch_rejects_adaptive_dt(gpu_lib):
    prm = _inst(22, 100).params.copy()
    prm.tse = 2
    with pytest.raises(SimpError) as ex:
        Batch(prm, 1000, 100, 4)
    assert ex.value.code == SIMP_ERR_BADARG


def test_retired_basins_compacted_later(gpu_lib):
    """A basin that leaves a batch is retired at once (its slot reads as
    free, it is neither searched nor stepped) and dropped from memory by a
    later compaction, which runs once retired basins hold a quarter of the
    batch or an admission needs their slot.  The basins that stay give the
    same bits as alone throughout."""
    A = _inst(5, 1600)
    small = [_inst(10 + k, 100) for k in range(3)]
    prm = A.params
    with _batch(prm, slots=4) as alone:
        sa = alone.add(A)
        alone.step(30)
        ref = alone.get_state(sa)
    with _batch(prm, slots=4) as mix:
        sa = mix.add(A)
        ss = [mix.add(b) for b in small]       # every slot taken
        mix.step(10)
        mix.remove(ss[0])                      # 100 of 1,900 particles: kept in place for now
        assert mix.info(ss[0])["ntotal"] == 0
        rc = mix.lib.simp_gpu_batch_get_state(mix.h, ss[0], None, None, None, None, None, None, None, None)
        assert rc == SIMP_ERR_BADARG
        mix.step(10)
        mix.remove(ss[1])
        s_new = mix.add(_inst(20, 144))        # no free slot: the retired ones are compacted first
        assert s_new in (ss[0], ss[1])
        mix.step(10)
        got = mix.get_state(sa)
        assert mix.info(sa)["steps"] == 30
        assert mix.info(ss[2])["steps"] == 30
    _assert_bitwise(got, ref, "alone vs batch with retirements and a compaction")


def test_full_ensemble_against_oracle(gpu_lib, oracle_mod):
    """The batched workload at its full size (64 basins, 4,096..262,144
    particles each, 5.2M in all, mixed precision, its own dt): after 5 steps
    the three smallest basins and a median one against the FP64 oracle run
    alone, within the mixed form's bar (measured ~1e-9 in velocity)."""
    bs = basins.cfg4(64, steps=500)
    order = np.argsort([x.n for x in bs])
    with Batch(bs[0].params, sum(x.n for x in bs), sum(x.nb for x in bs), 64) as bt:
        slots = [bt.add(x) for x in bs]
        bt.step(5)
        for k in list(order[:3]) + [order[32]]:
            got = bt.get_state(slots[k])
            prm = bs[k].params.copy()
            prm.precision = PREC_FP64
            o = oracle_mod.Oracle.from_basin(bs[k], prm)
            o.step(5)
            so = o.get_state()
            for f in ("vx", "h", "A"):
                e = rel_l2(got[f], so[f])
                assert e < 1e-4, (bs[k].name, f, e)
