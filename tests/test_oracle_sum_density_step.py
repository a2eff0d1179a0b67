"""Summation density inside the step (den_alg = 1): the oracle's kept
kernel_zero against a numpy restatement, and the GPU's p_i rule against the
oracle's pair order.

The reference keeps kernel_zero per particle (0 from initialize.f90:60) and
sets it in each right-hand side's pair loop for the p_i of every pair, to
W(0) at the pair's hsml (kernel.f90:503); sum_density then adds
kernel_zero(i) m_i to both sums (density.f90:78-79).  A particle that is
p_i of no pair keeps an earlier value (0 at the start).  The gather-form
GPU pass finds which particle of a pair the search makes p_i, and which of
several pairs comes last in the serial pair order, from the particles'
indices and reference buckets alone; the second test checks that rule on
the oracle's own pair lists.
"""
import numpy as np
import pytest

from helpers import rel_l2
from simp_b200 import basins


def _basin(jitter=0.0, hspread=0.0, seed=3, n=400):
    b = basins.cfg1() if n is None else basins.instance(0, n)
    rng = np.random.default_rng(seed)
    b.x = b.x + jitter * b.dx * rng.uniform(-1.0, 1.0, b.x.shape)
    b.hsml = b.hsml * (1.0 + hspread * rng.uniform(-1.0, 1.0, b.n))
    b.h = b.h * np.linspace(0.9, 1.1, b.n)
    b.rho = b.h * 900.0
    return b


def _ref_bin(v, bs):
    q = v / bs
    return (np.sign(q) * np.floor(np.abs(q) + 0.5)).astype(np.int64)


def _restated_sum_density(oracle_mod, b, prm, res):
    """density.f90:41-100 with kernel_zero set per pair for p_i."""
    n = b.n
    k0 = np.zeros(n)
    num = np.zeros(n)
    den = np.zeros(n)
    w = np.zeros(res["nip"])
    for k in range(res["nip"]):
        i, j = res["p_i"][k] - 1, res["p_j"][k] - 1
        dx, dy = b.x[i] - b.x[j]
        w[k], _, _, z = oracle_mod.kernel(prm, res["r_ij"][k], res["hsml_ij"][k], dx, dy)
        k0[i] = z
    num[:] = k0 * b.mass
    den[:] = k0 * b.mass / b.rho
    for k in range(res["nip"]):
        i, j = res["p_i"][k] - 1, res["p_j"][k] - 1
        den[i] += b.mass[j] * w[k] / b.rho[j]
        den[j] += b.mass[i] * w[k] / b.rho[i]
        num[i] += b.mass[j] * w[k]
        num[j] += b.mass[i] * w[k]
    return num / den, k0


@pytest.mark.parametrize("nnps", [1, 2])
def test_kept_kernel_zero_restated(oracle_mod, nnps):
    b = _basin(jitter=0.3, hspread=0.2)
    prm = b.params.copy()
    prm.den_alg = 1
    prm.nnps_algorithm = nnps
    o = oracle_mod.Oracle.from_basin(b, prm)
    got = o.sum_density(k0_mode=0)
    res = o.nnps()
    want, k0 = _restated_sum_density(oracle_mod, b, prm, res)
    assert rel_l2(got, want) < 1e-14
    # some particles are p_i of no pair: no self term, unlike W(0) at their hsml
    never = k0 == 0.0
    assert never.any() and not never.all()
    own = o.sum_density(k0_mode=1)
    assert np.all(np.abs(got[never] - own[never]) > 1e-6 * own[never])


@pytest.mark.parametrize("nnps", [1, 2])
@pytest.mark.parametrize("hspread", [0.0, 0.2])
def test_p_i_rule_matches_the_serial_pair_order(oracle_mod, nnps, hspread):
    """The rule of the GPU pass: direct search, p_i is the lower index; bucket
    search, the lower index within a bucket, else the particle whose bucket
    has the other's right, up, up-right or up-left of it, emitted in that
    order after the bucket's own pairs, each bucket in index order.  The
    largest (category, index) key picks the serial order's last pair."""
    b = _basin(jitter=0.45, hspread=hspread, seed=5, n=900)
    prm = b.params.copy()
    prm.nnps_algorithm = nnps
    o = oracle_mod.Oracle.from_basin(b, prm)
    res = o.nnps()
    pi, pj = res["p_i"] - 1, res["p_j"] - 1
    last_serial = np.full(b.n, -1)
    for k in range(res["nip"]):
        last_serial[pi[k]] = pj[k]
    bs = 2.0 * b.hsml.min()
    bx, by = _ref_bin(b.x[:, 0], bs), _ref_bin(b.x[:, 1], bs)
    best = np.full(b.n, -1, np.int64)
    best_j = np.full(b.n, -1)
    cats = {(1, 0): 1, (0, 1): 2, (1, 1): 3, (-1, 1): 4}
    for i, j in zip(np.concatenate([pi, pj]), np.concatenate([pj, pi])):   # every (i, j) of the gather form
        if nnps == 1:
            cat = 0 if j > i else -1
        else:
            d = (int(bx[j] - bx[i]), int(by[j] - by[i]))
            cat = (0 if j > i else -1) if d == (0, 0) else cats.get(d, -1)
        if cat < 0:
            continue
        key = (cat << 32) | int(j)
        if key > best[i]:
            best[i], best_j[i] = key, j
    assert np.array_equal(best_j, last_serial)
    assert (last_serial < 0).any()
