"""The checked debug build (libsimp_gpu_checked.so, SIMP_CHECK_BOUNDS):
device index checks on every neighbour index, stencil cell, sort slot and
shared-memory slot, which set a flag and skip the access instead of
trapping; an entry point whose kernels tripped one returns SIMP_ERR_BOUNDS.
On correct inputs nothing trips: every call returns 0, and since the checks
do not touch the arithmetic the results are bitwise those of the default
build.  (The reference has only its capacity STOPs, nnps.f90:415-423; this
build is the index-level counterpart the GPU pool allows without a
sanitizer.)
"""
import numpy as np
import pytest

from helpers import smooth_velocity
from simp_b200 import _lib, basins, build
from simp_b200.params import PASSES_TILED, PREC_MIXED
from simp_b200.simp import Simp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def checked_lib(gpu_lib):
    build.build(variant="checked")
    return _lib.load(build.LIB_CHECKED)


def _run(b, prm, lib, tiled=False):
    g = Simp.from_basin(b, prm, lib=lib)
    if tiled:
        g.set_passes(PASSES_TILED, 128, 1024)
    out = {"pairs": g.nnps(), "rhs": g.single_step(3600.0), "rho": g.sum_density()}
    g.time_integration(20)
    out["state"] = g.get_state()
    g.close()
    return out


@pytest.mark.parametrize("form", ["fp64", "mixed", "tiled"])
def test_checked_build_runs_clean_and_bitwise(gpu_lib, checked_lib, form):
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=2.0, seed=60)   # fast enough to rebuild lists and re-sort
    prm = b.params.copy()
    prm.dt = 5.0
    if form == "mixed":
        prm.precision = PREC_MIXED
    got = _run(b, prm, checked_lib, tiled=form == "tiled")    # (raises SimpError on a tripped check)
    want = _run(b, prm, None, tiled=form == "tiled")
    assert got["pairs"]["nip"] == want["pairs"]["nip"]
    for k in ("dxdt", "dvxdt", "dhdt", "dAdt"):
        assert np.array_equal(got["rhs"][k], want["rhs"][k]), k
    assert np.array_equal(got["rho"], want["rho"])
    for k in ("x", "vx", "h", "A", "rho"):
        assert np.array_equal(got["state"][k], want["state"][k]), k
