"""Snapshot output of a basin on the GPU (output.f90:61-78) and a restart from
it (the spin-up reader, initialize.f90:234-330), through the C ABI."""
import numpy as np
import pytest

from helpers import rel_l2, smooth_velocity
from simp_b200 import basins, snapshot
from simp_b200.simp import Simp

pytestmark = pytest.mark.gpu

# the files keep 8 significant digits
TOL_FILE = 6e-8


def test_write_output_and_restart(gpu_lib, tmp_path):
    b = basins.cfg1()
    b.vx = smooth_velocity(b.x, b.L, amp=0.3, seed=5)
    d = str(tmp_path)
    snapshot.create_output(d)
    snapshot.write_walls(d, b.xb, b.massb)
    g = Simp.from_basin(b)
    g.keep_diag(True)
    g.time_integration(5)
    g.write_output(d)
    g.time_integration(5)
    g.write_output(d)
    st = g.get_state()
    dg = g.get_diag()
    r = snapshot.particle_reading(d, -1)
    assert r["current_time"] == pytest.approx(st["current_time"], rel=1e-8)
    assert r["ntotalb"] == b.nb
    for k in ("x", "vx", "mass", "hsml", "A", "h"):
        np.testing.assert_allclose(r[k], st[k], rtol=TOL_FILE, atol=0, err_msg=k)
    s = np.loadtxt(tmp_path / "particle_state.csv", delimiter=",")[b.n:]
    for col, k in ((2, "p"), (6, "eps11"), (8, "eps22"), (11, "sig22")):
        np.testing.assert_allclose(s[:, col], dg[k], rtol=TOL_FILE, atol=1e-300, err_msg=k)
    # restart from the file and continue next to the original
    w = snapshot.boundary_reading(d)
    g2 = Simp(b.params, b.n, b.nb)
    g2.set_state(r["x"], r["vx"], r["mass"], r["rho"], r["hsml"], r["A"], r["h"], w["xb"], w["massb"],
                 b.params.dt, r["current_time"])
    g.time_integration(5)
    g2.time_integration(5)
    a, c = g.get_state(), g2.get_state()
    for k in ("x", "vx", "h"):
        assert rel_l2(c[k], a[k]) < 1e-6, (k, rel_l2(c[k], a[k]))
