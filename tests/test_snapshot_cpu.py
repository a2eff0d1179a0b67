"""The reference's snapshot files written and read by the library's host code
(no GPU): the Fortran edit descriptors of output.f90:61-64 and
boundaries.f90:31, the files the reference's own plotting script reads
(python/src/data_visualization.py:37-63), and the spin-up reader.

Expected lines follow the Fortran rules for Iw and Ew.dEe output: the
mantissa 0.d1...dd rounded to d digits, the exponent with e digits, the
optional leading zero written only when the field has room (so negative
values start with "-.").
"""
import numpy as np
import pytest

from simp_b200 import _lib, snapshot
from simp_b200.simp import SIMP_ERR_BADARG, SIMP_ERR_MAXN, SimpError


@pytest.fixture(scope="module")
def lib():
    from simp_b200 import build
    build.build()
    return _lib.load()


def _state(n, seed=0):
    rng = np.random.default_rng(seed)
    st = {"x": rng.uniform(0, 2.0e5, (n, 2)), "vx": rng.normal(0, 0.3, (n, 2)),
          "mass": rng.uniform(1e9, 4e9, n), "hsml": np.full(n, 4800.0),
          "A": rng.uniform(0.8, 1.0, n), "h": rng.uniform(0.5, 2.0, n)}
    dg = {k: rng.normal(0, 1e-7, n) for k in ("eps11", "eps12", "eps22")}
    dg.update({k: rng.normal(0, 2e4, n) for k in ("p", "sig11", "sig12", "sig22")})
    return st, dg


def _lines(path):
    with open(path) as f:
        return f.read().splitlines()


def test_fortran_edit_descriptors(lib, tmp_path):
    d = str(tmp_path)
    snapshot.create_output(d)
    st = {"x": np.array([[1500.0, 2000.0], [0.0, -2.5e-4]]), "vx": np.array([[0.1, -0.2], [0.0, 0.0]]),
          "mass": np.array([123456789.0, 0.999999999]), "hsml": np.array([1e-310, 4800.0]),
          "A": np.array([1.0, 1.0]), "h": np.array([1.0, 1.0])}
    zero = np.zeros(2)
    dg = {"p": np.array([-2.5e-7, 0.0]), "eps11": zero, "eps12": zero, "eps22": zero,
          "sig11": zero, "sig12": zero, "sig22": zero}
    snapshot.output(d, 7200.0, st, dg, ntotalb=75)
    mom = _lines(tmp_path / "particle_momentum.csv")
    assert mom[0] == "       1 , 0.15000000E+001 , 0.20000000E+001 , 0.10000000E+002 , -.20000000E+002"
    assert mom[1] == "       2 , 0.00000000E+000 , -.25000000E-006 , 0.00000000E+000 , 0.00000000E+000"
    sta = _lines(tmp_path / "particle_state.csv")
    assert sta[0].startswith("       1 , 0.12345679E+009 , -.25000000E-006 , 0.10000000E-309 , "
                             "0.10000000E+001 , 0.10000000E+001 , 0.00000000E+000")
    assert sta[1].startswith("       2 , 0.10000000E+001 , 0.00000000E+000 , 0.48000000E+004")
    assert len(sta[0]) == 8 + 11 * 18
    assert _lines(tmp_path / "particle_other.csv") == ["       2 ,      75 , 0.20000000E+001"]
    snapshot.write_walls(d, np.array([[1500.0, -1500.0], [1e123, 0.0]]), np.array([2.5e9, 1.0]))
    assert _lines(tmp_path / "boundary_particles.csv") == [
        "     1 , 0.15000000E+01 , -.15000000E+01 , 0.25000000E+10",
        "     2 , 0.10000000+121 , 0.00000000E+00 , 0.10000000E+01"]


def test_reference_plotting_script_reads_the_files(lib, tmp_path):
    """data_visualization.py:37-63 loads the files with np.loadtxt(delimiter=',')
    and splits them into 5, 12 and 3 columns."""
    d = str(tmp_path)
    snapshot.create_output(d)
    st, dg = _state(300, seed=1)
    for t in (0.0, 3600.0, 7200.0):
        snapshot.output(d, t, st, dg, ntotalb=12)
    m = np.loadtxt(tmp_path / "particle_momentum.csv", delimiter=",")
    s = np.loadtxt(tmp_path / "particle_state.csv", delimiter=",")
    o = np.loadtxt(tmp_path / "particle_other.csv", delimiter=",")
    assert m.shape == (900, 5) and s.shape == (900, 12) and o.shape == (3, 3)
    assert int(np.sum(m[:, 0] == 1)) == 3                       # ntimestep, :42
    assert np.array_equal(o[:, 2], [0.0, 1.0, 2.0])
    np.testing.assert_allclose(m[:300, 1:3], st["x"] / 1000, rtol=6e-8)
    np.testing.assert_allclose(m[:300, 3:5], st["vx"] * 100, rtol=6e-8)
    np.testing.assert_allclose(s[:300, 10], dg["sig12"], rtol=6e-8)


def test_spin_up_reader_round_trip(lib, tmp_path):
    d = str(tmp_path)
    snapshot.create_output(d)
    st0, dg0 = _state(500, seed=2)
    st1, dg1 = _state(500, seed=3)
    snapshot.output(d, 3600.0, st0, dg0, ntotalb=20)
    snapshot.output(d, 5400.0, st1, dg1, ntotalb=20)
    for k, (st, t) in ((0, (st0, 3600.0)), (-1, (st1, 5400.0)), (1, (st1, 5400.0)), (-2, (st0, 3600.0))):
        r = snapshot.particle_reading(d, k)
        assert r["current_time"] == pytest.approx(t, rel=1e-12)
        assert r["ntotalb"] == 20
        for key in ("x", "vx", "mass", "hsml", "A", "h"):
            np.testing.assert_allclose(r[key], st[key], rtol=6e-8, atol=0, err_msg=key)
        np.testing.assert_array_equal(r["rho"], r["h"] * 900.0)
    xb = np.array([[-1000.0, 0.0], [-1000.0, 2666.6666666], [201000.0, 5.5e4]])
    mb = np.full(3, 3.6e9)
    snapshot.write_walls(d, xb, mb)
    w = snapshot.boundary_reading(d)
    np.testing.assert_allclose(w["xb"], xb, rtol=6e-8)
    np.testing.assert_allclose(w["massb"], mb, rtol=6e-8)


def test_reader_errors(lib, tmp_path):
    d = str(tmp_path)
    with pytest.raises(SimpError) as ex:
        snapshot.particle_reading(d)                      # no files
    assert ex.value.code == SIMP_ERR_BADARG
    snapshot.create_output(d)
    with pytest.raises(SimpError) as ex:
        snapshot.particle_reading(d)                      # no snapshot yet
    assert ex.value.code == SIMP_ERR_BADARG
    st, dg = _state(50)
    snapshot.output(d, 0.0, st, dg)
    with pytest.raises(SimpError) as ex:
        snapshot.particle_reading(d, 0, cap=49)           # initialize.f90:276-283
    assert ex.value.code == SIMP_ERR_MAXN
    with pytest.raises(SimpError) as ex:
        snapshot.particle_reading(d, 1)
    assert ex.value.code == SIMP_ERR_BADARG
    with open(tmp_path / "particle_state.csv", "a") as f:  # a torn record
        f.write("      51 , 0.1\n")
    snapshot.output(d, 1.0, st, dg)
    with pytest.raises(SimpError):
        snapshot.particle_reading(d, 1)
