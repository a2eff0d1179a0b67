"""Map-driven domains (initialize.f90:102-228, boundaries.f90:164-312,
607-772) on the host: particle lattice, wall lines and normals, checked
against their defining geometry; and a map basin stepped by the oracle."""
import numpy as np
import pytest

from simp_b200 import domain
from simp_b200.params import basin_params


def _lshape(nx=8, ny=6):
    """Ice (1) on an L-shaped region inside a land (0) frame."""
    m = np.zeros((nx, ny), dtype=np.int32)
    m[1:nx - 1, 1:ny - 1] = 1
    m[nx // 2:nx - 1, 1:ny // 2] = 0          # a land notch
    return m


def test_particle_placing_lattice():
    m = _lshape()
    p = domain.particle_placing(m, 4000.0, 1000.0, x_mingeom=10000.0, y_maxgeom=90000.0)
    n_ice = int((m == 1).sum())
    assert p["x"].shape == (16 * n_ice, 2)                      # res_ratio 4: 16 per cell
    assert np.allclose(p["hsml"], 3 * 1000.0)                   # hsml_multiplicity * dx
    assert np.allclose(p["mass"], 900.0 * 1000.0 ** 2)
    # every particle inside an ice cell, at sub-cell centres (cell m spans
    # [m - 1/2, m + 1/2] map cells from x_mingeom; rows go down from y_maxgeom)
    cx = np.floor((p["x"][:, 0] - 10000.0) / 4000.0 + 0.5).astype(int)
    cy = np.floor((90000.0 - p["x"][:, 1]) / 4000.0 + 0.5).astype(int)
    assert np.all(m[cx, cy] == 1)
    frac = ((p["x"][:, 0] - 10000.0) / 1000.0 + 2.0) % 1.0
    assert np.allclose(frac, 0.5, atol=1e-6)
    # nearest-neighbour spacing of the lattice
    d = np.hypot(*(p["x"][1] - p["x"][0]))
    assert d == pytest.approx(1000.0, rel=1e-6)


def test_particle_placing_errors():
    with pytest.raises(domain.DomainError):
        domain.particle_placing(_lshape(), 1000.0, 4000.0, 0.0, 0.0)          # too coarse
    with pytest.raises(domain.DomainError):
        domain.particle_placing(_lshape(), 4000.0, 1000.0, 0.0, 0.0, maxn=10)


def test_wall_lines_and_normals():
    m = _lshape()
    xb, nrm = domain.boundary_placing_1(m, 4000.0, 4000.0, 10000.0, 90000.0)
    bppg = 3                                                     # 4000 / (4000 / 3)
    # one line of bppg wall particles per land/ice edge
    edges = 0
    nx, ny = m.shape
    for a in range(nx):
        for b in range(ny):
            if m[a, b] != 0:
                continue
            for da, db in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                if 0 <= a + da < nx and 0 <= b + db < ny and m[a + da, b + db] == 1:
                    edges += 1
    assert xb.shape == (bppg * edges, 2)
    # the normal points from the wall into the ice: a step of half a map cell
    # along it lands in an ice cell, a step against it in land
    for sgn, want in ((1.0, 1), (-1.0, 0)):
        q = xb + sgn * 2000.0 * nrm
        cx = np.floor((q[:, 0] - 10000.0) / 4000.0 + 0.5).astype(int)
        cy = np.floor((90000.0 - q[:, 1]) / 4000.0 + 0.5).astype(int)
        assert np.all(m[cx, cy] == want)
    assert np.allclose(np.hypot(nrm[:, 0], nrm[:, 1]), 1.0)


def test_boundary_normal_refit():
    """Straight walls keep their axis normals; at a corner the fitted normal
    is diagonal, unit length, pointing into the ice quadrant."""
    m = _lshape()
    xb, nrm = domain.boundary_placing_1(m, 4000.0, 4000.0, 10000.0, 90000.0)
    fit = domain.boundary_normal(xb, nrm)
    assert np.allclose(np.hypot(fit[:, 0], fit[:, 1]), 1.0)
    straight = np.all(fit == nrm, axis=1)
    assert straight.mean() > 0.6
    # refitted normals keep the sign of the placed ones' components
    assert np.all(fit[:, 0] * nrm[:, 0] >= 0) and np.all(fit[:, 1] * nrm[:, 1] >= 0)


def test_map_basin_steps_in_the_oracle(oracle_mod):
    prm = basin_params(1000.0, dt=1.0, wind=(8.0, 3.0))
    b = domain.basin_from_map(_lshape(), 4000.0, 1000.0, 10000.0, 90000.0, prm)
    o = oracle_mod.Oracle.from_basin(b)
    o.step(3)
    st = o.get_state()
    assert np.all(np.isfinite(st["x"])) and st["current_time"] == pytest.approx(3.0)
    assert b.nb > 0 and b.bn.shape == b.xb.shape


def test_multilayer_walls():
    """boundary_placing_2: hsml_multiplicity lines per edge, spaced
    max(hsml) / hsml_multiplicity into the land; a land cell touching ice
    only diagonally gets two edges."""
    m = np.zeros((5, 5), dtype=np.int32)
    m[1:4, 1:4] = 1
    xb1, _ = domain.boundary_placing_1(m, 4000.0, 4000.0, 0.0, 50000.0)
    xb2 = domain.boundary_placing_2(m, 4000.0, 4000.0, 0.0, 50000.0, max_hsml=3000.0, hsml_multiplicity=3)
    # straight edges: 3 layers of the single-layer wall, plus the 4 corner
    # cells (diagonal ice neighbour only): 2 edges x 3 wall particles x 3 layers each
    assert xb2.shape[0] == 3 * xb1.shape[0] + 4 * 2 * 3 * 3
    # the first layer of each edge is the single-layer wall
    first = xb2[::3]
    assert set(map(tuple, np.round(xb1, 6))) <= set(map(tuple, np.round(first, 6)))
    # successive layers step 1000 m along one axis, away from the ice
    # square's centre
    c = np.array([2.0 * 4000.0, 50000.0 - 2.0 * 4000.0])
    for a, b in ((0, 1), (1, 2)):
        step = xb2[b::3] - xb2[a::3]
        assert np.allclose(np.sort(np.abs(step), axis=1), [0.0, 1000.0])
        assert np.all(np.abs(xb2[b::3] - c).sum(axis=1) > np.abs(xb2[a::3] - c).sum(axis=1))


def test_multilayer_walls_refuse_wang_force():
    prm = basin_params(1000.0)
    prm.bfa = 2
    with pytest.raises(domain.DomainError):
        domain.basin_from_map(_lshape(), 4000.0, 1000.0, 0.0, 0.0, prm, b_setup=2)
