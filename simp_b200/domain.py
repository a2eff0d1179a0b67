"""Map-driven domains: particles, wall particles and wall normals generated
from an ice/land map, as the reference's initialisation does
(in_out/initialize.f90:102-228 particle_placing, in_out/boundaries.f90:164-312
boundary_placing_1, :607-772 boundary_normal).

The reference reads its maps from modules that are not part of the project
(`domain`, `boundary_domain`); here they are arguments.  Their coordinates
and resolutions are taken as double precision.  The reference's default-real
literals (1./2.) make the in-cell offsets single-precision expressions; they
are evaluated in float32 here as gfortran evaluates them.

Host code: initialisation runs once per basin and is not on the step path.
"""
from __future__ import annotations

import numpy as np

from .basins import RHO_ICE, Basin
from .params import SimpParams

f32 = np.float32


class DomainError(ValueError):
    pass


def particle_placing(ice_map, map_resolution: float, resolution: float, x_mingeom: float,
                     y_maxgeom: float, hsml_multiplicity: int = 3, maxn: int | None = None) -> dict:
    """Particles of every ice cell (map(m, n) == 1; m along x, n along y
    from the top): res_ratio^2 particles per cell on a regular sub-lattice
    (initialize.f90:141-185), at rest, h = A = 1, rho = rho_ice h,
    mass = rho (hsml / hsml_multiplicity)^2, hsml = hsml_multiplicity *
    map_resolution / res_ratio (:188-197)."""
    ice_map = np.asarray(ice_map)
    x_numcell, y_numcell = ice_map.shape
    res_ratio = int(np.floor(map_resolution / resolution + 0.5))   # NINT of a positive ratio
    nppg = res_ratio ** 2
    if nppg == 0:
        raise DomainError("Resolution desired too coarse by comparison to the domain map resolution.")
    ntotal = int(np.count_nonzero(ice_map == 1)) * nppg
    if maxn is not None and ntotal > maxn:
        raise DomainError("Resolution desired too high, the number of particles generated is higher "
                          "than the maximum allowed.")
    xs, ys = [], []
    kk, ll = np.meshgrid(np.arange(res_ratio), np.arange(res_ratio), indexing="ij")
    kk, ll = kk.ravel(), ll.ravel()                              # k outer, l inner (:166-176)
    for n in range(y_numcell):
        for m in range(x_numcell):
            if ice_map[m, n] != 1:
                continue
            ox = (f32(-0.5) + f32(m)) + (kk.astype(f32) + f32(0.5)) / f32(res_ratio)
            oy = (f32(0.5) - f32(n)) - (ll.astype(f32) + f32(0.5)) / f32(res_ratio)
            xs.append(x_mingeom + ox.astype(np.float64) * map_resolution)
            ys.append(y_maxgeom + oy.astype(np.float64) * map_resolution)
    x = np.stack([np.concatenate(xs), np.concatenate(ys)], axis=1) if xs else np.zeros((0, 2))
    hsml = np.full(ntotal, hsml_multiplicity * map_resolution / res_ratio)
    h = np.ones(ntotal)
    A = np.ones(ntotal)
    rho = RHO_ICE * h
    mass = rho * (hsml / hsml_multiplicity) ** 2
    return {"x": np.ascontiguousarray(x), "vx": np.zeros((ntotal, 2)), "hsml": hsml, "h": h, "A": A,
            "rho": rho, "mass": mass, "max_hsml": 10.0 * float(hsml.max()) if ntotal else 0.0}


def boundary_placing_1(bmap, bmap_resolution: float, b_length: float, bx_mingeom: float,
                       by_maxgeom: float, map_factor: float = 1.0, maxnb: int | None = None):
    """One line of wall particles, b_length / 3 apart, on every edge between
    a land cell (bmap == 0) and an ice cell (bmap == 1), with the unit
    normal pointing into the ice (boundaries.f90:196-297).  Land cells are
    taken with the first map index fastest."""
    bmap = np.asarray(bmap)
    bx_numcell, by_numcell = bmap.shape
    bppg = int(np.floor(bmap_resolution / (b_length / 3) + 0.5))
    if bppg == 0:
        raise DomainError("Boundary map resolution too high by comparison to the boundary particle resolution.")
    half = f32(0.5) * f32(map_factor)
    xb, nrm = [], []
    for m in range(1, by_numcell + 1):
        for n in range(1, bx_numcell + 1):
            if bmap[n - 1, m - 1] != 0:
                continue
            for k in range(bppg):
                t = (f32(k) + f32(0.5)) / f32(bppg)
                if n + 1 <= bx_numcell and bmap[n, m - 1] == 1:             # :206-221
                    xb.append((bx_mingeom + float(f32(n) - half) * bmap_resolution,
                               by_maxgeom + float(f32(-m + 1) + half - t) * bmap_resolution))
                    nrm.append((1.0, 0.0))
            for k in range(bppg):
                t = (f32(k) + f32(0.5)) / f32(bppg)
                if n - 1 >= 1 and bmap[n - 2, m - 1] == 1:                  # :224-239
                    xb.append((bx_mingeom + float(f32(n - 1) - half) * bmap_resolution,
                               by_maxgeom + float(f32(-m + 1) + half - t) * bmap_resolution))
                    nrm.append((-1.0, 0.0))
            for k in range(bppg):
                t = (f32(k) + f32(0.5)) / f32(bppg)
                if m + 1 <= by_numcell and bmap[n - 1, m] == 1:             # :242-257
                    xb.append((bx_mingeom + float(f32(n - 1) - half + t) * bmap_resolution,
                               by_maxgeom + float(f32(-m) + half) * bmap_resolution))
                    nrm.append((0.0, -1.0))
            for k in range(bppg):
                t = (f32(k) + f32(0.5)) / f32(bppg)
                if m - 1 >= 1 and bmap[n - 1, m - 2] == 1:                  # :260-275
                    xb.append((bx_mingeom + float(f32(n - 1) - half + t) * bmap_resolution,
                               by_maxgeom + float(f32(-m + 1) + half) * bmap_resolution))
                    nrm.append((0.0, 1.0))
    xb = np.ascontiguousarray(np.array(xb, dtype=np.float64).reshape(-1, 2))
    nrm = np.ascontiguousarray(np.array(nrm, dtype=np.float64).reshape(-1, 2))
    if maxnb is not None and xb.shape[0] > maxnb:
        raise DomainError("The number of boundary particles generated is higher than the maximum allowed.")
    return xb, nrm


def boundary_placing_2(bmap, bmap_resolution: float, b_length: float, bx_mingeom: float, by_maxgeom: float,
                       max_hsml: float, hsml_multiplicity: int = 3, map_factor: float = 1.0,
                       maxnb: int | None = None) -> np.ndarray:
    """Walls of hsml_multiplicity lines, max(hsml) / hsml_multiplicity
    apart and reaching into the land cell, on every land/ice edge, and on
    the two edges of a land cell whose only ice neighbour is diagonal
    (boundaries.f90:319-599).  No normals: the Wang force is not allowed with
    these walls (boundaries.f90:76-83).  Map cells outside the map count as
    land."""
    bmap = np.asarray(bmap)
    bx_numcell, by_numcell = bmap.shape
    bppg = int(np.floor(bmap_resolution / (b_length / 3) + 0.5))
    if bppg == 0:
        raise DomainError("Boundary map resolution too high by comparison to the boundary particle resolution.")
    spacing = max_hsml / hsml_multiplicity
    half = f32(0.5) * f32(map_factor)
    res = bmap_resolution
    out = []

    def ice(a, b):           # 1-based map indices
        return 1 <= a <= bx_numcell and 1 <= b <= by_numcell and bmap[a - 1, b - 1] == 1

    def lines(fx, fy):
        for k in range(bppg):
            t = (f32(k) + f32(0.5)) / f32(bppg)
            for l in range(hsml_multiplicity):
                out.append((fx(t, l), fy(t, l)))

    def left(n, m):          # :339-350
        lines(lambda t, l: bx_mingeom + float(f32(n) - half) * res - l * spacing,
              lambda t, l: by_maxgeom + float(f32(-m + 1) + half - t) * res)

    def right(n, m):         # :352-363
        lines(lambda t, l: bx_mingeom + float(f32(n - 1) - half) * res + l * spacing,
              lambda t, l: by_maxgeom + float(f32(-m + 1) + half - t) * res)

    def up(n, m):            # :365-376
        lines(lambda t, l: bx_mingeom + float(f32(n - 1) - half + t) * res,
              lambda t, l: by_maxgeom + float(f32(-m) + half) * res + l * spacing)

    def down(n, m):          # :378-389
        lines(lambda t, l: bx_mingeom + float(f32(n - 1) - half + t) * res,
              lambda t, l: by_maxgeom + float(f32(-m + 1) + half) * res - l * spacing)

    for m in range(1, by_numcell + 1):
        for n in range(1, bx_numcell + 1):
            if bmap[n - 1, m - 1] != 0:
                continue
            if ice(n + 1, m):
                left(n, m)
            if ice(n - 1, m):
                right(n, m)
            if ice(n, m + 1):
                up(n, m)
            if ice(n, m - 1):
                down(n, m)
            # a diagonal ice neighbour only (:391-470 and :472-583)
            if ice(n, m - 1) or ice(n, m + 1) or ice(n - 1, m) or ice(n + 1, m):
                continue
            if ice(n + 1, m - 1):
                left(n, m)
                down(n, m)
            if ice(n - 1, m + 1):
                right(n, m)
                up(n, m)
            if ice(n + 1, m + 1):
                left(n, m)
                up(n, m)
            if ice(n - 1, m - 1):
                down(n, m)
                right(n, m)
    xb = np.ascontiguousarray(np.array(out, dtype=np.float64).reshape(-1, 2))
    if maxnb is not None and xb.shape[0] > maxnb:
        raise DomainError("The number of boundary particles generated is higher than the maximum allowed.")
    return xb


def boundary_normal(xb, b_normal) -> np.ndarray:
    """Normals refitted from each wall particle and its two nearest wall
    neighbours (boundaries.f90:607-772), as the reference computes them for
    the Wang boundary force: a vertical or horizontal triple keeps an axis
    normal, otherwise the slope of a least-squares line through the three
    (in units of 100 m; two terms of its normal equations use metres, as the
    reference's do), and the sign of each component is flipped when any of
    the three had a negative component in the placed normals."""
    xb = np.asarray(xb, dtype=np.float64).reshape(-1, 2)
    nb = xb.shape[0]
    orientation = np.trunc(np.asarray(b_normal, dtype=np.float64).reshape(-1, 2)).astype(np.int64)
    xt = xb / 100
    out = np.zeros((nb, 2))
    for i in range(nb):
        d1 = d2 = 1e20
        n1 = n2 = -1
        for j in range(nb):
            if j == i:
                continue
            d = np.sqrt((xb[i, 0] - xb[j, 0]) ** 2 + (xb[i, 1] - xb[j, 1]) ** 2)
            if d < d1:
                if d1 < d2:
                    d2, n2 = d1, n1
                d1, n1 = d, j
            elif d < d2:
                d2, n2 = d, j
        if abs((xb[i, 0] + xb[n1, 0] + xb[n2, 0]) / 3.0 - xb[i, 0]) < 1e-20:
            bn = [1.0, 0.0]
        elif abs((xb[i, 1] + xb[n1, 1] + xb[n2, 1]) / 3.0 - xb[i, 1]) < 1e-20:
            bn = [0.0, 1.0]
        else:
            m11 = xt[i, 0] ** 2 + xt[n1, 0] ** 2 + xt[n2, 0] ** 2
            m12 = xt[i, 0] + xt[n1, 0] + xb[n2, 0]
            m22 = 3.0
            det = m11 * m22 - m12 * m12
            inv = np.array([[m22, -m12], [-m12, m11]]) / det
            v1 = xt[i, 1] * xt[i, 0] + xt[n1, 1] * xt[n1, 0] + xt[n2, 1] * xt[n2, 0]
            v2 = xt[i, 1] + xb[n1, 1] + xb[n2, 1]
            tang0 = inv[0, 0] * v1 + inv[0, 1] * v2
            b0 = np.sqrt(1 / (tang0 ** (-2) + 1))
            bn = [b0, abs(b0 / tang0)]
            if orientation[i, 0] == 0:
                bn = [bn[1], bn[0]]
        if np.any(orientation[[i, n1, n2], 0] < 0):
            bn[0] = -bn[0]
        if np.any(orientation[[i, n1, n2], 1] < 0):
            bn[1] = -bn[1]
        out[i] = bn
    return out


def basin_from_map(ice_map, map_resolution: float, resolution: float, x_mingeom: float, y_maxgeom: float,
                   params: SimpParams, bmap=None, bmap_resolution: float | None = None,
                   map_factor: float = 1.0, b_setup: int = 1, name: str = "map_basin") -> Basin:
    """A basin of a map domain: the particles of particle_placing and, with a
    boundary map (the ice map itself when none is given), the walls of
    boundary_placing_1 (b_setup = 1) or boundary_placing_2 (b_setup = 2)
    with massb = mean(mass) (boundaries.f90:52, 72), and the normals of
    boundary_placing_1 (refitted by boundary_normal when bfa = 2)."""
    part = particle_placing(ice_map, map_resolution, resolution, x_mingeom, y_maxgeom,
                            params.hsml_multiplicity)
    bmap = np.asarray(ice_map if bmap is None else bmap)
    bres = map_resolution if bmap_resolution is None else bmap_resolution
    if b_setup == 2:
        if params.bfa == 2:
            raise DomainError("The boundary force cannot be with bfa 2 if the boundary layer has multiple "
                              "set of particles.")
        xb = boundary_placing_2(bmap, bres, params.b_length, x_mingeom, y_maxgeom, float(part["hsml"].max()),
                                params.hsml_multiplicity, map_factor)
        nrm = np.zeros_like(xb)
    else:
        xb, nrm = boundary_placing_1(bmap, bres, params.b_length, x_mingeom, y_maxgeom, map_factor)
    if params.bfa == 2 and xb.shape[0] >= 3:
        nrm = boundary_normal(xb, nrm)
    n = part["x"].shape[0]
    massb = np.full(xb.shape[0], part["mass"].sum() / max(n, 1))
    ext = max(ice_map.shape) * map_resolution
    return Basin(name=name, dx=map_resolution / max(1, int(np.floor(map_resolution / resolution + 0.5))), L=ext,
                 x=part["x"], vx=part["vx"], mass=part["mass"], rho=part["rho"], hsml=part["hsml"],
                 A=part["A"], h=part["h"], xb=xb, massb=massb, params=params, bn=nrm,
                 meta={"map_shape": tuple(ice_map.shape), "max_hsml": part["max_hsml"]})
