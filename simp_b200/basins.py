"""Seeded synthetic sea-ice basins.

The reference builds its initial state from a land/ice map
(in_out/initialize.f90:102-228: particle_placing) and places wall particles
from a boundary map (in_out/boundaries.f90:164-312: boundary_placing_1).  The
workloads here are square basins generated from a seed instead; what is kept
from the reference is the initial-state semantics:

- particles on a square lattice of spacing dx, one per lattice cell centre
  (initialize.f90:178-181), here with a seeded uniform jitter of +/-0.05 dx;
- rho = rho_ice * h (initialize.f90:196, diagnostic density),
  mass = rho * dx^2 (initialize.f90:197 with hsml / hsml_multiplicity = dx);
- SIMP support radius hsml = 2.4 dx (smoothing length 1.2 dx of a cubic
  spline with support 2h);
- wall particles on straight lines at spacing b_length / 3
  (boundaries.f90:204), massb = mean(mass) (boundaries.f90:52).

Arrays use the reference's Fortran layout: 2-vectors as (n, 2) C-contiguous
float64 arrays, which is the interleaved x(dim, n) column-major layout.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .params import (PREC_FP64, PREC_MIXED, SKF_CUBIC, SimpParams,
                     basin_params)

RHO_ICE = 900.0


@dataclass
class Basin:
    name: str
    dx: float
    L: float
    x: np.ndarray
    vx: np.ndarray
    mass: np.ndarray
    rho: np.ndarray
    hsml: np.ndarray
    A: np.ndarray
    h: np.ndarray
    xb: np.ndarray
    massb: np.ndarray
    params: SimpParams
    steps: int = 0
    meta: dict = field(default_factory=dict)
    bn: np.ndarray | None = None   # wall normals b_normal(2, nb), into the ice

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    @property
    def nb(self) -> int:
        return int(self.xb.shape[0])

    def state_bytes_fp64(self) -> int:
        return self.n * 8 * 13 + self.nb * 8 * 3


def _lattice(nside: int, dx: float, rng: np.random.Generator, jitter: float = 0.05):
    c = (np.arange(nside, dtype=np.float64) + 0.5) * dx
    X, Y = np.meshgrid(c, c, indexing="xy")
    x = np.stack([X.ravel(), Y.ravel()], axis=1)
    x += rng.uniform(-jitter, jitter, size=x.shape) * dx
    return np.ascontiguousarray(x)


def _wall_line(p0, p1, spacing):
    """Wall particles centred on segments of length ``spacing`` along p0->p1."""
    p0 = np.asarray(p0, np.float64)
    p1 = np.asarray(p1, np.float64)
    length = float(np.hypot(*(p1 - p0)))
    k = max(1, int(math.ceil(length / spacing - 1e-9)))
    t = (np.arange(k) + 0.5) / k
    return p0[None, :] + t[:, None] * (p1 - p0)[None, :]


def _walls(L: float, dx: float, b_length: float, sides: str):
    """Wall particles of the requested sides and their unit normals, which
    point into the ice as the reference's b_normal does
    (boundaries.f90:232-287)."""
    s = b_length / 3.0
    lo, hi = -0.5 * dx, L + 0.5 * dx
    segs, normals = [], []
    for side, p0, p1, nrm in (("+x", (hi, lo), (hi, hi), (-1.0, 0.0)),
                              ("-x", (lo, lo), (lo, hi), (1.0, 0.0)),
                              ("+y", (lo, hi), (hi, hi), (0.0, -1.0)),
                              ("-y", (lo, lo), (hi, lo), (0.0, 1.0))):
        if side in sides:
            w = _wall_line(p0, p1, s)
            segs.append(w)
            normals.append(np.tile(nrm, (w.shape[0], 1)))
    if not segs:
        return np.zeros((0, 2)), np.zeros((0, 2))
    return (np.ascontiguousarray(np.concatenate(segs, axis=0)),
            np.ascontiguousarray(np.concatenate(normals, axis=0)))


def make_basin(nside: int, dx: float, seed: int, *, name: str = "basin",
               walls: str = "+x", wind=(10.0, 0.0), vortex=None,
               h=None, A=None, precision: int = PREC_FP64,
               skf: int = SKF_CUBIC, dt: float = 1.0, steps: int = 0,
               jitter: float = 0.05) -> Basin:
    rng = np.random.default_rng(seed)
    L = nside * dx
    x = _lattice(nside, dx, rng, jitter)
    n = x.shape[0]
    hh = np.ones(n) if h is None else np.broadcast_to(np.asarray(h, np.float64), (n,)).copy()
    AA = np.ones(n) if A is None else np.broadcast_to(np.asarray(A, np.float64), (n,)).copy()
    rho = RHO_ICE * hh
    mass = rho * dx * dx
    hsml = np.full(n, 2.4 * dx)
    prm = basin_params(dx, skf=skf, dt=dt, wind=wind, precision=precision, vortex=vortex)
    xb, bn = _walls(L, dx, prm.b_length, walls)
    massb = np.full(xb.shape[0], mass.sum() / n)
    return Basin(name=name, dx=dx, L=L, x=x, vx=np.zeros((n, 2)), mass=mass,
                 rho=rho, hsml=hsml, A=AA, h=hh, xb=xb, massb=massb, bn=bn,
                 params=prm, steps=steps, meta={"seed": seed, "nside": nside})


def smooth_velocity(x: np.ndarray, L: float, amp: float = 0.3, seed: int = 0) -> np.ndarray:
    """A smooth, non-trivial velocity field (shear + divergence + rotation)
    for exercising the rheology from a state not at rest."""
    rng = np.random.default_rng(seed)
    k = 2.0 * np.pi / L
    p = rng.uniform(0, 2 * np.pi, size=4)
    u = amp * (np.sin(k * x[:, 0] + p[0]) * np.cos(2 * k * x[:, 1] + p[1]) + 0.3)
    v = amp * (np.cos(3 * k * x[:, 0] + p[2]) * np.sin(k * x[:, 1] + p[3]) - 0.2)
    return np.ascontiguousarray(np.stack([u, v], axis=1))


def _gauss_smooth(field2d: np.ndarray, sigma_cells: float) -> np.ndarray:
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(field2d, sigma=sigma_cells, mode="nearest")


# --- the five workloads ----------------------------------------------------

def cfg1(seed: int = 1) -> Basin:
    """2,500 particles, 50x50 lattice, dx = 2 km, wall on +x, wind 10 m/s +x,
    cubic spline, fixed dt = 1 s, 200 steps, FP64."""
    return make_basin(50, 2000.0, seed, name="cfg1_2500", walls="+x",
                      wind=(10.0, 0.0), steps=200)


def cfg2(seed: int = 2) -> Basin:
    """262,144 particles, 512x512 lattice, dx = 500 m in a 256 km basin,
    same physics as cfg1, 1,000 steps, FP64."""
    return make_basin(512, 500.0, seed, name="cfg2_262144", walls="+x",
                      wind=(10.0, 0.0), steps=1000)


# The reference's viscous-plastic time-step bound (time_step.f90:155):
# dt <= rho_ice hsml^2 delta_min / (P_star (1 + k_t)), with hsml = 2.4 dx.
# Above it the explicit scheme amplifies any rounding difference (a
# reordered FP64 sum included) by a factor per step; below it mixed and FP64
# trajectories stay close for thousands of steps.
def vp_dt_bound(dx: float) -> float:
    return RHO_ICE * (2.4 * dx) ** 2 * 2.0e-9 / 2.75e4


def cfg3(seed: int = 3, nside: int = 1024, dt: float = 1.0e-5) -> Basin:
    """1,048,576 particles (1024x1024, dx = 250 m, 256 km), walls on four
    sides, cyclonic vortex wind of peak 15 m/s and radius 25 km centred in the
    middle 50% of the domain, h ~ U(0.5, 2), A ~ U(0.8, 1) smoothed with a
    5 km Gaussian, 2,000 steps, mixed precision.  dt = 1e-5 s, under the VP
    bound (2.4e-5 s at dx = 250 m, halved for h up to 2)."""
    dx = 256000.0 / nside
    rng = np.random.default_rng(seed + 1000)
    L = nside * dx
    cx, cy = rng.uniform(0.25, 0.75, size=2) * L
    h = rng.uniform(0.5, 2.0, size=(nside, nside))
    A = rng.uniform(0.8, 1.0, size=(nside, nside))
    sig = 5000.0 / dx
    h = _gauss_smooth(h, sig).ravel()
    A = np.minimum(_gauss_smooth(A, sig).ravel(), 1.0)
    return make_basin(nside, dx, seed, name=f"cfg3_{nside * nside}", walls="+x-x+y-y",
                      vortex=(cx, cy, 15.0, 25000.0), h=h, A=A,
                      precision=PREC_MIXED, steps=2000, dt=dt)


def instance(k: int, n_target: int, dx: float = 1000.0, steps: int = 500,
             precision: int = PREC_MIXED, seed_base: int = 4, dt: float = 1.0e-4) -> Basin:
    """One basin of a batched ensemble or a served request: square lattice of
    about n_target particles, dx = 1 km, walls on four sides, uniform wind of
    speed U(5, 20) m/s and direction U(0, 2 pi), h ~ U(0.5, 2) m and
    A ~ U(0.8, 1) drawn per instance.  dt = 1e-4 s, under the VP bound
    (3.8e-4 s at dx = 1 km, halved for h up to 2)."""
    rng = np.random.default_rng(seed_base + k)
    nside = max(2, int(round(math.sqrt(n_target))))
    speed = rng.uniform(5.0, 20.0)
    ang = rng.uniform(0.0, 2.0 * math.pi)
    hv = rng.uniform(0.5, 2.0)
    Av = rng.uniform(0.8, 1.0)
    return make_basin(nside, dx, int(rng.integers(1 << 31)), name=f"inst{k}",
                      walls="+x-x+y-y", wind=(speed * math.cos(ang), speed * math.sin(ang)),
                      h=hv, A=Av, precision=precision, steps=steps, dt=dt)


def cfg4_sizes(count: int = 64, seed: int = 4, lo: int = 4096, hi: int = 262144):
    """Particle counts log-uniform in [lo, hi], snapped to square lattices."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count))
    sides = np.maximum(2, np.round(np.sqrt(n))).astype(int)
    return [int(s * s) for s in sides]


def cfg4(count: int = 64, seed: int = 4, steps: int = 500):
    return [instance(k, n, steps=steps, seed_base=seed) for k, n in
            enumerate(cfg4_sizes(count, seed))]
