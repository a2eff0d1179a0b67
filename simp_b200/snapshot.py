"""The reference's snapshot files (in_out/output.f90:61-78,
boundaries.f90:52-63) written by the library, and the spin-up reader that
loads them back (initialize.f90:234-330, boundaries.f90:119-160), with the
reference's routine names.

The formatting and parsing are host code inside libsimp_gpu.so; only
``Simp.write_output`` reads the device.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .simp import SimpError

RHO_ICE = 900.0


def _chk(rc: int):
    if rc != 0:
        raise SimpError(rc, _lib.load().simp_csv_last_error().decode())


def _enc(folder: str) -> bytes:
    return str(folder).encode()


def create_output(folder: str) -> None:
    """Empty particle_momentum.csv, particle_state.csv, particle_other.csv
    (initialize.f90:83-95)."""
    _chk(_lib.load().simp_csv_create_output(_enc(folder)))


def output(folder: str, current_time: float, state: dict, diag: dict, ntotalb: int = 0) -> None:
    """Appends one snapshot from host arrays, as `output` does: state holds
    x, vx (n, 2), mass, hsml, A, h; diag holds p, eps11, eps12, eps22,
    sig11, sig12, sig22."""
    n = int(np.asarray(state["mass"]).shape[0])
    arrs = [np.ascontiguousarray(state["x"], np.float64), np.ascontiguousarray(state["vx"], np.float64)]
    arrs += [np.ascontiguousarray(state[k], np.float64) for k in ("mass",)]
    arrs += [np.ascontiguousarray(diag["p"], np.float64)]
    arrs += [np.ascontiguousarray(state[k], np.float64) for k in ("hsml", "A", "h")]
    arrs += [np.ascontiguousarray(diag[k], np.float64) for k in ("eps11", "eps12", "eps22", "sig11", "sig12", "sig22")]
    _chk(_lib.load().simp_csv_append_snapshot(_enc(folder), n, int(ntotalb), float(current_time),
                                              *[_lib.dptr(a) for a in arrs]))


def write_walls(folder: str, xb, massb) -> None:
    """boundary_particles.csv (boundaries.f90:52-63)."""
    xb = np.ascontiguousarray(xb, np.float64).reshape(-1, 2)
    massb = np.ascontiguousarray(massb, np.float64)
    _chk(_lib.load().simp_csv_write_walls(_enc(folder), xb.shape[0], _lib.dptr(xb), _lib.dptr(massb)))


def particle_reading(folder: str, snapshot: int = -1, cap: int | None = None) -> dict:
    """One snapshot of the particle files in SI units (x in m, vx in m/s,
    current_time in s), with rho = h rho_ice (the files hold no density)."""
    lib = _lib.load()
    n, nb = ctypes.c_int32(), ctypes.c_int32()
    t = ctypes.c_double()
    _chk(lib.simp_csv_read_snapshot(_enc(folder), int(snapshot), 0, ctypes.byref(n), ctypes.byref(nb),
                                    ctypes.byref(t), *([None] * 7)))
    out = {"x": np.zeros((n.value, 2)), "vx": np.zeros((n.value, 2))}
    for k in ("mass", "p", "hsml", "A", "h"):
        out[k] = np.zeros(n.value)
    cap = n.value if cap is None else int(cap)
    _chk(lib.simp_csv_read_snapshot(_enc(folder), int(snapshot), cap, ctypes.byref(n), ctypes.byref(nb),
                                    ctypes.byref(t),
                                    *[_lib.dptr(out[k]) for k in ("x", "vx", "mass", "p", "hsml", "A", "h")]))
    out["rho"] = out["h"] * RHO_ICE
    out["ntotalb"] = nb.value
    out["current_time"] = t.value
    return out


def boundary_reading(folder: str, cap: int | None = None) -> dict:
    """boundary_particles.csv in SI units."""
    lib = _lib.load()
    nb = ctypes.c_int32()
    _chk(lib.simp_csv_read_walls(_enc(folder), 0, ctypes.byref(nb), None, None))
    xb, massb = np.zeros((nb.value, 2)), np.zeros(nb.value)
    cap = nb.value if cap is None else int(cap)
    _chk(lib.simp_csv_read_walls(_enc(folder), cap, ctypes.byref(nb), _lib.dptr(xb), _lib.dptr(massb)))
    return {"xb": xb, "massb": massb}
