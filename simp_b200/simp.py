"""Host-side mirror of SIMP's hot-path interface over the GPU library.

The reference drives its physics through argument-less subroutines on module
globals: NNPS (neighbor/nnps.f90:5), single_step (integration/single_step.f90:5),
density (phy_quantities/density.f90:5), predictor_corrector and the
time_integration loop (integration/time_integration.f90:38-71, 155-282).
``Simp`` holds those globals resident on the GPU and offers the same
operations under the same names.  Errors the reference turns into a STOP
banner raise ``SimpError`` carrying the banner text and the status code.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .params import SimpForcing, SimpParams

SIMP_OK = 0
SIMP_ERR_BADARG = 1
SIMP_ERR_MAXN = 2
SIMP_ERR_PAIR_CAP = 3
SIMP_ERR_IND_INT = 4
SIMP_ERR_CUDA = 5
SIMP_ERR_NONFINITE = 6
SIMP_ERR_TIMEOUT = 7
SIMP_ERR_NOMEM = 8
SIMP_ERR_STATE = 9
SIMP_ERR_BOUNDS = 10
SIMP_ERR_CANCELLED = 11

DIAG_NAMES = ("eps11", "eps12", "eps22", "zeta", "eta", "p", "sig11", "sig12", "sig22")


class SimpError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[SIMP error {code}] {message}")
        self.code = code
        self.message = message


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        a = a.reshape(shape)
    return a


class Simp:
    """One resident basin: ntotal particles, ntotalb wall particles."""

    def __init__(self, params: SimpParams, maxn: int, maxnb: int, lib=None):
        # lib: another build of the library (the checked debug build), else the default one
        self.lib = lib if lib is not None else _lib.load()
        self.params = params.copy()
        h = ctypes.c_void_p()
        rc = self.lib.simp_gpu_create(ctypes.byref(self.params), int(maxn), int(maxnb), ctypes.byref(h))
        self.h = h.value
        if rc != SIMP_OK:
            msg = self.lib.simp_gpu_last_error(self.h).decode() if self.h else "create failed"
            self.close()
            raise SimpError(rc, msg)
        self.maxn, self.maxnb = int(maxn), int(maxnb)
        self.ntotal = 0
        self.ntotalb = 0

    # -- lifecycle --------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.simp_gpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc: int):
        if rc != SIMP_OK:
            raise SimpError(rc, self.lib.simp_gpu_last_error(self.h).decode())

    @classmethod
    def from_basin(cls, b, params: SimpParams | None = None, maxn: int | None = None, lib=None):
        prm = b.params if params is None else params
        s = cls(prm, maxn or b.n, max(b.nb, 1), lib=lib)
        s.set_state(b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h, b.xb, b.massb, prm.dt, 0.0)
        if prm.bfa == 2 and b.nb > 0 and getattr(b, "bn", None) is not None:
            s.set_wall_normals(b.bn)
        return s

    # -- state ------------------------------------------------------------
    def set_state(self, x, vx, mass, rho, hsml, A, h, xb, massb, dt: float, current_time: float = 0.0):
        n = int(np.asarray(mass).shape[0])
        nb = int(np.asarray(massb).shape[0])
        arrs = (_f64(x, (n, 2)), _f64(vx, (n, 2)), _f64(mass), _f64(rho), _f64(hsml), _f64(A), _f64(h),
                _f64(xb, (nb, 2)) if nb else np.zeros((1, 2)), _f64(massb) if nb else np.zeros(1))
        p = [_lib.dptr(a) for a in arrs]
        self._chk(self.lib.simp_gpu_set_state(self.h, n, p[0], p[1], p[2], p[3], p[4], p[5], p[6], nb,
                                              p[7], p[8], float(dt), float(current_time)))
        self.ntotal, self.ntotalb = n, nb

    def get_state(self) -> dict:
        n = self.ntotal
        out = {"x": np.zeros((n, 2)), "vx": np.zeros((n, 2))}
        for k in ("mass", "rho", "hsml", "A", "h"):
            out[k] = np.zeros(n)
        dt, t = ctypes.c_double(), ctypes.c_double()
        self._chk(self.lib.simp_gpu_get_state(self.h, *[_lib.dptr(out[k]) for k in
                                                        ("x", "vx", "mass", "rho", "hsml", "A", "h")],
                                              ctypes.byref(dt), ctypes.byref(t)))
        out["dt"], out["current_time"] = dt.value, t.value
        return out

    def write_output(self, folder: str):
        """Appends a snapshot to the reference's output files (output.f90:61-78)."""
        self._chk(self.lib.simp_gpu_write_output(self.h, str(folder).encode()))

    def set_wall_normals(self, b_normal: np.ndarray):
        """b_normal(2, ntotalb) of the walls (Wang boundary force, bfa = 2)."""
        bn = np.ascontiguousarray(b_normal, dtype=np.float64).reshape(-1, 2)
        self._chk(self.lib.simp_gpu_set_wall_normals(self.h, bn.shape[0], _lib.dptr(bn)))

    def set_forcing(self, forcing: SimpForcing):
        """Wind of this basin (and of later set_state calls)."""
        self._chk(self.lib.simp_gpu_set_forcing(self.h, ctypes.byref(forcing)))
        for name, _ in SimpForcing._fields_:
            if name != "reserved0":
                setattr(self.params, name, getattr(forcing, name))

    def set_passes(self, impl: int, threads: int = 256, cap: int = 1024):
        """Pair-pass implementation (params.PASSES_*): 0 per-particle gathers
        with the kinematic pass's form chosen by size, 1 shared-memory tiles,
        2 gathers with a one-kernel kinematic pass, 3 with a two-kernel one."""
        self._chk(self.lib.simp_gpu_set_passes(self.h, int(impl), int(threads), int(cap)))

    def get_passes(self):
        a, b, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._chk(self.lib.simp_gpu_get_passes(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def autotune(self, reps: int = 3) -> float:
        """Picks the fastest pass implementation and tile shape for the
        current state; returns its milliseconds per right-hand side."""
        ms = ctypes.c_double()
        self._chk(self.lib.simp_gpu_autotune(self.h, int(reps), ctypes.byref(ms)))
        return ms.value

    def keep_diag(self, keep: bool = True):
        self._chk(self.lib.simp_gpu_keep_diag(self.h, 1 if keep else 0))

    def get_diag(self) -> dict:
        out = {k: np.zeros(self.ntotal) for k in DIAG_NAMES}
        self._chk(self.lib.simp_gpu_get_diag(self.h, *[_lib.dptr(out[k]) for k in DIAG_NAMES]))
        return out

    # -- reference operations ----------------------------------------------
    def nnps(self, cap: int | None = None, bcap: int | None = None) -> dict:
        """Pair lists with the reference's bucket-search semantics (nnps.f90)."""
        cap = 40 * self.ntotal if cap is None else int(cap)
        bcap = 40 * self.ntotal if bcap is None else int(bcap)
        nip, bnip = ctypes.c_int32(), ctypes.c_int32()
        pi, pj = np.zeros(max(cap, 1), np.int32), np.zeros(max(cap, 1), np.int32)
        r, hm = np.zeros(max(cap, 1)), np.zeros(max(cap, 1))
        bpi, bpj = np.zeros(max(bcap, 1), np.int32), np.zeros(max(bcap, 1), np.int32)
        br = np.zeros(max(bcap, 1))
        rc = self.lib.simp_gpu_nnps(self.h, ctypes.byref(nip), _lib.iptr(pi), _lib.iptr(pj), _lib.dptr(r),
                                    _lib.dptr(hm), cap, ctypes.byref(bnip), _lib.iptr(bpi), _lib.iptr(bpj),
                                    _lib.dptr(br), bcap)
        m, mb = min(nip.value, cap), min(bnip.value, bcap)
        res = dict(nip=nip.value, p_i=pi[:m], p_j=pj[:m], r_ij=r[:m], hsml_ij=hm[:m],
                   bnip=bnip.value, bp_i=bpi[:mb], bp_j=bpj[:mb], br_ij=br[:mb])
        self._chk(rc)
        return res

    def interaction_stats(self) -> dict:
        a, b, d = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        s = ctypes.c_int64()
        self._chk(self.lib.simp_gpu_interaction_stats(self.h, ctypes.byref(a), ctypes.byref(b),
                                                      ctypes.byref(s), ctypes.byref(d)))
        return dict(maxip=a.value, minip=b.value, sumip=s.value, noip=d.value)

    def single_step(self, current_time: float) -> dict:
        n = self.ntotal
        out = dict(dxdt=np.zeros((n, 2)), dvxdt=np.zeros((n, 2)), dhdt=np.zeros(n), dAdt=np.zeros(n))
        self._chk(self.lib.simp_gpu_single_step(self.h, float(current_time), _lib.dptr(out["dxdt"]),
                                                _lib.dptr(out["dvxdt"]), _lib.dptr(out["dhdt"]),
                                                _lib.dptr(out["dAdt"])))
        return out

    def sum_density(self) -> np.ndarray:
        out = np.zeros(self.ntotal)
        self._chk(self.lib.simp_gpu_sum_density(self.h, _lib.dptr(out)))
        return out

    def time_integration(self, nsteps: int):
        """nsteps iterations of the reference's time loop; returns (t, dt)."""
        t, dt = ctypes.c_double(), ctypes.c_double()
        self._chk(self.lib.simp_gpu_step(self.h, int(nsteps), ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    def predictor_corrector(self):
        return self.time_integration(1)

    def step_enqueue(self, nsteps: int):
        """nsteps iterations without waiting for them (simp_gpu_step without
        outputs): the next get_state returns their status with the state, the
        next time_integration, single_step or nnps waits for them first."""
        self._chk(self.lib.simp_gpu_step(self.h, int(nsteps), None, None))


class Batch:
    """A batch of resident basins stepped together (one launch per kernel per
    sub-step for the whole batch).

    Every basin keeps its own grid, forcing, current_time and re-sort
    schedule, so its trajectory is bitwise the same alone or in any mix.
    Basins join with ``add`` (returns a slot) and leave with ``remove``.
    The batch shares one parameter set with a fixed time step (tse = 0) and
    fixed smoothing lengths (sle = 0).
    """

    def __init__(self, params: SimpParams, maxn: int, maxnb: int, max_instances: int):
        self.lib = _lib.load()
        self.params = params.copy()
        h = ctypes.c_void_p()
        rc = self.lib.simp_gpu_create_batch(ctypes.byref(self.params), int(maxn), int(maxnb),
                                            int(max_instances), ctypes.byref(h))
        self.h = h.value
        if rc != SIMP_OK:
            msg = self.lib.simp_gpu_last_error(self.h).decode() if self.h else "create failed"
            self.close()
            raise SimpError(rc, msg)
        self.sizes: dict[int, int] = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.simp_gpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc: int):
        if rc != SIMP_OK:
            raise SimpError(rc, self.lib.simp_gpu_last_error(self.h).decode())

    def add(self, b, forcing: SimpForcing | None = None) -> int:
        """Admit basin ``b`` (a ``Basin``); returns its slot."""
        f = SimpForcing.of(b.params) if forcing is None else forcing
        n, nb = b.n, b.nb
        arrs = (_f64(b.x, (n, 2)), _f64(b.vx, (n, 2)), _f64(b.mass), _f64(b.rho), _f64(b.hsml),
                _f64(b.A), _f64(b.h), _f64(b.xb, (nb, 2)) if nb else np.zeros((1, 2)),
                _f64(b.massb) if nb else np.zeros(1))
        p = [_lib.dptr(a) for a in arrs]
        slot = ctypes.c_int32()
        self._chk(self.lib.simp_gpu_batch_add(self.h, ctypes.byref(f), n, *p[:7], nb, p[7], p[8],
                                              ctypes.byref(slot)))
        self.sizes[slot.value] = n
        return slot.value

    def remove(self, slot: int):
        self._chk(self.lib.simp_gpu_batch_remove(self.h, int(slot)))
        self.sizes.pop(int(slot), None)

    def get_state(self, slot: int) -> dict:
        n = self.sizes[int(slot)]
        out = {"x": np.zeros((n, 2)), "vx": np.zeros((n, 2))}
        for k in ("mass", "rho", "hsml", "A", "h"):
            out[k] = np.zeros(n)
        t = ctypes.c_double()
        self._chk(self.lib.simp_gpu_batch_get_state(self.h, int(slot), *[_lib.dptr(out[k]) for k in
                                                                        ("x", "vx", "mass", "rho", "hsml",
                                                                         "A", "h")], ctypes.byref(t)))
        out["current_time"] = t.value
        return out

    def info(self, slot: int) -> dict:
        n, fl = ctypes.c_int32(), ctypes.c_int32()
        st = ctypes.c_int64()
        self._chk(self.lib.simp_gpu_batch_info(self.h, int(slot), ctypes.byref(n), ctypes.byref(st),
                                               ctypes.byref(fl)))
        return dict(ntotal=n.value, steps=st.value, flags=fl.value)

    def step(self, nsteps: int = 1):
        """nsteps predictor-corrector steps of every basin in the batch."""
        t, dt = ctypes.c_double(), ctypes.c_double()
        self._chk(self.lib.simp_gpu_step(self.h, int(nsteps), ctypes.byref(t), ctypes.byref(dt)))

    def kernel_launches(self) -> int:
        return int(self.lib.simp_gpu_kernel_launches(self.h))


def version() -> str:
    return _lib.load().simp_gpu_version().decode()
