"""ctypes front end of the CPU FP64 oracle (libsimp_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/, the
smoke entry point and the bench's CPU-baseline / reference legs use it.
Parity status: unpinned against the Fortran reference (no Fortran compiler
here and no reference fixtures exist); pinned to known-answer tests derived
from the mathematics (tests/golden/).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsimp_oracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "simp_oracle.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_last_error.argtypes = [ctypes.c_void_p]
        L.orc_set_state.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_dp] * 7 + [ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_double]
        L.orc_get_state.argtypes = [ctypes.c_void_p] + [_dp] * 9
        L.orc_nnps.argtypes = [ctypes.c_void_p, _ip, _ip, _ip, _dp, _dp, ctypes.c_int, _ip, _ip, _ip, _dp, ctypes.c_int]
        L.orc_single_step.argtypes = [ctypes.c_void_p, ctypes.c_double, _dp, _dp, _dp, _dp]
        L.orc_get_diag.argtypes = [ctypes.c_void_p] + [_dp] * 9
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_sum_density.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_kernel.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp]
        L.orc_boundary_w.restype = ctypes.c_double
        L.orc_boundary_w.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.orc_boundary_fdwdq.restype = ctypes.c_double
        L.orc_boundary_fdwdq.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.orc_set_wall_normals.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_set_regularization_form.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_interaction_stats.argtypes = [ctypes.c_void_p, _ip, _ip, ctypes.POINTER(ctypes.c_longlong), _ip]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _pi(a):
    return None if a is None else a.ctypes.data_as(_ip)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"oracle error {code}: {msg}")
        self.code = code


class Oracle:
    """One FP64 CPU instance of the reference's hot path."""

    def __init__(self, params, maxn: int, maxnb: int):
        self.params = params
        self.h = lib().orc_create(ctypes.byref(params), int(maxn), int(maxnb))
        self.n = 0
        self.nb = 0

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise OracleError(rc, lib().orc_last_error(self.h).decode())

    @classmethod
    def from_basin(cls, b, params=None):
        prm = b.params if params is None else params
        o = cls(prm, b.n, max(b.nb, 1))
        o.set_state(b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h, b.xb, b.massb, prm.dt, 0.0)
        if prm.bfa == 2 and b.nb > 0 and getattr(b, "bn", None) is not None:
            o.set_wall_normals(b.bn)
        return o

    def set_regularization_form(self, literal: bool):
        """Regularisation pair loops: per pair (False, the library's form) or
        the reference's serial loops literally (True)."""
        self._chk(lib().orc_set_regularization_form(self.h, 1 if literal else 0))

    def set_wall_normals(self, b_normal):
        bn = np.ascontiguousarray(b_normal, np.float64).reshape(-1, 2)
        self._keep_bn = bn
        self._chk(lib().orc_set_wall_normals(self.h, bn.shape[0], _p(bn)))

    def set_state(self, x, vx, mass, rho, hsml, A, h, xb, massb, dt, t):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (x, vx, mass, rho, hsml, A, h, xb, massb)]
        self._keep = arrs
        x, vx, mass, rho, hsml, A, h, xb, massb = arrs
        self.n = mass.shape[0]
        self.nb = massb.shape[0]
        self._chk(lib().orc_set_state(self.h, self.n, _p(x), _p(vx), _p(mass), _p(rho), _p(hsml),
                                      _p(A), _p(h), self.nb, _p(xb), _p(massb), float(dt), float(t)))

    def get_state(self):
        n = self.n
        out = {k: np.zeros((n, 2)) for k in ("x", "vx")}
        out.update({k: np.zeros(n) for k in ("mass", "rho", "hsml", "A", "h")})
        dt = ctypes.c_double()
        t = ctypes.c_double()
        self._chk(lib().orc_get_state(self.h, _p(out["x"]), _p(out["vx"]), _p(out["mass"]), _p(out["rho"]),
                                      _p(out["hsml"]), _p(out["A"]), _p(out["h"]), ctypes.byref(dt), ctypes.byref(t)))
        out["dt"] = dt.value
        out["current_time"] = t.value
        return out

    def nnps(self, cap=None, bcap=None):
        cap = cap if cap is not None else 40 * self.n + 16
        bcap = bcap if bcap is not None else 40 * self.n + 16
        nip = ctypes.c_int32()
        bnip = ctypes.c_int32()
        pi = np.zeros(cap, np.int32)
        pj = np.zeros(cap, np.int32)
        r = np.zeros(cap)
        hm = np.zeros(cap)
        bpi = np.zeros(bcap, np.int32)
        bpj = np.zeros(bcap, np.int32)
        br = np.zeros(bcap)
        rc = lib().orc_nnps(self.h, ctypes.byref(nip), _pi(pi), _pi(pj), _p(r), _p(hm), cap,
                            ctypes.byref(bnip), _pi(bpi), _pi(bpj), _p(br), bcap)
        m, mb = min(nip.value, cap), min(bnip.value, bcap)
        res = dict(nip=nip.value, p_i=pi[:m], p_j=pj[:m], r_ij=r[:m], hsml_ij=hm[:m],
                   bnip=bnip.value, bp_i=bpi[:mb], bp_j=bpj[:mb], br_ij=br[:mb], rc=rc)
        return res

    def interaction_stats(self):
        a, b, d = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        s = ctypes.c_longlong()
        lib().orc_interaction_stats(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(s), ctypes.byref(d))
        return dict(maxip=a.value, minip=b.value, sumip=s.value, noip=d.value)

    def single_step(self, current_time: float):
        n = self.n
        dxdt, dvxdt = np.zeros((n, 2)), np.zeros((n, 2))
        dhdt, dAdt = np.zeros(n), np.zeros(n)
        self._chk(lib().orc_single_step(self.h, float(current_time), _p(dxdt), _p(dvxdt), _p(dhdt), _p(dAdt)))
        return dict(dxdt=dxdt, dvxdt=dvxdt, dhdt=dhdt, dAdt=dAdt)

    def get_diag(self):
        n = self.n
        names = ("eps11", "eps12", "eps22", "zeta", "eta", "p", "sig11", "sig12", "sig22")
        out = {k: np.zeros(n) for k in names}
        self._chk(lib().orc_get_diag(self.h, *[_p(out[k]) for k in names]))
        return out

    def step(self, nsteps: int):
        t = ctypes.c_double()
        dt = ctypes.c_double()
        self._chk(lib().orc_step(self.h, int(nsteps), ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    def sum_density(self, k0_mode: int = 1):
        out = np.zeros(self.n)
        self._chk(lib().orc_sum_density(self.h, int(k0_mode), _p(out)))
        return out


def kernel(params, r, hij, dx, dy):
    w, gx, gy, k0 = (ctypes.c_double() for _ in range(4))
    lib().orc_kernel(ctypes.byref(params), float(r), float(hij), float(dx), float(dy),
                     ctypes.byref(w), ctypes.byref(gx), ctypes.byref(gy), ctypes.byref(k0))
    return w.value, gx.value, gy.value, k0.value


def boundary_w(params, br):
    return float(lib().orc_boundary_w(ctypes.byref(params), float(br)))


def boundary_fdwdq(params, br):
    """factor * dW/dq of the boundary kernel (bdwdx = -that / b_length * (bdx / br) * scale_h)."""
    return float(lib().orc_boundary_fdwdq(ctypes.byref(params), float(br)))
