"""Served request stream: the Python face of include/simp_serve.h, the
seeded request sampler of the served workload, and the serial plain-FP64
path it is compared with.

The reference has no serving layer (one basin per process, simp.f90); the
scheduler itself (admission by a device-memory budget, continuous batching,
FP64 spot-check replicas) is native code in csrc/serve.cu.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _lib, basins
from .params import (PREC_FP64, PREC_MIXED, RequestStats, ServerConfig,
                     ServerStats, SimpForcing)
from .simp import SIMP_OK, Simp, SimpError


@dataclass
class Request:
    basin: basins.Basin
    nsteps: int
    arrival_s: float


def sample_stream(count: int, seed: int = 5, rate_hz: float = 20.0, n_lo: int = 1024,
                  n_hi: int = 1048576, steps_lo: int = 100, steps_hi: int = 2000,
                  steps_scale: float = 1.0, precision: int = PREC_MIXED) -> list[Request]:
    """Poisson arrivals at ``rate_hz``; particle counts log-uniform in
    [n_lo, n_hi] (square lattices, dx = 1 km); step counts uniform in
    [steps_lo, steps_hi] times ``steps_scale``; per-request wind, thickness
    and concentration as in the batched ensemble (basins.instance)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, size=count)
    arrivals = np.cumsum(gaps) - gaps[0]
    sizes = np.exp(rng.uniform(math.log(n_lo), math.log(n_hi), size=count))
    steps = rng.integers(steps_lo, steps_hi + 1, size=count)
    out = []
    for k in range(count):
        b = basins.instance(k, int(sizes[k]), precision=precision, seed_base=seed * 100000)
        out.append(Request(b, max(1, int(round(steps[k] * steps_scale))), float(arrivals[k])))
    return out


class Server:
    """Continuous-batching server over one batch context (include/simp_serve.h)."""

    def __init__(self, params, hbm_budget_bytes: float, max_instances: int = 256,
                 max_request_particles: int = 1048576, quantum_steps: int = 16, spot_every: int = 0):
        self.lib = _lib.load()
        self.params = params.copy()
        self.cfg = ServerConfig(float(hbm_budget_bytes), int(max_instances), int(max_request_particles),
                                int(quantum_steps), int(spot_every))
        h = ctypes.c_void_p()
        rc = self.lib.simp_server_create(ctypes.byref(self.params), ctypes.byref(self.cfg), ctypes.byref(h))
        self.h = h.value
        if rc != SIMP_OK:
            msg = self.lib.simp_server_last_error(self.h).decode() if self.h else "server create failed"
            self.close()
            raise SimpError(rc, msg)
        self._keep = []          # arrays that must outlive their request
        self.outputs = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.simp_server_destroy(self.h)
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

    def _chk(self, rc):
        if rc != SIMP_OK:
            raise SimpError(rc, self.lib.simp_server_last_error(self.h).decode())

    def submit(self, req: Request, forcing: SimpForcing | None = None) -> int:
        b = req.basin
        n, nb = b.n, b.nb
        f = SimpForcing.of(b.params) if forcing is None else forcing
        ins = [np.ascontiguousarray(a, dtype=np.float64) for a in
               (b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h,
                b.xb if nb else np.zeros((1, 2)), b.massb if nb else np.zeros(1))]
        outs = {"x": np.zeros((n, 2)), "vx": np.zeros((n, 2)), "h": np.zeros(n), "A": np.zeros(n)}
        rid = ctypes.c_int64()
        P = _lib.dptr
        self._chk(self.lib.simp_server_submit(self.h, ctypes.byref(f), n, *[P(a) for a in ins[:7]], nb,
                                              P(ins[7]), P(ins[8]), int(req.nsteps), float(req.arrival_s),
                                              P(outs["x"]), P(outs["vx"]), P(outs["h"]), P(outs["A"]),
                                              ctypes.byref(rid)))
        self._keep.append((f, ins))
        self.outputs[rid.value] = outs
        return rid.value

    def run(self):
        self._chk(self.lib.simp_server_run(self.h))

    def cancel(self, rid: int, at_s: float = -1.0):
        """Cancels request rid at the first scheduling decision at or after
        at_s seconds into the run (at_s < 0: the next one); callable from
        another thread while run() is in progress."""
        self._chk(self.lib.simp_server_cancel(self.h, int(rid), float(at_s)))

    def request(self, rid: int) -> dict:
        st = RequestStats()
        self._chk(self.lib.simp_server_request(self.h, int(rid), ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in RequestStats._fields_ if f != "reserved0"}

    def stats(self) -> dict:
        st = ServerStats()
        self._chk(self.lib.simp_server_stats_get(self.h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_ if f != "reserved0"}


def serial_fp64(requests: list[Request], honor_arrivals: bool = True) -> dict:
    """The same requests one at a time through the plain FP64 single-basin
    path (one context sized for the largest request, set_state, nsteps
    steps, get_state), first come first served."""
    maxn = max(r.basin.n for r in requests)
    maxnb = max(max(r.basin.nb for r in requests), 1)
    order = sorted(range(len(requests)), key=lambda k: requests[k].arrival_s)
    prm0 = requests[0].basin.params.copy()
    prm0.precision = PREC_FP64
    sim = Simp(prm0, maxn, maxnb)
    lat, done, ps = [], [], 0
    t0 = time.perf_counter()
    try:
        for k in order:
            r = requests[k]
            if honor_arrivals:
                wait = r.arrival_s - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
            b = r.basin
            prm = b.params.copy()
            prm.precision = PREC_FP64
            sim.set_forcing(SimpForcing.of(prm))
            sim.set_state(b.x, b.vx, b.mass, b.rho, b.hsml, b.A, b.h, b.xb, b.massb, prm.dt, 0.0)
            sim.time_integration(r.nsteps)
            sim.get_state()
            t = time.perf_counter() - t0
            lat.append(t - r.arrival_s)
            done.append(t)
            ps += b.n * r.nsteps
    finally:
        sim.close()
    makespan = max(done)
    return {"particle_steps": ps, "makespan_s": makespan, "value": ps / makespan,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99))}
