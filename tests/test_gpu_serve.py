"""Served request stream (include/simp_serve.h): continuous batching with
admission by a device-memory budget and FP64 spot-check replicas.

- every served result is bitwise the result of the same request stepped
  alone (a batch of one), whatever else shared the batch meanwhile;
- at the served time step (1e-4 s, under the reference's viscous-plastic
  bound) the spot-checked mixed results agree with their FP64 replicas
  within 1e-6 (above the bound any rounding difference, a reordered FP64
  sum included, is amplified every step: test_gpu_mixed);
- arrival <= admission <= completion, budget-limited admission, errors.
"""
import numpy as np
import pytest

from simp_b200 import serve
from simp_b200.params import PREC_MIXED
from simp_b200.simp import SIMP_ERR_MAXN, Batch, SimpError

pytestmark = pytest.mark.gpu

GB = 1e9


def _stream(count=8, seed=31, n_hi=20000, steps=(20, 60), rate=200.0, dt=None):
    reqs = serve.sample_stream(count, seed=seed, rate_hz=rate, n_lo=1024, n_hi=n_hi,
                               steps_lo=steps[0], steps_hi=steps[1])
    if dt is not None:
        for r in reqs:
            r.basin.params.dt = dt
    return reqs


def _alone(r):
    with Batch(r.basin.params, r.basin.n, max(r.basin.nb, 1), 1) as bt:
        s = bt.add(r.basin)
        bt.step(r.nsteps)
        return bt.get_state(s)


def test_served_equals_alone(gpu_lib):
    reqs = _stream()
    with serve.Server(reqs[0].basin.params, 2 * GB, max_instances=16, max_request_particles=20000,
                      quantum_steps=7) as srv:
        ids = [srv.submit(r) for r in reqs]
        srv.run()
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["peak_resident_requests"] > 1          # requests overlapped
        for rid, r in zip(ids, reqs):
            q = srv.request(rid)
            assert q["status"] == 0 and q["steps"] == r.nsteps
            assert q["arrival_s"] <= q["admitted_s"] <= q["completed_s"]
            ref = _alone(r)
            out = srv.outputs[rid]
            for k in ("x", "vx", "h", "A"):
                assert np.array_equal(out[k], ref[k]), (rid, k)
        assert st["particle_steps"] == sum(r.basin.n * r.nsteps for r in reqs)


def test_spot_checks(gpu_lib):
    reqs = _stream(count=6, seed=32)
    assert reqs[0].basin.params.dt == 1e-4
    with serve.Server(reqs[0].basin.params, 2 * GB, max_instances=16, max_request_particles=20000,
                      quantum_steps=16, spot_every=2) as srv:
        ids = [srv.submit(r) for r in reqs]
        srv.run()
        checked = 0
        for rid in ids:
            q = srv.request(rid)
            if q["spot_checked"]:
                checked += 1
                assert 0.0 <= q["err_v"] < 1e-6, q
                assert 0.0 <= q["err_h"] < 1e-6, q
        assert checked == 3


def test_budget_limits_residency(gpu_lib):
    """A budget that holds about one large request: requests queue for room
    and all still complete, each with the same bits as alone."""
    reqs = _stream(count=5, seed=33, n_hi=8000, steps=(5, 15))
    big = max(r.basin.n for r in reqs)
    budget = 1.2 * big * 1800.0
    with serve.Server(reqs[0].basin.params, budget, max_instances=8, max_request_particles=big,
                      quantum_steps=4) as srv:
        ids = [srv.submit(r) for r in reqs]
        srv.run()
        st = srv.stats()
        assert st["completed"] == len(reqs)
        assert st["peak_resident_particles"] <= st["capacity_particles"]
        for rid, r in zip(ids, reqs):
            assert np.array_equal(srv.outputs[rid]["vx"], _alone(r)["vx"])


def test_submit_too_large(gpu_lib):
    reqs = _stream(count=1, seed=34, n_hi=5000)
    with serve.Server(reqs[0].basin.params, 1 * GB, max_instances=4, max_request_particles=1000) as srv:
        with pytest.raises(SimpError) as ex:
            srv.submit(reqs[0])
        assert ex.value.code == SIMP_ERR_MAXN


def test_serial_fp64_baseline_runs(gpu_lib):
    reqs = _stream(count=3, seed=35, steps=(5, 10))
    r = serve.serial_fp64(reqs, honor_arrivals=False)
    assert r["particle_steps"] == sum(q.basin.n * q.nsteps for q in reqs)
    assert r["value"] > 0 and r["p50_s"] <= r["p99_s"]
    assert reqs[0].basin.params.precision == PREC_MIXED


def test_cancel_resident_and_pending(gpu_lib):
    """Host-injected cancellation: a resident request that cannot finish is
    cancelled mid-run and leaves the batch between steps; a request that has
    not arrived is cancelled before admission.  Both report
    SIMP_ERR_CANCELLED with their outputs untouched; every other request
    completes with the same bits as stepped alone."""
    from simp_b200.simp import SIMP_ERR_CANCELLED
    reqs = _stream(count=6, seed=36, steps=(20, 60))
    reqs[1].nsteps = 10 ** 7          # cannot finish before its cancellation
    reqs[4].arrival_s = 30.0          # would arrive long after the others are done
    with serve.Server(reqs[0].basin.params, 2 * GB, max_instances=16, max_request_particles=20000,
                      quantum_steps=8, spot_every=1) as srv:
        ids = [srv.submit(r) for r in reqs]
        srv.cancel(ids[1], at_s=0.05)
        srv.cancel(ids[4], at_s=0.0)
        srv.run()
        st = srv.stats()
        assert st["cancelled"] == 2 and st["completed"] == 4 and st["failed"] == 0
        q1, q4 = srv.request(ids[1]), srv.request(ids[4])
        assert q1["status"] == SIMP_ERR_CANCELLED and 0 < q1["steps"] < reqs[1].nsteps
        assert q1["admitted_s"] <= 0.05 <= q1["completed_s"]
        assert q4["status"] == SIMP_ERR_CANCELLED and q4["steps"] == 0 and q4["admitted_s"] < 0
        for rid in (ids[1], ids[4]):
            assert all(not np.any(v) for v in srv.outputs[rid].values())
        assert st["makespan_s"] < 20.0    # the cancelled request was not waited for
        for k, (rid, r) in enumerate(zip(ids, reqs)):
            if k in (1, 4):
                continue
            q = srv.request(rid)
            assert q["status"] == 0 and q["steps"] == r.nsteps
            ref = _alone(r)
            for f in ("x", "vx", "h", "A"):
                assert np.array_equal(srv.outputs[rid][f], ref[f]), (rid, f)


def test_cancel_from_another_thread(gpu_lib):
    """simp_server_cancel while simp_server_run steps on the calling thread."""
    import threading
    import time
    from simp_b200.simp import SIMP_ERR_CANCELLED
    reqs = _stream(count=3, seed=37, steps=(10, 20))
    reqs[0].nsteps = 10 ** 7
    with serve.Server(reqs[0].basin.params, 2 * GB, max_instances=8, max_request_particles=20000,
                      quantum_steps=4) as srv:
        ids = [srv.submit(r) for r in reqs]

        def later():
            time.sleep(0.2)
            srv.cancel(ids[0])

        th = threading.Thread(target=later)
        th.start()
        srv.run()
        th.join()
        q = srv.request(ids[0])
        assert q["status"] == SIMP_ERR_CANCELLED and 0 < q["steps"] < reqs[0].nsteps
        assert srv.stats()["completed"] == 2
