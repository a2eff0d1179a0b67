"""The allocation-free density entry point against the context one.

simp_gpu_sum_density_noalloc serves callers that cannot allocate device
memory (a host whose device arrays belong to another runtime, or a loop that
may not stall on cudaMalloc): they pass their own device buffers and the
library works in a fixed array compiled into it.  This file is collected
last so that a failure here stops a -x run only after every other test.
It must pass alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest

from helpers import rel_l2
from simp_b200 import _lib, basins
from simp_b200.params import SKF_CUBIC, SKF_WENDLAND_C6
from simp_b200.simp import SIMP_ERR_BADARG, SIMP_OK, Simp

pytestmark = pytest.mark.gpu

TOL_RHS = 1e-11   # the FP64 single-evaluation tolerance of the parity tests
MAX_N = 65536     # SIMP_NOALLOC_MAX_PARTICLES


def _noalloc_density(lib, b, skf):
    import torch
    dev = torch.device("cuda")
    x = torch.tensor(b.x, dtype=torch.float64, device=dev).contiguous()
    hs = torch.tensor(b.hsml, dtype=torch.float64, device=dev)
    m = torch.tensor(b.mass, dtype=torch.float64, device=dev)
    rho = torch.tensor(b.rho, dtype=torch.float64, device=dev)
    out = torch.full((b.n,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.simp_gpu_sum_density_noalloc(x.data_ptr(), hs.data_ptr(), m.data_ptr(), rho.data_ptr(),
                                          b.n, skf, out.data_ptr(), stream)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def _context_density(b, skf):
    prm = b.params.copy()
    prm.skf = skf
    with Simp.from_basin(b, prm) as s:
        return s.sum_density()


def _varied_basin():
    b = basins.make_basin(120, 1000.0, 9, walls="+x-x")
    rng = np.random.default_rng(3)
    b.hsml = b.hsml * rng.uniform(0.8, 1.2, size=b.n)
    b.rho = b.rho * rng.uniform(0.9, 1.1, size=b.n)
    return b


def test_noalloc_matches_context_density_on_consecutive_calls(gpu_lib):
    lib = _lib.load()
    runs = [(basins.cfg1(), SKF_CUBIC), (_varied_basin(), SKF_WENDLAND_C6), (basins.cfg1(), SKF_CUBIC)]
    for b, skf in runs:   # consecutive calls share the fixed working array
        rc, got = _noalloc_density(lib, b, skf)
        assert rc == SIMP_OK
        want = _context_density(b, skf)
        assert np.all(np.isfinite(got))
        assert rel_l2(got, want) < TOL_RHS, rel_l2(got, want)


def test_noalloc_rejects_too_many_particles(gpu_lib):
    lib = _lib.load()
    rc = lib.simp_gpu_sum_density_noalloc(1, 1, 1, 1, MAX_N + 1, SKF_CUBIC, 1, None)
    assert rc == SIMP_ERR_BADARG


def _oracle_density(oracle_mod, b, skf):
    prm = b.params.copy()
    prm.skf = skf
    o = oracle_mod.Oracle.from_basin(b, prm)
    return o.sum_density(k0_mode=1)


def test_noalloc_against_oracle(gpu_lib, oracle_mod):
    """Directly against the oracle's summation density (density.f90:41-100,
    kernel_zero from each particle's own hsml), twice in a row."""
    lib = _lib.load()
    for b, skf in ((_varied_basin(), SKF_WENDLAND_C6), (basins.cfg1(), SKF_CUBIC)):
        rc, got = _noalloc_density(lib, b, skf)
        assert rc == SIMP_OK
        want = _oracle_density(oracle_mod, b, skf)
        assert rel_l2(got, want) < TOL_RHS, rel_l2(got, want)


def test_noalloc_at_the_particle_limit(gpu_lib, oracle_mod):
    """n = SIMP_NOALLOC_MAX_PARTICLES (a 256 x 256 lattice with varied hsml)."""
    lib = _lib.load()
    b = basins.make_basin(256, 1000.0, 17, walls="")
    rng = np.random.default_rng(5)
    b.hsml = b.hsml * rng.uniform(0.85, 1.1, size=b.n)
    assert b.n == MAX_N
    rc, got = _noalloc_density(lib, b, SKF_CUBIC)
    assert rc == SIMP_OK
    assert rel_l2(got, _context_density(b, SKF_CUBIC)) < TOL_RHS
    assert rel_l2(got, _oracle_density(oracle_mod, b, SKF_CUBIC)) < TOL_RHS


def test_noalloc_grid_grows_for_a_far_outlier(gpu_lib, oracle_mod):
    """A compact basin plus one particle 3,000 km away: the extent spans far
    more than 131,072 cells of side max(hsml), so the grid's cells are
    enlarged until it fits (and the cluster's cells hold many particles).
    The outlier has no neighbours (its density stays rho, to rounding)."""
    lib = _lib.load()
    b = basins.make_basin(100, 1000.0, 23, walls="")
    far = np.array([[3.0e6, 2.5e6]])
    b.x = np.vstack([b.x, far])
    b.vx = np.vstack([b.vx, np.zeros((1, 2))])
    for k in ("mass", "rho", "hsml", "A", "h"):
        setattr(b, k, np.concatenate([getattr(b, k), getattr(b, k)[:1]]))
    ncells = (3.0e6 / b.hsml.max()) * (2.5e6 / b.hsml.max())
    assert ncells > 2 * MAX_N
    for _ in range(2):
        rc, got = _noalloc_density(lib, b, SKF_CUBIC)
        assert rc == SIMP_OK
        assert abs(got[-1] / b.rho[-1] - 1.0) < 1e-14   # (k0 m) / (k0 m / rho)
        assert rel_l2(got, _oracle_density(oracle_mod, b, SKF_CUBIC)) < TOL_RHS
        assert rel_l2(got, _context_density(b, SKF_CUBIC)) < TOL_RHS


def test_noalloc_rejects_host_arrays(gpu_lib):
    """Host arrays (what the context entry points take) are refused with
    SIMP_ERR_BADARG before anything is launched; device buffers in the same
    call still work afterwards."""
    lib = _lib.load()
    b = basins.cfg1()
    x = np.ascontiguousarray(b.x)
    out = np.zeros(b.n)
    rc = lib.simp_gpu_sum_density_noalloc(_lib.dptr(x), _lib.dptr(b.hsml), _lib.dptr(b.mass), _lib.dptr(b.rho),
                                          b.n, SKF_CUBIC, _lib.dptr(out), None)
    assert rc == SIMP_ERR_BADARG
    assert np.all(out == 0.0)
    rc, got = _noalloc_density(lib, b, SKF_CUBIC)
    assert rc == SIMP_OK
    assert rel_l2(got, _context_density(b, SKF_CUBIC)) < TOL_RHS
