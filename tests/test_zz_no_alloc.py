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
