"""GPU test of pl_ppe_solve_noalloc, the allocation-free PPE entry point.

Callers that cannot call cudaMalloc while they solve (a host program whose
device memory belongs to another allocator, or a loop that must not stall on
cudaMalloc) use it: it takes the FP64 scratch of the tridiagonal sweep from a
fixed array inside the library.  This file sorts last so that a run stopping at the first failure
has already run every other test; it also passes on its own."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the mixed-precision PPE tolerance used elsewhere: FP32 transforms
TOL_MIXED = 1e-6


def _rhs(nx, ny, nz, dzf, seed):
    rng = np.random.default_rng(seed)
    r = rng.standard_normal((nz, ny, nx))
    wgt = dzf[1:-1]
    r -= (r.mean(axis=(1, 2)) * wgt).sum() / wgt.sum()
    return r.astype(np.float32)


def test_noalloc_matches_allocating_solve(gpu):
    import torch
    plb = gpu
    L = plb.lib()
    nx, ny, nz = 128, 96, 64
    zf = 0.5 * (1.0 + np.tanh((np.arange(nz + 1) / nz - 0.5) * 1.8) / np.tanh(0.9))
    dzf = np.empty(nz + 2)
    dzf[1:-1] = 2.0 * np.diff(zf)
    dzf[0], dzf[-1] = dzf[1], dzf[-2]
    s = plb.DevicePoissonSolver(nx, ny, nz, 2 * np.pi / nx, np.pi / ny, dzf, nparts=0, precision=plb.PL_MIXED)
    for call, seed in enumerate((1, 2)):  # two calls in a row share the fixed scratch
        r = _rhs(nx, ny, nz, dzf, seed)
        ref = torch.tensor(r, device="cuda").contiguous()
        s.solve(ref)  # the allocating entry point
        got = torch.tensor(r, device="cuda").contiguous()
        rc = L.pl_ppe_solve_noalloc(s._h, C.c_void_p(got.data_ptr()), None)
        assert rc == 0, L.pl_last_error().decode()
        torch.cuda.synchronize()
        a, b = got.double(), ref.double()
        err = ((a - a.mean()) - (b - b.mean())).abs().max().item() / (b - b.mean()).abs().max().item()
        assert err <= TOL_MIXED, (call, err)


def test_noalloc_rejects_oversized_plan(gpu):
    import torch
    plb = gpu
    L = plb.lib()
    nx, ny, nz = 256, 128, 128  # 4,194,304 values > 2,097,152
    dzf = np.full(nz + 2, 2.0 / nz)
    s = plb.DevicePoissonSolver(nx, ny, nz, 2 * np.pi / nx, np.pi / ny, dzf, nparts=0, precision=plb.PL_MIXED)
    x = torch.zeros((nz, ny, nx), dtype=torch.float32, device="cuda")
    rc = L.pl_ppe_solve_noalloc(s._h, C.c_void_p(x.data_ptr()), None)
    assert rc == -1
    assert "exceeds the fixed scratch" in L.pl_last_error().decode()
