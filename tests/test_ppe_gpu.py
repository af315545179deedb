"""GPU parity of the pressure Poisson solver against the reference.

Golden vectors come from the reference's own C solver (tests/golden, built from
src/src_c unmodified); live cases use the oracle's bit-exact restatement of it.
The (kx,ky) = (0,0) system of the Neumann problem is singular up to round-off
(its last pivot is round-off, mod_poisson_solver.c:337-342), so p is defined up
to an additive constant that differs with the summation order of any two
implementations: p is compared modulo its mean, with max|diff| / max|p|.
FP64 tolerance: 1e-12 relative (the FP64 path's parity bar)."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def relerr_modmean(a, b):
    a = a - a.mean()
    b = b - b.mean()
    return np.abs(a - b).max() / np.abs(b).max()


def partitions(nz, nparts):
    """z-partitions of decomp_2d.c:261-283 (0-based start, size)"""
    size, nu = nz // nparts, nz % nparts
    sz = [size if m < nparts - nu else size + 1 for m in range(nparts)]
    return [(sum(sz[:m]), sz[m]) for m in range(nparts)]


def relerr_pdd(a, b, nparts):
    """PDD with two partitions has a single interface whose 2x2 reduced system
    is the exact one, and for the (kx,ky) = (0,0) mode that system inherits
    the singularity of the Neumann problem (det = w*v - 1 is round-off): the
    reference's solution then carries an arbitrary constant per partition,
    fixed by round-off.  Compare modulo one constant per partition there;
    with P >= 3 the truncated interface systems are regular and one global
    constant is the only freedom."""
    if nparts != 2:
        return relerr_modmean(a, b)
    a = a.copy()
    b = b.copy()
    for k0, ke in partitions(a.shape[0], nparts):
        a[k0:k0 + ke] -= a[k0:k0 + ke].mean()
        b[k0:k0 + ke] -= b[k0:k0 + ke].mean()
    return np.abs(a - b).max() / np.abs(b).max()


GOLDEN_PPE = sorted(glob.glob(os.path.join(GOLDEN, "ppe_*.npz")))


@pytest.mark.parametrize("path", GOLDEN_PPE, ids=[os.path.basename(p)[:-4] for p in GOLDEN_PPE])
def test_reference_abi_vs_golden(gpu, path):
    """init/execute/free_poisson_solver through the C ABI on the ghosted host
    array, against the reference's own output."""
    plb = gpu
    d = np.load(path)
    nx, ny, nz = int(d["nx"]), int(d["ny"]), int(d["nz"])
    nparts = int(d["p_col"]) if int(d["pdd"]) else 0
    var = np.full((nz + 2, ny + 2, nx + 2), 7.25)  # ghosts must stay untouched
    var[1:-1, 1:-1, 1:-1] = d["rhs"]
    with plb.PoissonSolver(nx, ny, nz, float(d["dx"]), float(d["dy"]), d["dzf"], nparts=nparts) as s:
        s.execute(var)
    assert relerr_pdd(var[1:-1, 1:-1, 1:-1], d["p"], nparts) < TOL64
    ghost = var.copy()
    ghost[1:-1, 1:-1, 1:-1] = 7.25
    assert np.all(ghost == 7.25)


@pytest.mark.parametrize("path", GOLDEN_PPE[:3], ids=[os.path.basename(p)[:-4] for p in GOLDEN_PPE[:3]])
def test_device_ppe_vs_golden(gpu, path):
    import torch
    plb = gpu
    d = np.load(path)
    nx, ny, nz = int(d["nx"]), int(d["ny"]), int(d["nz"])
    nparts = int(d["p_col"]) if int(d["pdd"]) else 0
    s = plb.DevicePoissonSolver(nx, ny, nz, float(d["dx"]), float(d["dy"]), d["dzf"], nparts=nparts)
    x = torch.tensor(d["rhs"], dtype=torch.float64, device="cuda").contiguous()
    s.solve(x)
    torch.cuda.synchronize()
    assert relerr_pdd(x.cpu().numpy(), d["p"], nparts) < TOL64
    # repeated solves are deterministic (no races in the kernels)
    y = torch.tensor(d["rhs"], dtype=torch.float64, device="cuda").contiguous()
    s.solve(y)
    torch.cuda.synchronize()
    assert torch.equal(x, y)


# Thomas keeps its swept values in tensor memory for nz % 8 == 0: all of them
# for nz <= 256 (768x32x256: two rounds of columns per CTA; 16x8x8: one 8-row
# group, exactly one CTA of 128 columns; 8x6x16: one CTA with 80 idle
# threads), 256 of them for taller columns with the rest in HBM (32x24x264,
# 32x24x512); in HBM alone for other nz.  PDD: each partition in tensor
# memory for up to 8 partitions of multiples of 8 rows (256x192x32/4,
# 64x48x32/2), one thread per (column, partition) with the swept values in
# HBM otherwise up to 32 partitions (64x48x40/8, 96x72x30/4, 32x24x96/12,
# 32x24x100/12), one thread per column beyond (32x24x96/40)
@pytest.mark.parametrize("nx,ny,nz,nparts", [(64, 64, 64, 0), (128, 96, 48, 0), (256, 192, 32, 4),
                                            (64, 48, 40, 8), (96, 72, 30, 4), (64, 48, 32, 2),
                                            (64, 48, 30, 0), (32, 24, 264, 0), (768, 32, 256, 0),
                                            (16, 8, 8, 0), (8, 6, 16, 0), (32, 24, 512, 0),
                                            (32, 24, 96, 12), (32, 24, 100, 12), (32, 24, 96, 40)])
def test_ppe_vs_oracle_live(gpu, oracle_mod, nx, ny, nz, nparts):
    """Sizes beyond the fixtures (radix-3 lengths, uneven PDD partitions)."""
    import torch
    plb, O = gpu, oracle_mod
    g = O.Grid(nx, ny, nz, stretch=1.8)
    rng = np.random.default_rng(nx + ny + nz)
    r = rng.standard_normal((nz, ny, nx))
    wgt = g.dzf_global[1:-1]
    r -= (r.mean(axis=(1, 2)) * wgt).sum() / wgt.sum()
    var = np.zeros(g.shape)
    var[1:-1, 1:-1, 1:-1] = r
    O.PPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global, nparts=nparts).execute(var)
    s = plb.DevicePoissonSolver(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global, nparts=nparts)
    x = torch.tensor(r, dtype=torch.float64, device="cuda").contiguous()
    s.solve(x)
    torch.cuda.synchronize()
    assert relerr_pdd(x.cpu().numpy(), var[1:-1, 1:-1, 1:-1], nparts) < TOL64


@pytest.mark.parametrize("mx,my", [(1, 0), (0, 1), (3, 2), (16, 12), (32, 0)])
def test_ppe_single_modes(gpu, oracle_mod, mx, my):
    """Manufactured solution: p = cos(2 pi mx x/Lx + 0.3) cos(2 pi my y/Ly),
    uniform in z, solves L p = lambda p exactly (lambda the discrete
    eigenvalue, mod_fft_fftw.inc:115-118).  Tolerance relative to the input
    amplitude: high modes have |lambda| >> 1, so p is much smaller than f."""
    import torch
    plb, O = gpu, oracle_mod
    nx, ny, nz = 64, 48, 16
    g = O.Grid(nx, ny, nz, stretch=2.0)
    x = (np.arange(nx) + 0.5) * g.g.dx
    y = (np.arange(ny) + 0.5) * g.g.dy
    f = (np.cos(2 * np.pi * mx * x / g.g.lx + 0.3)[None, None, :] * np.cos(2 * np.pi * my * y / g.g.ly)[None, :, None]
         * np.ones((nz, 1, 1)))
    lam = 2 * (np.cos(2 * np.pi * mx / nx) - 1) / g.g.dx ** 2 + 2 * (np.cos(2 * np.pi * my / ny) - 1) / g.g.dy ** 2
    s = plb.DevicePoissonSolver(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global)
    t = torch.tensor(f, dtype=torch.float64, device="cuda").contiguous()
    s.solve(t)
    torch.cuda.synchronize()
    got = t.cpu().numpy()
    assert np.abs((got - got.mean()) - (f / lam - (f / lam).mean())).max() < 1e-13 * np.abs(f).max()


def test_ppe_linearity_full_size(gpu):
    """Size-independent property at the 512x384x256 bench size: the solver is
    linear (solve(a x + b y) = a solve(x) + b solve(y), modulo the null mode)."""
    import torch
    plb = gpu
    nx, ny, nz = 512, 384, 256
    dzf = np.full(nz + 2, 2.0 / nz)
    s = plb.DevicePoissonSolver(nx, ny, nz, 2 * np.pi / nx, np.pi / ny, dzf)
    gen = torch.Generator(device="cuda").manual_seed(3)
    xa = torch.randn((nz, ny, nx), dtype=torch.float64, device="cuda", generator=gen)
    xb = torch.randn((nz, ny, nx), dtype=torch.float64, device="cuda", generator=gen)
    xa -= xa.mean()
    xb -= xb.mean()
    xc = 2.0 * xa - 0.5 * xb
    for t in (xa, xb, xc):
        s.solve(t)
    torch.cuda.synchronize()
    lhs = xc - xc.mean()
    rhs = 2.0 * (xa - xa.mean()) - 0.5 * (xb - xb.mean())
    assert ((lhs - rhs).abs().max() / rhs.abs().max()).item() < 1e-11
