"""The multi-GPU z-slab step of the library, checked on one GPU.

G slabs (pl_channel_create_slab) live in one process on the one device and
slab.LocalTransport moves their planes with device copies between the phases,
in the schedule of slab.step; each slab's kernels are separate launches that
wait on nothing but the host.  The result is compared with the one-GPU
channel solving the same global problem with PDD over the same G partitions
(trid_parts = G), which the oracle pins to the reference's multi-rank PDD:
FP64 to 1e-12 (only Mean_h's sum runs in another order), mixed at FP32
rounding of the increments.  The projected divergence itself is round-off,
so it is held to a bound rather than matched."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gather(slabs, which):
    parts = [s.get_field(which) for s in slabs]
    inner = [p[1:-1] for p in parts]
    return np.concatenate([parts[0][:1]] + inner + [parts[-1][-1:]], axis=0)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nx,ny,nz,G", [(64, 48, 32, 2), (64, 48, 30, 4), (32, 16, 24, 3)])
def test_slabs_match_one_gpu_pdd(gpu, precision, nx, ny, nz, G):
    plb = gpu
    from powerllel_channel_b200 import slab as S
    prec = plb.PL_FP64 if precision == "fp64" else plb.PL_MIXED
    cfg = plb.ChannelConfig(nx=nx, ny=ny, nz=nz, stretch_ratio=1.5, re_tau=180.0, trid_parts=G, precision=prec)
    nsteps = 5
    one = plb.Channel(cfg)
    one.init_flow(42, 0.1)
    one.step(nsteps)
    ref = [one.get_field(q) for q in range(3)]
    dref = one.diagnostics()
    one.close()
    if precision == "mixed":
        # the FP64 path with the same partitions: the mixed bar
        cfg64 = plb.ChannelConfig(nx=nx, ny=ny, nz=nz, stretch_ratio=1.5, re_tau=180.0, trid_parts=G)
        f64 = plb.Channel(cfg64)
        f64.init_flow(42, 0.1)
        f64.step(nsteps)
        ref64 = [f64.get_field(q) for q in range(3)]
        f64.close()

    slabs = [S.Slab(cfg, r, G) for r in range(G)]
    nzs = [s.nz for s in slabs]
    assert nzs == S.slab_sizes(nz, G)[1]
    tr = S.LocalTransport(slabs)
    S.init_flow(slabs, tr, nzs, 42, 0.1)
    for _ in range(nsteps):
        S.step(slabs, tr, nzs)
    got = [_gather(slabs, q) for q in range(3)]
    d = S.diagnostics([s.diagnostics() for s in slabs])
    errs = [rel(a, b) for a, b in zip(got, ref)]
    print(f"{precision} {nx}x{ny}x{nz} over {G} slabs: max rel err u v w {errs}, div {d['div_max']} vs "
          f"{dref['div_max']}")
    tol = 1e-12 if precision == "fp64" else 1e-7
    assert max(errs) < tol
    # With two partitions PDD is exact and the projected divergence is
    # round-off of the fields' last bits, which Mean_h's summation order
    # already changes: both stay at round-off (FP64) or at the FP32
    # resolution of the full pressure that the mixed path solves for under
    # PDD (measured 2.7e-10).  With more, PDD's truncation leaves a
    # divergence of its own (4.5e-3 at 64x48x30 over 4), which both match.
    if dref["div_max"] > 1e-8:
        assert abs(d["div_max"] - dref["div_max"]) <= (1e-9 if precision == "fp64" else 1e-5) * dref["div_max"]
    else:
        dbar = 1e-12 if precision == "fp64" else 1e-9
        assert d["div_max"] <= dbar and dref["div_max"] <= dbar
    assert abs(d["cfl_max"] - dref["cfl_max"]) <= tol * dref["cfl_max"]
    if precision == "fp64":
        assert tuple(d["cfl_ijk"]) == tuple(dref["cfl_ijk"])
    assert d["nan_count"] == 0
    if precision == "mixed":
        l2 = [float(np.linalg.norm((a - b)[1:-1, 1:-1, 1:-1]) / np.linalg.norm(b[1:-1, 1:-1, 1:-1]))
              for a, b in zip(got, ref64)]
        print("  mixed slabs vs FP64 one-GPU, rel L2 u v w:", l2)
        assert max(l2) <= 1e-5
    for s in slabs:
        s.close()
