"""GPU runs of the benchmark configurations against the oracle.

C2: FP64, 256x192x128, Re_tau 550, stretch 1.8, PDD with 4 wall-normal
partitions, perturbation 0.05 from seed 7, 100 steps, against the oracle
(the C restatement of the stencils around the restated PDD solve, which is
bit-identical to the reference's own forked-rank PDD build on the golden
vectors), and the standalone PPE solve of a seeded zero-mean N(0,1)
right-hand side.

C3: the benchmark workload, 512x384x256, Re_tau 1000, stretch 2.0, Thomas,
perturbation 0.1 from seed 11: the FP64 path after 10 and 100 steps and the
mixed path after 100 steps, against the oracle step with the reference's own
C PPE (oracle/_ref, built unmodified), run in a subprocess.

C4: mixed precision at scale, 1024x768x512, Re_tau 2000, stretch 2.0, PDD
with 8 partitions: both paths after 5 steps against the oracle (restated PDD
PPE), and the mixed path against the FP64 path after 50 steps.

Every comparison reports max and L2 errors per field: velocities directly
(relative to the field's max |.| and L2 norm), the pressure modulo its mean
(the Neumann null mode).  The FP64 bar is 1e-12 relative at every step count
(measured on B200: at most 2.5e-14 after 100 steps).  The pressure's bar is
1e-10: the reference fixes the null-mode constant by dividing round-off by
the round-off last pivot of the (0,0) system, so p carries a large arbitrary
constant and its digits below eps times that constant are noise in either
implementation (measured 4e-12).
"""
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def rel_l2(a, b):
    a = a[1:-1, 1:-1, 1:-1]
    b = b[1:-1, 1:-1, 1:-1]
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def field_errors(got, ref, name):
    """max and L2 relative errors of interior arrays; p modulo its mean"""
    a = np.asarray(got, dtype=np.float64)
    b = np.asarray(ref, dtype=np.float64)
    if name == "p":
        a = a - a.mean()
        b = b - b.mean()
    d = a - b
    return {"max": float(np.abs(d).max() / np.abs(b).max()),
            "l2": float(np.sqrt((d * d).sum() / (b * b).sum()))}


def interior(ch, q):
    return ch.get_field(q)[1:-1, 1:-1, 1:-1]


def test_c2_fp64_pdd4_100_steps_match_oracle(gpu, oracle_mod):
    plb, O = gpu, oracle_mod
    nx, ny, nz, nparts = 256, 192, 128, 4
    cfg = plb.ChannelConfig(nx=nx, ny=ny, nz=nz, stretch_ratio=1.8, re_tau=550.0, trid_parts=nparts, dt=1e-4)
    ch = plb.Channel(cfg)
    ch.init_flow(7, 0.05)
    g = O.Grid(nx, ny, nz, stretch=1.8, re_tau=550.0, dt=1e-4)
    u, v, w, p = g.init_flow(7, 0.05)
    ppe = O.PPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global, nparts=nparts)
    u1, v1, w1 = g.zeros(), g.zeros(), g.zeros()
    for _ in range(10):
        g.step(ppe, u, v, w, u1, v1, w1, p)
    ch.step(10)
    gu, gv, gw, _ = ch.get_fields()
    errs10 = [rel(a, b) for a, b in ((gu, u), (gv, v), (gw, w))]
    for _ in range(90):
        g.step(ppe, u, v, w, u1, v1, w1, p)
    ch.step(90)
    gu, gv, gw, _ = ch.get_fields()
    errs = [rel(a, b) for a, b in ((gu, u), (gv, v), (gw, w))]
    print("C2 max rel err u v w after 10 steps:", errs10, "after 100 steps:", errs)
    assert max(errs10) < TOL64
    assert max(errs) < TOL64
    d = ch.diagnostics()
    div_o, _ = g.max_div(u, v, w)
    assert abs(d["div_max"] - div_o) <= 1e-6 * div_o
    ch.close()


def test_c2_standalone_ppe_pdd4(gpu, oracle_mod):
    import torch
    plb, O = gpu, oracle_mod
    nx, ny, nz, nparts = 256, 192, 128, 4
    g = O.Grid(nx, ny, nz, stretch=1.8)
    rng = np.random.default_rng(7)
    r = rng.standard_normal((nz, ny, nx))
    wgt = g.dzf_global[1:-1]
    r -= (r.mean(axis=(1, 2)) * wgt).sum() / wgt.sum()
    var = np.zeros((nz + 2, ny + 2, nx + 2))
    var[1:-1, 1:-1, 1:-1] = r
    O.PPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global, nparts=nparts).execute(var)
    s = plb.DevicePoissonSolver(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global, nparts=nparts)
    x = torch.tensor(r, dtype=torch.float64, device="cuda").contiguous()
    s.solve(x)
    torch.cuda.synchronize()
    got = x.cpu().numpy()
    ref = var[1:-1, 1:-1, 1:-1]
    # with P >= 3 partitions the truncated interface systems are regular:
    # the Neumann null mode (one global constant) is the only freedom
    err = np.abs((got - got.mean()) - (ref - ref.mean())).max() / np.abs(ref).max()
    print("C2 standalone PDD4 PPE rel err (modulo the mean):", err)
    assert err < TOL64


def test_c3_bench_workload_vs_oracle(gpu):
    """The benchmark workload against the oracle with the reference's own PPE:
    FP64 after 10 and 100 steps at the FP64 bar, and the mixed path after 100
    steps at its bar (velocity rel. L2 <= 1e-5, max |div u| <= 1e-10)."""
    from oracle import run_channel as R
    plb = gpu
    kw = dict(stretch=2.0, re_tau=1000.0, dt=1e-4, seed=11, noise=0.1)
    grid = (512, 384, 256)
    res = {}
    with tempfile.TemporaryDirectory() as td:
        meta = R.run(td, grid, [10, 100], **kw)
        print("oracle:", meta["what"], f"{np.mean(meta['step_seconds'][1:]):.2f} s/step,", meta["threads"], "threads")
        for name, prec in (("fp64", plb.PL_FP64), ("mixed", plb.PL_MIXED)):
            cfg = plb.ChannelConfig(nx=grid[0], ny=grid[1], nz=grid[2], stretch_ratio=2.0, re_tau=1000.0,
                                    dt=1e-4, precision=prec)
            ch = plb.Channel(cfg)
            ch.init_flow(11, 0.1)
            ch.step(10)
            if name == "fp64":
                ref = R.load(td, 10)
                res[(name, 10)] = {q: field_errors(interior(ch, i), ref[i], q) for i, q in enumerate("uvwp")}
            ch.step(90)
            ref = R.load(td, 100)
            res[(name, 100)] = {q: field_errors(interior(ch, i), ref[i], q) for i, q in enumerate("uvwp")}
            res[(name, "div")] = ch.diagnostics()["div_max"]
            ch.close()
    for k, v in res.items():
        print("C3", k, v)
    for q in "uvw":
        assert res[("fp64", 10)][q]["max"] < TOL64, (q, res[("fp64", 10)][q])
        assert res[("fp64", 100)][q]["max"] < TOL64, (q, res[("fp64", 100)][q])
        assert res[("mixed", 100)][q]["l2"] <= 1e-5, (q, res[("mixed", 100)][q])
    assert res[("fp64", 10)]["p"]["max"] < 1e-10
    assert res[("fp64", 100)]["p"]["max"] < 1e-10
    assert res[("fp64", "div")] <= 1e-10
    assert res[("mixed", "div")] <= 1e-10


def test_c4_mixed_pdd8_vs_oracle_and_fp64(gpu, oracle_mod):
    """1024x768x512, PDD with 8 partitions: both paths after 5 steps against
    the oracle (restated PDD PPE, all host threads), then 45 more steps and the
    mixed path against the FP64 path.  PDD's truncation of the interface
    systems is the reference's algorithm, so both paths leave the oracle's
    projection divergence."""
    plb, O = gpu, oracle_mod
    nx, ny, nz, nparts = 1024, 768, 512, 8
    g = O.Grid(nx, ny, nz, stretch=2.0, re_tau=2000.0, dt=1e-4)
    u, v, w, p = g.init_flow(11, 0.1)
    u1, v1, w1 = g.zeros(), g.zeros(), g.zeros()
    ppe = O.PPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global, nparts=nparts)
    for _ in range(5):
        g.step(ppe, u, v, w, u1, v1, w1, p)
    del u1, v1, w1, ppe
    div_o, _ = g.max_div(u, v, w)
    ref = (u, v, w, p)
    chans, errs5 = {}, {}
    for name, prec in (("fp64", plb.PL_FP64), ("mixed", plb.PL_MIXED)):
        cfg = plb.ChannelConfig(nx=nx, ny=ny, nz=nz, stretch_ratio=2.0, re_tau=2000.0, trid_parts=nparts, dt=1e-4,
                                precision=prec)
        ch = plb.Channel(cfg)
        ch.init_flow(11, 0.1)
        ch.step(5)
        # one component at a time to bound host memory (3.2 GB per field)
        errs5[name] = {q: field_errors(interior(ch, i), ref[i][1:-1, 1:-1, 1:-1], q) for i, q in enumerate("uvwp")}
        errs5[name]["div"] = ch.diagnostics()["div_max"]
        chans[name] = ch
    del ref, u, v, w, p
    print("C4 after 5 steps vs oracle:", errs5, "oracle div", div_o)
    for q in "uvw":
        assert errs5["fp64"][q]["max"] < TOL64, (q, errs5["fp64"][q])
        assert errs5["mixed"][q]["l2"] <= 1e-5, (q, errs5["mixed"][q])
    assert errs5["fp64"]["p"]["max"] < 1e-10
    assert abs(errs5["fp64"]["div"] - div_o) <= 1e-6 * div_o
    assert abs(errs5["mixed"]["div"] - div_o) <= 1e-3 * div_o
    for ch in chans.values():
        ch.step(45)
        ch.synchronize()
    f64, mix = chans["fp64"], chans["mixed"]
    errs = []
    for q in range(3):
        a, b = mix.get_field(q), f64.get_field(q)
        errs.append(rel_l2(a, b))
        del a, b
    dm, df = mix.diagnostics(), f64.diagnostics()
    print("C4 50 steps, rel L2 mixed vs FP64 (u v w):", errs, "div", dm["div_max"], df["div_max"])
    assert max(errs) <= 1e-5
    assert dm["nan_count"] == 0
    assert abs(dm["div_max"] - df["div_max"]) <= 1e-3 * df["div_max"]
    f64.close()
    mix.close()
