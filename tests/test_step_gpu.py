"""GPU parity of the RK2 projection step (FP64 path) against the oracle.

Every phase is compared on the same input state; the whole step is compared
after several steps.  Velocities are compared directly (max|diff| / max|u|), the pressure modulo its
mean (the Neumann null mode, see test_ppe_gpu) relative to max|p|.
FP64 tolerance 1e-12 relative."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def rel_modmean(a, b):
    """pressure: modulo the Neumann null mode (its mean), relative to the stored
    field's magnitude -- the reference fixes the null-mode constant by
    dividing round-off by the round-off last pivot, so digits below
    eps*max|p| carry no information in either implementation"""
    a = a[1:-1, 1:-1, 1:-1]
    b = b[1:-1, 1:-1, 1:-1]
    return np.abs((a - a.mean()) - (b - b.mean())).max() / max(np.abs(b).max(), 1e-300)


def make_pair(plb, O, nx, ny, nz, stretch=1.5, re_tau=180.0, nparts=0, seed=42, noise=0.1, dt=1e-4):
    cfg = plb.ChannelConfig(nx=nx, ny=ny, nz=nz, stretch_ratio=stretch, re_tau=re_tau, trid_parts=nparts, dt=dt)
    ch = plb.Channel(cfg)
    ch.init_flow(seed, noise)
    g = O.Grid(nx, ny, nz, stretch=stretch, re_tau=re_tau, dt=dt)
    return ch, g


def test_init_flow_matches_oracle(gpu, oracle_mod):
    plb, O = gpu, oracle_mod
    ch, g = make_pair(plb, O, 32, 24, 16)
    u, v, w, p = ch.get_fields()
    uo, vo, wo, po = g.init_flow(42, 0.1)
    assert np.array_equal(v, vo) and np.array_equal(w, wo)  # op-by-op identical
    assert rel(u, uo) < 1e-15                                 # mean normalisation sums in another order
    assert np.all(p == 0)


def _state(plb, O, nx=48, ny=36, nz=24, nsteps=2):
    """a developed (non-initial) state from the oracle, loaded into both"""
    ch, g = make_pair(plb, O, nx, ny, nz)
    u, v, w, p = g.init_flow(7, 0.2)
    ppe = O.PPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global)
    u1, v1, w1 = g.zeros(), g.zeros(), g.zeros()
    for _ in range(nsteps):
        g.step(ppe, u, v, w, u1, v1, w1, p)
    ch.set_fields(u, v, w)
    return ch, g, ppe, (u, v, w)


def test_phase_rk1(gpu, oracle_mod):
    plb, O = gpu, oracle_mod
    ch, g, _, (u, v, w) = _state(plb, O)
    u1, v1, w1 = g.rk1(u, v, w)
    g.bound_vel(u1, v1, w1)
    ch.phase("rk1")
    for which, ref in ((4, u1), (5, v1), (6, w1)):
        assert rel(ch.get_field(which), ref) < TOL64, which


def test_phase_rk2_rhs_ppe_correct(gpu, oracle_mod):
    """RK2, calcRHS, PPE, correct+force on the same state, each compared."""
    plb, O = gpu, oracle_mod
    ch, g, ppe, (u, v, w) = _state(plb, O)
    u1, v1, w1 = g.rk1(u, v, w)
    g.bound_vel(u1, v1, w1)
    g.rk2(u, v, w, u1, v1, w1)
    g.bound_vel(u, v, w)
    ch.phase("rk1")
    ch.phase("rk2")
    for which, ref in ((0, u), (1, v), (2, w)):
        assert rel(ch.get_field(which), ref) < TOL64, which
    p = g.zeros()
    g.calc_rhs(u, v, w, p)
    ch.phase("calc_rhs")
    got = ch.get_field(3)
    # div(u)/dt cancels terms of size |u|/(dx dt): measure the error on that scale
    scale = (np.abs(u).max() * g.g.dx_inv + np.abs(v).max() * g.g.dy_inv
             + np.abs(w).max() * g.arr1d("dzf_inv").max()) / g.g.dt
    assert np.abs(got[1:-1, 1:-1, 1:-1] - p[1:-1, 1:-1, 1:-1]).max() < 1e-14 * scale
    ppe.execute(p)
    g.bound_p(p)
    ch.phase("poisson")
    assert rel_modmean(ch.get_field(3), p) < TOL64
    g.correct_vel(p, u, v, w)
    g.force_vel(u, v, w)
    g.bound_vel(u, v, w)
    ch.phase("correct_force")
    for which, ref in ((0, u), (1, v), (2, w)):
        assert rel(ch.get_field(which), ref) < TOL64, which


@pytest.mark.parametrize("nparts", [0, 4])
def test_steps_match_oracle(gpu, oracle_mod, nparts):
    """Ten whole steps from the seeded initial field (C1 settings, 64^3,
    Re_tau 180, stretch 1.5, noise 0.1, seed 42; PDD with 4 partitions too)."""
    plb, O = gpu, oracle_mod
    nx = ny = nz = 64
    ch, g = make_pair(plb, O, nx, ny, nz, nparts=nparts)
    u, v, w, p = g.init_flow(42, 0.1)
    ppe = O.PPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global, nparts=nparts)
    u1, v1, w1 = g.zeros(), g.zeros(), g.zeros()
    for _ in range(10):
        g.step(ppe, u, v, w, u1, v1, w1, p)
    ch.step(10)
    gu, gv, gw, gp = ch.get_fields()
    for a, b in ((gu, u), (gv, v), (gw, w)):
        assert rel(a, b) < TOL64
    assert rel_modmean(gp, p) < 1e-10
    d = ch.diagnostics()
    div_o, ijk = g.max_div(u, v, w)
    if nparts == 0:
        assert d["div_max"] < 1e-12 and div_o < 1e-12
    else:
        # PDD truncates the low-wavenumber systems (the reference's algorithm),
        # so the projection leaves a divergence; it must be the reference's
        assert abs(d["div_max"] - div_o) < 1e-9 * div_o and tuple(d["div_ijk"]) == ijk
    cfl_o, cijk = g.max_cfl(u, v, w)
    assert abs(d["cfl_max"] - cfl_o) < 1e-12 * cfl_o and tuple(d["cfl_ijk"]) == cijk
    assert d["nan_count"] == 0


def test_step_fixture(gpu):
    """The golden step (oracle stencils + the reference's own PPE), 5 steps."""
    plb = gpu
    d = np.load(os.path.join(GOLDEN, "step_32x24x16_5.npz"))
    cfg = plb.ChannelConfig(nx=int(d["nx"]), ny=int(d["ny"]), nz=int(d["nz"]), stretch_ratio=float(d["stretch"]),
                            re=float(d["re"]), dt=float(d["dt"]))
    ch = plb.Channel(cfg)
    ch.init_flow(int(d["seed"]), float(d["noise"]))
    ch.step(int(d["nsteps"]))
    u, v, w, p = ch.get_fields()
    for a, b in ((u, d["u"]), (v, d["v"]), (w, d["w"])):
        assert rel(a, b) < TOL64


def test_diagnostics_locate_divergence(gpu, oracle_mod):
    """calcMaxDiv / calcMaxCFL with location on a divergent field; NaN count."""
    plb, O = gpu, oracle_mod
    ch, g = make_pair(plb, O, 32, 24, 16)
    u, v, w, _ = g.init_flow(11, 0.3)
    u[5, 7, 9] += 3.0
    ch.set_fields(u, v, w)
    d = ch.diagnostics()
    dv, ijk = g.max_div(u, v, w)
    cv, cijk = g.max_cfl(u, v, w)
    assert abs(d["div_max"] - dv) <= 1e-13 * dv and tuple(d["div_ijk"]) == ijk
    assert abs(d["cfl_max"] - cv) <= 1e-13 * cv and tuple(d["cfl_ijk"]) == cijk
    u[3, 4, 5] = np.nan
    ch.set_fields(u, v, w)
    assert ch.diagnostics()["nan_count"] >= 1


def test_full_size_step_invariants(gpu):
    """512x384x256 (the bench size), size-independent properties after 3
    steps: divergence at round-off, bulk velocity held at vel_force by forceVel,
    no NaN, deterministic rerun."""
    plb = gpu
    cfg = plb.ChannelConfig(nx=512, ny=384, nz=256, stretch_ratio=2.0, re_tau=1000.0)
    res = []
    for _ in range(2):
        ch = plb.Channel(cfg)
        ch.init_flow(11, 0.1)
        ch.step(3)
        d = ch.diagnostics()
        assert d["div_max"] < 1e-10 and d["nan_count"] == 0
        u = ch.get_field(0)
        res.append(u)
        ch.close()
    assert np.array_equal(res[0], res[1])
    # forceVel holds the dz-weighted bulk velocity (Mean_h) at vel_force = 1
    nz = 256
    zf = 0.5 * (1.0 + np.tanh((np.arange(nz + 1) / nz - 0.5) * 2.0) / np.tanh(1.0))
    dzf = 2.0 * np.diff(zf)
    u = res[0][1:-1, 1:-1, 1:-1]
    bulk = (u.mean(axis=(1, 2)) * dzf / 2.0).sum()
    assert abs(bulk - 1.0) < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("path", ["step", "phases"])
def test_convecting_frame_matches_oracle(gpu, oracle_mod, precision, path):
    """u_crf = 0.3: the convecting reference frame (transform2CRF,
    mod_calcVel.f90:26-50; the u_crf advection terms of :93, 115, 137; the u
    wall value -u_crf of imposeBCVel, mod_updateBound.f90:57-108).  "step"
    runs pl_channel_step (the fused RK kernels' u_crf specialisations at
    64x48x32); "phases" runs the separate RK1, RK2, calcRHS, Poisson and
    correction kernels.  FP64 against the oracle at 1e-12; mixed at 1e-7
    (FP32 stencils: 3 steps leave a few 1e-9)."""
    plb, O = gpu, oracle_mod
    nx, ny, nz, nsteps, u_crf = 64, 48, 32, 3, 0.3
    prec = plb.PL_FP64 if precision == "fp64" else plb.PL_MIXED
    cfg = plb.ChannelConfig(nx=nx, ny=ny, nz=nz, stretch_ratio=1.5, re_tau=180.0, u_crf=u_crf, precision=prec)
    ch = plb.Channel(cfg)
    ch.init_flow(42, 0.1)
    for _ in range(nsteps):
        if path == "step":
            ch.step(1)
        else:
            for ph in ("rk1", "rk2", "calc_rhs", "poisson", "correct_force"):
                ch.phase(ph)
    g = O.Grid(nx, ny, nz, stretch=1.5, re_tau=180.0, u_crf=u_crf)
    u, v, w, p = g.init_flow(42, 0.1)
    ppe = O.PPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global)
    u1, v1, w1 = g.zeros(), g.zeros(), g.zeros()
    for _ in range(nsteps):
        g.step(ppe, u, v, w, u1, v1, w1, p)
    gu, gv, gw, _ = ch.get_fields()
    errs = [rel(a, b) for a, b in ((gu, u), (gv, v), (gw, w))]
    print(f"u_crf {u_crf} {precision} {path}: max rel err u v w", errs)
    # the u wall ghosts hold 2*(-u_crf) - u(1): the frame velocity reached them
    assert np.abs(gu[0, 1:-1, 1:-1] + gu[1, 1:-1, 1:-1] + 2 * u_crf).max() < 1e-12
    assert max(errs) < (TOL64 if precision == "fp64" else 1e-7)
    ch.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nx,ny,nz", [(64, 48, 32), (192, 48, 24), (768, 16, 16)])
def test_step_matches_phases(gpu, precision, nx, ny, nz):
    """pl_channel_step fuses calcRHS into the Poisson solve's forward x
    transform; the phase entries run calcRHS and the solve as separate
    kernels.  FP64: the same numbers bit for bit.  Mixed: the FP64 plane
    sums of the (0,0) mode are summed in another order, so agreement to
    round-off."""
    plb = gpu
    prec = plb.PL_FP64 if precision == "fp64" else plb.PL_MIXED
    cfg = plb.ChannelConfig(nx=nx, ny=ny, nz=nz, stretch_ratio=1.5, re_tau=180.0, precision=prec)
    a, b = plb.Channel(cfg), plb.Channel(cfg)
    a.init_flow(5, 0.1)
    b.init_flow(5, 0.1)
    for _ in range(6):
        a.step(1)
        for ph in ("rk", "calc_rhs", "poisson", "correct_force"):
            b.phase(ph)
    da, db = a.diagnostics(), b.diagnostics()
    fa, fb = a.get_fields(), b.get_fields()
    if precision == "fp64":
        for x, y in zip(fa, fb):
            assert np.array_equal(x, y)
        assert da == db
    else:
        errs = [rel(x, y) for x, y in zip(fa[:3], fb[:3])]
        print("mixed step vs phases, max rel err u v w:", errs)
        assert max(errs) < 1e-11
    a.close()
    b.close()
