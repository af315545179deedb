"""CPU tests of the oracle itself: the restatement against the reference's own
build (golden fixtures and, when the reference tree is present, live runs),
against the published FFT definition, and against exact discrete identities."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN


def mm(a):
    return a - a.mean()


def test_fft_restatement_matches_definition(oracle_mod):
    """R2HC / HC2R of the FFTW manual, checked against numpy's rfft repacked
    into half-complex order (every length class the solver meets: 2^a, 3*2^a,
    odd, prime)."""
    import ctypes as C
    O = oracle_mod
    H = C.CDLL(O.LIB_PATH)
    H.hc_fft_plan_create.restype = C.c_void_p
    H.hc_fft_plan_create.argtypes = [C.c_int]
    H.hc_fft_plan_destroy.argtypes = [C.c_void_p]
    H.hc_fft_r2hc.argtypes = [C.c_void_p, O._dp, C.c_long]
    H.hc_fft_hc2r.argtypes = [C.c_void_p, O._dp, C.c_long]
    rng = np.random.default_rng(0)
    for n in [1, 2, 3, 4, 6, 8, 12, 16, 64, 96, 192, 384, 512, 768, 1024, 7, 15, 30]:
        x = rng.standard_normal(n)
        p = H.hc_fft_plan_create(n)
        y = x.copy()
        H.hc_fft_r2hc(p, O._ptr(y), 1)
        X = np.fft.rfft(x)
        hc = np.zeros(n)
        hc[: n // 2 + 1] = X.real
        for k in range(1, (n + 1) // 2):
            hc[n - k] = X[k].imag
        assert np.abs(y - hc).max() <= 1e-14 * max(1.0, np.abs(hc).max()), n
        z = y.copy()
        H.hc_fft_hc2r(p, O._ptr(z), 1)
        assert np.abs(z - n * x).max() <= 1e-14 * n * np.abs(x).max(), n
        H.hc_fft_plan_destroy(p)


GOLDEN_PPE = sorted(glob.glob(os.path.join(GOLDEN, "ppe_*.npz")))


@pytest.mark.parametrize("path", GOLDEN_PPE, ids=[os.path.basename(p)[:-4] for p in GOLDEN_PPE])
def test_oracle_ppe_bitexact_vs_reference_golden(oracle_mod, path):
    """The restated PPE reproduces the reference's own output bit for bit
    (same pivots, same FFT restatement, same operation order)."""
    O = oracle_mod
    d = np.load(path)
    nx, ny, nz = int(d["nx"]), int(d["ny"]), int(d["nz"])
    nparts = int(d["p_col"]) if int(d["pdd"]) else 0
    var = np.zeros((nz + 2, ny + 2, nx + 2))
    var[1:-1, 1:-1, 1:-1] = d["rhs"]
    s = O.PPE(nx, ny, nz, float(d["dx"]), float(d["dy"]), d["dzf"], nparts=nparts)
    s.execute(var)
    assert np.array_equal(var[1:-1, 1:-1, 1:-1], d["p"])


def _applyL(p, dx, dy, dzf):
    """The discrete operator the PPE inverts: periodic second differences in x,
    y; in z the staggered operator with zero-gradient walls."""
    nz, ny, nx = p.shape
    P = np.zeros((nz + 2, ny + 2, nx + 2))
    P[1:-1, 1:-1, 1:-1] = p
    P[:, :, 0], P[:, :, -1] = P[:, :, -2], P[:, :, 1]
    P[:, 0, :], P[:, -1, :] = P[:, -2, :], P[:, 1, :]
    P[0], P[-1] = P[1], P[-2]
    c = P[1:-1, 1:-1, 1:-1]
    lap = (P[1:-1, 1:-1, 2:] - 2 * c + P[1:-1, 1:-1, :-2]) / dx ** 2 + (P[1:-1, 2:, 1:-1] - 2 * c + P[1:-1, :-2, 1:-1]) / dy ** 2
    for k in range(1, nz + 1):
        dzc_p = 0.5 * (dzf[k] + dzf[k + 1])
        dzc_m = 0.5 * (dzf[k - 1] + dzf[k])
        lap[k - 1] += ((P[k + 1] - P[k])[1:-1, 1:-1] / dzc_p - (P[k] - P[k - 1])[1:-1, 1:-1] / dzc_m) / dzf[k]
    return lap


@pytest.mark.parametrize("path", [p for p in GOLDEN_PPE if "thomas" in p or "pdd1" in p],
                         ids=lambda p: os.path.basename(p)[:-4])
def test_reference_ppe_solves_poisson(path):
    """Thomas (and PDD with one partition) invert the discrete operator to
    round-off: pins the golden vectors as solutions, independently of any
    implementation."""
    d = np.load(path)
    p = d["p"]
    res = _applyL(p, float(d["dx"]), float(d["dy"]), d["dzf"]) - d["rhs"]
    assert np.abs(res).max() < 1e-11 * max(1.0, np.abs(d["rhs"]).max())


def test_pdd_one_partition_equals_thomas(oracle_mod):
    """PDD with P = 1 is Thomas bit for bit (both spikes vanish at the walls)."""
    O = oracle_mod
    g = O.Grid(32, 24, 16, stretch=1.8)
    rng = np.random.default_rng(5)
    var = np.zeros(g.shape)
    var[1:-1, 1:-1, 1:-1] = rng.standard_normal((16, 24, 32))
    a, b = var.copy(), var.copy()
    O.PPE(32, 24, 16, g.g.dx, g.g.dy, g.dzf_global, nparts=0).execute(a)
    O.PPE(32, 24, 16, g.g.dx, g.g.dy, g.dzf_global, nparts=1).execute(b)
    assert np.array_equal(a, b)


def test_pdd_truncation_depends_on_partitions(oracle_mod):
    """PDD truncates the reduced system: accurate for high wavenumbers, not for
    the (0,0) family; the result depends on P, so P must match the reference."""
    d = np.load(os.path.join(GOLDEN, "ppe_pdd4_32x24x32.npz"))
    d2 = np.load(os.path.join(GOLDEN, "ppe_pdd2_32x24x32.npz"))
    assert not np.allclose(mm(d["p"]), mm(d2["p"]), rtol=0, atol=1e-6)


def test_step_oracle_matches_golden(oracle_mod):
    """Init + 5 steps of the restated step with the restated PPE reproduce the
    fixture made with the reference PPE, bit for bit."""
    O = oracle_mod
    d = np.load(os.path.join(GOLDEN, "step_32x24x16_5.npz"))
    nx, ny, nz = int(d["nx"]), int(d["ny"]), int(d["nz"])
    g = O.Grid(nx, ny, nz, stretch=float(d["stretch"]), re=float(d["re"]), dt=float(d["dt"]))
    u, v, w, p = g.init_flow(int(d["seed"]), float(d["noise"]))
    assert np.array_equal(u, d["u0"]) and np.array_equal(v, d["v0"]) and np.array_equal(w, d["w0"])
    ppe = O.PPE(nx, ny, nz, g.g.dx, g.g.dy, g.dzf_global)
    u1, v1, w1 = g.zeros(), g.zeros(), g.zeros()
    for _ in range(int(d["nsteps"])):
        g.step(ppe, u, v, w, u1, v1, w1, p)
    assert np.array_equal(u, d["u"]) and np.array_equal(v, d["v"]) and np.array_equal(w, d["w"])
    assert g.max_div(u, v, w)[0] < 1e-12


def test_projection_identity(oracle_mod):
    """div(grad p) on the MAC grid is exactly the operator the PPE inverts, so
    correctVel(PPE(calcRHS(u))) leaves a divergence of round-off size even for a
    strongly divergent random field (the reference's div_limit is 1e-9)."""
    O = oracle_mod
    g = O.Grid(32, 24, 16, stretch=1.5)
    u, v, w, p = g.init_flow(3, 0.5)
    assert g.max_div(u, v, w)[0] > 1.0
    g.calc_rhs(u, v, w, p)
    O.PPE(32, 24, 16, g.g.dx, g.g.dy, g.dzf_global).execute(p)
    g.bound_p(p)
    g.correct_vel(p, u, v, w)
    g.bound_vel(u, v, w)
    assert g.max_div(u, v, w)[0] < 1e-11


def test_stencil_consistency(oracle_mod):
    """Manufactured smooth fields: the restated RK1 increment converges at
    second order to dt*(nu*lap(u) - div(u u)) on a uniform mesh."""
    O = oracle_mod
    errs = []
    for n in (16, 32):
        g = O.Grid(n, n, n, lx=2 * np.pi, ly=2 * np.pi, lz=2 * np.pi, mesh_type=0, stretch=0.0, re=1.0,
                   dt=1.0, is_forced=(0, 0, 0))
        h = 2 * np.pi / n
        xc = (np.arange(n) + 0.5) * h
        xf = (np.arange(n) + 1.0) * h
        Z, Y, X = np.meshgrid(xc, xc, xf, indexing="ij")  # u at x-faces
        u = np.zeros(g.shape)
        v = np.zeros(g.shape)
        w = np.zeros(g.shape)
        u[1:-1, 1:-1, 1:-1] = np.sin(X) * np.cos(Y)
        g.bound_vel(u, v, w)
        # walls make the z direction non-periodic: compare away from them
        u1, _, _ = g.rk1(u, v, w)
        du = (u1 - u)[1:-1, 1:-1, 1:-1]
        # exact: nu*lap(u) - d(uu)/dx - d(uv)/dy with v = w = 0 (z-uniform)
        exact = -2 * np.sin(X) * np.cos(Y) - 2 * np.sin(X) * np.cos(X) * np.cos(Y) ** 2
        sl = slice(2, -2)
        errs.append(np.abs(du[sl] - exact[sl]).max())
    assert errs[1] < errs[0] / 3.5, errs
