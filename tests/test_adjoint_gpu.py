"""GPU tests of the body-force forward step and the hand-written discrete
adjoint (pl_adjoint_ke_gradient), against the torch FP64 autograd reference
of the same step (adjoint_ref.py) and against central finite differences.

The torch.autograd.Function below exists only in this test harness: it
routes J(u0, v0, w0, f) through the library's forward sweep and its
backward through the library's adjoint."""
import numpy as np
import pytest
import torch

import adjoint_ref as A

pytestmark = pytest.mark.gpu


def _mesh_and_channel(plb, nx, ny, nz, stretch, re, dt, seed, noise):
    cfg = plb.ChannelConfig(nx=nx, ny=ny, nz=nz, stretch_ratio=stretch, re=re, dt=dt, precision=plb.PL_FP64)
    ch = plb.Channel(cfg)
    ch.init_flow(seed, noise)
    m = A.Mesh(nx, ny, nz, stretch=stretch, re=re, dt=dt)
    return m, ch


def _download(ch):
    nx, ny, nz = ch.cfg.nx, ch.cfg.ny, ch.cfg.nz
    x = np.zeros((3, nz + 2, ny, nx))
    ch.download_compact(x.ctypes.data)
    ch.synchronize()
    return x


def _upload(ch, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    ch.upload_compact(x.ctypes.data)
    ch.synchronize()


def _fill_bc(x):
    """wall fills of (3, nz+2, ny, nx) fields (u_crf = 0)"""
    x = x.copy()
    nz = x.shape[1] - 2
    x[0, 0], x[0, nz + 1] = -x[0, 1], -x[0, nz]
    x[1, 0], x[1, nz + 1] = -x[1, 1], -x[1, nz]
    x[2, 0] = x[2, nz] = x[2, nz + 1] = 0.0
    return x


def _relmax(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("grid", [(32, 24, 16), (24, 18, 12)])  # fused RK kernel / separate RK1, RK2 kernels
def test_body_force_step_matches_reference(gpu, grid):
    plb = gpu
    nx, ny, nz = grid
    m, ch = _mesh_and_channel(plb, nx, ny, nz, 1.8, 300.0, 1e-3, 3, 0.2)
    f = (0.7, -0.4, 0.3)
    ch.set_body_force(f)
    x0 = _download(ch)
    ch.step(3)
    ch.synchronize()
    got = _download(ch)
    u, v, w = (torch.tensor(q) for q in x0)
    for _ in range(3):
        u, v, w = A.step(m, u, v, w, f)
    K = slice(1, nz + 1)
    for q, ref in zip(got, (u, v, w)):
        assert _relmax(q[K], ref[K].numpy()) < 1e-11
    ch.close()


def test_adjoint_matches_autograd_reference(gpu):
    plb = gpu
    nx, ny, nz = 32, 24, 16
    m, ch = _mesh_and_channel(plb, nx, ny, nz, 1.8, 200.0, 1e-3, 5, 0.3)
    f = np.array([0.3, 0.1, -0.2])
    ch.set_body_force(f)
    x0 = _download(ch)
    g = [torch.zeros((nz + 2, ny, nx), dtype=torch.float64, device="cuda") for _ in range(3)]
    nsteps, every = 7, 3  # segments of 3, 3 and 1 steps
    J, gf = ch.adjoint_ke_gradient(nsteps, every, *(t.data_ptr() for t in g))
    torch.cuda.synchronize()
    # the fields are back at x0
    assert np.array_equal(_download(ch), x0)
    K = slice(1, nz + 1)
    Jr, gu, gv, gw, gfr = A.gradient(m, x0[0][K], x0[1][K], x0[2][K], f, nsteps)
    assert abs(J - Jr) <= 1e-12 * abs(Jr)
    got = [t.cpu().numpy() for t in g]
    print("adjoint vs autograd: J rel", abs(J - Jr) / abs(Jr), "grad rel max",
          [_relmax(got[c][K], r) for c, r in enumerate((gu, gv, gw))], "df rel", np.abs(gf - gfr).max() / np.abs(gfr).max())
    assert _relmax(got[0][K], gu) < 1e-9
    assert _relmax(got[1][K], gv) < 1e-9
    assert _relmax(got[2][K], gw) < 1e-9
    assert np.abs(gf - gfr).max() <= 1e-9 * np.abs(gfr).max()
    # ghost planes and the top wall of w carry no gradient
    assert not got[0][0].any() and not got[0][nz + 1].any() and not got[2][nz].any()
    ch.close()


class KineticEnergyAfterSteps(torch.autograd.Function):
    """J(u0, v0, w0, f): kinetic energy after `nsteps` library steps from the
    BC-filled fields (nz+2, ny, nx) with body force f. backward() returns the
    library's adjoint gradient."""

    @staticmethod
    def forward(ctx, u0, v0, w0, f, ch, nsteps, every):
        _upload(ch, torch.stack([u0, v0, w0]).detach().numpy())
        ch.set_body_force(f.detach().numpy())
        g = [torch.zeros(u0.shape, dtype=torch.float64, device="cuda") for _ in range(3)]
        J, gf = ch.adjoint_ke_gradient(nsteps, every, *(t.data_ptr() for t in g))
        ctx.save_for_backward(*(t.cpu() for t in g), torch.tensor(gf))
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        gu, gv, gw, gf = ctx.saved_tensors
        return gJ * gu, gJ * gv, gJ * gw, gJ * gf, None, None, None


def _direction(rng, x0, m):
    """a seeded direction: random multiples of the initial field, of a
    wall-normal profile and of a few low Fourier modes per component"""
    nx, ny, nz = m.nx, m.ny, m.nz
    xs = (np.arange(nx) + 0.5) * m.dx
    ys = (np.arange(ny) + 0.5) * m.dy
    zc = np.cumsum(np.r_[0.0, 0.5 * (m.dzf_np[:-1] + m.dzf_np[1:])]) - 0.5 * m.dzf_np[0]
    d = np.zeros_like(x0)
    for c in range(3):
        d[c] += rng.standard_normal() * x0[c]
        prof = np.sin(np.pi * rng.integers(1, 4) * zc / m.lz)
        d[c] += rng.standard_normal() * prof[:, None, None]
        for _ in range(3):
            kx, ky = rng.integers(0, 4), rng.integers(0, 4)
            ph, ps = rng.uniform(0, 2 * np.pi, 2)
            mode = np.cos(2 * np.pi * kx * xs / m.lx + ph)[None, None, :] * np.cos(2 * np.pi * ky * ys / m.ly + ps)[None, :, None]
            d[c] += rng.standard_normal() * mode * prof[:, None, None]
    return d, rng.standard_normal(3)


def test_adjoint_agrees_with_central_differences_256x192x128(gpu):
    """Gradient of the kinetic energy after 200 FP64 steps at 256x192x128
    (Re_tau 550, stretch 1.8, perturbation 0.05 from seed 7, Thomas PPE)
    w.r.t. the initial velocity and a uniform body force, checkpoint every
    20 steps; central differences with eps = 1e-6 on 16 seeded directions
    agree to 1e-6 relative."""
    plb = gpu
    nx, ny, nz = 256, 192, 128
    re = plb.re_from_retau(550.0)
    m, ch = _mesh_and_channel(plb, nx, ny, nz, 1.8, re, 1e-4, 7, 0.05)
    nsteps, every, eps = 200, 20, 1e-6
    x0 = _download(ch)
    f0 = np.zeros(3)
    xt = [torch.tensor(q, requires_grad=True) for q in x0]
    ft = torch.tensor(f0, requires_grad=True)
    J = KineticEnergyAfterSteps.apply(xt[0], xt[1], xt[2], ft, ch, nsteps, every)
    J.backward()
    grads = np.stack([t.grad.numpy() for t in xt])
    gf = ft.grad.numpy()

    def J_at(x, f):
        _upload(ch, _fill_bc(x))
        ch.set_body_force(f)
        ch.step(nsteps)
        return ch.kinetic_energy()

    rng = np.random.default_rng(2024)
    worst = 0.0
    for _ in range(16):
        d, df = _direction(rng, x0, m)
        fd = (J_at(x0 + eps * d, f0 + eps * df) - J_at(x0 - eps * d, f0 - eps * df)) / (2 * eps)
        ad = float((grads * d).sum() + (gf * df).sum())
        worst = max(worst, abs(ad - fd) / abs(fd))
        print(f"direction: fd {fd:.12e} adjoint {ad:.12e} rel {abs(ad - fd) / abs(fd):.3e}")
    print("J", float(J.detach()), "dJ/df", gf, "worst rel", worst)
    assert worst <= 1e-6, worst
    ch.close()


def test_adjoint_rejects_mixed_and_pdd(gpu):
    plb = gpu
    ch = plb.Channel(plb.ChannelConfig(nx=32, ny=24, nz=16, precision=plb.PL_MIXED))
    g = torch.zeros(3, dtype=torch.float64, device="cuda")
    with pytest.raises(plb.PowerLLELError, match="FP64 path"):
        ch.adjoint_ke_gradient(2, 1, g.data_ptr(), g.data_ptr(), g.data_ptr())
    with pytest.raises(plb.PowerLLELError, match="FP64 path only"):
        ch.set_body_force((1.0, 0.0, 0.0))
    ch.close()
    ch = plb.Channel(plb.ChannelConfig(nx=32, ny=24, nz=16, trid_parts=2))
    with pytest.raises(plb.PowerLLELError, match="Thomas"):
        ch.adjoint_ke_gradient(2, 1, g.data_ptr(), g.data_ptr(), g.data_ptr())
    ch.close()
