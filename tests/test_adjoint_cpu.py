"""CPU checks of the discrete-adjoint reference and of the hand-derived
transposed momentum stencil that the CUDA adjoint kernel evaluates."""
import numpy as np
import pytest
import torch

import adjoint_ref as A


def _state(m, rng, amp=1.0):
    u0 = torch.tensor(1.0 + amp * rng.standard_normal((m.nz, m.ny, m.nx)))
    v0 = torch.tensor(amp * rng.standard_normal((m.nz, m.ny, m.nx)))
    w0 = torch.tensor(amp * rng.standard_normal((m.nz, m.ny, m.nx)))
    return A.state_from_interior(m, u0, v0, w0)


def _adjoint_field(m, rng, wlast_zero=True):
    z = lambda: torch.zeros((1, m.ny, m.nx), dtype=A.DT)
    f = [torch.cat([z(), torch.tensor(rng.standard_normal((m.nz, m.ny, m.nx))), z()], 0) for _ in range(3)]
    if wlast_zero:
        f[2][m.nz] = 0.0
    return f


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("u_crf", [0.0, 0.3])
def test_transposed_rhs_matches_autograd(u_crf):
    rng = np.random.default_rng(3)
    m = A.Mesh(8, 6, 6, stretch=1.8, re=50.0, u_crf=u_crf)
    u, v, w = _state(m, rng)
    r = _adjoint_field(m, rng)
    K = slice(1, m.nz + 1)
    xi = [q[K].clone().requires_grad_(True) for q in (u, v, w)]
    ug, vg, wg = A.state_from_interior(m, *xi)
    ru, rv, rw = A.rhs(m, ug, vg, wg)
    (ru * r[0][K] + rv * r[1][K] + rw * r[2][K]).sum().backward()
    su, sv, sw = A.transposed_rhs(m, u, v, w, *r)
    assert _rel(su, xi[0].grad) < 1e-12
    assert _rel(sv, xi[1].grad) < 1e-12
    gw = xi[2].grad.clone()
    gw[m.nz - 1] = 0.0  # level nz of w is a wall face, not a degree of freedom
    assert _rel(sw, gw) < 1e-12


def test_adjoint_step_matches_autograd():
    rng = np.random.default_rng(5)
    m = A.Mesh(8, 6, 8, stretch=1.8, re=30.0, dt=2e-3)
    f = (0.3, -0.2, 0.1)
    u, v, w = _state(m, rng, 0.3)
    xbar = _adjoint_field(m, rng)
    K = slice(1, m.nz + 1)
    xi = [q[K].clone().requires_grad_(True) for q in (u, v, w)]
    ft = torch.tensor(f, dtype=A.DT, requires_grad=True)
    out = A.step(m, *A.state_from_interior(m, *xi), ft)
    sum((o[K] * b[K]).sum() for o, b in zip(out, xbar)).backward()
    X, fbar = A.adjoint_step(m, (u, v, w), xbar, f)
    assert _rel(X[0][K], xi[0].grad) < 1e-10
    assert _rel(X[1][K], xi[1].grad) < 1e-10
    gw = xi[2].grad.clone()
    gw[m.nz - 1] = 0.0
    assert _rel(X[2][K], gw) < 1e-10
    assert _rel(fbar, ft.grad) < 1e-10


def test_reference_gradient_matches_central_differences():
    rng = np.random.default_rng(7)
    m = A.Mesh(8, 6, 6, stretch=1.5, re=40.0, dt=2e-3)
    nsteps = 3
    u0 = 1.0 + 0.2 * rng.standard_normal((m.nz, m.ny, m.nx))
    v0 = 0.2 * rng.standard_normal((m.nz, m.ny, m.nx))
    w0 = 0.2 * rng.standard_normal((m.nz, m.ny, m.nx))
    f = np.array([0.5, 0.2, -0.1])
    J, gu, gv, gw, gf = A.gradient(m, u0, v0, w0, f, nsteps)
    eps = 1e-6
    for d in range(3):
        du, dv, dw = (rng.standard_normal(u0.shape) for _ in range(3))
        df = rng.standard_normal(3)
        Jp = A.objective(m, *(torch.tensor(a + eps * b) for a, b in ((u0, du), (v0, dv), (w0, dw))),
                         torch.tensor(f + eps * df), nsteps)
        Jm = A.objective(m, *(torch.tensor(a - eps * b) for a, b in ((u0, du), (v0, dv), (w0, dw))),
                         torch.tensor(f - eps * df), nsteps)
        fd = float(Jp - Jm) / (2 * eps)
        ad = float((gu * du).sum() + (gv * dv).sum() + (gw * dw).sum() + (gf * df).sum())
        assert abs(fd - ad) <= 1e-6 * abs(fd), (d, fd, ad)
