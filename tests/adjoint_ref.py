"""FP64 discrete-adjoint reference of the RK2 projection step (test code).

The forward map is one step of the channel solver: the RK1/RK2 momentum
stencils (src/mod_calcVel.f90:52-426), the wall and periodic fills
(src/mod_updateBound.f90:57-108, 274-330), calcRHS (src/mod_calcRHS.f90:11-36),
the PPE (src/src_c/mod_poisson_solver.c), correctVel and forceVel
(src/mod_calcVel.f90:428-509). It is written with torch FP64 tensor
operations, so torch.autograd gives its exact discrete adjoint (reverse-mode
differentiation of the same arithmetic).

It differs from the library's forward in one place only: the PPE's linear
system is solved with torch FFTs and a dense solve per wavenumber pair, and
the (0,0) mode is gauged by p(nz) = 0. The reference leaves that constant to
round-off. u, v, w are unchanged up to rounding, because correctVel uses only
pressure differences.

A uniform body force f = (fx, fy, fz) is added to the momentum right-hand
side of both RK stages: u1 = u + dt (RHS(u) + f), and
u = (u1 + dt (RHS(u1) + f) + u) / 2. The reference has no body force. forceVel
stays on: it shifts u by vel_force - Mean_h(u) after the projection.

Objective: J = 1/2 dx dy [ sum_{k=1..nz} dzf_k sum_ij (u^2 + v^2)
                         + sum_{k=1..nz-1} dzc_k sum_ij w^2 ].
This is the kinetic energy integrated over the staggered cells.

Layout: every field is a (nz+2, ny, nx) tensor [k][j][i]. k = 0 and nz+1 are
the wall ghost planes. x and y are periodic through index wrap (torch.roll),
as in the library's device layout.

``transposed_rhs`` restates, with whole-array operations, the hand-derived
transposed momentum stencil that the CUDA adjoint kernel evaluates point by
point. It is checked here against autograd on the CPU.
"""
from __future__ import annotations

import math

import numpy as np
import torch

DT = torch.float64


class Mesh:
    """Grid and run parameters (mod_mesh.f90:26-84, tanh stretching :120-162)."""

    def __init__(self, nx, ny, nz, lx=2 * math.pi, ly=math.pi, lz=2.0, stretch=1.5, re=1000.0, dt=1e-4,
                 u_crf=0.0, vel_force=1.0, forced=True):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.lx, self.ly, self.lz = lx, ly, lz
        self.dx, self.dy = lx / nx, ly / ny
        self.dxi, self.dyi = 1.0 / self.dx, 1.0 / self.dy
        self.re_inv = 1.0 / re
        self.dt, self.u_crf = dt, u_crf
        self.vel_force, self.forced = vel_force, forced
        dzf = np.zeros(nz + 2)
        if stretch == 0.0:
            dzf[:] = lz / nz
        else:
            zf = np.zeros(nz + 1)
            for k in range(1, nz + 1):
                zf[k] = 0.5 * (1.0 + math.tanh((k / nz - 0.5) * stretch) / math.tanh(stretch / 2.0))
            dzf[1:nz + 1] = lz * np.diff(zf)
            dzf[0], dzf[nz + 1] = dzf[1], dzf[nz]
        dzc = np.zeros(nz + 2)
        dzc[:nz + 1] = 0.5 * (dzf[:nz + 1] + dzf[1:])
        dzc[nz + 1] = dzc[nz]
        self.dzf_np, self.dzc_np = dzf, dzc
        t = lambda a: torch.tensor(a, dtype=DT)[:, None, None]
        self.dzf, self.dzc = t(dzf), t(dzc)
        self.dzf_inv, self.dzc_inv = t(1.0 / dzf), t(1.0 / dzc)
        self.dzflzi = t(dzf / lz)


def xp(a):
    return torch.roll(a, -1, dims=2)


def xm(a):
    return torch.roll(a, 1, dims=2)


def yp(a):
    return torch.roll(a, -1, dims=1)


def ym(a):
    return torch.roll(a, 1, dims=1)


def fill_bc(m: Mesh, u, v, w):
    """imposeNoSlipBC on the wall planes (x, y periodic by wrap)."""
    nz = m.nz
    bc = 0.0 - m.u_crf
    u = torch.cat([2 * bc - u[1:2], u[1:nz + 1], 2 * bc - u[nz:nz + 1]], 0)
    v = torch.cat([-v[1:2], v[1:nz + 1], -v[nz:nz + 1]], 0)
    z = torch.zeros_like(w[0:1])
    w = torch.cat([z, w[1:nz], z, z], 0)
    return u, v, w


def with_interior(m: Mesh, full, interior):
    return torch.cat([full[0:1], interior, full[m.nz + 1:]], 0)


def rhs(m: Mesh, u, v, w):
    """(visc - conv) of the three momentum equations on levels 1..nz
    (timeIntVelRK1_kernel, mod_calcVel.f90:74-138)."""
    nz = m.nz
    K, Kp, Km = slice(1, nz + 1), slice(2, nz + 2), slice(0, nz)
    dxi, dyi, re_inv, u_crf = m.dxi, m.dyi, m.re_inv, m.u_crf
    f_k, f_kp, f_km = m.dzf[K], m.dzf[Kp], m.dzf[Km]
    ci_k, ci_km = m.dzc_inv[K], m.dzc_inv[Km]
    fi_k, fi_kp = m.dzf_inv[K], m.dzf_inv[Kp]
    U, V, W = u[K], v[K], w[K]
    Ukp, Ukm, Vkp, Vkm, Wkm = u[Kp], u[Km], v[Kp], v[Km], w[Km]

    ue, uw = U + xp(U), xm(U) + U
    un, us = U + yp(U), ym(U) + U
    ut = (U * f_kp + Ukp * f_k) * ci_k
    ub = (U * f_km + Ukm * f_k) * ci_km
    vn, vs = V + xp(V), ym(V) + xp(ym(V))
    wt, wb = W + xp(W), Wkm + xp(Wkm)
    conv = 0.25 * ((ue * ue - uw * uw) * dxi + (un * vn - us * vs) * dyi + (ut * wt - ub * wb) * fi_k)
    conv = conv + 0.5 * u_crf * (ue - uw) * dxi
    visc = (((xp(U) - U) * dxi - (U - xm(U)) * dxi) * dxi + ((yp(U) - U) * dyi - (U - ym(U)) * dyi) * dyi +
            ((Ukp - U) * ci_k - (U - Ukm) * ci_km) * fi_k) * re_inv
    ru = visc - conv

    ve, vw = V + xp(V), xm(V) + V
    vn, vs = V + yp(V), ym(V) + V
    vt = (V * f_kp + Vkp * f_k) * ci_k
    vb = (V * f_km + Vkm * f_k) * ci_km
    ue, uw = U + yp(U), xm(U) + xm(yp(U))
    wt, wb = W + yp(W), Wkm + yp(Wkm)
    conv = 0.25 * ((ue * ve - uw * vw) * dxi + (vn * vn - vs * vs) * dyi + (wt * vt - wb * vb) * fi_k)
    conv = conv + 0.5 * u_crf * (ve - vw) * dxi
    visc = (((xp(V) - V) * dxi - (V - xm(V)) * dxi) * dxi + ((yp(V) - V) * dyi - (V - ym(V)) * dyi) * dyi +
            ((Vkp - V) * ci_k - (V - Vkm) * ci_km) * fi_k) * re_inv
    rv = visc - conv

    Wkp = w[Kp]
    we, ww = W + xp(W), xm(W) + W
    wn, ws = W + yp(W), ym(W) + W
    wt, wb = W + Wkp, W + Wkm
    ue = (U * f_kp + Ukp * f_k) * ci_k
    uw = xm(ue)
    vn = (V * f_kp + Vkp * f_k) * ci_k
    vs = ym(vn)
    conv = 0.25 * ((ue * we - uw * ww) * dxi + (vn * wn - vs * ws) * dyi + (wt * wt - wb * wb) * ci_k)
    conv = conv + 0.5 * u_crf * (we - ww) * dxi
    visc = (((xp(W) - W) * dxi - (W - xm(W)) * dxi) * dxi + ((yp(W) - W) * dyi - (W - ym(W)) * dyi) * dyi +
            ((Wkp - W) * fi_kp - (W - Wkm) * fi_k) * ci_k) * re_inv
    rw = visc - conv
    return ru, rv, rw


def trid_coeffs(m: Mesh):
    """set_trid_coeff (mod_poisson_solver.c:40-103), Neumann at both walls."""
    nz, dzf = m.nz, m.dzf_np
    a = np.array([2.0 / (dzf[k] * (dzf[k - 1] + dzf[k])) for k in range(1, nz + 1)])
    c = np.array([2.0 / (dzf[k] * (dzf[k + 1] + dzf[k])) for k in range(1, nz + 1)])
    b = -a - c
    b[0] += a[0]
    a[0] = 0.0
    b[-1] += c[-1]
    c[-1] = 0.0
    return a, b, c


def ppe(m: Mesh, r):
    """Solve L p = r (r: (nz, ny, nx)) for the discrete Poisson operator of
    the PPE; the (0,0) mode is gauged by p(nz) = 0."""
    nx, ny, nz = m.nx, m.ny, m.nz
    nxh = nx // 2 + 1
    R = torch.fft.fft(torch.fft.rfft(r, dim=2), dim=1)  # (nz, ny, nxh)
    lx = 2.0 * (np.cos(2 * np.pi * np.arange(nxh) / nx) - 1.0) * m.dxi ** 2
    ly = 2.0 * (np.cos(2 * np.pi * np.arange(ny) / ny) - 1.0) * m.dyi ** 2
    a, b, c = trid_coeffs(m)
    A = np.zeros((ny, nxh, nz, nz))
    idx = np.arange(nz)
    A[:, :, idx, idx] = b[None, None, :] + (ly[:, None] + lx[None, :])[:, :, None]
    A[:, :, idx[1:], idx[:-1]] = a[1:]
    A[:, :, idx[:-1], idx[1:]] = c[:-1]
    A[0, 0, nz - 1, :] = 0.0
    A[0, 0, nz - 1, nz - 1] = 1.0
    mask = torch.ones((nz, ny, nxh), dtype=DT)
    mask[nz - 1, 0, 0] = 0.0
    R = R * mask
    At = torch.tensor(A, dtype=torch.complex128)
    X = torch.linalg.solve(At, R.permute(1, 2, 0).unsqueeze(-1)).squeeze(-1).permute(2, 0, 1)
    return torch.fft.irfft(torch.fft.ifft(X, dim=1), n=nx, dim=2)


def step(m: Mesh, u, v, w, f=(0.0, 0.0, 0.0)):
    """One RK2 projection step (main.f90:137-208) on BC-filled fields."""
    nz, dt = m.nz, m.dt
    K, Kp, Km = slice(1, nz + 1), slice(2, nz + 2), slice(0, nz)
    ru, rv, rw = rhs(m, u, v, w)
    u1, v1, w1 = fill_bc(m, with_interior(m, u, u[K] + dt * (ru + f[0])), with_interior(m, v, v[K] + dt * (rv + f[1])),
                         with_interior(m, w, w[K] + dt * (rw + f[2])))
    ru, rv, rw = rhs(m, u1, v1, w1)
    u2 = with_interior(m, u, (u1[K] + dt * (ru + f[0]) + u[K]) * 0.5)
    v2 = with_interior(m, v, (v1[K] + dt * (rv + f[1]) + v[K]) * 0.5)
    w2 = with_interior(m, w, (w1[K] + dt * (rw + f[2]) + w[K]) * 0.5)
    u2, v2, w2 = fill_bc(m, u2, v2, w2)
    dti = 1.0 / dt
    r = ((u2[K] - xm(u2[K])) * (dti * m.dxi) + (v2[K] - ym(v2[K])) * (dti * m.dyi) +
         (w2[K] - w2[Km]) * dti * m.dzf_inv[K])
    p = ppe(m, r)
    pg = torch.cat([p[0:1], p, p[nz - 1:nz]], 0)
    u3 = u2[K] - (xp(pg[K]) - pg[K]) * (dt * m.dxi)
    v3 = v2[K] - (yp(pg[K]) - pg[K]) * (dt * m.dyi)
    w3 = w2[K] - (pg[Kp] - pg[K]) * dt * m.dzc_inv[K]
    if m.forced:
        mean = (u3 * m.dzflzi[K]).sum() / m.nx / m.ny
        u3 = u3 + (m.vel_force - mean)
    return fill_bc(m, with_interior(m, u2, u3), with_interior(m, v2, v3), with_interior(m, w2, w3))


def kinetic_energy(m: Mesh, u, v, w):
    nz = m.nz
    K = slice(1, nz + 1)
    s = (m.dzf[K] * (u[K] ** 2 + v[K] ** 2)).sum() + (m.dzc[1:nz] * w[1:nz] ** 2).sum()
    return 0.5 * m.dx * m.dy * s


def state_from_interior(m: Mesh, u0, v0, w0):
    """Ghosted, BC-filled fields from (nz, ny, nx) interior arrays; w0's
    level nz (a wall face) is overwritten by zero."""
    z = torch.zeros_like(u0[0:1])
    g = lambda a: torch.cat([z, a, z], 0)
    return fill_bc(m, g(u0), g(v0), g(w0))


def objective(m: Mesh, u0, v0, w0, f, nsteps):
    u, v, w = state_from_interior(m, u0, v0, w0)
    for _ in range(nsteps):
        u, v, w = step(m, u, v, w, f)
    return kinetic_energy(m, u, v, w)


def gradient(m: Mesh, u0, v0, w0, f, nsteps):
    """(J, dJ/du0, dJ/dv0, dJ/dw0, dJ/df) by reverse-mode AD; the field
    gradients are (nz, ny, nx) arrays over the interior."""
    x = [torch.tensor(np.asarray(a), dtype=DT, requires_grad=True) for a in (u0, v0, w0)]
    ft = torch.tensor(np.asarray(f, dtype=np.float64), dtype=DT, requires_grad=True)
    J = objective(m, x[0], x[1], x[2], ft, nsteps)
    J.backward()
    return float(J.detach()), x[0].grad.numpy(), x[1].grad.numpy(), x[2].grad.numpy(), ft.grad.numpy()


# ----------------------------------------------------------------------------
# Hand-derived transposed momentum stencil (what the CUDA adjoint kernel does)
# ----------------------------------------------------------------------------
def transposed_rhs(m: Mesh, u, v, w, au, av, aw):
    """S = E^T J_R(u,v,w)^T (au, av, aw): the transposed Jacobian of the
    momentum right-hand side, wall fills included, applied to the adjoint
    fields (same layout; ghost planes and aw's level nz hold zero). Returns
    the interior levels 1..nz; sw's level nz is zero.

    The convective terms are written as face fluxes shared by two equations:
    Pxy = (u(o) + u(o+j)) (v(o) + v(o+i)) is the y flux of u and the x flux of
    v. Pxz = ut wt is the z flux of u and the x flux of w. Pyz = vt wn is the
    z flux of v and the y flux of w. The diagonal fluxes are (u(o) + u(o+i))^2,
    (v(o) + v(o+j))^2 and (w(o) + w(o+k))^2. The adjoint of a flux difference
    -0.25 (F(o) - F(o-1)) h_o is Fbar(o) = -0.25 (h_o r(o) - h_{o+1} r(o+1)).
    """
    nz = m.nz
    dxi, dyi, re_inv, u_crf = m.dxi, m.dyi, m.re_inv, m.u_crf
    f, ci, fi = m.dzf, m.dzc_inv, m.dzf_inv
    # level-shifted views over the interior levels 1..nz ("c") and the levels
    # 0..nz-1 ("m", the plane below)
    L = lambda a, s: a[1 + s:nz + 1 + s]
    U, V, W = L(u, 0), L(v, 0), L(w, 0)
    Um, Vm, Wm = L(u, -1), L(v, -1), L(w, -1)
    Up, Vp, Wp = L(u, 1), L(v, 1), L(w, 1)
    RU, RV, RW = L(au, 0), L(av, 0), L(aw, 0)
    RUp, RVp, RWp = L(au, 1), L(av, 1), L(aw, 1)
    RUm, RVm, RWm = L(au, -1), L(av, -1), L(aw, -1)
    f_c, f_p, f_m = L(f, 0), L(f, 1), L(f, -1)
    ci_c, ci_m, ci_p = L(ci, 0), L(ci, -1), L(ci, 1)
    fi_c, fi_p, fi_m = L(fi, 0), L(fi, 1), L(fi, -1)

    # flux adjoints at the faces of cell o (level c) and of the plane below
    # (level m, i.e. o - k)
    Au_x = -0.25 * dxi * (RU - xp(RU))
    Av_y = -0.25 * dyi * (RV - yp(RV))
    Au_y = -0.25 * dyi * (RU - yp(RU))
    Av_x = -0.25 * dxi * (RV - xp(RV))
    Aw_x = -0.25 * dxi * (RW - xp(RW))
    Aw_y = -0.25 * dyi * (RW - yp(RW))
    Au_z = -0.25 * (RU * fi_c - RUp * fi_p)
    Av_z = -0.25 * (RV * fi_c - RVp * fi_p)
    Aw_z = -0.25 * (RW * ci_c - RWp * ci_p)
    Aw_x_m = -0.25 * dxi * (RWm - xp(RWm))
    Aw_y_m = -0.25 * dyi * (RWm - yp(RWm))
    Au_z_m = -0.25 * (RUm * fi_m - RU * fi_c)
    Av_z_m = -0.25 * (RVm * fi_m - RV * fi_c)
    Aw_z_m = -0.25 * (RWm * ci_m - RW * ci_c)
    Pxy = Au_y + Av_x
    Pxz = Au_z + Aw_x
    Pyz = Av_z + Aw_y
    Pxz_m = Au_z_m + Aw_x_m
    Pyz_m = Av_z_m + Aw_y_m

    # base-state interpolants
    ue = U + xp(U)
    un = U + yp(U)
    vn = V + xp(V)
    vnv = V + yp(V)
    wt = W + xp(W)
    wn = W + yp(W)
    wtw = W + Wp
    wtw_m = Wm + W
    ut = (U * f_p + Up * f_c) * ci_c
    vt = (V * f_p + Vp * f_c) * ci_c
    wt_m = Wm + xp(Wm)
    wn_m = Wm + yp(Wm)

    su = (2 * ue * Au_x + 2 * xm(ue) * xm(Au_x) + vn * Pxy + ym(vn) * ym(Pxy) +
          f_p * ci_c * wt * Pxz + f_m * ci_m * wt_m * Pxz_m)
    sv = (2 * vnv * Av_y + 2 * ym(vnv) * ym(Av_y) + un * Pxy + xm(un) * xm(Pxy) +
          f_p * ci_c * wn * Pyz + f_m * ci_m * wn_m * Pyz_m)
    sw = (2 * wtw * Aw_z + 2 * wtw_m * Aw_z_m + ut * Pxz + xm(ut) * xm(Pxz) + vt * Pyz + ym(vt) * ym(Pyz))

    # u_crf advection, adjoint of -0.5 u_crf (q(i+1) - q(i-1)) dx_inv
    su = su - 0.5 * u_crf * dxi * (xm(RU) - xp(RU))
    sv = sv - 0.5 * u_crf * dxi * (xm(RV) - xp(RV))
    sw = sw - 0.5 * u_crf * dxi * (xm(RW) - xp(RW))

    # viscous terms: x, y symmetric; z through the face fluxes, with the
    # wall-ghost chain (q(0) = 2bc - q(1), q(nz+1) = 2bc - q(nz)) doubling
    # the wall face coefficients of u and v
    lap = lambda R: (xp(R) - 2 * R + xm(R)) * dxi * dxi + (yp(R) - 2 * R + ym(R)) * dyi * dyi
    kk = torch.arange(1, nz + 1)[:, None, None]
    cb = torch.where(kk == nz, 2.0, 1.0).to(DT)
    ca = torch.where(kk == 1, 2.0, 1.0).to(DT)
    Vb_u = re_inv * (RU * fi_c - RUp * fi_p)
    Vb_u_m = re_inv * (RUm * fi_m - RU * fi_c)
    Vb_v = re_inv * (RV * fi_c - RVp * fi_p)
    Vb_v_m = re_inv * (RVm * fi_m - RV * fi_c)
    Vb_w = re_inv * (RW * ci_c - RWp * ci_p)
    Vb_w_m = re_inv * (RWm * ci_m - RW * ci_c)
    su = su + re_inv * lap(RU) - cb * ci_c * Vb_u + ca * ci_m * Vb_u_m
    sv = sv + re_inv * lap(RV) - cb * ci_c * Vb_v + ca * ci_m * Vb_v_m
    sw = sw + re_inv * lap(RW) - fi_p * Vb_w + fi_c * Vb_w_m
    sw = torch.cat([sw[:nz - 1], torch.zeros_like(sw[nz - 1:])], 0)
    return su, sv, sw


def adjoint_step(m: Mesh, x, xbar, f=(0.0, 0.0, 0.0)):
    """Reverse of one step at base state x = (u, v, w) (BC-filled): given the
    adjoint of the step's output (interior levels 1..nz, ghosted layout with
    zero ghost planes), return (adjoint of x, adjoint of f). Composition the
    CUDA adjoint follows: forceVel^T, W P W^-1 (the projection in the
    dz-weighted inner product), RK2^T, RK1^T."""
    nz, dt = m.nz, m.dt
    K = slice(1, nz + 1)
    z = lambda a: with_interior(m, torch.zeros_like(a), a[K])
    u, v, w = x
    # stage-1 field
    ru, rv, rw = rhs(m, u, v, w)
    y1 = fill_bc(m, with_interior(m, u, u[K] + dt * (ru + f[0])), with_interior(m, v, v[K] + dt * (rv + f[1])),
                 with_interior(m, w, w[K] + dt * (rw + f[2])))
    au, av, aw = xbar
    if m.forced:
        S = au[K].sum()
        au = with_interior(m, au, au[K] - m.dzflzi[K] / (m.nx * m.ny) * S)
    # projection adjoint: scale by 1/W, project, scale by W
    wu = m.dzf[K]
    ww = m.dzc[K].clone()
    ww[nz - 1] = 1.0
    zu, zv, zw = au[K] / wu, av[K] / wu, aw[K] / ww
    zw = torch.cat([zw[:nz - 1], torch.zeros_like(zw[nz - 1:])], 0)
    Z = [with_interior(m, torch.zeros_like(au), q) for q in (zu, zv, zw)]
    dti = 1.0 / dt
    r = ((Z[0][K] - xm(Z[0][K])) * (dti * m.dxi) + (Z[1][K] - ym(Z[1][K])) * (dti * m.dyi) +
         (Z[2][K] - Z[2][0:nz]) * dti * m.dzf_inv[K])
    p = ppe(m, r)
    pg = torch.cat([p[0:1], p, p[nz - 1:nz]], 0)
    b2u = (Z[0][K] - (xp(pg[K]) - pg[K]) * (dt * m.dxi)) * wu
    b2v = (Z[1][K] - (yp(pg[K]) - pg[K]) * (dt * m.dyi)) * wu
    b2w = (Z[2][K] - (pg[2:nz + 2] - pg[K]) * dt * m.dzc_inv[K]) * ww
    b2w = torch.cat([b2w[:nz - 1], torch.zeros_like(b2w[nz - 1:])], 0)
    B2 = [with_interior(m, torch.zeros_like(au), q) for q in (b2u, b2v, b2w)]
    fbar = 0.5 * dt * torch.stack([q[K].sum() for q in B2])
    # RK2^T: y2 = (y1 + dt (R(y1) + f) + x) / 2
    s = transposed_rhs(m, *y1, *B2)
    B1 = [with_interior(m, torch.zeros_like(au), 0.5 * q[K] + 0.5 * dt * sq) for q, sq in zip(B2, s)]
    fbar = fbar + dt * torch.stack([q[K].sum() for q in B1])
    # RK1^T: y1 = x + dt (R(x) + f)
    s = transposed_rhs(m, u, v, w, *B1)
    X = [with_interior(m, torch.zeros_like(au), 0.5 * q2[K] + q1[K] + dt * sq) for q2, q1, sq in zip(B2, B1, s)]
    X[2] = with_interior(m, X[2], torch.cat([X[2][1:nz], torch.zeros_like(X[2][nz:nz + 1])], 0))
    return X, fbar
