// stencil_rhs.cuh -- the momentum right-hand side of the RK stages, shared by
// the point-per-thread kernels (stencil.cu) and the fused RK kernel
// (rk_fused.cu).  Values are fetched through an accessor and neighbour
// offsets, so the same expressions serve global memory and shared-memory
// plane rings.
#pragma once

#include "stencil.cuh"

namespace pl {

// ------------------------------------------------------------------------
// momentum right-hand side (timeIntVelRK1_kernel, mod_calcVel.f90:74-138;
// timeIntVelRK2_kernel evaluates the same expressions on u1, :262-326)
// ------------------------------------------------------------------------
struct Nb {
    size_t c, xm, xp, ym, yp, zm, zp, xpym, xmyp, xpzm, xmzp, ypzm, ymzp;
};

__device__ __forceinline__ Nb neighbours(int i, int j, int k, int nx, int ny)
{
    const int im = (i == 0) ? nx - 1 : i - 1, ip = (i == nx - 1) ? 0 : i + 1;
    const int jm = (j == 0) ? ny - 1 : j - 1, jp = (j == ny - 1) ? 0 : j + 1;
    const size_t sk = (size_t)nx * ny;
    const size_t row = (size_t)nx * j + sk * k, rowm = (size_t)nx * jm + sk * k, rowp = (size_t)nx * jp + sk * k;
    Nb n;
    n.c = row + i;
    n.xm = row + im;
    n.xp = row + ip;
    n.ym = rowm + i;
    n.yp = rowp + i;
    n.zm = n.c - sk;
    n.zp = n.c + sk;
    n.xpym = rowm + ip; // (i+1, j-1)
    n.xmyp = rowp + im; // (i-1, j+1)
    n.xpzm = n.xp - sk; // (i+1, k-1)
    n.xmzp = n.xm + sk; // (i-1, k+1)
    n.ypzm = n.yp - sk; // (j+1, k-1)
    n.ymzp = n.ym + sk; // (j-1, k+1)
    return n;
}

// Field accessor: plain load converted to the compute type.
template <typename TS, typename TC> struct LoadF {
    const TS *__restrict__ a;
    __device__ __forceinline__ TC operator()(size_t q) const { return (TC)__ldg(a + q); }
};

// Accessor of the mixed path's stage-1 field u1 = u + d1 (u FP64, d1 FP32),
// rounded to FP32 for the FP32 stencil arithmetic.
struct LoadSum {
    const double *__restrict__ a;
    const float *__restrict__ d;
    __device__ __forceinline__ float operator()(size_t q) const
    {
        return (float)(__ldg(a + q) + (double)__ldg(d + q));
    }
};

// shared-memory ring offsets fit in 32 bits
struct Nb32 {
    int c, xm, xp, ym, yp, zm, zp, xpym, xmyp, xpzm, xmzp, ypzm, ymzp;
};

// the run and mesh constants of one k-plane of the momentum stencil
template <typename TC> struct RhsConst {
    TC dx_inv, dy_inv, re_inv, u_crf;
    TC dzf_k, dzf_kp, dzf_km, dzci_k, dzci_km, dzfi_k, dzfi_kp;
};

template <typename TC>
__device__ __forceinline__ RhsConst<TC> rhs_const(const StepParams &p, const MeshDev &m, int k)
{
    RhsConst<TC> c;
    c.dx_inv = (TC)p.dx_inv;
    c.dy_inv = (TC)p.dy_inv;
    c.re_inv = (TC)p.re_inv;
    c.u_crf = (TC)p.u_crf;
    c.dzf_k = (TC)__ldg(m.dzf + k);
    c.dzf_kp = (TC)__ldg(m.dzf + k + 1);
    c.dzf_km = (TC)__ldg(m.dzf + k - 1);
    c.dzci_k = (TC)__ldg(m.dzc_inv + k);
    c.dzci_km = (TC)__ldg(m.dzc_inv + k - 1);
    c.dzfi_k = (TC)__ldg(m.dzf_inv + k);
    c.dzfi_kp = (TC)__ldg(m.dzf_inv + k + 1);
    return c;
}

// the momentum right-hand sides with the plane's constants given; CRF false
// drops the u_crf advection terms (exact when u_crf == 0: they add zero)
template <typename TC, bool CRF, typename AU, typename AV, typename AW, typename NB>
__device__ __forceinline__ void momentum_rhs_c(const AU &u, const AV &v, const AW &w, const NB &n,
                                               const RhsConst<TC> &cst, TC &ru, TC &rv, TC &rw)
{
    const TC dx_inv = cst.dx_inv, dy_inv = cst.dy_inv, re_inv = cst.re_inv, u_crf = cst.u_crf;
    const TC dzf_k = cst.dzf_k, dzf_kp = cst.dzf_kp, dzf_km = cst.dzf_km;
    const TC dzci_k = cst.dzci_k, dzci_km = cst.dzci_km;
    const TC dzfi_k = cst.dzfi_k, dzfi_kp = cst.dzfi_kp;
    const TC h = (TC)0.25, half = (TC)0.5;

    const TC uc = u(n.c), uxp = u(n.xp), uxm = u(n.xm), uyp = u(n.yp), uym = u(n.ym), uzp = u(n.zp), uzm = u(n.zm);
    const TC vc = v(n.c), vxp = v(n.xp), vxm = v(n.xm), vyp = v(n.yp), vym = v(n.ym), vzp = v(n.zp), vzm = v(n.zm);
    const TC wc = w(n.c), wxp = w(n.xp), wxm = w(n.xm), wyp = w(n.yp), wym = w(n.ym), wzp = w(n.zp), wzm = w(n.zm);
    TC ue, uw, un, us, ut, ub, vn, vs, wt, wb, ve, vw, vt, vb, we, ww, wn, ws;
    TC dqe, dqw, dqn, dqs, dqt, dqb, conv, visc;

    // u-equation (:74-94)
    ue = (uc + uxp);
    uw = (uxm + uc);
    un = (uc + uyp);
    us = (uym + uc);
    ut = (uc * dzf_kp + uzp * dzf_k) * dzci_k;
    ub = (uc * dzf_km + uzm * dzf_k) * dzci_km;
    vn = (vc + vxp);
    vs = (vym + v(n.xpym));
    wt = (wc + wxp);
    wb = (wzm + w(n.xpzm));
    dqe = (uxp - uc) * dx_inv;
    dqw = (uc - uxm) * dx_inv;
    dqn = (uyp - uc) * dy_inv;
    dqs = (uc - uym) * dy_inv;
    dqt = (uzp - uc) * dzci_k;
    dqb = (uc - uzm) * dzci_km;
    conv = h * ((ue * ue - uw * uw) * dx_inv + (un * vn - us * vs) * dy_inv + (ut * wt - ub * wb) * dzfi_k);
    if (CRF) conv = conv + half * u_crf * (ue - uw) * dx_inv;
    visc = ((dqe - dqw) * dx_inv + (dqn - dqs) * dy_inv + (dqt - dqb) * dzfi_k) * re_inv;
    ru = visc - conv;

    // v-equation (:96-116)
    ve = (vc + vxp);
    vw = (vxm + vc);
    vn = (vc + vyp);
    vs = (vym + vc);
    vt = (vc * dzf_kp + vzp * dzf_k) * dzci_k;
    vb = (vc * dzf_km + vzm * dzf_k) * dzci_km;
    ue = (uc + uyp);
    uw = (uxm + u(n.xmyp));
    wt = (wc + wyp);
    wb = (wzm + w(n.ypzm));
    dqe = (vxp - vc) * dx_inv;
    dqw = (vc - vxm) * dx_inv;
    dqn = (vyp - vc) * dy_inv;
    dqs = (vc - vym) * dy_inv;
    dqt = (vzp - vc) * dzci_k;
    dqb = (vc - vzm) * dzci_km;
    conv = h * ((ue * ve - uw * vw) * dx_inv + (vn * vn - vs * vs) * dy_inv + (wt * vt - wb * vb) * dzfi_k);
    if (CRF) conv = conv + half * u_crf * (ve - vw) * dx_inv;
    visc = ((dqe - dqw) * dx_inv + (dqn - dqs) * dy_inv + (dqt - dqb) * dzfi_k) * re_inv;
    rv = visc - conv;

    // w-equation (:118-138)
    we = (wc + wxp);
    ww = (wxm + wc);
    wn = (wc + wyp);
    ws = (wym + wc);
    wt = (wc + wzp);
    wb = (wc + wzm);
    ue = (uc * dzf_kp + uzp * dzf_k) * dzci_k;
    uw = (uxm * dzf_kp + u(n.xmzp) * dzf_k) * dzci_k;
    vn = (vc * dzf_kp + vzp * dzf_k) * dzci_k;
    vs = (vym * dzf_kp + v(n.ymzp) * dzf_k) * dzci_k;
    dqe = (wxp - wc) * dx_inv;
    dqw = (wc - wxm) * dx_inv;
    dqn = (wyp - wc) * dy_inv;
    dqs = (wc - wym) * dy_inv;
    dqt = (wzp - wc) * dzfi_kp;
    dqb = (wc - wzm) * dzfi_k;
    conv = h * ((ue * we - uw * ww) * dx_inv + (vn * wn - vs * ws) * dy_inv + (wt * wt - wb * wb) * dzci_k);
    if (CRF) conv = conv + half * u_crf * (we - ww) * dx_inv;
    visc = ((dqe - dqw) * dx_inv + (dqn - dqs) * dy_inv + (dqt - dqb) * dzci_k) * re_inv;
    rw = visc - conv;
}

template <typename TC, typename AU, typename AV, typename AW, typename NB = Nb>
__device__ __forceinline__ void momentum_rhs(const AU &u, const AV &v, const AW &w, const NB &n, int k,
                                             const StepParams &p, const MeshDev &m, TC &ru, TC &rv, TC &rw)
{
    momentum_rhs_c<TC, true>(u, v, w, n, rhs_const<TC>(p, m, k), ru, rv, rw);
}


// wall fills of imposeNoSlipBC for the plane just written (k == 1 or nz),
// where that side is a wall (wlo, whi: see StepParams)
template <typename T>
__device__ __forceinline__ void wall_fill(T *u, T *v, T *w, size_t c, int k, size_t sk, int nz, T bcu, T uval,
                                          T vval, int wlo = 1, int whi = 1)
{
    if (wlo && k == 1) {
        u[c - sk] = (T)2.0 * bcu - uval;
        v[c - sk] = -vval;
        w[c - sk] = (T)0;
    }
    if (whi && k == nz) {
        u[c + sk] = (T)2.0 * bcu - uval;
        v[c + sk] = -vval;
        w[c] = (T)0;
        w[c + sk] = (T)0;
    }
}

// block-wide sum of three values; result valid in thread 0
__device__ __forceinline__ void block_sum3(double &a, double &b, double &c)
{
    __shared__ double sh[3][32];
    const int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
    const int wid = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
        sh[0][wid] = a;
        sh[1][wid] = b;
        sh[2][wid] = c;
    }
    __syncthreads();
    if (wid == 0) {
        a = lane < nw ? sh[0][lane] : 0.0;
        b = lane < nw ? sh[1][lane] : 0.0;
        c = lane < nw ? sh[2][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
            c += __shfl_down_sync(0xffffffffu, c, o);
        }
    }
}

// ------------------------------------------------------------------------
// Mean_h of the new streamwise velocity, fused into the RK2 kernels.
// forceVel (mod_calcVel.f90:463-476) shifts u by vel_force - Mean_h(u) after
// correctVel.  correctVel changes sum_i u by -dt/dx * sum_i (p_{i+1} - p_i),
// which telescopes to zero on the periodic x lines, so Mean_h of the
// corrected u equals Mean_h of the RK2 output (up to round-off): the shift is
// computed here and applied by the correction kernel, saving a pass.
// Block partials are summed by the last block in a fixed order
// (deterministic).
// ------------------------------------------------------------------------
struct MeanRed {
    double *partial;        // one per block
    unsigned int *counter;  // zero between launches
    double *scalar;         // [0] = Mean_h, [3] = vel_force - Mean_h
    double dnx, dny, vel_force;
};

__device__ __forceinline__ void mean_reduce(double su, const MeanRed &r)
{
    double z0 = 0.0, z1 = 0.0;
    block_sum3(su, z0, z1);
    __shared__ bool last;
    const int t = threadIdx.x + threadIdx.y * blockDim.x;
    const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
    if (t == 0) {
        const size_t b = blockIdx.x + (size_t)gridDim.x * (blockIdx.y + (size_t)gridDim.y * blockIdx.z);
        r.partial[b] = su;
        __threadfence();
        last = (atomicAdd(r.counter, 1u) == nb - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int nthr = blockDim.x * blockDim.y;
    double s = 0.0;
    for (unsigned int q = t; q < nb; q += nthr) s += __ldcg(r.partial + q);
    z0 = z1 = 0.0;
    __syncthreads();
    block_sum3(s, z0, z1);
    if (t == 0) {
        const double mean = s / r.dnx / r.dny;
        r.scalar[0] = mean;
        r.scalar[3] = r.vel_force - mean;
        r.scalar[6] = s; // the plane-weighted sum itself (z slabs add theirs across ranks)
        *r.counter = 0u;
    }
}

} // namespace pl
