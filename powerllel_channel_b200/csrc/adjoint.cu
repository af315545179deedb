// adjoint.cu -- hand-written discrete adjoint of the FP64 RK2 projection step
// and the gradient of the kinetic energy after n steps with respect to the
// initial velocity and a uniform body force.
//
// The reference has no adjoint.  The forward map differentiated is the step of
// channel.cu, FP64 path, Thomas PPE (main.f90:137-208 plus the body force
// f added to the momentum right-hand side of both RK stages):
//   y1 = x + dt (R(E x) + f)                 RK1, E = wall/periodic fill
//   y2 = (y1 + dt (R(E y1) + f) + x) / 2     RK2
//   y3 = P y2                                calcRHS, PPE, correctVel
//   x' = y3 + (vel_force - Mean_h(y3)) e_x   forceVel
// Its adjoint, in reverse order:
//   forceVel^T : ybar3 = xbar' - (dzf_k / (lz nx ny)) sum(xbar'_u) e_x
//   P^T        : ybar2 = W P W^-1 ybar3, with W = dzf_k for u, v and dzc_k
//                for w: P is symmetric in the cell-volume inner product
//                (summation by parts of calcRHS against correctVel), so the
//                forward calcRHS + PPE + correctVel kernels apply it
//   RK2^T      : ybar1 = ybar2/2 + (dt/2) S(y1; ybar2)
//   RK1^T      : xbar  = ybar2/2 + ybar1 + dt S(x; ybar1)
//   fbar      += (dt/2) sum(ybar2) + dt sum(ybar1)     (per component)
// with S(q; r) = E^T J_R(E q)^T r, the transposed momentum stencil below.
// The degrees of freedom are u, v on levels 1..nz and w on levels 1..nz-1
// (w(nz) is the top wall).
//
// Checkpointing: the forward run stores the state every `every` steps; the
// reverse sweep recomputes each segment forward from its checkpoint, keeping
// the segment's states, and then runs the adjoint steps of the segment
// backwards.  Memory: ceil(n/every) + every states of 3 fields.
#include <algorithm>
#include <cmath>
#include <vector>

#include "channel.cuh"
#include "stencil_rhs.cuh"

using namespace pl;

namespace {

constexpr int SUM_PARTS = 8; // partial sums per level in the plane reductions

dim3 adj_block() { return dim3(64, 4, 1); }
dim3 adj_grid(const StepParams &p) { return dim3((p.nx + 63) / 64, (p.ny + 3) / 4, p.nz); }

// out = alpha r + beta S(q; r) + gamma e at every degree of freedom; the
// output's ghost planes are not written, and its w on level nz is zero.
// q: base state (BC-filled); r: adjoint fields with zero ghost planes and
// zero w on level nz.  Each flux of the momentum stencil shared by two
// equations (Pxy: y flux of u and x flux of v; Pxz: z flux of u and x flux
// of w; Pyz: z flux of v and y flux of w) gets one adjoint, the sum of the
// adjoints of its two uses; the adjoint of a flux difference
// -0.25 (F(o) - F(o-1)) h_o is -0.25 (h_o r(o) - h_{o+1} r(o+1)).
__global__ void __launch_bounds__(256) k_adj_rk(const double *__restrict__ u, const double *__restrict__ v,
                                                const double *__restrict__ w, const double *__restrict__ ru,
                                                const double *__restrict__ rv, const double *__restrict__ rw,
                                                const double *__restrict__ eu, const double *__restrict__ ev,
                                                const double *__restrict__ ew, double *__restrict__ ou,
                                                double *__restrict__ ov, double *__restrict__ ow, double alpha,
                                                double beta, double gamma, StepParams p, MeshDev m)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + 1;
    if (i >= p.nx || j >= p.ny) return;
    const Nb n = neighbours(i, j, k, p.nx, p.ny);
    const double dxi = p.dx_inv, dyi = p.dy_inv, re = p.re_inv, q = 0.25;
    const double f_c = __ldg(m.dzf + k), f_p = __ldg(m.dzf + k + 1), f_m = __ldg(m.dzf + k - 1);
    const double ci_c = __ldg(m.dzc_inv + k), ci_m = __ldg(m.dzc_inv + k - 1), ci_p = __ldg(m.dzc_inv + k + 1);
    const double fi_c = __ldg(m.dzf_inv + k), fi_p = __ldg(m.dzf_inv + k + 1), fi_m = __ldg(m.dzf_inv + k - 1);

    const double Uc = __ldg(u + n.c), Uxp = __ldg(u + n.xp), Uxm = __ldg(u + n.xm), Uyp = __ldg(u + n.yp),
                 Uzp = __ldg(u + n.zp), Uxmyp = __ldg(u + n.xmyp), Uxmzp = __ldg(u + n.xmzp);
    const double Vc = __ldg(v + n.c), Vxp = __ldg(v + n.xp), Vym = __ldg(v + n.ym), Vyp = __ldg(v + n.yp),
                 Vzp = __ldg(v + n.zp), Vxpym = __ldg(v + n.xpym), Vymzp = __ldg(v + n.ymzp);
    const double Wc = __ldg(w + n.c), Wxp = __ldg(w + n.xp), Wyp = __ldg(w + n.yp), Wzp = __ldg(w + n.zp),
                 Wzm = __ldg(w + n.zm), Wxpzm = __ldg(w + n.xpzm), Wypzm = __ldg(w + n.ypzm);

    const double RUc = __ldg(ru + n.c), RUxp = __ldg(ru + n.xp), RUxm = __ldg(ru + n.xm), RUyp = __ldg(ru + n.yp),
                 RUym = __ldg(ru + n.ym), RUzp = __ldg(ru + n.zp), RUzm = __ldg(ru + n.zm),
                 RUxmyp = __ldg(ru + n.xmyp), RUxmzp = __ldg(ru + n.xmzp);
    const double RVc = __ldg(rv + n.c), RVxp = __ldg(rv + n.xp), RVxm = __ldg(rv + n.xm), RVyp = __ldg(rv + n.yp),
                 RVym = __ldg(rv + n.ym), RVzp = __ldg(rv + n.zp), RVzm = __ldg(rv + n.zm),
                 RVxpym = __ldg(rv + n.xpym), RVymzp = __ldg(rv + n.ymzp);
    const double RWc = __ldg(rw + n.c), RWxp = __ldg(rw + n.xp), RWxm = __ldg(rw + n.xm), RWyp = __ldg(rw + n.yp),
                 RWym = __ldg(rw + n.ym), RWzp = __ldg(rw + n.zp), RWzm = __ldg(rw + n.zm),
                 RWxpzm = __ldg(rw + n.xpzm), RWypzm = __ldg(rw + n.ypzm);

    // flux adjoints at the faces of cell g and of its x-, y- and z-neighbours below
    const double Aux_c = -q * dxi * (RUc - RUxp), Aux_m = -q * dxi * (RUxm - RUc);
    const double Avy_c = -q * dyi * (RVc - RVyp), Avy_m = -q * dyi * (RVym - RVc);
    const double Awz_c = -q * (RWc * ci_c - RWzp * ci_p), Awz_m = -q * (RWzm * ci_m - RWc * ci_c);
    const double Pxy_c = -q * dyi * (RUc - RUyp) - q * dxi * (RVc - RVxp);
    const double Pxy_ym = -q * dyi * (RUym - RUc) - q * dxi * (RVym - RVxpym);
    const double Pxy_xm = -q * dyi * (RUxm - RUxmyp) - q * dxi * (RVxm - RVc);
    const double Pxz_c = -q * (RUc * fi_c - RUzp * fi_p) - q * dxi * (RWc - RWxp);
    const double Pxz_zm = -q * (RUzm * fi_m - RUc * fi_c) - q * dxi * (RWzm - RWxpzm);
    const double Pxz_xm = -q * (RUxm * fi_c - RUxmzp * fi_p) - q * dxi * (RWxm - RWc);
    const double Pyz_c = -q * (RVc * fi_c - RVzp * fi_p) - q * dyi * (RWc - RWyp);
    const double Pyz_zm = -q * (RVzm * fi_m - RVc * fi_c) - q * dyi * (RWzm - RWypzm);
    const double Pyz_ym = -q * (RVym * fi_c - RVymzp * fi_p) - q * dyi * (RWym - RWc);

    // convective part: flux adjoint times the derivative of the flux
    const double ut_c = (Uc * f_p + Uzp * f_c) * ci_c, ut_xm = (Uxm * f_p + Uxmzp * f_c) * ci_c;
    const double vt_c = (Vc * f_p + Vzp * f_c) * ci_c, vt_ym = (Vym * f_p + Vymzp * f_c) * ci_c;
    double su = 2.0 * (Uc + Uxp) * Aux_c + 2.0 * (Uxm + Uc) * Aux_m + (Vc + Vxp) * Pxy_c + (Vym + Vxpym) * Pxy_ym +
                f_p * ci_c * (Wc + Wxp) * Pxz_c + f_m * ci_m * (Wzm + Wxpzm) * Pxz_zm;
    double sv = 2.0 * (Vc + Vyp) * Avy_c + 2.0 * (Vym + Vc) * Avy_m + (Uc + Uyp) * Pxy_c + (Uxm + Uxmyp) * Pxy_xm +
                f_p * ci_c * (Wc + Wyp) * Pyz_c + f_m * ci_m * (Wzm + Wypzm) * Pyz_zm;
    double sw = 2.0 * (Wc + Wzp) * Awz_c + 2.0 * (Wzm + Wc) * Awz_m + ut_c * Pxz_c + ut_xm * Pxz_xm + vt_c * Pyz_c +
                vt_ym * Pyz_ym;

    // u_crf advection: adjoint of -0.5 u_crf (q(i+1) - q(i-1)) dx_inv
    const double hc = 0.5 * p.u_crf * dxi;
    su -= hc * (RUxm - RUxp);
    sv -= hc * (RVxm - RVxp);
    sw -= hc * (RWxm - RWxp);

    // viscous part; the wall ghosts q(0) = 2bc - q(1), q(nz+1) = 2bc - q(nz)
    // of u and v double the wall-face coefficients
    const double dxi2 = dxi * dxi, dyi2 = dyi * dyi;
    const double ca = (k == 1) ? 2.0 : 1.0, cb = (k == p.nz) ? 2.0 : 1.0;
    su += re * ((RUxp - 2.0 * RUc + RUxm) * dxi2 + (RUyp - 2.0 * RUc + RUym) * dyi2) -
          cb * ci_c * re * (RUc * fi_c - RUzp * fi_p) + ca * ci_m * re * (RUzm * fi_m - RUc * fi_c);
    sv += re * ((RVxp - 2.0 * RVc + RVxm) * dxi2 + (RVyp - 2.0 * RVc + RVym) * dyi2) -
          cb * ci_c * re * (RVc * fi_c - RVzp * fi_p) + ca * ci_m * re * (RVzm * fi_m - RVc * fi_c);
    sw += re * ((RWxp - 2.0 * RWc + RWxm) * dxi2 + (RWyp - 2.0 * RWc + RWym) * dyi2) -
          fi_p * re * (RWc * ci_c - RWzp * ci_p) + fi_c * re * (RWzm * ci_m - RWc * ci_c);

    double xu = alpha * RUc + beta * su, xv = alpha * RVc + beta * sv, xw = alpha * RWc + beta * sw;
    if (eu) {
        xu += gamma * __ldg(eu + n.c);
        xv += gamma * __ldg(ev + n.c);
        xw += gamma * __ldg(ew + n.c);
    }
    ou[n.c] = xu;
    ov[n.c] = xv;
    ow[n.c] = (k == p.nz) ? 0.0 : xw;
}

// per-level partial sums of three fields over the degrees of freedom:
// MODE 0: sums of a, b, c; MODE 1: kinetic-energy terms dzf (a^2 + b^2) and
// dzc c^2.  part[((k-1) * SUM_PARTS + q) * 3 + comp], fixed summation order.
template <int MODE>
__global__ void __launch_bounds__(256) k_level_sums(const double *__restrict__ a, const double *__restrict__ b,
                                                    const double *__restrict__ c, StepParams p, MeshDev m,
                                                    double *__restrict__ part)
{
    __shared__ double sh[3][256];
    const int k = blockIdx.y + 1, q = blockIdx.x, t = threadIdx.x;
    const size_t sk = (size_t)p.nx * p.ny, n = sk;
    const size_t chunk = (n + SUM_PARTS - 1) / SUM_PARTS;
    const size_t beg = chunk * q, end = min(n, beg + chunk);
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    const double *pa = a + sk * k, *pb = b + sk * k, *pc = c + sk * k;
    for (size_t x = beg + t; x < end; x += 256) {
        const double va = __ldg(pa + x), vb = __ldg(pb + x), vc = __ldg(pc + x);
        if (MODE == 0) {
            s0 += va;
            s1 += vb;
            s2 += vc;
        } else {
            s0 += va * va;
            s1 += vb * vb;
            s2 += vc * vc;
        }
    }
    if (k == p.nz) s2 = 0.0; // w(nz) is the wall
    sh[0][t] = s0;
    sh[1][t] = s1;
    sh[2][t] = s2;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (t < h) {
            sh[0][t] += sh[0][t + h];
            sh[1][t] += sh[1][t + h];
            sh[2][t] += sh[2][t + h];
        }
        __syncthreads();
    }
    if (t == 0) {
        double *o = part + ((size_t)(k - 1) * SUM_PARTS + q) * 3;
        if (MODE == 0) {
            o[0] = sh[0][0];
            o[1] = sh[1][0];
            o[2] = sh[2][0];
        } else {
            const double fz = __ldg(m.dzf + k), cz = 1.0 / __ldg(m.dzc_inv + k);
            o[0] = fz * sh[0][0];
            o[1] = fz * sh[1][0];
            o[2] = cz * sh[2][0];
        }
    }
}

// out[c] = (accumulate ? out[c] : 0) + coef * sum of the level partials, in k order
__global__ void k_sums_finish(const double *__restrict__ part, int nz, double coef, int accumulate,
                              double *__restrict__ out)
{
    const int c = threadIdx.x;
    if (c >= 3) return;
    double s = 0.0;
    for (int x = 0; x < nz * SUM_PARTS; x++) s += part[(size_t)x * 3 + c];
    out[c] = (accumulate ? out[c] : 0.0) + coef * s;
}

// forceVel^T and division by the cell volumes: z = W^-1 (xbar - c_k S e_x),
// c_k = dzf_k / (lz nx ny), S = sum of xbar_u (scal[0]) when x is forced
__global__ void __launch_bounds__(256) k_adj_prep(const double *__restrict__ au, const double *__restrict__ av,
                                                  const double *__restrict__ aw, double *__restrict__ zu,
                                                  double *__restrict__ zv, double *__restrict__ zw,
                                                  const double *__restrict__ scal, int forced_x, StepParams p,
                                                  MeshDev m)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + 1;
    if (i >= p.nx || j >= p.ny) return;
    const size_t g = (size_t)i + (size_t)p.nx * j + (size_t)p.nx * p.ny * k;
    const double fi = __ldg(m.dzf_inv + k);
    double xu = au[g];
    if (forced_x) xu -= __ldg(m.dzflzi + k) / ((double)p.nx * p.ny) * scal[0];
    zu[g] = xu * fi;
    zv[g] = av[g] * fi;
    zw[g] = (k == p.nz) ? 0.0 : aw[g] * __ldg(m.dzc_inv + k);
}

// correctVel on z with the solved p, then multiplication by the cell
// volumes: ybar2 = W (z - dt G p), in place; p interior-only, p(nz+1) = p(nz)
__global__ void __launch_bounds__(256) k_adj_correct(const double *__restrict__ pp, double *zu, double *zv,
                                                     double *zw, StepParams p, MeshDev m)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + 1;
    if (i >= p.nx || j >= p.ny) return;
    const size_t sk = (size_t)p.nx * p.ny;
    const int ip = (i == p.nx - 1) ? 0 : i + 1, jp = (j == p.ny - 1) ? 0 : j + 1;
    const size_t g = (size_t)i + (size_t)p.nx * j + sk * k;
    const size_t c0 = (size_t)i + (size_t)p.nx * j + sk * (k - 1);
    const double p0 = __ldg(pp + c0);
    const double pxp = __ldg(pp + (size_t)ip + (size_t)p.nx * j + sk * (k - 1));
    const double pyp = __ldg(pp + (size_t)i + (size_t)p.nx * jp + sk * (k - 1));
    const double dt = p.dt, fz = __ldg(m.dzf + k);
    zu[g] = (zu[g] - (pxp - p0) * (dt * p.dx_inv)) * fz;
    zv[g] = (zv[g] - (pyp - p0) * (dt * p.dy_inv)) * fz;
    if (k == p.nz) {
        zw[g] = 0.0;
    } else {
        const double pzp = __ldg(pp + c0 + sk), ci = __ldg(m.dzc_inv + k);
        zw[g] = (zw[g] - (pzp - p0) * dt * ci) / ci;
    }
}

// seed of the reverse sweep: dJ/dx_N = dx dy W x_N
__global__ void __launch_bounds__(256) k_adj_seed(const double *__restrict__ u, const double *__restrict__ v,
                                                  const double *__restrict__ w, double *__restrict__ au,
                                                  double *__restrict__ av, double *__restrict__ aw, double dxdy,
                                                  StepParams p, MeshDev m)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + 1;
    if (i >= p.nx || j >= p.ny) return;
    const size_t g = (size_t)i + (size_t)p.nx * j + (size_t)p.nx * p.ny * k;
    const double fz = __ldg(m.dzf + k);
    au[g] = dxdy * fz * u[g];
    av[g] = dxdy * fz * v[g];
    aw[g] = (k == p.nz) ? 0.0 : dxdy / __ldg(m.dzc_inv + k) * w[g];
}

struct AdjWork {
    std::vector<double *> owned;
    double *ck = nullptr, *seg = nullptr;           // checkpoints, segment states (3 fields each)
    double *xa = nullptr, *y2 = nullptr, *y1 = nullptr; // adjoint fields (3 fields each)
    double *part = nullptr, *scal = nullptr, *fbar = nullptr;
    ~AdjWork()
    {
        for (double *p : owned) cudaFree(p);
    }
    bool alloc(double **p, size_t n, cudaStream_t st)
    {
        if (cudaMalloc(p, sizeof(double) * n) != cudaSuccess) return false;
        owned.push_back(*p);
        return cudaMemsetAsync(*p, 0, sizeof(double) * n, st) == cudaSuccess;
    }
};

int level_sums(int mode, const double *a, const double *b, const double *c, const pl_channel *ch, double *part,
               double coef, int accumulate, double *out)
{
    dim3 g(SUM_PARTS, ch->nz);
    if (mode == 0)
        k_level_sums<0><<<g, 256, 0, ch->stream>>>(a, b, c, ch->sp, ch->m, part);
    else
        k_level_sums<1><<<g, 256, 0, ch->stream>>>(a, b, c, ch->sp, ch->m, part);
    PL_CHECK_LAUNCH();
    k_sums_finish<<<1, 32, 0, ch->stream>>>(part, ch->nz, coef, accumulate, out);
    PL_CHECK_LAUNCH();
    return 0;
}

int copy3(double *du, double *dv, double *dw, const double *su, const double *sv, const double *sw, size_t nf,
          cudaStream_t st)
{
    PL_CUDA_TRY(cudaMemcpyAsync(du, su, sizeof(double) * nf, cudaMemcpyDeviceToDevice, st));
    PL_CUDA_TRY(cudaMemcpyAsync(dv, sv, sizeof(double) * nf, cudaMemcpyDeviceToDevice, st));
    PL_CUDA_TRY(cudaMemcpyAsync(dw, sw, sizeof(double) * nf, cudaMemcpyDeviceToDevice, st));
    return 0;
}

// one adjoint step at base state x (3 fields): W.xa holds xbar_{n+1} on entry
// and xbar_n on return; fbar accumulates
int adjoint_step(pl_channel *c, const double *xu, const double *xv, const double *xw, AdjWork &W)
{
    const size_t nf = c->nf;
    const StepParams &p = c->sp;
    cudaStream_t st = c->stream;
    double *au = W.xa, *av = W.xa + nf, *aw = W.xa + 2 * nf;
    double *bu = W.y2, *bv = W.y2 + nf, *bw = W.y2 + 2 * nf;
    double *cu = W.y1, *cv = W.y1 + nf, *cw = W.y1 + 2 * nf;
    // stage-1 state y1 = RK1(x) (with its wall fill) into u1, v1, w1
    if (launch_rk1_fp64(xu, xv, xw, c->u1, c->v1, c->w1, p, c->m, st)) return -1;
    // forceVel^T, W^-1
    const int fx = c->cfg.is_forced[0];
    if (fx && level_sums(0, au, av, aw, c, W.part, 1.0, 0, W.scal)) return -1;
    k_adj_prep<<<adj_grid(p), adj_block(), 0, st>>>(au, av, aw, bu, bv, bw, W.scal, fx, p, c->m);
    PL_CHECK_LAUNCH();
    // P, then W
    if (launch_calc_rhs_fp64(bu, bv, bw, c->p, p, c->m, st)) return -1;
    if (ppe_solve_fp64(&c->ppe, c->p, st)) return -1;
    k_adj_correct<<<adj_grid(p), adj_block(), 0, st>>>(c->p, bu, bv, bw, p, c->m);
    PL_CHECK_LAUNCH();
    if (level_sums(0, bu, bv, bw, c, W.part, 0.5 * p.dt, 1, W.fbar)) return -1;
    // RK2^T at y1
    k_adj_rk<<<adj_grid(p), adj_block(), 0, st>>>(c->u1, c->v1, c->w1, bu, bv, bw, nullptr, nullptr, nullptr, cu, cv,
                                                  cw, 0.5, 0.5 * p.dt, 0.0, p, c->m);
    PL_CHECK_LAUNCH();
    if (level_sums(0, cu, cv, cw, c, W.part, p.dt, 1, W.fbar)) return -1;
    // RK1^T at x
    k_adj_rk<<<adj_grid(p), adj_block(), 0, st>>>(xu, xv, xw, cu, cv, cw, bu, bv, bw, au, av, aw, 1.0, p.dt, 0.5, p,
                                                  c->m);
    PL_CHECK_LAUNCH();
    return 0;
}

} // namespace

extern "C" int pl_channel_set_body_force(pl_channel *c, const double f[3])
{
    if (c->cfg.precision != PL_FP64 && (f[0] != 0.0 || f[1] != 0.0 || f[2] != 0.0)) {
        set_error("pl_channel_set_body_force: the body force is defined for the FP64 path only");
        return -1;
    }
    for (int d = 0; d < 3; d++) c->sp.fb[d] = f[d];
    return 0;
}

extern "C" int pl_channel_kinetic_energy(pl_channel *c, double *ke)
{
    double *part = nullptr, *out = nullptr;
    PL_CUDA_TRY(cudaMalloc(&part, sizeof(double) * (3 * SUM_PARTS * (size_t)c->nz + 4)));
    out = part + 3 * SUM_PARTS * (size_t)c->nz;
    int rc = level_sums(1, c->u, c->v, c->w, c, part, 1.0, 0, out);
    double h[3] = {0, 0, 0};
    if (!rc && cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) rc = -1;
    if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = -1;
    cudaFree(part);
    if (rc) {
        set_error("pl_channel_kinetic_energy: device error");
        return -1;
    }
    const double dx = c->cfg.lx / c->nx, dy = c->cfg.ly / c->ny;
    *ke = 0.5 * dx * dy * (h[0] + h[1] + h[2]);
    return 0;
}

extern "C" int pl_adjoint_ke_gradient(pl_channel *c, int nsteps, int every, double *ke, double *d_gu, double *d_gv,
                                      double *d_gw, double grad_f[3])
{
    if (c->cfg.precision != PL_FP64) {
        set_error("pl_adjoint_ke_gradient: the adjoint is defined for the FP64 path");
        return -1;
    }
    if (c->cfg.trid_parts > 1) {
        set_error("pl_adjoint_ke_gradient: needs the Thomas PPE (trid_parts 0 or 1); PDD's truncated solve is "
                  "not an exact inverse, so the transposed projection differs from the forward one");
        return -1;
    }
    if (nsteps < 0 || every < 1) {
        set_error("pl_adjoint_ke_gradient: nsteps must be >= 0 and every >= 1");
        return -1;
    }
    const size_t nf = c->nf;
    const StepParams &p = c->sp;
    cudaStream_t st = c->stream;
    const int nck = (nsteps + every - 1) / every;
    const int nseg = std::min(every, std::max(nsteps, 1));
    AdjWork W;
    if (!W.alloc(&W.ck, 3 * nf * (size_t)std::max(nck, 1), st) || !W.alloc(&W.seg, 3 * nf * (size_t)nseg, st) ||
        !W.alloc(&W.xa, 3 * nf, st) || !W.alloc(&W.y2, 3 * nf, st) || !W.alloc(&W.y1, 3 * nf, st) ||
        !W.alloc(&W.part, 3 * SUM_PARTS * (size_t)c->nz + 16, st)) {
        set_error("pl_adjoint_ke_gradient: out of device memory for checkpoints and adjoint fields");
        return -1;
    }
    W.scal = W.part + 3 * SUM_PARTS * (size_t)c->nz;
    W.fbar = W.scal + 4;
    auto state = [&](double *base, int slot) { return base + 3 * nf * (size_t)slot; };

    // forward sweep with checkpoints
    if (launch_fill_bc_vel(c->u, c->v, c->w, p, st)) return -1;
    if (copy3(state(W.ck, 0), state(W.ck, 0) + nf, state(W.ck, 0) + 2 * nf, c->u, c->v, c->w, nf, st)) return -1;
    for (int n = 0; n < nsteps; n++) {
        if (n % every == 0) {
            double *s = state(W.ck, n / every);
            if (copy3(s, s + nf, s + 2 * nf, c->u, c->v, c->w, nf, st)) return -1;
        }
        if (pl_channel_step(c, 1)) return -1;
    }
    double *keout = W.scal + 8;
    if (level_sums(1, c->u, c->v, c->w, c, W.part, 1.0, 0, keout)) return -1;
    double h[3];
    PL_CUDA_TRY(cudaMemcpyAsync(h, keout, sizeof(h), cudaMemcpyDeviceToHost, st));
    PL_CUDA_TRY(cudaStreamSynchronize(st));
    const double dx = c->cfg.lx / c->nx, dy = c->cfg.ly / c->ny;
    *ke = 0.5 * dx * dy * (h[0] + h[1] + h[2]);
    k_adj_seed<<<adj_grid(p), adj_block(), 0, st>>>(c->u, c->v, c->w, W.xa, W.xa + nf, W.xa + 2 * nf, dx * dy, p,
                                                    c->m);
    PL_CHECK_LAUNCH();

    // reverse sweep, segment by segment
    for (int s = nck - 1; s >= 0; s--) {
        const int n0 = s * every, n1 = std::min(nsteps, n0 + every);
        const double *ck = state(W.ck, s);
        if (copy3(c->u, c->v, c->w, ck, ck + nf, ck + 2 * nf, nf, st)) return -1;
        for (int n = n0; n < n1; n++) {
            double *x = state(W.seg, n - n0);
            if (copy3(x, x + nf, x + 2 * nf, c->u, c->v, c->w, nf, st)) return -1;
            if (n < n1 - 1 && pl_channel_step(c, 1)) return -1;
        }
        for (int n = n1 - 1; n >= n0; n--) {
            const double *x = state(W.seg, n - n0);
            if (adjoint_step(c, x, x + nf, x + 2 * nf, W)) return -1;
        }
    }

    // results; the fields are left at the initial state
    if (copy3(d_gu, d_gv, d_gw, W.xa, W.xa + nf, W.xa + 2 * nf, nf, st)) return -1;
    const double *x0 = state(W.ck, 0);
    if (copy3(c->u, c->v, c->w, x0, x0 + nf, x0 + 2 * nf, nf, st)) return -1;
    PL_CUDA_TRY(cudaMemcpyAsync(grad_f, W.fbar, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    PL_CUDA_TRY(cudaStreamSynchronize(st));
    return 0;
}
