// stencil.cu -- RK2 momentum stencils, divergence, projection, forcing, wall
// fills, diagnostics and the initial field.
//
// One thread per grid point, (i, j) over the block, k over blockIdx.z;
// neighbour values come through L1/L2 (each field is streamed from HBM once).
// x and y neighbours wrap periodically; the wall ghost planes k = 0, nz+1 are
// stored and refreshed by the kernel that writes the adjacent interior plane,
// which reproduces imposeNoSlipBC (mod_updateBound.f90:274-330) applied after
// the periodic fills.
#include "stencil.cuh"
#include "stencil_rhs.cuh"

namespace pl {

#define PL_POINT_INDEX()                                                                   \
    const int i = blockIdx.x * blockDim.x + threadIdx.x;                                   \
    const int j = blockIdx.y * blockDim.y + threadIdx.y;                                   \
    const int k = blockIdx.z + 1;                                                          \
    if (i >= p.nx || j >= p.ny) return;                                                    \
    const size_t sk = (size_t)p.nx * p.ny;

// RK1: u1 = u + dt*(visc - conv) (mod_calcVel.f90:94,116,138) + wall fill
__global__ void __launch_bounds__(256) k_rk1_fp64(const double *__restrict__ u, const double *__restrict__ v,
                                                  const double *__restrict__ w, double *__restrict__ u1,
                                                  double *__restrict__ v1, double *__restrict__ w1, StepParams p,
                                                  MeshDev m)
{
    PL_POINT_INDEX();
    const Nb n = neighbours(i, j, k, p.nx, p.ny);
    double ru, rv, rw;
    momentum_rhs<double>(LoadF<double, double>{u}, LoadF<double, double>{v}, LoadF<double, double>{w}, n, k, p, m,
                         ru, rv, rw);
    const double nu = __ldg(u + n.c) + p.dt * (ru + p.fb[0]);
    const double nv = __ldg(v + n.c) + p.dt * (rv + p.fb[1]);
    u1[n.c] = nu;
    v1[n.c] = nv;
    if (k != p.nz) w1[n.c] = __ldg(w + n.c) + p.dt * (rw + p.fb[2]);
    wall_fill<double>(u1, v1, w1, n.c, k, sk, p.nz, 0.0 - p.u_crf, nu, nv);
}

// RK2: u = (u1 + dt*(visc - conv)(u1) + u) * 0.5 (:282,304,326) + wall fill.
// u is read at the centre only, so the update is in place.
__global__ void __launch_bounds__(256) k_rk2_fp64(double *u, double *v, double *w, const double *__restrict__ u1,
                                                  const double *__restrict__ v1, const double *__restrict__ w1,
                                                  StepParams p, MeshDev m)
{
    PL_POINT_INDEX();
    const Nb n = neighbours(i, j, k, p.nx, p.ny);
    double ru, rv, rw;
    momentum_rhs<double>(LoadF<double, double>{u1}, LoadF<double, double>{v1}, LoadF<double, double>{w1}, n, k, p,
                         m, ru, rv, rw);
    const double nu = (__ldg(u1 + n.c) + p.dt * (ru + p.fb[0]) + u[n.c]) * 0.5;
    const double nv = (__ldg(v1 + n.c) + p.dt * (rv + p.fb[1]) + v[n.c]) * 0.5;
    u[n.c] = nu;
    v[n.c] = nv;
    if (k != p.nz) w[n.c] = (__ldg(w1 + n.c) + p.dt * (rw + p.fb[2]) + w[n.c]) * 0.5;
    wall_fill<double>(u, v, w, n.c, k, sk, p.nz, 0.0 - p.u_crf, nu, nv);
}

// calcRHS (mod_calcRHS.f90:19-33): rhs = div(u)/dt into the interior-only array
__global__ void __launch_bounds__(256) k_calc_rhs_fp64(const double *__restrict__ u, const double *__restrict__ v,
                                                       const double *__restrict__ w, double *__restrict__ rhs,
                                                       StepParams p, MeshDev m)
{
    PL_POINT_INDEX();
    const Nb n = neighbours(i, j, k, p.nx, p.ny);
    const double dti = 1.0 / p.dt, dtidxi = dti * p.dx_inv, dtidyi = dti * p.dy_inv;
    rhs[n.c - sk] = (__ldg(u + n.c) - __ldg(u + n.xm)) * dtidxi + (__ldg(v + n.c) - __ldg(v + n.ym)) * dtidyi +
                    (__ldg(w + n.c) - __ldg(w + n.zm)) * dti * __ldg(m.dzf_inv + k);
}

// correctVel (mod_calcVel.f90:436-450) + dz-weighted sums for Mean_h
// (mod_utils.f90:105-131) of the corrected components + wall fill of v.
// p is interior-only; p(nz+1) = p(nz) (imposeZeroGradBC) makes the w
// correction of the top plane zero.
template <typename TP>
__global__ void __launch_bounds__(256) k_correct(const TP *__restrict__ pp, double *u, double *v, double *w,
                                                 StepParams p, MeshDev m, double *partial)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + 1;
    double su = 0.0, sv = 0.0, sw = 0.0;
    if (i < p.nx && j < p.ny) {
        const size_t sk = (size_t)p.nx * p.ny;
        const Nb n = neighbours(i, j, k, p.nx, p.ny);
        const double dt = p.dt, dtdxi = dt * p.dx_inv, dtdyi = dt * p.dy_inv;
        const size_t pc = n.c - sk;
        const double p0 = (double)__ldg(pp + pc);
        const double pxp = (double)__ldg(pp + n.xp - sk), pyp = (double)__ldg(pp + n.yp - sk);
        const double pzp = (k < p.nz) ? (double)__ldg(pp + pc + sk) : p0;
        const double nu = u[n.c] - (pxp - p0) * dtdxi;
        const double nv = v[n.c] - (pyp - p0) * dtdyi;
        const double nw = w[n.c] - (pzp - p0) * dt * __ldg(m.dzc_inv + k);
        u[n.c] = nu;
        v[n.c] = nv;
        w[n.c] = nw;
        // wall fill of the corrected u, v (w(0) = w(nz) = 0 are unchanged);
        // a forced component is refilled after its shift by k_force
        const double bcu = 0.0 - p.u_crf;
        if (k == 1) {
            u[n.c - sk] = 2.0 * bcu - nu;
            v[n.c - sk] = -nv;
        }
        if (k == p.nz) {
            u[n.c + sk] = 2.0 * bcu - nu;
            v[n.c + sk] = -nv;
        }
        const double wz = __ldg(m.dzflzi + k);
        su = nu * wz;
        sv = nv * wz;
        sw = nw * wz;
    }
    block_sum3(su, sv, sw);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const size_t b = blockIdx.x + (size_t)gridDim.x * (blockIdx.y + (size_t)gridDim.y * blockIdx.z);
        const size_t nb = (size_t)gridDim.x * gridDim.y * gridDim.z;
        partial[b] = su;
        partial[nb + b] = sv;
        partial[2 * nb + b] = sw;
    }
}

// fixed-order final sum of the block partials (deterministic), then
// Mean_h = sum / nx / ny and the forceVel shift vel_force - mean
__global__ void k_finish_means(const double *partial, int nb, double dnx, double dny, double f0, double f1,
                               double f2, double *scalar)
{
    const int comp = blockIdx.x;
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[(size_t)comp * nb + b];
    __shared__ double sh[1024];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double mean = sh[0] / dnx / dny; // Mean_h/nx_global/ny_global (mod_utils.f90:128)
        scalar[comp] = mean;
        if (comp == 0) scalar[6] = sh[0]; // the sum itself (z slabs add theirs across ranks)
        const double f = comp == 0 ? f0 : (comp == 1 ? f1 : f2);
        scalar[3 + comp] = f - mean;
    }
}

// forceVel (mod_calcVel.f90:463-506) + wall fill of the forced components
__global__ void __launch_bounds__(256) k_force(double *u, double *v, double *w, StepParams p, int fx, int fy,
                                               int fz, const double *scalar)
{
    PL_POINT_INDEX();
    const size_t c = (size_t)i + (size_t)p.nx * j + sk * k;
    const double bcu = 0.0 - p.u_crf;
    if (fx) {
        const double nu = u[c] + scalar[3];
        u[c] = nu;
        if (k == 1) u[c - sk] = 2.0 * bcu - nu;
        if (k == p.nz) u[c + sk] = 2.0 * bcu - nu;
    }
    if (fy) {
        const double nv = v[c] + scalar[4];
        v[c] = nv;
        if (k == 1) v[c - sk] = -nv;
        if (k == p.nz) v[c + sk] = -nv;
    }
    if (fz) {
        if (k != p.nz) w[c] = w[c] + scalar[5];
    }
}

// ------------------------------------------------------------------------
// diagnostics (checkNaN, calcMaxCFL, calcMaxDiv: mod_utils.f90:193-394)
// ------------------------------------------------------------------------
// lexicographic (value desc, linear index asc): the first strict maximum in
// k, j, i order, as the sequential loops of the reference find it
__device__ __forceinline__ void better(double &v, long long &ix, double ov, long long oix)
{
    if (ov > v || (ov == v && oix < ix)) {
        v = ov;
        ix = oix;
    }
}

__global__ void __launch_bounds__(256) k_diag(const double *__restrict__ u, const double *__restrict__ v,
                                              const double *__restrict__ w, StepParams p, MeshDev m,
                                              double *part, long long *ipart)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + 1;
    double dv = -1.0, cv = -1.0, nan = 0.0;
    long long di = 0x7fffffffffffffffLL, ci = 0x7fffffffffffffffLL;
    if (i < p.nx && j < p.ny) {
        const Nb n = neighbours(i, j, k, p.nx, p.ny);
        const double dzfi = __ldg(m.dzf_inv + k);
        const double uc = __ldg(u + n.c), vc = __ldg(v + n.c), wc = __ldg(w + n.c);
        const double um = __ldg(u + n.xm), vm = __ldg(v + n.ym), wm = __ldg(w + n.zm);
        dv = fabs((uc - um) * p.dx_inv + (vc - vm) * p.dy_inv + (wc - wm) * dzfi);
        cv = fabs((uc + um) * 0.5) * p.dx_inv + fabs((vc + vm) * 0.5) * p.dy_inv + fabs((wc + wm) * 0.5) * dzfi;
        const long long lin = (long long)i + (long long)p.nx * (j + (long long)p.ny * (k - 1));
        di = ci = lin;
        nan = (uc != uc) + (vc != vc) + (wc != wc);
        if (k == 1) nan += (__ldg(u + n.zm) != __ldg(u + n.zm)) + (vm != vm) + (wm != wm);
        if (k == p.nz)
            nan += (__ldg(u + n.zp) != __ldg(u + n.zp)) + (__ldg(v + n.zp) != __ldg(v + n.zp)) +
                   (__ldg(w + n.zp) != __ldg(w + n.zp));
        // NaN compares false: map a NaN residual to +inf so it is reported
        if (dv != dv) dv = __longlong_as_double(0x7ff0000000000000LL);
        if (cv != cv) cv = __longlong_as_double(0x7ff0000000000000LL);
    }
    for (int o = 16; o > 0; o >>= 1) {
        double odv = __shfl_down_sync(0xffffffffu, dv, o), ocv = __shfl_down_sync(0xffffffffu, cv, o);
        long long odi = __shfl_down_sync(0xffffffffu, di, o), oci = __shfl_down_sync(0xffffffffu, ci, o);
        nan += __shfl_down_sync(0xffffffffu, nan, o);
        better(dv, di, odv, odi);
        better(cv, ci, ocv, oci);
    }
    __shared__ double sd[32], sc[32], sn[32];
    __shared__ long long sdi[32], sci[32];
    const int t = threadIdx.x + threadIdx.y * blockDim.x, lane = t & 31, wid = t >> 5;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    if (lane == 0) {
        sd[wid] = dv;
        sc[wid] = cv;
        sn[wid] = nan;
        sdi[wid] = di;
        sci[wid] = ci;
    }
    __syncthreads();
    if (t == 0) {
        for (int q = 1; q < nw; q++) {
            better(dv, di, sd[q], sdi[q]);
            better(cv, ci, sc[q], sci[q]);
            nan += sn[q];
        }
        const size_t b = blockIdx.x + (size_t)gridDim.x * (blockIdx.y + (size_t)gridDim.y * blockIdx.z);
        const size_t nb = (size_t)gridDim.x * gridDim.y * gridDim.z;
        part[b] = dv;
        part[nb + b] = cv;
        part[2 * nb + b] = nan;
        ipart[b] = di;
        ipart[nb + b] = ci;
    }
}

// the block partials reduced by one CTA: max |div| and max CFL with the
// first location among equal values (better() is associative and
// commutative, so the tree gives the scan's result), the NaN count summed
// (whole numbers, exact in any order)
constexpr int DIAG_FIN_THREADS = 1024;
__global__ void __launch_bounds__(DIAG_FIN_THREADS) k_diag_finish(const double *part, const long long *ipart, int nb,
                                                                  StepParams p, double *out, int *loc)
{
    __shared__ double sdv[DIAG_FIN_THREADS], scv[DIAG_FIN_THREADS], snan[DIAG_FIN_THREADS];
    __shared__ long long sdi[DIAG_FIN_THREADS], sci[DIAG_FIN_THREADS];
    const int t = threadIdx.x;
    double dv = -1.0, cv = -1.0, nan = 0.0;
    long long di = 0x7fffffffffffffffLL, ci = 0x7fffffffffffffffLL;
    for (int b = t; b < nb; b += DIAG_FIN_THREADS) {
        better(dv, di, part[b], ipart[b]);
        better(cv, ci, part[nb + b], ipart[nb + b]);
        nan += part[2 * nb + b];
    }
    sdv[t] = dv;
    sdi[t] = di;
    scv[t] = cv;
    sci[t] = ci;
    snan[t] = nan;
    __syncthreads();
    for (int o = DIAG_FIN_THREADS / 2; o > 0; o >>= 1) {
        if (t < o) {
            better(sdv[t], sdi[t], sdv[t + o], sdi[t + o]);
            better(scv[t], sci[t], scv[t + o], sci[t + o]);
            snan[t] += snan[t + o];
        }
        __syncthreads();
    }
    if (t != 0) return;
    dv = sdv[0];
    di = sdi[0];
    cv = scv[0];
    ci = sci[0];
    out[0] = dv;
    out[1] = cv * p.dt;
    out[2] = snan[0];
    const long long nxy = (long long)p.nx * p.ny;
    loc[0] = (int)(di % p.nx) + 1;
    loc[1] = (int)((di / p.nx) % p.ny) + 1;
    loc[2] = (int)(di / nxy) + 1;
    loc[3] = (int)(ci % p.nx) + 1;
    loc[4] = (int)((ci / p.nx) % p.ny) + 1;
    loc[5] = (int)(ci / nxy) + 1;
}

// ------------------------------------------------------------------------
// initial field (mod_initFlow.f90:28-78 with the repository PRNG)
// ------------------------------------------------------------------------
__device__ __forceinline__ double splitmix_uniform(uint64_t seed, uint64_t n)
{
    uint64_t z = seed + (n + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void __launch_bounds__(256) k_init_fill(double *u, double *v, double *w, const double *prof,
                                                   uint64_t seed, double noise, StepParams p)
{
    PL_POINT_INDEX();
    const size_t c = (size_t)i + (size_t)p.nx * j + sk * k;
    // the counter is the point's global index, so a z slab draws the same
    // numbers as the whole domain
    const uint64_t nint = (uint64_t)p.nx * p.ny * (p.nzg > 0 ? p.nzg : p.nz);
    const uint64_t lin = (uint64_t)i + (uint64_t)p.nx * ((uint64_t)j + (uint64_t)p.ny * (uint64_t)(p.kofs + k - 1));
    // var + 2*(rn - 0.5)*norm (mod_initFlow.f90:372), rounded op by op like the
    // reference (no fused multiply-add)
    u[c] = __dadd_rn(__ldg(prof + k), __dmul_rn(__dmul_rn(2.0, splitmix_uniform(seed, lin) - 0.5), noise));
    v[c] = __dadd_rn(0.0, __dmul_rn(__dmul_rn(2.0, splitmix_uniform(seed, nint + lin) - 0.5), noise));
    w[c] = __dadd_rn(0.0, __dmul_rn(__dmul_rn(2.0, splitmix_uniform(seed, 2 * nint + lin) - 0.5), noise));
}

__global__ void __launch_bounds__(256) k_sum_comp(const double *__restrict__ var, StepParams p, MeshDev m,
                                                  double *partial, int comp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + 1;
    double s = 0.0, z0 = 0.0, z1 = 0.0;
    if (i < p.nx && j < p.ny) {
        const size_t c = (size_t)i + (size_t)p.nx * j + (size_t)p.nx * p.ny * k;
        s = __ldg(var + c) * __ldg(m.dzflzi + k);
    }
    block_sum3(s, z0, z1);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const size_t b = blockIdx.x + (size_t)gridDim.x * (blockIdx.y + (size_t)gridDim.y * blockIdx.z);
        const size_t nb = (size_t)gridDim.x * gridDim.y * gridDim.z;
        partial[(size_t)comp * nb + b] = s;
    }
}

// u = u/meanold*u_ref (if meanold != 0), transform2CRF u -= u_crf, wall fills
__global__ void __launch_bounds__(256) k_init_finish(double *u, double *v, double *w, StepParams p, double u_ref,
                                                     const double *scalar)
{
    PL_POINT_INDEX();
    const size_t c = (size_t)i + (size_t)p.nx * j + sk * k;
    const double meanold = scalar[0];
    double nu = u[c];
    if (meanold != 0.0) nu = nu / meanold * u_ref;
    nu = nu - p.u_crf;
    u[c] = nu;
    wall_fill<double>(u, v, w, c, k, sk, p.nz, 0.0 - p.u_crf, nu, v[c], p.wlo, p.whi);
}

__global__ void __launch_bounds__(256) k_fill_bc(double *u, double *v, double *w, StepParams p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= p.nx || j >= p.ny) return;
    const size_t sk = (size_t)p.nx * p.ny;
    const double bcu = 0.0 - p.u_crf;
    const size_t c1 = (size_t)i + (size_t)p.nx * j + sk, cn = c1 + sk * (p.nz - 1);
    u[c1 - sk] = 2.0 * bcu - u[c1];
    v[c1 - sk] = -v[c1];
    w[c1 - sk] = 0.0;
    u[cn + sk] = 2.0 * bcu - u[cn];
    v[cn + sk] = -v[cn];
    w[cn] = 0.0;
    w[cn + sk] = 0.0;
}

// RK2 (FP64) with the fused Mean_h of the new u
__global__ void __launch_bounds__(256) k_rk2m_fp64(double *u, double *v, double *w, const double *__restrict__ u1,
                                                   const double *__restrict__ v1, const double *__restrict__ w1,
                                                   StepParams p, MeshDev m, MeanRed red)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + 1;
    const size_t sk = (size_t)p.nx * p.ny;
    double su = 0.0;
    if (i < p.nx && j < p.ny) {
        const Nb n = neighbours(i, j, k, p.nx, p.ny);
        double ru, rv, rw;
        momentum_rhs<double>(LoadF<double, double>{u1}, LoadF<double, double>{v1}, LoadF<double, double>{w1}, n, k,
                             p, m, ru, rv, rw);
        const double nu = (__ldg(u1 + n.c) + p.dt * (ru + p.fb[0]) + u[n.c]) * 0.5;
        const double nv = (__ldg(v1 + n.c) + p.dt * (rv + p.fb[1]) + v[n.c]) * 0.5;
        u[n.c] = nu;
        v[n.c] = nv;
        if (k != p.nz) w[n.c] = (__ldg(w1 + n.c) + p.dt * (rw + p.fb[2]) + w[n.c]) * 0.5;
        wall_fill<double>(u, v, w, n.c, k, sk, p.nz, 0.0 - p.u_crf, nu, nv);
        su = nu * __ldg(m.dzflzi + k);
    }
    mean_reduce(su, red);
}


// ------------------------------------------------------------------------
// mixed precision (u, v, w, p in FP64; stage increments and PPE in FP32)
// ------------------------------------------------------------------------

// RK1: d1 = dt * (visc - conv)(u) in FP32, i.e. u1 = u + d1.  Wall fill of
// u1 (imposeNoSlipBC) in increment form: u1(0) = 2 bc - u1(1) and u(0) = 2 bc
// - u(1) give d1(0) = -d1(1); w1 = w = 0 on the walls gives d1w = 0 there.
__global__ void __launch_bounds__(256) k_rk1_mixed(const double *__restrict__ u, const double *__restrict__ v,
                                                   const double *__restrict__ w, float *__restrict__ du,
                                                   float *__restrict__ dv, float *__restrict__ dw, StepParams p,
                                                   MeshDev m)
{
    PL_POINT_INDEX();
    const Nb n = neighbours(i, j, k, p.nx, p.ny);
    float ru, rv, rw;
    momentum_rhs<float>(LoadF<double, float>{u}, LoadF<double, float>{v}, LoadF<double, float>{w}, n, k, p, m, ru,
                        rv, rw);
    const float dtf = (float)p.dt;
    const float a = dtf * ru, b = dtf * rv;
    du[n.c] = a;
    dv[n.c] = b;
    if (k != p.nz) dw[n.c] = dtf * rw;
    wall_fill<float>(du, dv, dw, n.c, k, sk, p.nz, 0.0f, a, b);
}

// RK2: u_new = (u1 + dt*(visc - conv)(u1) + u) * 0.5 with u1 = u + d1, the
// right-hand side in FP32 and the update in FP64; out of place (u is read
// at the neighbours to rebuild u1).  Fused Mean_h of u_new.
__global__ void __launch_bounds__(256) k_rk2_mixed(const double *__restrict__ u, const double *__restrict__ v,
                                                   const double *__restrict__ w, const float *__restrict__ du,
                                                   const float *__restrict__ dv, const float *__restrict__ dw,
                                                   double *__restrict__ uo, double *__restrict__ vo,
                                                   double *__restrict__ wo, StepParams p, MeshDev m, MeanRed red,
                                                   const float *__restrict__ pq, int pinc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + 1;
    const size_t sk = (size_t)p.nx * p.ny;
    double su = 0.0;
    if (i < p.nx && j < p.ny) {
        const Nb n = neighbours(i, j, k, p.nx, p.ny);
        float ru, rv, rw;
        momentum_rhs<float>(LoadSum{u, du}, LoadSum{v, dv}, LoadSum{w, dw}, n, k, p, m, ru, rv, rw);
        const float dtf = (float)p.dt;
        const double uc = __ldg(u + n.c), vc = __ldg(v + n.c), wc = __ldg(w + n.c);
        double nu = ((uc + (double)__ldg(du + n.c)) + (double)(dtf * ru) + uc) * 0.5;
        double nv = ((vc + (double)__ldg(dv + n.c)) + (double)(dtf * rv) + vc) * 0.5;
        double nw = ((wc + (double)__ldg(dw + n.c)) + (double)(dtf * rw) + wc) * 0.5;
        if (pinc) { // u_hat = u* - dt G p_pred (FP64): its divergence is the increment's residual
            const size_t pc = n.c - sk;
            const double q0 = __ldg(pq + pc), qxp = __ldg(pq + n.xp - sk), qyp = __ldg(pq + n.yp - sk);
            const double qzp = (k < p.nz) ? (double)__ldg(pq + pc + sk) : q0;
            nu = nu - (qxp - q0) * (p.dt * p.dx_inv);
            nv = nv - (qyp - q0) * (p.dt * p.dy_inv);
            nw = nw - (qzp - q0) * p.dt * __ldg(m.dzc_inv + k);
        }
        uo[n.c] = nu;
        vo[n.c] = nv;
        if (k != p.nz) wo[n.c] = nw;
        wall_fill<double>(uo, vo, wo, n.c, k, sk, p.nz, 0.0 - p.u_crf, nu, nv);
        su = nu * __ldg(m.dzflzi + k);
    }
    mean_reduce(su, red);
}

// Mixed residual: r = div(u)/dt in FP64, stored in FP32 (the increment's
// right-hand side), with the FP64 plane sums of r (the (kx,ky) = (0,0)
// right-hand side, solved in FP64).  For an incremental projection u is
// u_hat = u* - dt G p_pred (stored by the RK kernel), so r = div(u*)/dt -
// L p_pred, L being exactly the operator the PPE inverts; p_pred = 2 p_n -
// p_{n-1} makes r the second difference of p in time, and every FP32 error
// of the increment solve scales with |r|.
// Two adjacent points (i, i+1), i even, per thread: 16-byte loads of the
// u, v, w pairs and of the v and w pairs at j-1 and k-1, one float2 store,
// and one warp reduction per two points.  nx is even (the transforms pair
// lines), so every pair is 16-byte aligned and lies in one row.
constexpr int RHS_BX = 32, RHS_BY = 8; // threads; a block covers 64 x 8 points of a plane
__global__ void __launch_bounds__(RHS_BX *RHS_BY) k_rhs_mixed(const double *__restrict__ u, const double *__restrict__ v,
                                                              const double *__restrict__ w, float *__restrict__ r,
                                                              double *__restrict__ warp_part, StepParams p, MeshDev m)
{
    const int i = 2 * (blockIdx.x * RHS_BX + threadIdx.x);
    const int j = blockIdx.y * RHS_BY + threadIdx.y;
    const int k = blockIdx.z + 1;
    const size_t sk = (size_t)p.nx * p.ny;
    double val = 0.0;
    if (i < p.nx && j < p.ny) {
        const int im = (i == 0) ? p.nx - 1 : i - 1, jm = (j == 0) ? p.ny - 1 : j - 1;
        const size_t row = (size_t)p.nx * j + sk * k, c = row + i;
        const size_t ym = (size_t)p.nx * jm + sk * k + i;
        const double dti = 1.0 / p.dt, dtidxi = dti * p.dx_inv, dtidyi = dti * p.dy_inv;
        const double2 uc = __ldg(reinterpret_cast<const double2 *>(u + c));
        const double uxm = __ldg(u + row + im);
        const double2 vc = __ldg(reinterpret_cast<const double2 *>(v + c));
        const double2 vym = __ldg(reinterpret_cast<const double2 *>(v + ym));
        const double2 wc = __ldg(reinterpret_cast<const double2 *>(w + c));
        const double2 wzm = __ldg(reinterpret_cast<const double2 *>(w + c - sk));
        // the expressions of k_calc_rhs_fp64, per point
        const double r0 = (uc.x - uxm) * dtidxi + (vc.x - vym.x) * dtidyi + (wc.x - wzm.x) * dti * __ldg(m.dzf_inv + k);
        const double r1 = (uc.y - uc.x) * dtidxi + (vc.y - vym.y) * dtidyi + (wc.y - wzm.y) * dti * __ldg(m.dzf_inv + k);
        *reinterpret_cast<float2 *>(r + c - sk) = make_float2((float)r0, (float)r1);
        val = r0 + r1;
    }
    // warp partials (no block barrier); summed per plane in a fixed order
    for (int o = 16; o > 0; o >>= 1) val += __shfl_down_sync(0xffffffffu, val, o);
    const int t = threadIdx.x + threadIdx.y * RHS_BX;
    if ((t & 31) == 0) {
        constexpr int wpb = (RHS_BX * RHS_BY) >> 5;
        const size_t b = blockIdx.x + (size_t)gridDim.x * blockIdx.y;
        warp_part[((size_t)blockIdx.z * gridDim.x * gridDim.y + b) * wpb + (t >> 5)] = val;
    }
}

static inline dim3 rhs_mixed_grid(const StepParams &p)
{
    return dim3((p.nx / 2 + RHS_BX - 1) / RHS_BX, (p.ny + RHS_BY - 1) / RHS_BY, p.nz);
}

// correctVel + forceVel (shift from the fused mean) + wall fill, for two
// adjacent points (i, i+1), i even, per thread: the u, v, w pairs and the
// pressure pairs move as 16-byte (FP32 pressure: 8-byte) accesses (nx is
// even, so every pair is aligned and lies in one row).  Per point the
// expressions are correctVel's (mod_calcVel.f90:436-450) in its order.
template <typename TP> struct PairOf;
template <> struct PairOf<double> {
    using type = double2;
};
template <> struct PairOf<float> {
    using type = float2;
};

template <typename TP>
__global__ void __launch_bounds__(RHS_BX *RHS_BY) k_correct_force(const TP *__restrict__ pp, double *u, double *v,
                                                                   double *w, StepParams p, MeshDev m, int forced_x,
                                                                   const double *scalar)
{
    using P2 = typename PairOf<TP>::type;
    const int i = 2 * (blockIdx.x * RHS_BX + threadIdx.x);
    const int j = blockIdx.y * RHS_BY + threadIdx.y;
    const int k = blockIdx.z + 1;
    if (i >= p.nx || j >= p.ny) return;
    const size_t sk = (size_t)p.nx * p.ny;
    const int ip2 = (i + 2 == p.nx) ? 0 : i + 2, jp = (j == p.ny - 1) ? 0 : j + 1;
    const size_t c = (size_t)p.nx * j + sk * k + i, pc = c - sk;
    const double dt = p.dt, dtdxi = dt * p.dx_inv, dtdyi = dt * p.dy_inv;
    const P2 p0 = __ldg(reinterpret_cast<const P2 *>(pp + pc));
    const double p0a = (double)p0.x, p0b = (double)p0.y;
    const double pxpb = (double)__ldg(pp + (size_t)p.nx * j + sk * (k - 1) + ip2); // (i+2, j)
    const P2 py = __ldg(reinterpret_cast<const P2 *>(pp + (size_t)p.nx * jp + sk * (k - 1) + i));
    double pza = p0a, pzb = p0b;
    if (k < p.nz || !p.whi) { // at a slab interface plane nz + 1 is the neighbour's first (a halo)
        const P2 pz = __ldg(reinterpret_cast<const P2 *>(pp + pc + sk));
        pza = (double)pz.x;
        pzb = (double)pz.y;
    }
    const double2 uu = *reinterpret_cast<const double2 *>(u + c);
    const double2 vv = *reinterpret_cast<const double2 *>(v + c);
    const double2 ww = *reinterpret_cast<const double2 *>(w + c);
    double nua = uu.x - (p0b - p0a) * dtdxi, nub = uu.y - (pxpb - p0b) * dtdxi;
    if (forced_x) {
        nua = nua + __ldg(scalar + 3);
        nub = nub + __ldg(scalar + 3);
    }
    const double nva = vv.x - ((double)py.x - p0a) * dtdyi, nvb = vv.y - ((double)py.y - p0b) * dtdyi;
    const double dzi = __ldg(m.dzc_inv + k);
    const double nwa = ww.x - (pza - p0a) * dt * dzi, nwb = ww.y - (pzb - p0b) * dt * dzi;
    *reinterpret_cast<double2 *>(u + c) = make_double2(nua, nub);
    *reinterpret_cast<double2 *>(v + c) = make_double2(nva, nvb);
    *reinterpret_cast<double2 *>(w + c) = make_double2(nwa, nwb);
    const double bcu = 0.0 - p.u_crf;
    if (p.wlo && k == 1) {
        *reinterpret_cast<double2 *>(u + c - sk) = make_double2(2.0 * bcu - nua, 2.0 * bcu - nub);
        *reinterpret_cast<double2 *>(v + c - sk) = make_double2(-nva, -nvb);
    }
    if (p.whi && k == p.nz) {
        *reinterpret_cast<double2 *>(u + c + sk) = make_double2(2.0 * bcu - nua, 2.0 * bcu - nub);
        *reinterpret_cast<double2 *>(v + c + sk) = make_double2(-nva, -nvb);
    }
}

// per-plane sums of the warp partials (fixed order): mode0[k] = sum_ij r
__global__ void k_plane_sums(const double *part, int nper, int nz, double *mode0)
{
    const int k = blockIdx.x;
    if (k >= nz) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < nper; b += blockDim.x) s += part[(size_t)k * nper + b];
    __shared__ double sh[256];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) mode0[k] = sh[0];
}

// ------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------
static inline dim3 point_block() { return dim3(64, 4, 1); }
static inline dim3 point_grid(const StepParams &p)
{
    return dim3((p.nx + 63) / 64, (p.ny + 3) / 4, p.nz);
}

int launch_rk1_fp64(const double *u, const double *v, const double *w, double *u1, double *v1, double *w1,
                    const StepParams &p, const MeshDev &m, cudaStream_t st)
{
    k_rk1_fp64<<<point_grid(p), point_block(), 0, st>>>(u, v, w, u1, v1, w1, p, m);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_rk2_fp64(double *u, double *v, double *w, const double *u1, const double *v1, const double *w1,
                    const StepParams &p, const MeshDev &m, cudaStream_t st)
{
    k_rk2_fp64<<<point_grid(p), point_block(), 0, st>>>(u, v, w, u1, v1, w1, p, m);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_calc_rhs_fp64(const double *u, const double *v, const double *w, double *rhs, const StepParams &p,
                         const MeshDev &m, cudaStream_t st)
{
    k_calc_rhs_fp64<<<point_grid(p), point_block(), 0, st>>>(u, v, w, rhs, p, m);
    PL_CHECK_LAUNCH();
    return 0;
}

static int nblocks(const StepParams &p)
{
    dim3 g = point_grid(p);
    return (int)(g.x * g.y * g.z);
}

int launch_correct_fp64(const double *p_, double *u, double *v, double *w, const StepParams &p, const MeshDev &m,
                        const int forced[3], ReduceBuf &rb, cudaStream_t st)
{
    (void)forced;
    if (nblocks(p) > rb.max_blocks) {
        set_error("reduction buffer too small");
        return -1;
    }
    k_correct<double><<<point_grid(p), point_block(), 0, st>>>(p_, u, v, w, p, m, rb.partial);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_force_fp64(double *u, double *v, double *w, const StepParams &p, const int forced[3],
                      const double vel_force[3], ReduceBuf &rb, cudaStream_t st)
{
    if (!(forced[0] || forced[1] || forced[2])) return 0;
    k_finish_means<<<3, 1024, 0, st>>>(rb.partial, nblocks(p), (double)p.nx, (double)p.ny, vel_force[0], vel_force[1],
                                       vel_force[2], rb.scalar);
    PL_CHECK_LAUNCH();
    k_force<<<point_grid(p), point_block(), 0, st>>>(u, v, w, p, forced[0], forced[1], forced[2], rb.scalar);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_diagnostics_fp64(const double *u, const double *v, const double *w, const StepParams &p,
                            const MeshDev &m, double *d_out, int *d_loc, double *d_part, long long *d_ipart,
                            int max_blocks, cudaStream_t st)
{
    if (nblocks(p) > max_blocks) {
        set_error("diagnostics buffer too small");
        return -1;
    }
    k_diag<<<point_grid(p), point_block(), 0, st>>>(u, v, w, p, m, d_part, d_ipart);
    PL_CHECK_LAUNCH();
    k_diag_finish<<<1, DIAG_FIN_THREADS, 0, st>>>(d_part, d_ipart, nblocks(p), p, d_out, d_loc);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_init_fill(double *u, double *v, double *w, const double *prof, uint64_t seed, double noise,
                     const StepParams &p, cudaStream_t st)
{
    k_init_fill<<<point_grid(p), point_block(), 0, st>>>(u, v, w, prof, seed, noise, p);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_mean_sum(const double *var, const StepParams &p, const MeshDev &m, ReduceBuf &rb, int comp,
                    cudaStream_t st)
{
    if (nblocks(p) > rb.max_blocks) {
        set_error("reduction buffer too small");
        return -1;
    }
    k_sum_comp<<<point_grid(p), point_block(), 0, st>>>(var, p, m, rb.partial, comp);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_init_finish(double *u, double *v, double *w, const StepParams &p, double u_ref, ReduceBuf &rb,
                       cudaStream_t st)
{
    k_finish_means<<<3, 1024, 0, st>>>(rb.partial, nblocks(p), (double)p.nx, (double)p.ny, 0.0, 0.0, 0.0, rb.scalar);
    PL_CHECK_LAUNCH();
    k_init_finish<<<point_grid(p), point_block(), 0, st>>>(u, v, w, p, u_ref, rb.scalar);
    PL_CHECK_LAUNCH();
    return 0;
}

// Mean_h from the sum of u dzf/lz over all z slabs (scalar[6], summed across
// the ranks by the caller): scalar[0] = Mean_h, scalar[3] = vel_force - Mean_h
__global__ void k_mean_from_sum(double *scalar, double dnx, double dny, double vel_force)
{
    const double mean = scalar[6] / dnx / dny;
    scalar[0] = mean;
    scalar[3] = vel_force - mean;
}

int launch_mean_from_sum(double *scalar, const StepParams &p, double vel_force, cudaStream_t st)
{
    k_mean_from_sum<<<1, 1, 0, st>>>(scalar, (double)p.nx, (double)p.ny, vel_force);
    PL_CHECK_LAUNCH();
    return 0;
}

// the block partials of launch_mean_sum (component 0) reduced: scalar[0] =
// this grid's Mean_h, scalar[6] = its sum
int launch_mean_partials(const StepParams &p, ReduceBuf &rb, cudaStream_t st)
{
    k_finish_means<<<1, 1024, 0, st>>>(rb.partial, nblocks(p), (double)p.nx, (double)p.ny, 0.0, 0.0, 0.0, rb.scalar);
    PL_CHECK_LAUNCH();
    return 0;
}

// initial-field normalisation u / Mean_h(u) u_ref from the summed scalar[6]
int launch_init_finish_sum(double *u, double *v, double *w, const StepParams &p, double u_ref, ReduceBuf &rb,
                           cudaStream_t st)
{
    k_mean_from_sum<<<1, 1, 0, st>>>(rb.scalar, (double)p.nx, (double)p.ny, 0.0);
    PL_CHECK_LAUNCH();
    k_init_finish<<<point_grid(p), point_block(), 0, st>>>(u, v, w, p, u_ref, rb.scalar);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_fill_bc_vel(double *u, double *v, double *w, const StepParams &p, cudaStream_t st)
{
    dim3 g((p.nx + 63) / 64, (p.ny + 3) / 4, 1);
    k_fill_bc<<<g, point_block(), 0, st>>>(u, v, w, p);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_rk2m_fp64(double *u, double *v, double *w, const double *u1, const double *v1, const double *w1,
                     const StepParams &p, const MeshDev &m, MeanState &ms, cudaStream_t st)
{
    if (nblocks(p) > ms.max_blocks) {
        set_error("mean buffer too small");
        return -1;
    }
    MeanRed r{ms.partial, ms.counter, ms.scalar, (double)p.nx, (double)p.ny, ms.vel_force};
    k_rk2m_fp64<<<point_grid(p), point_block(), 0, st>>>(u, v, w, u1, v1, w1, p, m, r);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_correct_force_fp64(const double *p_, double *u, double *v, double *w, const StepParams &p,
                              const MeshDev &m, int forced_x, const double *scalar, cudaStream_t st)
{
    k_correct_force<double><<<rhs_mixed_grid(p), dim3(RHS_BX, RHS_BY), 0, st>>>(p_, u, v, w, p, m, forced_x, scalar);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_correct_force_f32(const float *p_, double *u, double *v, double *w, const StepParams &p, const MeshDev &m,
                             int forced_x, const double *scalar, cudaStream_t st)
{
    k_correct_force<float><<<rhs_mixed_grid(p), dim3(RHS_BX, RHS_BY), 0, st>>>(p_, u, v, w, p, m, forced_x, scalar);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_rk1_mixed(const double *u, const double *v, const double *w, float *d1u, float *d1v, float *d1w,
                     const StepParams &p, const MeshDev &m, cudaStream_t st)
{
    k_rk1_mixed<<<point_grid(p), point_block(), 0, st>>>(u, v, w, d1u, d1v, d1w, p, m);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_rk2_mixed(const double *u, const double *v, const double *w, const float *d1u, const float *d1v,
                     const float *d1w, double *uo, double *vo, double *wo, const StepParams &p, const MeshDev &m,
                     MeanState &ms, const float *pq, int pinc, cudaStream_t st)
{
    if (nblocks(p) > ms.max_blocks) {
        set_error("mean buffer too small");
        return -1;
    }
    MeanRed r{ms.partial, ms.counter, ms.scalar, (double)p.nx, (double)p.ny, ms.vel_force};
    k_rk2_mixed<<<point_grid(p), point_block(), 0, st>>>(u, v, w, d1u, d1v, d1w, uo, vo, wo, p, m, r, pq, pinc);
    PL_CHECK_LAUNCH();
    return 0;
}

int warp_partials_per_plane(const StepParams &p)
{
    const dim3 g = rhs_mixed_grid(p);
    return (int)(g.x * g.y) * ((RHS_BX * RHS_BY) / 32);
}

int launch_plane_sums(const double *part, int nper, int nz, double *mode0, cudaStream_t st)
{
    k_plane_sums<<<nz, 256, 0, st>>>(part, nper, nz, mode0);
    PL_CHECK_LAUNCH();
    return 0;
}

int launch_rhs_mixed(const double *u, const double *v, const double *w, float *r, double *warp_part, double *mode0,
                     const StepParams &p, const MeshDev &m, cudaStream_t st)
{
    if (p.nx % 2 != 0) {
        set_error("the mixed right-hand side needs an even nx");
        return -1;
    }
    k_rhs_mixed<<<rhs_mixed_grid(p), dim3(RHS_BX, RHS_BY), 0, st>>>(u, v, w, r, warp_part, p, m);
    PL_CHECK_LAUNCH();
    k_plane_sums<<<p.nz, 256, 0, st>>>(warp_part, warp_partials_per_plane(p), p.nz, mode0);
    PL_CHECK_LAUNCH();
    return 0;
}

} // namespace pl
