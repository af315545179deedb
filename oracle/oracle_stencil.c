/*
 * oracle_stencil.c -- restatement of the Fortran side of the RK2 projection
 * step for one rank.  TEST INFRASTRUCTURE ONLY.
 *
 * Fortran array u(0:nx+1, 0:ny+1, 0:nz+1) maps to u[IX(i,j,k)] with the same
 * (i,j,k).  Every function follows the cited reference lines statement by
 * statement, in the same floating-point evaluation order; OpenMP reductions
 * (Mean_h, calcMaxDiv) are summed/scanned sequentially in k, j, i order.
 *
 * Parity of this file is pinned only indirectly (no Fortran compiler exists in
 * this environment and the reference ships no test vectors): by the
 * manufactured-solution and invariant tests in tests/ (consistency of each
 * stencil with its continuous operator, discrete div(grad p) = Poisson
 * operator, projection to round-off divergence) and by agreement with the
 * independently written CUDA kernels.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define IX(i, j, k) ((size_t)(i) + (size_t)(g->nx + 2) * ((size_t)(j) + (size_t)(g->ny + 2) * (size_t)(k)))

int orc_grid_init(orc_grid *g, int nx, int ny, int nz, double lx, double ly, double lz, int mesh_type,
                  int stretch_func, double stretch, double re, double u_ref, double l_ref, double dt,
                  double u_crf, const int is_forced[3], const double vel_force[3])
{
    memset(g, 0, sizeof(*g));
    g->nx = nx;
    g->ny = ny;
    g->nz = nz;
    g->lx = lx;
    g->ly = ly;
    g->lz = lz;
    g->re = re;
    g->u_ref = u_ref;
    g->l_ref = l_ref;
    g->re_inv = u_ref * l_ref / re; /* mod_parameters.f90:187 */
    g->dt = dt;
    g->u_crf = u_crf;
    for (int d = 0; d < 3; d++) {
        g->is_forced[d] = is_forced[d];
        g->vel_force[d] = vel_force[d];
    }
    const int n1 = nz + 2;
    g->dzf_global = (double *)calloc(n1, sizeof(double));
    g->zc_global = (double *)calloc(n1, sizeof(double));
    g->dzf = (double *)calloc(n1, sizeof(double));
    g->dzf_inv = (double *)calloc(n1, sizeof(double));
    g->dzc = (double *)calloc(n1, sizeof(double));
    g->dzc_inv = (double *)calloc(n1, sizeof(double));
    g->dzflzi = (double *)calloc(n1, sizeof(double));

    /* mod_mesh.f90:42-45 */
    g->dx = lx / nx;
    g->dy = ly / ny;
    g->dx_inv = 1.0 / g->dx;
    g->dy_inv = 1.0 / g->dy;

    /* initMeshByFunc, mod_mesh.f90:130-159 */
    const double pi = acos(-1.0);
    double *dzf = g->dzf_global;
    if (stretch == 0.0 || mesh_type == 0) {
        for (int k = 0; k < n1; k++) dzf[k] = lz / nz;
    } else {
        double *zf = (double *)calloc(nz + 1, sizeof(double));
        zf[0] = 0.0;
        for (int k = 1; k <= nz; k++) {
            double z0 = k / (1.0 * nz);
            if (stretch_func == 0)
                zf[k] = 0.5 * (1.0 + tanh((z0 - 0.5) * stretch) / tanh(stretch / 2.0));
            else
                zf[k] = 0.5 * (1.0 + sin((z0 - 0.5) * stretch * pi) / sin(stretch * pi / 2.0));
        }
        for (int k = 1; k <= nz; k++) dzf[k] = lz * (zf[k] - zf[k - 1]);
        dzf[0] = dzf[1];
        dzf[nz + 1] = dzf[nz];
        free(zf);
    }
    /* mod_mesh.f90:60-72 (one rank: st(3) = 1, sz(3) = nz) */
    g->zc_global[0] = -0.5 * dzf[0];
    for (int k = 1; k <= nz + 1; k++) g->zc_global[k] = g->zc_global[k - 1] + 0.5 * (dzf[k - 1] + dzf[k]);
    for (int k = 0; k <= nz + 1; k++) {
        g->dzf[k] = dzf[k];
        g->dzf_inv[k] = 1.0 / g->dzf[k];
    }
    for (int k = 0; k <= nz; k++) {
        g->dzc[k] = 0.5 * (g->dzf[k] + g->dzf[k + 1]);
        g->dzc_inv[k] = 1.0 / g->dzc[k];
    }
    /* dzc(nz+1) is never assigned by the reference and never read */
    g->dzc[nz + 1] = g->dzc[nz];
    g->dzc_inv[nz + 1] = g->dzc_inv[nz];
    for (int k = 0; k <= nz + 1; k++) g->dzflzi[k] = g->dzf[k] / lz;
    return 0;
}

void orc_grid_free(orc_grid *g)
{
    free(g->dzf_global);
    free(g->zc_global);
    free(g->dzf);
    free(g->dzf_inv);
    free(g->dzc);
    free(g->dzc_inv);
    free(g->dzflzi);
    memset(g, 0, sizeof(*g));
}

double orc_uniform(uint64_t seed, uint64_t n)
{
    uint64_t z = seed + (n + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* ---- boundary fills (mod_updateBound.f90) ----------------------------- */

/* y: periodic self-exchange of updateHalo (:364-396, south/north at :378-383)
 * over all i, all k; x: imposePeriodicBC idir=1 (:241-272) over all j, k */
static void periodic_xy(const orc_grid *g, double *var)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    for (int k = 0; k <= nz + 1; k++)
        for (int i = 0; i <= nx + 1; i++) {
            var[IX(i, ny + 1, k)] = var[IX(i, 1, k)];
            var[IX(i, 0, k)] = var[IX(i, ny, k)];
        }
    for (int k = 0; k <= nz + 1; k++)
        for (int j = 0; j <= ny + 1; j++) {
            var[IX(0, j, k)] = var[IX(nx, j, k)];
            var[IX(nx + 1, j, k)] = var[IX(1, j, k)];
        }
}

/* imposeNoSlipBC (:274-330) */
static void noslip(const orc_grid *g, int ibound, int centered, double *var, double bcvalue)
{
    const int nx = g->nx, ny = g->ny, n = g->nz;
    for (int j = 0; j <= ny + 1; j++)
        for (int i = 0; i <= nx + 1; i++) {
            if (ibound == 0) {
                if (centered)
                    var[IX(i, j, 0)] = 2.0 * bcvalue - var[IX(i, j, 1)];
                else
                    var[IX(i, j, 0)] = bcvalue;
            } else {
                if (centered)
                    var[IX(i, j, n + 1)] = 2.0 * bcvalue - var[IX(i, j, n)];
                else {
                    var[IX(i, j, n)] = bcvalue;
                    var[IX(i, j, n + 1)] = bcvalue;
                }
            }
        }
}

/* updateBoundVel (:30-55) = updateHalo + imposeBCVel (:57-108) */
void orc_update_bound_vel(const orc_grid *g, double *u, double *v, double *w)
{
    periodic_xy(g, u);
    periodic_xy(g, v);
    periodic_xy(g, w);
    const double bc_u = 0.0 - g->u_crf;
    noslip(g, 0, 1, u, bc_u);
    noslip(g, 0, 1, v, 0.0);
    noslip(g, 0, 0, w, 0.0);
    noslip(g, 1, 1, u, bc_u);
    noslip(g, 1, 1, v, 0.0);
    noslip(g, 1, 0, w, 0.0);
}

/* updateBoundP (:186-239) with imposeZeroGradBC (:332-362) */
void orc_update_bound_p(const orc_grid *g, double *p)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    periodic_xy(g, p);
    for (int j = 0; j <= ny + 1; j++)
        for (int i = 0; i <= nx + 1; i++) {
            p[IX(i, j, 0)] = p[IX(i, j, 1)];
        }
    for (int j = 0; j <= ny + 1; j++)
        for (int i = 0; i <= nx + 1; i++) {
            p[IX(i, j, nz + 1)] = p[IX(i, j, nz)];
        }
}

/* ---- momentum stencils (mod_calcVel.f90) ------------------------------ */

/* the three momentum right-hand sides, timeIntVelRK1_kernel :74-138 (and
 * identically timeIntVelRK2_kernel :262-326), evaluated on (u,v,w) */
static inline void rhs_uvw(const orc_grid *g, const double *u, const double *v, const double *w, int i, int j, int k,
                           double *ru, double *rv, double *rw)
{
    const double dx_inv = g->dx_inv, dy_inv = g->dy_inv, re_inv = g->re_inv, u_crf = g->u_crf;
    const double *dzf = g->dzf, *dzc_inv = g->dzc_inv, *dzf_inv = g->dzf_inv;
    double conv, visc;
    double uw, ue, us, un, ub, ut, ww, we, ws, wn, wb, wt, vw, ve, vs, vn, vb, vt;
    double dqw, dqe, dqs, dqn, dqb, dqt;

    ue = (u[IX(i, j, k)] + u[IX(i + 1, j, k)]);
    uw = (u[IX(i - 1, j, k)] + u[IX(i, j, k)]);
    un = (u[IX(i, j, k)] + u[IX(i, j + 1, k)]);
    us = (u[IX(i, j - 1, k)] + u[IX(i, j, k)]);
    ut = (u[IX(i, j, k)] * dzf[k + 1] + u[IX(i, j, k + 1)] * dzf[k]) * dzc_inv[k];
    ub = (u[IX(i, j, k)] * dzf[k - 1] + u[IX(i, j, k - 1)] * dzf[k]) * dzc_inv[k - 1];
    vn = (v[IX(i, j, k)] + v[IX(i + 1, j, k)]);
    vs = (v[IX(i, j - 1, k)] + v[IX(i + 1, j - 1, k)]);
    wt = (w[IX(i, j, k)] + w[IX(i + 1, j, k)]);
    wb = (w[IX(i, j, k - 1)] + w[IX(i + 1, j, k - 1)]);
    dqe = (u[IX(i + 1, j, k)] - u[IX(i, j, k)]) * dx_inv;
    dqw = (u[IX(i, j, k)] - u[IX(i - 1, j, k)]) * dx_inv;
    dqn = (u[IX(i, j + 1, k)] - u[IX(i, j, k)]) * dy_inv;
    dqs = (u[IX(i, j, k)] - u[IX(i, j - 1, k)]) * dy_inv;
    dqt = (u[IX(i, j, k + 1)] - u[IX(i, j, k)]) * dzc_inv[k];
    dqb = (u[IX(i, j, k)] - u[IX(i, j, k - 1)]) * dzc_inv[k - 1];
    conv = 0.25 * ((ue * ue - uw * uw) * dx_inv + (un * vn - us * vs) * dy_inv + (ut * wt - ub * wb) * dzf_inv[k]);
    conv = conv + 0.5 * u_crf * (ue - uw) * dx_inv;
    visc = ((dqe - dqw) * dx_inv + (dqn - dqs) * dy_inv + (dqt - dqb) * dzf_inv[k]) * re_inv;
    *ru = visc - conv;

    ve = (v[IX(i, j, k)] + v[IX(i + 1, j, k)]);
    vw = (v[IX(i - 1, j, k)] + v[IX(i, j, k)]);
    vn = (v[IX(i, j, k)] + v[IX(i, j + 1, k)]);
    vs = (v[IX(i, j - 1, k)] + v[IX(i, j, k)]);
    vt = (v[IX(i, j, k)] * dzf[k + 1] + v[IX(i, j, k + 1)] * dzf[k]) * dzc_inv[k];
    vb = (v[IX(i, j, k)] * dzf[k - 1] + v[IX(i, j, k - 1)] * dzf[k]) * dzc_inv[k - 1];
    ue = (u[IX(i, j, k)] + u[IX(i, j + 1, k)]);
    uw = (u[IX(i - 1, j, k)] + u[IX(i - 1, j + 1, k)]);
    wt = (w[IX(i, j, k)] + w[IX(i, j + 1, k)]);
    wb = (w[IX(i, j, k - 1)] + w[IX(i, j + 1, k - 1)]);
    dqe = (v[IX(i + 1, j, k)] - v[IX(i, j, k)]) * dx_inv;
    dqw = (v[IX(i, j, k)] - v[IX(i - 1, j, k)]) * dx_inv;
    dqn = (v[IX(i, j + 1, k)] - v[IX(i, j, k)]) * dy_inv;
    dqs = (v[IX(i, j, k)] - v[IX(i, j - 1, k)]) * dy_inv;
    dqt = (v[IX(i, j, k + 1)] - v[IX(i, j, k)]) * dzc_inv[k];
    dqb = (v[IX(i, j, k)] - v[IX(i, j, k - 1)]) * dzc_inv[k - 1];
    conv = 0.25 * ((ue * ve - uw * vw) * dx_inv + (vn * vn - vs * vs) * dy_inv + (wt * vt - wb * vb) * dzf_inv[k]);
    conv = conv + 0.5 * u_crf * (ve - vw) * dx_inv;
    visc = ((dqe - dqw) * dx_inv + (dqn - dqs) * dy_inv + (dqt - dqb) * dzf_inv[k]) * re_inv;
    *rv = visc - conv;

    we = (w[IX(i, j, k)] + w[IX(i + 1, j, k)]);
    ww = (w[IX(i - 1, j, k)] + w[IX(i, j, k)]);
    wn = (w[IX(i, j, k)] + w[IX(i, j + 1, k)]);
    ws = (w[IX(i, j - 1, k)] + w[IX(i, j, k)]);
    wt = (w[IX(i, j, k)] + w[IX(i, j, k + 1)]);
    wb = (w[IX(i, j, k)] + w[IX(i, j, k - 1)]);
    ue = (u[IX(i, j, k)] * dzf[k + 1] + u[IX(i, j, k + 1)] * dzf[k]) * dzc_inv[k];
    uw = (u[IX(i - 1, j, k)] * dzf[k + 1] + u[IX(i - 1, j, k + 1)] * dzf[k]) * dzc_inv[k];
    vn = (v[IX(i, j, k)] * dzf[k + 1] + v[IX(i, j, k + 1)] * dzf[k]) * dzc_inv[k];
    vs = (v[IX(i, j - 1, k)] * dzf[k + 1] + v[IX(i, j - 1, k + 1)] * dzf[k]) * dzc_inv[k];
    dqe = (w[IX(i + 1, j, k)] - w[IX(i, j, k)]) * dx_inv;
    dqw = (w[IX(i, j, k)] - w[IX(i - 1, j, k)]) * dx_inv;
    dqn = (w[IX(i, j + 1, k)] - w[IX(i, j, k)]) * dy_inv;
    dqs = (w[IX(i, j, k)] - w[IX(i, j - 1, k)]) * dy_inv;
    dqt = (w[IX(i, j, k + 1)] - w[IX(i, j, k)]) * dzf_inv[k + 1];
    dqb = (w[IX(i, j, k)] - w[IX(i, j, k - 1)]) * dzf_inv[k];
    conv = 0.25 * ((ue * we - uw * ww) * dx_inv + (vn * wn - vs * ws) * dy_inv + (wt * wt - wb * wb) * dzc_inv[k]);
    conv = conv + 0.5 * u_crf * (we - ww) * dx_inv;
    visc = ((dqe - dqw) * dx_inv + (dqn - dqs) * dy_inv + (dqt - dqb) * dzc_inv[k]) * re_inv;
    *rw = visc - conv;
}

/* timeIntVelRK1_kernel (:52-146): u1 = u + dt*(visc - conv) */
void orc_rk1(const orc_grid *g, const double *u, const double *v, const double *w, double *u1, double *v1,
             double *w1)
{
    const double dt = g->dt;
    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= g->nz; k++)
        for (int j = 1; j <= g->ny; j++)
            for (int i = 1; i <= g->nx; i++) {
                double ru, rv, rw;
                rhs_uvw(g, u, v, w, i, j, k, &ru, &rv, &rw);
                u1[IX(i, j, k)] = u[IX(i, j, k)] + dt * ru;
                v1[IX(i, j, k)] = v[IX(i, j, k)] + dt * rv;
                w1[IX(i, j, k)] = w[IX(i, j, k)] + dt * rw;
            }
}

/* timeIntVelRK2_kernel (:240-334): u = (u1 + dt*(visc - conv)(u1) + u)/2 */
void orc_rk2(const orc_grid *g, double *u, double *v, double *w, const double *u1, const double *v1,
             const double *w1)
{
    const double dt = g->dt;
    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= g->nz; k++)
        for (int j = 1; j <= g->ny; j++)
            for (int i = 1; i <= g->nx; i++) {
                double ru, rv, rw;
                rhs_uvw(g, u1, v1, w1, i, j, k, &ru, &rv, &rw);
                u[IX(i, j, k)] = (u1[IX(i, j, k)] + dt * ru + u[IX(i, j, k)]) * 0.5;
                v[IX(i, j, k)] = (v1[IX(i, j, k)] + dt * rv + v[IX(i, j, k)]) * 0.5;
                w[IX(i, j, k)] = (w1[IX(i, j, k)] + dt * rw + w[IX(i, j, k)]) * 0.5;
            }
}

/* calcRHS, mod_calcRHS.f90:11-36 (into the interior of p) */
void orc_calc_rhs(const orc_grid *g, const double *u, const double *v, const double *w, double *rhs)
{
    const double dti = 1.0 / g->dt, dtidxi = dti * g->dx_inv, dtidyi = dti * g->dy_inv;
    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= g->nz; k++)
        for (int j = 1; j <= g->ny; j++)
            for (int i = 1; i <= g->nx; i++)
                rhs[IX(i, j, k)] = (u[IX(i, j, k)] - u[IX(i - 1, j, k)]) * dtidxi +
                                   (v[IX(i, j, k)] - v[IX(i, j - 1, k)]) * dtidyi +
                                   (w[IX(i, j, k)] - w[IX(i, j, k - 1)]) * dti * g->dzf_inv[k];
}

/* correctVel, mod_calcVel.f90:428-453 */
void orc_correct_vel(const orc_grid *g, const double *p, double *u, double *v, double *w)
{
    const double dt = g->dt, dtdxi = dt * g->dx_inv, dtdyi = dt * g->dy_inv;
    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= g->nz; k++)
        for (int j = 1; j <= g->ny; j++)
            for (int i = 1; i <= g->nx; i++) {
                u[IX(i, j, k)] = u[IX(i, j, k)] - (p[IX(i + 1, j, k)] - p[IX(i, j, k)]) * dtdxi;
                v[IX(i, j, k)] = v[IX(i, j, k)] - (p[IX(i, j + 1, k)] - p[IX(i, j, k)]) * dtdyi;
                w[IX(i, j, k)] = w[IX(i, j, k)] - (p[IX(i, j, k + 1)] - p[IX(i, j, k)]) * dt * g->dzc_inv[k];
            }
}

/* Mean_h, mod_utils.f90:105-131 (one rank: the ALLREDUCE is the identity) */
double orc_mean_h(const orc_grid *g, const double *var)
{
    /* the reference sums with an OpenMP reduction over k (thread-count
     * dependent order); here each k-plane is summed in j, i order and the
     * plane sums are added in k order, for any thread count */
    double *plane = (double *)calloc((size_t)g->nz + 1, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= g->nz; k++) {
        double s = 0.0;
        for (int j = 1; j <= g->ny; j++)
            for (int i = 1; i <= g->nx; i++) s = s + var[IX(i, j, k)] * g->dzflzi[k];
        plane[k] = s;
    }
    double m = 0.0;
    for (int k = 1; k <= g->nz; k++) m = m + plane[k];
    free(plane);
    m = m / g->nx / g->ny;
    return m;
}

/* forceVel, mod_calcVel.f90:455-509 */
void orc_force_vel(const orc_grid *g, double *u, double *v, double *w)
{
    double *f[3] = {u, v, w};
    for (int d = 0; d < 3; d++) {
        if (!g->is_forced[d]) continue;
        double mean = orc_mean_h(g, f[d]);
        double force = g->vel_force[d] - mean;
        #pragma omp parallel for schedule(static)
        for (int k = 1; k <= g->nz; k++)
            for (int j = 1; j <= g->ny; j++)
                for (int i = 1; i <= g->nx; i++) f[d][IX(i, j, k)] = f[d][IX(i, j, k)] + force;
    }
}

/* calcMaxDiv, mod_utils.f90:257-318 (first strict maximum in k,j,i order) */
double orc_max_div(const orc_grid *g, const double *u, const double *v, const double *w, int ijk[3])
{
    double mx = 0.0;
    int bi = 1, bj = 1, bk = 1;
    for (int k = 1; k <= g->nz; k++)
        for (int j = 1; j <= g->ny; j++)
            for (int i = 1; i <= g->nx; i++) {
                double d = fabs((u[IX(i, j, k)] - u[IX(i - 1, j, k)]) * g->dx_inv +
                                (v[IX(i, j, k)] - v[IX(i, j - 1, k)]) * g->dy_inv +
                                (w[IX(i, j, k)] - w[IX(i, j, k - 1)]) * g->dzf_inv[k]);
                if (d > mx) {
                    mx = d;
                    bi = i;
                    bj = j;
                    bk = k;
                }
            }
    if (ijk) {
        ijk[0] = bi;
        ijk[1] = bj;
        ijk[2] = bk;
    }
    return mx;
}

/* calcMaxCFL, mod_utils.f90:193-255 */
double orc_max_cfl(const orc_grid *g, const double *u, const double *v, const double *w, int ijk[3])
{
    double mx = 0.0;
    int bi = 1, bj = 1, bk = 1;
    for (int k = 1; k <= g->nz; k++)
        for (int j = 1; j <= g->ny; j++)
            for (int i = 1; i <= g->nx; i++) {
                double c = fabs((u[IX(i, j, k)] + u[IX(i - 1, j, k)]) * 0.5) * g->dx_inv +
                           fabs((v[IX(i, j, k)] + v[IX(i, j - 1, k)]) * 0.5) * g->dy_inv +
                           fabs((w[IX(i, j, k)] + w[IX(i, j, k - 1)]) * 0.5) * g->dzf_inv[k];
                if (c > mx) {
                    mx = c;
                    bi = i;
                    bj = j;
                    bk = k;
                }
            }
    if (ijk) {
        ijk[0] = bi;
        ijk[1] = bj;
        ijk[2] = bk;
    }
    return mx * g->dt;
}

/* checkNaN, mod_utils.f90:352-394 (whole array, ghosts included) */
int orc_has_nan(const orc_grid *g, const double *var)
{
    size_t n = (size_t)(g->nx + 2) * (g->ny + 2) * (g->nz + 2);
    for (size_t q = 0; q < n; q++)
        if (var[q] != var[q]) return 1;
    return 0;
}

/* initFlow, mod_initFlow.f90:28-78 ('poi', init_with_noise), then
 * transform2CRF and updateBoundVel/updateBoundP (main.f90:98-102).  The
 * gfortran random_number stream (seeds 123/456/789) is replaced by one
 * SplitMix64 stream: u, then v, then w, each interior i-fastest. */
void orc_init_flow(const orc_grid *g, uint64_t seed, double noise, double *u, double *v, double *w, double *p)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const size_t ng = (size_t)(nx + 2) * (ny + 2) * (nz + 2), nint = (size_t)nx * ny * nz;
    memset(u, 0, sizeof(double) * ng);
    memset(v, 0, sizeof(double) * ng);
    memset(w, 0, sizeof(double) * ng);
    memset(p, 0, sizeof(double) * ng);
    for (int k = 1; k <= nz; k++) {
        double zn = g->zc_global[k] / g->lz;
        double prof = 6.0 * (1.0 - zn) * zn * g->u_ref;
        for (int j = 1; j <= ny; j++)
            for (int i = 1; i <= nx; i++) u[IX(i, j, k)] = prof;
    }
    double *f[3] = {u, v, w};
    for (int d = 0; d < 3; d++)
        for (int k = 1; k <= nz; k++)
            for (int j = 1; j <= ny; j++)
                for (int i = 1; i <= nx; i++) {
                    uint64_t n = (uint64_t)d * nint + (uint64_t)(i - 1) + (uint64_t)nx * ((uint64_t)(j - 1) + (uint64_t)ny * (uint64_t)(k - 1));
                    double rn = orc_uniform(seed, n);
                    f[d][IX(i, j, k)] = f[d][IX(i, j, k)] + 2.0 * (rn - 0.5) * noise;
                }
    double meanold = orc_mean_h(g, u);
    if (meanold != 0.0)
        for (int k = 1; k <= nz; k++)
            for (int j = 1; j <= ny; j++)
                for (int i = 1; i <= nx; i++) u[IX(i, j, k)] = u[IX(i, j, k)] / meanold * g->u_ref;
    for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
            for (int i = 1; i <= nx; i++) u[IX(i, j, k)] = u[IX(i, j, k)] - g->u_crf;
    orc_update_bound_vel(g, u, v, w);
    orc_update_bound_p(g, p);
}

/* main.f90:137-208, blocking-halo build (identical values to NB_HALO on one
 * rank: the non-blocking path only reorders the same copies). */
void orc_step(const orc_grid *g, orc_ppe_fn ppe, void *ppe_ctx, double *u, double *v, double *w, double *u1,
              double *v1, double *w1, double *p)
{
    orc_rk1(g, u, v, w, u1, v1, w1);
    orc_update_bound_vel(g, u1, v1, w1);
    orc_rk2(g, u, v, w, u1, v1, w1);
    orc_update_bound_vel(g, u, v, w);
    orc_calc_rhs(g, u, v, w, p);
    ppe(ppe_ctx, p);
    orc_update_bound_p(g, p);
    orc_correct_vel(g, p, u, v, w);
    orc_force_vel(g, u, v, w);
    orc_update_bound_vel(g, u, v, w);
}
