/*
 * oracle_ppe.c -- restatement of the reference's C pressure Poisson solver
 * (src/src_c/mod_poisson_solver.c) for one process.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference solves  L p = rhs  with real FFTs in x and y (R2HC, FFTW
 * guru plans, init_fft mod_fft_fftw.inc:35-90, execute_fft :92-95) and one wall-normal tridiagonal
 * system per half-complex slot (i,j), eigenvalue lambda_x(i)/dx^2 +
 * lambda_y(j)/dy^2 (mod_poisson_solver.c:226-242, get_eigen_values
 * mod_fft_fftw.inc:110-133).
 * Thomas (ssolve_trid :311-359) in the default build; PDD (init_pdd_array
 * :105-176, psolve_trid :361-466) over p_col z-partitions in the _PDD build.
 * With p_row = 1 every pencil transpose is an identity, so the P partitions
 * are kept here as P consecutive z-chunks of one array and each MPI_Sendrecv
 * of the reference becomes a copy between adjacent chunks.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "hc_fft.h"
#include "oracle.h"

struct orc_ppe {
    int nx, ny, nz, nparts, pdd;
    double norm;
    int *kst, *ksz;        /* chunk start (0-based global k) and size */
    double *a, *c;         /* per chunk, nz entries in chunk order */
    double *b;             /* pivots, nx*ny*nz, chunk-major in k */
    double *v, *w;         /* PDD spikes */
    double *tmp_v;         /* per chunk: upper neighbour's v plane at k=0 */
    double *lambdaxy;
    hc_fft_plan *px, *py;
    double *work;
};

/* decomp_2d.c:261-283: 1-based st/en, size; last blocks get the extra points */
static void distribute(int num, int nprocs, int *st, int *en, int *sz)
{
    int size = num / nprocs;
    int nu = num - size * nprocs;
    int nl = nprocs - nu;
    st[0] = 1;
    sz[0] = size;
    en[0] = size;
    for (int i = 1; i < nl; i++) {
        st[i] = st[i - 1] + size;
        sz[i] = size;
        en[i] = en[i - 1] + size;
    }
    size++;
    for (int i = nl; i < nprocs; i++) {
        st[i] = en[i - 1] + 1;
        sz[i] = size;
        en[i] = en[i - 1] + size;
    }
    en[nprocs - 1] = num;
    sz[nprocs - 1] = num - st[nprocs - 1] + 1;
}

/* mod_poisson_solver.c:40-103 for c_or_f = 'c', bctype "NN"; dzf has n+2
 * entries (local indices 0..n+1); bottom/top say whether that end is a wall
 * (neighbour == MPI_PROC_NULL). */
static void set_trid_coeff_c_nn(int n, const double *dzf, int bottom, int top, double *a, double *b, double *c)
{
    for (int k = 0; k < n; k++) {
        a[k] = 2.0 / (dzf[k + 1] * (dzf[k] + dzf[k + 1]));
        c[k] = 2.0 / (dzf[k + 1] * (dzf[k + 2] + dzf[k + 1]));
    }
    for (int i = 0; i < n; i++) b[i] = -a[i] - c[i];
    const double factor = 1.0; /* 'N' */
    if (bottom) {
        b[0] += factor * a[0];
        a[0] *= fabs(factor) - 1.0;
    }
    if (top) {
        b[n - 1] += factor * c[n - 1];
        c[n - 1] *= fabs(factor) - 1.0;
    }
}

/* get_eigen_values, mod_fft_fftw.inc:115-118, "PP" */
static void eigen_pp(int n, double *lambda)
{
    const double pi = acos(-1.0);
    for (int i = 1; i <= n; i++) lambda[i - 1] = 2.0 * (cos(2.0 * pi * (i - 1.0) / n) - 1.0);
}

orc_ppe *orc_ppe_init(int nx, int ny, int nz, double dx, double dy, const double *dzf_global, int nparts)
{
    orc_ppe *s = (orc_ppe *)calloc(1, sizeof(*s));
    s->nx = nx;
    s->ny = ny;
    s->nz = nz;
    s->pdd = nparts >= 1;
    s->nparts = nparts >= 1 ? nparts : 1;
    const int P = s->nparts;
    const size_t nxy = (size_t)nx * ny, n = nxy * nz;
    s->kst = (int *)malloc(sizeof(int) * P);
    s->ksz = (int *)malloc(sizeof(int) * P);
    int *en = (int *)malloc(sizeof(int) * P);
    distribute(nz, P, s->kst, en, s->ksz);
    for (int m = 0; m < P; m++) s->kst[m] -= 1;
    free(en);

    /* init_fft: normfactor 1/(1*nx*1*ny) for PP,PP (mod_fft_fftw.inc:89) */
    s->norm = 1.0 / (1.0 * nx * 1.0 * ny);
    s->px = hc_fft_plan_create(nx);
    s->py = hc_fft_plan_create(ny);
    s->work = (double *)malloc(sizeof(double) * n);

    /* eigenvalues (mod_poisson_solver.c:227-242) */
    double *lx = (double *)malloc(sizeof(double) * nx), *ly = (double *)malloc(sizeof(double) * ny);
    eigen_pp(nx, lx);
    for (int i = 0; i < nx; i++) lx[i] /= (dx * dx);
    eigen_pp(ny, ly);
    for (int i = 0; i < ny; i++) ly[i] /= (dy * dy);
    s->lambdaxy = (double *)malloc(sizeof(double) * nxy);
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) s->lambdaxy[i + (size_t)j * nx] = lx[i] + ly[j];
    free(lx);
    free(ly);

    s->a = (double *)malloc(sizeof(double) * nz);
    s->c = (double *)malloc(sizeof(double) * nz);
    s->b = (double *)malloc(sizeof(double) * n);
    if (s->pdd) {
        s->v = (double *)calloc(n, sizeof(double));
        s->w = (double *)calloc(n, sizeof(double));
        s->tmp_v = (double *)calloc(nxy * P, sizeof(double));
    }
    double *btmp = (double *)malloc(sizeof(double) * nz);
    for (int m = 0; m < P; m++) {
        const int k0 = s->kst[m], ke = s->ksz[m];
        double *a = s->a + k0, *c = s->c + k0, *bt = btmp + k0;
        double *b = s->b + nxy * k0;
        /* local dzf: dzf_global[st_trid[2]-1+i], i = 0..ke+1 (c:251-253) */
        set_trid_coeff_c_nn(ke, dzf_global + k0, m == 0, m == P - 1, a, bt, c);
        /* b = b_tmp + lambda; LU pivots (c:255-276) */
        for (int k = 0; k < ke; k++)
            for (size_t ij = 0; ij < nxy; ij++) b[ij + nxy * k] = bt[k] + s->lambdaxy[ij];
        for (int k = 1; k < ke; k++)
            for (size_t ij = 0; ij < nxy; ij++) {
                double a_tmp = a[k] / b[ij + nxy * (k - 1)];
                b[ij + nxy * k] -= (a_tmp * c[k - 1]);
            }
        if (s->pdd) {
            /* init_pdd_array (c:105-170), before the plane exchange */
            double *v = s->v + nxy * k0, *w = s->w + nxy * k0;
            for (size_t ij = 0; ij < nxy; ij++) {
                v[ij] = a[0];
                w[ij + nxy * (ke - 1)] = c[ke - 1];
            }
            a[0] = 0.0;
            c[ke - 1] = 0.0;
            for (int k = 1; k < ke; k++)
                for (size_t ij = 0; ij < nxy; ij++) {
                    double a_tmp = a[k] / b[ij + nxy * (k - 1)];
                    v[ij + nxy * k] -= a_tmp * v[ij + nxy * (k - 1)];
                    w[ij + nxy * k] -= a_tmp * w[ij + nxy * (k - 1)];
                }
            for (size_t ij = 0; ij < nxy; ij++) {
                double bb = b[ij + nxy * (ke - 1)];
                if (bb != 0.0) {
                    v[ij + nxy * (ke - 1)] /= bb;
                    w[ij + nxy * (ke - 1)] /= bb;
                } else {
                    v[ij + nxy * (ke - 1)] = 0.0;
                    w[ij + nxy * (ke - 1)] = 0.0;
                }
            }
            for (int k = ke - 2; k >= 0; k--)
                for (size_t ij = 0; ij < nxy; ij++) {
                    v[ij + nxy * k] = (v[ij + nxy * k] - c[k] * v[ij + nxy * (k + 1)]) / b[ij + nxy * k];
                    w[ij + nxy * k] = (w[ij + nxy * k] - c[k] * w[ij + nxy * (k + 1)]) / b[ij + nxy * k];
                }
        }
    }
    free(btmp);
    if (s->pdd) {
        /* MPI_Sendrecv(v[k=0] -> lower, tmp_v <- upper) (c:172-174) */
        for (int m = 0; m + 1 < P; m++)
            memcpy(s->tmp_v + nxy * m, s->v + nxy * s->kst[m + 1], sizeof(double) * nxy);
    }
    return s;
}

/* ssolve_trid (c:311-359) on one chunk; psolve_trid's local part (c:368-408)
 * is the same recurrence (it reads a[k] for k >= 1 and c[k] for k <= ke-2
 * only, so the PDD zeroing of a[0], c[ke-1] does not enter it). */
static void thomas_chunk(size_t nxy, int ke, const double *a, const double *c, const double *b, double *x)
{
    /* the columns ij are independent: threads split them (same arithmetic per
     * column as the serial loops) */
    for (int k = 1; k < ke; k++)
#pragma omp parallel for schedule(static)
        for (size_t ij = 0; ij < nxy; ij++) {
            double a_tmp = a[k] / b[ij + nxy * (k - 1)];
            x[ij + nxy * k] -= a_tmp * x[ij + nxy * (k - 1)];
        }
#pragma omp parallel for schedule(static)
    for (size_t ij = 0; ij < nxy; ij++) {
        double bb = b[ij + nxy * (ke - 1)];
        if (bb != 0)
            x[ij + nxy * (ke - 1)] /= bb;
        else
            x[ij + nxy * (ke - 1)] = 0;
    }
    for (int k = ke - 2; k >= 0; k--)
#pragma omp parallel for schedule(static)
        for (size_t ij = 0; ij < nxy; ij++)
            x[ij + nxy * k] = (x[ij + nxy * k] - c[k] * x[ij + nxy * (k + 1)]) / b[ij + nxy * k];
}

static void solve_trid(orc_ppe *s, double *x)
{
    const size_t nxy = (size_t)s->nx * s->ny;
    const int P = s->nparts;
    for (int m = 0; m < P; m++)
        thomas_chunk(nxy, s->ksz[m], s->a + s->kst[m], s->c + s->kst[m], s->b + nxy * s->kst[m],
                     x + nxy * s->kst[m]);
    if (!s->pdd) return;
    /* psolve_trid (c:415-464): exchange bottom planes, reduced 2x2 solve at
     * each internal interface (truncated PDD), pass y3 upwards, correct. */
    double *y1 = (double *)calloc(nxy * P, sizeof(double));
    double *y2 = (double *)calloc(nxy * P, sizeof(double));
    double *y3 = (double *)calloc(nxy * P, sizeof(double));
    for (int m = 0; m + 1 < P; m++) {
        const int ke = s->ksz[m];
        const double *wt = s->w + nxy * (s->kst[m] + ke - 1);
        const double *xt = x + nxy * (s->kst[m] + ke - 1);
        const double *tmp_var = x + nxy * s->kst[m + 1]; /* upper neighbour's var[k=0] */
        const double *tmp_v = s->tmp_v + nxy * m;
#pragma omp parallel for schedule(static)
        for (size_t ij = 0; ij < nxy; ij++) {
            double det_pdd = wt[ij] * tmp_v[ij] - ((double)1.0);
            y2[nxy * m + ij] = (xt[ij] * tmp_v[ij] - tmp_var[ij]) / det_pdd;
            y3[nxy * m + ij] = (tmp_var[ij] * wt[ij] - xt[ij]) / det_pdd;
        }
    }
    /* MPI_Sendrecv(y3 -> upper, y1 <- lower) (c:444-446) */
    for (int m = 1; m < P; m++) memcpy(y1 + nxy * m, y3 + nxy * (m - 1), sizeof(double) * nxy);
    for (int m = 0; m < P; m++) {
        const int k0 = s->kst[m], ke = s->ksz[m];
#pragma omp parallel for schedule(static)
        for (int k = 0; k < ke; k++)
            for (size_t ij = 0; ij < nxy; ij++) {
                size_t g = ij + nxy * (size_t)(k0 + k);
                x[g] = x[g] - s->v[g] * y1[nxy * m + ij] - s->w[g] * y2[nxy * m + ij];
            }
    }
    free(y1);
    free(y2);
    free(y3);
}

/* execute_poisson_solver (c:468-605) on the ghosted (nx+2)(ny+2)(nz+2) array */
void orc_ppe_execute(orc_ppe *s, double *var)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const size_t gx = (size_t)nx + 2, gxy = gx * (ny + 2), nxy = (size_t)nx * ny;
    double *x = s->work;
    /* every line transform is independent: threads split the lines */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++) {
        for (int j = 0; j < ny; j++) {
            memcpy(&x[(size_t)k * nxy + (size_t)j * nx], &var[(size_t)(k + 1) * gxy + (size_t)(j + 1) * gx + 1],
                   sizeof(double) * nx);
            hc_fft_r2hc(s->px, &x[(size_t)k * nxy + (size_t)j * nx], 1);
        }
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++) hc_fft_r2hc(s->py, &x[(size_t)k * nxy + i], nx);
    solve_trid(s, x);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++) hc_fft_hc2r(s->py, &x[(size_t)k * nxy + i], nx);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++) {
            double *src = &x[(size_t)k * nxy + (size_t)j * nx];
            hc_fft_hc2r(s->px, src, 1);
            double *dst = &var[(size_t)(k + 1) * gxy + (size_t)(j + 1) * gx + 1];
            for (int i = 0; i < nx; i++) dst[i] = src[i] * s->norm;
        }
}

void orc_ppe_execute_cb(void *ctx, double *var) { orc_ppe_execute((orc_ppe *)ctx, var); }

/* One partition m of the PDD solve, as the rank that holds it runs it
 * (psolve_trid, mod_poisson_solver.c:361-466, on p_col ranks with p_row = 1):
 * the three parts between the two MPI_Sendrecv calls.  x is the partition's
 * ksz[m] planes (layout [k][j][i], no ghosts); xs its FP64 sweep buffer;
 * planes tvar, y1, y2, y3 are nx*ny.  Same operations, in the same order, as
 * orc_ppe_execute's transforms and solve_trid for that partition. */
void orc_slab_forward(orc_ppe *s, int m, const double *x, double *xs)
{
    const int nx = s->nx, ny = s->ny, ke = s->ksz[m];
    const size_t nxy = (size_t)nx * ny;
    memcpy(xs, x, sizeof(double) * nxy * ke);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < ke; k++)
        for (int j = 0; j < ny; j++) hc_fft_r2hc(s->px, &xs[(size_t)k * nxy + (size_t)j * nx], 1);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < ke; k++)
        for (int i = 0; i < nx; i++) hc_fft_r2hc(s->py, &xs[(size_t)k * nxy + i], nx);
    thomas_chunk(nxy, ke, s->a + s->kst[m], s->c + s->kst[m], s->b + nxy * s->kst[m], xs);
}

void orc_slab_iface(orc_ppe *s, int m, const double *xs, const double *tvar, double *y2, double *y3)
{
    const size_t nxy = (size_t)s->nx * s->ny;
    const int ke = s->ksz[m];
    const double *wt = s->w + nxy * (s->kst[m] + ke - 1);
    const double *xt = xs + nxy * (ke - 1);
    const double *tmp_v = s->tmp_v + nxy * m;
#pragma omp parallel for schedule(static)
    for (size_t ij = 0; ij < nxy; ij++) {
        double det_pdd = wt[ij] * tmp_v[ij] - ((double)1.0);
        y2[ij] = (xt[ij] * tmp_v[ij] - tvar[ij]) / det_pdd;
        y3[ij] = (tvar[ij] * wt[ij] - xt[ij]) / det_pdd;
    }
}

/* y1 (NULL: no lower neighbour) and y2 (NULL: no upper one) are zero there */
void orc_slab_finish(orc_ppe *s, int m, double *xs, const double *y1, const double *y2, double *out)
{
    const int nx = s->nx, ny = s->ny, k0 = s->kst[m], ke = s->ksz[m];
    const size_t nxy = (size_t)nx * ny;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < ke; k++)
        for (size_t ij = 0; ij < nxy; ij++) {
            const size_t g = ij + nxy * (size_t)k, gg = ij + nxy * (size_t)(k0 + k);
            const double a1 = y1 ? y1[ij] : 0.0, a2 = y2 ? y2[ij] : 0.0;
            xs[g] = xs[g] - s->v[gg] * a1 - s->w[gg] * a2;
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < ke; k++)
        for (int i = 0; i < nx; i++) hc_fft_hc2r(s->py, &xs[(size_t)k * nxy + i], nx);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < ke; k++)
        for (int j = 0; j < ny; j++) {
            double *src = &xs[(size_t)k * nxy + (size_t)j * nx];
            hc_fft_hc2r(s->px, src, 1);
            double *dst = &out[(size_t)k * nxy + (size_t)j * nx];
            for (int i = 0; i < nx; i++) dst[i] = src[i] * s->norm;
        }
}

void orc_slab_extent(const orc_ppe *s, int m, int *kst, int *ksz)
{
    *kst = s->kst[m];
    *ksz = s->ksz[m];
}


const double *orc_ppe_pivots(const orc_ppe *s) { return s->b; }

void orc_ppe_free(orc_ppe *s)
{
    if (!s) return;
    free(s->kst);
    free(s->ksz);
    free(s->a);
    free(s->c);
    free(s->b);
    free(s->v);
    free(s->w);
    free(s->tmp_v);
    free(s->lambdaxy);
    hc_fft_plan_destroy(s->px);
    hc_fft_plan_destroy(s->py);
    free(s->work);
    free(s);
}
