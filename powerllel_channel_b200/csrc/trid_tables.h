// trid_tables.h -- host construction of the wall-normal tridiagonal data of
// the PPE (plain C++, no CUDA: also compiled on the CPU by the host-logic
// tests).
//
// Restates, per eigenvalue class, src/src_c/mod_poisson_solver.c:
//   set_trid_coeff (:40-103) with c_or_f = 'c' and bctype "NN",
//   eigenvalues lambda = lambda_x/dx^2 + lambda_y/dy^2 (:227-242,
//   mod_fft_fftw.inc:115-118), pivots b (:255-276), PDD spikes v, w and the
//   exchanged plane tmp_v (init_pdd_array :105-176).
// A class is (ix, jy) with ix <= nx/2, jy <= ny/2: half-complex slots p and
// n-p carry the same eigenvalue (cos is even), so every per-column quantity
// is stored once per class, layout [k][jy][ix].
#pragma once

#include <cmath>
#include <vector>

namespace pl {

struct TridTables {
    int nx = 0, ny = 0, nz = 0, nparts = 0, ncx = 0, ncy = 0;
    std::vector<int> kst, ksz;     // partition start (0-based) and size (decomp_2d.c:261-283)
    std::vector<double> a, bt, c;  // rows of each partition (global k), after the wall corrections
    std::vector<double> mult;      // a[k]/b[k-1]; 0 at a partition's first row
    std::vector<double> rb;        // 1/b[k], 0 where b == 0 (the guard of :337-342)
    std::vector<double> v, w, tmpv; // PDD only
    // Two-ended (twisted) sweep of a Thomas column, nz even: rows below
    // p = nz/2 keep the LU multipliers and reciprocal pivots above; rows
    // p .. nz-1 hold the elimination from the top wall, tmult[k] =
    // c[k]/e[k+1] (0 at nz-1) and trb[k] = 1/e[k], e[nz-1] = b[nz-1],
    // e[k] = b[k] - tmult[k] a[k+1].  Rows nz and nz+1 hold the 2x2 system
    // that joins the halves, d x_{p-1} + c[p-1] x_p = xs_{p-1} and
    // a[p] x_{p-1} + e[p] x_p = ys_p: x_{p-1} = xs tmult[nz] - ys tmult[nz+1],
    // x_p = ys trb[nz] - xs trb[nz+1].  Where that system is singular (the
    // (0,0) class: zero row sums) the rows give the gauge x_p = 0.
    std::vector<double> tmult, trb;
};

// decomp_2d.c:261-283, 0-based starts
inline void trid_distribute(int num, int nprocs, std::vector<int> &st0, std::vector<int> &sz)
{
    std::vector<int> st(nprocs), en(nprocs);
    sz.assign(nprocs, 0);
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
    st0.resize(nprocs);
    for (int i = 0; i < nprocs; i++) st0[i] = st[i] - 1;
}

// nparts 0: Thomas over the whole column; nparts >= 1: PDD partitions
inline void trid_build(TridTables &t, int nx, int ny, int nz, double dx, double dy, const double *dzf_global,
                       int nparts, bool twisted = false)
{
    t = TridTables();
    t.nx = nx;
    t.ny = ny;
    t.nz = nz;
    t.nparts = nparts;
    t.ncx = nx / 2 + 1;
    t.ncy = ny / 2 + 1;
    const int P = nparts >= 1 ? nparts : 1;
    trid_distribute(nz, P, t.kst, t.ksz);

    const double pi = acos(-1.0);
    std::vector<double> lx(nx), ly(ny);
    for (int i = 1; i <= nx; i++) lx[i - 1] = 2.0 * (cos(2.0 * pi * (i - 1.0) / nx) - 1.0);
    for (int i = 0; i < nx; i++) lx[i] /= (dx * dx);
    for (int i = 1; i <= ny; i++) ly[i - 1] = 2.0 * (cos(2.0 * pi * (i - 1.0) / ny) - 1.0);
    for (int i = 0; i < ny; i++) ly[i] /= (dy * dy);

    const size_t ncls = (size_t)t.ncx * t.ncy;
    std::vector<double> b(nz);
    t.a.assign(nz, 0.0);
    t.bt.assign(nz, 0.0);
    t.c.assign(nz, 0.0);
    std::vector<double> &a = t.a, &bt = t.bt;
    t.mult.assign(ncls * nz, 0.0);
    t.rb.assign(ncls * nz, 0.0);
    twisted = twisted && nparts == 0 && nz % 2 == 0 && nz >= 4;
    if (twisted) {
        t.tmult.assign(ncls * (nz + 2), 0.0);
        t.trb.assign(ncls * (nz + 2), 0.0);
    }
    std::vector<double> e(twisted ? nz : 0);
    if (nparts >= 1) {
        t.v.assign(ncls * nz, 0.0);
        t.w.assign(ncls * nz, 0.0);
        t.tmpv.assign(ncls * P, 0.0);
    }
    std::vector<double> &c = t.c;
    for (int m = 0; m < P; m++) {
        const int k0 = t.kst[m], ke = t.ksz[m];
        const double *dzf = dzf_global + k0; // dzf_global[st-1+i], i = 0..ke+1 (:251-253)
        for (int k = 0; k < ke; k++) {
            a[k0 + k] = 2.0 / (dzf[k + 1] * (dzf[k] + dzf[k + 1]));
            c[k0 + k] = 2.0 / (dzf[k + 1] * (dzf[k + 2] + dzf[k + 1]));
        }
        for (int k = 0; k < ke; k++) bt[k0 + k] = -a[k0 + k] - c[k0 + k];
        const double factor = 1.0; // 'N'
        if (m == 0) {              // bottom wall (neighbour == MPI_PROC_NULL)
            bt[k0] += factor * a[k0];
            a[k0] *= fabs(factor) - 1.0;
        }
        if (m == P - 1) { // top wall
            bt[k0 + ke - 1] += factor * c[k0 + ke - 1];
            c[k0 + ke - 1] *= fabs(factor) - 1.0;
        }
    }
    for (int jy = 0; jy < t.ncy; jy++)
        for (int ix = 0; ix < t.ncx; ix++) {
            const size_t cl = (size_t)ix + (size_t)t.ncx * jy;
            const double lam = lx[ix] + ly[jy];
            for (int m = 0; m < P; m++) {
                const int k0 = t.kst[m], ke = t.ksz[m];
                for (int k = 0; k < ke; k++) b[k0 + k] = bt[k0 + k] + lam;
                for (int k = 1; k < ke; k++) {
                    double a_tmp = a[k0 + k] / b[k0 + k - 1];
                    b[k0 + k] -= (a_tmp * c[k0 + k - 1]);
                    t.mult[cl + ncls * (k0 + k)] = a_tmp;
                }
                for (int k = 0; k < ke; k++)
                    t.rb[cl + ncls * (k0 + k)] = (b[k0 + k] != 0.0) ? 1.0 / b[k0 + k] : 0.0;
                if (nparts >= 1) {
                    // init_pdd_array: v = L^-1 (a[0] e_0), w = L^-1 (c[ke-1] e_{ke-1})
                    std::vector<double> vv(ke, 0.0), ww(ke, 0.0);
                    vv[0] = a[k0];
                    ww[ke - 1] = c[k0 + ke - 1];
                    for (int k = 1; k < ke; k++) {
                        double a_tmp = a[k0 + k] / b[k0 + k - 1];
                        vv[k] -= a_tmp * vv[k - 1];
                        ww[k] -= a_tmp * ww[k - 1];
                    }
                    if (b[k0 + ke - 1] != 0.0) {
                        vv[ke - 1] /= b[k0 + ke - 1];
                        ww[ke - 1] /= b[k0 + ke - 1];
                    } else {
                        vv[ke - 1] = 0.0;
                        ww[ke - 1] = 0.0;
                    }
                    for (int k = ke - 2; k >= 0; k--) {
                        vv[k] = (vv[k] - c[k0 + k] * vv[k + 1]) / b[k0 + k];
                        ww[k] = (ww[k] - c[k0 + k] * ww[k + 1]) / b[k0 + k];
                    }
                    for (int k = 0; k < ke; k++) {
                        t.v[cl + ncls * (k0 + k)] = vv[k];
                        t.w[cl + ncls * (k0 + k)] = ww[k];
                    }
                }
            }
            if (nparts >= 1)
                for (int m = 0; m + 1 < P; m++) t.tmpv[cl + ncls * m] = t.v[cl + ncls * t.kst[m + 1]];
            if (twisted) {
                const int p = nz / 2;
                for (int k = 0; k < p; k++) {
                    t.tmult[cl + ncls * k] = t.mult[cl + ncls * k];
                    t.trb[cl + ncls * k] = t.rb[cl + ncls * k];
                }
                e[nz - 1] = bt[nz - 1] + lam;
                for (int k = nz - 2; k >= p; k--) {
                    const double mu = c[k] / e[k + 1];
                    e[k] = (bt[k] + lam) - mu * a[k + 1];
                    t.tmult[cl + ncls * k] = mu;
                }
                for (int k = p; k < nz; k++) t.trb[cl + ncls * k] = (e[k] != 0.0) ? 1.0 / e[k] : 0.0;
                // b[p-1] is the LU pivot d_{p-1} (eliminated in place above)
                const double d = b[p - 1], ep = e[p], det = d * ep - c[p - 1] * a[p];
                double E, C, D, A;
                if (!(fabs(det) > 1e-13 * fabs(d * ep))) { // singular: gauge x_p = 0
                    E = (d != 0.0) ? 1.0 / d : 0.0;
                    C = D = A = 0.0;
                } else {
                    const double idet = 1.0 / det;
                    E = ep * idet;
                    C = c[p - 1] * idet;
                    D = d * idet;
                    A = a[p] * idet;
                }
                t.tmult[cl + ncls * nz] = E;
                t.tmult[cl + ncls * (nz + 1)] = C;
                t.trb[cl + ncls * nz] = D;
                t.trb[cl + ncls * (nz + 1)] = A;
            }
        }
}

} // namespace pl
