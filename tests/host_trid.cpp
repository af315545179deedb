// host_trid.cpp -- CPU test helper: builds the library's tridiagonal tables
// (powerllel_channel_b200/csrc/trid_tables.h, the same header the CUDA code
// uses) and replays the Thomas / PDD column algorithm of the k_thomas / k_pdd
// kernels on the CPU, so the host logic is testable without a GPU.
// Compiled by tests/test_host_logic.py with g++.
#include <cstring>

#include "../powerllel_channel_b200/csrc/trid_tables.h"

using namespace pl;

static void thomas_column(const TridTables &t, double *x, size_t col, size_t cls, size_t stride, size_t cs, int k0,
                          int ke)
{
    double xp = x[col + (size_t)k0 * stride];
    for (int k = k0 + 1; k < k0 + ke; k++) {
        xp = x[col + (size_t)k * stride] - t.mult[cls + (size_t)k * cs] * xp;
        x[col + (size_t)k * stride] = xp;
    }
    const int kl = k0 + ke - 1;
    xp = xp * t.rb[cls + (size_t)kl * cs];
    x[col + (size_t)kl * stride] = xp;
    for (int k = kl - 1; k >= k0; k--) {
        xp = (x[col + (size_t)k * stride] - t.c[k] * xp) * t.rb[cls + (size_t)k * cs];
        x[col + (size_t)k * stride] = xp;
    }
}

extern "C" int host_trid_solve(int nx, int ny, int nz, double dx, double dy, const double *dzf, int nparts, double *x)
{
    TridTables t;
    trid_build(t, nx, ny, nz, dx, dy, dzf, nparts);
    const size_t stride = (size_t)nx * ny, cs = (size_t)t.ncx * t.ncy;
    std::vector<double> xs(x, x + stride * nz);
    for (int py = 0; py < ny; py++)
        for (int px = 0; px < nx; px++) {
            const size_t col = (size_t)px + (size_t)nx * py;
            const int ix = px < nx - px ? px : nx - px, jy = py < ny - py ? py : ny - py;
            const size_t cls = (size_t)ix + (size_t)t.ncx * jy;
            if (nparts == 0) {
                thomas_column(t, x, col, cls, stride, cs, 0, nz);
                continue;
            }
            for (int m = 0; m < nparts; m++) thomas_column(t, xs.data(), col, cls, stride, cs, t.kst[m], t.ksz[m]);
            double y1 = 0.0;
            for (int m = 0; m < nparts; m++) {
                double y2 = 0.0, y3 = 0.0;
                if (m + 1 < nparts) {
                    const int kt = t.kst[m] + t.ksz[m] - 1;
                    const double wt = t.w[cls + (size_t)kt * cs], tv = t.tmpv[cls + (size_t)m * cs];
                    const double xt = xs[col + (size_t)kt * stride], tvar = xs[col + (size_t)t.kst[m + 1] * stride];
                    const double det = wt * tv - 1.0;
                    y2 = (xt * tv - tvar) / det;
                    y3 = (tvar * wt - xt) / det;
                }
                for (int k = t.kst[m]; k < t.kst[m] + t.ksz[m]; k++) {
                    const size_t g = col + (size_t)k * stride, gc = cls + (size_t)k * cs;
                    x[g] = xs[g] - t.v[gc] * y1 - t.w[gc] * y2;
                }
                y1 = y3;
            }
        }
    return 0;
}

// the two-ended sweep of k_thomas_th (mixed path): the LU elimination on rows
// below p = nz/2, the elimination from the top wall on rows p .. nz-1, the
// 2x2 system of rows p-1 and p, back substitution outwards (nz even)
// round_swept != 0: the swept values kept for the backward pass are rounded
// to FP32, as k_thomas_th2 keeps them in tensor memory (the recurrences and
// the junction stay FP64)
extern "C" int host_trid_solve_twisted(int nx, int ny, int nz, double dx, double dy, const double *dzf, double *x,
                                       int round_swept)
{
    TridTables t;
    trid_build(t, nx, ny, nz, dx, dy, dzf, 0, true);
    if (t.tmult.empty()) return -1;
    const size_t stride = (size_t)nx * ny, cs = (size_t)t.ncx * t.ncy;
    const int p = nz / 2;
    std::vector<double> xs(nz);
    for (int py = 0; py < ny; py++)
        for (int px = 0; px < nx; px++) {
            const size_t col = (size_t)px + (size_t)nx * py;
            const int ix = px < nx - px ? px : nx - px, jy = py < ny - py ? py : ny - py;
            const size_t cls = (size_t)ix + (size_t)t.ncx * jy;
            auto M = [&](int k) { return t.tmult[cls + (size_t)k * cs]; };
            auto R = [&](int k) { return t.trb[cls + (size_t)k * cs]; };
            double sl = 0.0, su = 0.0;
            auto keep = [&](double v) { return round_swept ? (double)(float)v : v; };
            for (int k = 0; k < p; k++) xs[k] = keep(sl = x[col + (size_t)k * stride] - M(k) * sl);
            for (int k = nz - 1; k >= p; k--) xs[k] = keep(su = x[col + (size_t)k * stride] - M(k) * su);
            double wl = sl * M(nz) - su * M(nz + 1), wu = su * R(nz) - sl * R(nz + 1);
            x[col + (size_t)(p - 1) * stride] = wl;
            x[col + (size_t)p * stride] = wu;
            for (int k = p - 2; k >= 0; k--) x[col + (size_t)k * stride] = wl = (xs[k] - t.c[k] * wl) * R(k);
            for (int k = p + 1; k < nz; k++) x[col + (size_t)k * stride] = wu = (xs[k] - t.a[k] * wu) * R(k);
        }
    return 0;
}
