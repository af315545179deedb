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
