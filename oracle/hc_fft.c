/*
 * hc_fft.c -- restated FFTW R2HC / HC2R semantics for the CPU oracle.
 * TEST INFRASTRUCTURE ONLY (see hc_fft.h); never linked into the product.
 *
 * Algorithm: recursive decimation-in-time Cooley-Tukey over the prime factors
 * of the length, direct O(r^2) butterflies per radix r, twiddles evaluated in
 * long double.  Even real lengths use the standard packing of the real line
 * into a half-length complex line (even samples -> real part, odd samples ->
 * imaginary part) followed by the split E_k + w^k O_k.
 */
#include "hc_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct hc_fft_plan {
    int n;       /* real length */
    int m;       /* complex length actually transformed */
    double *tw;  /* exp(-2 pi i k / m), k < m, interleaved */
    double *twn; /* exp(-2 pi i k / n), k <= n/2, interleaved (packing) */
};

static double *make_twiddles(int n, int count)
{
    double *t = (double *)malloc(sizeof(double) * 2 * (size_t)(count > 0 ? count : 1));
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < count; k++) {
        long double a = -two_pi * (long double)k / (long double)n;
        t[2 * k] = (double)cosl(a);
        t[2 * k + 1] = (double)sinl(a);
    }
    return t;
}

static int smallest_factor(int n)
{
    if (n % 2 == 0) return 2;
    for (int r = 3; r * r <= n; r += 2)
        if (n % r == 0) return r;
    return n;
}

/* out[0..n) = DFT_n of in[0], in[is], ..., with twiddle table tw for length
 * n*tws (exp(-2 pi i e / (n*tws))).  sign = -1 forward, +1 backward. */
static void cfft_rec(int n, const double *in, ptrdiff_t is, double *out,
                     const double *tw, int tws, int sign)
{
    if (n == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    int r = smallest_factor(n);
    int m = n / r;
    for (int q = 0; q < r; q++)
        cfft_rec(m, in + 2 * q * is, is * r, out + 2 * (size_t)q * m, tw, tws * r, sign);

    double tre[64], tim[64];
    double *hre = tre, *him = tim;
    if (r > 64) {
        hre = (double *)malloc(sizeof(double) * r);
        him = (double *)malloc(sizeof(double) * r);
    }
    double *res = (double *)malloc(sizeof(double) * 2 * (size_t)r);
    for (int k = 0; k < m; k++) {
        for (int q = 0; q < r; q++) {
            long e = ((long)q * k) % n;
            double wr = tw[2 * e * tws], wi = -sign * tw[2 * e * tws + 1];
            double yr = out[2 * ((size_t)q * m + k)], yi = out[2 * ((size_t)q * m + k) + 1];
            hre[q] = yr * wr - yi * wi;
            him[q] = yr * wi + yi * wr;
        }
        for (int s = 0; s < r; s++) {
            double ar = 0.0, ai = 0.0;
            for (int q = 0; q < r; q++) {
                long e = ((long)((q * (long)s) % r)) * m;
                double wr = tw[2 * e * tws], wi = -sign * tw[2 * e * tws + 1];
                ar += hre[q] * wr - him[q] * wi;
                ai += hre[q] * wi + him[q] * wr;
            }
            res[2 * s] = ar;
            res[2 * s + 1] = ai;
        }
        for (int s = 0; s < r; s++) {
            out[2 * (k + (size_t)s * m)] = res[2 * s];
            out[2 * (k + (size_t)s * m) + 1] = res[2 * s + 1];
        }
    }
    free(res);
    if (r > 64) {
        free(hre);
        free(him);
    }
}

void hc_fft_complex(int n, int sign, const double *in, double *out)
{
    double *tw = make_twiddles(n, n);
    cfft_rec(n, in, 1, out, tw, 1, sign);
    free(tw);
}

hc_fft_plan *hc_fft_plan_create(int n)
{
    hc_fft_plan *p = (hc_fft_plan *)calloc(1, sizeof(*p));
    p->n = n;
    p->m = (n % 2 == 0) ? n / 2 : n;
    p->tw = make_twiddles(p->m, p->m);
    p->twn = make_twiddles(n, n / 2 + 1);
    return p;
}

void hc_fft_plan_destroy(hc_fft_plan *p)
{
    if (!p) return;
    free(p->tw);
    free(p->twn);
    free(p);
}

void hc_fft_r2hc(const hc_fft_plan *p, double *x, ptrdiff_t stride)
{
    const int n = p->n, m = p->m;
    if (n == 1) return;
    double *z = (double *)malloc(sizeof(double) * 4 * (size_t)m);
    double *Z = z + 2 * (size_t)m;
    if (n % 2 == 0) {
        for (int j = 0; j < m; j++) {
            z[2 * j] = x[(2 * j) * stride];
            z[2 * j + 1] = x[(2 * j + 1) * stride];
        }
        cfft_rec(m, z, 1, Z, p->tw, 1, -1);
        for (int k = 0; k <= m; k++) {
            int k1 = k % m, k2 = (m - k) % m;
            double zr = Z[2 * k1], zi = Z[2 * k1 + 1];
            double cr = Z[2 * k2], ci = -Z[2 * k2 + 1];
            double er = 0.5 * (zr + cr), ei = 0.5 * (zi + ci);
            /* O = -i (Zk - conj Z_{m-k}) / 2 */
            double or_ = 0.5 * (zi - ci), oi = -0.5 * (zr - cr);
            double wr = p->twn[2 * k], wi = p->twn[2 * k + 1];
            double xr = er + (wr * or_ - wi * oi);
            double xi = ei + (wr * oi + wi * or_);
            x[k * stride] = xr;
            if (k > 0 && k < m) x[(n - k) * stride] = xi;
        }
    } else {
        for (int j = 0; j < n; j++) {
            z[2 * j] = x[j * stride];
            z[2 * j + 1] = 0.0;
        }
        cfft_rec(n, z, 1, Z, p->tw, 1, -1);
        for (int k = 0; k <= n / 2; k++) {
            x[k * stride] = Z[2 * k];
            if (k > 0) x[(n - k) * stride] = Z[2 * k + 1];
        }
    }
    free(z);
}

void hc_fft_hc2r(const hc_fft_plan *p, double *x, ptrdiff_t stride)
{
    const int n = p->n, m = p->m;
    if (n == 1) return;
    double *Z = (double *)malloc(sizeof(double) * 4 * (size_t)m);
    double *z = Z + 2 * (size_t)m;
    if (n % 2 == 0) {
        for (int k = 0; k < m; k++) {
            int k2 = m - k; /* 1..m */
            double xr = x[k * stride];
            double xi = (k > 0) ? x[(n - k) * stride] : 0.0;
            double cr = x[k2 * stride];
            double ci = (k2 < m) ? -x[(n - k2) * stride] : 0.0;
            double er = 0.5 * (xr + cr), ei = 0.5 * (xi + ci);
            double dr = 0.5 * (xr - cr), di = 0.5 * (xi - ci);
            /* O = D * w^{-k} (w^{-k} = conj of twn[k]) */
            double wr = p->twn[2 * k], wi = -p->twn[2 * k + 1];
            double or_ = dr * wr - di * wi, oi = dr * wi + di * wr;
            /* Z = E + i O */
            Z[2 * k] = er - oi;
            Z[2 * k + 1] = ei + or_;
        }
        cfft_rec(m, Z, 1, z, p->tw, 1, +1);
        for (int j = 0; j < m; j++) {
            x[(2 * j) * stride] = 2.0 * z[2 * j];
            x[(2 * j + 1) * stride] = 2.0 * z[2 * j + 1];
        }
    } else {
        for (int k = 0; k < n; k++) {
            int kk = (k <= n / 2) ? k : n - k;
            double re = x[kk * stride];
            double im = (kk > 0) ? x[(n - kk) * stride] : 0.0;
            if (k > n / 2) im = -im;
            Z[2 * k] = re;
            Z[2 * k + 1] = im;
        }
        cfft_rec(n, Z, 1, z, p->tw, 1, +1);
        for (int j = 0; j < n; j++) x[j * stride] = z[2 * j];
    }
    free(Z);
}
