/*
 * hc_fft.h -- CPU restatement of the real-to-half-complex transforms that the
 * reference obtains from FFTW3 (third-party, pinned at 3.3.8 by
 * examples/template/build_th2a.sh:29; >= 3.3.4 per README.md:17).
 *
 * TEST INFRASTRUCTURE ONLY: part of the CPU oracle.  Nothing in the product
 * (powerllel_channel_b200/) links or calls this code.
 *
 * The reference calls FFTW_R2HC / FFTW_HC2R through fftw_plan_guru_r2r
 * (src/src_c/mod_fft_fftw.inc:1-5, 56-63, 76-83) for the periodic ("PP")
 * directions.  Their published definitions (FFTW manual, "The Halfcomplex-format
 * DFT" and "Real even/odd DFTs"):
 *
 *   R2HC:  r_k =  sum_j x_j cos(2 pi j k / n)         k = 0 .. n/2
 *          i_k = -sum_j x_j sin(2 pi j k / n)         k = 1 .. (n-1)/2
 *          stored in place as  r_0, r_1, ..., r_{n/2}, i_{(n+1)/2-1}, ..., i_1
 *   HC2R:  the unnormalised inverse: x_j = sum_k X_k e^{+2 pi i j k / n} with
 *          X the Hermitian spectrum encoded by the half-complex array, so
 *          HC2R(R2HC(x)) = n x.
 *
 * This file restates those definitions with an O(n log n) mixed-radix complex
 * FFT (any n; radix 2,3,4,5 and a direct DFT for other prime factors) with
 * twiddles evaluated in long double.  No FFTW source is used.
 */
#ifndef ORACLE_HC_FFT_H
#define ORACLE_HC_FFT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hc_fft_plan hc_fft_plan;

/* plan for real length n (n >= 1) */
hc_fft_plan *hc_fft_plan_create(int n);
void hc_fft_plan_destroy(hc_fft_plan *p);

/* in-place on a strided real line: x[0], x[stride], ..., x[(n-1)*stride] */
void hc_fft_r2hc(const hc_fft_plan *p, double *x, ptrdiff_t stride);
void hc_fft_hc2r(const hc_fft_plan *p, double *x, ptrdiff_t stride);

/* Cooley-Tukey complex DFT of length n, sign = -1 forward, +1 backward,
 * unnormalised; in/out interleaved (re,im) arrays of length 2n.  Exposed for
 * tests of the restatement itself. */
void hc_fft_complex(int n, int sign, const double *in, double *out);

#ifdef __cplusplus
}
#endif

#endif
