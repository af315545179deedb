/*
 * fftw_shim.c -- the guru r2r subset declared in shim/fftw3.h, implemented on
 * top of the oracle's restated R2HC / HC2R (oracle/hc_fft.c).
 * TEST INFRASTRUCTURE ONLY.
 *
 * Plan semantics follow the FFTW3 guru interface as the reference uses it
 * (src/src_c/mod_fft_fftw.inc:35-95): one transform dimension
 * {n, is, os} and one "howmany" loop dimension {n, is, os}; in-place
 * (in == out).  Execution may be called concurrently on different arrays
 * (the reference calls it inside OpenMP loops), so a plan holds no scratch.
 */
#include "fftw3.h"

#include <stdio.h>
#include <stdlib.h>

#include "../hc_fft.h"

struct oracle_fftw_plan_s {
    int n, is, os;
    int hm_n, hm_is, hm_os;
    fftw_r2r_kind kind;
    hc_fft_plan *hc;
};

fftw_plan fftw_plan_guru_r2r(int rank, const fftw_iodim *dims, int howmany_rank,
                             const fftw_iodim *howmany_dims, double *in, double *out,
                             const fftw_r2r_kind *kind, unsigned flags)
{
    (void)in;
    (void)out;
    (void)flags;
    if (rank != 1 || howmany_rank > 1) {
        fprintf(stderr, "oracle fftw shim: only rank-1 transforms with <=1 loop dimension\n");
        abort();
    }
    if (kind[0] != FFTW_R2HC && kind[0] != FFTW_HC2R) {
        fprintf(stderr, "oracle fftw shim: r2r kind %d is not restated (periodic only)\n", (int)kind[0]);
        abort();
    }
    struct oracle_fftw_plan_s *p = (struct oracle_fftw_plan_s *)calloc(1, sizeof(*p));
    p->n = dims[0].n;
    p->is = dims[0].is;
    p->os = dims[0].os;
    if (howmany_rank == 1) {
        p->hm_n = howmany_dims[0].n;
        p->hm_is = howmany_dims[0].is;
        p->hm_os = howmany_dims[0].os;
    } else {
        p->hm_n = 1;
    }
    if (p->is != p->os || p->hm_is != p->hm_os) {
        fprintf(stderr, "oracle fftw shim: only in-place layouts (is == os)\n");
        abort();
    }
    p->kind = kind[0];
    p->hc = hc_fft_plan_create(p->n);
    return p;
}

void fftw_execute_r2r(const fftw_plan p, double *in, double *out)
{
    if (in != out) {
        fprintf(stderr, "oracle fftw shim: only in-place execution\n");
        abort();
    }
    for (int h = 0; h < p->hm_n; h++) {
        double *line = in + (ptrdiff_t)h * p->hm_is;
        if (p->kind == FFTW_R2HC)
            hc_fft_r2hc(p->hc, line, p->is);
        else
            hc_fft_hc2r(p->hc, line, p->is);
    }
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    hc_fft_plan_destroy(p->hc);
    free(p);
}
