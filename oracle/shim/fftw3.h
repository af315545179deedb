/*
 * fftw3.h -- minimal stand-in for the FFTW3 guru real-to-real interface, so
 * that the reference's own src/src_c/mod_fft.c (+ mod_fft_fftw.inc) compiles
 * unmodified for the CPU oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * Declares exactly what mod_fft_fftw.inc uses (types fftw_plan, fftw_iodim,
 * fftw_r2r_kind; flags FFTW_MEASURE; fftw_plan_guru_r2r, fftw_execute_r2r,
 * fftw_destroy_plan).  Names and argument meaning follow the public FFTW3 API
 * documentation; the implementation (fftw_shim.c) is this repository's own
 * restatement of the R2HC / HC2R definitions (oracle/hc_fft.c).  The
 * REDFT/RODFT kinds are accepted by name but rejected at plan time: the
 * channel configuration uses only the periodic kinds.
 */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FFTW_R2HC = 0,
    FFTW_HC2R = 1,
    FFTW_DHT = 2,
    FFTW_REDFT00 = 3,
    FFTW_REDFT01 = 4,
    FFTW_REDFT10 = 5,
    FFTW_REDFT11 = 6,
    FFTW_RODFT00 = 7,
    FFTW_RODFT01 = 8,
    FFTW_RODFT10 = 9,
    FFTW_RODFT11 = 10
} fftw_r2r_kind;

typedef struct {
    int n;
    int is;
    int os;
} fftw_iodim;

typedef struct oracle_fftw_plan_s *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_guru_r2r(int rank, const fftw_iodim *dims, int howmany_rank,
                             const fftw_iodim *howmany_dims, double *in, double *out,
                             const fftw_r2r_kind *kind, unsigned flags);
void fftw_execute_r2r(const fftw_plan p, double *in, double *out);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
