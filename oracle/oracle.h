/*
 * oracle.h -- CPU oracle for the PowerLLEL_Channel RK2 projection step.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py may load this library, and only
 * as the checker or the timed CPU baseline.  The product
 * (powerllel_channel_b200/) never links, loads or calls it.
 *
 * Restatement, in plain C and in the reference's own data layout, of:
 *   - src/src_c/mod_poisson_solver.c  (PPE: set_trid_coeff, pivots, Thomas,
 *     PDD with P in-process z-chunks, execute)          -> oracle_ppe.c
 *   - src/src_c/mod_fft_fftw.inc      (eigenvalues, normalisation)
 *   - FFTW3 R2HC/HC2R (third party)                      -> hc_fft.c
 *   - src/mod_calcVel.f90, mod_calcRHS.f90, mod_updateBound.f90,
 *     mod_utils.f90 (Mean_h, calcMaxDiv, calcMaxCFL, checkNaN),
 *     mod_mesh.f90, mod_initFlow.f90, main.f90:131-208 -> oracle_stencil.c
 *
 * Field layout is the reference's: Fortran order, i fastest, one ghost layer,
 * u(0:nx+1, 0:ny+1, 0:nz+1) (mod_variables.f90:21-41) on one rank.
 */
#ifndef ORACLE_H
#define ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny, nz;
    double lx, ly, lz;
    double dx, dy, dx_inv, dy_inv;
    double re, re_inv, u_ref, l_ref, dt, u_crf;
    int is_forced[3];
    double vel_force[3];
    /* 1-D mesh arrays, index 0..nz+1 (mod_mesh.f90:32-39) */
    double *dzf_global, *zc_global;
    double *dzf, *dzf_inv, *dzc, *dzc_inv, *dzflzi;
} orc_grid;

/* mod_mesh.f90:26-84 + initMeshByFunc :120-162.  mesh_type 0 uniform,
 * 1 stretched (stretch_func 0 tanh, 1 sin); stretch == 0 -> uniform. */
int orc_grid_init(orc_grid *g, int nx, int ny, int nz, double lx, double ly, double lz, int mesh_type,
                  int stretch_func, double stretch, double re, double u_ref, double l_ref, double dt,
                  double u_crf, const int is_forced[3], const double vel_force[3]);
void orc_grid_free(orc_grid *g);

/* counter-based SplitMix64 uniform in [0,1): value number n of stream seed */
double orc_uniform(uint64_t seed, uint64_t n);

/* mod_initFlow.f90:19-81 ('poi' + noise) with the repository PRNG, then
 * transform2CRF and the boundary fills of main.f90:98-102 */
void orc_init_flow(const orc_grid *g, uint64_t seed, double noise, double *u, double *v, double *w, double *p);

void orc_rk1(const orc_grid *g, const double *u, const double *v, const double *w, double *u1, double *v1,
             double *w1);
void orc_rk2(const orc_grid *g, double *u, double *v, double *w, const double *u1, const double *v1,
             const double *w1);
void orc_update_bound_vel(const orc_grid *g, double *u, double *v, double *w);
void orc_update_bound_p(const orc_grid *g, double *p);
void orc_calc_rhs(const orc_grid *g, const double *u, const double *v, const double *w, double *rhs);
void orc_correct_vel(const orc_grid *g, const double *p, double *u, double *v, double *w);
double orc_mean_h(const orc_grid *g, const double *var);
void orc_force_vel(const orc_grid *g, double *u, double *v, double *w);
double orc_max_div(const orc_grid *g, const double *u, const double *v, const double *w, int ijk[3]);
double orc_max_cfl(const orc_grid *g, const double *u, const double *v, const double *w, int ijk[3]);
int orc_has_nan(const orc_grid *g, const double *var);

/* ---- PPE restatement (mod_poisson_solver.c) ------------------------- */
typedef struct orc_ppe orc_ppe;
/* nparts == 0: Thomas in one z-pencil (default build); nparts >= 1: PDD
 * with nparts z-partitions, i.e. p_row = 1, p_col = nparts (_PDD build). */
orc_ppe *orc_ppe_init(int nx, int ny, int nz, double dx, double dy, const double *dzf_global, int nparts);
void orc_ppe_execute(orc_ppe *s, double *var);
void orc_ppe_free(orc_ppe *s);
/* pivots b in the solver's layout (i fastest, then j, then k) and the 1-D a,c
 * coefficients after init (for bit-level checks against the reference) */
const double *orc_ppe_pivots(const orc_ppe *s);

/* ---- one time step of main.f90:131-208 ------------------------------ */
typedef void (*orc_ppe_fn)(void *ctx, double *var);
void orc_ppe_execute_cb(void *ctx, double *var); /* ctx = orc_ppe* */
/* one PDD partition m, as the rank holding it runs it (see oracle_ppe.c) */
void orc_slab_forward(orc_ppe *s, int m, const double *x, double *xs);
void orc_slab_iface(orc_ppe *s, int m, const double *xs, const double *tvar, double *y2, double *y3);
void orc_slab_finish(orc_ppe *s, int m, double *xs, const double *y1, const double *y2, double *out);
void orc_slab_extent(const orc_ppe *s, int m, int *kst, int *ksz);
void orc_step(const orc_grid *g, orc_ppe_fn ppe, void *ppe_ctx, double *u, double *v, double *w, double *u1,
              double *v1, double *w1, double *p);

#ifdef __cplusplus
}
#endif

#endif
