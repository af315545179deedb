/*
 * powerllel_b200.h -- C ABI of the B200 implementation of PowerLLEL_Channel's
 * RK2 projection step (libpowerllel_b200.so).
 *
 * Plain C: pointers, sizes and status codes; no CUDA or torch types.  Device
 * pointers are passed as void*, streams as void* (a cudaStream_t, or NULL for
 * the library's own stream).  Every function returning int returns 0 on
 * success and -1 on failure, with the reason in pl_last_error().
 *
 * Part 1 is the reference's own PPE interface, unchanged, so that a build of
 * the Fortran driver links this library in place of src/src_c/mod_poisson_
 * solver.c + mod_fft.c.  Parts 2-4 are the device-resident extensions.
 */
#ifndef POWERLLEL_B200_H
#define POWERLLEL_B200_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================================================================
 * 1. Reference PPE interface (drop-in)
 * ====================================================================== */

/* Replaces init_poisson_solver, src/src_c/mod_poisson_solver.c:178-309
 * (Fortran interface src/mod_poisson_solver.f90:61-75).  Same arguments:
 * global sizes, dx, dy, dzf_global[0..nz+1], NUL-terminated BC strings
 * (only "PP","PP","NN" -- the channel -- is supported, as in main.f90:80),
 * neighbour table [pencil][W,E,S,N,B,T] compared against MPI_PROC_NULL.
 * Reads decomp_main (decomp_2d.h) when the caller's process defines it (the
 * reference decomp_2d.c kept in the link) and requires the whole domain on
 * this rank; without it the global sizes define a 1x1 decomposition.
 * Solver: Thomas by default (the default build, src/CMakeLists.txt:8); PDD
 * with P z-partitions after pl_set_trid_partitions(P) (the USE_PDD build
 * run on P ranks, p_row = 1, p_col = P).  Errors abort the process, as the
 * reference's decomposition errors do (decomp_2d.c:114-121). */
void init_poisson_solver(int nx_global, int ny_global, int nz_global, double dx, double dy,
                         double *dzf_global, char bctype_x[], char bctype_y[], char bctype_z[],
                         int neighbor_xyz[3][6]);

/* Replaces execute_poisson_solver, mod_poisson_solver.c:468-605: solves in
 * place on the caller's ghosted host array var[(nx+2)(ny+2)(nz+2)] (Fortran
 * order); only the interior is read and overwritten. */
void execute_poisson_solver(double *var);

/* Replaces free_poisson_solver, mod_poisson_solver.c:607-632. */
void free_poisson_solver(void);

/* PDD partition count used by the next init_poisson_solver: 0 = Thomas,
 * P >= 1 = PDD with P z-partitions (no reference counterpart: the reference
 * selects PDD at build time with USE_PDD and takes P from p_col). */
int pl_set_trid_partitions(int nparts);

/* Message of the last failure of the calling thread ("" if none). */
const char *pl_last_error(void);

/* ======================================================================
 * 2. Device-resident PPE
 * ====================================================================== */

enum { PL_FP64 = 0, PL_MIXED = 1 };

typedef struct pl_ppe pl_ppe;

/* Same setup as init_poisson_solver (mod_poisson_solver.c:178-309) as an
 * object: nparts 0 = Thomas, P >= 1 = PDD; precision PL_FP64 or PL_MIXED. */
int pl_ppe_create(pl_ppe **out, int nx, int ny, int nz, double dx, double dy, const double *dzf_global,
                  int nparts, int precision);
/* In place on a device array of nx*ny*nz values (double for PL_FP64, float
 * for PL_MIXED), layout [k][j][i], i fastest, no ghosts, starting on a
 * boundary of two elements (16 bytes for PL_FP64, 8 for PL_MIXED; every
 * cudaMalloc'd array does): other arrays are rejected with an error.
 * Asynchronous on `stream`.  Same operator as execute_poisson_solver
 * (:468-605). */
int pl_ppe_solve(pl_ppe *s, void *d_var, void *stream);
int pl_ppe_destroy(pl_ppe *s);

/* Allocation-free variant of pl_ppe_solve, for callers that cannot call
 * cudaMalloc while they solve: a host program whose device memory is owned by
 * another allocator (a pool that claimed the GPU's memory at start-up), or a
 * loop that must not stall on cudaMalloc, which can wait for the device to go
 * idle.  No counterpart in the reference.  The plan must be made with
 * PL_MIXED and nparts = 0 (Thomas).  The solve runs the same x and y
 * transforms as pl_ppe_solve, but always the tridiagonal kernel that keeps
 * its FP64 forward-swept values in device memory (pl_ppe_solve keeps them in
 * tensor memory where nz allows), and that memory is a fixed 16 MiB array
 * inside the library instead of the plan's buffer; it calls no cudaMalloc or
 * cudaFree.  d_var as for pl_ppe_solve (8-byte boundary).  The results
 * agree with pl_ppe_solve's to FP32 rounding, modulo
 * the (0,0) mode's free constant where pl_ppe_solve runs the two-ended sweep
 * (16 <= nz <= 256, nz % 16 == 0), which takes its own gauge.
 * Limit: nx*ny*nz <= 2,097,152 (e.g. 128^3); larger plans are rejected with an
 * error.  The array's device address is looked up on the first call on each
 * device (and again after the device's context is recreated).  Every call on a
 * device shares the array:
 * calls that overlap on the GPU (other streams, other threads) race;
 * serialise them.  The plan's other tables are read-only and are shared
 * safely. */
int pl_ppe_solve_noalloc(pl_ppe *s, void *d_var, void *stream);

/* ======================================================================
 * 3. Whole time step (main.f90:131-208) on device-resident fields
 * ====================================================================== */

typedef struct {
    int nx, ny, nz;          /* global grid, nx and ny even (mod_parameters.f90:264-267) */
    double lx, ly, lz;       /* domain */
    int mesh_type;           /* 0 uniform, 1 stretched (mod_mesh.f90:134-158) */
    int stretch_func;        /* 0 tanh, 1 sin */
    double stretch_ratio;
    double re, u_ref, l_ref; /* re_inv = u_ref*l_ref/re (mod_parameters.f90:187) */
    double dt, u_crf;
    int is_forced[3];
    double vel_force[3];
    int trid_parts;          /* 0 Thomas, P >= 1 PDD */
    int precision;           /* PL_FP64 or PL_MIXED */
} pl_channel_config;

typedef struct pl_channel pl_channel;

typedef struct {
    double div_max;   /* max |div u| (calcMaxDiv, mod_utils.f90:257-318) */
    double cfl_max;   /* max CFL, times dt (calcMaxCFL, :193-255) */
    int div_ijk[3];   /* 1-based location of div_max */
    int cfl_ijk[3];
    int nan_count;    /* NaNs in u, v, w incl. wall ghosts (checkNaN, :352-394) */
} pl_diag;

int pl_channel_create(pl_channel **out, const pl_channel_config *cfg);
int pl_channel_destroy(pl_channel *c);
/* initFlow 'poi' + noise (mod_initFlow.f90:19-81) with a counter-based
 * SplitMix64 stream (u, then v, then w, interior i-fastest; value n is
 * splitmix64(seed + (n+1)*0x9E3779B97F4A7C15) >> 11 scaled by 2^-53), then
 * transform2CRF and the boundary fills (main.f90:98-102). */
int pl_channel_init_flow(pl_channel *c, uint64_t seed, double noise_intensity);
/* nsteps RK2 projection steps, asynchronous on the channel's stream.  Where
 * nx is one of the compile-time transform lengths, calcRHS runs inside the
 * Poisson solve's forward x transform (the per-phase entries below run it as
 * its own kernel; in FP64 both give the same numbers bit for bit). */
int pl_channel_step(pl_channel *c, int nsteps);
int pl_channel_synchronize(pl_channel *c);
int pl_channel_diagnostics(pl_channel *c, pl_diag *out);
/* host copies in the reference's ghosted Fortran layout (nx+2)(ny+2)(nz+2);
 * any pointer may be NULL.  p is the last pressure (interior + ghosts). */
int pl_channel_get_fields(pl_channel *c, double *u, double *v, double *w, double *p);
int pl_channel_set_fields(pl_channel *c, const double *u, const double *v, const double *w);
/* one field (numbering of pl_channel_field) to a host array in the ghosted
 * layout, converted to double; the stage-1 fields of the mixed path are
 * returned as u1 = u + increment */
int pl_channel_get_field(pl_channel *c, int which, double *host_ghosted);
/* host copies in the device layout nx*ny*(nz+2) per component (wall ghost
 * planes included), u then v then w; with pinned memory these are single
 * DMA transfers (used for end-to-end timing) */
int pl_channel_upload_compact(pl_channel *c, const double *uvw);
int pl_channel_download_compact(pl_channel *c, double *uvw);
/* device pointers of the current fields (for per-phase entries and tests):
 * which = 0..2 u,v,w (FP64, nx*ny*(nz+2)), 3 = p (interior), 4..6 = stage-1
 * fields u1,v1,w1 (FP64 path) or stage-1 increments (mixed path, FP32) */
void *pl_channel_field(pl_channel *c, int which);
void *pl_channel_stream(pl_channel *c);

/* ======================================================================
 * 4. Per-phase entries on the channel's device fields (one kernel each,
 *    asynchronous; the step calls them in this order)
 * ====================================================================== */
int pl_phase_rk(pl_channel *c);         /* both stages in one kernel when nx % 32 == 0 and ny % 8 == 0
                                           (what pl_channel_step runs), else rk1 then rk2 */
int pl_phase_rk1(pl_channel *c);        /* timeIntVelRK1 + updateBoundVel(u1) */
int pl_phase_rk2(pl_channel *c);        /* timeIntVelRK2 + updateBoundVel(u) */
int pl_phase_calc_rhs(pl_channel *c);   /* calcRHS into p */
int pl_phase_poisson(pl_channel *c);    /* execute_poisson_solver(p) */
int pl_phase_correct_force(pl_channel *c); /* updateBoundP, correctVel, forceVel, updateBoundVel */

/* Per-kernel device time: runs nsteps steps with a CUDA event between every
 * kernel launch (same kernels and order as pl_channel_step) and writes the
 * mean milliseconds per step of each launch slot to ms[0..nslots) and its
 * name to names (nslots*32 bytes, NUL-padded).  Returns the slot count, or -1. */
int pl_channel_profile(pl_channel *c, int nsteps, double *ms, char *names, int max_slots);


/* ======================================================================
 * 5. Discrete adjoint (FP64 path, Thomas PPE).  No counterpart in the
 *    reference: the reference has neither a body force nor an adjoint.
 * ====================================================================== */
/* Uniform body force f added to the momentum right-hand side of both RK
 * stages: u1 = u + dt (RHS(u) + f), u = (u1 + dt (RHS(u1) + f) + u) / 2.
 * Zero by default (the reference's step).  FP64 path only; forceVel stays on. */
int pl_channel_set_body_force(pl_channel *c, const double f[3]);
/* J = 1/2 dx dy [ sum_{k=1..nz} dzf_k sum_ij (u^2 + v^2) + sum_{k=1..nz-1} dzc_k sum_ij w^2 ]
 * of the current fields (kinetic energy over the staggered cells). */
int pl_channel_kinetic_energy(pl_channel *c, double *ke);
/* Gradient of J after nsteps steps from the current fields x0, by the
 * hand-written discrete adjoint with a checkpoint every `every` steps
 * (segments recomputed forward).  Writes J(x_nsteps) to *ke, dJ/du0, dJ/dv0,
 * dJ/dw0 to the device arrays d_gu, d_gv, d_gw (device layout nx*ny*(nz+2),
 * wall planes and w's level nz zero) and dJ/df to grad_f (host).  The
 * gradient is with respect to the degrees of freedom: u, v on levels 1..nz,
 * w on levels 1..nz-1.  On return u, v, w hold x0 again; p and the stage-1
 * fields are overwritten.  Device memory: (ceil(nsteps/every) + every + 9)
 * fields.  Errors: mixed precision, PDD (trid_parts > 1), nsteps < 0, every < 1. */
int pl_adjoint_ke_gradient(pl_channel *c, int nsteps, int every, double *ke, double *d_gu, double *d_gv,
                           double *d_gw, double grad_f[3]);


/* ======================================================================
 * 6. Statistics and monitors (src/mod_statistics.f90, src/mod_monitor.f90),
 *    computed on the device; the reference writes them to text and HDF5
 *    files, here the caller receives the values.
 * ====================================================================== */
/* bits of `which`, in the order of stat_which_var: */
#define PL_STAT_U (1u << 0)
#define PL_STAT_V (1u << 1)
#define PL_STAT_W (1u << 2)
#define PL_STAT_U2 (1u << 3)
#define PL_STAT_V2 (1u << 4)
#define PL_STAT_W2 (1u << 5)
#define PL_STAT_UV (1u << 6)
#define PL_STAT_UW (1u << 7)
#define PL_STAT_VW (1u << 8)
#define PL_STAT_P (1u << 9)
#define PL_STAT_P2 (1u << 10)
/* allocStat + initStat (mod_statistics.f90:21-124): device sums, nx*ny*nz
 * doubles per selected variable, sampled from nt_init_stat every
 * sample_interval steps */
int pl_stat_enable(pl_channel *c, unsigned which, int nt_init_stat, int sample_interval);
int pl_stat_init(pl_channel *c); /* initStat: zero the sums and the counters */
/* calcStat (:126-192) at step nt: adds the cell-centred u (+u_crf), v, w,
 * their products, p and p^2 when (nt - nt_init_stat) % sample_interval == 0 */
int pl_stat_sample(pl_channel *c, int nt);
/* stat_info: first step, last sampled step, number of samples */
int pl_stat_info(pl_channel *c, int *nts, int *nte, int *nspl);
/* one sum (which = 0..10, the bit index) to a host array [k][j][i], nx*ny*nz */
int pl_stat_get(pl_channel *c, int which, double *host);
int pl_stat_disable(pl_channel *c); /* freeStat */
/* calcAndWriteSkf (mod_monitor.f90:264-296): wall 0 = bottom (k = 1), 1 = top
 * (k = nz); tau_w = <re_inv (u + u_crf)> / (dzf/2), u_tau = sqrt(tau_w),
 * cf = tau_w / (u_ref^2 / 2) */
int pl_monitor_skin_friction(pl_channel *c, int wall, double *u_tau, double *cf);
/* calcAndWriteForcing (:298-318): Mean_h of the forced components (0 for the
 * others), u_crf added to u */
int pl_monitor_forcing(pl_channel *c, double vel_mean[3]);
/* extractAndWriteProbePoint (:197-219): u + u_crf, v, w, p at the 1-based
 * point (i, j, k) */
int pl_monitor_probe(pl_channel *c, int i, int j, int k, double out[4]);
/* extractAndWriteRegion (:320-376): cell-centred u (+u_crf), v, w and p over
 * ijk = {i0, i1, j0, j1, k0, k1} (1-based, inclusive, clipped to the domain
 * as initMonitor does); host_uvwp receives the four arrays one after the
 * other, each [k][j][i] over the clipped region */
int pl_monitor_region(pl_channel *c, const int ijk[6], double *host_uvwp);

/* ======================================================================
 * 5. z slabs: one GPU per slab of a multi-GPU run
 *
 * The reference decomposes the domain over p_row x p_col MPI ranks
 * (decomp_2d.c:45-130); with p_row = 1 the x- and y-pencils coincide, the x
 * and y transforms stay local and the tridiagonal systems are solved by PDD
 * with one partition per rank (mod_poisson_solver.c:105-176, 361-466).  A
 * slab holds planes kst+1 .. kst+nz of the global grid (distributed as
 * decomp_2d.c:261-283 distributes them), its walls where it touches one, and
 * two halo planes of u, v, w beyond each interface.  Every entry below is one
 * phase of the step between two exchanges; the host moves the planes
 * pl_slab_plane names between the ranks (in order, see
 * powerllel_channel_b200/slab.py):
 *   pl_slab_rk; sum plane 8 over the ranks; pl_slab_mean_finish;
 *   w plane nz -> upper neighbour's plane 0;  pl_slab_rhs_sweep;
 *   plane 4 (0) -> lower neighbour's 5;      pl_slab_pdd_iface;
 *   plane 6 -> upper neighbour's 7;          pl_slab_finish;
 *   plane 3 (0) -> lower neighbour's 3 (nz); pl_slab_correct;
 *   u, v, w planes 1, 2 -> lower's nz+1, nz+2 and nz-1, nz -> upper's -1, 0.
 * Counterparts: the MPI_Sendrecv calls of psolve_trid (:415-417, 444-446),
 * updateHalo (mod_updateBound.f90:364-396) and the MPI_ALLREDUCE of Mean_h
 * (mod_utils.f90:127); the plane tmp_v exchanged once in init_pdd_array
 * (:172-174) is computed by every rank from the global tables instead.
 * ====================================================================== */

/* cfg describes the global problem; trid_parts must equal z_ranks */
int pl_channel_create_slab(pl_channel **out, const pl_channel_config *cfg, int z_rank, int z_ranks);
/* out = {kst, nz (the slab's planes), z_rank, z_ranks} */
int pl_slab_info(pl_channel *c, int out[4]);
/* device address of an exchanged plane, *bytes its size: field 0, 1, 2 = u,
 * v, w plane k (-1 .. nz+2); 3 = the pressure the correction reads (FP64 p,
 * or the mixed path's FP32 solution), interior plane k (0 .. nz; nz is the
 * upper neighbour's first); 4 = the PDD sweep buffer, plane k; 5 = the upper
 * neighbour's first swept plane (received); 6 = y3 (sent up); 7 = y1
 * (received from below); 8 = the RK's sum of u dzf/lz; 9 = the initial
 * field's sum of u dzf/lz (both one double, summed over the ranks in place) */
void *pl_slab_plane(pl_channel *c, int field, int k, size_t *bytes);
/* initFlow in two halves around the cross-rank sum of plane 9 */
int pl_slab_init_fill(pl_channel *c, uint64_t seed, double noise);
int pl_slab_init_finish(pl_channel *c);
int pl_slab_rk(pl_channel *c);
int pl_slab_mean_finish(pl_channel *c);
int pl_slab_rhs_sweep(pl_channel *c);
int pl_slab_pdd_iface(pl_channel *c);
int pl_slab_finish(pl_channel *c);
int pl_slab_correct(pl_channel *c);

#ifdef __cplusplus
}
#endif

#endif
