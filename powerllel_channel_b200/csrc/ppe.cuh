// ppe.cuh -- pressure Poisson solver (PPE) on one B200: host-side plan.
//
// Restates src/src_c/mod_poisson_solver.c for one GPU holding the whole
// domain (the reference's 1x1 decomposition, where every pencil transpose is
// an identity: mod_poisson_solver.c:195-206,501,538,578):
//   forward R2HC along x and y, one tridiagonal system per half-complex slot
//   (Thomas, :311-359, or PDD over P z-partitions, :105-176 and :361-466),
//   backward HC2R along y and x, scale by 1/(nx*ny) (:587-599).
#pragma once

#include <vector>

#include "common.cuh"
#include "fft.cuh"

namespace pl {

enum Precision { PREC_FP64 = 0, PREC_MIXED = 1 };

struct Ppe {
    int nx = 0, ny = 0, nz = 0;
    int nparts = 0; // 0: Thomas, >= 1: PDD with nparts z-partitions
    int prec = PREC_FP64;
    int ncx = 0, ncy = 0; // eigenvalue classes: nx/2+1, ny/2+1
    double norm = 1.0;
    std::vector<int> kst, ksz; // partition start (0-based) and size

    // FFT plans (both precisions share the radix lists)
    FftPlanDev<double2> px64{}, py64{};
    FftPlanDev<float2> px32{}, py32{};
    double2 *d_twx64 = nullptr, *d_twy64 = nullptr;
    float2 *d_twx32 = nullptr, *d_twy32 = nullptr;

    // tridiagonal coefficients, per eigenvalue class (ix <= nx/2, jy <= ny/2)
    // layout [k][jy][ix]; mult[k] = a[k]/b[k-1] (k-th row of each partition,
    // 0 at a partition's first row), rb[k] = 1/b[k] (0 where b == 0)
    double *d_mult = nullptr, *d_rb = nullptr;
    double *d_c = nullptr;   // c[k], nz (partition-local values)
    double *d_a = nullptr, *d_bt = nullptr; // a[k], b_tmp[k]: the z rows of the operator
    double *d_v = nullptr, *d_w = nullptr; // PDD spikes, class tables
    // mixed-path Thomas, 16 <= nz <= 256, nz % 16 == 0: the two-ended
    // sweep's tables (TridTables::tmult, trb; nz + 2 rows of tcs values, tcs
    // = the class count rounded up to even, so that every row starts on a
    // 16-byte boundary), else null
    double *d_tmult = nullptr, *d_trb = nullptr;
    size_t tcs = 0;
    double *d_tmpv = nullptr;              // PDD: v of partition m+1 at its k=0, [m][jy][ix]
    double *d_scratch = nullptr;           // mixed path: FP64 forward-sweep values
    size_t scratch_elems = 0;

    // (0,0) mode (mixed path): FP64 plane sums of the right-hand side
    double *d_mode0 = nullptr;

    // z slab of a multi-GPU run: this plan holds partition `rank` of the
    // global PDD system over `nranks` partitions (one per GPU); the tables
    // above are that partition's rows (nz = its plane count), d_tmpv its
    // interface plane (the upper neighbour's v at its first row).  Per-column
    // interface values: tvar (the upper neighbour's first swept row,
    // received), y2, y3 (the interface solve), y1 (the lower neighbour's y3,
    // received); nx*ny doubles each.
    int slab = 0, has_up = 0, has_down = 0;
    double *d_tvar = nullptr, *d_y1 = nullptr, *d_y2 = nullptr, *d_y3 = nullptr;

    // optional per-launch marker (profiling): called after every kernel launch
    void (*mark)(void *ctx, const char *name) = nullptr;
    void *mark_ctx = nullptr;
};

int ppe_create(Ppe *s, int nx, int ny, int nz, double dx, double dy, const double *dzf_global, int nparts,
               int prec);

void ppe_destroy(Ppe *s);

// In-place solve on the interior-only device array (layout [k][j][i]).
int ppe_solve_fp64(Ppe *s, double *d_var, cudaStream_t st);
// mode0 (optional, FP64 [nz]): the plane sums of the right-hand side; when
// given, the (kx,ky) = (0,0) system is solved from them in FP64 instead of
// from the FP32 transform, with its free constant fixed: x[nz-1] = 0 under
// Thomas, y3 = 0 at the singular interface of a two-partition PDD.
// Mixed step: the pressure update applied to the FP32 solution dp of the
// increment solve, fused into the inverse x transform where the layout
// allows (one kernel otherwise): p_new = (incremental ? q : 0) + dp stored
// in p (in place of p_n), and the next prediction qnext = qmode ?
// 2 p_new - p_n : p_new (FP32, interior-only layout).  The projection's
// accuracy does not rest on these values: the RK kernel subtracts dt G q
// from whatever q holds and the FP64 residual of the next increment solve
// takes up the difference.
// The ghosted velocity fields and factors of calcRHS
// (rhs = (u_i - u_{i-1}) dt^-1 dx^-1 + (v_j - v_{j-1}) dt^-1 dy^-1
//        + (w_k - w_{k-1}) dt^-1 dzf_k^-1, mod_calcRHS.f90:19-33) for the
// forward x transform with calcRHS fused in; dtidxi = (1/dt) (1/dx),
// dtidyi = (1/dt) (1/dy), dti = 1/dt as the stencil kernels form them.
struct DivIn {
    const double *u, *v, *w; // [k = 0..nz+1][j][i]
    const double *dzf_inv;   // index 0..nz+1
    double dtidxi, dtidyi, dti;
};
// Forward x transform of rhs = div(u)/dt computed on the fly, into the
// interior-only array out (T = double: the FP64 solve's, float: the mixed
// one's); part (optional, nz * ny/2 doubles): per line pair, the FP64 sum of
// its rhs values.  Returns 1 (nothing launched) where the fused kernel does
// not apply: nx not a compile-time transform length.
template <typename T> int ppe_xfwd_div(Ppe *s, const DivIn &d, T *out, double *part, cudaStream_t st);
// FP64 solve when d_var already holds the forward x transform
int ppe_solve_fp64_from_x(Ppe *s, double *d_var, cudaStream_t st);

struct PressureUpdate {
    const float *q = nullptr;
    float *p = nullptr, *qnext = nullptr;
    int incremental = 0, qmode = 0;
};
int ppe_solve_fp32(Ppe *s, float *d_var, const double *mode0, cudaStream_t st, const PressureUpdate *pu = nullptr);
// the same solve when d_var already holds the forward x transform
int ppe_solve_fp32_from_x(Ppe *s, float *d_var, const double *mode0, cudaStream_t st,
                          const PressureUpdate *pu = nullptr);

// the plan of z slab `rank` of `nranks` (nz_global planes distributed as
// decomp_2d.c:261-283 distributes them; PDD across the slabs)
int ppe_create_slab(Ppe *s, int nx, int ny, int nz_global, double dx, double dy, const double *dzf_global,
                    int nranks, int rank, int prec);
// Slab solve, in three parts around the two PDD plane exchanges
// (psolve_trid, mod_poisson_solver.c:361-466):
//   ppe_slab_forward_from_x: y transform of d_var (which holds the x
//     transform), the FP64 copy into the sweep buffer, the local sweep
//     (mode0, mixed path: this slab's plane sums of the right-hand side,
//     the (0,0) column's FP64 right-hand side);
//   [the caller sends the sweep buffer's first plane (d_scratch) to the lower
//    neighbour and receives the upper neighbour's into d_tvar]
//   ppe_slab_iface: y2, y3 of the interface with the upper neighbour
//     (gauge00: the mixed path over two slabs, whose (0,0) interface system
//     is singular: y3 = 0 there);
//   [the caller sends d_y3 to the upper neighbour, receives d_y1 from the lower]
//   ppe_slab_backward: x = xs - v y1 - w y2 into d_var, inverse y and x
//     transforms (with the mixed path's pressure update when pu is given).
template <typename T> int ppe_slab_forward_from_x(Ppe *s, T *d_var, cudaStream_t st, const double *mode0);
// the same from the right-hand side itself (x transform first)
template <typename T> int ppe_slab_forward(Ppe *s, T *d_var, cudaStream_t st, const double *mode0);
int ppe_slab_iface(Ppe *s, cudaStream_t st, int gauge00);
template <typename T> int ppe_slab_backward(Ppe *s, T *d_var, cudaStream_t st, const PressureUpdate *pu);


// Solve reading from / writing to a strided device array (the reference's
// ghosted layout): element (i,j,k), 0-based interior, at base[off + i +
// j*sj + k*sk].  The interior-only work array receives the transform.
int ppe_solve_fp64_strided(Ppe *s, const double *in, double *out, size_t off, size_t sj, size_t sk,
                           double *d_work, cudaStream_t st);

// out[q] = (double)in[q], q < n
int launch_widen(const float *in, double *out, size_t n, cudaStream_t st);

} // namespace pl

// the C ABI's opaque PPE handle (include/powerllel_b200.h)
struct pl_ppe {
    pl::Ppe s;
};
