// channel.cu -- the C ABI: the reference's PPE interface (drop-in), the
// device-resident PPE object, and the whole RK2 projection step.
//
// Step order (main.f90:137-208): RK1 -> RK2 -> calcRHS -> PPE -> correctVel ->
// forceVel, with updateBoundVel / updateBoundP folded into the kernels that
// write the fields (see stencil.cu).
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <utility>
#include <string>
#include <vector>

#include "../../include/powerllel_b200.h"
#include "channel.cuh"
#include "trid_tables.h"

namespace pl {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }
const char *get_error() { return g_err.c_str(); }

} // namespace pl

using namespace pl;

// ------------------------------------------------------------------------
// decomp_main of the reference's decomp_2d.h, read when the process defines
// it (layout identical to struct DECOMP_2D_INFO, decomp_2d.h:27-51).
// ------------------------------------------------------------------------
typedef struct DECOMP_2D_INFO {
    int *x1cnts, *x1disp, *y1cnts, *y1disp, *y2cnts, *y2disp, *z2cnts, *z2disp;
    int x1count, y1count, y2count, z2count;
    int xst[3], xen[3], xsz[3];
    int yst[3], yen[3], ysz[3];
    int zst[3], zen[3], zsz[3];
    int *x1st, *x1en, *x1dist, *y1st, *y1en, *y1dist, *y2st, *y2en, *y2dist, *z2st, *z2en, *z2dist;
    bool even;
} pl_decomp_2d_info;

extern "C" {
extern pl_decomp_2d_info decomp_main __attribute__((weak));
}

// ------------------------------------------------------------------------
// 1. Reference PPE interface
// ------------------------------------------------------------------------
namespace {
std::mutex g_legacy_mu;
Ppe g_legacy;
bool g_legacy_live = false;
int g_legacy_parts = 0;
double *g_legacy_stage = nullptr;
double *g_legacy_work = nullptr;
int g_gnx = 0, g_gny = 0, g_gnz = 0;

[[noreturn]] void legacy_abort(const std::string &msg)
{
    std::fprintf(stderr, "powerllel_b200 ERROR: %s\n", msg.c_str());
    std::fflush(stderr);
    std::abort();
}
} // namespace

extern "C" int pl_set_trid_partitions(int nparts)
{
    if (nparts < 0) {
        set_error("pl_set_trid_partitions: nparts must be >= 0");
        return -1;
    }
    g_legacy_parts = nparts;
    return 0;
}

extern "C" const char *pl_last_error(void) { return get_error(); }

extern "C" void init_poisson_solver(int nx_global, int ny_global, int nz_global, double dx, double dy,
                                    double *dzf_global, char bctype_x[], char bctype_y[], char bctype_z[],
                                    int neighbor_xyz[3][6])
{
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    if (g_legacy_live) legacy_abort("init_poisson_solver called twice without free_poisson_solver");
    if (std::strcmp(bctype_x, "PP") || std::strcmp(bctype_y, "PP") || std::strcmp(bctype_z, "NN"))
        legacy_abort("only the channel boundary types PP, PP, NN are implemented");
    if (&decomp_main != nullptr) {
        const int *xs = decomp_main.xsz;
        if (xs[0] != 0 && (xs[0] != nx_global || xs[1] != ny_global || xs[2] != nz_global))
            legacy_abort("decomp_main describes a multi-rank decomposition; this library holds the whole domain "
                         "on one GPU (p_row = p_col = 1)");
    }
    (void)neighbor_xyz; // one rank: every wall neighbour is MPI_PROC_NULL, y/x periodic
    if (ppe_create(&g_legacy, nx_global, ny_global, nz_global, dx, dy, dzf_global, g_legacy_parts, PREC_FP64))
        legacy_abort(std::string("init_poisson_solver: ") + get_error());
    const size_t ng = (size_t)(nx_global + 2) * (ny_global + 2) * (nz_global + 2);
    if (cudaMalloc(&g_legacy_stage, sizeof(double) * ng) != cudaSuccess ||
        cudaMalloc(&g_legacy_work, sizeof(double) * (size_t)nx_global * ny_global * nz_global) != cudaSuccess)
        legacy_abort("init_poisson_solver: device allocation failed");
    g_gnx = nx_global;
    g_gny = ny_global;
    g_gnz = nz_global;
    g_legacy_live = true;
}

extern "C" void execute_poisson_solver(double *var)
{
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    if (!g_legacy_live) legacy_abort("execute_poisson_solver before init_poisson_solver");
    const size_t gx = (size_t)g_gnx + 2, gxy = gx * (g_gny + 2), ng = gxy * (g_gnz + 2);
    if (cudaMemcpy(g_legacy_stage, var, sizeof(double) * ng, cudaMemcpyHostToDevice) != cudaSuccess)
        legacy_abort("execute_poisson_solver: host to device copy failed");
    if (ppe_solve_fp64_strided(&g_legacy, g_legacy_stage, g_legacy_stage, 1 + gx + gxy, gx, gxy, g_legacy_work,
                               nullptr))
        legacy_abort(std::string("execute_poisson_solver: ") + get_error());
    if (cudaMemcpy(var, g_legacy_stage, sizeof(double) * ng, cudaMemcpyDeviceToHost) != cudaSuccess)
        legacy_abort("execute_poisson_solver: device to host copy failed");
}

extern "C" void free_poisson_solver(void)
{
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    if (!g_legacy_live) return;
    ppe_destroy(&g_legacy);
    cudaFree(g_legacy_stage);
    cudaFree(g_legacy_work);
    g_legacy_stage = g_legacy_work = nullptr;
    g_legacy_live = false;
}

// ------------------------------------------------------------------------
// 2. Device-resident PPE
// ------------------------------------------------------------------------
extern "C" int pl_ppe_create(pl_ppe **out, int nx, int ny, int nz, double dx, double dy, const double *dzf_global,
                             int nparts, int precision)
{
    *out = nullptr;
    if (precision != PL_FP64 && precision != PL_MIXED) {
        set_error("pl_ppe_create: precision must be PL_FP64 or PL_MIXED");
        return -1;
    }
    pl_ppe *p = new pl_ppe();
    if (ppe_create(&p->s, nx, ny, nz, dx, dy, dzf_global, nparts, precision)) {
        ppe_destroy(&p->s);
        delete p;
        return -1;
    }
    *out = p;
    return 0;
}

extern "C" int pl_ppe_solve(pl_ppe *p, void *d_var, void *stream)
{
    if (!p || !d_var) {
        set_error("pl_ppe_solve: null argument");
        return -1;
    }
    // the y transform reads and writes adjacent column pairs as one complex
    // value: the array must start on a boundary of two elements (checked
    // before the plan is read)
    const uintptr_t a = reinterpret_cast<uintptr_t>(d_var);
    if (a % 8 != 0 || (a % 16 != 0 && p->s.prec == PREC_FP64)) {
        set_error(std::string("pl_ppe_solve: d_var must be aligned to ") + (a % 8 != 0 ? "8" : "16") +
                  " bytes (two elements: 8 for PL_MIXED, 16 for PL_FP64)");
        return -1;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (p->s.prec == PREC_FP64) return ppe_solve_fp64(&p->s, (double *)d_var, st);
    return ppe_solve_fp32(&p->s, (float *)d_var, nullptr, st);
}

extern "C" int pl_ppe_destroy(pl_ppe *p)
{
    if (!p) return 0;
    ppe_destroy(&p->s);
    delete p;
    return 0;
}

// ------------------------------------------------------------------------
// 3. Whole step
// ------------------------------------------------------------------------

static void channel_mark(void *ctx, const char *name)
{
    pl_channel *c = (pl_channel *)ctx;
    if (!c->prof_events) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, c->stream);
    c->prof_events->push_back(e);
    c->prof_names->push_back(name);
}

// mod_mesh.f90:26-84 with initMeshByFunc :120-162 (one rank)
static void build_mesh(pl_channel *c)
{
    const pl_channel_config &g = c->cfg;
    const int nz = g.nz, n1 = nz + 2;
    c->dzf_global.assign(n1, 0.0);
    c->zc_global.assign(n1, 0.0);
    const double pi = acos(-1.0);
    if (g.stretch_ratio == 0.0 || g.mesh_type == 0) {
        for (int k = 0; k < n1; k++) c->dzf_global[k] = g.lz / nz;
    } else {
        std::vector<double> zf(nz + 1, 0.0);
        for (int k = 1; k <= nz; k++) {
            double z0 = k / (1.0 * nz);
            if (g.stretch_func == 0)
                zf[k] = 0.5 * (1.0 + tanh((z0 - 0.5) * g.stretch_ratio) / tanh(g.stretch_ratio / 2.0));
            else
                zf[k] = 0.5 * (1.0 + sin((z0 - 0.5) * g.stretch_ratio * pi) / sin(g.stretch_ratio * pi / 2.0));
        }
        for (int k = 1; k <= nz; k++) c->dzf_global[k] = g.lz * (zf[k] - zf[k - 1]);
        c->dzf_global[0] = c->dzf_global[1];
        c->dzf_global[nz + 1] = c->dzf_global[nz];
    }
    c->zc_global[0] = -0.5 * c->dzf_global[0];
    for (int k = 1; k <= nz + 1; k++)
        c->zc_global[k] = c->zc_global[k - 1] + 0.5 * (c->dzf_global[k - 1] + c->dzf_global[k]);
    c->dzf = c->dzf_global;
    c->dzf_inv.assign(n1, 0.0);
    c->dzc.assign(n1, 0.0);
    c->dzc_inv.assign(n1, 0.0);
    c->dzflzi.assign(n1, 0.0);
    for (int k = 0; k <= nz + 1; k++) c->dzf_inv[k] = 1.0 / c->dzf[k];
    for (int k = 0; k <= nz; k++) {
        c->dzc[k] = 0.5 * (c->dzf[k] + c->dzf[k + 1]);
        c->dzc_inv[k] = 1.0 / c->dzc[k];
    }
    c->dzc[nz + 1] = c->dzc[nz]; // never assigned nor read by the reference
    c->dzc_inv[nz + 1] = c->dzc_inv[nz];
    for (int k = 0; k <= nz + 1; k++) c->dzflzi[k] = c->dzf[k] / g.lz;
    // Poiseuille profile, setProfile_Poiseuille (mod_initFlow.f90:83-97)
    c->prof.assign(n1, 0.0);
    for (int k = 1; k <= nz; k++) {
        double zn = c->zc_global[k] / g.lz;
        c->prof[k] = 6.0 * (1.0 - zn) * zn * g.u_ref;
    }
}

static void channel_free(pl_channel *c)
{
    pl_stat_disable(c);
    cudaFree(c->d_mesh);
    // velocity-like fields start hx planes before their plane 0
    const size_t hoff = (size_t)c->hx * c->nx * c->ny;
    for (double *f : {c->u, c->v, c->w, c->u1, c->v1, c->w1, c->ub, c->vb, c->wb})
        if (f) cudaFree(f - hoff);
    cudaFree(c->p);
    cudaFree(c->p32);
    cudaFree(c->pm32);
    cudaFree(c->pb32);
    if (c->mxtab) cudaFree(c->mxtab - (size_t)12 * c->hx);
    cudaFree(c->d1u);
    cudaFree(c->d1v);
    cudaFree(c->d1w);
    cudaFree(c->r32);
    cudaFree(c->plane_part);
    cudaFree(c->mode0);
    cudaFree(c->ms.partial);
    cudaFree(c->ms.counter);
    cudaFree(c->rb.partial);
    cudaFree(c->rb.scalar);
    cudaFree(c->d_diag);
    cudaFree(c->d_loc);
    cudaFree(c->d_dpart);
    cudaFree(c->d_dipart);
    ppe_destroy(&c->ppe);
    if (c->stream) cudaStreamDestroy(c->stream);
}

// one GPU holding the whole domain (zn = 1), or z slab zr of zn
static int channel_create(pl_channel **out, const pl_channel_config *cfg, int zr, int zn)
{
    *out = nullptr;
    if (cfg->precision != PL_FP64 && cfg->precision != PL_MIXED) {
        set_error("pl_channel_create: precision must be PL_FP64 or PL_MIXED");
        return -1;
    }
    if (cfg->nx < 2 || cfg->ny < 2 || cfg->nz < 2 || (cfg->nx & 1) || (cfg->ny & 1) || (cfg->nz & 1)) {
        set_error("pl_channel_create: nx, ny, nz must be even (mod_parameters.f90:264-267)");
        return -1;
    }
    int kst = 0, nzl = cfg->nz;
    if (zn > 1) {
        // p_row = 1, p_col = zn: the z planes distributed as decomp_2d.c:261-283
        // distributes them, and the PDD partitions are the slabs
        if (zr < 0 || zr >= zn || cfg->trid_parts != zn) {
            set_error("pl_channel_create_slab: needs 0 <= z_rank < z_ranks and trid_parts == z_ranks (PDD across "
                      "the slabs, one partition per GPU)");
            return -1;
        }
        std::vector<int> st, sz;
        trid_distribute(cfg->nz, zn, st, sz);
        for (int q = 0; q < zn; q++)
            if (sz[q] < 2) {
                set_error("pl_channel_create_slab: every slab needs at least 2 planes");
                return -1;
            }
        kst = st[zr];
        nzl = sz[zr];
    }
    pl_channel *c = new pl_channel();
    c->cfg = *cfg;
    c->nx = cfg->nx;
    c->ny = cfg->ny;
    c->nz = nzl;
    c->zrank = zn > 1 ? zr : 0;
    c->zranks = zn > 1 ? zn : 1;
    c->kst = kst;
    c->hx = zn > 1 ? 1 : 0;
    c->nf = (size_t)c->nx * c->ny * (c->nz + 2);
    c->np = (size_t)c->nx * c->ny * c->nz;
    build_mesh(c); // the global mesh (cfg->nz planes)
    c->sp.nx = c->nx;
    c->sp.ny = c->ny;
    c->sp.nz = c->nz;
    c->sp.dx_inv = 1.0 / (cfg->lx / cfg->nx);
    c->sp.dy_inv = 1.0 / (cfg->ly / cfg->ny);
    c->sp.re_inv = cfg->u_ref * cfg->l_ref / cfg->re;
    c->sp.dt = cfg->dt;
    c->sp.u_crf = cfg->u_crf;
    c->sp.wlo = c->zrank == 0;
    c->sp.whi = c->zrank == c->zranks - 1;
    c->sp.kofs = kst;
    c->sp.nzg = cfg->nz;
    const double dx = cfg->lx / cfg->nx, dy = cfg->ly / cfg->ny;
    auto fail = [&](void) {
        channel_free(c);
        delete c;
        return -1;
    };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("pl_channel_create: stream creation failed");
        return fail();
    }
    // the device mesh over the local planes -hx .. nz+1+hx (global plane
    // kst + k; beyond the global range only at a wall, where nothing reads it)
    const int hx = c->hx;
    const size_t n1 = c->nz + 2 + 2 * hx;
    {
        std::vector<double> loc(4 * n1);
        const int nzg = cfg->nz;
        for (size_t q = 0; q < n1; q++) {
            int kg = kst + (int)q - hx;
            kg = kg < 0 ? 0 : (kg > nzg + 1 ? nzg + 1 : kg);
            loc[q] = c->dzf[kg];
            loc[n1 + q] = c->dzf_inv[kg];
            loc[2 * n1 + q] = c->dzc_inv[kg];
            loc[3 * n1 + q] = c->dzflzi[kg];
        }
        if (cudaMalloc(&c->d_mesh, sizeof(double) * n1 * 4) != cudaSuccess) return fail();
        cudaMemcpy(c->d_mesh, loc.data(), sizeof(double) * 4 * n1, cudaMemcpyHostToDevice);
    }
    c->m.dzf = c->d_mesh + hx;
    c->m.dzf_inv = c->d_mesh + n1 + hx;
    c->m.dzc_inv = c->d_mesh + 2 * n1 + hx;
    c->m.dzflzi = c->d_mesh + 3 * n1 + hx;
    const bool mixed = cfg->precision == PL_MIXED;
    auto dalloc = [&](double **f, size_t n) {
        if (cudaMalloc(f, sizeof(double) * n) != cudaSuccess) return false;
        cudaMemset(*f, 0, sizeof(double) * n);
        return true;
    };
    auto falloc = [&](float **f, size_t n) {
        if (cudaMalloc(f, sizeof(float) * n) != cudaSuccess) return false;
        cudaMemset(*f, 0, sizeof(float) * n);
        return true;
    };
    // both RK stages in one kernel where the grid tiles: 32 x 8 (FP64
    // kernel) or 32 x 16 (mixed kernel); else the two stage kernels
    c->fused_rk = mixed ? rk_mixed_supported(c->sp) : rk_fused_supported(c->sp);
    if (zn > 1 && !c->fused_rk) {
        set_error("pl_channel_create_slab: the slab step needs the fused RK kernel: nx % 32 == 0 and ny % 8 == 0 "
                  "(FP64) or ny % 16 == 0 (mixed)");
        return fail();
    }
    // velocity-like fields with hx halo planes beyond each wall plane
    const size_t sk = (size_t)c->nx * c->ny;
    auto valloc = [&](double **f) {
        if (!dalloc(f, c->nf + 2 * hx * sk)) return false;
        *f += hx * sk;
        return true;
    };
    const size_t npx = c->np + hx * sk; // pressure with the upper neighbour's first plane
    bool ok = valloc(&c->u) && valloc(&c->v) && valloc(&c->w) && dalloc(&c->p, npx) && valloc(&c->ub) &&
              valloc(&c->vb) && valloc(&c->wb);
    if (ok && !mixed && zn == 1) ok = valloc(&c->u1) && valloc(&c->v1) && valloc(&c->w1);
    if (ok && mixed) {
        ok = falloc(&c->p32, c->np) && falloc(&c->pb32, c->np) && falloc(&c->pm32, c->np) &&
             falloc(&c->mxtab, (size_t)12 * n1) && falloc(&c->r32, npx) && dalloc(&c->mode0, c->nz) &&
             dalloc(&c->plane_part, (size_t)std::max(warp_partials_per_plane(c->sp), c->sp.ny / 2) * c->nz);
        if (ok) c->mxtab += (size_t)12 * hx;
        if (ok && zn == 1) ok = falloc(&c->d1u, c->nf) && falloc(&c->d1v, c->nf) && falloc(&c->d1w, c->nf);
    }
    if (!ok) {
        set_error("pl_channel_create: out of device memory for the fields");
        return fail();
    }
    // the mixed path solves for the pressure increment (Thomas); with PDD the
    // reference's truncated solve is not an exact inverse, so the full
    // pressure is solved each step as in the reference
    c->incremental = (cfg->trid_parts == 0) ? 1 : 0;
    const int pprec = mixed ? PREC_MIXED : PREC_FP64;
    if (zn > 1 ? ppe_create_slab(&c->ppe, c->nx, c->ny, cfg->nz, dx, dy, c->dzf_global.data(), zn, c->zrank, pprec)
               : ppe_create(&c->ppe, c->nx, c->ny, c->nz, dx, dy, c->dzf_global.data(), cfg->trid_parts, pprec))
        return fail();
    if (mixed) {
        const std::vector<float> tab = rk_mixed_table(c->sp, c->dzf, c->dzf_inv, c->dzc_inv, kst - hx, n1);
        if (cudaMemcpy(c->mxtab - (size_t)12 * hx, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
            set_error("pl_channel_create: upload of the mixed RK coefficients failed");
            return fail();
        }
    }
    c->max_blocks = ((c->nx + 63) / 64) * ((c->ny + 3) / 4) * c->nz;
    if (c->fused_rk && !mixed && rk_fused_blocks(c->sp) > c->max_blocks) c->max_blocks = rk_fused_blocks(c->sp);
    if (c->fused_rk && mixed && rk_mixed_blocks(c->sp) > c->max_blocks) c->max_blocks = rk_mixed_blocks(c->sp);
    c->rb.max_blocks = c->max_blocks;
    if (cudaMalloc(&c->rb.partial, sizeof(double) * 3 * c->max_blocks) != cudaSuccess ||
        cudaMalloc(&c->rb.scalar, sizeof(double) * 8) != cudaSuccess ||
        cudaMalloc(&c->d_diag, sizeof(double) * 4) != cudaSuccess ||
        cudaMalloc(&c->d_loc, sizeof(int) * 8) != cudaSuccess ||
        cudaMalloc(&c->d_dpart, sizeof(double) * 3 * c->max_blocks) != cudaSuccess ||
        cudaMalloc(&c->d_dipart, sizeof(long long) * 2 * c->max_blocks) != cudaSuccess ||
        cudaMalloc(&c->ms.partial, sizeof(double) * c->max_blocks) != cudaSuccess ||
        cudaMalloc(&c->ms.counter, sizeof(unsigned int)) != cudaSuccess) {
        set_error("pl_channel_create: out of device memory for reductions");
        return fail();
    }
    cudaMemset(c->ms.counter, 0, sizeof(unsigned int));
    cudaMemset(c->rb.scalar, 0, sizeof(double) * 8);
    c->ms.scalar = c->rb.scalar;
    c->ms.max_blocks = c->max_blocks;
    c->ms.vel_force = cfg->vel_force[0];
    if (cfg->is_forced[1] || cfg->is_forced[2]) {
        set_error("pl_channel_create: forcing is implemented for x only (is_forced = T,F,F, the channel)");
        return fail();
    }
    if (cudaDeviceSynchronize() != cudaSuccess) {
        set_error("pl_channel_create: device error during setup");
        return fail();
    }
    *out = c;
    return 0;
}

extern "C" int pl_channel_create(pl_channel **out, const pl_channel_config *cfg)
{
    return channel_create(out, cfg, 0, 1);
}

extern "C" int pl_channel_create_slab(pl_channel **out, const pl_channel_config *cfg, int z_rank, int z_ranks)
{
    if (z_ranks < 2) {
        set_error("pl_channel_create_slab: z_ranks must be >= 2 (pl_channel_create holds the whole domain)");
        return -1;
    }
    return channel_create(out, cfg, z_rank, z_ranks);
}

extern "C" int pl_channel_destroy(pl_channel *c)
{
    if (!c) return 0;
    cudaStreamSynchronize(c->stream);
    channel_free(c);
    delete c;
    return 0;
}

// initFlow (mod_initFlow.f90:28-78) up to the Mean_h normalisation: the
// Poiseuille profile plus the seeded noise (global-index counters), and the
// plane-weighted sum of u in rb.scalar[6]
static int init_fill(pl_channel *c, uint64_t seed, double noise)
{
    double *dprof = nullptr;
    PL_CUDA_TRY(cudaMalloc(&dprof, sizeof(double) * (c->nz + 2)));
    PL_CUDA_TRY(cudaMemcpy(dprof, c->prof.data() + c->kst, sizeof(double) * (c->nz + 2), cudaMemcpyHostToDevice));
    PL_CUDA_TRY(cudaMemsetAsync(c->u, 0, sizeof(double) * c->nf, c->stream));
    PL_CUDA_TRY(cudaMemsetAsync(c->v, 0, sizeof(double) * c->nf, c->stream));
    PL_CUDA_TRY(cudaMemsetAsync(c->w, 0, sizeof(double) * c->nf, c->stream));
    PL_CUDA_TRY(cudaMemsetAsync(c->p, 0, sizeof(double) * c->np, c->stream));
    for (float *q : {c->p32, c->pb32, c->pm32})
        if (q) PL_CUDA_TRY(cudaMemsetAsync(q, 0, sizeof(float) * c->np, c->stream));
    c->p_stale = false;
    c->nsolve = 0;
    int rc = launch_init_fill(c->u, c->v, c->w, dprof, seed, noise, c->sp, c->stream);
    if (!rc) rc = launch_mean_sum(c->u, c->sp, c->m, c->rb, 0, c->stream);
    if (!rc) rc = launch_mean_partials(c->sp, c->rb, c->stream);
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    cudaFree(dprof);
    return rc;
}

extern "C" int pl_channel_init_flow(pl_channel *c, uint64_t seed, double noise)
{
    if (c->zranks > 1) {
        set_error("pl_channel_init_flow: a z slab needs the cross-rank Mean_h: pl_slab_init_fill, the sum of "
                  "pl_slab_plane(c, 9, 0) over the ranks, pl_slab_init_finish");
        return -1;
    }
    int rc = init_fill(c, seed, noise);
    if (!rc) rc = launch_init_finish(c->u, c->v, c->w, c->sp, c->cfg.u_ref, c->rb, c->stream);
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return rc;
}

static inline bool is_mixed(const pl_channel *c) { return c->cfg.precision == PL_MIXED; }

const double *pl::channel_p64(pl_channel *c)
{
    if (c->p32 && c->p_stale) {
        if (launch_widen(c->p32, c->p, c->np, c->stream) == 0) c->p_stale = false;
    }
    return c->p;
}

// mixed path pressure prediction: the first two projections after the
// initial field solve for the full pressure (the first one removes the
// initial divergence, an outlier in time); then the increment over p_n, and
// from the fourth on over the extrapolation 2 p_n - p_{n-1}.  The prediction
// for the next projection is written by the solve's inverse x transform into
// pb and rotated into pm.  For an incremental projection the RK kernel stores
// u_hat = u* - dt G p_pred, so the residual is div(u_hat) / dt and the
// correction uses the FP32 increment alone.
static int mixed_incremental(const pl_channel *c) { return (c->incremental && c->nsolve >= 2) ? 1 : 0; }

extern "C" int pl_phase_rk1(pl_channel *c)
{
    int rc = is_mixed(c) ? launch_rk1_mixed(c->u, c->v, c->w, c->d1u, c->d1v, c->d1w, c->sp, c->m, c->stream)
                         : launch_rk1_fp64(c->u, c->v, c->w, c->u1, c->v1, c->w1, c->sp, c->m, c->stream);
    channel_mark(c, "rk1");
    return rc;
}

extern "C" int pl_phase_rk2(pl_channel *c)
{
    int rc;
    if (is_mixed(c)) {
        rc = launch_rk2_mixed(c->u, c->v, c->w, c->d1u, c->d1v, c->d1w, c->ub, c->vb, c->wb, c->sp, c->m, c->ms,
                              c->pm32, mixed_incremental(c), c->stream);
        std::swap(c->u, c->ub);
        std::swap(c->v, c->vb);
        std::swap(c->w, c->wb);
    } else {
        rc = launch_rk2m_fp64(c->u, c->v, c->w, c->u1, c->v1, c->w1, c->sp, c->m, c->ms, c->stream);
    }
    channel_mark(c, "rk2");
    return rc;
}

extern "C" int pl_phase_calc_rhs(pl_channel *c)
{
    int rc;
    if (is_mixed(c))
        rc = launch_rhs_mixed(c->u, c->v, c->w, c->r32, c->plane_part, c->mode0, c->sp, c->m, c->stream);
    else
        rc = launch_calc_rhs_fp64(c->u, c->v, c->w, c->p, c->sp, c->m, c->stream);
    channel_mark(c, "calc_rhs");
    return rc;
}

// The mixed increment solve's pressure update: its inverse x transform also
// forms p_n <- prediction + increment (in place) and, in pb, the next
// prediction, extrapolated from the third projection on.
static PressureUpdate mixed_pressure_update(const pl_channel *c)
{
    PressureUpdate pu;
    pu.q = c->pm32;
    pu.p = c->p32;
    pu.qnext = c->pb32;
    pu.incremental = mixed_incremental(c);
    pu.qmode = (c->nsolve + 1 >= 3) ? 1 : 0;
    return pu;
}

extern "C" int pl_phase_poisson(pl_channel *c)
{
    if (is_mixed(c)) {
        const PressureUpdate pu = mixed_pressure_update(c);
        c->p_stale = true;
        return ppe_solve_fp32(&c->ppe, c->r32, c->mode0, c->stream, &pu);
    }
    return ppe_solve_fp64(&c->ppe, c->p, c->stream);
}

// calcRHS + the Poisson solve, with calcRHS fused into the solve's forward x
// transform where the transform length allows (the right-hand side then
// never crosses HBM); otherwise the two phases.  The FP64 right-hand side
// and its transform are the same numbers either way; the mixed path's FP64
// plane sums are summed per line pair instead of per warp.
static int phase_rhs_poisson(pl_channel *c)
{
    DivIn d;
    d.u = c->u;
    d.v = c->v;
    d.w = c->w;
    d.dzf_inv = c->m.dzf_inv;
    d.dti = 1.0 / c->sp.dt;
    d.dtidxi = d.dti * c->sp.dx_inv;
    d.dtidyi = d.dti * c->sp.dy_inv;
    if (is_mixed(c)) {
        const int rc = ppe_xfwd_div<float>(&c->ppe, d, c->r32, c->plane_part, c->stream);
        if (rc < 0) return -1;
        if (rc == 0) {
            if (launch_plane_sums(c->plane_part, c->sp.ny / 2, c->nz, c->mode0, c->stream)) return -1;
            channel_mark(c, "rhs_xfft");
            const PressureUpdate pu = mixed_pressure_update(c);
            c->p_stale = true;
            return ppe_solve_fp32_from_x(&c->ppe, c->r32, c->mode0, c->stream, &pu);
        }
    } else {
        const int rc = ppe_xfwd_div<double>(&c->ppe, d, c->p, nullptr, c->stream);
        if (rc < 0) return -1;
        if (rc == 0) {
            channel_mark(c, "rhs_xfft");
            return ppe_solve_fp64_from_x(&c->ppe, c->p, c->stream);
        }
    }
    return (pl_phase_calc_rhs(c) || pl_phase_poisson(c)) ? -1 : 0;
}

extern "C" int pl_phase_correct_force(pl_channel *c)
{
    // mixed: the RK kernel applied -dt G p_pred, the increment remains
    const int rc = is_mixed(c) ? launch_correct_force_f32(c->r32, c->u, c->v, c->w, c->sp, c->m,
                                                          c->cfg.is_forced[0], c->ms.scalar, c->stream)
                               : launch_correct_force_fp64(c->p, c->u, c->v, c->w, c->sp, c->m, c->cfg.is_forced[0],
                                                           c->ms.scalar, c->stream);
    if (is_mixed(c)) {
        std::swap(c->pm32, c->pb32); // the prediction written by the solve
        c->nsolve++;
    }
    channel_mark(c, "correct_force");
    return rc;
}

// both RK stages in one kernel (out of place) when the grid tiles (32 x 8 FP64,
// 32 x 16 mixed), else the two stage kernels
extern "C" int pl_phase_rk(pl_channel *c)
{
    int rc;
    if (!c->fused_rk) {
        rc = pl_phase_rk1(c);
        if (!rc) rc = pl_phase_rk2(c);
        return rc;
    }
    rc = is_mixed(c) ? launch_rk_mixed(c->u, c->v, c->w, c->ub, c->vb, c->wb, c->sp, c->m, c->mxtab, c->ms, c->pm32,
                                       mixed_incremental(c), c->stream)
                     : launch_rk_fused_fp64(c->u, c->v, c->w, c->ub, c->vb, c->wb, c->sp, c->m, c->ms, c->stream);
    std::swap(c->u, c->ub);
    std::swap(c->v, c->vb);
    std::swap(c->w, c->wb);
    channel_mark(c, "rk_fused");
    return rc;
}

extern "C" int pl_channel_profile(pl_channel *c, int nsteps, double *ms, char *names, int max_slots)
{
    if (nsteps < 1) {
        set_error("pl_channel_profile: nsteps must be >= 1");
        return -1;
    }
    std::vector<cudaEvent_t> ev;
    std::vector<std::string> nm;
    c->prof_events = &ev;
    c->prof_names = &nm;
    c->ppe.mark = channel_mark;
    c->ppe.mark_ctx = c;
    int rc = 0;
    channel_mark(c, "start");
    for (int s = 0; s < nsteps && rc == 0; s++) rc = pl_channel_step(c, 1);
    c->ppe.mark = nullptr;
    c->prof_events = nullptr;
    c->prof_names = nullptr;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    int nslot = ((int)ev.size() - 1) / nsteps;
    if (rc == 0 && e == cudaSuccess) {
        for (int q = 0; q < nslot && q < max_slots; q++) {
            double acc = 0.0;
            for (int s = 0; s < nsteps; s++) {
                float t = 0.f;
                cudaEventElapsedTime(&t, ev[(size_t)s * nslot + q], ev[(size_t)s * nslot + q + 1]);
                acc += t;
            }
            ms[q] = acc / nsteps;
            if (names) {
                std::memset(names + 32 * q, 0, 32);
                std::strncpy(names + 32 * q, nm[q + 1].c_str(), 31);
            }
        }
    }
    for (auto x : ev) cudaEventDestroy(x);
    if (rc) return -1;
    if (e != cudaSuccess) {
        set_error(std::string("pl_channel_profile: ") + cudaGetErrorString(e));
        return -1;
    }
    return nslot;
}

extern "C" int pl_channel_step(pl_channel *c, int nsteps)
{
    for (int s = 0; s < nsteps; s++) {
        if (pl_phase_rk(c) || phase_rhs_poisson(c) || pl_phase_correct_force(c)) return -1;
    }
    return 0;
}

extern "C" int pl_channel_synchronize(pl_channel *c)
{
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return 0;
}

extern "C" int pl_channel_diagnostics(pl_channel *c, pl_diag *out)
{
    if (launch_diagnostics_fp64(c->u, c->v, c->w, c->sp, c->m, c->d_diag, c->d_loc, c->d_dpart, c->d_dipart,
                                c->max_blocks, c->stream))
        return -1;
    double h[3];
    int loc[6];
    PL_CUDA_TRY(cudaMemcpyAsync(h, c->d_diag, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    PL_CUDA_TRY(cudaMemcpyAsync(loc, c->d_loc, sizeof(loc), cudaMemcpyDeviceToHost, c->stream));
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    out->div_max = h[0];
    out->cfl_max = h[1];
    out->nan_count = (int)h[2];
    for (int q = 0; q < 3; q++) {
        out->div_ijk[q] = loc[q];
        out->cfl_ijk[q] = loc[3 + q];
    }
    return 0;
}

// device layout [k][j][i] (k = 0..nz+1) <-> reference ghosted (nx+2)(ny+2)(nz+2)
static void expand_ghosted(const pl_channel *c, const double *src, double *dst, int planes_src, int k_off)
{
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const size_t gx = nx + 2, gxy = gx * (ny + 2);
    for (int k = 0; k <= nz + 1; k++) {
        int ks = k + k_off; // source plane
        if (ks < 0) ks = 0;
        if (ks >= planes_src) ks = planes_src - 1;
        for (int j = 0; j <= ny + 1; j++) {
            const int js = (j == 0) ? ny - 1 : (j == ny + 1 ? 0 : j - 1);
            const double *row = src + (size_t)nx * ((size_t)js + (size_t)ny * ks);
            double *drow = dst + gx * j + gxy * k;
            drow[0] = row[nx - 1];
            std::memcpy(drow + 1, row, sizeof(double) * nx);
            drow[nx + 1] = row[0];
        }
    }
}

extern "C" int pl_channel_get_fields(pl_channel *c, double *u, double *v, double *w, double *p)
{
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    std::vector<double> tmp(c->nf);
    double *dev[3] = {c->u, c->v, c->w};
    double *host[3] = {u, v, w};
    for (int q = 0; q < 3; q++) {
        if (!host[q]) continue;
        PL_CUDA_TRY(cudaMemcpy(tmp.data(), dev[q], sizeof(double) * c->nf, cudaMemcpyDeviceToHost));
        expand_ghosted(c, tmp.data(), host[q], c->nz + 2, 0);
    }
    if (p) {
        channel_p64(c);
        PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
        PL_CUDA_TRY(cudaMemcpy(tmp.data(), c->p, sizeof(double) * c->np, cudaMemcpyDeviceToHost));
        // interior planes 0..nz-1 become k = 1..nz; ghosts p(0) = p(1), p(nz+1) = p(nz)
        expand_ghosted(c, tmp.data(), p, c->nz, -1);
    }
    return 0;
}

extern "C" int pl_channel_get_field(pl_channel *c, int which, double *host)
{
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (which < 0 || which > 6 || !host) {
        set_error("pl_channel_get_field: which must be 0..6");
        return -1;
    }
    std::vector<double> tmp(c->nf);
    if (which == 3) {
        channel_p64(c);
        PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
        PL_CUDA_TRY(cudaMemcpy(tmp.data(), c->p, sizeof(double) * c->np, cudaMemcpyDeviceToHost));
        expand_ghosted(c, tmp.data(), host, c->nz, -1);
        return 0;
    }
    if (which >= 4 && is_mixed(c)) {
        // u1 = u + d1 (the stage-1 field the mixed path keeps as an increment)
        std::vector<float> inc(c->nf);
        const double *base = which == 4 ? c->u : (which == 5 ? c->v : c->w);
        const float *d = which == 4 ? c->d1u : (which == 5 ? c->d1v : c->d1w);
        PL_CUDA_TRY(cudaMemcpy(tmp.data(), base, sizeof(double) * c->nf, cudaMemcpyDeviceToHost));
        PL_CUDA_TRY(cudaMemcpy(inc.data(), d, sizeof(float) * c->nf, cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < c->nf; q++) tmp[q] += (double)inc[q];
        expand_ghosted(c, tmp.data(), host, c->nz + 2, 0);
        return 0;
    }
    const double *src = (const double *)pl_channel_field(c, which);
    PL_CUDA_TRY(cudaMemcpy(tmp.data(), src, sizeof(double) * c->nf, cudaMemcpyDeviceToHost));
    expand_ghosted(c, tmp.data(), host, c->nz + 2, 0);
    return 0;
}

extern "C" int pl_channel_set_fields(pl_channel *c, const double *u, const double *v, const double *w)
{
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->nsolve = 0; // a new state: the pressure history no longer applies
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const size_t gx = nx + 2, gxy = gx * (ny + 2);
    std::vector<double> tmp(c->nf);
    const double *host[3] = {u, v, w};
    double *dev[3] = {c->u, c->v, c->w};
    for (int q = 0; q < 3; q++) {
        if (!host[q]) continue;
        for (int k = 0; k <= nz + 1; k++)
            for (int j = 0; j < ny; j++)
                std::memcpy(tmp.data() + (size_t)nx * ((size_t)j + (size_t)ny * k), host[q] + 1 + gx * (j + 1) + gxy * k,
                            sizeof(double) * nx);
        PL_CUDA_TRY(cudaMemcpy(dev[q], tmp.data(), sizeof(double) * c->nf, cudaMemcpyHostToDevice));
    }
    return 0;
}

extern "C" int pl_channel_upload_compact(pl_channel *c, const double *uvw)
{
    double *dev[3] = {c->u, c->v, c->w};
    for (int q = 0; q < 3; q++)
        PL_CUDA_TRY(cudaMemcpyAsync(dev[q], uvw + q * c->nf, sizeof(double) * c->nf, cudaMemcpyHostToDevice,
                                    c->stream));
    return 0;
}

extern "C" int pl_channel_download_compact(pl_channel *c, double *uvw)
{
    double *dev[3] = {c->u, c->v, c->w};
    for (int q = 0; q < 3; q++)
        PL_CUDA_TRY(cudaMemcpyAsync(uvw + q * c->nf, dev[q], sizeof(double) * c->nf, cudaMemcpyDeviceToHost,
                                    c->stream));
    return 0;
}

extern "C" void *pl_channel_field(pl_channel *c, int which)
{
    switch (which) {
    case 0: return c->u;
    case 1: return c->v;
    case 2: return c->w;
    case 3: return (void *)channel_p64(c);
    case 4: return is_mixed(c) ? (void *)c->d1u : (void *)c->u1;
    case 5: return is_mixed(c) ? (void *)c->d1v : (void *)c->v1;
    case 6: return is_mixed(c) ? (void *)c->d1w : (void *)c->w1;
    default: return nullptr;
    }
}

extern "C" void *pl_channel_stream(pl_channel *c) { return (void *)c->stream; }

// ------------------------------------------------------------------------
// 4. z slabs of a multi-GPU run: the phases of one step between the
//    exchanges, which the host performs (powerllel_channel_b200/slab.py)
// ------------------------------------------------------------------------
extern "C" int pl_slab_info(pl_channel *c, int out[4])
{
    out[0] = c->kst;
    out[1] = c->nz;
    out[2] = c->zrank;
    out[3] = c->zranks;
    return 0;
}

extern "C" void *pl_slab_plane(pl_channel *c, int field, int k, size_t *bytes)
{
    const size_t sk = (size_t)c->nx * c->ny;
    const bool mixed = is_mixed(c);
    if (bytes) *bytes = sizeof(double) * sk;
    switch (field) {
    case 0: return c->u + sk * (k + 1) - sk;
    case 1: return c->v + sk * (k + 1) - sk;
    case 2: return c->w + sk * (k + 1) - sk;
    case 3: // the pressure the correction reads (plane k of the interior, nz = the halo)
        if (mixed) {
            if (bytes) *bytes = sizeof(float) * sk;
            return c->r32 + sk * k;
        }
        return c->p + sk * k;
    case 4: return c->ppe.d_scratch + sk * k;
    case 5: return c->ppe.d_tvar;
    case 6: return c->ppe.d_y3;
    case 7: return c->ppe.d_y1;
    case 8:
        if (bytes) *bytes = sizeof(double);
        return c->ms.scalar + 6;
    case 9:
        if (bytes) *bytes = sizeof(double);
        return c->rb.scalar + 6;
    default: set_error("pl_slab_plane: field must be 0..9"); return nullptr;
    }
}

extern "C" int pl_slab_init_fill(pl_channel *c, uint64_t seed, double noise) { return init_fill(c, seed, noise); }

extern "C" int pl_slab_init_finish(pl_channel *c)
{
    const int rc = launch_init_finish_sum(c->u, c->v, c->w, c->sp, c->cfg.u_ref, c->rb, c->stream);
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return rc;
}

extern "C" int pl_slab_rk(pl_channel *c)
{
    if (!c->fused_rk) {
        set_error("pl_slab_rk: the slab step needs the fused RK kernel");
        return -1;
    }
    return pl_phase_rk(c);
}

extern "C" int pl_slab_mean_finish(pl_channel *c)
{
    return launch_mean_from_sum(c->ms.scalar, c->sp, c->ms.vel_force, c->stream);
}

// calcRHS fused into the forward x transform, the y transform, the local PDD sweep
extern "C" int pl_slab_rhs_sweep(pl_channel *c)
{
    DivIn d;
    d.u = c->u;
    d.v = c->v;
    d.w = c->w;
    d.dzf_inv = c->m.dzf_inv;
    d.dti = 1.0 / c->sp.dt;
    d.dtidxi = d.dti * c->sp.dx_inv;
    d.dtidyi = d.dti * c->sp.dy_inv;
    int rc = is_mixed(c) ? ppe_xfwd_div<float>(&c->ppe, d, c->r32, c->plane_part, c->stream)
                         : ppe_xfwd_div<double>(&c->ppe, d, c->p, nullptr, c->stream);
    if (rc < 0) return -1;
    if (rc > 0) {
        // no fused divergence + x transform for this nx: calcRHS, then the
        // solve's own forward x transform
        if (pl_phase_calc_rhs(c)) return -1;
        return is_mixed(c) ? ppe_slab_forward<float>(&c->ppe, c->r32, c->stream, c->mode0)
                           : ppe_slab_forward<double>(&c->ppe, c->p, c->stream, nullptr);
    }
    if (is_mixed(c) && launch_plane_sums(c->plane_part, c->sp.ny / 2, c->nz, c->mode0, c->stream)) return -1;
    channel_mark(c, "rhs_xfft");
    return is_mixed(c) ? ppe_slab_forward_from_x<float>(&c->ppe, c->r32, c->stream, c->mode0)
                       : ppe_slab_forward_from_x<double>(&c->ppe, c->p, c->stream, nullptr);
}

extern "C" int pl_slab_pdd_iface(pl_channel *c)
{
    return ppe_slab_iface(&c->ppe, c->stream, is_mixed(c) && c->zranks == 2);
}

extern "C" int pl_slab_finish(pl_channel *c)
{
    if (is_mixed(c)) {
        const PressureUpdate pu = mixed_pressure_update(c);
        c->p_stale = true;
        return ppe_slab_backward<float>(&c->ppe, c->r32, c->stream, &pu);
    }
    return ppe_slab_backward<double>(&c->ppe, c->p, c->stream, nullptr);
}

extern "C" int pl_slab_correct(pl_channel *c) { return pl_phase_correct_force(c); }
