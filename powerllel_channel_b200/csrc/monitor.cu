// monitor.cu -- device statistics and run monitors of the channel:
//   calcStat (src/mod_statistics.f90:126-192): running sums of the
//     cell-centred velocities, their products, p and p^2, every
//     sample_interval steps from nt_init_stat on;
//   outputMonitor (src/mod_monitor.f90:160-320): bulk velocities (Mean_h),
//     a probe point, the wall skin friction (u_tau, cf) of the bottom and top
//     walls, and the cell-centred extract of a region.
// The reference writes these to text and HDF5 files; here they are returned
// to the caller (host values or host arrays), which owns the output format.
#include <algorithm>
#include <cmath>

#include "channel.cuh"

using namespace pl;

namespace {

constexpr int NSTAT = 11; // u v w u2 v2 w2 uv uw vw p p2, the order of stat_which_var

dim3 mon_block() { return dim3(64, 4, 1); }
dim3 mon_grid(const StepParams &p) { return dim3((p.nx + 63) / 64, (p.ny + 3) / 4, p.nz); }

struct StatPtrs {
    double *a[NSTAT]; // nullptr where the variable is not sampled
};

// one sample of calcStat: uc = (u(i-1)+u(i))/2 + u_crf, vc, wc likewise at
// the cell centre (periodic x, y; w(k=0) is the wall), then the sums
__global__ void __launch_bounds__(256) k_stat_sample(const double *__restrict__ u, const double *__restrict__ v,
                                                     const double *__restrict__ w, const double *__restrict__ pp,
                                                     StatPtrs s, StepParams p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z + 1;
    if (i >= p.nx || j >= p.ny) return;
    const size_t sk = (size_t)p.nx * p.ny;
    const int im = (i == 0) ? p.nx - 1 : i - 1, jm = (j == 0) ? p.ny - 1 : j - 1;
    const size_t c = (size_t)i + (size_t)p.nx * j + sk * k;
    const double uc = (__ldg(u + (size_t)im + (size_t)p.nx * j + sk * k) + __ldg(u + c)) * 0.5 + p.u_crf;
    const double vc = (__ldg(v + (size_t)i + (size_t)p.nx * jm + sk * k) + __ldg(v + c)) * 0.5;
    const double wc = (__ldg(w + c - sk) + __ldg(w + c)) * 0.5;
    const size_t o = c - sk; // statistics and p: interior-only layout
    const double pv = __ldg(pp + o);
    const double val[NSTAT] = {uc, vc, wc, uc * uc, vc * vc, wc * wc, uc * vc, uc * wc, vc * wc, pv, pv * pv};
#pragma unroll
    for (int q = 0; q < NSTAT; q++)
        if (s.a[q]) s.a[q][o] += val[q];
}

// deterministic sums over the (i, j) plane k of var (ghosted velocity layout):
// part[b] for each of `nb` blocks, then k_sum_finish adds them in order
__global__ void __launch_bounds__(256) k_plane_part(const double *__restrict__ var, int k, StepParams p,
                                                    double *__restrict__ part)
{
    __shared__ double sh[256];
    const size_t sk = (size_t)p.nx * p.ny;
    double s = 0.0;
    for (size_t q = (size_t)blockIdx.x * 256 + threadIdx.x; q < sk; q += (size_t)gridDim.x * 256)
        s += __ldg(var + sk * k + q);
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// Mean_h (mod_utils.f90:105-131): sum of var * dzf/lz over the interior / (nx ny);
// per-level partials in k order
__global__ void __launch_bounds__(256) k_meanh_part(const double *__restrict__ var, StepParams p, MeshDev m,
                                                    double *__restrict__ part)
{
    __shared__ double sh[256];
    const int k = blockIdx.x + 1;
    const size_t sk = (size_t)p.nx * p.ny;
    double s = 0.0;
    for (size_t q = threadIdx.x; q < sk; q += 256) s += __ldg(var + sk * k + q);
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0] * __ldg(m.dzflzi + k);
}

__global__ void k_sum_finish(const double *__restrict__ part, int n, double *__restrict__ out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < n; q++) s += part[q];
        *out = s;
    }
}

// extractRegion (mod_monitor.f90:323-376): cell-centred u, v, w (+u_crf on u)
// and p over [i0, i1] x [j0, j1] x [k0, k1] (1-based, inclusive), into a
// buffer laid out [k][j][i] over the region
__global__ void __launch_bounds__(256) k_region(const double *__restrict__ u, const double *__restrict__ v,
                                                const double *__restrict__ w, const double *__restrict__ pp,
                                                StepParams p, int i0, int j0, int k0, int ni, int nj, int nk,
                                                double *__restrict__ out)
{
    const size_t n = (size_t)ni * nj * nk;
    const size_t sk = (size_t)p.nx * p.ny;
    for (size_t q = (size_t)blockIdx.x * 256 + threadIdx.x; q < n; q += (size_t)gridDim.x * 256) {
        const int a = (int)(q % ni), b = (int)((q / ni) % nj), cc = (int)(q / ((size_t)ni * nj));
        const int i = i0 - 1 + a, j = j0 - 1 + b, k = k0 + cc; // 0-based i, j; ghosted k
        const int im = (i == 0) ? p.nx - 1 : i - 1, jm = (j == 0) ? p.ny - 1 : j - 1;
        const size_t c = (size_t)i + (size_t)p.nx * j + sk * k;
        out[q] = 0.5 * (__ldg(u + (size_t)im + (size_t)p.nx * j + sk * k) + __ldg(u + c)) + p.u_crf;
        out[n + q] = 0.5 * (__ldg(v + (size_t)i + (size_t)p.nx * jm + sk * k) + __ldg(v + c));
        out[2 * n + q] = 0.5 * (__ldg(w + c - sk) + __ldg(w + c));
        out[3 * n + q] = __ldg(pp + c - sk);
    }
}

int host_scalar(pl_channel *c, const double *d, double *h)
{
    PL_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return 0;
}

// the pressure the monitors report: p of the current state, FP64 in both
// paths (the mixed path widens its FP32 pressure on demand)
const double *state_p(pl_channel *c) { return pl::channel_p64(c); }

} // namespace

// ---------------------------------------------------------------------------
// statistics (allocStat / initStat / calcStat / freeStat)
// ---------------------------------------------------------------------------
struct pl_stats {
    double *a[NSTAT] = {};
    int nt_init = 0, interval = 1;
    int nts = 0, nte = 0, nspl = 0; // stat_info of mod_parameters (first step, last step, samples)
};

static pl_stats *stats_of(pl_channel *c) { return reinterpret_cast<pl_stats *>(c->stats); }

extern "C" int pl_stat_enable(pl_channel *c, unsigned which, int nt_init_stat, int sample_interval)
{
    if (sample_interval < 1) {
        set_error("pl_stat_enable: sample_interval must be >= 1");
        return -1;
    }
    if (c->stats) {
        set_error("pl_stat_enable: statistics already enabled (pl_stat_disable first)");
        return -1;
    }
    pl_stats *s = new pl_stats();
    s->nt_init = nt_init_stat;
    s->interval = sample_interval;
    for (int q = 0; q < NSTAT; q++) {
        if (!(which & (1u << q))) continue;
        if (cudaMalloc(&s->a[q], sizeof(double) * c->np) != cudaSuccess) {
            for (int r = 0; r < NSTAT; r++) cudaFree(s->a[r]);
            delete s;
            set_error("pl_stat_enable: out of device memory for the statistics");
            return -1;
        }
    }
    c->stats = s;
    return pl_stat_init(c);
}

extern "C" int pl_stat_init(pl_channel *c)
{
    pl_stats *s = stats_of(c);
    if (!s) {
        set_error("pl_stat_init: statistics not enabled");
        return -1;
    }
    s->nts = s->nt_init + 1;
    s->nte = s->nt_init;
    s->nspl = 0;
    for (int q = 0; q < NSTAT; q++)
        if (s->a[q]) PL_CUDA_TRY(cudaMemsetAsync(s->a[q], 0, sizeof(double) * c->np, c->stream));
    return 0;
}

extern "C" int pl_stat_sample(pl_channel *c, int nt)
{
    pl_stats *s = stats_of(c);
    if (!s) {
        set_error("pl_stat_sample: statistics not enabled");
        return -1;
    }
    if ((nt - s->nt_init) % s->interval != 0) return 0; // not a sampling step (calcStat :135)
    s->nte += s->interval;
    s->nspl += 1;
    StatPtrs sp;
    for (int q = 0; q < NSTAT; q++) sp.a[q] = s->a[q];
    k_stat_sample<<<mon_grid(c->sp), mon_block(), 0, c->stream>>>(c->u, c->v, c->w, state_p(c), sp, c->sp);
    PL_CHECK_LAUNCH();
    return 0;
}

extern "C" int pl_stat_info(pl_channel *c, int *nts, int *nte, int *nspl)
{
    pl_stats *s = stats_of(c);
    if (!s) {
        set_error("pl_stat_info: statistics not enabled");
        return -1;
    }
    *nts = s->nts;
    *nte = s->nte;
    *nspl = s->nspl;
    return 0;
}

extern "C" int pl_stat_get(pl_channel *c, int which, double *host)
{
    pl_stats *s = stats_of(c);
    if (!s || which < 0 || which >= NSTAT || !s->a[which]) {
        set_error("pl_stat_get: that statistic is not being sampled");
        return -1;
    }
    PL_CUDA_TRY(cudaMemcpyAsync(host, s->a[which], sizeof(double) * c->np, cudaMemcpyDeviceToHost, c->stream));
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return 0;
}

extern "C" int pl_stat_disable(pl_channel *c)
{
    pl_stats *s = stats_of(c);
    if (!s) return 0;
    cudaStreamSynchronize(c->stream);
    for (int q = 0; q < NSTAT; q++) cudaFree(s->a[q]);
    delete s;
    c->stats = nullptr;
    return 0;
}

// ---------------------------------------------------------------------------
// monitors
// ---------------------------------------------------------------------------
extern "C" int pl_monitor_skin_friction(pl_channel *c, int wall, double *u_tau, double *cf)
{
    if (wall != 0 && wall != 1) {
        set_error("pl_monitor_skin_friction: wall must be 0 (bottom) or 1 (top)");
        return -1;
    }
    // calcAndWriteSkf (:264-296): tau_w = mean of re_inv (u(k_wall) + u_crf) / dz,
    // dz = dzf(k_wall)/2, k_wall = 1 or nz
    const int kw = wall == 0 ? 1 : c->nz;
    constexpr int NB = 64;
    double *part = nullptr;
    PL_CUDA_TRY(cudaMalloc(&part, sizeof(double) * (NB + 1)));
    k_plane_part<<<NB, 256, 0, c->stream>>>(c->u, kw, c->sp, part);
    k_sum_finish<<<1, 32, 0, c->stream>>>(part, NB, part + NB);
    double sum = 0.0;
    int rc = (cudaGetLastError() == cudaSuccess) ? host_scalar(c, part + NB, &sum) : -1;
    cudaFree(part);
    if (rc) {
        set_error("pl_monitor_skin_friction: device error");
        return -1;
    }
    const double n = (double)c->nx * c->ny;
    const double dz = 0.5 * c->dzf[kw];
    const double re_inv = c->cfg.u_ref * c->cfg.l_ref / c->cfg.re;
    const double tau_w = re_inv * (sum + n * c->cfg.u_crf) / dz / n;
    *u_tau = std::sqrt(tau_w);
    *cf = tau_w / (0.5 * c->cfg.u_ref * c->cfg.u_ref);
    return 0;
}

extern "C" int pl_monitor_forcing(pl_channel *c, double vel_mean[3])
{
    // calcAndWriteForcing (:298-318): Mean_h of the forced components, u_crf added to u
    double *part = nullptr;
    PL_CUDA_TRY(cudaMalloc(&part, sizeof(double) * ((size_t)c->nz + 1)));
    const double *f[3] = {c->u, c->v, c->w};
    int rc = 0;
    for (int d = 0; d < 3 && rc == 0; d++) {
        vel_mean[d] = 0.0;
        if (!c->cfg.is_forced[d]) continue;
        k_meanh_part<<<c->nz, 256, 0, c->stream>>>(f[d], c->sp, c->m, part);
        k_sum_finish<<<1, 32, 0, c->stream>>>(part, c->nz, part + c->nz);
        double s = 0.0;
        rc = (cudaGetLastError() == cudaSuccess) ? host_scalar(c, part + c->nz, &s) : -1;
        vel_mean[d] = s / c->nx / c->ny;
    }
    cudaFree(part);
    if (rc) {
        set_error("pl_monitor_forcing: device error");
        return -1;
    }
    vel_mean[0] += c->cfg.u_crf;
    return 0;
}

extern "C" int pl_monitor_probe(pl_channel *c, int i, int j, int k, double out[4])
{
    // extractAndWriteProbePoint (:197-219): u + u_crf, v, w, p at (i, j, k), 1-based
    if (i < 1 || i > c->nx || j < 1 || j > c->ny || k < 1 || k > c->nz) {
        set_error("pl_monitor_probe: the point is outside the domain");
        return -1;
    }
    const size_t sk = (size_t)c->nx * c->ny;
    const size_t g = (size_t)(i - 1) + (size_t)c->nx * (j - 1) + sk * k;
    const double *src[4] = {c->u + g, c->v + g, c->w + g, state_p(c) + g - sk};
    for (int q = 0; q < 4; q++)
        PL_CUDA_TRY(cudaMemcpyAsync(out + q, src[q], sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PL_CUDA_TRY(cudaStreamSynchronize(c->stream));
    out[0] += c->cfg.u_crf;
    return 0;
}

extern "C" int pl_monitor_region(pl_channel *c, const int ijk[6], double *host_uvwp)
{
    // extractAndWriteRegion (:320-376) with the region clipped to the domain
    // as initMonitor does (:120-126); host_uvwp receives u, v, w, p one after
    // the other, each [k][j][i] over the clipped region
    const int i0 = std::max(ijk[0], 1), i1 = std::min(ijk[1], c->nx);
    const int j0 = std::max(ijk[2], 1), j1 = std::min(ijk[3], c->ny);
    const int k0 = std::max(ijk[4], 1), k1 = std::min(ijk[5], c->nz);
    if (i1 < i0 || j1 < j0 || k1 < k0) {
        set_error("pl_monitor_region: the region does not meet the domain");
        return -1;
    }
    const int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
    const size_t n = (size_t)ni * nj * nk;
    double *d = nullptr;
    PL_CUDA_TRY(cudaMalloc(&d, sizeof(double) * 4 * n));
    const int grid = (int)std::min<size_t>((n + 255) / 256, 4096);
    k_region<<<grid, 256, 0, c->stream>>>(c->u, c->v, c->w, state_p(c), c->sp, i0, j0, k0, ni, nj, nk, d);
    int rc = cudaGetLastError() == cudaSuccess ? 0 : -1;
    if (!rc && cudaMemcpyAsync(host_uvwp, d, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
        rc = -1;
    if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = -1;
    cudaFree(d);
    if (rc) {
        set_error("pl_monitor_region: device error");
        return -1;
    }
    return 0;
}
