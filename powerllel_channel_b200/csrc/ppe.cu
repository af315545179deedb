// ppe.cu -- kernels and host plan of the pressure Poisson solver.
//
// Reference: src/src_c/mod_poisson_solver.c (init :178-309, Thomas :311-359,
// PDD :105-176/:361-466, execute :468-605), src/src_c/mod_fft_fftw.inc
// (init_fft :35-90, execute_fft :92-95, get_eigen_values :110-133).
//
// Kernels (one launch each per solve):
//   k_xfft<fwd>  rows of the k-plane, two rows per complex line (x: contiguous)
//   k_yfft<fwd>  columns of the k-plane, two columns per complex line
//   k_thomas / k_pdd   one wall-normal system per (x-slot, y-slot) column
// Pivots and PDD spikes depend on the column only through its eigenvalue
// lambda_x(ix) + lambda_y(jy), and slots p and n-p of a half-complex array
// share the eigenvalue, so they are stored once per class
// (ix <= nx/2, jy <= ny/2): a quarter of the reference's b array.
#include <algorithm>
#include <cstdint>
#include <cuda.h> // CUcontext (the driver entry point is fetched through the runtime)
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "ppe.cuh"
#include "tmem.cuh"
#include "trid_tables.h"

namespace pl {

// ------------------------------------------------------------------------
// FFT kernels
// ------------------------------------------------------------------------

// x direction.  CTA = `pb` row pairs (j = 2p, 2p+1) of plane k.  Input element
// (i,j,k) at in[in_off + i + j*in_sj + k*in_sk]; output in the interior-only
// layout (fwd) or at out[out_off + i + j*out_sj + k*out_sk] (bwd).
template <typename T, bool FWD>
__global__ void __launch_bounds__(256) k_xfft(const T *__restrict__ in, size_t in_off, size_t in_sj, size_t in_sk,
                                              T *__restrict__ out, size_t out_off, size_t out_sj, size_t out_sk,
                                              FftPlanDev<typename cplx_of<T>::type> plan, int ny, int pb, T scale)
{
    using V = typename cplx_of<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = plan.n; // = nx
    V *buf0 = reinterpret_cast<V *>(smem_raw);
    V *buf1 = buf0 + fpad_elems<V>(pb * n);
    const int k = blockIdx.y;
    const int p0 = blockIdx.x * pb;
    const int nb = min(pb, ny / 2 - p0);
    const int tid = threadIdx.x, nthr = blockDim.x;

    for (int e = tid; e < nb * 2 * n; e += nthr) {
        const int m = e % n, r = (e / n) & 1, b = e / (2 * n);
        const int j = 2 * (p0 + b) + r;
        T val = in[in_off + (size_t)m + (size_t)j * in_sj + (size_t)k * in_sk];
        reinterpret_cast<T *>(&buf0[fpad<V>(b * n + m)])[r] = val;
    }
    __syncthreads();
    if (FWD) {
        V *res = fft_batch<V, true, false>(buf0, buf1, plan, nb, 1, n, tid, nthr);
        for (int e = tid; e < nb * n; e += nthr) {
            const int m = e % n, b = e / n;
            V A = res[fpad<V>(b * n + m)], Bc = res[fpad<V>(b * n + (m == 0 ? 0 : n - m))];
            V h = split_hc(A, Bc, m, n);
            const int j = 2 * (p0 + b);
            out[out_off + (size_t)m + (size_t)j * out_sj + (size_t)k * out_sk] = h.x;
            out[out_off + (size_t)m + (size_t)(j + 1) * out_sj + (size_t)k * out_sk] = h.y;
        }
    } else {
        for (int e = tid; e < nb * n; e += nthr) {
            const int m = e % n, b = e / n;
            V P = buf0[fpad<V>(b * n + m)], Q = buf0[fpad<V>(b * n + (m == 0 ? 0 : n - m))];
            buf1[fpad<V>(b * n + m)] = merge_hc(P, Q, m, n);
        }
        __syncthreads();
        V *res = fft_batch<V, false, false>(buf1, buf0, plan, nb, 1, n, tid, nthr);
        for (int e = tid; e < nb * n; e += nthr) {
            const int m = e % n, b = e / n;
            V z = res[fpad<V>(b * n + m)];
            const int j = 2 * (p0 + b);
            out[out_off + (size_t)m + (size_t)j * out_sj + (size_t)k * out_sk] = z.x * scale;
            out[out_off + (size_t)m + (size_t)(j + 1) * out_sj + (size_t)k * out_sk] = z.y * scale;
        }
    }
}

// y direction, in place on the interior-only array.  Columns 2c, 2c+1 of a row
// are adjacent, so the complex line of pair c is the V-typed column c of the
// plane viewed as [ny][nx/2] complex.  CTA = `w` pairs of plane k.
template <typename T, bool FWD>
__global__ void __launch_bounds__(256) k_yfft(T *__restrict__ data, FftPlanDev<typename cplx_of<T>::type> plan,
                                              int nx, int w)
{
    using V = typename cplx_of<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = plan.n; // = ny
    const int ncol = nx / 2;
    V *buf0 = reinterpret_cast<V *>(smem_raw);
    V *buf1 = buf0 + fpad_elems<V>(w * n);
    const int k = blockIdx.y;
    const int c0 = blockIdx.x * w;
    const int nb = min(w, ncol - c0);
    const int tid = threadIdx.x, nthr = blockDim.x;
    V *plane = reinterpret_cast<V *>(data) + (size_t)k * n * ncol;

    for (int e = tid; e < nb * n; e += nthr) {
        const int c = e % nb, m = e / nb;
        buf0[fpad<V>(m * w + c)] = plane[(size_t)m * ncol + c0 + c];
    }
    __syncthreads();
    if (FWD) {
        V *res = fft_batch<V, true, true>(buf0, buf1, plan, nb, w, 1, tid, nthr);
        for (int e = tid; e < nb * n; e += nthr) {
            const int c = e % nb, m = e / nb;
            V A = res[fpad<V>(m * w + c)], Bc = res[fpad<V>((m == 0 ? 0 : n - m) * w + c)];
            plane[(size_t)m * ncol + c0 + c] = split_hc(A, Bc, m, n);
        }
    } else {
        for (int e = tid; e < nb * n; e += nthr) {
            const int c = e % nb, m = e / nb;
            V P = buf0[fpad<V>(m * w + c)], Q = buf0[fpad<V>((m == 0 ? 0 : n - m) * w + c)];
            buf1[fpad<V>(m * w + c)] = merge_hc(P, Q, m, n);
        }
        __syncthreads();
        V *res = fft_batch<V, false, true>(buf1, buf0, plan, nb, w, 1, tid, nthr);
        for (int e = tid; e < nb * n; e += nthr) {
            const int c = e % nb, m = e / nb;
            plane[(size_t)m * ncol + c0 + c] = res[fpad<V>(m * w + c)];
        }
    }
}

// Compile-time-length version of k_xfft (same layout, same arithmetic): N is
// the line length, the batch per CTA is a constant, and the twiddle table is
// staged in shared memory.  Used for the strided (ghosted) layout of the
// host-pointer drop-in.
template <int N> __host__ __device__ constexpr int ct_x_lines() { return N >= 1024 ? 1 : 1024 / N; }

template <typename T, int N, bool FWD>
__global__ void __launch_bounds__(256) k_xfft_ct(const T *__restrict__ in, size_t in_off, size_t in_sj, size_t in_sk,
                                                 T *__restrict__ out, size_t out_off, size_t out_sj, size_t out_sk,
                                                 const typename cplx_of<T>::type *__restrict__ twg, int ny, T scale)
{
    using V = typename cplx_of<T>::type;
    constexpr int NB = ct_x_lines<N>(), BUF = fpad_elems<V>(NB * N);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *buf0 = reinterpret_cast<V *>(smem_raw);
    V *buf1 = buf0 + BUF;
    V *tw = buf1 + BUF;
    const int k = blockIdx.y;
    const int p0 = blockIdx.x * NB;
    const int nb = min(NB, ny / 2 - p0);
    const int tid = threadIdx.x;
    ct_build_twiddles<V, N, 256>(twg, tw, tid);
    for (int e = tid; e < nb * 2 * N; e += 256) {
        const int m = e % N, r = (e / N) & 1, b = e / (2 * N);
        const int j = 2 * (p0 + b) + r;
        T val = in[in_off + (size_t)m + (size_t)j * in_sj + (size_t)k * in_sk];
        reinterpret_cast<T *>(&buf0[fpad<V>(b * N + m)])[r] = val;
    }
    __syncthreads();
    if (FWD) {
        V *res = ct_batch<V, true, false, N, NB, 1, N, 256>(buf0, buf1, nb, tw, tid);
        for (int e = tid; e < nb * N; e += 256) {
            const int m = e % N, b = e / N;
            V A = res[fpad<V>(b * N + m)], Bc = res[fpad<V>(b * N + (m == 0 ? 0 : N - m))];
            V h = split_hc(A, Bc, m, N);
            const int j = 2 * (p0 + b);
            out[out_off + (size_t)m + (size_t)j * out_sj + (size_t)k * out_sk] = h.x;
            out[out_off + (size_t)m + (size_t)(j + 1) * out_sj + (size_t)k * out_sk] = h.y;
        }
    } else {
        for (int e = tid; e < nb * N; e += 256) {
            const int m = e % N, b = e / N;
            V P = buf0[fpad<V>(b * N + m)], Q = buf0[fpad<V>(b * N + (m == 0 ? 0 : N - m))];
            buf1[fpad<V>(b * N + m)] = merge_hc(P, Q, m, N);
        }
        __syncthreads();
        V *res = ct_batch<V, false, false, N, NB, 1, N, 256>(buf1, buf0, nb, tw, tid);
        for (int e = tid; e < nb * N; e += 256) {
            const int m = e % N, b = e / N;
            V z = res[fpad<V>(b * N + m)];
            const int j = 2 * (p0 + b);
            out[out_off + (size_t)m + (size_t)j * out_sj + (size_t)k * out_sk] = z.x * scale;
            out[out_off + (size_t)m + (size_t)(j + 1) * out_sj + (size_t)k * out_sk] = z.y * scale;
        }
    }
}

// threadIdx.x through a volatile move: index arithmetic derived from it inside
// a persistent loop is recomputed per iteration instead of being hoisted and
// held in registers across the whole loop (which cost occupancy)
__device__ __forceinline__ int opaque_tid()
{
    int t;
    asm volatile("mov.u32 %0, %%tid.x;" : "=r"(t));
    return t;
}

// pressure update of one point o (PressureUpdate in ppe.cuh); dp is the
// FP32 increment
__device__ __forceinline__ void pressure_update(const PressureUpdate &pu, size_t o, float dp)
{
    const float pn = (pu.incremental ? __ldg(pu.q + o) : 0.f) + dp;
    const float pold = __ldg(pu.p + o);
    // the prediction first: storing over the just-read p before another
    // stream measured markedly slower on B200
    pu.qnext[o] = pu.qmode ? 2.f * pn - pold : pn;
    pu.p[o] = pn;
}

// the same from the staged prediction q and old pressure pold of point o
__device__ __forceinline__ void pressure_update_staged(const PressureUpdate &pu, size_t o, float dp, float q,
                                                       float pold)
{
    const float pn = (pu.incremental ? q : 0.f) + dp;
    pu.qnext[o] = pu.qmode ? 2.f * pn - pold : pn;
    pu.p[o] = pn;
}

__global__ void __launch_bounds__(256) k_pressure_update(const float *__restrict__ dp, PressureUpdate pu, size_t n)
{
    for (size_t o = (size_t)blockIdx.x * 256 + threadIdx.x; o < n; o += (size_t)gridDim.x * 256)
        pressure_update(pu, o, __ldg(dp + o));
}

// Persistent versions on the compact layout [k][j][i] (the device solves).
// Each CTA walks line groups g = blockIdx.x, + gridDim.x, ...  The raw data
// of the next group is copied global -> shared with cp.async into a staging
// buffer while the current group is transformed in place in the work
// buffer, so load latency overlaps the butterflies without holding the data
// in registers.  The staging copy into the work buffer pairs the two real
// lines into complex values (and, for the inverse, merges the half-complex
// spectra).  The y kernel moves whole 32-byte sectors: W column pairs of V
// per row (W * sizeof(V) = 64 bytes when N allows).
// (FP64: the forward transform measured faster with 8 columns at N = 384,
// 0.173 -> 0.160 ms at 512x384x256, the inverse with 4, 0.177 against 0.182)
template <typename V, int N, bool FWD> __host__ __device__ constexpr int pf_y_cols()
{
    return sizeof(V) == 8 ? ((3072 / N) >= 8 ? 8 : ((3072 / N) >= 4 ? 4 : 2))
                          : (FWD && (3072 / N) >= 8 ? 8 : ((1536 / N) >= 4 ? 4 : ((1536 / N) >= 2 ? 2 : 1)));
}

// threads per CTA of the persistent x kernel, and line pairs per group: one
// radix-8 stage of a group is one butterfly per thread
template <typename T> __host__ __device__ constexpr int pf_y_threads() { return 256; }
template <typename T> __host__ __device__ constexpr int pf_x_threads() { return sizeof(T) == 8 ? 64 : 256; }
template <typename T, int N> __host__ __device__ constexpr int pf_x_lines()
{
    return (pf_x_threads<T>() * 8 / N) < 1 ? 1 : pf_x_threads<T>() * 8 / N;
}
// shared memory of the persistent kernels, in V elements: work buffer,
// staging buffer (rounded to an even count), per-stage twiddle table
template <typename T, int N> __host__ __device__ constexpr int pf_x_smem_elems()
{
    using V = typename cplx_of<T>::type;
    return (fpad_elems<V>(pf_x_lines<T, N>() * N) + 1) / 2 * 2 + pf_x_lines<T, N>() * N + N;
}
// ... and with the mixed pressure update fused (FP32 inverse): the group's
// rows of the prediction q and of the old pressure, staged (bytes)
template <typename T, int N> __host__ __device__ constexpr int pf_x_pu_bytes()
{
    return 2 * 2 * pf_x_lines<T, N>() * N * 4;
}
template <typename T, int N, bool FWD> __host__ __device__ constexpr int pf_y_smem_elems()
{
    using V = typename cplx_of<T>::type;
    return (fpad_elems<V>(pf_y_cols<V, N, FWD>() * N) + 1) / 2 * 2 + pf_y_cols<V, N, FWD>() * N + N;
}

// PU (FP32 inverse only): the pressure update of the mixed path is fused
// into the last stage; the group's rows of q and of the old pressure are
// copied into shared memory when the group starts, so their latency hides
// behind its butterflies instead of sitting in the epilogue.
template <typename T, int N, bool FWD, bool PU = false>
__global__ void __launch_bounds__(pf_x_threads<T>()) k_xfft_pf(const T *__restrict__ in, T *__restrict__ out,
                                                               const typename cplx_of<T>::type *__restrict__ twg,
                                                               int ny, int total, T scale, PressureUpdate pu)
{
    static_assert(!PU || (sizeof(T) == 4 && !FWD), "the fused pressure update is the FP32 inverse's");
    using V = typename cplx_of<T>::type;
    constexpr int NT = pf_x_threads<T>();
    constexpr int NB = pf_x_lines<T, N>(), BUF = (fpad_elems<V>(NB * N) + 1) / 2 * 2;
    constexpr int CH = 16 / sizeof(T); // T values per 16-byte copy
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *buf = reinterpret_cast<V *>(smem_raw);
    T *stage = reinterpret_cast<T *>(buf + BUF); // 2 NB rows of N values, 16-byte aligned
    V *tw = reinterpret_cast<V *>(stage + 2 * NB * N);
    float *pst = reinterpret_cast<float *>(tw + N); // PU: [2][2 NB N], q then the old pressure
    const int tid = threadIdx.x;
    const int gpk = (ny / 2 + NB - 1) / NB; // groups per k-plane
    ct_build_twiddles<V, N, NT>(twg, tw, tid);
    // PU: the group's rows of q and p (the run the group writes), one commit group
    auto fetch_pu = [&](int g) {
        const int k = g / gpk, p0 = (g % gpk) * NB, cnt = min(NB, ny / 2 - p0) * 2 * N;
        const size_t o = (size_t)k * N * ny + (size_t)2 * p0 * N;
        for (int e = tid * 4; e < cnt; e += NT * 4) {
            if (pu.incremental) cp_async_16(pst + e, pu.q + o + e);
            cp_async_16(pst + 2 * NB * N + e, pu.p + o + e);
        }
        cp_async_commit();
    };
    // rows 2 p0 .. 2 p0 + 2 nb - 1 of plane k are one contiguous run
    auto fetch = [&](int g) {
        const int k = g / gpk, p0 = (g % gpk) * NB, cnt = min(NB, ny / 2 - p0) * 2 * N;
        const T *src = in + (size_t)k * N * ny + (size_t)2 * p0 * N;
        for (int e = tid * CH; e < cnt; e += NT * CH) cp_async_16(stage + e, src + e);
        cp_async_commit();
    };
    if (blockIdx.x < total) fetch(blockIdx.x);
    for (int g = blockIdx.x; g < total; g += gridDim.x) {
        const int tid = opaque_tid();
        const int k = g / gpk, p0 = (g % gpk) * NB, nb = min(NB, ny / 2 - p0);
        cp_async_wait<0>(); // this thread's copies of group g have landed
        __syncthreads();    // ... and everyone's; the previous group is done with buf (and pst)
        if (PU) fetch_pu(g);
        // first stage straight from the staged rows: line b pairs rows 2b, 2b+1
        auto in = [&](int b, int m) {
            const T *r0 = stage + 2 * b * N, *r1 = r0 + N;
            V z;
            if (FWD) {
                z.x = r0[m];
                z.y = r1[m];
            } else {
                const int mc = (m == 0) ? 0 : N - m;
                V P, Q;
                P.x = r0[m];
                P.y = r1[m];
                Q.x = r0[mc];
                Q.y = r1[mc];
                z = merge_hc(P, Q, m, N);
            }
            return z;
        };
        ct_first_stage<V, FWD, false, N, NB, 1, N, NT>(buf, nb, in, tid);
        __syncthreads();
        if (g + (int)gridDim.x < total)
            fetch(g + gridDim.x);
        else if (PU)
            cp_async_commit(); // one group after fetch_pu(g), as in the other rounds
        T *dst = out + (size_t)k * N * ny + (size_t)2 * p0 * N;
        if constexpr (FWD) {
            ct_batch_ip<V, FWD, false, N, NB, 1, N, NT, 1, ct_nstages(N) - 1>(buf, nb, tw, tid);
            // the last stage splits line b into its two half-complex rows from registers
            auto put = [&](int b, int m, V A, V Bc) {
                const V h = split_hc(A, Bc, m, N);
                dst[(size_t)2 * b * N + m] = h.x;
                dst[(size_t)(2 * b + 1) * N + m] = h.y;
            };
            ct_last_stage_pairs<V, FWD, false, N, NB, 1, N, NT>(buf, nb, tw, tid, put);
        } else {
            ct_batch_ip<V, FWD, false, N, NB, 1, N, NT, 1, ct_nstages(N) - 1>(buf, nb, tw, tid);
            if (PU) {
                cp_async_wait<1>(); // fetch_pu(g) landed (the next group's fetch may be in flight)
                __syncthreads();
            }
            // the last stage writes the two real rows of line b from registers
            auto put = [&](int b, int m, V z) {
                const T d0 = z.x * scale, d1 = z.y * scale;
                dst[(size_t)2 * b * N + m] = d0; // mixed: the increment itself, for the correction
                dst[(size_t)(2 * b + 1) * N + m] = d1;
                if (PU) {
                    const int r = 2 * b * N + m;
                    const size_t o = (size_t)k * N * ny + (size_t)2 * p0 * N + r;
                    pressure_update_staged(pu, o, (float)d0, pst[r], pst[2 * NB * N + r]);
                    pressure_update_staged(pu, o + N, (float)d1, pst[r + N], pst[2 * NB * N + r + N]);
                }
            };
            ct_last_stage<V, FWD, false, N, NB, 1, N, NT>(buf, nb, tw, tid, put);
        }
    }
    cp_async_wait<0>();
}

template <typename T, int N, bool FWD>
// CTAs per SM the register budget is cut for, as measured fastest at
// N = 384: up to 80 registers (three CTAs) for FP32 lines up to 512 and for
// the FP64 inverse (a spill of 4-16 bytes, served from L1, costs less than
// the third CTA gains), 128 (two) for the FP64 forward, which would spill
// 80 bytes at 80; longer lines keep more registers rather than spill
__global__ void __launch_bounds__(pf_y_threads<T>(),
                                  sizeof(T) == 4 ? (N <= 512 ? 3 : 2) : (N <= 512 ? (FWD ? 2 : 3) : 1))
    k_yfft_pf(T *__restrict__ data, const typename cplx_of<T>::type *__restrict__ twg,
                                                 int nx, int total)
{
    using V = typename cplx_of<T>::type;
    constexpr int NT = pf_y_threads<T>();
    constexpr int W = pf_y_cols<V, N, FWD>(), BUF = (fpad_elems<V>(W * N) + 1) / 2 * 2, RAW = W * N;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ncol = nx / 2;
    V *buf = reinterpret_cast<V *>(smem_raw);
    V *stage = buf + BUF; // [m][c], dense
    V *tw = stage + RAW;
    const int tid = threadIdx.x;
    const int gpk = (ncol + W - 1) / W;
    ct_build_twiddles<V, N, NT>(twg, tw, tid);
    auto fetch = [&](int g) {
        const int k = g / gpk, c0 = (g % gpk) * W, nb = min(W, ncol - c0);
        const V *plane = reinterpret_cast<const V *>(data) + (size_t)k * N * ncol;
        if (sizeof(V) == 8 && W % 2 == 0 && ncol % 2 == 0) {
            // FP32: two columns per 16-byte copy (c0 and c even, rows of even
            // length: 16-byte aligned); a lone last column takes an 8-byte one
            for (int e = 2 * tid; e < RAW; e += 2 * NT) {
                const int c = e % W, m = e / W;
                if (c + 1 < nb)
                    cp_async_16(stage + e, plane + (size_t)m * ncol + c0 + c);
                else if (c < nb)
                    cp_async_8(stage + e, plane + (size_t)m * ncol + c0 + c);
            }
        } else {
            for (int e = tid; e < RAW; e += NT) {
                const int c = e % W, m = e / W;
                if (c < nb) {
                    if (sizeof(V) == 16)
                        cp_async_16(stage + e, plane + (size_t)m * ncol + c0 + c);
                    else
                        cp_async_8(stage + e, plane + (size_t)m * ncol + c0 + c);
                }
            }
        }
        cp_async_commit();
    };
    if (blockIdx.x < total) fetch(blockIdx.x);
    for (int g = blockIdx.x; g < total; g += gridDim.x) {
        const int k = g / gpk, c0 = (g % gpk) * W, nb = min(W, ncol - c0);
        V *plane = reinterpret_cast<V *>(data) + (size_t)k * N * ncol;
        cp_async_wait<0>();
        __syncthreads();
        // first stage straight from the staged columns ([m][c])
        auto in = [&](int c, int m) {
            if (FWD) return stage[m * W + c];
            return merge_hc(stage[m * W + c], stage[(m == 0 ? 0 : N - m) * W + c], m, N);
        };
        ct_first_stage<V, FWD, true, N, W, W, 1, NT>(buf, nb, in, tid);
        __syncthreads();
        if (g + (int)gridDim.x < total) fetch(g + gridDim.x);
        if constexpr (FWD) {
            ct_batch_ip<V, FWD, true, N, W, W, 1, NT, 1, ct_nstages(N) - 1>(buf, nb, tw, tid);
            auto put = [&](int c, int m, V A, V Bc) { plane[(size_t)m * ncol + c0 + c] = split_hc(A, Bc, m, N); };
            ct_last_stage_pairs<V, FWD, true, N, W, W, 1, NT>(buf, nb, tw, tid, put);
        } else {
            ct_batch_ip<V, FWD, true, N, W, W, 1, NT, 1, ct_nstages(N) - 1>(buf, nb, tw, tid);
            auto put = [&](int c, int m, V z) { plane[(size_t)m * ncol + c0 + c] = z; };
            ct_last_stage<V, FWD, true, N, W, W, 1, NT>(buf, nb, tw, tid, put);
        }
    }
    cp_async_wait<0>();
}
// calcRHS (mod_calcRHS.f90:19-33) fused into the forward x transform.  One
// group is one line pair (rows 2p, 2p+1 of interior plane k); its staging
// holds, as FP64 rows of the ghosted fields (plane kg = k + 1): u rows 2p,
// 2p+1; v rows 2p-1 (periodic), 2p, 2p+1; w rows 2p, 2p+1 of planes kg and
// kg - 1.  The first Stockham stage forms rhs = div(u)/dt of the two rows
// with k_calc_rhs_fp64's expression (u_{i-1} is in the same periodic row)
// and pairs them into one complex line, so neither the right-hand side nor
// its re-read crosses HBM.  When `part` is given, each group also writes the
// FP64 sum of its rhs values (in a fixed order) for the plane sums of the
// mixed path's (0,0) mode.
constexpr int XDIV_THREADS = 64;

template <typename T, int N> __host__ __device__ constexpr int xdiv_smem_bytes()
{
    using V = typename cplx_of<T>::type;
    // work buffer, 9 staged FP64 rows, per-stage twiddles, 2 warp sums
    return (int)(sizeof(V) * ((fpad_elems<V>(N) + 1) / 2 * 2) + 8 * 9 * N + sizeof(V) * N + 16);
}

template <typename T, int N>
__global__ void __launch_bounds__(XDIV_THREADS) k_xfft_div_pf(DivIn d, T *__restrict__ out,
                                                              const typename cplx_of<T>::type *__restrict__ twg,
                                                              int ny, int total, double *__restrict__ part)
{
    using V = typename cplx_of<T>::type;
    constexpr int NT = XDIV_THREADS, BUF = (fpad_elems<V>(N) + 1) / 2 * 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *buf = reinterpret_cast<V *>(smem_raw);
    double *stage = reinterpret_cast<double *>(buf + BUF); // rows: u0 u1 | v- v0 v1 | w0 w1 | w0m w1m
    V *tw = reinterpret_cast<V *>(stage + 9 * N);
    double *wsum = reinterpret_cast<double *>(tw + N);
    const int tid = threadIdx.x;
    const int gpk = ny / 2;
    const size_t sk = (size_t)N * ny;
    ct_build_twiddles<V, N, NT>(twg, tw, tid);
    auto copy_rows = [&](double *dst, const double *src, int n) {
        for (int e = tid * 2; e < n; e += NT * 2) cp_async_16(dst + e, src + e);
    };
    auto fetch = [&](int g) {
        const int k = g / gpk, p = g % gpk, kg = k + 1;
        const size_t r0 = sk * kg + (size_t)2 * p * N;
        copy_rows(stage, d.u + r0, 2 * N);
        copy_rows(stage + 2 * N, d.v + sk * kg + (size_t)(p == 0 ? ny - 1 : 2 * p - 1) * N, N);
        copy_rows(stage + 3 * N, d.v + r0, 2 * N);
        copy_rows(stage + 5 * N, d.w + r0, 2 * N);
        copy_rows(stage + 7 * N, d.w + r0 - sk, 2 * N);
        cp_async_commit();
    };
    if (blockIdx.x < total) fetch(blockIdx.x);
    for (int g = blockIdx.x; g < total; g += gridDim.x) {
        const int k = g / gpk, p = g % gpk;
        const double dtidzi_k = __ldg(d.dzf_inv + k + 1);
        cp_async_wait<0>();
        __syncthreads();
        double acc = 0.0;
        auto in = [&](int, int m) {
            const int mm = (m == 0) ? N - 1 : m - 1;
            const double *u0 = stage, *u1 = stage + N, *vm = stage + 2 * N, *v0 = stage + 3 * N, *v1 = stage + 4 * N;
            const double *w0 = stage + 5 * N, *w1 = stage + 6 * N, *w0m = stage + 7 * N, *w1m = stage + 8 * N;
            const double r0 = (u0[m] - u0[mm]) * d.dtidxi + (v0[m] - vm[m]) * d.dtidyi + (w0[m] - w0m[m]) * d.dti * dtidzi_k;
            const double r1 = (u1[m] - u1[mm]) * d.dtidxi + (v1[m] - v0[m]) * d.dtidyi + (w1[m] - w1m[m]) * d.dti * dtidzi_k;
            acc += r0 + r1;
            V z;
            z.x = (T)r0;
            z.y = (T)r1;
            return z;
        };
        ct_first_stage<V, true, false, N, 1, 1, N, NT>(buf, 1, in, tid);
        if (part != nullptr) { // the group's sum, in a fixed order
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
            if ((tid & 31) == 0) wsum[tid >> 5] = acc;
        }
        __syncthreads();
        if (part != nullptr && tid == 0) part[g] = wsum[0] + wsum[1];
        if (g + (int)gridDim.x < total) fetch(g + gridDim.x);
        T *dst = out + (size_t)k * N * ny + (size_t)2 * p * N;
        ct_batch_ip<V, true, false, N, 1, 1, N, NT, 1, ct_nstages(N) - 1>(buf, 1, tw, tid);
        auto put = [&](int, int m, V A, V Bc) {
            const V h = split_hc(A, Bc, m, N);
            dst[m] = h.x;
            dst[N + m] = h.y;
        };
        ct_last_stage_pairs<V, true, false, N, 1, 1, N, NT>(buf, 1, tw, tid, put);
    }
    cp_async_wait<0>();
}

// ------------------------------------------------------------------------
// Tridiagonal kernels (FP64 arithmetic in both precision modes)
// ------------------------------------------------------------------------

struct TridDev {
    int nx, ny, nz, ncx, ncy;
    const double *mult, *rb, *c;
};

__device__ __forceinline__ size_t trid_class(int px, int py, const TridDev &t)
{
    const int ix = min(px, t.nx - px), jy = min(py, t.ny - py);
    return (size_t)ix + (size_t)t.ncx * jy;
}

// rows per load batch of the Thomas sweeps: measured best at 4 for FP64
// data (in place) and 8 for the FP32 input with the FP64 sweep scratch
template <typename T> __host__ __device__ constexpr int trid_unroll() { return sizeof(T) == 8 ? 4 : 8; }

// Thomas on rows [k0, k0+ke) of one column.  Reads the right-hand side from
// `xin` (type T), keeps the forward-swept values in `xs` (double; may alias
// xin when T is double) and writes the solution to `xout` (type TO, T by
// default; may alias xs).
template <typename T, typename TO = T>
__device__ __forceinline__ void thomas_column(const T *xin, double *xs, TO *xout, size_t col, size_t cls,
                                              size_t stride, size_t cstride, int k0, int ke, const TridDev &t)
{
    constexpr int TRID_UNROLL = trid_unroll<T>();
    // forward elimination: x_k -= (a_k / b_{k-1}) x_{k-1}   (ssolve_trid :319-330)
    double xp = (double)xin[col + (size_t)k0 * stride];
    xs[col + (size_t)k0 * stride] = xp;
    for (int kb = 1; kb < ke; kb += TRID_UNROLL) {
        double xv[TRID_UNROLL], mv[TRID_UNROLL];
#pragma unroll
        for (int u = 0; u < TRID_UNROLL; u++) {
            const int k = k0 + kb + u;
            if (kb + u < ke) {
                xv[u] = (double)xin[col + (size_t)k * stride];
                mv[u] = __ldg(t.mult + cls + (size_t)k * cstride);
            }
        }
#pragma unroll
        for (int u = 0; u < TRID_UNROLL; u++) {
            if (kb + u < ke) {
                xp = xv[u] - mv[u] * xp;
                xs[col + (size_t)(k0 + kb + u) * stride] = xp;
            }
        }
    }
    // last row: x /= b, or 0 where b == 0 (:332-344); rb holds 1/b or 0
    const int kl = k0 + ke - 1;
    xp = xp * __ldg(t.rb + cls + (size_t)kl * cstride);
    xout[col + (size_t)kl * stride] = (TO)xp;
    // back substitution: x_k = (x_k - c_k x_{k+1}) / b_k   (:346-356)
    for (int kb = ke - 2; kb >= 0; kb -= TRID_UNROLL) {
        double xv[TRID_UNROLL], rv[TRID_UNROLL];
#pragma unroll
        for (int u = 0; u < TRID_UNROLL; u++) {
            const int k = k0 + kb - u;
            if (kb - u >= 0) {
                xv[u] = xs[col + (size_t)k * stride];
                rv[u] = __ldg(t.rb + cls + (size_t)k * cstride);
            }
        }
#pragma unroll
        for (int u = 0; u < TRID_UNROLL; u++) {
            const int k = k0 + kb - u;
            if (kb - u >= 0) {
                xp = (xv[u] - __ldg(t.c + k) * xp) * rv[u];
                xout[col + (size_t)k * stride] = (TO)xp;
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(128) k_thomas(const T *xin, double *xs, T *xout, TridDev t, const double *mode0)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    if (px >= t.nx) return;
    const size_t col = (size_t)px + (size_t)t.nx * py, stride = (size_t)t.nx * t.ny;
    const size_t cls = trid_class(px, py, t), cstride = (size_t)t.ncx * t.ncy;
    if (mode0 != nullptr && col == 0) {
        // Mixed path, (kx,ky) = (0,0): the Neumann system is singular (its
        // last pivot is round-off), so its FP32-transformed right-hand side
        // is not consistent to the precision the division needs.  Solve it in
        // FP64 from the FP64 plane sums of the right-hand side, with the
        // gauge x[nz-1] = 0 fixing the free constant.
        double xp = mode0[0];
        xs[0] = xp;
        for (int k = 1; k < t.nz; k++) {
            xp = mode0[k] - __ldg(t.mult + (size_t)k * cstride) * xp;
            xs[(size_t)k * stride] = xp;
        }
        double xn = 0.0;
        xout[(size_t)(t.nz - 1) * stride] = (T)0;
        for (int k = t.nz - 2; k >= 0; k--) {
            xn = (xs[(size_t)k * stride] - __ldg(t.c + k) * xn) * __ldg(t.rb + (size_t)k * cstride);
            xout[(size_t)k * stride] = (T)xn;
        }
        return;
    }
    thomas_column<T>(xin, xs, xout, col, cls, stride, cstride, 0, t.nz, t);
}

// Thomas with the forward-swept values in tensor memory.  The in-place sweep
// above writes every swept value to HBM and reads it back (32 B/point in
// FP64), because the 402 MB of a 512x384x256 sweep does not stay in L2.
// Here each of the 128 threads of a CTA (one per SM: its shared memory is
// over half the SM's) keeps the swept values of its column in its own TMEM
// lane (up to 256 rows; see below for taller columns), so HBM sees the
// right-hand side once, the solution once and the class tables.  The loads are per-thread cp.async copies into a ring of
// TTM_NS groups of TTM_G rows in shared memory, TTM_NS - 1 groups ahead;
// each thread reads only its own copies, so the pipeline has no barrier and
// no wait other than cp.async.wait_group on the thread's own copies.  The
// copy stream of a round is the forward groups (rhs + multipliers) then the
// backward groups (reciprocal pivots), and runs on into the next round's
// columns.  The arithmetic is thomas_column's, operation for operation.
//
// A lane holds 256 doubles.  Taller columns (nz <= TTM_MAX_NZ) keep their
// bottom TTM_TM_ROWS - TTM_TOP_ROWS and top TTM_TOP_ROWS rows in tensor
// memory and the rows between in an HBM scratch (FP64: in place), which the
// backward sweep prefetches through the copy ring.  The top rows stay on
// chip because the ring runs NS - 1 groups ahead: a backward group's
// prefetch is issued after the forward store of its rows only from the
// NS/2-th group below the top on.
constexpr int TTM_THREADS = 128, TTM_G = 8, TTM_NS = 8, TTM_MAX_NZ = 1024, TTM_TM_ROWS = 256, TTM_TOP_ROWS = 32;
static_assert(TTM_TOP_ROWS >= (TTM_NS / 2) * TTM_G, "the HBM rows' prefetch must follow their store");

template <typename T> __host__ __device__ constexpr size_t ttm_smem_bytes(int nz)
{
    // table ring [NS][G][128] (double), rhs ring [NS][G][128] (T), (0,0)-mode
    // rhs ring [NS][G] (double), c_k [TTM_MAX_NZ], TMEM address slot, and for
    // FP32 right-hand sides of tall columns a ring of the HBM rows (double;
    // FP64 reuses the rhs ring); at least 116 KB so that two CTAs never share
    // an SM (each may take all 512 TMEM columns)
    const size_t b = (size_t)TTM_NS * TTM_G * TTM_THREADS * (8 + sizeof(T)) + TTM_NS * TTM_G * 8 + TTM_MAX_NZ * 8 +
                     16 + ((sizeof(T) == 4 && nz > TTM_TM_ROWS) ? (size_t)TTM_NS * TTM_G * TTM_THREADS * 8 : 0);
    return b < 116 * 1024 ? 116 * 1024 : b;
}

// Processing order of the y rows: 0, 1, ny-1, 2, ny-2, ..., ny/2 (ny even),
// so that rows py and ny - py, which share their class tables, run together.
__device__ __forceinline__ int trid_pair_row(int b, int ny)
{
    if (b == 0) return 0;
    if (b == ny - 1) return ny / 2;
    const int jy = (b + 1) / 2;
    return (b & 1) ? jy : ny - jy;
}

// One thread's column in one round of the persistent loop.
struct TtmColumn {
    bool valid;
    size_t col, cls;
};

// TALL: nz > TTM_TM_ROWS (the HBM-scratch rows exist); a compile-time switch,
// so that shorter columns run the tensor-memory path alone
// TO: the solution's type (T by default; the slab sweep writes FP64).
// GAUGE: the (0,0) column (mode0 given) takes x[nz-1] = 0, the free
// constant of the singular whole-column system; a slab's partition system is
// regular and solves that column from the plane sums without it.
template <typename T, bool TALL, typename TO = T, bool GAUGE = true>
__global__ void __launch_bounds__(TTM_THREADS, 1)
    k_thomas_tmem(const T *xin, TO *xout, double *xsc, TridDev t, const double *mode0, int rounds, uint32_t tcols)
{
    constexpr int G = TTM_G, NS = TTM_NS, NT = TTM_THREADS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *cring = reinterpret_cast<double *>(smem_raw);          // [NS][G][NT] mult (fwd) / rb (bwd)
    T *xring = reinterpret_cast<T *>(cring + NS * G * NT);           // [NS][G][NT] right-hand side
    double *zring = reinterpret_cast<double *>(xring + NS * G * NT); // [NS][G] (0,0) mode right-hand side
    double *csh = zring + NS * G;                                    // [nz] c_k
    uint32_t *tslot = reinterpret_cast<uint32_t *>(csh + TTM_MAX_NZ);
    double *sring = sizeof(T) == 8 ? reinterpret_cast<double *>(xring) : csh + TTM_MAX_NZ + 2; // HBM rows, bwd
    const int tid = threadIdx.x, warp = tid >> 5;
    const int nz = t.nz, ngf = nz / G, per_round = 2 * ngf;
    // rows [kb, kt) live in the HBM scratch (none when nz <= TTM_TM_ROWS);
    // row k < kb sits at TMEM cell 2k, row k >= kt at 2 (kb + k - kt)
    const int kb = TALL ? TTM_TM_ROWS - TTM_TOP_ROWS : nz, kt = TALL ? nz - TTM_TOP_ROWS : nz;
    auto in_hbm = [&](int k0) { return TALL && k0 >= kb && k0 < kt; }; // k0: first row of an 8-row group
    auto tcell = [&](int k0) { return TALL ? 2 * (k0 < kb ? k0 : kb + k0 - kt) : 2 * k0; };
    const size_t stride = (size_t)t.nx * t.ny, cstride = (size_t)t.ncx * t.ncy;
    const int ncol = t.nx * t.ny;

    for (int k = tid; k < nz; k += NT) csh[k] = __ldg(t.c + k);
    if (warp == 0) tmem_alloc(tslot, tcols);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tbase = *tslot + ((uint32_t)(warp * 32) << 16);

    auto column = [&](int r) {
        TtmColumn c{false, 0, 0};
        const int q = (r * (int)gridDim.x + (int)blockIdx.x) * NT + tid;
        if (q < ncol) {
            const int b = q / t.nx, px = q - b * t.nx, py = trid_pair_row(b, t.ny);
            c = TtmColumn{true, (size_t)px + (size_t)t.nx * py, trid_class(px, py, t)};
        }
        return c;
    };
    // the (0,0) mode of the mixed path: column 0, which is thread 0's of
    // CTA 0 in round 0 (processing row 0 is y row 0)
    const bool zcta = (mode0 != nullptr) && blockIdx.x == 0;

    // copy stream: round ir, group ig, ring slot islot; the source pointers
    // walk down (forward) and up (backward) the current column row by row
    int ir = 0, ig = 0, islot = 0;
    TtmColumn ic = column(0);
    const T *xsrc = xin + ic.col;
    const double *msrc = t.mult + ic.cls, *rsrc = t.rb + ic.cls + (size_t)(nz - 1) * cstride;
    const double *ssrc = xsc + ic.col + (size_t)(nz - 1) * stride;
    auto issue_next = [&]() {
        if (ir < rounds) {
            double *cdst = cring + islot * G * NT + tid;
            if (ig < ngf) {
                T *xdst = xring + islot * G * NT + tid;
                const bool z = zcta && ir == 0 && tid == 0;
                if (ic.valid) {
#pragma unroll
                    for (int u = 0; u < G; u++) {
                        cp_async_8(cdst + u * NT, msrc);
                        if (z)
                            cp_async_8(zring + islot * G + u, mode0 + ig * G + u);
                        else if (sizeof(T) == 8)
                            cp_async_8(xdst + u * NT, xsrc);
                        else
                            cp_async_4(xdst + u * NT, xsrc);
                        msrc += cstride;
                        xsrc += stride;
                    }
                }
            } else if (ic.valid) {
                const bool hb = in_hbm(nz - (ig - ngf + 1) * G);
                double *sdst = sring + islot * G * NT + tid;
#pragma unroll
                for (int u = 0; u < G; u++) {
                    cp_async_8(cdst + u * NT, rsrc);
                    rsrc -= cstride;
                    if constexpr (TALL) {
                        if (hb) cp_async_8(sdst + u * NT, ssrc);
                        ssrc -= stride;
                    }
                }
            }
            if (++ig == per_round) {
                ig = 0;
                if (++ir < rounds) {
                    ic = column(ir);
                    xsrc = xin + ic.col;
                    msrc = t.mult + ic.cls;
                    rsrc = t.rb + ic.cls + (size_t)(nz - 1) * cstride;
                    ssrc = xsc + ic.col + (size_t)(nz - 1) * stride;
                }
            }
        }
        cp_async_commit(); // one group per step, empty or not
        islot = (islot + 1 == NS) ? 0 : islot + 1;
    };

    for (int q = 0; q < NS - 1; q++) issue_next();
    int slot = 0;
    for (int r = 0; r < rounds; r++) {
        const TtmColumn cc = column(r);
        const bool zr = zcta && r == 0; // warp-uniform
        // forward elimination: x_k -= (a_k / b_{k-1}) x_{k-1}   (ssolve_trid :319-330);
        // mult is 0 at k = 0, where it leaves x_0 as it is
        double xp = 0.0;
        for (int g = 0; g < ngf; g++) {
            cp_async_wait<NS - 2>(); // this step's group has landed
            const double *cs = cring + slot * G * NT + tid;
            const T *xs = xring + slot * G * NT + tid;
            double xv[G], mv[G];
#pragma unroll
            for (int u = 0; u < G; u++) {
                xv[u] = (double)xs[u * NT];
                mv[u] = cs[u * NT];
            }
            if (zr && tid == 0) {
#pragma unroll
                for (int u = 0; u < G; u++) xv[u] = zring[slot * G + u];
            }
            issue_next(); // refills the slot consumed one step ago
            uint32_t v[2 * G];
            const bool hb = in_hbm(g * G); // warp-uniform
#pragma unroll
            for (int u = 0; u < G; u++) {
                xp = xv[u] - mv[u] * xp;
                v[2 * u] = (uint32_t)__double2loint(xp);
                v[2 * u + 1] = (uint32_t)__double2hiint(xp);
                if (hb && cc.valid) xsc[cc.col + (size_t)(g * G + u) * stride] = xp;
            }
            if (!hb) {
                __syncwarp();
                tmem_st16(tbase + tcell(g * G), v);
            }
            slot = (slot + 1 == NS) ? 0 : slot + 1;
        }
        tmem_wait_st();
        // back substitution from the top row: x_k = (x_k - c_k x_{k+1}) / b_k
        // (:346-356); at k = nz-1, with x_{nz} = 0, it is x /= b (:332-344),
        // and the (0,0) mode takes the gauge x[nz-1] = 0 there
        xp = 0.0;
        TO *dst = xout + cc.col + (size_t)(nz - 1) * stride;
        for (int h = 0; h < ngf; h++) {
            const int ktop = nz - 1 - h * G; // rows ktop, ktop-1, ..., ktop-G+1
            uint32_t v[2 * G];
            const bool hb = in_hbm(ktop - G + 1); // warp-uniform
            if (!hb) {
                __syncwarp();
                tmem_ld16_start(tbase + tcell(ktop - G + 1), v);
            }
            cp_async_wait<NS - 2>();
            const double *cs = cring + slot * G * NT + tid;
            double rv[G], cv[G];
#pragma unroll
            for (int u = 0; u < G; u++) {
                rv[u] = cs[u * NT];
                cv[u] = csh[ktop - u];
            }
            if (GAUGE && zr && tid == 0 && h == 0) rv[0] = 0.0;
            issue_next();
            if (!hb) tmem_wait_ld(v);
            const double *ss = sring + slot * G * NT + tid;
#pragma unroll
            for (int u = 0; u < G; u++) {
                const int i = G - 1 - u;
                const double x = hb ? ss[u * NT] : __hiloint2double((int)v[2 * i + 1], (int)v[2 * i]);
                xp = (x - cv[u] * xp) * rv[u];
                if (cc.valid) *dst = (TO)xp;
                dst -= stride;
            }
            slot = (slot + 1 == NS) ? 0 : slot + 1;
        }
    }
    cp_async_wait<0>();
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after_sync();
        tmem_free(*tslot, tcols);
    }
}

// rows per ring group of the two-ended sweep below
constexpr int TTW_G = 8;

// Two-ended Thomas with one thread per half column (mixed path; 16 <= nz <=
// 256, nz % 16 == 0), the tables TridTables::tmult and trb (rows of tcs
// values).  A 256-thread CTA solves 128
// columns per round: threads 0-127 sweep the lower halves (rows 0 .. p-1, the
// LU elimination), threads 128-255 the upper halves (rows nz-1 .. p, the
// elimination from the top wall), each thread one chain of nz steps.  Both
// threads of a column share a tensor-memory lane (warps w and w+4 reach the
// same lanes): the lower half's swept rows at cells 2k, the upper half's at
// cells nz + 2(k - p).  They meet at the 2x2 system of rows p-1 and p through
// shared memory, one barrier per round.  (One thread per column with both
// chains interleaved ran at 0.179 ms against 0.186 for the one-ended sweep;
// this kernel, two warps per scheduler, at 0.177 ms, at 512x384x256: the
// per-row instruction latency binds, not the FP64 recurrence alone.)
constexpr int TTH_NS = 4;

template <typename T> __host__ __device__ constexpr size_t tth_smem_bytes()
{
    // ring [NS][G][256] of table values (double) and right-hand sides (T),
    // (0,0)-mode ring [NS][2][G], c_k and a_k [256], junction values [2][2][128],
    // TMEM address slot; at least 116 KB so that two CTAs never share an SM
    const size_t b = (size_t)TTH_NS * TTW_G * 2 * TTM_THREADS * (8 + sizeof(T)) + TTH_NS * 2 * TTW_G * 8 +
                     2 * TTM_TM_ROWS * 8 + 4 * TTM_THREADS * 8 + 16;
    return b < 116 * 1024 ? 116 * 1024 : b;
}

template <typename T>
__global__ void __launch_bounds__(2 * TTM_THREADS, 1)
    k_thomas_th(const T *xin, T *xout, const double *tm, const double *tr, const double *ak, const double *ck,
                int nx, int ny, int nz, int ncx, int ncy, long long tcs, const double *mode0, int rounds,
                uint32_t tcols)
{
    constexpr int G = TTW_G, NS = TTH_NS, NC = TTM_THREADS, NT = 2 * NC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *cring = reinterpret_cast<double *>(smem_raw);          // [NS][G][NT] tables
    T *xring = reinterpret_cast<T *>(cring + NS * G * NT);           // [NS][G][NT] right-hand side
    double *zring = reinterpret_cast<double *>(xring + NS * G * NT); // [NS][2][G] (0,0) mode
    double *csh = zring + NS * 2 * G;                                // c_k
    double *ash = csh + TTM_TM_ROWS;                                 // a_k
    double *jv = ash + TTM_TM_ROWS;                                  // [2 parities][2 halves][NC]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(jv + 4 * NC);
    const int tid = threadIdx.x, warp = tid >> 5, half = tid >= NC ? 1 : 0, lt = tid - half * NC;
    const int p = nz / 2, ngh = p / G, per_round = 2 * ngh;
    const long long stride = (long long)nx * ny, cstride = tcs;
    const int ncol = nx * ny;
    TridDev td{nx, ny, nz, ncx, ncy, nullptr, nullptr, nullptr};
    // this half's walk: forward from its wall towards the middle, backward
    // from the middle towards its wall
    const long long fx = half ? -stride : stride, fm = half ? -cstride : cstride, br = half ? cstride : -cstride;
    const int kx0 = half ? nz - 1 : 0, kr0 = half ? p : p - 1;

    for (int k = tid; k < nz; k += NT) {
        csh[k] = __ldg(ck + k);
        ash[k] = __ldg(ak + k);
    }
    if (warp == 0) tmem_alloc(tslot, tcols);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tbase = *tslot + ((uint32_t)((warp & 3) * 32) << 16) + (half ? (uint32_t)nz : 0u);

    auto column = [&](int r) {
        TtmColumn c{false, 0, 0};
        const int q = (r * (int)gridDim.x + (int)blockIdx.x) * NC + lt;
        if (q < ncol) {
            const int b = q / nx, px = q - b * nx, py = trid_pair_row(b, ny);
            c = TtmColumn{true, (size_t)px + (size_t)nx * py, trid_class(px, py, td)};
        }
        return c;
    };
    const bool zcta = (mode0 != nullptr) && blockIdx.x == 0;

    // copy stream: forward group g brings this half's rows kx0 +- (g G + u)
    // of the right-hand side and of tm, backward group h its rows
    // kr0 -+ (h G + u) of tr
    int ir = 0, ig = 0, islot = 0;
    TtmColumn ic = column(0);
    const T *xp_ = xin + ic.col + kx0 * stride;
    const double *mp_ = tm + ic.cls + kx0 * cstride, *rp_ = tr + ic.cls + kr0 * cstride;
    auto issue_next = [&]() {
        if (ir < rounds) {
            double *cdst = cring + islot * G * NT + tid;
            if (ig < ngh) {
                T *xdst = xring + islot * G * NT + tid;
                const bool z = zcta && ir == 0 && lt == 0;
                if (ic.valid) {
#pragma unroll
                    for (int u = 0; u < G; u++) {
                        cp_async_8(cdst + u * NT, mp_);
                        if (z)
                            cp_async_8(zring + (islot * 2 + half) * G + u,
                                       mode0 + (half ? nz - 1 - ig * G - u : ig * G + u));
                        else if (sizeof(T) == 8)
                            cp_async_8(xdst + u * NT, xp_);
                        else
                            cp_async_4(xdst + u * NT, xp_);
                        mp_ += fm;
                        xp_ += fx;
                    }
                }
            } else if (ic.valid) {
#pragma unroll
                for (int u = 0; u < G; u++) {
                    cp_async_8(cdst + u * NT, rp_);
                    rp_ += br;
                }
            }
            if (++ig == per_round) {
                ig = 0;
                if (++ir < rounds) {
                    ic = column(ir);
                    xp_ = xin + ic.col + kx0 * stride;
                    mp_ = tm + ic.cls + kx0 * cstride;
                    rp_ = tr + ic.cls + kr0 * cstride;
                }
            }
        }
        cp_async_commit(); // one group per step, empty or not
        islot = (islot + 1 == NS) ? 0 : islot + 1;
    };

    for (int q = 0; q < NS - 1; q++) issue_next();
    int slot = 0;
    for (int r = 0; r < rounds; r++) {
        const TtmColumn cc = column(r);
        const bool zr = zcta && r == 0 && lt == 0;
        // the junction's 2x2 coefficients, needed after the forward sweep
        const double jE = __ldg(tm + cc.cls + (size_t)nz * cstride), jC = __ldg(tm + cc.cls + (size_t)(nz + 1) * cstride);
        const double jD = __ldg(tr + cc.cls + (size_t)nz * cstride), jA = __ldg(tr + cc.cls + (size_t)(nz + 1) * cstride);
        // forward: s_k = r_k - m_k s_{k -+ 1} from this half's wall
        double s = 0.0;
        for (int g = 0; g < ngh; g++) {
            cp_async_wait<NS - 2>(); // this step's group has landed
            const double *cs = cring + slot * G * NT + tid;
            const T *xs = xring + slot * G * NT + tid;
            double xv[G], mv[G];
#pragma unroll
            for (int u = 0; u < G; u++) {
                xv[u] = (double)xs[u * NT];
                mv[u] = cs[u * NT];
            }
            if (zr) {
#pragma unroll
                for (int u = 0; u < G; u++) xv[u] = zring[(slot * 2 + half) * G + u];
            }
            issue_next(); // refills the slot consumed one step ago
            double sv[G];
#pragma unroll
            for (int u = 0; u < G; u++) sv[u] = s = xv[u] - mv[u] * s;
            // cells of the 8-row block in ascending row order: the upper
            // half walks its rows downwards (two branches, so that every
            // index is a constant and the block stays in registers)
            uint32_t v[2 * G];
            if (half) {
#pragma unroll
                for (int u = 0; u < G; u++) {
                    v[2 * (G - 1 - u)] = (uint32_t)__double2loint(sv[u]);
                    v[2 * (G - 1 - u) + 1] = (uint32_t)__double2hiint(sv[u]);
                }
            } else {
#pragma unroll
                for (int u = 0; u < G; u++) {
                    v[2 * u] = (uint32_t)__double2loint(sv[u]);
                    v[2 * u + 1] = (uint32_t)__double2hiint(sv[u]);
                }
            }
            __syncwarp();
            tmem_st16(tbase + 2 * (half ? p - G - g * G : g * G), v);
            slot = (slot + 1 == NS) ? 0 : slot + 1;
        }
        tmem_wait_st();
        // rows p-1 and p from the 2x2 system that joins the halves
        double *jr = jv + (r & 1) * 2 * NC;
        jr[half * NC + lt] = s;
        __syncthreads();
        const double xs_ = jr[lt], ys_ = jr[NC + lt];
        const double xj = half ? ys_ * jD - xs_ * jA : xs_ * jE - ys_ * jC;
        // backward from the middle: x_k = (s_k - c_k x_{k+1}) / d_k below,
        // x_k = (s_k - a_k x_{k-1}) / e_k above
        double w = 0.0;
        T *dst = xout + cc.col + kr0 * stride;
        for (int h = 0; h < ngh; h++) {
            uint32_t v[2 * G];
            __syncwarp();
            tmem_ld16_start(tbase + 2 * (half ? h * G : p - G - h * G), v);
            cp_async_wait<NS - 2>();
            const double *cs = cring + slot * G * NT + tid;
            double rv[G], cf[G];
#pragma unroll
            for (int u = 0; u < G; u++) {
                rv[u] = cs[u * NT];
                cf[u] = half ? ash[p + h * G + u] : csh[p - 1 - h * G - u];
            }
            issue_next();
            tmem_wait_ld(v);
            double sv[G];
            if (half) {
#pragma unroll
                for (int u = 0; u < G; u++) sv[u] = __hiloint2double((int)v[2 * u + 1], (int)v[2 * u]);
            } else {
#pragma unroll
                for (int u = 0; u < G; u++)
                    sv[u] = __hiloint2double((int)v[2 * (G - 1 - u) + 1], (int)v[2 * (G - 1 - u)]);
            }
#pragma unroll
            for (int u = 0; u < G; u++) {
                w = (u == 0 && h == 0) ? xj : (sv[u] - cf[u] * w) * rv[u];
                if (cc.valid) *dst = (T)w;
                dst -= fx;
            }
            slot = (slot + 1 == NS) ? 0 : slot + 1;
        }
    }
    cp_async_wait<0>();
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after_sync();
        tmem_free(*tslot, tcols);
    }
}

// The same sweep at two CTAs per SM (k_thomas_th2; nx % 128 == 0 and a
// right-hand side on a 16-byte boundary), row k's swept value at cell k of
// the column's lane.  The recurrences run in FP64 in registers; the copy of
// each swept value kept for the backward pass is rounded to FP32, one cell
// per row, so a column takes nz cells of a lane and two CTAs share an SM's
// 512 tensor-memory
// columns: twice the chains in flight for the per-row instruction latency
// that bounds the sweep.  The backward recurrence x_k = (s_k - c x_{k-+1})/d_k
// is contractive, so the rounding of s_k enters x_k once, at the relative
// size of the FP32 result's own rounding.
//
// The CTA's 128 columns of a round are one run of a plane row (nx % 128 ==
// 0) and their eigenvalue classes one window of at most 128 consecutive
// classes, so the ring is filled cooperatively with 16-byte copies: a row of
// the right-hand side is 32 copies, a row of a table 65, for the whole CTA
// (per-thread 4- and 8-byte copies, one per row and column, saturated the
// memory-instruction queues at two CTAs per SM).  A barrier per 8-row group
// publishes them.  A round takes 1.66-1.69 times as long as a round of
// k_thomas_th (the barriers, and two CTAs' chains sharing the schedulers),
// so the launcher takes this kernel only where it needs that many times
// fewer rounds (0.162 against 0.176 ms at 512x384x256, 11 rounds against 6).
constexpr int TTH2_CW = 130;       // class window of a round: 128 classes, from an even start
constexpr int TTH2_CH = TTH2_CW / 2; // 16-byte copies per table row

__host__ __device__ constexpr size_t tth2_slot_bytes()
{
    // right-hand side [2 halves][G][128] (float), table rows [2][G][CW] (double)
    return (size_t)2 * TTW_G * TTM_THREADS * 4 + (size_t)2 * TTW_G * TTH2_CW * 8;
}

__host__ __device__ constexpr size_t tth2_smem_bytes()
{
    // ring of NS slots, (0,0)-mode ring [NS][2][G], c_k and a_k [256],
    // junction values [2][2][128], TMEM address slot; at least 78 KB so that
    // at most two CTAs (two times nz <= 256 tensor-memory columns) share an SM
    const size_t b = (size_t)TTH_NS * tth2_slot_bytes() + TTH_NS * 2 * TTW_G * 8 + 2 * TTM_TM_ROWS * 8 +
                     4 * TTM_THREADS * 8 + 16;
    return b < 78 * 1024 ? 78 * 1024 : b;
}

__global__ void __launch_bounds__(2 * TTM_THREADS, 2)
    k_thomas_th2(const float *xin, float *xout, const double *tm, const double *tr, const double *ak, const double *ck,
                int nx, int ny, int nz, int ncx, int ncy, long long tcs, const double *mode0, int rounds,
                uint32_t tcols)
{
    constexpr int G = TTW_G, NS = TTH_NS, NC = TTM_THREADS, NT = 2 * NC, CW = TTH2_CW, CH = TTH2_CH;
    constexpr int SLOT = (int)tth2_slot_bytes();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char *ring = smem_raw;                                            // [NS] slots
    double *zring = reinterpret_cast<double *>(smem_raw + (size_t)NS * SLOT); // [NS][2][G] (0,0) mode
    double *csh = zring + NS * 2 * G;                                         // c_k
    double *ash = csh + TTM_TM_ROWS;                                          // a_k
    double *jv = ash + TTM_TM_ROWS;                                           // [2 parities][2 halves][NC]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(jv + 4 * NC);
    const int tid = threadIdx.x, warp = tid >> 5, half = tid >= NC ? 1 : 0, lt = tid - half * NC;
    const int p = nz / 2, ngh = p / G, per_round = 2 * ngh;
    const long long stride = (long long)nx * ny;
    const int ncol = nx * ny;
    TridDev td{nx, ny, nz, ncx, ncy, nullptr, nullptr, nullptr};
    const long long fx = half ? -stride : stride;

    for (int k = tid; k < nz; k += NT) {
        csh[k] = __ldg(ck + k);
        ash[k] = __ldg(ak + k);
    }
    if (warp == 0) tmem_alloc(tslot, tcols);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tbase = *tslot + ((uint32_t)((warp & 3) * 32) << 16);

    // the CTA's run of round r: its first column (plane offset; -1 past the
    // last column) and the even start of its class window
    struct Run {
        long long col0, cbase;
    };
    auto run = [&](int r) {
        Run u{-1, 0};
        const int q0 = (r * (int)gridDim.x + (int)blockIdx.x) * NC;
        if (q0 < ncol) {
            const int b = q0 / nx, px0 = q0 - b * nx, py = trid_pair_row(b, ny);
            const int ixmin = min(px0, nx - px0 - (NC - 1)), jy = min(py, ny - py);
            u.col0 = (long long)px0 + (long long)nx * py;
            u.cbase = ((long long)ixmin + (long long)ncx * jy) & ~1ll;
        }
        return u;
    };
    auto column = [&](int r) {
        TtmColumn c{false, 0, 0};
        const int q = (r * (int)gridDim.x + (int)blockIdx.x) * NC + lt;
        if (q < ncol) {
            const int b = q / nx, px = q - b * nx, py = trid_pair_row(b, ny);
            c = TtmColumn{true, (size_t)px + (size_t)nx * py, trid_class(px, py, td)};
        }
        return c;
    };
    const bool zcta = (mode0 != nullptr) && blockIdx.x == 0;

    // copy stream: step ig < ngh of a round brings the right-hand side and
    // tm rows of forward group ig of both halves (lower: rows ig G + u,
    // upper: nz-1 - ig G - u), step ngh + h the tr rows of backward group h
    // (lower: p-1 - h G - u, upper: p + h G + u)
    int ir = 0, ig = 0, islot = 0;
    Run irun = run(0);
    auto issue_next = [&]() {
        if (ir < rounds) {
            unsigned char *sl = ring + (size_t)islot * SLOT;
            float *xr = reinterpret_cast<float *>(sl);
            double *tb = reinterpret_cast<double *>(sl + (size_t)2 * G * NC * 4);
            if (irun.col0 >= 0) {
                const bool fwd = ig < ngh;
                const int gg = fwd ? ig : ig - ngh;
                auto row = [&](int h, int u) {
                    return fwd ? (h ? nz - 1 - gg * G - u : gg * G + u) : (h ? p + gg * G + u : p - 1 - gg * G - u);
                };
                if (fwd) {
#pragma unroll
                    for (int e = tid; e < 2 * G * (NC / 4); e += NT) {
                        const int h = e / (G * (NC / 4)), u = (e / (NC / 4)) % G, c = e % (NC / 4);
                        cp_async_16(xr + (h * G + u) * NC + 4 * c, xin + irun.col0 + row(h, u) * stride + 4 * c);
                    }
                    if (zcta && ir == 0 && lt == 0) {
#pragma unroll
                        for (int u = 0; u < G; u++)
                            cp_async_8(zring + (islot * 2 + half) * G + u, mode0 + row(half, u));
                    }
                }
                const double *src = fwd ? tm : tr;
#pragma unroll
                for (int e = tid; e < 2 * G * CH; e += NT) {
                    const int h = e / (G * CH), u = (e / CH) % G, c = e % CH;
                    cp_async_16(tb + (h * G + u) * CW + 2 * c, src + irun.cbase + row(h, u) * tcs + 2 * c);
                }
            }
            if (++ig == per_round) {
                ig = 0;
                if (++ir < rounds) irun = run(ir);
            }
        }
        cp_async_commit(); // one group per step, empty or not
        islot = (islot + 1 == NS) ? 0 : islot + 1;
    };

    for (int q = 0; q < NS - 1; q++) issue_next();
    int slot = 0;
    for (int r = 0; r < rounds; r++) {
        const TtmColumn cc = column(r);
        const int coff = (int)((long long)cc.cls - run(r).cbase); // this column's place in the class window
        const bool zr = zcta && r == 0 && lt == 0;
        // the junction's 2x2 coefficients, needed after the forward sweep
        const double jE = __ldg(tm + cc.cls + nz * tcs), jC = __ldg(tm + cc.cls + (nz + 1) * tcs);
        const double jD = __ldg(tr + cc.cls + nz * tcs), jA = __ldg(tr + cc.cls + (nz + 1) * tcs);
        // forward: s_k = r_k - m_k s_{k -+ 1} from this half's wall
        double s = 0.0;
        for (int g = 0; g < ngh; g++) {
            cp_async_wait<NS - 2>(); // this step's group has landed (every thread's share)
            __syncthreads();
            const unsigned char *sl = ring + (size_t)slot * SLOT;
            const float *xs = reinterpret_cast<const float *>(sl) + half * G * NC + lt;
            const double *cs = reinterpret_cast<const double *>(sl + (size_t)2 * G * NC * 4) + half * G * CW + coff;
            double xv[G], mv[G];
#pragma unroll
            for (int u = 0; u < G; u++) {
                xv[u] = (double)xs[u * NC];
                mv[u] = cs[u * CW];
            }
            if (zr) {
#pragma unroll
                for (int u = 0; u < G; u++) xv[u] = zring[(slot * 2 + half) * G + u];
            }
            issue_next(); // refills the slot consumed one step ago
            double sv[G];
#pragma unroll
            for (int u = 0; u < G; u++) sv[u] = s = xv[u] - mv[u] * s;
            // cells of the 8-row block in ascending row order: the upper
            // half walks its rows downwards (two branches, so that every
            // index is a constant and the block stays in registers)
            uint32_t v[G];
            if (half) {
#pragma unroll
                for (int u = 0; u < G; u++) v[G - 1 - u] = __float_as_uint(__double2float_rn(sv[u]));
            } else {
#pragma unroll
                for (int u = 0; u < G; u++) v[u] = __float_as_uint(__double2float_rn(sv[u]));
            }
            __syncwarp();
            tmem_st8(tbase + (half ? nz - G - g * G : g * G), v);
            slot = (slot + 1 == NS) ? 0 : slot + 1;
        }
        tmem_wait_st();
        // rows p-1 and p from the 2x2 system that joins the halves
        double *jr = jv + (r & 1) * 2 * NC;
        jr[half * NC + lt] = s;
        __syncthreads();
        const double xs_ = jr[lt], ys_ = jr[NC + lt];
        const double xj = half ? ys_ * jD - xs_ * jA : xs_ * jE - ys_ * jC;
        // backward from the middle: x_k = (s_k - c_k x_{k+1}) / d_k below,
        // x_k = (s_k - a_k x_{k-1}) / e_k above
        double w = 0.0;
        float *dst = xout + cc.col + (half ? p : p - 1) * stride;
        for (int h = 0; h < ngh; h++) {
            uint32_t v[G];
            __syncwarp();
            tmem_ld8_start(tbase + (half ? p + h * G : p - G - h * G), v);
            cp_async_wait<NS - 2>();
            __syncthreads();
            const double *cs =
                reinterpret_cast<const double *>(ring + (size_t)slot * SLOT + (size_t)2 * G * NC * 4) +
                half * G * CW + coff;
            double rv[G], cf[G];
#pragma unroll
            for (int u = 0; u < G; u++) {
                rv[u] = cs[u * CW];
                cf[u] = half ? ash[p + h * G + u] : csh[p - 1 - h * G - u];
            }
            issue_next();
            tmem_wait_ld(v);
            double sv[G];
            if (half) {
#pragma unroll
                for (int u = 0; u < G; u++) sv[u] = (double)__uint_as_float(v[u]);
            } else {
#pragma unroll
                for (int u = 0; u < G; u++) sv[u] = (double)__uint_as_float(v[G - 1 - u]);
            }
#pragma unroll
            for (int u = 0; u < G; u++) {
                w = (u == 0 && h == 0) ? xj : (sv[u] - cf[u] * w) * rv[u];
                if (cc.valid) *dst = (float)w;
                dst -= fx;
            }
            slot = (slot + 1 == NS) ? 0 : slot + 1;
        }
    }
    cp_async_wait<0>();
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after_sync();
        tmem_free(*tslot, tcols);
    }
}

constexpr int PDD_MAX_PARTS = 64;

struct PddDev {
    int nparts;
    int kst[PDD_MAX_PARTS], ksz[PDD_MAX_PARTS];
    const double *v, *w, *tmpv;
};

// PDD (psolve_trid :361-466) for all nparts z-partitions of one column:
// local Thomas per partition, then for each internal interface the truncated
// 2x2 reduced system (:423-438), y3 of partition m becoming y1 of m+1
// (:444-446), and the correction x -= v*y1 + w*y2 (:452-464).  The bottom
// partition keeps y1 = 0 and the top one y2 = 0, as in the reference where
// those arrays are zeroed at init and never received.
//
// Mixed path (mode0 given): the (0,0) column takes its FP64 right-hand side
// from the plane sums, as in k_thomas.  Its matrix has zero row sums, so a
// partition's spike towards a wall-bounded neighbour is the constant -1; with
// two partitions both spikes of the one interface are, its reduced system is
// singular (det = wt tv - 1 is round-off) and the reference's division leaves
// x with an arbitrary constant far above FP32's resolution of x.  There the
// system's free parameter is fixed by y3 = 0 (x moves by a constant only)
// and y2 comes from its second row, y2 + tv y3 = tvar.  With three or more
// partitions every truncated interface system is regular.
__device__ __forceinline__ bool pdd_gauge00(const double *mode0, size_t col, int nparts)
{
    return mode0 != nullptr && col == 0 && nparts == 2;
}

template <typename T>
__global__ void __launch_bounds__(128) k_pdd(double *xs, T *xout, TridDev t, PddDev p, const double *mode0)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    if (px >= t.nx) return;
    const size_t col = (size_t)px + (size_t)t.nx * py, stride = (size_t)t.nx * t.ny;
    const size_t cls = trid_class(px, py, t), cstride = (size_t)t.ncx * t.ncy;
    if (mode0 != nullptr && col == 0)
        for (int k = 0; k < t.nz; k++) xs[(size_t)k * stride] = mode0[k];
    // local solves in FP64, in place in xs
    for (int m = 0; m < p.nparts; m++)
        thomas_column<double>(xs, xs, xs, col, cls, stride, cstride, p.kst[m], p.ksz[m], t);
    double y1 = 0.0;
    for (int m = 0; m < p.nparts; m++) {
        double y2 = 0.0, y3 = 0.0;
        if (m + 1 < p.nparts) {
            const int kt = p.kst[m] + p.ksz[m] - 1;
            const double wt = __ldg(p.w + cls + (size_t)kt * cstride);
            const double tv = __ldg(p.tmpv + cls + (size_t)m * cstride);
            const double xt = xs[col + (size_t)kt * stride];
            const double tvar = xs[col + (size_t)p.kst[m + 1] * stride];
            const double det = wt * tv - 1.0;
            y2 = (xt * tv - tvar) / det;
            y3 = (tvar * wt - xt) / det;
            if (pdd_gauge00(mode0, col, p.nparts)) {
                y2 = tvar;
                y3 = 0.0;
            }
        }
        for (int k = p.kst[m]; k < p.kst[m] + p.ksz[m]; k++) {
            const size_t g = col + (size_t)k * stride;
            const size_t gc = cls + (size_t)k * cstride;
            xout[g] = (T)(xs[g] - __ldg(p.v + gc) * y1 - __ldg(p.w + gc) * y2);
        }
        y1 = y3;
    }
}

// PDD with one thread per (column, partition), P <= 32: a 32 x P block
// holds 32 adjacent columns (coalesced rows) and all their partitions.  Each
// thread solves its partition's local system, reading the right-hand side
// (FP32 or FP64) straight from the transform array; after the block's
// barrier it forms the interface systems on both sides of its partition
// from the neighbours' rows of the FP64 sweep buffer (y1 from the interface
// below, y2 from the one above) and corrects its own rows.  The values are
// k_pdd's, expression for expression; P threads per column instead of one
// run the local sweeps side by side, and no widening or copy of the
// right-hand side precedes them.
template <typename T>
__global__ void __launch_bounds__(1024) k_pdd_par(const T *xin, double *xs, T *xout, TridDev t, PddDev p,
                                                  const double *mode0)
{
    const int m = threadIdx.y;
    const int q = blockIdx.x * 32 + threadIdx.x, ncol = t.nx * t.ny;
    const bool valid = q < ncol;
    const int qq = valid ? q : 0, px = qq % t.nx, py = qq / t.nx;
    const size_t col = (size_t)qq, stride = (size_t)t.nx * t.ny;
    const size_t cls = trid_class(px, py, t), cstride = (size_t)t.ncx * t.ncy;
    const int k0 = p.kst[m], ke = p.ksz[m];
    if (valid) {
        if (mode0 != nullptr && col == 0) { // mixed path: the (0,0) column from the FP64 plane sums
            for (int k = k0; k < k0 + ke; k++) xs[(size_t)k * stride] = mode0[k];
            thomas_column<double>(xs, xs, xs, col, cls, stride, cstride, k0, ke, t);
        } else {
            thomas_column<T, double>(xin, xs, xs, col, cls, stride, cstride, k0, ke, t);
        }
    }
    __syncthreads();
    if (!valid) return;
    // the truncated 2x2 system at the top of partition mm (:423-438)
    auto iface = [&](int mm, double &y2, double &y3) {
        const int kt = p.kst[mm] + p.ksz[mm] - 1;
        const double wt = __ldg(p.w + cls + (size_t)kt * cstride);
        const double tv = __ldg(p.tmpv + cls + (size_t)mm * cstride);
        const double xt = xs[col + (size_t)kt * stride];
        const double tvar = xs[col + (size_t)p.kst[mm + 1] * stride];
        const double det = wt * tv - 1.0;
        y2 = (xt * tv - tvar) / det;
        y3 = (tvar * wt - xt) / det;
        if (pdd_gauge00(mode0, col, p.nparts)) {
            y2 = tvar;
            y3 = 0.0;
        }
    };
    double y1 = 0.0, y2 = 0.0, unused;
    if (m > 0) iface(m - 1, unused, y1); // y3 of the interface below is this partition's y1 (:444-446)
    if (m + 1 < p.nparts) iface(m, y2, unused);
    for (int k = k0; k < k0 + ke; k++) {
        const size_t g = col + (size_t)k * stride;
        const size_t gc = cls + (size_t)k * cstride;
        xout[g] = (T)(xs[g] - __ldg(p.v + gc) * y1 - __ldg(p.w + gc) * y2);
    }
}

// PDD with one thread per (column, partition) and each partition's swept
// values in tensor memory (P <= 8, every partition a multiple of 8 rows):
// the local sweep writes its forward-swept rows to the thread's lane, the
// back substitution reads them and writes the local solution over them, and
// the correction reads that; HBM sees the right-hand side, the solution and
// the class tables only.  Warp m holds partition m (lane quarter m % 4;
// warps m and m+4 use the next 2 kmax cells).  The partitions' first and
// last local values meet in shared memory for the interface systems.  The
// values are k_pdd's, expression for expression.
constexpr int PTM_G = 8;

__host__ __device__ constexpr int pdd_tm_static_smem() { return 2 * 8 * 32 * 8 + 16; }

template <typename T>
__global__ void __launch_bounds__(256) k_pdd_tm(const T *xin, T *xout, TridDev t, PddDev p, const double *mode0,
                                                int kmax, uint32_t tcols)
{
    constexpr int G = PTM_G;
    __shared__ double edge[2][8][32]; // [first / last local value][partition][column]
    __shared__ uint32_t tslot;
    const int cx = threadIdx.x, m = threadIdx.y;
    const int q = blockIdx.x * 32 + cx, ncol = t.nx * t.ny;
    const bool valid = q < ncol;
    const int qq = valid ? q : 0, px = qq % t.nx, py = qq / t.nx;
    const size_t col = (size_t)qq, stride = (size_t)t.nx * t.ny;
    const size_t cls = trid_class(px, py, t), cstride = (size_t)t.ncx * t.ncy;
    const int k0 = p.kst[m], ke = p.ksz[m], ng = ke / G;
    const bool z = mode0 != nullptr && valid && col == 0; // mixed path: the (0,0) column from the plane sums

    if (m == 0) tmem_alloc(&tslot, tcols);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tb = tslot + ((uint32_t)((m & 3) * 32) << 16) + (uint32_t)((m >> 2) * 2 * kmax);

    // forward elimination of the partition (ssolve_trid :319-330; the
    // multiplier is 0 at its first row)
    double xp = 0.0;
    for (int g = 0; g < ng; g++) {
        double xv[G], mv[G];
#pragma unroll
        for (int u = 0; u < G; u++) {
            const int k = k0 + g * G + u;
            xv[u] = z ? mode0[k] : (double)xin[col + (size_t)k * stride];
            mv[u] = __ldg(t.mult + cls + (size_t)k * cstride);
        }
        uint32_t v[2 * G];
#pragma unroll
        for (int u = 0; u < G; u++) {
            xp = xv[u] - mv[u] * xp;
            v[2 * u] = (uint32_t)__double2loint(xp);
            v[2 * u + 1] = (uint32_t)__double2hiint(xp);
        }
        __syncwarp();
        tmem_st16(tb + 2 * g * G, v);
    }
    tmem_wait_st();
    // back substitution (:332-356): x = (x - c x_{k+1}) / b, with x_{k+1} = 0
    // above the partition's last row; the local solution replaces the swept rows
    double w = 0.0, first = 0.0, last = 0.0;
    for (int g = ng - 1; g >= 0; g--) {
        uint32_t v[2 * G];
        __syncwarp();
        tmem_ld16_start(tb + 2 * g * G, v);
        double rv[G], cv[G];
#pragma unroll
        for (int u = 0; u < G; u++) {
            const int k = k0 + g * G + u;
            rv[u] = __ldg(t.rb + cls + (size_t)k * cstride);
            cv[u] = __ldg(t.c + k);
        }
        tmem_wait_ld(v);
#pragma unroll
        for (int u = G - 1; u >= 0; u--) {
            const double s = __hiloint2double((int)v[2 * u + 1], (int)v[2 * u]);
            w = (s - cv[u] * w) * rv[u];
            if (g == ng - 1 && u == G - 1) last = w;
            v[2 * u] = (uint32_t)__double2loint(w);
            v[2 * u + 1] = (uint32_t)__double2hiint(w);
        }
        __syncwarp();
        tmem_st16(tb + 2 * g * G, v);
    }
    first = w;
    tmem_wait_st();
    edge[0][m][cx] = first;
    edge[1][m][cx] = last;
    __syncthreads();
    // the truncated 2x2 systems at the partition's two interfaces (:423-438)
    auto iface = [&](int mm, double &y2, double &y3) {
        const int kt = p.kst[mm] + p.ksz[mm] - 1;
        const double wt = __ldg(p.w + cls + (size_t)kt * cstride);
        const double tv = __ldg(p.tmpv + cls + (size_t)mm * cstride);
        const double xt = edge[1][mm][cx], tvar = edge[0][mm + 1][cx];
        const double det = wt * tv - 1.0;
        y2 = (xt * tv - tvar) / det;
        y3 = (tvar * wt - xt) / det;
        if (pdd_gauge00(mode0, col, p.nparts)) {
            y2 = tvar;
            y3 = 0.0;
        }
    };
    double y1 = 0.0, y2 = 0.0, unused;
    if (m > 0) iface(m - 1, unused, y1);
    if (m + 1 < p.nparts) iface(m, y2, unused);
    // correction x = x_local - v y1 - w y2 (:452-464)
    for (int g = 0; g < ng; g++) {
        uint32_t v[2 * G];
        __syncwarp();
        tmem_ld16_start(tb + 2 * g * G, v);
        double vv[G], wv[G];
#pragma unroll
        for (int u = 0; u < G; u++) {
            const size_t gc = cls + (size_t)(k0 + g * G + u) * cstride;
            vv[u] = __ldg(p.v + gc);
            wv[u] = __ldg(p.w + gc);
        }
        tmem_wait_ld(v);
        if (valid) {
#pragma unroll
            for (int u = 0; u < G; u++) {
                const double x = __hiloint2double((int)v[2 * u + 1], (int)v[2 * u]);
                xout[col + (size_t)(k0 + g * G + u) * stride] = (T)(x - vv[u] * y1 - wv[u] * y2);
            }
        }
    }
    tmem_fence_before_sync();
    __syncthreads();
    if (m == 0) {
        tmem_fence_after_sync();
        tmem_free(tslot, tcols);
    }
}

// PDD of one z slab per GPU (psolve_trid, mod_poisson_solver.c:361-466, for
// the rank that holds the partition): the local sweep, the interface solve
// with the upper neighbour, and the correction, as three kernels around the
// two plane exchanges.  Per column the arithmetic is k_pdd's for that
// partition, operation for operation, the mixed path's (0,0) column included
// (mode0: this slab's plane sums; gauge on the lower rank of two).
__global__ void __launch_bounds__(128) k_pdd_sweep(double *xs, TridDev t, const double *mode0)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    if (px >= t.nx) return;
    const size_t col = (size_t)px + (size_t)t.nx * py, stride = (size_t)t.nx * t.ny;
    const size_t cls = trid_class(px, py, t), cstride = (size_t)t.ncx * t.ncy;
    if (mode0 != nullptr && col == 0)
        for (int k = 0; k < t.nz; k++) xs[(size_t)k * stride] = mode0[k];
    thomas_column<double>(xs, xs, xs, col, cls, stride, cstride, 0, t.nz, t);
}

// the reduced 2x2 system at the top interface (:423-438): tvar is the upper
// neighbour's first swept row, tmpv its v at that row
__global__ void __launch_bounds__(256) k_pdd_iface(const double *xs, const double *tvar, const double *w,
                                                   const double *tmpv, double *y2, double *y3, TridDev t,
                                                   int gauge00)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    if (px >= t.nx) return;
    const size_t col = (size_t)px + (size_t)t.nx * py, stride = (size_t)t.nx * t.ny;
    const size_t cls = trid_class(px, py, t), cstride = (size_t)t.ncx * t.ncy;
    const int kt = t.nz - 1;
    const double wt = __ldg(w + cls + (size_t)kt * cstride);
    const double tv = __ldg(tmpv + cls);
    const double xt = xs[col + (size_t)kt * stride];
    const double tva = tvar[col];
    const double det = wt * tv - 1.0;
    y2[col] = (xt * tv - tva) / det;
    y3[col] = (tva * wt - xt) / det;
    if (gauge00 && col == 0) {
        y2[col] = tva;
        y3[col] = 0.0;
    }
}

// x = xs - v y1 - w y2 (:454-465); y1 = 0 without a lower neighbour, y2 = 0
// without an upper one (the reference's zero-initialised arrays)
template <typename T>
__global__ void __launch_bounds__(128) k_pdd_fix(const double *xs, T *xout, const double *v, const double *w,
                                                 const double *y1, const double *y2, int has_down, int has_up,
                                                 TridDev t)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    if (px >= t.nx) return;
    const size_t col = (size_t)px + (size_t)t.nx * py, stride = (size_t)t.nx * t.ny;
    const size_t cls = trid_class(px, py, t), cstride = (size_t)t.ncx * t.ncy;
    const double a1 = has_down ? y1[col] : 0.0, a2 = has_up ? y2[col] : 0.0;
    for (int k = 0; k < t.nz; k++) {
        const size_t g = col + (size_t)k * stride;
        const size_t gc = cls + (size_t)k * cstride;
        xout[g] = (T)(xs[g] - __ldg(v + gc) * a1 - __ldg(w + gc) * a2);
    }
}

// mixed path: widen the FP32 right-hand side into the FP64 sweep buffer
__global__ void k_widen(const float *__restrict__ in, double *__restrict__ out, size_t n)
{
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        out[q] = (double)in[q];
}

int launch_widen(const float *in, double *out, size_t n, cudaStream_t st)
{
    k_widen<<<1184, 256, 0, st>>>(in, out, n);
    PL_CHECK_LAUNCH();
    return 0;
}

// ------------------------------------------------------------------------
// Host plan
// ------------------------------------------------------------------------

// radix plan: 8s first, then one 4 or 2, then 3s (a leftover 2 merged with a
// 3 into a 6): few stages, so few shared-memory round trips
static int factor_radices(int n, int *radix, int *nstages)
{
    int s = 0, m = n;
    while (m % 8 == 0 && s < FFT_MAX_STAGES) {
        radix[s++] = 8;
        m /= 8;
    }
    int two = 0;
    if (m % 4 == 0) {
        radix[s++] = 4;
        m /= 4;
    } else if (m % 2 == 0) {
        two = 1;
        m /= 2;
    }
    int threes = 0;
    while (m % 3 == 0) {
        threes++;
        m /= 3;
    }
    if (m != 1) return -1;
    if (two && threes) {
        radix[s++] = 6;
        threes--;
    } else if (two) {
        radix[s++] = 2;
    }
    while (threes-- > 0 && s < FFT_MAX_STAGES) radix[s++] = 3;
    *nstages = s;
    return 0;
}

template <typename V> static int upload_twiddles(int n, V **dptr)
{
    std::vector<V> h(n);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int t = 0; t < n; t++) {
        long double a = -two_pi * (long double)t / (long double)n;
        h[t].x = (decltype(h[t].x))cosl(a);
        h[t].y = (decltype(h[t].y))sinl(a);
    }
    PL_CUDA_TRY(cudaMalloc(dptr, sizeof(V) * n));
    PL_CUDA_TRY(cudaMemcpy(*dptr, h.data(), sizeof(V) * n, cudaMemcpyHostToDevice));
    return 0;
}

template <typename V> static void set_plan(FftPlanDev<V> &p, int n, const int *radix, int ns, const V *tw)
{
    p.n = n;
    p.nstages = ns;
    for (int s = 0; s < ns; s++) p.radix[s] = radix[s];
    p.tw = tw;
}

int ppe_create(Ppe *s, int nx, int ny, int nz, double dx, double dy, const double *dzf_global, int nparts,
               int prec)
{
    *s = Ppe();
    if (nx < 2 || ny < 2 || nz < 1 || (nx & 1) || (ny & 1)) {
        set_error("ppe_create: nx and ny must be even and >= 2, nz >= 1 (the reference requires even sizes, "
                  "mod_parameters.f90:264-267)");
        return -1;
    }
    if (nparts < 0 || nparts > PDD_MAX_PARTS || nparts > nz) {
        set_error("ppe_create: PDD partition count must be in [0, min(nz, 64)]");
        return -1;
    }
    s->nx = nx;
    s->ny = ny;
    s->nz = nz;
    s->nparts = nparts;
    s->prec = prec;
    s->ncx = nx / 2 + 1;
    s->ncy = ny / 2 + 1;
    s->norm = 1.0 / (1.0 * nx * 1.0 * ny); // mod_fft_fftw.inc:89, PP/PP
    const int P = nparts >= 1 ? nparts : 1;

    int rx[FFT_MAX_STAGES], ry[FFT_MAX_STAGES], nsx = 0, nsy = 0;
    if (factor_radices(nx, rx, &nsx) || factor_radices(ny, ry, &nsy)) {
        set_error("ppe_create: nx and ny must be of the form 2^a 3^b");
        return -1;
    }
    if (upload_twiddles<double2>(nx, &s->d_twx64) || upload_twiddles<double2>(ny, &s->d_twy64) ||
        upload_twiddles<float2>(nx, &s->d_twx32) || upload_twiddles<float2>(ny, &s->d_twy32))
        return -1;
    set_plan(s->px64, nx, rx, nsx, s->d_twx64);
    set_plan(s->py64, ny, ry, nsy, s->d_twy64);
    set_plan(s->px32, nx, rx, nsx, s->d_twx32);
    set_plan(s->py32, ny, ry, nsy, s->d_twy32);

    // tridiagonal coefficients, pivots and PDD spikes per eigenvalue class
    TridTables tt;
    const bool twisted = prec == PREC_MIXED && nparts == 0 && nz % (2 * TTW_G) == 0 && nz >= 2 * TTW_G &&
                         nz <= TTM_TM_ROWS;
    trid_build(tt, nx, ny, nz, dx, dy, dzf_global, nparts, twisted);
    if (prec == PREC_MIXED && nparts == 0) {
        // The (0,0) class has lambda = 0: its Neumann system is singular and
        // its last pivot is round-off, so the reference's division at row
        // nz-1 gives x a constant of order 1e7 |x| that an FP32 result cannot
        // carry.  The mixed plan takes the gauge x[nz-1] = 0 there instead,
        // as the sweeps' plane-sum branch does; the FP64 plan keeps the
        // reference's pivots.
        tt.rb[(size_t)(nz - 1) * ((size_t)s->ncx * s->ncy)] = 0.0;
    }
    s->kst = tt.kst;
    s->ksz = tt.ksz;
    const size_t ncls = (size_t)s->ncx * s->ncy;
    const std::vector<double> &mult = tt.mult, &rb = tt.rb, &c = tt.c, &v = tt.v, &w = tt.w, &tmpv = tt.tmpv;
    PL_CUDA_TRY(cudaMalloc(&s->d_a, sizeof(double) * nz));
    PL_CUDA_TRY(cudaMalloc(&s->d_bt, sizeof(double) * nz));
    PL_CUDA_TRY(cudaMemcpy(s->d_a, tt.a.data(), sizeof(double) * nz, cudaMemcpyHostToDevice));
    PL_CUDA_TRY(cudaMemcpy(s->d_bt, tt.bt.data(), sizeof(double) * nz, cudaMemcpyHostToDevice));
    PL_CUDA_TRY(cudaMalloc(&s->d_mult, sizeof(double) * ncls * nz));
    PL_CUDA_TRY(cudaMalloc(&s->d_rb, sizeof(double) * ncls * nz));
    PL_CUDA_TRY(cudaMalloc(&s->d_c, sizeof(double) * nz));
    PL_CUDA_TRY(cudaMemcpy(s->d_mult, mult.data(), sizeof(double) * ncls * nz, cudaMemcpyHostToDevice));
    PL_CUDA_TRY(cudaMemcpy(s->d_rb, rb.data(), sizeof(double) * ncls * nz, cudaMemcpyHostToDevice));
    PL_CUDA_TRY(cudaMemcpy(s->d_c, c.data(), sizeof(double) * nz, cudaMemcpyHostToDevice));
    if (nparts >= 1) {
        PL_CUDA_TRY(cudaMalloc(&s->d_v, sizeof(double) * ncls * nz));
        PL_CUDA_TRY(cudaMalloc(&s->d_w, sizeof(double) * ncls * nz));
        PL_CUDA_TRY(cudaMalloc(&s->d_tmpv, sizeof(double) * ncls * P));
        PL_CUDA_TRY(cudaMemcpy(s->d_v, v.data(), sizeof(double) * ncls * nz, cudaMemcpyHostToDevice));
        PL_CUDA_TRY(cudaMemcpy(s->d_w, w.data(), sizeof(double) * ncls * nz, cudaMemcpyHostToDevice));
        PL_CUDA_TRY(cudaMemcpy(s->d_tmpv, tmpv.data(), sizeof(double) * ncls * P, cudaMemcpyHostToDevice));
    }
    if (twisted) {
        // rows of an even number of values: the sweep copies 16-byte pairs
        s->tcs = (ncls + 1) / 2 * 2;
        const size_t tb = sizeof(double) * s->tcs * (nz + 2);
        PL_CUDA_TRY(cudaMalloc(&s->d_tmult, tb));
        PL_CUDA_TRY(cudaMalloc(&s->d_trb, tb));
        PL_CUDA_TRY(cudaMemset(s->d_tmult, 0, tb));
        PL_CUDA_TRY(cudaMemset(s->d_trb, 0, tb));
        PL_CUDA_TRY(cudaMemcpy2D(s->d_tmult, sizeof(double) * s->tcs, tt.tmult.data(), sizeof(double) * ncls,
                                 sizeof(double) * ncls, nz + 2, cudaMemcpyHostToDevice));
        PL_CUDA_TRY(cudaMemcpy2D(s->d_trb, sizeof(double) * s->tcs, tt.trb.data(), sizeof(double) * ncls,
                                 sizeof(double) * ncls, nz + 2, cudaMemcpyHostToDevice));
    }
    if (prec == PREC_MIXED || nparts >= 1) {
        s->scratch_elems = (size_t)nx * ny * nz;
        PL_CUDA_TRY(cudaMalloc(&s->d_scratch, sizeof(double) * s->scratch_elems));
    }
    // kernels with > 48 KB of dynamic shared memory
    PL_CUDA_TRY(cudaFuncSetAttribute(k_yfft<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_yfft<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_yfft<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_yfft<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_xfft<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_xfft<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_xfft<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    PL_CUDA_TRY(cudaFuncSetAttribute(k_xfft<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    return 0;
}

int ppe_create_slab(Ppe *s, int nx, int ny, int nz_global, double dx, double dy, const double *dzf_global,
                    int nranks, int rank, int prec)
{
    if (nranks < 2 || rank < 0 || rank >= nranks) {
        set_error("ppe_create_slab: needs 2 or more slabs and 0 <= rank < nranks");
        return -1;
    }
    // the FFT plans and every table of the global PDD system, then this
    // partition's rows of them
    Ppe g;
    if (ppe_create(&g, nx, ny, nz_global, dx, dy, dzf_global, nranks, prec)) {
        ppe_destroy(&g);
        return -1;
    }
    const int k0 = g.kst[rank], nzl = g.ksz[rank];
    if (nzl < 2) {
        ppe_destroy(&g);
        set_error("ppe_create_slab: every slab needs at least 2 planes");
        return -1;
    }
    *s = g; // plans, twiddles and sizes; the tables are replaced below
    s->nz = nzl;
    s->nparts = 1;
    s->kst.assign(1, 0);
    s->ksz.assign(1, nzl);
    s->slab = 1;
    s->has_down = rank > 0;
    s->has_up = rank < nranks - 1;
    s->d_tmult = s->d_trb = s->d_mult = s->d_rb = s->d_c = s->d_a = s->d_bt = s->d_v = s->d_w = s->d_tmpv =
        s->d_scratch = nullptr;
    const size_t ncls = (size_t)s->ncx * s->ncy, nxy = (size_t)nx * ny;
    auto slice = [&](const double *src, size_t per_plane, int k_from, int nk, double **dst) -> int {
        PL_CUDA_TRY(cudaMalloc(dst, sizeof(double) * per_plane * nk));
        PL_CUDA_TRY(cudaMemcpy(*dst, src + per_plane * k_from, sizeof(double) * per_plane * nk,
                               cudaMemcpyDeviceToDevice));
        return 0;
    };
    int rc = slice(g.d_mult, ncls, k0, nzl, &s->d_mult) || slice(g.d_rb, ncls, k0, nzl, &s->d_rb) ||
             slice(g.d_c, 1, k0, nzl, &s->d_c) || slice(g.d_a, 1, k0, nzl, &s->d_a) ||
             slice(g.d_bt, 1, k0, nzl, &s->d_bt) || slice(g.d_v, ncls, k0, nzl, &s->d_v) ||
             slice(g.d_w, ncls, k0, nzl, &s->d_w) || slice(g.d_tmpv, ncls, rank, 1, &s->d_tmpv);
    // the global plan's own tables and scratch go; its plans and twiddles stay in s
    cudaFree(g.d_mult);
    cudaFree(g.d_rb);
    cudaFree(g.d_c);
    cudaFree(g.d_a);
    cudaFree(g.d_bt);
    cudaFree(g.d_v);
    cudaFree(g.d_w);
    cudaFree(g.d_tmpv);
    cudaFree(g.d_scratch);
    if (rc) return -1;
    s->scratch_elems = nxy * nzl;
    PL_CUDA_TRY(cudaMalloc(&s->d_scratch, sizeof(double) * s->scratch_elems));
    PL_CUDA_TRY(cudaMalloc(&s->d_tvar, sizeof(double) * nxy * 4));
    s->d_y1 = s->d_tvar + nxy;
    s->d_y2 = s->d_y1 + nxy;
    s->d_y3 = s->d_y2 + nxy;
    PL_CUDA_TRY(cudaMemset(s->d_tvar, 0, sizeof(double) * nxy * 4));
    return 0;
}


void ppe_destroy(Ppe *s)
{
    cudaFree(s->d_twx64);
    cudaFree(s->d_twy64);
    cudaFree(s->d_twx32);
    cudaFree(s->d_twy32);
    cudaFree(s->d_mult);
    cudaFree(s->d_rb);
    cudaFree(s->d_tmult);
    cudaFree(s->d_trb);
    cudaFree(s->d_c);
    cudaFree(s->d_a);
    cudaFree(s->d_bt);
    cudaFree(s->d_v);
    cudaFree(s->d_w);
    cudaFree(s->d_tmpv);
    cudaFree(s->d_scratch);
    cudaFree(s->d_mode0);
    cudaFree(s->d_tvar);
    *s = Ppe();
}

// launch geometry ---------------------------------------------------------
static int x_pairs_per_cta(int nx, int ny)
{
    int pb = 1024 / nx;
    if (pb < 1) pb = 1;
    if (pb > ny / 2) pb = ny / 2;
    return pb;
}

static int y_cols_per_cta(int nx, int ny)
{
    int w = 2048 / ny;
    if (w < 1) w = 1;
    if (w > 8) w = 8;
    if (w > nx / 2) w = nx / 2;
    return w;
}

static int sm_count()
{
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 1;
    }
    return n;
}

template <typename K> static int persistent_grid(K kernel, size_t shm, int total, int threads = 256)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, shm) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return std::max(1, std::min(total, per_sm * sm_count()));
}

template <typename T, int N, bool FWD>
static int launch_x_ct(const Ppe *s, const T *in, size_t in_off, size_t in_sj, size_t in_sk, T *out, size_t out_off,
                       size_t out_sj, size_t out_sk, T scale, cudaStream_t st, const PressureUpdate *pu, bool *fused)
{
    using V = typename cplx_of<T>::type;
    constexpr int NB = ct_x_lines<N>();
    const size_t shm = sizeof(V) * (2 * (size_t)fpad_elems<V>(NB * N) + N);
    const V *tw = reinterpret_cast<const V *>(sizeof(T) == 8 ? (const void *)s->d_twx64 : (const void *)s->d_twx32);
    const size_t sk = (size_t)N * s->ny;
    const bool aligned = ((uintptr_t)in % 16 == 0) && ((uintptr_t)out % 16 == 0);
    if (aligned && in_off == 0 && out_off == 0 && in_sj == (size_t)N && out_sj == (size_t)N && in_sk == sk &&
        out_sk == sk) {
        constexpr int NT = pf_x_threads<T>(), NBP = pf_x_lines<T, N>();
        const int total = ((s->ny / 2 + NBP - 1) / NBP) * s->nz;
        if constexpr (sizeof(T) == 4 && !FWD) {
            if (pu != nullptr) {
                const size_t shmp = sizeof(V) * (size_t)pf_x_smem_elems<T, N>() + pf_x_pu_bytes<T, N>();
                auto kern = k_xfft_pf<T, N, false, true>;
                if (shmp > 48 * 1024)
                    PL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmp));
                kern<<<persistent_grid(kern, shmp, total, NT), NT, shmp, st>>>(in, out, tw, s->ny, total, scale, *pu);
                PL_CHECK_LAUNCH();
                *fused = true;
                return 0;
            }
        }
        const size_t shmp = sizeof(V) * (size_t)pf_x_smem_elems<T, N>();
        if (shmp > 48 * 1024)
            PL_CUDA_TRY(
                cudaFuncSetAttribute(k_xfft_pf<T, N, FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmp));
        k_xfft_pf<T, N, FWD><<<persistent_grid(k_xfft_pf<T, N, FWD>, shmp, total, NT), NT, shmp, st>>>(
            in, out, tw, s->ny, total, scale, PressureUpdate{});
        PL_CHECK_LAUNCH();
        *fused = false;
        return 0;
    }
    if (shm > 48 * 1024)
        PL_CUDA_TRY(cudaFuncSetAttribute(k_xfft_ct<T, N, FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    dim3 grid((s->ny / 2 + NB - 1) / NB, s->nz);
    k_xfft_ct<T, N, FWD><<<grid, 256, shm, st>>>(in, in_off, in_sj, in_sk, out, out_off, out_sj, out_sk, tw, s->ny,
                                                 scale);
    PL_CHECK_LAUNCH();
    return 0;
}

template <typename T, int N, bool FWD> static int launch_y_ct(const Ppe *s, T *data, cudaStream_t st)
{
    using V = typename cplx_of<T>::type;
    constexpr int W = pf_y_cols<V, N, FWD>();
    const size_t shm = sizeof(V) * (size_t)pf_y_smem_elems<T, N, FWD>();
    if (shm > 48 * 1024)
        PL_CUDA_TRY(cudaFuncSetAttribute(k_yfft_pf<T, N, FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    const V *tw = reinterpret_cast<const V *>(sizeof(T) == 8 ? (const void *)s->d_twy64 : (const void *)s->d_twy32);
    const int total = ((s->nx / 2 + W - 1) / W) * s->nz;
    k_yfft_pf<T, N, FWD><<<persistent_grid(k_yfft_pf<T, N, FWD>, shm, total, pf_y_threads<T>()), pf_y_threads<T>(), shm,
                           st>>>(data, tw, s->nx, total);
    PL_CHECK_LAUNCH();
    return 0;
}

// line lengths with compile-time kernels; other 2^a 3^b lengths use the
// runtime-length kernels
#define PL_FFT_CT_SIZES(X) X(64) X(128) X(192) X(256) X(384) X(512) X(768) X(1024)

template <typename T> static int launch_pressure_update(const Ppe *s, const T *dp, const PressureUpdate *pu, cudaStream_t st)
{
    if (sizeof(T) != 4) {
        set_error("pressure update: FP32 increments only");
        return -1;
    }
    const size_t n = (size_t)s->nx * s->ny * s->nz;
    const int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 16);
    k_pressure_update<<<grid, 256, 0, st>>>(reinterpret_cast<const float *>(dp), *pu, n);
    PL_CHECK_LAUNCH();
    return 0;
}

template <typename T>
static int launch_x(const Ppe *s, bool fwd, const T *in, size_t in_off, size_t in_sj, size_t in_sk, T *out,
                    size_t out_off, size_t out_sj, size_t out_sk, T scale, cudaStream_t st,
                    const PressureUpdate *pu = nullptr)
{
    using V = typename cplx_of<T>::type;
    bool fused = false;
    int rc = 1;
    switch (s->nx) {
#define PL_X_CASE(n)                                                                                               \
    case n:                                                                                                        \
        rc = fwd ? launch_x_ct<T, n, true>(s, in, in_off, in_sj, in_sk, out, out_off, out_sj, out_sk, scale, st,    \
                                           pu, &fused)                                                              \
                 : launch_x_ct<T, n, false>(s, in, in_off, in_sj, in_sk, out, out_off, out_sj, out_sk, scale, st,   \
                                            pu, &fused);                                                            \
        break;
        PL_FFT_CT_SIZES(PL_X_CASE)
#undef PL_X_CASE
    default:
        break;
    }
    if (rc == 0) return (pu && !fused) ? launch_pressure_update(s, out, pu, st) : 0;
    if (rc < 0) return rc;
    const int pb = x_pairs_per_cta(s->nx, s->ny);
    dim3 grid((s->ny / 2 + pb - 1) / pb, s->nz);
    const size_t shm = 2 * sizeof(V) * (size_t)fpad_elems<V>(pb * s->nx);
    const FftPlanDev<V> &plan = *reinterpret_cast<const FftPlanDev<V> *>(
        sizeof(T) == 8 ? (const void *)&s->px64 : (const void *)&s->px32);
    if (fwd)
        k_xfft<T, true><<<grid, 256, shm, st>>>(in, in_off, in_sj, in_sk, out, out_off, out_sj, out_sk, plan, s->ny,
                                                pb, scale);
    else
        k_xfft<T, false><<<grid, 256, shm, st>>>(in, in_off, in_sj, in_sk, out, out_off, out_sj, out_sk, plan,
                                                 s->ny, pb, scale);
    PL_CHECK_LAUNCH();
    return pu ? launch_pressure_update(s, out, pu, st) : 0;
}

template <typename T> static int launch_y(const Ppe *s, bool fwd, T *data, cudaStream_t st)
{
    using V = typename cplx_of<T>::type;
    switch (s->ny) {
#define PL_Y_CASE(n)                                                                                               \
    case n:                                                                                                        \
        if ((uintptr_t)data % 16 == 0)                                                                             \
            return fwd ? launch_y_ct<T, n, true>(s, data, st) : launch_y_ct<T, n, false>(s, data, st);             \
        break;
        PL_FFT_CT_SIZES(PL_Y_CASE)
#undef PL_Y_CASE
    default:
        break;
    }
    const int w = y_cols_per_cta(s->nx, s->ny);
    dim3 grid((s->nx / 2 + w - 1) / w, s->nz);
    const size_t shm = 2 * sizeof(V) * (size_t)fpad_elems<V>(w * s->ny);
    const FftPlanDev<V> &plan = *reinterpret_cast<const FftPlanDev<V> *>(
        sizeof(T) == 8 ? (const void *)&s->py64 : (const void *)&s->py32);
    if (fwd)
        k_yfft<T, true><<<grid, 256, shm, st>>>(data, plan, s->nx, w);
    else
        k_yfft<T, false><<<grid, 256, shm, st>>>(data, plan, s->nx, w);
    PL_CHECK_LAUNCH();
    return 0;
}

template <typename T> static int launch_trid(Ppe *s, T *x, cudaStream_t st, const double *mode0 = nullptr)
{
    TridDev t{s->nx, s->ny, s->nz, s->ncx, s->ncy, s->d_mult, s->d_rb, s->d_c};
    dim3 grid((s->nx + 127) / 128, s->ny);
    if (sizeof(T) == 4 && s->nparts == 0 && s->d_tmult != nullptr) {
        // the two-ended sweep (mixed path): one thread per half column, one
        // 256-thread CTA per SM (k_thomas_th), or two with FP32 copies of the
        // swept values (k_thomas_th2) where its rounds, 1.68 times as long,
        // are that many times fewer
        const int ncol = s->nx * s->ny, cpr = TTM_THREADS;
        const int ctas1 = std::max(1, std::min(sm_count(), (ncol + cpr - 1) / cpr));
        const int rounds1 = (ncol + ctas1 * cpr - 1) / (ctas1 * cpr);
        const int ctas2 = std::max(1, std::min(2 * sm_count(), (ncol + cpr - 1) / cpr));
        const int rounds2 = (ncol + ctas2 * cpr - 1) / (ctas2 * cpr);
        if constexpr (sizeof(T) == 4) {
            if (s->nx % TTM_THREADS == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0 &&
                168 * rounds2 < 100 * rounds1) {
                const size_t shm = tth2_smem_bytes();
                uint32_t tcols = 32;
                while (tcols < (uint32_t)s->nz) tcols *= 2;
                PL_CUDA_TRY(cudaFuncSetAttribute(k_thomas_th2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
                k_thomas_th2<<<ctas2, 2 * TTM_THREADS, shm, st>>>(x, x, s->d_tmult, s->d_trb, s->d_a, s->d_c, s->nx,
                                                                   s->ny, s->nz, s->ncx, s->ncy, (long long)s->tcs,
                                                                   mode0, rounds2, tcols);
                PL_CHECK_LAUNCH();
                return 0;
            }
        }
        const size_t shm = tth_smem_bytes<T>();
        uint32_t tcols = 32;
        while (tcols < 2u * (uint32_t)s->nz) tcols *= 2;
        PL_CUDA_TRY(cudaFuncSetAttribute(k_thomas_th<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        k_thomas_th<T><<<ctas1, 2 * TTM_THREADS, shm, st>>>(x, x, s->d_tmult, s->d_trb, s->d_a, s->d_c, s->nx, s->ny,
                                                              s->nz, s->ncx, s->ncy, (long long)s->tcs, mode0, rounds1,
                                                              tcols);
        PL_CHECK_LAUNCH();
        return 0;
    }
    double *xs = (sizeof(T) == 8 && s->nparts == 0) ? reinterpret_cast<double *>(x) : s->d_scratch;
    if (s->nparts == 0 && s->nz % TTM_G == 0 && s->nz <= TTM_MAX_NZ &&
        (s->nz <= TTM_TM_ROWS || sizeof(T) == 8 || s->d_scratch != nullptr)) {
        // swept values in TMEM (taller columns partly in the HBM scratch: in
        // place for FP64, the FP64 sweep scratch for FP32): one 128-thread CTA
        // per SM, persistent over the columns
        const size_t shm = ttm_smem_bytes<T>(s->nz);
        const int ncol = s->nx * s->ny;
        const int ctas = std::max(1, std::min(sm_count(), (ncol + TTM_THREADS - 1) / TTM_THREADS));
        const int rounds = (ncol + ctas * TTM_THREADS - 1) / (ctas * TTM_THREADS);
        uint32_t tcols = 32;
        while (tcols < 2u * (uint32_t)std::min(s->nz, TTM_TM_ROWS)) tcols *= 2;
        double *xsc = sizeof(T) == 8 ? reinterpret_cast<double *>(x) : s->d_scratch;
        if (s->nz > TTM_TM_ROWS) {
            PL_CUDA_TRY(
                cudaFuncSetAttribute(k_thomas_tmem<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
            k_thomas_tmem<T, true><<<ctas, TTM_THREADS, shm, st>>>(x, x, xsc, t, mode0, rounds, tcols);
        } else {
            PL_CUDA_TRY(
                cudaFuncSetAttribute(k_thomas_tmem<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
            k_thomas_tmem<T, false><<<ctas, TTM_THREADS, shm, st>>>(x, x, xsc, t, mode0, rounds, tcols);
        }
    } else if (s->nparts == 0) {
        k_thomas<T><<<grid, 128, 0, st>>>(x, xs, x, t, mode0);
    } else if (s->nparts <= 32) {
        PddDev p{};
        p.nparts = s->nparts;
        int kmax = 0;
        bool groups = true;
        for (int m = 0; m < s->nparts; m++) {
            p.kst[m] = s->kst[m];
            p.ksz[m] = s->ksz[m];
            kmax = std::max(kmax, s->ksz[m]);
            groups = groups && s->ksz[m] >= PTM_G && s->ksz[m] % PTM_G == 0;
        }
        p.v = s->d_v;
        p.w = s->d_w;
        p.tmpv = s->d_tmpv;
        const int ncol = s->nx * s->ny;
        const int cells = ((s->nparts + 3) / 4) * 2 * kmax; // TMEM columns of one CTA
        if (groups && s->nparts <= 8 && cells <= 512) {
            // partitions in tensor memory; the dynamic shared memory (unused)
            // caps the CTAs on an SM at what its 512 TMEM columns hold
            uint32_t tcols = 32;
            while (tcols < (uint32_t)cells) tcols *= 2;
            const int per_sm = std::max(1, std::min(512 / (int)tcols, 2048 / (32 * s->nparts)));
            const int dyn = std::max(0, 233472 / per_sm - 1024 - pdd_tm_static_smem() - 512);
            if (dyn > 48 * 1024)
                PL_CUDA_TRY(cudaFuncSetAttribute(k_pdd_tm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
            k_pdd_tm<T><<<(ncol + 31) / 32, dim3(32, s->nparts), dyn, st>>>(x, x, t, p, sizeof(T) == 4 ? mode0 : nullptr,
                                                                             kmax, tcols);
        } else {
            k_pdd_par<T><<<(ncol + 31) / 32, dim3(32, s->nparts), 0, st>>>(x, s->d_scratch, x, t, p,
                                                                          sizeof(T) == 4 ? mode0 : nullptr);
        }
    } else {
        if (sizeof(T) == 4) {
            k_widen<<<1184, 256, 0, st>>>(reinterpret_cast<const float *>(x), xs, s->scratch_elems);
            PL_CHECK_LAUNCH();
        } else {
            PL_CUDA_TRY(cudaMemcpyAsync(xs, x, sizeof(double) * s->scratch_elems, cudaMemcpyDeviceToDevice, st));
        }
        PddDev p{};
        p.nparts = s->nparts;
        for (int m = 0; m < s->nparts; m++) {
            p.kst[m] = s->kst[m];
            p.ksz[m] = s->ksz[m];
        }
        p.v = s->d_v;
        p.w = s->d_w;
        p.tmpv = s->d_tmpv;
        k_pdd<T><<<grid, 128, 0, st>>>(xs, x, t, p, sizeof(T) == 4 ? mode0 : nullptr);
    }
    PL_CHECK_LAUNCH();
    return 0;
}

static inline void mark(const Ppe *s, const char *name)
{
    if (s->mark) s->mark(s->mark_ctx, name);
}

int ppe_solve_fp64_strided(Ppe *s, const double *in, double *out, size_t off, size_t sj, size_t sk,
                           double *d_work, cudaStream_t st)
{
    const size_t nxl = s->nx, nxy = (size_t)s->nx * s->ny;
    if (launch_x<double>(s, true, in, off, sj, sk, d_work, 0, nxl, nxy, 1.0, st)) return -1;
    mark(s, "ppe_xfft_fwd");
    if (launch_y<double>(s, true, d_work, st)) return -1;
    mark(s, "ppe_yfft_fwd");
    if (launch_trid<double>(s, d_work, st)) return -1;
    mark(s, s->nparts ? "ppe_pdd" : "ppe_thomas");
    if (launch_y<double>(s, false, d_work, st)) return -1;
    mark(s, "ppe_yfft_bwd");
    if (launch_x<double>(s, false, d_work, 0, nxl, nxy, out, off, sj, sk, s->norm, st)) return -1;
    mark(s, "ppe_xfft_bwd");
    return 0;
}

template <typename T, int N> static int launch_xdiv(Ppe *s, const DivIn &d, T *out, double *part, cudaStream_t st)
{
    using V = typename cplx_of<T>::type;
    constexpr int shm = xdiv_smem_bytes<T, N>();
    const V *tw = reinterpret_cast<const V *>(sizeof(T) == 8 ? (const void *)s->d_twx64 : (const void *)s->d_twx32);
    if (shm > 48 * 1024)
        PL_CUDA_TRY(cudaFuncSetAttribute(k_xfft_div_pf<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, shm));
    const int total = (s->ny / 2) * s->nz;
    k_xfft_div_pf<T, N><<<persistent_grid(k_xfft_div_pf<T, N>, shm, total, XDIV_THREADS), XDIV_THREADS, shm, st>>>(
        d, out, tw, s->ny, total, part);
    PL_CHECK_LAUNCH();
    return 0;
}

template <typename T> int ppe_xfwd_div(Ppe *s, const DivIn &d, T *out, double *part, cudaStream_t st)
{
    switch (s->nx) {
#define PL_XDIV_CASE(n)                                                                                               \
    case n:                                                                                                          \
        return launch_xdiv<T, n>(s, d, out, part, st);
        PL_FFT_CT_SIZES(PL_XDIV_CASE)
#undef PL_XDIV_CASE
    default:
        return 1;
    }
}
template int ppe_xfwd_div<double>(Ppe *, const DivIn &, double *, double *, cudaStream_t);
template int ppe_xfwd_div<float>(Ppe *, const DivIn &, float *, double *, cudaStream_t);

int ppe_solve_fp64_from_x(Ppe *s, double *d_var, cudaStream_t st)
{
    const size_t nxl = s->nx, nxy = (size_t)s->nx * s->ny;
    if (launch_y<double>(s, true, d_var, st)) return -1;
    mark(s, "ppe_yfft_fwd");
    if (launch_trid<double>(s, d_var, st)) return -1;
    mark(s, s->nparts ? "ppe_pdd" : "ppe_thomas");
    if (launch_y<double>(s, false, d_var, st)) return -1;
    mark(s, "ppe_yfft_bwd");
    if (launch_x<double>(s, false, d_var, 0, nxl, nxy, d_var, 0, nxl, nxy, s->norm, st)) return -1;
    mark(s, "ppe_xfft_bwd");
    return 0;
}

int ppe_solve_fp64(Ppe *s, double *d_var, cudaStream_t st)
{
    const size_t nxl = s->nx, nxy = (size_t)s->nx * s->ny;
    return ppe_solve_fp64_strided(s, d_var, d_var, 0, nxl, nxy, d_var, st);
}

int ppe_solve_fp32(Ppe *s, float *d_var, const double *mode0, cudaStream_t st, const PressureUpdate *pu)
{
    const size_t nxl = s->nx, nxy = (size_t)s->nx * s->ny;
    if (launch_x<float>(s, true, d_var, 0, nxl, nxy, d_var, 0, nxl, nxy, 1.0f, st)) return -1;
    mark(s, "ppe_xfft_fwd");
    return ppe_solve_fp32_from_x(s, d_var, mode0, st, pu);
}

int ppe_solve_fp32_from_x(Ppe *s, float *d_var, const double *mode0, cudaStream_t st, const PressureUpdate *pu)
{
    const size_t nxl = s->nx, nxy = (size_t)s->nx * s->ny;
    if (launch_y<float>(s, true, d_var, st)) return -1;
    mark(s, "ppe_yfft_fwd");
    if (launch_trid<float>(s, d_var, st, mode0)) return -1;
    mark(s, s->nparts ? "ppe_pdd" : "ppe_thomas");
    if (launch_y<float>(s, false, d_var, st)) return -1;
    mark(s, "ppe_yfft_bwd");
    if (launch_x<float>(s, false, d_var, 0, nxl, nxy, d_var, 0, nxl, nxy, (float)s->norm, st, pu)) return -1;
    mark(s, "ppe_xfft_bwd");
    return 0;
}

template <typename T> int ppe_slab_forward_from_x(Ppe *s, T *d_var, cudaStream_t st, const double *mode0)
{
    if (launch_y<T>(s, true, d_var, st)) return -1;
    mark(s, "ppe_yfft_fwd");
    if (s->nz % TTM_G == 0 && s->nz <= TTM_TM_ROWS) {
        // the partition's sweep in tensor memory, reading the right-hand side
        // as stored and writing the local solution to the FP64 sweep buffer
        TridDev t{s->nx, s->ny, s->nz, s->ncx, s->ncy, s->d_mult, s->d_rb, s->d_c};
        const size_t shm = ttm_smem_bytes<T>(s->nz);
        const int ncol = s->nx * s->ny;
        const int ctas = std::max(1, std::min(sm_count(), (ncol + TTM_THREADS - 1) / TTM_THREADS));
        const int rounds = (ncol + ctas * TTM_THREADS - 1) / (ctas * TTM_THREADS);
        uint32_t tcols = 32;
        while (tcols < 2u * (uint32_t)s->nz) tcols *= 2;
        auto kern = k_thomas_tmem<T, false, double, false>;
        PL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        kern<<<ctas, TTM_THREADS, shm, st>>>(d_var, s->d_scratch, s->d_scratch, t, mode0, rounds, tcols);
        PL_CHECK_LAUNCH();
        mark(s, "ppe_pdd_sweep");
        return 0;
    }
    if (sizeof(T) == 4) {
        k_widen<<<1184, 256, 0, st>>>(reinterpret_cast<const float *>(d_var), s->d_scratch, s->scratch_elems);
        PL_CHECK_LAUNCH();
    } else {
        PL_CUDA_TRY(cudaMemcpyAsync(s->d_scratch, d_var, sizeof(double) * s->scratch_elems, cudaMemcpyDeviceToDevice,
                                    st));
    }
    TridDev t{s->nx, s->ny, s->nz, s->ncx, s->ncy, s->d_mult, s->d_rb, s->d_c};
    k_pdd_sweep<<<dim3((s->nx + 127) / 128, s->ny), 128, 0, st>>>(s->d_scratch, t, mode0);
    PL_CHECK_LAUNCH();
    mark(s, "ppe_pdd_sweep");
    return 0;
}
template int ppe_slab_forward_from_x<double>(Ppe *, double *, cudaStream_t, const double *);
template int ppe_slab_forward_from_x<float>(Ppe *, float *, cudaStream_t, const double *);

template <typename T> int ppe_slab_forward(Ppe *s, T *d_var, cudaStream_t st, const double *mode0)
{
    const size_t nxl = s->nx, nxy = (size_t)s->nx * s->ny;
    if (launch_x<T>(s, true, d_var, 0, nxl, nxy, d_var, 0, nxl, nxy, (T)1, st)) return -1;
    mark(s, "ppe_xfft_fwd");
    return ppe_slab_forward_from_x<T>(s, d_var, st, mode0);
}
template int ppe_slab_forward<double>(Ppe *, double *, cudaStream_t, const double *);
template int ppe_slab_forward<float>(Ppe *, float *, cudaStream_t, const double *);

int ppe_slab_iface(Ppe *s, cudaStream_t st, int gauge00)
{
    if (!s->has_up) return 0;
    TridDev t{s->nx, s->ny, s->nz, s->ncx, s->ncy, s->d_mult, s->d_rb, s->d_c};
    k_pdd_iface<<<dim3((s->nx + 255) / 256, s->ny), 256, 0, st>>>(s->d_scratch, s->d_tvar, s->d_w, s->d_tmpv, s->d_y2,
                                                                   s->d_y3, t, gauge00);
    PL_CHECK_LAUNCH();
    return 0;
}

template <typename T> int ppe_slab_backward(Ppe *s, T *d_var, cudaStream_t st, const PressureUpdate *pu)
{
    const size_t nxl = s->nx, nxy = (size_t)s->nx * s->ny;
    TridDev t{s->nx, s->ny, s->nz, s->ncx, s->ncy, s->d_mult, s->d_rb, s->d_c};
    k_pdd_fix<T><<<dim3((s->nx + 127) / 128, s->ny), 128, 0, st>>>(s->d_scratch, d_var, s->d_v, s->d_w, s->d_y1,
                                                                   s->d_y2, s->has_down, s->has_up, t);
    PL_CHECK_LAUNCH();
    mark(s, "ppe_pdd_fix");
    if (launch_y<T>(s, false, d_var, st)) return -1;
    mark(s, "ppe_yfft_bwd");
    if (launch_x<T>(s, false, d_var, 0, nxl, nxy, d_var, 0, nxl, nxy, (T)s->norm, st, pu)) return -1;
    mark(s, "ppe_xfft_bwd");
    return 0;
}
template int ppe_slab_backward<double>(Ppe *, double *, cudaStream_t, const PressureUpdate *);
template int ppe_slab_backward<float>(Ppe *, float *, cudaStream_t, const PressureUpdate *);

} // namespace pl

// ------------------------------------------------------------------------
// Allocation-free solve (pl_ppe_solve_noalloc in include/powerllel_b200.h).
//
// Some callers cannot call cudaMalloc while they solve: a host program whose
// device memory is owned by another allocator (a pool that claimed the GPU's
// memory at start-up), or a loop that must not stall on cudaMalloc, which can
// wait for the device to go idle.  For them the mixed-precision Thomas solve
// runs the HBM-scratch sweep kernel (k_thomas), whose FP64 forward-swept
// values go to this fixed device array instead of the buffer pl_ppe_create
// allocates.  The array is file-scope device memory: every GPU that loads
// the library holds it (16 MiB) until the process exits.
// ------------------------------------------------------------------------
namespace pl {

constexpr size_t NOALLOC_SCRATCH_DOUBLES = (size_t)1 << 21; // 16 MiB: nx*ny*nz <= 2,097,152
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

// Device address of g_noalloc_scratch.  In host code the symbol names a
// host-side stand-in, not device memory, so the address is looked up with
// cudaGetSymbolAddress once per device and context (with that device
// current); a new context on the device (after cudaDeviceReset) looks it up
// again, since the array then lives at a new address.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);

static CtxGetCurrentFn ctx_get_current()
{
    static CtxGetCurrentFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(f);
    }
    return fn;
}

static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[64] = {nullptr};
static CUcontext g_noalloc_ctx[64] = {nullptr};

static int noalloc_scratch(double **out)
{
    int dev = -1;
    PL_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("pl_ppe_solve_noalloc: device ordinal out of range");
        return -1;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    CtxGetCurrentFn get = ctx_get_current();
    auto current = [&]() {
        CUcontext c = nullptr;
        if (get && get(&c) != CUDA_SUCCESS) c = nullptr;
        return c;
    };
    const CUcontext ctx = current(); // null: no context is current in this thread yet
    if (!g_noalloc_ptr[dev] || ctx == nullptr || ctx != g_noalloc_ctx[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch); // makes the device's context current
        if (e != cudaSuccess || ptr == nullptr) {
            set_error(std::string("pl_ppe_solve_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return -1;
        }
        g_noalloc_ptr[dev] = static_cast<double *>(ptr);
        g_noalloc_ctx[dev] = current();
    }
    *out = g_noalloc_ptr[dev];
    return 0;
}

static int ppe_solve_fp32_noalloc(Ppe *s, float *d_var, cudaStream_t st)
{
    if (s->prec != PREC_MIXED || s->nparts != 0) {
        set_error("pl_ppe_solve_noalloc: the plan must be PL_MIXED with Thomas (nparts = 0)");
        return -1;
    }
    const size_t n = (size_t)s->nx * s->ny * s->nz;
    if (n > NOALLOC_SCRATCH_DOUBLES) {
        set_error("pl_ppe_solve_noalloc: nx*ny*nz = " + std::to_string(n) + " exceeds the fixed scratch of " +
                  std::to_string(NOALLOC_SCRATCH_DOUBLES) + " values; use pl_ppe_solve");
        return -1;
    }
    double *xs = nullptr;
    if (noalloc_scratch(&xs)) return -1;
    const size_t nxl = s->nx, nxy = (size_t)s->nx * s->ny;
    if (launch_x<float>(s, true, d_var, 0, nxl, nxy, d_var, 0, nxl, nxy, 1.0f, st)) return -1;
    if (launch_y<float>(s, true, d_var, st)) return -1;
    // every value of the scratch is written by the forward sweep before the
    // backward sweep reads it, so nothing needs clearing between calls
    TridDev t{s->nx, s->ny, s->nz, s->ncx, s->ncy, s->d_mult, s->d_rb, s->d_c};
    dim3 grid((s->nx + 127) / 128, s->ny);
    k_thomas<float><<<grid, 128, 0, st>>>(d_var, xs, d_var, t, nullptr);
    PL_CHECK_LAUNCH();
    if (launch_y<float>(s, false, d_var, st)) return -1;
    if (launch_x<float>(s, false, d_var, 0, nxl, nxy, d_var, 0, nxl, nxy, (float)s->norm, st)) return -1;
    return 0;
}

} // namespace pl

extern "C" int pl_ppe_solve_noalloc(pl_ppe *p, void *d_var, void *stream)
{
    if (!p || !d_var) {
        pl::set_error("pl_ppe_solve_noalloc: null argument");
        return -1;
    }
    if (reinterpret_cast<uintptr_t>(d_var) % 8 != 0) { // column pairs of the y transform, as pl_ppe_solve
        pl::set_error("pl_ppe_solve_noalloc: d_var must be aligned to 8 bytes (two elements)");
        return -1;
    }
    return pl::ppe_solve_fp32_noalloc(&p->s, (float *)d_var, (cudaStream_t)stream);
}
