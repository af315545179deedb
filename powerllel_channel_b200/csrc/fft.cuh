// fft.cuh -- shared-memory batched complex FFT engine and the real<->half-complex
// pairing used by the PPE kernels.
//
// The reference transforms each periodic direction with FFTW's R2HC / HC2R
// (src/src_c/mod_fft_fftw.inc:35-95): forward unnormalised, output in FFTW's
// half-complex order r_0..r_{n/2}, i_{(n+1)/2-1}..i_1; backward unnormalised.
// Here two real lines are packed into one complex line (z = a + i b), one
// complex FFT of length n is run, and the two half-complex spectra are split
// out of it (and merged back before the inverse).  Every stored value is the
// half-complex slot FFTW would produce, so the tridiagonal stage sees the same
// unknowns as the reference.
//
// The complex FFT is a Stockham autosort decimation-in-time transform over a
// batch held in shared memory, ping-ponging between two buffers, with radix
// 8, 6, 4, 3 and 2 passes (each thread keeps one butterfly in registers).
// Twiddles exp(-2 pi i t / n) come from a table computed on
// the host in long double.
#pragma once

#include "common.cuh"

namespace pl {

constexpr int FFT_MAX_STAGES = 16;

// A length-n transform plan: radix of each stage and the twiddle table
// (device pointer, n complex entries of type V).
template <typename V> struct FftPlanDev {
    int n;
    int nstages;
    int radix[FFT_MAX_STAGES];
    const V *tw; // exp(-2 pi i t / n), t < n
};

// Shared-memory index padding: one unused slot after every 128 bytes (8
// double2 or 16 float2), so the strided writes of a Stockham stage (stride R
// elements when Ns = 1) spread over all banks instead of a few.
template <typename V> __host__ __device__ constexpr int fpad(int i)
{
    return i + (i >> (sizeof(V) == 16 ? 3 : 4));
}
template <typename V> __host__ __device__ constexpr int fpad_elems(int n) { return fpad<V>(n) + 1; }

template <typename V, bool FWD>
__device__ __forceinline__ V twiddle(const V *tw, int t)
{
    V w = __ldg(tw + t);
    if (!FWD) w.y = -w.y;
    return w;
}

// R-point DFTs on registers.  FWD selects the sign of the exponent.
template <typename V, bool FWD> __device__ __forceinline__ void dft2(V &a0, V &a1)
{
    V t = a0;
    a0 = cadd(t, a1);
    a1 = csub(t, a1);
}

template <typename V, bool FWD> __device__ __forceinline__ void dft4(V &a0, V &a1, V &a2, V &a3)
{
    V t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), d = csub(a1, a3);
    V t3;
    if (FWD) { // -i * d
        t3.x = d.y;
        t3.y = -d.x;
    } else { // +i * d
        t3.x = -d.y;
        t3.y = d.x;
    }
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, t3);
    a3 = csub(t1, t3);
}

template <typename V, bool FWD> __device__ __forceinline__ void dft3(V &a0, V &a1, V &a2)
{
    using T = decltype(a0.x);
    const T c = T(-0.5);
    const T s = FWD ? T(-0.86602540378443864676372317075293618) : T(0.86602540378443864676372317075293618);
    V sum = cadd(a1, a2), dif = csub(a1, a2);
    V t;
    t.x = a0.x + c * sum.x;
    t.y = a0.y + c * sum.y;
    // i * s * dif
    V u;
    u.x = -s * dif.y;
    u.y = s * dif.x;
    a0 = cadd(a0, sum);
    a1 = cadd(t, u);
    a2 = csub(t, u);
}

// 8-point DFT: two 4-point DFTs (even, odd samples) and the w8^k combination
template <typename V, bool FWD> __device__ __forceinline__ void dft8(V *a)
{
    using T = decltype(a[0].x);
    const T h = T(0.70710678118654752440084436210484904);
    V e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
    V o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
    dft4<V, FWD>(e0, e1, e2, e3);
    dft4<V, FWD>(o0, o1, o2, o3);
    // w8^1 o1, w8^2 o2, w8^3 o3 with w8 = exp(-+ i pi/4)
    V t1, t2, t3;
    if (FWD) {
        t1.x = h * (o1.x + o1.y);
        t1.y = h * (o1.y - o1.x);
        t2.x = o2.y;
        t2.y = -o2.x;
        t3.x = h * (o3.y - o3.x);
        t3.y = -h * (o3.x + o3.y);
    } else {
        t1.x = h * (o1.x - o1.y);
        t1.y = h * (o1.x + o1.y);
        t2.x = -o2.y;
        t2.y = o2.x;
        t3.x = -h * (o3.x + o3.y);
        t3.y = h * (o3.x - o3.y);
    }
    a[0] = cadd(e0, o0);
    a[4] = csub(e0, o0);
    a[1] = cadd(e1, t1);
    a[5] = csub(e1, t1);
    a[2] = cadd(e2, t2);
    a[6] = csub(e2, t2);
    a[3] = cadd(e3, t3);
    a[7] = csub(e3, t3);
}

// 6-point DFT: two 3-point DFTs (even, odd samples) and the w6^k combination
template <typename V, bool FWD> __device__ __forceinline__ void dft6(V *a)
{
    using T = decltype(a[0].x);
    const T s3 = T(0.86602540378443864676372317075293618);
    V e0 = a[0], e1 = a[2], e2 = a[4];
    V o0 = a[1], o1 = a[3], o2 = a[5];
    dft3<V, FWD>(e0, e1, e2);
    dft3<V, FWD>(o0, o1, o2);
    // w6 = exp(-+ i pi/3) = (1/2, -+ s3), w6^2 = (-1/2, -+ s3)
    const T sg = FWD ? -s3 : s3;
    V t1, t2;
    t1.x = T(0.5) * o1.x - sg * o1.y;
    t1.y = T(0.5) * o1.y + sg * o1.x;
    t2.x = T(-0.5) * o2.x - sg * o2.y;
    t2.y = T(-0.5) * o2.y + sg * o2.x;
    a[0] = cadd(e0, o0);
    a[3] = csub(e0, o0);
    a[1] = cadd(e1, t1);
    a[4] = csub(e1, t1);
    a[2] = cadd(e2, t2);
    a[5] = csub(e2, t2);
}

// One Stockham stage over a batch of `nb` sequences of length n.
// Element (m, b) of a buffer lives at buf[fpad(m * sm + b * sb)].
// BATCH_FAST: consecutive threads take consecutive b (use when sb == 1).
template <typename V, bool FWD, bool BATCH_FAST>
__device__ __forceinline__ void fft_stage(const V *__restrict__ src, V *__restrict__ dst, int n, int nb, int sm,
                                          int sb, int R, int Ns, const V *tw, int tid, int nthr)
{
    const int nbf = n / R;           // butterflies per sequence
    const int tstep = n / (Ns * R);  // twiddle index step
    const int total = nbf * nb;
    for (int q = tid; q < total; q += nthr) {
        int b, j;
        if (BATCH_FAST) {
            b = q % nb;
            j = q / nb;
        } else {
            j = q % nbf;
            b = q / nbf;
        }
        const int base = b * sb;
        const int jm = j % Ns;
        const int idxD = (j / Ns) * Ns * R + jm;
        if (R == 8 || R == 6) {
            V a[8];
#pragma unroll
            for (int r = 0; r < 8; r++)
                if (r < R) a[r] = src[fpad<V>(base + (j + r * nbf) * sm)];
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < 8; r++)
                    if (r < R) a[r] = cmul(a[r], twiddle<V, FWD>(tw, r * jm * tstep));
            }
            if (R == 8)
                dft8<V, FWD>(a);
            else
                dft6<V, FWD>(a);
#pragma unroll
            for (int r = 0; r < 8; r++)
                if (r < R) dst[fpad<V>(base + (idxD + r * Ns) * sm)] = a[r];
        } else if (R == 4) {
            V a0 = src[fpad<V>(base + j * sm)], a1 = src[fpad<V>(base + (j + nbf) * sm)], a2 = src[fpad<V>(base + (j + 2 * nbf) * sm)], a3 = src[fpad<V>(base + (j + 3 * nbf) * sm)];
            if (Ns > 1) {
                a1 = cmul(a1, twiddle<V, FWD>(tw, jm * tstep));
                a2 = cmul(a2, twiddle<V, FWD>(tw, 2 * jm * tstep));
                a3 = cmul(a3, twiddle<V, FWD>(tw, 3 * jm * tstep));
            }
            dft4<V, FWD>(a0, a1, a2, a3);
            dst[fpad<V>(base + idxD * sm)] = a0;
            dst[fpad<V>(base + (idxD + Ns) * sm)] = a1;
            dst[fpad<V>(base + (idxD + 2 * Ns) * sm)] = a2;
            dst[fpad<V>(base + (idxD + 3 * Ns) * sm)] = a3;
        } else if (R == 2) {
            V a0 = src[fpad<V>(base + j * sm)], a1 = src[fpad<V>(base + (j + nbf) * sm)];
            if (Ns > 1) a1 = cmul(a1, twiddle<V, FWD>(tw, jm * tstep));
            dft2<V, FWD>(a0, a1);
            dst[fpad<V>(base + idxD * sm)] = a0;
            dst[fpad<V>(base + (idxD + Ns) * sm)] = a1;
        } else { // R == 3
            V a0 = src[fpad<V>(base + j * sm)], a1 = src[fpad<V>(base + (j + nbf) * sm)], a2 = src[fpad<V>(base + (j + 2 * nbf) * sm)];
            if (Ns > 1) {
                a1 = cmul(a1, twiddle<V, FWD>(tw, jm * tstep));
                a2 = cmul(a2, twiddle<V, FWD>(tw, 2 * jm * tstep));
            }
            dft3<V, FWD>(a0, a1, a2);
            dst[fpad<V>(base + idxD * sm)] = a0;
            dst[fpad<V>(base + (idxD + Ns) * sm)] = a1;
            dst[fpad<V>(base + (idxD + 2 * Ns) * sm)] = a2;
        }
    }
}

// Full transform; data starts in buf0, result pointer returned (buf0 or buf1).
// Ends with a __syncthreads().
template <typename V, bool FWD, bool BATCH_FAST>
__device__ V *fft_batch(V *buf0, V *buf1, const FftPlanDev<V> &p, int nb, int sm, int sb, int tid, int nthr)
{
    V *src = buf0, *dst = buf1;
    int Ns = 1;
    for (int s = 0; s < p.nstages; s++) {
        const int R = p.radix[s];
        fft_stage<V, FWD, BATCH_FAST>(src, dst, p.n, nb, sm, sb, R, Ns, p.tw, tid, nthr);
        __syncthreads();
        Ns *= R;
        V *t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// ---------------------------------------------------------------------------
// Compile-time sizes.  For the common line lengths the transform length, the
// radix sequence, the batch geometry and every index divisor are template
// constants, so a stage costs its butterfly arithmetic plus two shared-memory
// accesses per element; twiddles are read from a shared-memory copy of the
// table.  The radix sequence and the operations are those of the runtime
// engine above, so both give bitwise identical results.
// ---------------------------------------------------------------------------

// radix of stage s for length n (0 past the last stage): 8s first, then 4, or
// a 2 merged with one 3 into a 6, then 3s (the host's factor_radices order)
__host__ __device__ constexpr int ct_radix(int n, int s)
{
    int m = n, idx = 0;
    while (m % 8 == 0) {
        if (idx == s) return 8;
        idx++;
        m /= 8;
    }
    int two = 0;
    if (m % 4 == 0) {
        if (idx == s) return 4;
        idx++;
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
    if (two && threes) {
        if (idx == s) return 6;
        idx++;
        threes--;
    } else if (two) {
        if (idx == s) return 2;
        idx++;
    }
    while (threes-- > 0) {
        if (idx == s) return 3;
        idx++;
    }
    return 0;
}

// product of the radices of the stages before s (Stockham's Ns)
__host__ __device__ constexpr int ct_ns(int n, int s)
{
    int p = 1;
    for (int q = 0; q < s; q++) p *= ct_radix(n, q);
    return p;
}

template <typename V, bool FWD, int R> __device__ __forceinline__ void dft_r(V *a)
{
    if constexpr (R == 8)
        dft8<V, FWD>(a);
    else if constexpr (R == 6)
        dft6<V, FWD>(a);
    else if constexpr (R == 4)
        dft4<V, FWD>(a[0], a[1], a[2], a[3]);
    else if constexpr (R == 3)
        dft3<V, FWD>(a[0], a[1], a[2]);
    else
        dft2<V, FWD>(a[0], a[1]);
}

// Offset of stage s's twiddle block in the per-stage table: stage s (s >= 1)
// holds w^(r jm N/(NS R)) at [(r-1) NS + jm], r = 1..R-1, jm < NS, so the
// threads of a warp (consecutive jm) read consecutive entries.  The blocks
// add up to N - 1 entries.
__host__ __device__ constexpr int ct_twoff(int n, int s)
{
    int off = 0;
    for (int q = 1; q < s; q++) off += ct_ns(n, q) * (ct_radix(n, q) - 1);
    return off;
}

// Gather the per-stage twiddle table of length-N transforms from the global
// table tw[t] = exp(-2 pi i t / N) (same values, reordered).
template <typename V, int N, int NTHR>
__device__ __forceinline__ void ct_build_twiddles(const V *__restrict__ twg, V *__restrict__ tws, int tid)
{
    int s = 1;
    int off = 0;
#pragma unroll 1
    for (; ct_radix(N, s) != 0; s++) {
        const int R = ct_radix(N, s), NS = ct_ns(N, s), tstep = N / (NS * R);
        for (int idx = tid; idx < NS * (R - 1); idx += NTHR) {
            const int r = idx / NS + 1, jm = idx % NS;
            tws[off + idx] = __ldg(twg + r * jm * tstep);
        }
        off += NS * (R - 1);
    }
}

// One stage over NB sequences (nb <= NB present) of length N; element (m, b)
// at buf[fpad(m * SM + b * SB)]; BF: consecutive threads take consecutive b.
// tws: this stage's block of the per-stage twiddle table.
template <typename V, bool FWD, bool BF, int N, int R, int NS, int NB, int SM, int SB, int NTHR>
__device__ __forceinline__ void ct_stage(const V *__restrict__ src, V *__restrict__ dst, int nb,
                                         const V *__restrict__ tws, int tid)
{
    constexpr int NBF = N / R, TOTAL = NBF * NB;
    constexpr int ITERS = (TOTAL + NTHR - 1) / NTHR;
#pragma unroll
    for (int it = 0; it < ITERS; it++) {
        const int q = tid + it * NTHR;
        if (TOTAL % NTHR == 0 || q < TOTAL) {
            const int b = BF ? q % NB : q / NBF;
            const int j = BF ? q / NB : q % NBF;
            if (b < nb) {
                const int jm = j % NS;
                const int idxD = (j / NS) * NS * R + jm;
                const int base = b * SB;
                V a[R];
#pragma unroll
                for (int r = 0; r < R; r++) a[r] = src[fpad<V>(base + (j + r * NBF) * SM)];
                if (NS > 1) {
#pragma unroll
                    for (int r = 1; r < R; r++) {
                        V w = tws[(r - 1) * NS + jm];
                        if (!FWD) w.y = -w.y;
                        a[r] = cmul(a[r], w);
                    }
                }
                dft_r<V, FWD, R>(a);
#pragma unroll
                for (int r = 0; r < R; r++) dst[fpad<V>(base + (idxD + r * NS) * SM)] = a[r];
            }
        }
    }
}

// All stages from S on; tws is the per-stage twiddle table
// (ct_build_twiddles).  Returns the buffer holding the result.  Ends with a
// __syncthreads().
template <typename V, bool FWD, bool BF, int N, int NB, int SM, int SB, int NTHR, int S = 0>
__device__ __forceinline__ V *ct_batch(V *src, V *dst, int nb, const V *tws, int tid)
{
    if constexpr (ct_radix(N, S) == 0) {
        return src;
    } else {
        ct_stage<V, FWD, BF, N, ct_radix(N, S), ct_ns(N, S), NB, SM, SB, NTHR>(src, dst, nb,
                                                                              tws + (S > 0 ? ct_twoff(N, S) : 0), tid);
        __syncthreads();
        return ct_batch<V, FWD, BF, N, NB, SM, SB, NTHR, S + 1>(dst, src, nb, tws, tid);
    }
}

// In-place variant of ct_stage: every thread first loads, twiddles and
// transforms all of its butterflies in registers, then (after a barrier that
// the caller's previous stage ends with and one here) stores them over the
// same buffer.  Halves the shared memory of the ping-pong form.
template <typename V, bool FWD, bool BF, int N, int R, int NS, int NB, int SM, int SB, int NTHR>
__device__ __forceinline__ void ct_stage_ip(V *buf, int nb, const V *__restrict__ tws, int tid)
{
    constexpr int NBF = N / R, TOTAL = NBF * NB;
    constexpr int ITERS = (TOTAL + NTHR - 1) / NTHR;
    V a[ITERS][R];
#pragma unroll
    for (int it = 0; it < ITERS; it++) {
        const int q = tid + it * NTHR;
        if (TOTAL % NTHR == 0 || q < TOTAL) {
            const int b = BF ? q % NB : q / NBF;
            const int j = BF ? q / NB : q % NBF;
            if (b < nb) {
                const int jm = j % NS;
                const int base = b * SB;
#pragma unroll
                for (int r = 0; r < R; r++) a[it][r] = buf[fpad<V>(base + (j + r * NBF) * SM)];
                if (NS > 1) {
#pragma unroll
                    for (int r = 1; r < R; r++) {
                        V w = tws[(r - 1) * NS + jm];
                        if (!FWD) w.y = -w.y;
                        a[it][r] = cmul(a[it][r], w);
                    }
                }
                dft_r<V, FWD, R>(a[it]);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < ITERS; it++) {
        const int q = tid + it * NTHR;
        if (TOTAL % NTHR == 0 || q < TOTAL) {
            const int b = BF ? q % NB : q / NBF;
            const int j = BF ? q / NB : q % NBF;
            if (b < nb) {
                const int jm = j % NS;
                const int idxD = (j / NS) * NS * R + jm;
                const int base = b * SB;
#pragma unroll
                for (int r = 0; r < R; r++) buf[fpad<V>(base + (idxD + r * NS) * SM)] = a[it][r];
            }
        }
    }
}

// number of stages of a length-n transform
__host__ __device__ constexpr int ct_nstages(int n)
{
    int s = 0;
    while (ct_radix(n, s) != 0) s++;
    return s;
}

// Stages S .. SEND-1 (all remaining stages by default), in place in buf.
// Ends with a __syncthreads().
template <typename V, bool FWD, bool BF, int N, int NB, int SM, int SB, int NTHR, int S = 0,
          int SEND = ct_nstages(N)>
__device__ __forceinline__ void ct_batch_ip(V *buf, int nb, const V *tws, int tid)
{
    if constexpr (S < SEND) {
        ct_stage_ip<V, FWD, BF, N, ct_radix(N, S), ct_ns(N, S), NB, SM, SB, NTHR>(
            buf, nb, tws + (S > 0 ? ct_twoff(N, S) : 0), tid);
        __syncthreads();
        ct_batch_ip<V, FWD, BF, N, NB, SM, SB, NTHR, S + 1, SEND>(buf, nb, tws, tid);
    }
}

// The last stage, its outputs handed to `out(b, m, value)` (line b, element
// m) instead of stored back: the inverse kernels write them to global memory
// straight from registers.  For a fixed r consecutive threads hold
// consecutive m (BF = false) or consecutive b (BF = true).  Reads buf only,
// so it needs no barrier of its own; the caller's next write to buf must
// follow a __syncthreads().
template <typename V, bool FWD, bool BF, int N, int NB, int SM, int SB, int NTHR, typename OUT>
__device__ __forceinline__ void ct_last_stage(const V *buf, int nb, const V *tws, int tid, const OUT &out)
{
    constexpr int S = ct_nstages(N) - 1, R = ct_radix(N, S), NS = ct_ns(N, S);
    constexpr int NBF = N / R, TOTAL = NBF * NB;
    constexpr int ITERS = (TOTAL + NTHR - 1) / NTHR;
    static_assert(S > 0 && NS * R == N, "last stage of a multi-stage transform");
    tws += ct_twoff(N, S);
#pragma unroll
    for (int it = 0; it < ITERS; it++) {
        const int q = tid + it * NTHR;
        if (TOTAL % NTHR == 0 || q < TOTAL) {
            const int b = BF ? q % NB : q / NBF;
            const int j = BF ? q / NB : q % NBF; // j < NS: output index j + r NS
            if (b < nb) {
                const int base = b * SB;
                V a[R];
#pragma unroll
                for (int r = 0; r < R; r++) a[r] = buf[fpad<V>(base + (j + r * NBF) * SM)];
#pragma unroll
                for (int r = 1; r < R; r++) {
                    V w = tws[(r - 1) * NS + j];
                    if (!FWD) w.y = -w.y;
                    a[r] = cmul(a[r], w);
                }
                dft_r<V, FWD, R>(a);
#pragma unroll
                for (int r = 0; r < R; r++) out(b, j + r * NS, a[r]);
            }
        }
    }
}

// The first stage (NS = 1, no twiddles) with its inputs produced by `in(b, m)`
// (line b, element m) instead of read from the work buffer: the kernels
// read their staged raw data through it, pairing the two real lines (and,
// for the inverse, merging the half-complex spectra) on the fly.  Writes
// the stage's output to buf; the caller then runs the stages from S = 1.
template <typename V, bool FWD, bool BF, int N, int NB, int SM, int SB, int NTHR, typename IN>
__device__ __forceinline__ void ct_first_stage(V *__restrict__ buf, int nb, const IN &in, int tid)
{
    constexpr int R = ct_radix(N, 0), NBF = N / R, TOTAL = NBF * NB;
    constexpr int ITERS = (TOTAL + NTHR - 1) / NTHR;
#pragma unroll
    for (int it = 0; it < ITERS; it++) {
        const int q = tid + it * NTHR;
        if (TOTAL % NTHR == 0 || q < TOTAL) {
            const int b = BF ? q % NB : q / NBF;
            const int j = BF ? q / NB : q % NBF;
            if (b < nb) {
                V a[R];
#pragma unroll
                for (int r = 0; r < R; r++) a[r] = in(b, j + r * NBF);
                dft_r<V, FWD, R>(a);
                const int base = b * SB;
#pragma unroll
                for (int r = 0; r < R; r++) buf[fpad<V>(base + (j * R + r) * SM)] = a[r];
            }
        }
    }
}

// The last stage of a forward transform, its outputs handed in mirror
// pairs to `out(b, m, Z_m, Z_{N-m})` (line b; Z_N = Z_0) so that the
// half-complex split runs from registers.  Output m = j + r NS of butterfly
// j has its mirror N - m = (NS - j) + (R-1-r) NS in butterfly NS - j, so one
// thread takes the butterflies {t, NS - t} for t = 1 .. NS/2-1, and the
// thread t = 0 the two self-mirrored ones {0, NS/2}.  Reads buf only.
template <typename V, bool FWD, bool BF, int N, int NB, int SM, int SB, int NTHR, typename OUT>
__device__ __forceinline__ void ct_last_stage_pairs(const V *buf, int nb, const V *tws, int tid, const OUT &out)
{
    constexpr int S = ct_nstages(N) - 1, R = ct_radix(N, S), NS = ct_ns(N, S), H = NS / 2;
    constexpr int TOTAL = H * NB;
    constexpr int ITERS = (TOTAL + NTHR - 1) / NTHR;
    static_assert(S > 0 && NS * R == N && NS % 2 == 0, "last stage of a multi-stage even transform");
    tws += ct_twoff(N, S);
    auto butterfly = [&](int base, int j, V *a) {
#pragma unroll
        for (int r = 0; r < R; r++) a[r] = buf[fpad<V>(base + (j + r * NS) * SM)];
#pragma unroll
        for (int r = 1; r < R; r++) {
            V w = tws[(r - 1) * NS + j];
            if (!FWD) w.y = -w.y;
            a[r] = cmul(a[r], w);
        }
        dft_r<V, FWD, R>(a);
    };
#pragma unroll
    for (int it = 0; it < ITERS; it++) {
        const int q = tid + it * NTHR;
        if (TOTAL % NTHR == 0 || q < TOTAL) {
            const int b = BF ? q % NB : q / H;
            const int t = BF ? q / NB : q % H;
            if (b < nb) {
                const int base = b * SB, ja = t, jb = (t == 0) ? H : NS - t;
                V xa[R], xb[R];
                butterfly(base, ja, xa);
                butterfly(base, jb, xb);
#pragma unroll
                for (int r = 0; r < R; r++) {
                    out(b, ja + r * NS, xa[r], (t == 0) ? xa[(R - r) % R] : xb[R - 1 - r]);
                    out(b, jb + r * NS, xb[r], (t == 0) ? xb[R - 1 - r] : xa[R - 1 - r]);
                }
            }
        }
    }
}

// Asynchronous global -> shared copies (cp.async; completion is awaited with
// cp.async.wait_group, a hardware wait on this thread's own copies).
__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_4(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

// Split the spectrum Z of z = a + i b (length n, even) into the two FFTW
// half-complex arrays of a and b, returned as the pair (hc_a[m], hc_b[m]).
template <typename V> __device__ __forceinline__ V split_hc(V A, V Bc, int m, int n)
{
    using T = decltype(A.x);
    V r;
    if (2 * m <= n) {
        r.x = T(0.5) * (A.x + Bc.x);
        r.y = T(0.5) * (A.y + Bc.y);
    } else {
        r.x = T(0.5) * (Bc.y - A.y);
        r.y = T(0.5) * (A.x - Bc.x);
    }
    return r;
}

// Inverse of split_hc: from the half-complex pair P = (hc_a[m], hc_b[m]) and
// Q = (hc_a[n-m], hc_b[n-m]) rebuild Z_m = A_m + i B_m.
template <typename V> __device__ __forceinline__ V merge_hc(V P, V Q, int m, int n)
{
    V z;
    if (m == 0 || 2 * m == n) {
        z = P;
    } else if (2 * m < n) {
        z.x = P.x - Q.y;
        z.y = Q.x + P.y;
    } else {
        z.x = Q.x + P.y;
        z.y = Q.y - P.x;
    }
    return z;
}

} // namespace pl
