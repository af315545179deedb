// rk_fused.cu -- both RK2 stages of timeIntVelRK1 / timeIntVelRK2
// (mod_calcVel.f90:52-146, 240-334) with their wall fills in one kernel, FP64
// (the parity path; the mixed path's kernel is rk_mixed.cu).
//
// 2.5D blocking: a CTA owns a 32 x 8 tile of (i, j) and marches up a chunk of
// k-planes.  Shared-memory rings hold the last planes of u (halo 2 in x, y)
// and of the stage-1 field (halo 1): each plane of u is read from HBM once,
// the stage-1 field u1 = u + dt*RHS(u) never leaves the SM, and the stage-2
// update is written once.  HBM traffic per point: read u, v, w and write the
// new u, v, w, instead of writing and re-reading u1, v1, w1 between two
// kernels.
//
// The rings hold u and u1 in double; the expressions are the reference's,
// in the reference's order.
#include "fft.cuh" // cp.async helpers
#include "stencil.cuh"
#include "stencil_rhs.cuh"

namespace pl {

constexpr int FX = 32, FY = 8;          // tile
constexpr int UW = FX + 4, UH = FY + 4; // ring plane with a halo of 2
constexpr int UPS = UW * UH;            // 432 values per plane

constexpr int NS = 3; // planes per ring

template <typename R> struct RingLoad {
    const R *a;
    __device__ __forceinline__ R operator()(int q) const { return a[q]; }
};

// Neighbour codes known at compile time (plane -1/0/+1, dx, dy): with the
// three per-plane base pointers of RingLoad3 every stencil read becomes a
// shared-memory load at a constant offset from one of three registers.
__host__ __device__ constexpr int ring_enc(int pl, int dx, int dy) { return (pl + 1) * 1024 + (dy + 8) * 32 + (dx + 8); }
struct RingNbC {
    static constexpr int c = ring_enc(0, 0, 0), xm = ring_enc(0, -1, 0), xp = ring_enc(0, 1, 0), ym = ring_enc(0, 0, -1),
                         yp = ring_enc(0, 0, 1), zm = ring_enc(-1, 0, 0), zp = ring_enc(1, 0, 0), xpym = ring_enc(0, 1, -1),
                         xmyp = ring_enc(0, -1, 1), xpzm = ring_enc(-1, 1, 0), xmzp = ring_enc(1, -1, 0), ypzm = ring_enc(-1, 0, 1),
                         ymzp = ring_enc(1, 0, -1);
};

template <typename R> struct RingLoad3 {
    const R *pm, *pc, *pp; // the point's element in the planes below, at and above
    __device__ __forceinline__ R operator()(int code) const
    {
        const int pl = code / 1024 - 1, dy = (code / 32) % 32 - 8, dx = code % 32 - 8;
        const R *b = pl < 0 ? pm : (pl > 0 ? pp : pc);
        return b[dx + dy * UW];
    }
};

__device__ __forceinline__ Nb32 ring_nb(int x, int y, int s0, int sm, int sp)
{
    Nb32 n;
    const int xy = y * UW + x;
    n.c = s0 * UPS + xy;
    n.xm = n.c - 1;
    n.xp = n.c + 1;
    n.ym = n.c - UW;
    n.yp = n.c + UW;
    n.zm = sm * UPS + xy;
    n.zp = sp * UPS + xy;
    n.xpym = n.c + 1 - UW;
    n.xmyp = n.c - 1 + UW;
    n.xpzm = n.zm + 1;
    n.xmzp = n.zp - 1;
    n.ypzm = n.zm + UW;
    n.ymzp = n.zp - UW;
    return n;
}

template <bool CRF>
__global__ void __launch_bounds__(FX *FY, 3) k_rk_fused(const double *__restrict__ u, const double *__restrict__ v,
                                                       const double *__restrict__ w, double *__restrict__ uo,
                                                       double *__restrict__ vo, double *__restrict__ wo, StepParams p,
                                                       MeshDev m, MeanRed red, int kchunk)
{
    using R = double;
    constexpr int FS = NS * UPS; // ring size per field
    static_assert(NS == 3, "the ring slot rotation of the march assumes three-plane rings");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *ur = reinterpret_cast<R *>(smem_raw); // u, v, w rings
    R *qr = ur + 3 * FS;                     // u1 rings
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i0 = blockIdx.x * FX, j0 = blockIdx.y * FY;
    const int kbeg = blockIdx.z * kchunk + 1, kend = min(kbeg + kchunk - 1, p.nz);
    const size_t sk = (size_t)p.nx * p.ny;
    const R dt = (R)p.dt;
    const R bcu = (R)(0.0 - p.u_crf);

    // This thread's points of a ring plane and of the stage-1 (halo-1)
    // region, fixed for the whole march.  Each warp takes 32 consecutive x of
    // one row, so its shared-memory accesses are free of bank conflicts and
    // its global loads are whole 32-element row segments; the columns left
    // over are taken four (load) or one (stage 1) per row.
    //   ring plane, 36 x 12: slot 0 = x 2..33 of rows 0..7 (warp = row);
    //     slot 1 = x 2..33 of rows 8..11 (warps 0-3), and x 0, 1, 34, 35 of
    //     rows 0..11 (warp 4 and half of warp 5: 48 points)
    //   stage-1 region, x 1..34, y 1..10: slot 0 = x 2..33 of rows 1..8;
    //     slot 1 = x 2..33 of rows 9, 10 (warps 0, 1), and x 1, 34 of rows
    //     1..10 (20 lanes of warp 2)
    static_assert(FX == 32 && FY == 8 && UW == 36 && UH == 12, "slot maps of the 32 x 8 tile");
    const int lane = tx, wid = ty;
    int loff[2], lxy[2];
    bool lval1;
    {
        int lx[2], ly[2];
        lx[0] = 2 + lane;
        ly[0] = wid;
        if (wid < 4) {
            lx[1] = 2 + lane;
            ly[1] = 8 + wid;
        } else {
            const int e = (wid - 4) * 32 + lane, c = e % 4; // e < 48 on warps 4, 5
            lx[1] = c < 2 ? c : 32 + c;
            ly[1] = min(e / 4, UH - 1);
        }
        lval1 = wid < 5 || (wid == 5 && lane < 16);
#pragma unroll
        for (int sl = 0; sl < 2; sl++) {
            int gi = i0 - 2 + lx[sl], gj = j0 - 2 + ly[sl];
            gi += (gi < 0) ? p.nx : 0;
            gi -= (gi >= p.nx) ? p.nx : 0;
            gj += (gj < 0) ? p.ny : 0;
            gj -= (gj >= p.ny) ? p.ny : 0;
            loff[sl] = gi + p.nx * gj;
            lxy[sl] = ly[sl] * UW + lx[sl];
        }
    }
    // the rings hold the fields as loaded: a plane is copied asynchronously
    // (cp.async), in flight while stage 2 runs
    auto load_u_plane_async = [&](int kq, int s) {
        const long long gk = (long long)sk * kq; // kq >= -1 (a slab's lower halo)
#pragma unroll
        for (int sl = 0; sl < 2; sl++) {
            if (sl == 0 || lval1) {
                const long long g = gk + loff[sl];
                const int q = s * UPS + lxy[sl];
                cp_async_8(ur + 0 * FS + q, u + g);
                cp_async_8(ur + 1 * FS + q, v + g);
                cp_async_8(ur + 2 * FS + q, w + g);
            }
        }
        cp_async_commit();
    };

    int hxy[2];
    bool hval1;
    hxy[0] = (1 + wid) * UW + 2 + lane;
    if (wid < 2)
        hxy[1] = (9 + wid) * UW + 2 + lane;
    else
        hxy[1] = (1 + lane % 10) * UW + (lane < 10 ? 1 : 34);
    hval1 = wid < 2 || (wid == 2 && lane < 20);
    constexpr int HSLOTS = 2;

    // ring slots sm, s0, sp of the planes mq-1, mq, mq+1
    auto produce = [&](int mq, int sm, int s0, int sp, const RhsConst<R> &cst) {
#pragma unroll
        for (int sl = 0; sl < HSLOTS; sl++) {
            if (sl == 1 && !hval1) break;
            const int xy = hxy[sl];
            const int om = sm * UPS + xy, oc = s0 * UPS + xy, op = sp * UPS + xy;
            R ru, rv, rw;
            momentum_rhs_c<R, CRF>(RingLoad3<R>{ur + om, ur + oc, ur + op},
                                   RingLoad3<R>{ur + FS + om, ur + FS + oc, ur + FS + op},
                                   RingLoad3<R>{ur + 2 * FS + om, ur + 2 * FS + oc, ur + 2 * FS + op}, RingNbC{}, cst,
                                   ru, rv, rw);
            // u1 = u + dt*(visc - conv); w1(nz) = 0, the wall
            qr[oc] = ur[oc] + dt * (ru + (R)p.fb[0]);
            qr[FS + oc] = ur[FS + oc] + dt * (rv + (R)p.fb[1]);
            qr[2 * FS + oc] = (p.whi && mq == p.nz) ? (R)0 : ur[2 * FS + oc] + dt * (rw + (R)p.fb[2]);
        }
    };

    // imposeNoSlipBC on the stage-1 field: plane kg from plane ki (0 <- 1, nz+1 <- nz)
    auto wall = [&](int kg, int ki) {
        const int sg = kg % NS, si = ki % NS;
#pragma unroll
        for (int sl = 0; sl < HSLOTS; sl++) {
            if (sl == 1 && !hval1) break;
            const int xy = hxy[sl];
            qr[sg * UPS + xy] = (R)2 * bcu - qr[si * UPS + xy];
            qr[FS + sg * UPS + xy] = -qr[FS + si * UPS + xy];
            qr[2 * FS + sg * UPS + xy] = (R)0;
        }
    };

    double su = 0.0;
    // stage 2 at interior plane kq from the stage-1 planes kq-1, kq, kq+1
    auto stage2 = [&](int kq, int sm, int s0, int sp, const RhsConst<R> &cst) {
        const Nb32 n = ring_nb(tx + 2, ty + 2, s0, sm, sp);
        // global loads first, so their latency overlaps the stencil
        const size_t g = (size_t)(i0 + tx) + (size_t)p.nx * (j0 + ty) + sk * kq;
        const double uc = __ldg(u + g), vc = __ldg(v + g), wc = __ldg(w + g);
        R ru, rv, rw;
        {
            const int xy = (ty + 2) * UW + tx + 2;
            const int om = sm * UPS + xy, oc = s0 * UPS + xy, op = sp * UPS + xy;
            const R *b = qr;
            momentum_rhs_c<R, CRF>(RingLoad3<R>{b + om, b + oc, b + op},
                                   RingLoad3<R>{b + FS + om, b + FS + oc, b + FS + op},
                                   RingLoad3<R>{b + 2 * FS + om, b + 2 * FS + oc, b + 2 * FS + op}, RingNbC{}, cst, ru,
                                   rv, rw);
        }
        const double nu = ((double)qr[n.c] + p.dt * ((double)ru + p.fb[0]) + uc) * 0.5;
        const double nv = ((double)qr[FS + n.c] + p.dt * ((double)rv + p.fb[1]) + vc) * 0.5;
        const double nw = ((double)qr[2 * FS + n.c] + p.dt * ((double)rw + p.fb[2]) + wc) * 0.5;
        uo[g] = nu;
        vo[g] = nv;
        if (kq != p.nz || !p.whi) wo[g] = nw;
        wall_fill<double>(uo, vo, wo, g, kq, sk, p.nz, 0.0 - p.u_crf, nu, nv, p.wlo, p.whi);
        su += nu * __ldg(m.dzflzi + kq);
    };

    // Two barriers per plane: produce(mq) reads u planes mq-1..mq+1; then
    // stage2(mq-1), which reads only the stage-1 rings and global memory,
    // runs together with the load of u plane mq+2 into the slot of plane
    // mq-1 that produce(mq) has finished with, so the load's latency hides
    // behind the stage-2 arithmetic.
    //
    // The mesh constants of plane mq (cur) and mq-1 (prev) roll in
    // registers: moving up one plane loads three values, dzf(mq+2),
    // dzc_inv(mq+1) and dzf_inv(mq+2), instead of all eleven per evaluation.
    // stage 1 runs one plane beyond the chunk, but not on a wall plane
    // (whose u1 is the wall fill); at a slab interface it runs on the halo
    const int mstart = max(kbeg - 1, p.wlo ? 1 : 0), mend = min(kend + 1, p.whi ? p.nz : p.nz + 1);
    RhsConst<R> cur = rhs_const<R>(p, m, mstart), prev = cur; // prev is unused until mq = mstart + 1
    // ring slots of the planes mq-1, mq, mq+1, rotated once per plane
    // ring slot of plane k: (k + NS) % NS (k >= -1 at a slab interface)
    int sa = (mstart - 1 + NS) % NS, sb = mstart % NS, sc = (mstart + 1) % NS;
    load_u_plane_async(mstart - 1, sa);
    load_u_plane_async(mstart, sb);
    load_u_plane_async(mstart + 1, sc);
    cp_async_wait<0>();
    __syncthreads();
    for (int mq = mstart; mq <= mend; mq++) {
        produce(mq, sa, sb, sc, cur);
        __syncthreads();
        const bool next = mq + 2 <= mend + 1;
        // the copy of u plane mq+2 into the slot of plane mq-1 (which
        // nothing reads after produce(mq)) overlaps stage 2
        if (next) load_u_plane_async(mq + 2, sa);
        if (p.wlo && mq == 1) {
            wall(0, 1);
            __syncthreads();
        }
        // plane mq-2 sits in slot sc
        if (mq - 1 >= kbeg && mq - 1 <= kend) stage2(mq - 1, sc, sa, sb, prev);
        if (p.whi && mq == p.nz) {
            // the top wall plane reuses the ring slot of u1(nz-2), which
            // stage2(nz-1) above has just consumed
            __syncthreads();
            wall(p.nz + 1, p.nz);
            __syncthreads();
            if (p.nz >= kbeg && p.nz <= kend) stage2(p.nz, sa, sb, sc, cur);
        }
        if (next) cp_async_wait<0>(); // (mq + 2) % 3 == (mq - 1) % 3
        if (mq < mend) { // constants of plane mq + 1 <= nz: indices up to mq + 2 <= nz + 1
            prev = cur;
            cur.dzf_km = cur.dzf_k;
            cur.dzf_k = cur.dzf_kp;
            cur.dzf_kp = (R)__ldg(m.dzf + mq + 2);
            cur.dzci_km = cur.dzci_k;
            cur.dzci_k = (R)__ldg(m.dzc_inv + mq + 1);
            cur.dzfi_k = cur.dzfi_kp;
            cur.dzfi_kp = (R)__ldg(m.dzf_inv + mq + 2);
        }
        const int st = sa;
        sa = sb;
        sb = sc;
        sc = st;
        __syncthreads();
    }
    mean_reduce(su, red);
}

// z-chunks per tile column.  Measured on B200 at 512x384x256 (1.35-1.44 ms
// over 3..16 chunks, both paths fastest at 5): chunks of about 52 planes.
// A grid whose tiles x chunks would not fill one wave of resident CTAs takes
// more chunks, down to 16 planes each.
static int fused_chunks(const StepParams &p, long resident)
{
    const int tiles = (p.nx / FX) * (p.ny / FY);
    const int maxch = p.nz / 16 > 1 ? p.nz / 16 : 1;
    int nch = (p.nz + 26) / 52;
    if (nch < 1) nch = 1;
    while (nch < maxch && (long)tiles * nch < resident) nch++;
    return nch < maxch ? nch : maxch;
}

bool rk_fused_supported(const StepParams &p) { return p.nx % FX == 0 && p.ny % FY == 0 && p.nz >= 2; }

// an upper bound of the launch's CTA count (fused_chunks never exceeds nz/16)
int rk_fused_blocks(const StepParams &p) { return (p.nx / FX) * (p.ny / FY) * (p.nz / 16 > 1 ? p.nz / 16 : 1); }

static int sm_count_rk()
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

int launch_rk_fused_fp64(const double *u, const double *v, const double *w, double *uo, double *vo, double *wo,
                         const StepParams &p, const MeshDev &m, MeanState &ms, cudaStream_t st)
{
    if (!rk_fused_supported(p)) {
        set_error("fused RK kernel needs nx % 32 == 0 and ny % 8 == 0");
        return -1;
    }
    const size_t shm = sizeof(double) * 6 * NS * UPS;
    // u_crf == 0 (the channel's usual frame) drops the frame-velocity terms
    auto kern = (p.u_crf != 0.0) ? k_rk_fused<true> : k_rk_fused<false>;
    PL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    // prefer the largest shared-memory carve-out: several CTAs per SM
    PL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, FX * FY, shm) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int nch = fused_chunks(p, (long)per_sm * sm_count_rk());
    const int kchunk = (p.nz + nch - 1) / nch;
    dim3 grid(p.nx / FX, p.ny / FY, (p.nz + kchunk - 1) / kchunk);
    if ((int)(grid.x * grid.y * grid.z) > ms.max_blocks) {
        set_error("mean buffer too small for the fused RK kernel");
        return -1;
    }
    MeanRed r{ms.partial, ms.counter, ms.scalar, (double)p.nx, (double)p.ny, ms.vel_force};
    kern<<<grid, dim3(FX, FY), shm, st>>>(u, v, w, uo, vo, wo, p, m, r, kchunk);
    PL_CHECK_LAUNCH();
    return 0;
}

} // namespace pl
