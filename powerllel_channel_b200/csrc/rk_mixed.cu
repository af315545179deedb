// rk_mixed.cu -- the mixed-precision path's fused RK2 kernel: both stages of
// timeIntVelRK1 / timeIntVelRK2 (mod_calcVel.f90:52-146, 240-334) with their
// wall fills, in FP32 flux form.
//
// 2.5D blocking as in the FP64 kernel (rk_fused.cu), on a 32 x 16 tile of
// (i, j) whose 256 threads own two y-adjacent points each: a CTA marches up a
// chunk of k-planes; shared-memory rings hold
// the last three planes of u, v, w (FP32, halo 2) and of the stage-1 field
// u1 = u + d1 (FP32, halo 1); HBM sees u, v, w read once, the new fields
// written once and the FP32 pressure prediction read once.  The FP64 planes
// arrive through a three-slot staging ring filled by 16-byte cp.async copies
// two planes ahead of their conversion to FP32, so no load latency and no
// extra barrier sits on the march's critical path.
//
// The kernel is bound by instruction issue, not by HBM, so its layout
// serves the instruction count: the march is unrolled by three, so every
// ring slot is a compile-time constant and every ring access one base
// register plus an immediate; a thread's two points are evaluated in packed
// FP32 pairs (one two-lane instruction for both points, each lane rounded as
// the scalar operation); every thread copies the same two (row, column)
// pairs of the three fields, so the copy map costs four registers.
//
// The arithmetic is the reference's stencil rearranged into fluxes, which
// the FP64 path (the parity path) does not do:
//   * every convective edge product is formed once per point and serves the
//     two equations that share the edge: (u_c + u_yp)(v_c + v_xp) is the
//     north flux of u and the east flux of v (:84 un*vn, :107 ue*ve); the
//     u-to-w-face interpolation times (w_c + w_xp) is the top flux of u and
//     the east flux of w (:85 ut*wt, :129 ue*we); likewise v and w;
//   * the top fluxes of plane k are the bottom fluxes of plane k+1, so they
//     ride in registers up the march instead of being recomputed;
//   * (q_c + q_xp)^2 - (q_xm + q_c)^2 = (q_xp - q_xm)(q_xp + q_xm + 2 q_c), and
//     the viscous terms are one five-point combination per direction with
//     dt, 0.25, 1/Re and the mesh factors folded into per-plane coefficients;
//   * each thread evaluates its two points together, point B's terms being
//     point A's one row up: the pair's south fluxes are (A's south, A's
//     north), so no value crosses between the lanes of a pair;
//   * the stage-1 increment d1 = dt RHS(u) of the tile's own points stays in
//     the thread's registers from stage 1 of plane k to stage 2 of plane k
//     (the thread that forms it consumes it), so only u1 goes through
//     shared memory.
// About 70 FP32 operations and 25 shared-memory loads per stencil
// evaluation, against about 135 and 27 for the reference's form.
//
// Stage 2 forms u_hat = u + [ (d1 + d2)/2 - dt G p_pred ] with the bracket in
// FP32 and the sum in FP64: u, v, w stay FP64, and the projection residual of
// the increment solve is the FP64 divergence of the stored u_hat, whatever
// rounding the bracket carries.
#include <type_traits>
#include <vector>

#include "fft.cuh" // cp.async helpers
#include "stencil.cuh"
#include "stencil_rhs.cuh"

namespace pl {

namespace {

constexpr int MX = 32, MY = 16;         // tile; each thread owns the points (x, 2t) and (x, 2t+1)
constexpr int MW = MX + 4, MH = MY + 4; // ring plane with a halo of 2
constexpr int MPS = MW * MH;            // 720 values per plane
constexpr int MNS = 3;                  // planes per ring
constexpr int FST = MPS;                // ring layout [slot][field][xy]: field stride
constexpr int SST = 3 * MPS;            // ... and plane (slot) stride
constexpr int MT = 256;                 // threads
constexpr int MX_KCHUNK = 80;           // longest z-chunk (planes)

// rolling top fluxes of one point: E_uw(k+1/2), E_vw(k+1/2) and (w_k + w_{k+1})^2
struct Carry {
    float euw, evw, cw;
};

// the top fluxes of plane k at one point from the planes k (oc) and k+1 (op)
// of a ring (u, v, w at R, R + FST, R + 2 FST); a, b: plane k's weights of
// the face interpolation q_{k+1/2} = q_k a + q_{k+1} b
__device__ __forceinline__ Carry mx_top(const float *R, int oc, int op, float a, float b)
{
    const float *u = R, *v = R + FST, *w = R + 2 * FST;
    Carry c;
    const float wc = w[oc];
    c.euw = (u[oc] * a + u[op] * b) * (wc + w[oc + 1]);
    c.evw = (v[oc] * a + v[op] * b) * (wc + w[oc + MW]);
    const float wt = wc + w[op];
    c.cw = wt * wt;
    return c;
}

// dt * (momentum right-hand side) at one point from the planes k-1 (om), k
// (oc), k+1 (op) of a ring; cy holds the bottom fluxes on entry and the top
// fluxes on return.  Plane coefficients (dt folded in, MxPlane): a, b face
// weights; hzuv = dt/4 dzf_inv(k); azp, azm = dt/Re dzf_inv(k) dzc_inv(k),
// dzc_inv(k-1); ccuv = 2 cxx + 2 cyy + azp + azm; hzw = dt/4 dzc_inv(k);
// bzp, bzm = dt/Re dzc_inv(k) dzf_inv(k+1), dzf_inv(k); ccw likewise.
template <bool CRF>
__device__ __forceinline__ void mx_rhs(const float *R, int om, int oc, int op, const MxPlane &P, const MxConst &K,
                                       Carry &cy, float &du, float &dv, float &dw)
{
    const float *u = R, *v = R + FST, *w = R + 2 * FST;
    const float uc = u[oc], uxp = u[oc + 1], uxm = u[oc - 1], uyp = u[oc + MW], uym = u[oc - MW];
    const float uzp = u[op], uzm = u[om], uxmyp = u[oc - 1 + MW], uxmzp = u[op - 1];
    const float vc = v[oc], vxp = v[oc + 1], vxm = v[oc - 1], vyp = v[oc + MW], vym = v[oc - MW];
    const float vzp = v[op], vzm = v[om], vxpym = v[oc + 1 - MW], vymzp = v[op - MW];
    const float wc = w[oc], wxp = w[oc + 1], wxm = w[oc - 1], wyp = w[oc + MW], wym = w[oc - MW];
    const float wzp = w[op], wzm = w[om];

    // edge fluxes (products of face sums), each shared by two equations
    const float euv_n = (uc + uyp) * (vc + vxp);                // (i+1/2, j+1/2): u north, v east
    const float euv_s = (uym + uc) * (vym + vxpym);             // (i+1/2, j-1/2): u south
    const float euv_w = (uxm + uxmyp) * (vxm + vc);             // (i-1/2, j+1/2): v west
    const float euw_t = (uc * P.a + uzp * P.b) * (wc + wxp);    // (i+1/2, k+1/2): u top, w east
    const float euw_w = (uxm * P.a + uxmzp * P.b) * (wxm + wc); // (i-1/2, k+1/2): w west
    const float evw_t = (vc * P.a + vzp * P.b) * (wc + wyp);    // (j+1/2, k+1/2): v top, w north
    const float evw_s = (vym * P.a + vymzp * P.b) * (wym + wc); // (j-1/2, k+1/2): w south
    const float wt = wc + wzp;
    const float cw_t = wt * wt;

    // u: x self-flux difference (u_xp - u_xm)(u_xp + u_xm + 2 u_c)
    const float sxu = uxp + uxm, syu = uyp + uym, dxu = uxp - uxm;
    float r = K.cxx * sxu;
    r = fmaf(K.cyy, syu, r);
    r = fmaf(P.azp, uzp, r);
    r = fmaf(P.azm, uzm, r);
    r = fmaf(-P.ccuv, uc, r);
    r = fmaf(-K.hx, dxu * fmaf(2.f, uc, sxu), r);
    r = fmaf(-K.hy, euv_n - euv_s, r);
    r = fmaf(-P.hzuv, euw_t - cy.euw, r);
    if (CRF) r = fmaf(-K.ucx, dxu, r);
    du = r;

    // v: y self-flux difference
    const float sxv = vxp + vxm, syv = vyp + vym, dyv = vyp - vym;
    r = K.cxx * sxv;
    r = fmaf(K.cyy, syv, r);
    r = fmaf(P.azp, vzp, r);
    r = fmaf(P.azm, vzm, r);
    r = fmaf(-P.ccuv, vc, r);
    r = fmaf(-K.hx, euv_n - euv_w, r);
    r = fmaf(-K.hy, dyv * fmaf(2.f, vc, syv), r);
    r = fmaf(-P.hzuv, evw_t - cy.evw, r);
    if (CRF) r = fmaf(-K.ucx, vxp - vxm, r);
    dv = r;

    // w: z self-flux from the carried bottom square
    const float sxw = wxp + wxm, syw = wyp + wym;
    r = K.cxx * sxw;
    r = fmaf(K.cyy, syw, r);
    r = fmaf(P.bzp, wzp, r);
    r = fmaf(P.bzm, wzm, r);
    r = fmaf(-P.ccw, wc, r);
    r = fmaf(-K.hx, euw_t - euw_w, r);
    r = fmaf(-K.hy, evw_t - evw_s, r);
    r = fmaf(-P.hzw, cw_t - cy.cw, r);
    if (CRF) r = fmaf(-K.ucx, wxp - wxm, r);
    dw = r;

    cy.euw = euw_t;
    cy.evw = evw_t;
    cy.cw = cw_t;
}

// plane k's coefficients from the chunk's copy in shared memory (tab points
// at the first plane of the chunk's copy, k relative to it)
__device__ __forceinline__ MxPlane mx_plane(const float4 *tab, int k)
{
    const float4 x = tab[3 * k], y = tab[3 * k + 1], z = tab[3 * k + 2];
    MxPlane P;
    P.a = x.x;
    P.b = x.y;
    P.hzuv = x.z;
    P.azp = x.w;
    P.azm = y.x;
    P.ccuv = y.y;
    P.hzw = y.z;
    P.bzp = y.w;
    P.bzm = z.x;
    P.ccw = z.y;
    P.gz = z.z;
    return P;
}


// Packed FP32 pairs (Blackwell's two-lane FP32 instructions, each lane
// rounded as the scalar operation): .x belongs to point A, .y to point B.
typedef float2 f2;
__device__ __forceinline__ f2 add2(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 sub2(f2 a, f2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ f2 mul2(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 bc2(float s) { return make_float2(s, s); }
// values at offsets o (point A) and o + MW (point B) of a ring field
__device__ __forceinline__ f2 ld2(const float *q, int o) { return make_float2(q[o], q[o + MW]); }

// the carried top fluxes of the pair
struct Carry2 {
    f2 euw, evw, cw;
};

// dt * (momentum right-hand side) at the points A (oc) and B = A + y (oc + MW)
// of a ring in packed pairs.  Every term of B is its term of A one row up,
// so each pair is two loads one row apart: B's south fluxes (A's north
// ones) come out of the pair (south of A, north of A), with no exchange
// between the lanes.  cy: the pair's carried bottom fluxes (top fluxes on
// return); du, dv, dw: the pair's increments.
template <bool CRF>
__device__ __forceinline__ void mx_rhs2(const float *R, int om, int oc, int op, const MxPlane &P, const MxConst &K,
                                        Carry2 &cy, f2 &du, f2 &dv, f2 &dw)
{
    const float *u = R, *v = R + FST, *w = R + 2 * FST;
    const f2 uC = ld2(u, oc), uYP = ld2(u, oc + MW), uYM = ld2(u, oc - MW);
    const f2 uXP = ld2(u, oc + 1), uXM = ld2(u, oc - 1), uXMYP = ld2(u, oc - 1 + MW);
    const f2 uZP = ld2(u, op), uZM = ld2(u, om), uXMZP = ld2(u, op - 1);
    const f2 vC = ld2(v, oc), vYP = ld2(v, oc + MW), vYM = ld2(v, oc - MW);
    const f2 vXP = ld2(v, oc + 1), vXM = ld2(v, oc - 1), vXPYM = ld2(v, oc + 1 - MW);
    const f2 vZP = ld2(v, op), vZM = ld2(v, om), vYMZP = ld2(v, op - MW);
    const f2 wC = ld2(w, oc), wYP = ld2(w, oc + MW), wYM = ld2(w, oc - MW);
    const f2 wXP = ld2(w, oc + 1), wXM = ld2(w, oc - 1), wZP = ld2(w, op), wZM = ld2(w, om);
    const f2 a = bc2(P.a), b = bc2(P.b);

    // edge fluxes: (A, B) of the north, south, west, top faces
    const f2 euv_n = mul2(add2(uC, uYP), add2(vC, vXP));
    const f2 euv_s = mul2(add2(uYM, uC), add2(vYM, vXPYM)); // (south of A, north of A)
    const f2 euv_w = mul2(add2(uXM, uXMYP), add2(vXM, vC));
    const f2 euw_t = mul2(fma2(uC, a, mul2(uZP, b)), add2(wC, wXP));
    const f2 euw_w = mul2(fma2(uXM, a, mul2(uXMZP, b)), add2(wXM, wC));
    const f2 evw_t = mul2(fma2(vC, a, mul2(vZP, b)), add2(wC, wYP));
    const f2 evw_s = mul2(fma2(vYM, a, mul2(vYMZP, b)), add2(wYM, wC)); // (south of A, top of A)
    const f2 wt = add2(wC, wZP);
    const f2 cw_t = mul2(wt, wt);

    const f2 cxx = bc2(K.cxx), cyy = bc2(K.cyy), nhx = bc2(-K.hx), nhy = bc2(-K.hy);
    f2 r;
    {
        const f2 sx = add2(uXP, uXM), sy = add2(uYP, uYM), dx = sub2(uXP, uXM);
        r = mul2(cxx, sx);
        r = fma2(cyy, sy, r);
        r = fma2(bc2(P.azp), uZP, r);
        r = fma2(bc2(P.azm), uZM, r);
        r = fma2(bc2(-P.ccuv), uC, r);
        r = fma2(nhx, mul2(dx, fma2(bc2(2.f), uC, sx)), r);
        r = fma2(nhy, sub2(euv_n, euv_s), r);
        r = fma2(bc2(-P.hzuv), sub2(euw_t, cy.euw), r);
        if (CRF) r = fma2(bc2(-K.ucx), dx, r);
        du = r;
    }
    {
        const f2 sx = add2(vXP, vXM), sy = add2(vYP, vYM), dy = sub2(vYP, vYM);
        r = mul2(cxx, sx);
        r = fma2(cyy, sy, r);
        r = fma2(bc2(P.azp), vZP, r);
        r = fma2(bc2(P.azm), vZM, r);
        r = fma2(bc2(-P.ccuv), vC, r);
        r = fma2(nhx, sub2(euv_n, euv_w), r);
        r = fma2(nhy, mul2(dy, fma2(bc2(2.f), vC, sy)), r);
        r = fma2(bc2(-P.hzuv), sub2(evw_t, cy.evw), r);
        if (CRF) r = fma2(bc2(-K.ucx), sub2(vXP, vXM), r);
        dv = r;
    }
    {
        const f2 sx = add2(wXP, wXM), sy = add2(wYP, wYM);
        r = mul2(cxx, sx);
        r = fma2(cyy, sy, r);
        r = fma2(bc2(P.bzp), wZP, r);
        r = fma2(bc2(P.bzm), wZM, r);
        r = fma2(bc2(-P.ccw), wC, r);
        r = fma2(nhx, sub2(euw_t, euw_w), r);
        r = fma2(nhy, sub2(evw_t, evw_s), r);
        r = fma2(bc2(-P.hzw), sub2(cw_t, cy.cw), r);
        if (CRF) r = fma2(bc2(-K.ucx), sub2(wXP, wXM), r);
        dw = r;
    }
    cy.euw = euw_t;
    cy.evw = evw_t;
    cy.cw = cw_t;
}
} // namespace

template <bool CRF>
__global__ void __launch_bounds__(MT, 2) k_rk_mixed(const double *__restrict__ u, const double *__restrict__ v,
                                                   const double *__restrict__ w, double *__restrict__ uo,
                                                   double *__restrict__ vo, double *__restrict__ wo, StepParams p,
                                                   MeshDev m, const float4 *__restrict__ tab, MxConst K, MeanRed red,
                                                   int kchunk, const float *__restrict__ pq, int pinc)
{
    constexpr int NSTG = 3; // FP64 staging slots
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *stg = reinterpret_cast<double *>(smem_raw);    // FP64 staging, [slot][field][MPS]
    float *ur = reinterpret_cast<float *>(stg + NSTG * SST); // u, v, w rings, [plane slot][field][MPS]
    float *sr = ur + 3 * SST;                               // u1 = u + d1 rings
    // the chunk's plane coefficients (planes kbeg - 2 .. kbeg + kchunk + 1,
    // 3 float4 each) and dzf/lz: used every plane, so they live on chip
    // instead of in global loads whose latency would sit on the march
    float4 *ptab = reinterpret_cast<float4 *>(sr + 3 * SST);
    double *pzl = reinterpret_cast<double *>(ptab + 3 * (kchunk + 4));
    const int lane = threadIdx.x, wid = threadIdx.y;
    const int i0 = blockIdx.x * MX, j0 = blockIdx.y * MY;
    const int kbeg = blockIdx.z * kchunk + 1, kend = min(kbeg + kchunk - 1, p.nz);
    const size_t sk = (size_t)p.nx * p.ny;
    const int tid = lane + MX * wid;

    // Ring-plane loads (36 x 20 of u, v, w): 360 aligned pairs of doubles
    // per field and plane, pair q = row r, x pair c (q = 18 r + c); thread t
    // copies pair t of every field and, for t >= 152, pair t + 104 (warps
    // 0-3 carry the halo stencil instead).  Each pair is one 16-byte copy
    // (cp.async.cg: L2 only, no L1 pollution) into the FP64 staging slot, and
    // one 16-byte shared load, two conversions and an 8-byte store into the
    // FP32 ring, at the same offset within the slot.  The pair's position in
    // the plane (periodic in x and y; a pair never straddles the wrap, nx
    // being even) and in the slot are the same for the three fields and fixed
    // for the whole march.
    static_assert(MX == 32 && MY == 16 && MW == 36 && MH == 20, "pair maps of the 32 x 16 tile");
    constexpr int FPAIR = MH * (MW / 2), PAIR2 = MT - (FPAIR - MT); // 360 pairs per field; 152
    int soff[2], pk[2]; // the pair's element offset in a plane and its offset in a ring field
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int q = h == 0 ? tid : (tid >= PAIR2 ? tid + (FPAIR - MT) : 0);
        const int r = q / 18, c = q % 18;
        int gx = i0 - 2 + 2 * c, gy = j0 - 2 + r;
        gx += (gx < 0) ? p.nx : 0;
        gx -= (gx >= p.nx) ? p.nx : 0;
        gy += (gy < 0) ? p.ny : 0;
        gy -= (gy >= p.ny) ? p.ny : 0;
        soff[h] = gy * p.nx + gx;
        pk[h] = r * MW + 2 * c;
    }
    const bool pv2 = tid >= PAIR2;

    // Slots: plane k of the march sits in slot (k - mstart + 1) % 3 of the
    // staging ring and of both FP32 rings, so that with the march unrolled by
    // three every slot is a compile-time constant and every ring access one
    // per-thread base address plus an immediate offset.
    // copy u, v, w plane kq (in [-1, nz+2]; none past last) into staging
    // slot `slot`; one commit group per call, empty or not, so the wait counts
    // stay uniform
    auto issue = [&](int kq, int last, int slot) {
        if (kq <= last) {
            const long long off = (long long)sk * kq; // kq >= -1 (a slab's lower halo)
            double *d = stg + slot * SST;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                if (h == 0 || pv2) {
                    const long long o = off + soff[h];
                    cp_async_16(d + pk[h], u + o);
                    cp_async_16(d + FST + pk[h], v + o);
                    cp_async_16(d + 2 * FST + pk[h], w + o);
                }
            }
        }
        cp_async_commit();
    };

    // staging slot s (every thread's copies landed and a barrier passed) ->
    // FP32 ring slot s
    auto convert = [&](int s) {
        const double *d = stg + s * SST;
        float *o = ur + s * SST;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            if (h == 0 || pv2) {
#pragma unroll
                for (int f = 0; f < 3; f++) {
                    const double2 x = *reinterpret_cast<const double2 *>(d + f * FST + pk[h]);
                    *reinterpret_cast<float2 *>(o + f * FST + pk[h]) = make_float2((float)x.x, (float)x.y);
                }
            }
        }
    };

    // stage-1 points (halo-1 region, x 1..34, y 1..18 of the ring plane):
    // the pair = the thread's own points (x 2 + lane, y 2 + 2 wid and the row
    // above: its stage-2 points); the halo = rows 1 and 18 (warps 0, 1) and
    // columns 1, 34 of rows 1..18 (warp 2 and 4 lanes of warp 3)
    const int hxy0 = (2 + 2 * wid) * MW + 2 + lane;
    int hxy1;
    if (wid < 2) {
        hxy1 = (wid == 0 ? 1 : 18) * MW + 2 + lane;
    } else {
        const int e = (wid - 2) * 32 + lane; // < 36 on the valid lanes
        hxy1 = (1 + e % 18) * MW + (e < 18 ? 1 : 34);
    }
    const bool hval1 = wid < 3 || (wid == 3 && lane < 4);

    // the global points of the thread's stage-2 pair and their
    // pressure-prediction neighbours (+x, +y periodic)
    const int gi = i0 + lane, gjA = j0 + 2 * wid;
    const int gxp = (gi == p.nx - 1) ? 0 : gi + 1, gjB2 = (gjA + 2 >= p.ny) ? gjA + 2 - p.ny : gjA + 2;
    const size_t gA = (size_t)gi + (size_t)p.nx * gjA;

    // stage 1 runs one plane beyond the chunk, but not on a wall plane:
    // under the top wall the march's step at nz+1 forms the wall plane of u1
    // instead; at a slab interface stage 1 runs on the halo
    const int mstart = max(kbeg - 1, p.wlo ? 1 : 0), mend = min(kend + 1, p.nz + 1);
    const bool wall_step = p.whi && mend == p.nz + 1;
    const int last = wall_step ? p.nz + 1 : mend + 1; // the last u plane the march reads
    {
        const int k0 = max(kbeg - 2, p.wlo ? 0 : -1), np = min(kbeg + kchunk + 1, p.nz + (p.whi ? 1 : 2)) - k0 + 1;
        for (int q = tid; q < 3 * np; q += MT) ptab[q] = __ldg(tab + 3 * k0 + q);
        for (int q = tid; q < np; q += MT) pzl[q] = __ldg(m.dzflzi + k0 + q);
        ptab -= 3 * k0; // indexable by the global plane
        pzl -= k0;
    }
    // a plane is issued two iterations before its conversion at the end of
    // an iteration
    issue(mstart - 1, last, 0);
    issue(mstart, last, 1);
    issue(mstart + 1, last, 2);
    cp_async_wait<0>();
    __syncthreads();
    convert(0);
    convert(1);
    convert(2);
    __syncthreads();
    issue(mstart + 2, last, 0); // into the staging slots of mstart - 1 and mstart, converted above
    issue(mstart + 3, last, 1);
    cp_async_wait<1>(); // plane mstart + 2 landed; the barrier below publishes it
    __syncthreads();

    // bottom fluxes of the first stage-1 plane (the top fluxes of mstart - 1)
    const Carry zero = {0.f, 0.f, 0.f};
    auto pair = [](const Carry &x, const Carry &y) {
        return Carry2{make_float2(x.euw, y.euw), make_float2(x.evw, y.evw), make_float2(x.cw, y.cw)};
    };
    Carry cH;
    Carry2 c1, c2 = pair(zero, zero);
    {
        const MxPlane Pm = mx_plane(ptab, mstart - 1);
        c1 = pair(mx_top(ur, hxy0, SST + hxy0, Pm.a, Pm.b), mx_top(ur, hxy0 + MW, SST + hxy0 + MW, Pm.a, Pm.b));
        cH = hval1 ? mx_top(ur, hxy1, SST + hxy1, Pm.a, Pm.b) : zero;
    }
    // d1 of the own pair (u, v, w; .x point A, .y point B) at plane mq (this
    // iteration) and at mq - 1
    f2 d1[3] = {bc2(0.f), bc2(0.f), bc2(0.f)}, e1[3] = {bc2(0.f), bc2(0.f), bc2(0.f)};
    bool first2 = true;
    double su = 0.0;
    const float bcu2 = (float)(2.0 * (0.0 - p.u_crf));

    // the stage-2 centre values of the pair at plane kq: u, v, w (FP64) and
    // the pressure prediction at A, B and their +x, +y, +z neighbours (A's +y
    // neighbour is B)
    struct Centre {
        double u[2], v[2], w[2];
        float qA, qB, qxA, qxB, qyB, qzA, qzB;
    };
    auto centre = [&](int kq) {
        Centre c;
        const size_t g = gA + sk * kq;
        c.u[0] = __ldg(u + g);
        c.u[1] = __ldg(u + g + p.nx);
        c.v[0] = __ldg(v + g);
        c.v[1] = __ldg(v + g + p.nx);
        c.w[0] = __ldg(w + g);
        c.w[1] = __ldg(w + g + p.nx);
        const size_t pl = sk * (kq - 1);
        const size_t rowA = (size_t)p.nx * gjA + pl, rowB = rowA + p.nx, rowB2 = (size_t)p.nx * gjB2 + pl;
        c.qA = c.qB = c.qxA = c.qxB = c.qyB = c.qzA = c.qzB = 0.f;
        if (pinc) {
            c.qA = __ldg(pq + rowA + gi);
            c.qB = __ldg(pq + rowB + gi);
            c.qxA = __ldg(pq + rowA + gxp);
            c.qxB = __ldg(pq + rowB + gxp);
            c.qyB = __ldg(pq + rowB2 + gi);
            c.qzA = (kq < p.nz) ? __ldg(pq + rowA + sk + gi) : c.qA;
            c.qzB = (kq < p.nz) ? __ldg(pq + rowB + sk + gi) : c.qB;
        }
        return c;
    };

    // the pressure-prediction lines of centre(kq) into L1 ahead of their
    // loads, which follow the barrier (a prefetch holds no registers)
    auto pf = [](const void *a) { asm volatile("prefetch.global.L1 [%0];" ::"l"(a)); };
    auto prefetch = [&](int kq) {
        if (pinc) {
            const size_t pl = sk * (kq - 1);
            const size_t rowA = (size_t)p.nx * gjA + pl, rowB = rowA + p.nx, rowB2 = (size_t)p.nx * gjB2 + pl;
            pf(pq + rowA + gi);
            pf(pq + rowB + gi);
            pf(pq + rowA + gxp);
            pf(pq + rowB + gxp);
            pf(pq + rowB2 + gi);
            if (kq < p.nz) {
                pf(pq + rowA + sk + gi);
                pf(pq + rowB + sk + gi);
            }
        }
    };

    // stage 2 at interior plane kq from the stage-1 planes kq-1 (sm), kq (s0),
    // kq+1 (sp); e: the pair's d1 at kq
    auto stage2 = [&](int kq, int sm, int s0, int sp, const f2 *e, const Centre &cv) {
        const MxPlane P = mx_plane(ptab, kq);
        if (first2) { // bottom fluxes of u1 at kq: the top fluxes of plane kq - 1
            const MxPlane Pm = mx_plane(ptab, kq - 1);
            c2 = pair(mx_top(sr, sm * SST + hxy0, s0 * SST + hxy0, Pm.a, Pm.b),
                      mx_top(sr, sm * SST + hxy0 + MW, s0 * SST + hxy0 + MW, Pm.a, Pm.b));
            first2 = false;
        }
        f2 d[3];
        mx_rhs2<CRF>(sr, sm * SST + hxy0, s0 * SST + hxy0, sp * SST + hxy0, P, K, c2, d[0], d[1], d[2]);
        const f2 half = bc2(0.5f);
        f2 iu = mul2(half, add2(e[0], d[0])), iv = mul2(half, add2(e[1], d[1])), iw = mul2(half, add2(e[2], d[2]));
        if (pinc) {
            const f2 q = make_float2(cv.qA, cv.qB);
            iu = fma2(bc2(-K.gx), sub2(make_float2(cv.qxA, cv.qxB), q), iu);
            iv = fma2(bc2(-K.gy), sub2(make_float2(cv.qB, cv.qyB), q), iv);
            iw = fma2(bc2(-P.gz), sub2(make_float2(cv.qzA, cv.qzB), q), iw);
        }
        const size_t g = gA + sk * kq;
        const double zl = pzl[kq];
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const size_t gq = g + (size_t)q * p.nx;
            const double nu = cv.u[q] + (double)(q ? iu.y : iu.x), nv = cv.v[q] + (double)(q ? iv.y : iv.x),
                         nw = cv.w[q] + (double)(q ? iw.y : iw.x);
            uo[gq] = nu;
            vo[gq] = nv;
            if (kq != p.nz || !p.whi) wo[gq] = nw;
            wall_fill<double>(uo, vo, wo, gq, kq, sk, p.nz, 0.0 - p.u_crf, nu, nv, p.wlo, p.whi);
            su += nu * zl;
        }
    };

    // u1 = u + d1 at ring offset o (FP32), and its wall image at plane 0
    auto put1 = [&](int s, int sw, int xy, float du, float dv, float dw, bool bottom) {
        const float a = ur[s * SST + xy] + du, b = ur[s * SST + FST + xy] + dv;
        sr[s * SST + xy] = a;
        sr[s * SST + FST + xy] = b;
        sr[s * SST + 2 * FST + xy] = ur[s * SST + 2 * FST + xy] + dw;
        if (bottom) { // imposeNoSlipBC on u1: u1(0) = 2bc - u1(1), v1(0) = -v1(1), w1(0) = 0
            sr[sw * SST + xy] = bcu2 - a;
            sr[sw * SST + FST + xy] = -b;
            sr[sw * SST + 2 * FST + xy] = 0.f;
        }
    };
    // the top wall plane of u1 at ring slot st from plane nz at slot sn
    auto top1 = [&](int st, int sn, int xy) {
        sr[st * SST + xy] = bcu2 - sr[sn * SST + xy];
        sr[st * SST + FST + xy] = -sr[sn * SST + FST + xy];
        sr[st * SST + 2 * FST + xy] = 0.f;
    };

    // Two barriers per plane: stage 1 at plane mq reads u planes mq-1..mq+1
    // and writes u1 plane mq (under the top wall, at mq = nz+1, the wall
    // plane of u1 instead); then stage 2 at mq-1 reads u1 planes mq-2..mq,
    // and the staged u plane mq+2 is converted into the slot of plane mq-1.
    // PH = (mq - mstart) % 3: planes mq-1, mq, mq+1 in slots sa, sb, sc.
    auto march = [&](auto PH, int mq) {
        constexpr int sa = decltype(PH)::value, sb = (sa + 1) % MNS, sc = (sa + 2) % MNS;
        const bool do2 = (mq - 1 >= kbeg && mq - 1 <= kend);
        if (do2) prefetch(mq - 1);
        if (wall_step && mq == p.nz + 1) {
            // imposeNoSlipBC on u1 at the top wall, from u1 plane nz (slot sa)
            top1(sb, sa, hxy0);
            top1(sb, sa, hxy0 + MW);
            if (hval1) top1(sb, sa, hxy1);
        } else {
            const MxPlane P = mx_plane(ptab, mq);
            const bool top = p.whi && mq == p.nz, bottom = p.wlo && mq == 1;
            mx_rhs2<CRF>(ur, sa * SST + hxy0, sb * SST + hxy0, sc * SST + hxy0, P, K, c1, d1[0], d1[1], d1[2]);
            if (top) d1[2] = bc2(0.f); // w1(nz) = 0, the wall
            put1(sb, sa, hxy0, d1[0].x, d1[1].x, d1[2].x, bottom);
            put1(sb, sa, hxy0 + MW, d1[0].y, d1[1].y, d1[2].y, bottom);
            if (hval1) {
                float du, dv, dw;
                mx_rhs<CRF>(ur, sa * SST + hxy1, sb * SST + hxy1, sc * SST + hxy1, P, K, cH, du, dv, dw);
                if (top) dw = 0.f;
                put1(sb, sa, hxy1, du, dv, dw, bottom);
            }
        }
        __syncthreads();
        // plane mq-2 sits in slot sc
        if (do2) stage2(mq - 1, sc, sa, sb, e1, centre(mq - 1));
        // staged plane mq+2 (landed and published by the last iteration's
        // wait and barrier; its staging slot is sa) into the FP32 slot of
        // plane mq-1, which stage 1 above has finished with
        if (mq + 2 <= last) convert(sa);
        issue(mq + 4, last, sc); // into the staging slot of plane mq + 1, converted last iteration
        cp_async_wait<1>();      // plane mq + 3 landed (mq + 4 may be in flight)
#pragma unroll
        for (int q = 0; q < 3; q++) e1[q] = d1[q];
        __syncthreads();
    };
    for (int mq = mstart;;) {
        march(std::integral_constant<int, 0>{}, mq);
        if (++mq > mend) break;
        march(std::integral_constant<int, 1>{}, mq);
        if (++mq > mend) break;
        march(std::integral_constant<int, 2>{}, mq);
        if (++mq > mend) break;
    }
    cp_async_wait<0>();
    mean_reduce(su, red);
}

// z-chunks per tile column, as for the FP64 kernel: chunks of about 52
// planes, more where tiles x chunks would not fill one wave of resident CTAs
static int mx_chunks(const StepParams &p, long resident)
{
    const int tiles = (p.nx / MX) * (p.ny / MY);
    const int maxch = p.nz / 16 > 1 ? p.nz / 16 : 1;
    int nch = (p.nz + 26) / 52;
    if (nch < 1) nch = 1;
    while (nch < maxch && (long)tiles * nch < resident) nch++;
    return nch < maxch ? nch : maxch;
}

std::vector<float> rk_mixed_table(const StepParams &p, const std::vector<double> &dzf,
                                  const std::vector<double> &dzf_inv, const std::vector<double> &dzc_inv, int kg0,
                                  size_t np)
{
    // dzf, dzf_inv, dzc_inv: the global mesh, planes 0 .. nzg+1; entry q of
    // the table is global plane kg0 + q (entries beyond the global range,
    // only outside a wall, stay zero: nothing reads them)
    const int nzg = (int)dzf.size() - 2;
    std::vector<float> t(np * 12, 0.f);
    const double dt = p.dt, re = p.re_inv;
    const double cxx = dt * re * p.dx_inv * p.dx_inv, cyy = dt * re * p.dy_inv * p.dy_inv;
    for (size_t q = 0; q < np; q++) {
        const int k = kg0 + (int)q;
        if (k < 0 || k > nzg) continue;
        float *r = t.data() + (size_t)12 * q;
        r[0] = (float)(dzf[k + 1] * dzc_inv[k]); // a
        r[1] = (float)(dzf[k] * dzc_inv[k]);     // b
        if (k == 0) continue;
        const double azp = dt * re * dzf_inv[k] * dzc_inv[k], azm = dt * re * dzf_inv[k] * dzc_inv[k - 1];
        const double bzp = dt * re * dzc_inv[k] * dzf_inv[k + 1], bzm = dt * re * dzc_inv[k] * dzf_inv[k];
        r[2] = (float)(0.25 * dt * dzf_inv[k]); // hzuv
        r[3] = (float)azp;
        r[4] = (float)azm;
        r[5] = (float)(2.0 * cxx + 2.0 * cyy + azp + azm); // ccuv
        r[6] = (float)(0.25 * dt * dzc_inv[k]);            // hzw
        r[7] = (float)bzp;
        r[8] = (float)bzm;
        r[9] = (float)(2.0 * cxx + 2.0 * cyy + bzp + bzm); // ccw
        r[10] = (float)(dt * dzc_inv[k]);                  // gz
    }
    return t;
}

bool rk_mixed_supported(const StepParams &p) { return p.nx % MX == 0 && p.ny % MY == 0 && p.nz >= 2; }

int rk_mixed_blocks(const StepParams &p) { return (p.nx / MX) * (p.ny / MY) * (p.nz / 16 > 1 ? p.nz / 16 : 1); }

int launch_rk_mixed(const double *u, const double *v, const double *w, double *uo, double *vo, double *wo,
                    const StepParams &p, const MeshDev &m, const float *tab, MeanState &ms, const float *pq, int pinc,
                    cudaStream_t st)
{
    if (!rk_mixed_supported(p)) {
        set_error("mixed fused RK kernel needs nx % 32 == 0 and ny % 16 == 0");
        return -1;
    }
    // staging + rings + the chunk's coefficient table (room for chunks of up
    // to MX_KCHUNK planes; mx_chunks gives at most 78)
    const size_t shm = sizeof(double) * 3 * SST + sizeof(float) * 6 * SST +
                       (sizeof(float4) * 3 + sizeof(double)) * (MX_KCHUNK + 4);
    auto kern = (p.u_crf != 0.0) ? k_rk_mixed<true> : k_rk_mixed<false>;
    PL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    PL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
    int per_sm = 0, dev = 0, nsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, MT, shm) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int nch = mx_chunks(p, (long)per_sm * (nsm > 0 ? nsm : 1));
    const int kchunk = (p.nz + nch - 1) / nch;
    if (kchunk > MX_KCHUNK) {
        set_error("mixed fused RK kernel: z-chunk longer than its coefficient table");
        return -1;
    }
    dim3 grid(p.nx / MX, p.ny / MY, (p.nz + kchunk - 1) / kchunk);
    if ((int)(grid.x * grid.y * grid.z) > ms.max_blocks) {
        set_error("mean buffer too small for the mixed fused RK kernel");
        return -1;
    }
    MxConst K;
    K.hx = (float)(0.25 * p.dt * p.dx_inv);
    K.hy = (float)(0.25 * p.dt * p.dy_inv);
    K.cxx = (float)(p.dt * p.re_inv * p.dx_inv * p.dx_inv);
    K.cyy = (float)(p.dt * p.re_inv * p.dy_inv * p.dy_inv);
    K.ucx = (float)(0.5 * p.dt * p.u_crf * p.dx_inv);
    K.gx = (float)(p.dt * p.dx_inv);
    K.gy = (float)(p.dt * p.dy_inv);
    MeanRed r{ms.partial, ms.counter, ms.scalar, (double)p.nx, (double)p.ny, ms.vel_force};
    kern<<<grid, dim3(MX, MT / MX), shm, st>>>(u, v, w, uo, vo, wo, p, m, reinterpret_cast<const float4 *>(tab), K, r,
                                               kchunk, pq, pinc);
    PL_CHECK_LAUNCH();
    return 0;
}

} // namespace pl
