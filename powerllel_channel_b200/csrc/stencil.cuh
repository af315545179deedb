// stencil.cuh -- momentum, divergence, projection and boundary kernels of the
// RK2 projection step (Fortran reference: src/mod_calcVel.f90,
// src/mod_calcRHS.f90, src/mod_updateBound.f90, src/mod_utils.f90).
#pragma once

#include <vector>

#include "common.cuh"

namespace pl {

struct MeshDev {
    const double *dzf, *dzf_inv, *dzc_inv, *dzflzi; // index 0 .. nz+1 as in mod_mesh.f90:36-38
};

struct StepParams {
    int nx, ny, nz;
    double dx_inv, dy_inv, re_inv, dt, u_crf;
    double fb[3]; // uniform body force added to both RK stages (FP64 path; zero in the reference's step)
    // z slab of a multi-GPU run: wlo / whi = 1 where the slab's bottom / top
    // is a wall (imposeNoSlipBC), 0 at an interface with a neighbouring slab,
    // whose velocity planes -1, 0 (nz+1, nz+2) are halos filled by exchange
    int wlo = 1, whi = 1;
    int kofs = 0, nzg = 0; // the slab's first plane in the global grid, the global nz (0: nz)
};

// Reduction scratch: per-block partial results and the final scalars.
struct ReduceBuf {
    double *partial = nullptr; // >= max blocks * 3
    double *scalar = nullptr;  // [0..2] component means, [3..5] forcing shift, [6] u's plane-weighted sum
    int max_blocks = 0;
};

// FP64 step kernels (one launch each)
int launch_rk1_fp64(const double *u, const double *v, const double *w, double *u1, double *v1, double *w1,
                    const StepParams &p, const MeshDev &m, cudaStream_t st);
int launch_rk2_fp64(double *u, double *v, double *w, const double *u1, const double *v1, const double *w1,
                    const StepParams &p, const MeshDev &m, cudaStream_t st);
int launch_calc_rhs_fp64(const double *u, const double *v, const double *w, double *rhs, const StepParams &p,
                         const MeshDev &m, cudaStream_t st);
// correctVel + the dz-weighted sums of Mean_h for the forced components
int launch_correct_fp64(const double *p_, double *u, double *v, double *w, const StepParams &p, const MeshDev &m,
                        const int forced[3], ReduceBuf &rb, cudaStream_t st);
// forceVel shift (from the sums) + wall fill of the forced components
int launch_force_fp64(double *u, double *v, double *w, const StepParams &p, const int forced[3],
                      const double vel_force[3], ReduceBuf &rb, cudaStream_t st);

// Mean_h of the RK2 output reduced inside the RK2 kernel (deterministic
// last-block sum); scalar[3] = vel_force(1) - Mean_h, applied by the
// correction kernel (forceVel)
struct MeanState {
    double *partial = nullptr;       // >= max_blocks
    unsigned int *counter = nullptr; // zero-initialised once
    double *scalar = nullptr;        // >= 7 (as ReduceBuf::scalar)
    int max_blocks = 0;
    double vel_force = 0.0;
};

// fused RK1 + RK2 (rk_fused.cu): u -> (uo, vo, wo) out of place
bool rk_fused_supported(const StepParams &p);
int rk_fused_blocks(const StepParams &p);
int launch_rk_fused_fp64(const double *u, const double *v, const double *w, double *uo, double *vo, double *wo,
                         const StepParams &p, const MeshDev &m, MeanState &ms, cudaStream_t st);

// mixed path: both RK stages in FP32 flux form (rk_mixed.cu); with pinc,
// u_hat = u* - dt G pq is stored (pq: the FP32 pressure prediction,
// interior-only layout), whose divergence / dt is the increment's residual.
// tab: the per-plane coefficients of rk_mixed_table, 12 floats per plane
// k = 0..nz+1, on the device.
struct MxPlane {
    float a, b;                 // face weights: q_{k+1/2} = q_k a + q_{k+1} b
    float hzuv, azp, azm, ccuv; // u, v equations (dt folded in)
    float hzw, bzp, bzm, ccw;   // w equation
    float gz;                   // dt dzc_inv(k)
};
struct MxConst {
    float hx, hy, cxx, cyy, ucx, gx, gy;
};
bool rk_mixed_supported(const StepParams &p);
int rk_mixed_blocks(const StepParams &p);
// the table's np planes from global plane kg0 on (the mesh vectors are global)
std::vector<float> rk_mixed_table(const StepParams &p, const std::vector<double> &dzf,
                                  const std::vector<double> &dzf_inv, const std::vector<double> &dzc_inv, int kg0,
                                  size_t np);
int launch_rk_mixed(const double *u, const double *v, const double *w, double *uo, double *vo, double *wo,
                    const StepParams &p, const MeshDev &m, const float *tab, MeanState &ms, const float *pq, int pinc,
                    cudaStream_t st);

int launch_rk2m_fp64(double *u, double *v, double *w, const double *u1, const double *v1, const double *w1,
                     const StepParams &p, const MeshDev &m, MeanState &ms, cudaStream_t st);
int launch_correct_force_fp64(const double *p_, double *u, double *v, double *w, const StepParams &p,
                              const MeshDev &m, int forced_x, const double *scalar, cudaStream_t st);
// the same with an FP32 pressure (the mixed path's increment)
int launch_correct_force_f32(const float *p_, double *u, double *v, double *w, const StepParams &p,
                             const MeshDev &m, int forced_x, const double *scalar, cudaStream_t st);

// mixed precision: u, v, w, p in FP64; stage-1 increments and PPE in FP32
int launch_rk1_mixed(const double *u, const double *v, const double *w, float *d1u, float *d1v, float *d1w,
                     const StepParams &p, const MeshDev &m, cudaStream_t st);
int launch_rk2_mixed(const double *u, const double *v, const double *w, const float *d1u, const float *d1v,
                     const float *d1w, double *uo, double *vo, double *wo, const StepParams &p, const MeshDev &m,
                     MeanState &ms, const float *pq, int pinc, cudaStream_t st);
int launch_rhs_mixed(const double *u, const double *v, const double *w, float *r, double *warp_part, double *mode0,
                     const StepParams &p, const MeshDev &m, cudaStream_t st);
int warp_partials_per_plane(const StepParams &p);
// mode0[k] = sum over the nper partials of plane k, in a fixed order
int launch_plane_sums(const double *part, int nper, int nz, double *mode0, cudaStream_t st);

// diagnostics: out[0] = max|div| , out[1] = max CFL (already * dt), out[2] =
// NaN count over u,v,w (ghosts included); loc[0..2] ijk of the div max,
// loc[3..5] of the CFL max (1-based interior indices, reference convention)
int launch_diagnostics_fp64(const double *u, const double *v, const double *w, const StepParams &p,
                            const MeshDev &m, double *d_out, int *d_loc, double *d_part, long long *d_ipart,
                            int max_blocks, cudaStream_t st);

// initial field: Poiseuille profile + counter-based SplitMix64 noise
int launch_init_fill(double *u, double *v, double *w, const double *prof, uint64_t seed, double noise,
                     const StepParams &p, cudaStream_t st);
int launch_mean_sum(const double *var, const StepParams &p, const MeshDev &m, ReduceBuf &rb, int comp,
                    cudaStream_t st);
int launch_init_finish(double *u, double *v, double *w, const StepParams &p, double u_ref, ReduceBuf &rb,
                       cudaStream_t st);
int launch_fill_bc_vel(double *u, double *v, double *w, const StepParams &p, cudaStream_t st);
// z slabs: Mean_h and the forceVel shift from the cross-rank sum in
// scalar[6]; the initial-field normalisation likewise
int launch_mean_from_sum(double *scalar, const StepParams &p, double vel_force, cudaStream_t st);
int launch_mean_partials(const StepParams &p, ReduceBuf &rb, cudaStream_t st);
int launch_init_finish_sum(double *u, double *v, double *w, const StepParams &p, double u_ref, ReduceBuf &rb,
                           cudaStream_t st);

} // namespace pl
