// channel.cuh -- the device-resident channel object behind the pl_channel_*
// entry points, shared by the step (channel.cu) and its adjoint (adjoint.cu).
#pragma once

#include <string>
#include <vector>

#include "../../include/powerllel_b200.h"
#include "ppe.cuh"
#include "stencil.cuh"

struct pl_channel {
    pl_channel_config cfg{};
    int nx = 0, ny = 0, nz = 0;
    // z slab of a multi-GPU run (pl_channel_create_slab): nz above is the
    // slab's plane count, kst its first plane in the global grid (0-based);
    // hx = 1 extra halo plane below plane 0 and above nz+1 of every
    // velocity-like field (the fused RK kernels read two planes beyond the
    // slab), and one extra pressure plane (nz: the upper neighbour's first)
    int zrank = 0, zranks = 1, kst = 0, hx = 0;
    size_t nf = 0;  // elements of a velocity-like field, nx*ny*(nz+2)
    size_t np = 0;  // elements of p, nx*ny*nz
    pl::StepParams sp{};
    std::vector<double> dzf_global, zc_global, dzf, dzf_inv, dzc, dzc_inv, dzflzi, prof;
    double *d_mesh = nullptr;
    pl::MeshDev m{};
    // FP64 path: u,v,w = ua,va,wa; stage-1 fields u1,v1,w1; p
    // mixed path: u,v,w ping-pong between (ua,va,wa) and (ub,vb,wb); stage-1
    // increments d1u,d1v,d1w (FP32, the per-phase entries only); p32 = p_n
    // (FP32, updated in place by the solve); the pressure prediction for the
    // next projection in pm32, written into pb32 by the solve and swapped;
    // the PPE works in place on r32 (FP32); p (FP64) is p32 widened on demand
    // for readers (channel_p64); mxtab: the mixed RK kernel's per-plane
    // coefficients
    double *u = nullptr, *v = nullptr, *w = nullptr;
    double *u1 = nullptr, *v1 = nullptr, *w1 = nullptr;
    double *p = nullptr;
    double *ub = nullptr, *vb = nullptr, *wb = nullptr;
    float *p32 = nullptr, *pm32 = nullptr, *pb32 = nullptr, *mxtab = nullptr;
    bool p_stale = false; // mixed: p lags p32
    float *d1u = nullptr, *d1v = nullptr, *d1w = nullptr, *r32 = nullptr;
    double *plane_part = nullptr, *mode0 = nullptr;
    int incremental = 1;   // mixed path: solve for a pressure increment (Thomas)
    long long nsolve = 0;  // projections since the initial field (mixed prediction schedule)
    bool fused_rk = false; // both RK stages in one kernel (rk_fused.cu, rk_mixed.cu)
    pl::Ppe ppe;
    pl::ReduceBuf rb;
    pl::MeanState ms;
    double *d_diag = nullptr;
    int *d_loc = nullptr;
    double *d_dpart = nullptr;
    long long *d_dipart = nullptr;
    int max_blocks = 0;
    cudaStream_t stream = nullptr;
    void *stats = nullptr; // device statistics (monitor.cu), when enabled
    // profiling marks (pl_channel_profile)
    std::vector<cudaEvent_t> *prof_events = nullptr;
    std::vector<std::string> *prof_names = nullptr;
};

namespace pl {
// the FP64 pressure of the current state (the mixed path widens p32 into p
// on the channel's stream when it has changed)
const double *channel_p64(pl_channel *c);
} // namespace pl
