// common.cuh -- shared definitions of the B200 channel-flow step library.
//
// Device layout (all fields, both precisions): x fastest, then y, then z.
//   velocity-like fields  [k = 0 .. nz+1][j = 0 .. ny-1][i = 0 .. nx-1]
//       (wall ghost planes k = 0 and k = nz+1 are stored; x and y are periodic
//        and are indexed modulo nx / ny, so no x/y ghost cells exist)
//   pressure / PPE work    [k = 0 .. nz-1][j][i]   (interior only)
// The reference's ghosted Fortran array u(0:nx+1,0:ny+1,0:nz+1)
// (mod_variables.f90:21-41) maps to this layout by dropping the x/y ghosts,
// which on one rank always equal the periodic images of the interior
// (imposePeriodicBC, mod_updateBound.f90:241-272, and the self-exchange of
// updateHalo, :364-396).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

namespace pl {

// last error message of the calling host thread (C ABI: pl_last_error)
void set_error(const std::string &msg);
const char *get_error();

#define PL_CUDA_TRY(expr)                                                                  \
    do {                                                                                   \
        cudaError_t _e = (expr);                                                           \
        if (_e != cudaSuccess) {                                                           \
            ::pl::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e) + " at " +  \
                            __FILE__ + ":" + std::to_string(__LINE__));                    \
            return -1;                                                                     \
        }                                                                                  \
    } while (0)

#define PL_CHECK_LAUNCH()                                                                  \
    do {                                                                                   \
        cudaError_t _e = cudaGetLastError();                                               \
        if (_e != cudaSuccess) {                                                           \
            ::pl::set_error(std::string("kernel launch: ") + cudaGetErrorString(_e) +      \
                            " at " + __FILE__ + ":" + std::to_string(__LINE__));           \
            return -1;                                                                     \
        }                                                                                  \
    } while (0)

template <typename T> struct cplx_of;
template <> struct cplx_of<double> { using type = double2; };
template <> struct cplx_of<float> { using type = float2; };

template <typename V>
__host__ __device__ __forceinline__ V cmul(V a, V b)
{
    V r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

// a * conj(b)
template <typename V>
__host__ __device__ __forceinline__ V cmulc(V a, V b)
{
    V r;
    r.x = a.x * b.x + a.y * b.y;
    r.y = a.y * b.x - a.x * b.y;
    return r;
}

template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b)
{
    V r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    return r;
}

template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b)
{
    V r;
    r.x = a.x - b.x;
    r.y = a.y - b.y;
    return r;
}

__host__ __device__ __forceinline__ size_t idx3(int i, int j, int k, int nx, int ny)
{
    return (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * (size_t)k);
}

} // namespace pl
