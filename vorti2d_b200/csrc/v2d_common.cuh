// Shared definitions for the vorti2d B200 kernels: status codes, error
// reporting, launch helpers and the node-topology helpers every kernel uses.
//
// Node pointer (reference src/fortran/vorti2d_core.f90:10-13): 1-based
// k = imax*(j-1) + i.  Device code works 0-based: K = k-1 = imax*(j-1) + (i-1),
// so every field array is a row-major [jmax][imax] slab (i fastest) and a warp
// of consecutive K reads 32 consecutive doubles.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/vorti2d_b200.h"

namespace v2d {

// Last error message of the calling host thread (v2d_last_error()).
void set_error(const char *fmt, ...);

#define V2D_CUDA_TRY(expr)                                                          \
    do {                                                                            \
        cudaError_t _e = (expr);                                                    \
        if (_e != cudaSuccess) {                                                    \
            ::v2d::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,            \
                             cudaGetErrorString(_e));                               \
            return V2D_ECUDA;                                                       \
        }                                                                           \
    } while (0)

#define V2D_TRY(expr)                                                               \
    do {                                                                            \
        int _s = (expr);                                                            \
        if (_s != V2D_OK) return _s;                                                \
    } while (0)

#define V2D_ARG_CHECK(cond, ...)                                                    \
    do {                                                                            \
        if (!(cond)) {                                                              \
            ::v2d::set_error(__VA_ARGS__);                                          \
            return V2D_EARG;                                                        \
        }                                                                           \
    } while (0)

constexpr int kSMs = 148;  // B200: 2 dies x 74 SMs

inline int grid_for(long long n, int block, int per_sm_cap = 32)
{
    long long g = (n + block - 1) / block;
    long long cap = (long long)kSMs * per_sm_cap;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// Neighbour pointers with the O-grid branch-cut wrap, 0-based
// (reference vorti2d_core.f90:33-61): i=0 west -> imax-2, i=imax-1 east -> 1.
struct Nbr {
    int k, e, w, n, s, ne, nw, se, sw;
};

__host__ __device__ __forceinline__ Nbr wrap_neighbors(int i, int j, int imax)
{
    Nbr b;
    b.k = imax * j + i;
    b.n = b.k + imax;
    b.s = b.k - imax;
    int de, dw;
    if (i == 0) {
        de = 1; dw = imax - 2;
    } else if (i == imax - 1) {
        de = -(imax - 2); dw = -1;
    } else {
        de = 1; dw = -1;
    }
    b.e = b.k + de; b.w = b.k + dw;
    b.ne = b.n + de; b.nw = b.n + dw;
    b.se = b.s + de; b.sw = b.s + dw;
    return b;
}

// Grid-stride loop helper.
#define V2D_GRID_STRIDE(idx, count)                                                 \
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;          \
         idx < (long long)(count); idx += (long long)gridDim.x * blockDim.x)

}  // namespace v2d
