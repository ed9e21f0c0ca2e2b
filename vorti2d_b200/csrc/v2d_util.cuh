// Host/device utilities shared by the translation units: a stream-ordered
// device buffer, a deterministic exclusive scan and block reductions.
#pragma once

#include "v2d_common.cuh"

namespace v2d {

// Number of kernels this library has launched (graph replays count their
// kernel nodes); read through v2d_launch_count().
void count_launches(long long n);

// Device allocation from the stream-ordered pool; freed on destruction.
template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t s = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    int alloc(size_t count, cudaStream_t stream)
    {
        release();
        s = stream;
        n = count;
        if (count == 0) return V2D_OK;
        cudaError_t e = cudaMallocAsync((void **)&p, count * sizeof(T), stream);
        if (e != cudaSuccess) {
            p = nullptr;
            n = 0;
            set_error("device allocation of %zu bytes failed: %s", count * sizeof(T),
                      cudaGetErrorString(e));
            return V2D_ENOMEM;
        }
        return V2D_OK;
    }
    void release()
    {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
};

// Exclusive scan of n ints (d_in may equal d_out); *total receives the sum
// (device scalar).  Deterministic (fixed blocking).  Needs scratch of
// scan_scratch_ints(n) ints.
size_t scan_scratch_ints(long long n);
int exclusive_scan_i32(const int *d_in, int *d_out, long long n, int *d_total, int *d_scratch,
                       cudaStream_t s);

// Warp / block sum helpers (deterministic order for a fixed launch shape).
template <class T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sum; result valid in all threads.  smem: >= 32 elements.
template <class T>
__device__ __forceinline__ T block_sum(T v, T *smem)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) smem[wid] = v;
    __syncthreads();
    T r = (threadIdx.x < nw) ? smem[threadIdx.x] : T(0);
    if (wid == 0) r = warp_sum(r);
    if (threadIdx.x == 0) smem[0] = r;
    __syncthreads();
    r = smem[0];
    __syncthreads();
    return r;
}

}  // namespace v2d
