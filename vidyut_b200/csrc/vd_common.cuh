// Shared device utilities of the B200 library: error checks, launch
// accounting, block reductions, the grid descriptor.
#pragma once

#include <cuda_runtime.h>
#include <cstdio>
#include <string>

#define VD_CUDA_OK(call)                                                        \
    do                                                                          \
    {                                                                           \
        cudaError_t e_ = (call);                                                \
        if (e_ != cudaSuccess)                                                  \
            throw vd::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Every kernel of the library begins by waiting for the grids it depends
// on: launched with programmatic stream serialization (a dependent launch
// that may be scheduled while the previous kernel drains) it must not read
// before that kernel's writes are visible; launched normally the wait is a
// no-op.
#define VD_PDL_WAIT() asm volatile("griddepcontrol.wait;" ::: "memory")

namespace vd {

struct CudaError
{
    std::string msg;
    explicit CudaError(std::string m) : msg(std::move(m)) {}
    virtual ~CudaError() = default;
};

// A request the library does not support (returned as VD_ERR_UNSUPPORTED).
struct UnsupportedError : CudaError
{
    explicit UnsupportedError(std::string m) : CudaError(std::move(m)) {}
};

// A device allocation that failed for lack of memory (VD_ERR_OOM).
struct OomError : CudaError
{
    explicit OomError(std::string m) : CudaError(std::move(m)) {}
};

// Grid of one multigrid level (or of the state): cell counts, active
// dimension count, periodicity, storage layout.
//   natural (rb = 0): (i,j,k) -> i + nx*(j + ny*k)            (the state)
//   red-black split (rb = 1, nx even): the cells with (i+j+k) even come
//   first, then the odd ones, each half in natural order of (i/2, j, k):
//   (i,j,k) -> ((i+j+k)&1) * ncell/2 + (i>>1) + (nx/2)*(j + ny*k)
// so one Gauss-Seidel colour is a contiguous, unit-stride array.
struct GridDev
{
    int n[3];
    int dim;
    int per[3];
    int rb;
    __host__ __device__ long long ncell() const
    {
        return (long long)n[0] * n[1] * n[2];
    }
    __host__ __device__ long long idx(int i, int j, int k) const
    {
        const long long row = j + (long long)n[1] * k;
        if (!rb) return i + (long long)n[0] * row;
        return (long long)((i + j + k) & 1) * (ncell() >> 1) + (i >> 1) + (long long)(n[0] >> 1) * row;
    }
};

// Global launch counter (kernels launched by this library).
extern long long g_launches;

inline dim3 grid1d(long long n, int bs)
{
    long long b = (n + bs - 1) / bs;
    if (b < 1) b = 1;
    return dim3((unsigned)b);
}

// Max of non-negative values through their bit patterns (IEEE ordering of
// non-negative doubles equals unsigned ordering).
__device__ inline void atomic_max_nonneg(unsigned long long* addr, double v)
{
    atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

template <typename T>
__device__ inline T warp_sum(T v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Max that keeps a NaN: a residual norm taken over a state that went
// non-finite must not read as converged (fmax and `a > m ? a : m` drop it).
template <typename T>
__host__ __device__ __forceinline__ T nanmax(T m, T a)
{
    return (a > m || a != a) ? a : m;
}

template <typename T>
__device__ inline T warp_max(T v)
{
    for (int o = 16; o > 0; o >>= 1)
        v = nanmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum; `sh` must hold blockDim.x/32 entries.  All threads get it.
template <typename T>
__device__ inline T block_sum(T v, T* sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    T r = 0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w) r += sh[w];
    __syncthreads();
    return r;
}

template <typename T>
__device__ inline T block_max(T v, T* sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    T r = 0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w) r = nanmax(r, sh[w]);
    __syncthreads();
    return r;
}

} // namespace vd
