// FP64 CUDA-core throughput probe: the denominator of the explicit kernel's
// roofline (the WENO flux and chemistry are FP64 arithmetic on the CUDA
// cores, not tensor-core work).  Each thread runs independent chains of
// fused multiply-adds with enough chains in flight to hide the FMA latency;
// the host times the launch with CUDA events and reports FP64 FLOP/s
// (2 per FMA).  The chains are seeded from the thread index and their sum is
// written out, so the compiler keeps every FMA.
#include <cuda_runtime.h>

namespace {

constexpr int CHAINS = 8;

__global__ void __launch_bounds__(256) k_fp64_fma(double* out, int iters, double a, double b)
{
    double x[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) x[c] = 1e-3 * (threadIdx.x + c);
    for (int it = 0; it < iters; ++it)
    {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

} // namespace

// FP64 FMA throughput of the current device in GFLOP/s (best of `reps`
// launches of `blocks_per_sm` x SM-count blocks of 256 threads, `iters`
// FMA rounds of CHAINS chains per thread); 0 on error.
extern "C" double vd_fp64_peak_gflops(int blocks_per_sm, int iters, int reps)
{
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0.0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0.0;
    const int blocks = blocks_per_sm * nsm;
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * (size_t)blocks * 256) != cudaSuccess) return 0.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    for (int r = 0; r < reps + 1; ++r)
    {
        cudaEventRecord(e0);
        k_fp64_fma<<<blocks, 256>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * CHAINS * (double)iters * blocks * 256.0;
        if (r > 0 && ms > 0.f) best = flops / (ms * 1e-3) / 1e9 > best ? flops / (ms * 1e-3) / 1e9 : best;
    }
    const bool ok = cudaGetLastError() == cudaSuccess;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return ok ? best : 0.0;
}
