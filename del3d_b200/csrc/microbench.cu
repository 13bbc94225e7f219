// FP64 throughput of this GPU, measured with the arithmetic the predicate
// filters use: separate DADD and DMUL (the library is built with -fmad=false,
// so the filters never contract into DFMA).  The roofline of a filter kernel
// is its queries/s x FP64 operations per query against this figure.
// A measurement aid with no counterpart in the reference.
#include "common.cuh"

#include <cuda_runtime.h>

namespace d3g {
namespace {

constexpr int kChains = 8;

/// Each thread runs kChains independent x = x * m + c chains for `iters`
/// steps: 2 * kChains FP64 operations per step, kept separate (no FMA).
__global__ void __launch_bounds__(256) k_fp64_addmul(double* __restrict__ sink, int iters, double m, double c) {
    double x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = 1.0 + 1e-3 * (threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = __dadd_rn(__dmul_rn(x[k], m), c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    if (s == 12345.678) sink[blockIdx.x] = s;   // keeps the chains live; never true in practice
}

/// The same chains contracted into DFMA (one instruction, two FLOPs).
__global__ void __launch_bounds__(256) k_fp64_fma(double* __restrict__ sink, int iters, double m, double c) {
    double x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = 1.0 + 1e-3 * (threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = __fma_rn(x[k], m, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    if (s == 12345.678) sink[blockIdx.x] = s;
}

}  // namespace
}  // namespace d3g

using namespace d3g;

extern "C" int d3g_microbench_fp64(int64_t iters, double* addmul_ops_per_s, double* fma_per_s, void* stream) {
    if (iters < 1 || iters > (int64_t(1) << 30)) return D3G_ERR_INVALID_ARGUMENT;
    D3G_TRY(ensure_device());
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    D3G_CUDA(cudaGetDevice(&dev));
    D3G_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int block = 256, grid = sms * 8;
    DevBuf<double> sink;
    D3G_TRY(sink.alloc(size_t(grid), s));
    cudaEvent_t e0, e1;
    D3G_CUDA(cudaEventCreate(&e0));
    D3G_CUDA(cudaEventCreate(&e1));
    const double m = 0.9999999, c = 1e-7;
    const double threads = double(grid) * block;
    // warm-up, then one timed launch of each
    k_fp64_addmul<<<grid, block, 0, s>>>(sink.p, 64, m, c);
    k_fp64_fma<<<grid, block, 0, s>>>(sink.p, 64, m, c);
    float ms = 0.f;
    cudaEventRecord(e0, s);
    k_fp64_addmul<<<grid, block, 0, s>>>(sink.p, int(iters), m, c);
    cudaEventRecord(e1, s);
    D3G_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    if (addmul_ops_per_s) *addmul_ops_per_s = threads * double(iters) * kChains * 2.0 / (ms * 1e-3);
    cudaEventRecord(e0, s);
    k_fp64_fma<<<grid, block, 0, s>>>(sink.p, int(iters), m, c);
    cudaEventRecord(e1, s);
    D3G_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    if (fma_per_s) *fma_per_s = threads * double(iters) * kChains / (ms * 1e-3);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    sink.release();
    D3G_CUDA(cudaStreamSynchronize(s));
    return D3G_OK;
}
