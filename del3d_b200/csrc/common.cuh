// Shared host-side plumbing of the del3d_b200 library: status handling,
// stream-ordered device buffers, launch helpers.
#pragma once

#include "../../include/del3d_b200.h"
#include "predicates.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace d3g {

constexpr int kNumSMs = 148;   // B200: 2 dies x 74 SMs

/// Records a detail message for d3g_last_error() on the calling thread.
void set_error(const std::string& msg);

/// Maps device status bits to the C status code.
int status_from_bits(uint32_t bits);

#define D3G_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            ::d3g::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));       \
            return (e_ == cudaErrorMemoryAllocation) ? D3G_ERR_OOM : D3G_ERR_CUDA;       \
        }                                                                                \
    } while (0)

#define D3G_TRY(expr)                  \
    do {                               \
        int s_ = (expr);               \
        if (s_ != D3G_OK) return s_;   \
    } while (0)

/// A stream-ordered device allocation, freed on the same stream.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    int alloc(size_t count, cudaStream_t stream) {
        release();
        s = stream;
        n = count;
        if (count == 0) return D3G_OK;
        cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), stream);
        if (e != cudaSuccess) {
            p = nullptr;
            n = 0;
            set_error(std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
            return (e == cudaErrorMemoryAllocation) ? D3G_ERR_OOM : D3G_ERR_CUDA;
        }
        return D3G_OK;
    }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
};

inline unsigned grid_for(int64_t n, int block, int64_t cap = int64_t(kNumSMs) * 32) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return unsigned(g);
}

/// Host memory for result arrays, from a cache of pinned (page-locked) blocks:
/// device-to-host copies into it run at full PCIe rate, and a block handed back
/// by host_result_free is reused by later results instead of being pinned again.
/// Falls back to malloc if pinning fails.  host_result_free accepts any pointer
/// host_result_alloc returned (and null).
void* host_result_alloc(size_t bytes);
void host_result_free(void* p);
/// Unpins and frees the cached blocks not in use.
void host_result_trim();

/// Ensures a CUDA device is present and current, and prepares it.
int ensure_device();
/// Once per device: keeps freed stream-ordered allocations cached in the pool.
int prepare_device();

}  // namespace d3g
