// Shared host-side plumbing of the del3d_b200 library: status handling,
// stream-ordered device buffers, launch helpers.
#pragma once

#include "../../include/del3d_b200.h"
#include "predicates.cuh"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <string>
#include <utility>

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

/// Stream-ordered device memory.  Blocks of kBlockCacheMin bytes and more go
/// through a per-device cache: a freed block waits there, with an event that
/// marks the end of its last use, and serves a later request of about its size
/// on any stream (which first waits for that event).  Repeated builds of one
/// workload then make no large pool calls: a large cudaMallocAsync can hold the
/// calling thread for hundreds of milliseconds even when the pool already
/// reserves the memory, while the device sits idle.  Smaller blocks, and blocks
/// of a stream under graph capture, go to the pool directly.
constexpr size_t kBlockCacheMin = size_t(1) << 20;
/// Allocates at least `bytes` on `s`; `*cap` receives the block's size when it
/// belongs to the cache (0 otherwise) and `*dev` its device.
cudaError_t device_block_alloc(void** p, size_t bytes, cudaStream_t s, size_t* cap, int* dev);
/// Hands back a block from device_block_alloc after the work queued on `s`.
void device_block_free(void* p, size_t cap, cudaStream_t s, int dev);
/// Returns the current device's cached blocks not in use to the pool; the
/// device must be synchronised.
int device_block_trim();

/// A stream-ordered device allocation, freed on the same stream.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    size_t cap = 0;     // size of a cached block, 0 for a pool block
    int dev = -1;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    int alloc(size_t count, cudaStream_t stream) {
        release();
        s = stream;
        n = count;
        if (count == 0) return D3G_OK;
        cudaError_t e = device_block_alloc(reinterpret_cast<void**>(&p), count * sizeof(T), stream, &cap, &dev);
        if (e != cudaSuccess) {
            p = nullptr;
            n = 0;
            set_error(std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
            return (e == cudaErrorMemoryAllocation) ? D3G_ERR_OOM : D3G_ERR_CUDA;
        }
        return D3G_OK;
    }
    void release() {
        if (p) device_block_free(p, cap, s, dev);
        p = nullptr;
        n = 0;
        cap = 0;
    }
    /// Exchanges the blocks of two buffers (ping-pong passes).
    void swap(DevBuf& o) {
        std::swap(p, o.p);
        std::swap(n, o.n);
        std::swap(s, o.s);
        std::swap(cap, o.cap);
        std::swap(dev, o.dev);
    }
};

/// A named NVTX range over a scope: a host-side marker that costs nothing
/// without a profiler attached.  The build marks d3g.build, d3g.order,
/// d3g.insert, "d3g.level N" and d3g.output, and the server each batch
/// (d3g.server.batch), so a profiler can pick the kernels of one phase
/// (ncu --nvtx --nvtx-include).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
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
