// C ABI plumbing: status strings, error detail, host-pointer wrappers of the
// device entry points, synthetic input generators.
#include "common.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#include <string>
#include <vector>

namespace d3g {

int predicates_device(const double* d_pts, int64_t n_pts, const int32_t* d_idx, int64_t nq, int kind,
                      int8_t* d_out, cudaStream_t stream, d3g_predicate_stats* stats);
int orient2d_device(const double* d_six, int64_t nq, int8_t* d_out, cudaStream_t stream);

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int status_from_bits(uint32_t bits) {
    if (bits & ST_EXACT_CAPACITY) {
        set_error("coordinate exponent span too wide for the exact stage");
        return D3G_ERR_EXACT_CAPACITY;
    }
    if (bits & ST_CAVITY_CAPACITY) return D3G_ERR_CAVITY_CAPACITY;
    if (bits & ST_WALK_LIMIT) return D3G_ERR_WALK_LIMIT;
    if (bits & ST_TET_CAPACITY) return D3G_ERR_OOM;
    if (bits & ST_ROUND_LIMIT) return D3G_ERR_ROUND_LIMIT;
    if (bits & ST_INTERNAL) return D3G_ERR_INTERNAL;
    return D3G_OK;
}

int ensure_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_error(std::string("no CUDA device: ") + cudaGetErrorString(e));
        cudaGetLastError();
        return D3G_ERR_NO_DEVICE;
    }
    return prepare_device();
}

int prepare_device() {
    // The build allocates and frees gigabytes per call from the stream-ordered
    // pool; keep that memory in the pool instead of handing it back to the
    // driver at every synchronisation (d3g_release_cached_memory trims it).
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        set_error("no current CUDA device");
        return D3G_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = ~uint64_t(0);
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        cudaGetLastError();
        done[dev] = true;
    }
    return D3G_OK;
}

namespace {

struct PinnedCache {
    std::mutex mu;
    std::multimap<size_t, void*> free_blocks;     // size -> block, not in use
    std::map<void*, size_t> pinned;               // every pinned block -> size
    size_t cached_bytes = 0;                      // bytes in free_blocks
};

PinnedCache& pinned_cache() {
    static PinnedCache* c = new PinnedCache();    // lives until exit (blocks freed by trim)
    return *c;
}

// Blocks kept for reuse, at most this many bytes in all.
constexpr size_t kPinnedCacheBytes = size_t(16) << 30;

}  // namespace

void* host_result_alloc(size_t bytes) {
    if (bytes == 0) bytes = 16;
    PinnedCache& c = pinned_cache();
    {
        std::lock_guard<std::mutex> lock(c.mu);
        // Smallest cached block that fits, if it is not more than twice the need.
        auto it = c.free_blocks.lower_bound(bytes);
        if (it != c.free_blocks.end() && it->first <= 2 * bytes) {
            void* p = it->second;
            c.cached_bytes -= it->first;
            c.free_blocks.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) == cudaSuccess && p) {
        std::lock_guard<std::mutex> lock(c.mu);
        c.pinned[p] = bytes;
        return p;
    }
    cudaGetLastError();
    return malloc(bytes);
}

void host_result_free(void* p) {
    if (!p) return;
    PinnedCache& c = pinned_cache();
    std::vector<void*> evict;
    {
        std::lock_guard<std::mutex> lock(c.mu);
        auto it = c.pinned.find(p);
        if (it == c.pinned.end()) {
            free(p);
            return;
        }
        c.free_blocks.emplace(it->second, p);
        c.cached_bytes += it->second;
        // Over the cap: drop the smallest cached blocks first.
        while (c.cached_bytes > kPinnedCacheBytes && !c.free_blocks.empty()) {
            auto f = c.free_blocks.begin();
            c.cached_bytes -= f->first;
            c.pinned.erase(f->second);
            evict.push_back(f->second);
            c.free_blocks.erase(f);
        }
    }
    for (void* q : evict) cudaFreeHost(q);
}

void host_result_trim() {
    PinnedCache& c = pinned_cache();
    std::vector<void*> evict;
    {
        std::lock_guard<std::mutex> lock(c.mu);
        for (auto& kv : c.free_blocks) {
            c.pinned.erase(kv.second);
            evict.push_back(kv.second);
        }
        c.free_blocks.clear();
        c.cached_bytes = 0;
    }
    for (void* q : evict) cudaFreeHost(q);
}

namespace {

struct IdleBlock {
    void* p;
    cudaStream_t s;     // stream of its last use
    cudaEvent_t ev;     // recorded on s when the block was handed back
    uint64_t age;       // hand-back order: the oldest is evicted first
};

struct DeviceBlockCache {
    std::mutex mu;
    std::multimap<size_t, IdleBlock> idle;   // size -> block not in use
    std::vector<cudaEvent_t> events;         // spare events of this device
    size_t idle_bytes = 0;
    size_t limit = 0;                        // idle bytes kept: half the device memory
    uint64_t clock = 0;
};

constexpr int kMaxDevices = 64;

DeviceBlockCache& block_cache(int dev) {
    static DeviceBlockCache* c = new DeviceBlockCache[kMaxDevices];   // lives until exit
    return c[dev];
}

bool is_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return st != cudaStreamCaptureStatusNone;
}

cudaEvent_t take_event(DeviceBlockCache& c) {
    {
        std::lock_guard<std::mutex> lock(c.mu);
        if (!c.events.empty()) {
            cudaEvent_t ev = c.events.back();
            c.events.pop_back();
            return ev;
        }
    }
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return ev;
}

void give_event(DeviceBlockCache& c, cudaEvent_t ev) {
    std::lock_guard<std::mutex> lock(c.mu);
    c.events.push_back(ev);
}

/// Returns idle blocks to the pool in the order of `s`, after their last use.
void free_idle_on(DeviceBlockCache& c, std::vector<IdleBlock>& blocks, cudaStream_t s) {
    for (IdleBlock& b : blocks) {
        if (b.s != s && cudaStreamWaitEvent(s, b.ev, 0) != cudaSuccess) cudaGetLastError();
        if (cudaFreeAsync(b.p, s) != cudaSuccess) cudaGetLastError();
        give_event(c, b.ev);
    }
    blocks.clear();
}

}  // namespace

cudaError_t device_block_alloc(void** p, size_t bytes, cudaStream_t s, size_t* cap, int* dev) {
    *cap = 0;
    *dev = -1;
    int d = -1;
    if (bytes >= kBlockCacheMin && cudaGetDevice(&d) != cudaSuccess) {
        cudaGetLastError();
        d = -1;
    }
    if (bytes < kBlockCacheMin || d < 0 || d >= kMaxDevices || is_capturing(s))
        return cudaMallocAsync(p, bytes, s);
    DeviceBlockCache& c = block_cache(d);
    bool hit = false;
    size_t size = 0;
    IdleBlock b{};
    {
        std::lock_guard<std::mutex> lock(c.mu);
        if (c.limit == 0) {
            size_t free_b = 0, total_b = 0;
            if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) cudaGetLastError();
            c.limit = std::max<size_t>(total_b / 2, size_t(1) << 30);
        }
        // The smallest idle block that fits, if it wastes at most a quarter.
        auto it = c.idle.lower_bound(bytes);
        if (it != c.idle.end() && it->first - bytes <= bytes / 4) {
            hit = true;
            size = it->first;
            b = it->second;
            c.idle_bytes -= size;
            c.idle.erase(it);
        }
    }
    if (hit) {
        if (b.s == s || cudaStreamWaitEvent(s, b.ev, 0) == cudaSuccess) {
            give_event(c, b.ev);
            *p = b.p;
            *cap = size;
            *dev = d;
            return cudaSuccess;
        }
        cudaGetLastError();
        std::vector<IdleBlock> one{b};
        free_idle_on(c, one, b.s);
    }
    cudaError_t e = cudaMallocAsync(p, bytes, s);
    if (e == cudaErrorMemoryAllocation) {
        // Idle blocks of other sizes go back to the pool, which may then fit the request.
        cudaGetLastError();
        std::vector<IdleBlock> all;
        {
            std::lock_guard<std::mutex> lock(c.mu);
            for (auto& kv : c.idle) all.push_back(kv.second);
            c.idle.clear();
            c.idle_bytes = 0;
        }
        if (!all.empty()) {
            free_idle_on(c, all, s);
            e = cudaMallocAsync(p, bytes, s);
        }
    }
    if (e == cudaSuccess) {
        *cap = bytes;
        *dev = d;
    }
    return e;
}

void device_block_free(void* p, size_t cap, cudaStream_t s, int dev) {
    if (!p) return;
    if (cap == 0 || dev < 0 || dev >= kMaxDevices || is_capturing(s)) {
        cudaFreeAsync(p, s);
        return;
    }
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) cudaGetLastError();
    if (cur != dev && cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeAsync(p, s);
        return;
    }
    DeviceBlockCache& c = block_cache(dev);
    cudaEvent_t ev = take_event(c);
    if (!ev || cudaEventRecord(ev, s) != cudaSuccess) {
        cudaGetLastError();
        if (ev) give_event(c, ev);
        if (cudaFreeAsync(p, s) != cudaSuccess) cudaGetLastError();
    } else {
        std::vector<IdleBlock> evict;
        {
            std::lock_guard<std::mutex> lock(c.mu);
            c.idle.emplace(cap, IdleBlock{p, s, ev, ++c.clock});
            c.idle_bytes += cap;
            while (c.idle_bytes > c.limit && !c.idle.empty()) {
                auto oldest = c.idle.begin();
                for (auto it = c.idle.begin(); it != c.idle.end(); ++it)
                    if (it->second.age < oldest->second.age) oldest = it;
                c.idle_bytes -= oldest->first;
                evict.push_back(oldest->second);
                c.idle.erase(oldest);
            }
        }
        free_idle_on(c, evict, s);
    }
    if (cur != dev && cur >= 0 && cudaSetDevice(cur) != cudaSuccess) cudaGetLastError();
}

int device_block_trim() {
    int d = -1;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) {
        cudaGetLastError();
        return D3G_ERR_NO_DEVICE;
    }
    DeviceBlockCache& c = block_cache(d);
    std::vector<IdleBlock> all;
    std::vector<cudaEvent_t> events;
    {
        std::lock_guard<std::mutex> lock(c.mu);
        for (auto& kv : c.idle) all.push_back(kv.second);
        c.idle.clear();
        c.idle_bytes = 0;
        events.swap(c.events);
    }
    // The caller has synchronised the device: every idle block's last use is
    // over, and the legacy stream orders the frees (the stream of a block's last
    // use may be gone by now).
    cudaError_t first = cudaSuccess;
    auto note = [&](cudaError_t e) {
        if (e != cudaSuccess && first == cudaSuccess) first = e;
    };
    for (IdleBlock& b : all) {
        note(cudaFreeAsync(b.p, cudaStreamLegacy));
        note(cudaEventDestroy(b.ev));
    }
    for (cudaEvent_t ev : events) note(cudaEventDestroy(ev));
    if (first == cudaSuccess) return D3G_OK;
    cudaGetLastError();
    set_error(std::string("releasing cached device blocks: ") + cudaGetErrorString(first));
    return D3G_ERR_CUDA;
}

}  // namespace d3g

using namespace d3g;

extern "C" {

const char* d3g_status_string(int status) {
    switch (status) {
        case D3G_OK: return "ok";
        case D3G_ERR_INVALID_ARGUMENT: return "invalid argument";
        case D3G_ERR_INVALID_INPUT: return "invalid input";
        case D3G_ERR_OOM: return "out of device memory";
        case D3G_ERR_EXACT_CAPACITY: return "exact-stage capacity exceeded";
        case D3G_ERR_CAVITY_CAPACITY: return "conflict-region capacity exceeded";
        case D3G_ERR_WALK_LIMIT: return "point-location walk limit exceeded";
        case D3G_ERR_ROUND_LIMIT: return "insertion round limit exceeded";
        case D3G_ERR_CUDA: return "CUDA error";
        case D3G_ERR_INTERNAL: return "internal error";
        case D3G_ERR_NO_DEVICE: return "no CUDA device";
        case D3G_ERR_NOT_READY: return "not complete yet";
        default: return "unknown status";
    }
}

const char* d3g_last_error(void) { return g_last_error.c_str(); }

int d3g_release_cached_memory(void) {
    host_result_trim();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return D3G_ERR_NO_DEVICE;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return D3G_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return D3G_ERR_CUDA;
    D3G_TRY(device_block_trim());
    if (cudaDeviceSynchronize() != cudaSuccess) return D3G_ERR_CUDA;
    return cudaMemPoolTrimTo(pool, 0) == cudaSuccess ? D3G_OK : D3G_ERR_CUDA;
}

int d3g_predicate_arity(int kind) {
    switch (kind) {
        case D3G_ORIENT3D: return 4;
        case D3G_IN_SPHERE: return 5;
        case D3G_IN_SPHERE_UNPERTURBED: return 5;
        case D3G_COPLANAR_ORIENTATION3: return 3;
        case D3G_COPLANAR_ORIENTATION4: return 4;
        case D3G_COPLANAR_IN_CIRCLE: return 4;
        case D3G_COPLANAR_IN_CIRCLE_UNPERTURBED: return 4;
        case D3G_COLLINEAR: return 3;
        default: return 0;
    }
}

int d3g_predicates_device(const double* d_pts, int64_t n_pts, const int32_t* d_idx,
                          int64_t n_queries, int kind, int8_t* d_sign_out, void* stream,
                          d3g_predicate_stats* stats) {
    return predicates_device(d_pts, n_pts, d_idx, n_queries, kind, d_sign_out,
                             static_cast<cudaStream_t>(stream), stats);
}

int d3g_predicates(const double* pts, int64_t n_pts, const int32_t* idx, int64_t n_queries, int kind,
                   int8_t* sign_out, d3g_predicate_stats* stats) {
    const int k = d3g_predicate_arity(kind);
    if (k == 0 || n_pts < 0 || n_queries < 0) return D3G_ERR_INVALID_ARGUMENT;
    if (n_queries == 0) {
        if (stats) *stats = d3g_predicate_stats{0, 0};
        return D3G_OK;
    }
    if (!pts || !idx || !sign_out) return D3G_ERR_INVALID_ARGUMENT;
    D3G_TRY(ensure_device());
    cudaStream_t s = nullptr;
    DevBuf<double> dp;
    DevBuf<int32_t> di;
    DevBuf<int8_t> dout;
    D3G_TRY(dp.alloc(size_t(3 * n_pts > 0 ? 3 * n_pts : 1), s));
    D3G_TRY(di.alloc(size_t(k * n_queries), s));
    D3G_TRY(dout.alloc(size_t(n_queries), s));
    if (n_pts > 0) D3G_CUDA(cudaMemcpyAsync(dp.p, pts, sizeof(double) * 3 * n_pts, cudaMemcpyHostToDevice, s));
    D3G_CUDA(cudaMemcpyAsync(di.p, idx, sizeof(int32_t) * k * n_queries, cudaMemcpyHostToDevice, s));
    const int st = predicates_device(dp.p, n_pts, di.p, n_queries, kind, dout.p, s, stats);
    if (st != D3G_OK) return st;
    D3G_CUDA(cudaMemcpyAsync(sign_out, dout.p, size_t(n_queries), cudaMemcpyDeviceToHost, s));
    D3G_CUDA(cudaStreamSynchronize(s));
    return D3G_OK;
}

int d3g_orient2d(const double* six, int64_t n_queries, int8_t* sign_out) {
    if (n_queries < 0) return D3G_ERR_INVALID_ARGUMENT;
    if (n_queries == 0) return D3G_OK;
    if (!six || !sign_out) return D3G_ERR_INVALID_ARGUMENT;
    D3G_TRY(ensure_device());
    cudaStream_t s = nullptr;
    DevBuf<double> d6;
    DevBuf<int8_t> dout;
    D3G_TRY(d6.alloc(size_t(6 * n_queries), s));
    D3G_TRY(dout.alloc(size_t(n_queries), s));
    D3G_CUDA(cudaMemcpyAsync(d6.p, six, sizeof(double) * 6 * n_queries, cudaMemcpyHostToDevice, s));
    D3G_TRY(orient2d_device(d6.p, n_queries, dout.p, s));
    D3G_CUDA(cudaMemcpyAsync(sign_out, dout.p, size_t(n_queries), cudaMemcpyDeviceToHost, s));
    D3G_CUDA(cudaStreamSynchronize(s));
    return D3G_OK;
}

}  // extern "C"
