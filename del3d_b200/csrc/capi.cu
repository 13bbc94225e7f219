// C ABI plumbing: status strings, error detail, host-pointer wrappers of the
// device entry points, synthetic input generators.
#include "common.cuh"

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
