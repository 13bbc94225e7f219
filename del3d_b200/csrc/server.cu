// Request server: triangulation requests of any size, submitted from any host
// thread, built on one GPU with continuous batching.
//
// The reference builds one point set per call on one CPU thread and has no
// serving layer; this is the serving form of the same build (the tet set of
// every request is the one d3g_build returns for it alone).
//
// Design
//   * `slots` worker threads, each with its own non-blocking CUDA stream, so up
//     to `slots` batches run on the device at once and overlap there.
//   * A slot that becomes free takes the request at the head of the queue and,
//     behind it in arrival order, the requests of a similar size (within a
//     factor 4) for as long as they fit: at most max_batch_sets requests and
//     max_batch_points points per batch, and the estimated device memory of
//     everything in flight within hbm_budget_bytes.  The head is never
//     overtaken (a large request is not starved; it waits at the head until
//     memory frees up); one larger than the whole budget runs alone once
//     nothing else is in flight.  Requests that arrive while batches run are admitted
//     as soon as a slot and memory free up: the batch is formed when a slot
//     is free, not when a fixed window closes.
//   * A batch is one d3g_build_batch-style build (points copied in on the
//     slot's stream, tet tables, rounds and output on the device); each
//     request's cells are copied back to its own host buffer.  If a batch
//     fails (for instance one request holds a non-finite coordinate), each of
//     its requests is rebuilt alone so that only the bad one reports the error.
#include "build_api.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace d3g {
namespace {

/// Device bytes one batch needs, from its point count: tet tables (8 tets per
/// point at 57 B), per-worker scratch, spatial-sort and output-sort buffers,
/// plus the big-round scratch and small fixed buffers per batch.  Calibrated
/// against the pool's high-water mark (tests/test_server_gpu.py checks it).
constexpr int64_t kBytesPerPoint = 1600;
constexpr int64_t kBytesPerBatch = int64_t(160) << 20;

int64_t estimate_bytes(int64_t points) { return kBytesPerPoint * points; }

/// Batch formation: requests within a factor kSizeBand of the batch's first
/// request join it (and any request up to kSmallRequest points joins a batch
/// of small ones).
constexpr int64_t kSizeBand = 4;
constexpr int64_t kSmallRequest = 4096;

struct Request {
    int64_t ticket = 0;
    const double* xyz = nullptr;
    int64_t n = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int status = D3G_OK;
    std::string error;
    int32_t* cells = nullptr;
    int64_t n_cells = 0, n_vertices = 0;
    int32_t batch_sets = 0;
    bool done = false;
};

}  // namespace
}  // namespace d3g

struct d3g_server {
    d3g_server_options opt{};
    int device = 0;
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<d3g::Request*> queue;
    std::unordered_map<int64_t, d3g::Request*> requests;
    int64_t next_ticket = 1;
    int64_t bytes_in_use = 0, peak_bytes = 0;
    int in_flight_batches = 0;
    int64_t in_flight_requests = 0, peak_in_flight_requests = 0;
    int64_t submitted = 0, completed = 0, batches = 0, batched_requests = 0;
    bool stop = false;
    std::vector<std::thread> workers;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace d3g {
namespace {

void copy_error(Request* r, int status) {
    r->status = status;
    r->error = d3g_last_error();
}

/// Builds `batch` on `stream` and fills each request's result.  Returns the
/// status of the batch build (per-request statuses are set either way).
int run_batch(const std::vector<Request*>& batch, cudaStream_t stream) {
    NvtxRange nvtx_batch("d3g.server.batch");
    const int k = int(batch.size());
    std::vector<int64_t> off(size_t(k) + 1, 0);
    for (int i = 0; i < k; ++i) off[size_t(i) + 1] = off[size_t(i)] + batch[size_t(i)]->n;
    const int64_t total = off[size_t(k)];
    d3g_options o;
    d3g_options_default(&o);
    DeviceResult R;
    int st = D3G_OK;
    {
        DevBuf<double> dx;
        st = dx.alloc(size_t(3 * std::max<int64_t>(total, 1)), stream);
        for (int i = 0; st == D3G_OK && i < k; ++i) {
            const Request* r = batch[size_t(i)];
            if (r->n == 0) continue;
            const cudaError_t e = cudaMemcpyAsync(dx.p + 3 * off[size_t(i)], r->xyz, sizeof(double) * 3 * r->n,
                                                  cudaMemcpyHostToDevice, stream);
            if (e != cudaSuccess) {
                set_error(std::string("d3g_server: copy in: ") + cudaGetErrorString(e));
                st = D3G_ERR_CUDA;
            }
        }
        if (st == D3G_OK) st = build_on_stream(dx.p, off.data(), k, o, stream, R);
    }
    if (st == D3G_OK) {
        for (int i = 0; i < k && st == D3G_OK; ++i) {
            Request* r = batch[size_t(i)];
            const int64_t a = R.cell_off[size_t(i)], b = R.cell_off[size_t(i) + 1];
            r->n_cells = b - a;
            r->n_vertices = R.set_nv[size_t(i)];
            r->cells = static_cast<int32_t*>(host_result_alloc(sizeof(int4) * size_t(std::max<int64_t>(b - a, 1))));
            if (!r->cells) {
                set_error("d3g_server: host allocation failed");
                st = D3G_ERR_OOM;
                break;
            }
            if (b > a) {
                const cudaError_t e = cudaMemcpyAsync(r->cells, R.cells.p + a, sizeof(int4) * size_t(b - a),
                                                      cudaMemcpyDeviceToHost, stream);
                if (e != cudaSuccess) {
                    set_error(std::string("d3g_server: copy out: ") + cudaGetErrorString(e));
                    st = D3G_ERR_CUDA;
                }
            }
        }
        const cudaError_t e = cudaStreamSynchronize(stream);
        if (st == D3G_OK && e != cudaSuccess) {
            set_error(std::string("d3g_server: ") + cudaGetErrorString(e));
            st = D3G_ERR_CUDA;
        }
    }
    R.reset();
    cudaStreamSynchronize(stream);
    for (Request* r : batch) {
        r->batch_sets = k;
        if (st != D3G_OK) {
            host_result_free(r->cells);
            r->cells = nullptr;
            r->n_cells = r->n_vertices = 0;
            copy_error(r, st);
        } else {
            r->status = D3G_OK;
        }
    }
    return st;
}

void worker_main(d3g_server* sv) {
    cudaSetDevice(sv->device);
    cudaStream_t stream = nullptr;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) stream = nullptr;
    for (;;) {
        std::vector<Request*> batch;
        int64_t est = 0;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            auto admissible = [&]() {
                if (sv->queue.empty()) return false;
                const int64_t e = estimate_bytes(sv->queue.front()->n) + kBytesPerBatch;
                return sv->bytes_in_use + e <= sv->opt.hbm_budget_bytes || sv->in_flight_batches == 0;
            };
            sv->cv_work.wait(lk, [&]() { return (sv->stop && sv->queue.empty()) || admissible(); });
            if (sv->queue.empty()) break;
            int64_t pts = 0;
            est = kBytesPerBatch;
            const double t = sv->now();
            // The head of the queue always goes first (no request is overtaken
            // for good).  Behind it, only requests of a similar size join its
            // batch: a batch finishes with its largest set, so a small request
            // batched with a large one would wait for it.  Others keep their
            // place for the next free slot.
            Request* head = sv->queue.front();
            const int64_t lo = head->n / kSizeBand, hi = std::max<int64_t>(head->n * kSizeBand, kSmallRequest);
            for (auto it = sv->queue.begin(); it != sv->queue.end();) {
                Request* r = *it;
                const int64_t e = estimate_bytes(r->n);
                if (r != head) {
                    if (int64_t(batch.size()) >= sv->opt.max_batch_sets) break;
                    if (sv->bytes_in_use + est + e > sv->opt.hbm_budget_bytes) break;
                    if (r->n < lo || r->n > hi || pts + r->n > sv->opt.max_batch_points) {
                        ++it;
                        continue;
                    }
                }
                it = sv->queue.erase(it);
                r->t_admit = t;
                batch.push_back(r);
                pts += r->n;
                est += e;
            }
            sv->bytes_in_use += est;
            sv->peak_bytes = std::max(sv->peak_bytes, sv->bytes_in_use);
            sv->in_flight_batches += 1;
            sv->in_flight_requests += int64_t(batch.size());
            sv->peak_in_flight_requests = std::max(sv->peak_in_flight_requests, sv->in_flight_requests);
            sv->batches += 1;
            sv->batched_requests += int64_t(batch.size());
        }
        if (!stream) {
            set_error("d3g_server: could not create a stream");
            for (Request* r : batch) copy_error(r, D3G_ERR_CUDA);
        } else if (run_batch(batch, stream) != D3G_OK && batch.size() > 1) {
            for (Request* r : batch) {
                std::vector<Request*> one{r};
                run_batch(one, stream);
                r->batch_sets = int32_t(batch.size());
            }
        }
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            const double t = sv->now();
            for (Request* r : batch) {
                r->t_done = t;
                r->done = true;
            }
            sv->bytes_in_use -= est;
            sv->in_flight_batches -= 1;
            sv->in_flight_requests -= int64_t(batch.size());
            sv->completed += int64_t(batch.size());
        }
        sv->cv_done.notify_all();
        sv->cv_work.notify_all();
    }
    if (stream) cudaStreamDestroy(stream);
}

}  // namespace
}  // namespace d3g

using namespace d3g;

extern "C" {

void d3g_server_options_default(d3g_server_options* o) {
    if (!o) return;
    o->slots = 4;
    o->hbm_budget_bytes = 0;
    o->max_batch_sets = 1024;
    o->max_batch_points = int64_t(8) << 20;
    o->device = -1;
}

int d3g_server_create(const d3g_server_options* opts, d3g_server** out) {
    if (!out) return D3G_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    d3g_server_options o;
    d3g_server_options_default(&o);
    if (opts) o = *opts;
    if (o.slots < 1 || o.slots > 64 || o.max_batch_sets < 1 || o.max_batch_points < 1 || o.hbm_budget_bytes < 0) {
        set_error("d3g_server_create: slots must be 1..64, batch limits positive, budget >= 0");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    D3G_TRY(ensure_device());
    if (o.device >= 0) D3G_CUDA(cudaSetDevice(o.device));
    int dev = 0;
    D3G_CUDA(cudaGetDevice(&dev));
    D3G_TRY(prepare_device());
    if (o.hbm_budget_bytes == 0) {
        size_t free_b = 0, total_b = 0;
        D3G_CUDA(cudaMemGetInfo(&free_b, &total_b));
        o.hbm_budget_bytes = int64_t(free_b / 2);
    }
    o.device = dev;
    d3g_server* sv = new d3g_server();
    sv->opt = o;
    sv->device = dev;
    sv->t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < o.slots; ++i) sv->workers.emplace_back(worker_main, sv);
    *out = sv;
    return D3G_OK;
}

int d3g_server_submit(d3g_server* sv, const double* xyz, int64_t n, int64_t* ticket) {
    if (!sv || !ticket || n < 0 || (n > 0 && !xyz)) return D3G_ERR_INVALID_ARGUMENT;
    if (n > int64_t(INT32_MAX) / 8) {
        set_error("d3g_server_submit: request too large");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    Request* r = new Request();
    r->xyz = xyz;
    r->n = n;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stop) {
            delete r;
            set_error("d3g_server_submit: server is shutting down");
            return D3G_ERR_INVALID_ARGUMENT;
        }
        r->ticket = sv->next_ticket++;
        r->t_submit = sv->now();
        sv->requests[r->ticket] = r;
        sv->queue.push_back(r);
        sv->submitted += 1;
        *ticket = r->ticket;
    }
    sv->cv_work.notify_one();
    return D3G_OK;
}

int d3g_server_wait(d3g_server* sv, int64_t ticket, double timeout_s, d3g_request_result* out) {
    if (!sv || !out) return D3G_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof *out);
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->requests.find(ticket);
    if (it == sv->requests.end()) {
        set_error("d3g_server_wait: unknown or already collected ticket");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    Request* r = it->second;
    if (timeout_s < 0) {
        sv->cv_done.wait(lk, [&]() { return r->done; });
    } else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&]() { return r->done; })) {
        set_error("d3g_server_wait: not complete within the timeout");
        return D3G_ERR_NOT_READY;
    }
    sv->requests.erase(it);
    lk.unlock();
    out->status = r->status;
    out->n_points = r->n;
    out->n_vertices = r->n_vertices;
    out->n_cells = r->n_cells;
    out->cells = r->cells;
    out->t_submit = r->t_submit;
    out->t_admit = r->t_admit;
    out->t_done = r->t_done;
    out->batch_sets = r->batch_sets;
    const int st = r->status;
    if (st != D3G_OK) set_error(r->error);
    delete r;
    return st;
}

void d3g_request_result_free(d3g_request_result* r) {
    if (!r) return;
    host_result_free(r->cells);
    r->cells = nullptr;
    r->n_cells = 0;
}

int d3g_server_get_stats(d3g_server* sv, d3g_server_stats* out) {
    if (!sv || !out) return D3G_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(sv->mu);
    out->submitted = sv->submitted;
    out->completed = sv->completed;
    out->queued = int64_t(sv->queue.size());
    out->batches = sv->batches;
    out->batched_requests = sv->batched_requests;
    out->bytes_in_use = sv->bytes_in_use;
    out->peak_bytes_in_use = sv->peak_bytes;
    out->hbm_budget_bytes = sv->opt.hbm_budget_bytes;
    out->peak_in_flight_requests = sv->peak_in_flight_requests;
    out->slots = sv->opt.slots;
    return D3G_OK;
}

int d3g_server_destroy(d3g_server* sv) {
    if (!sv) return D3G_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    for (std::thread& t : sv->workers) t.join();
    for (auto& kv : sv->requests) {
        host_result_free(kv.second->cells);
        delete kv.second;
    }
    delete sv;
    return D3G_OK;
}

int d3g_pool_usage(int64_t* used, int64_t* used_high, int reset_high) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return D3G_ERR_NO_DEVICE;
    }
    cudaMemPool_t pool;
    D3G_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t u = 0, h = 0;
    D3G_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
    D3G_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &h));
    if (used) *used = int64_t(u);
    if (used_high) *used_high = int64_t(h);
    if (reset_high) {
        uint64_t zero = 0;
        D3G_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero));
    }
    return D3G_OK;
}

}  // extern "C"
