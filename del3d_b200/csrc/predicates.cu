// Batch predicate evaluation: the C ABI d3g_predicates / d3g_predicates_device.
//
// orient3d and in_sphere run in two kernels:
//   k_filter_*  one thread per query: gather the points, evaluate the filter;
//               certain queries write their sign, uncertain ones are appended
//               to a compacted queue with one warp-aggregated atomic per warp;
//   k_exact_*   one thread per queued query: the exact stage and, for
//               in_sphere, the symbolic perturbation.
// The filter kernel is bound by the point gathers (HBM/L2) and the FP64 pipe;
// the queue keeps the rare, long-running exact path out of its warps.
// The coplanar family, used only on hull-coplanar configurations, runs as one
// kernel per query.
#include "common.cuh"
#include "exact_wide.cuh"

#include <cuda.h>

#include <mutex>

namespace d3g {
namespace {

// The wide tier: at most this many calls queued per entry-point call (more
// report D3G_ERR_EXACT_CAPACITY), and this many evaluated at once (each with a
// kWideArenaLimbs piece of the arena: 148 KB).
constexpr int64_t kWideQueueCap = int64_t(1) << 20;
constexpr int64_t kWideSlots = 256;

__device__ __forceinline__ Pt load_pt(const double* __restrict__ pts, int32_t i) {
    const double* p = pts + 3 * int64_t(i);
    return Pt{__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}

__device__ __forceinline__ bool idx_ok(int32_t i, int64_t n) { return i >= 0 && int64_t(i) < n; }

/// Appends `q` to the queue if `push`; all lanes of the warp must call this.
__device__ __forceinline__ void warp_push(bool push, int64_t q, int64_t* queue,
                                          unsigned long long* count) {
    const unsigned mask = __ballot_sync(0xffffffffu, push);
    if (mask == 0) return;
    const int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == __ffs(mask) - 1) base = atomicAdd(count, (unsigned long long)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
    if (push) queue[base + __popc(mask & ((1u << lane) - 1u))] = q;
}

/// Limbs the exact stage needs for an orient3d / in_sphere call (0 when the
/// filter's own value is exact), as orient3d_degenerate / in_sphere_degenerate
/// choose them.
__device__ int orient3d_limbs(const Pt& a, const Pt& b, const Pt& c, const Pt& d) {
    Span s;
    s.add(a.x); s.add(a.y); s.add(a.z); s.add(b.x); s.add(b.y); s.add(b.z);
    s.add(c.x); s.add(c.y); s.add(c.z); s.add(d.x); s.add(d.y); s.add(d.z);
    return s.exact_in_double(3, 3) ? 0 : limbs_for(3 * (s.bits() + 1) + 3);
}
__device__ int in_sphere_limbs(const Pt& a, const Pt& b, const Pt& c, const Pt& d, const Pt& e) {
    Span s;
    s.add(a.x); s.add(a.y); s.add(a.z); s.add(b.x); s.add(b.y); s.add(b.z);
    s.add(c.x); s.add(c.y); s.add(c.z); s.add(d.x); s.add(d.y); s.add(d.z);
    s.add(e.x); s.add(e.y); s.add(e.z);
    return s.exact_in_double(5, 7) ? 0 : limbs_for(5 * (s.bits() + 1) + 7);
}

/// Queues query q for the wide tier (too wide for the exact stage's 16 limbs),
/// or reports the exact-stage capacity when the caller gave no wide queue (the
/// entry point that allocates nothing) or it is full.
__device__ void push_wide(int64_t q, int64_t* wq, unsigned long long* wcount, int64_t wcap, uint32_t* status) {
    if (!wq) {
        report(status, ST_EXACT_CAPACITY);
        return;
    }
    const unsigned long long k = atomicAdd(wcount, 1ull);
    if (int64_t(k) < wcap) wq[k] = q;
    else report(status, ST_EXACT_CAPACITY);
}

__global__ void __launch_bounds__(256) k_filter_orient3d(const double* __restrict__ pts, int64_t npts,
                                                         const int32_t* __restrict__ idx, int64_t nq,
                                                         int8_t* __restrict__ out, int64_t* queue,
                                                         unsigned long long* qcount, uint32_t* status) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t nq_pad = (nq + 31) & ~int64_t(31);
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nq_pad; q += stride) {
        bool push = false;
        if (q < nq) {
            const int4 t = *reinterpret_cast<const int4*>(idx + 4 * q);
            if (idx_ok(t.x, npts) && idx_ok(t.y, npts) && idx_ok(t.z, npts) && idx_ok(t.w, npts)) {
                const Orient3dFilter f = orient3d_filter(load_pt(pts, t.x), load_pt(pts, t.y),
                                                         load_pt(pts, t.z), load_pt(pts, t.w));
                out[q] = int8_t(f.certain ? -sign_of(f.det) : 0);
                push = !f.certain;
            } else {
                out[q] = 0;
                report(status, ST_INTERNAL);
            }
        }
        warp_push(push, q, queue, qcount);
    }
}

__global__ void __launch_bounds__(256) k_exact_orient3d(const double* __restrict__ pts,
                                                        const int32_t* __restrict__ idx,
                                                        int8_t* __restrict__ out,
                                                        const int64_t* __restrict__ queue,
                                                        const unsigned long long* qcount,
                                                        int64_t* wq, unsigned long long* wcount, int64_t wcap,
                                                        uint32_t* status) {
    const int64_t n = int64_t(*qcount);
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += int64_t(gridDim.x) * blockDim.x) {
        const int64_t q = queue[k];
        const int4 t = *reinterpret_cast<const int4*>(idx + 4 * q);
        const Pt a = load_pt(pts, t.x), b = load_pt(pts, t.y), c = load_pt(pts, t.z),
                 d = load_pt(pts, t.w);
        if (orient3d_limbs(a, b, c, d) > kMaxLimbs) {
            push_wide(q, wq, wcount, wcap, status);
            continue;
        }
        const Orient3dFilter f = orient3d_filter(a, b, c, d);
        out[q] = int8_t(orient3d_exact(a, b, c, d, f.det, status));
    }
}

__global__ void __launch_bounds__(256) k_filter_in_sphere(const double* __restrict__ pts, int64_t npts,
                                                          const int32_t* __restrict__ idx, int64_t nq,
                                                          int8_t* __restrict__ out, int64_t* queue,
                                                          unsigned long long* qcount, uint32_t* status) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t nq_pad = (nq + 31) & ~int64_t(31);
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nq_pad; q += stride) {
        bool push = false;
        if (q < nq) {
            const int32_t* t = idx + 5 * q;
            const int32_t i0 = t[0], i1 = t[1], i2 = t[2], i3 = t[3], i4 = t[4];
            if (idx_ok(i0, npts) && idx_ok(i1, npts) && idx_ok(i2, npts) && idx_ok(i3, npts) &&
                idx_ok(i4, npts)) {
                const InSphereFilter f =
                    in_sphere_filter(load_pt(pts, i0), load_pt(pts, i1), load_pt(pts, i2),
                                     load_pt(pts, i3), load_pt(pts, i4));
                out[q] = int8_t(f.certain ? -sign_of(f.det) : 0);
                push = !f.certain;
            } else {
                out[q] = 0;
                report(status, ST_INTERNAL);
            }
        }
        warp_push(push, q, queue, qcount);
    }
}

__global__ void __launch_bounds__(128) k_exact_in_sphere(const double* __restrict__ pts,
                                                         const int32_t* __restrict__ idx,
                                                         int8_t* __restrict__ out,
                                                         const int64_t* __restrict__ queue,
                                                         const unsigned long long* qcount,
                                                         int perturbed, int64_t* wq,
                                                         unsigned long long* wcount, int64_t wcap,
                                                         uint32_t* status) {
    const int64_t n = int64_t(*qcount);
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += int64_t(gridDim.x) * blockDim.x) {
        const int64_t q = queue[k];
        const int32_t* t = idx + 5 * q;
        const int64_t id[5] = {t[0], t[1], t[2], t[3], t[4]};
        const Pt a = load_pt(pts, t[0]), b = load_pt(pts, t[1]), c = load_pt(pts, t[2]),
                 d = load_pt(pts, t[3]), e = load_pt(pts, t[4]);
        // Too wide for 16 limbs: the wide tier (a tie-break then needs orient3d
        // calls of at most this width, so narrower calls never get there).
        if (in_sphere_limbs(a, b, c, d, e) > kMaxLimbs) {
            push_wide(q, wq, wcount, wcap, status);
            continue;
        }
        const InSphereFilter f = in_sphere_filter(a, b, c, d, e);
        const int s = in_sphere_degenerate(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, d.x, d.y, d.z, e.x, e.y,
                                           e.z, id[0], id[1], id[2], id[3], id[4], f.det, perturbed, status);
        out[q] = int8_t(s);
    }
}

// ---- the wide tier ------------------------------------------------------------
//
// Calls whose exact value needs more than the exact stage's 16 limbs (coordinate
// spans beyond about 200 binades in one in_sphere call, 330 in one orient3d
// call).  One thread per call, its integers in its own piece of an arena the
// host allocates for the calls queued (exact_wide.cuh); rare and slow by design,
// but every finite input gets the reference's sign.

/// orient3d for the tie-break of a wide in_sphere call: the filter, then the
/// exact stage's tiers, then the arena when 16 limbs are not enough.
struct Orient3dWide {
    Arena* arena;
    uint32_t* status;
    __device__ int operator()(const Pt& A, const Pt& B, const Pt& C, const Pt& D) const {
        const Orient3dFilter f = orient3d_filter(A, B, C, D);
        if (f.certain) return -sign_of(f.det);
        const int L = orient3d_limbs(A, B, C, D);
        if (L <= kMaxLimbs) return orient3d_exact(A, B, C, D, f.det, status);
        Span s;
        s.add(A.x); s.add(A.y); s.add(A.z); s.add(B.x); s.add(B.y); s.add(B.z);
        s.add(C.x); s.add(C.y); s.add(C.z); s.add(D.x); s.add(D.y); s.add(D.z);
        const int64_t mark = arena->used;
        const int r = orient3d_num<WideG>(A, B, C, D, NumFrom<WideG>{s.emin, L, arena});
        if (!arena->overflow) arena->used = mark;
        return r;
    }
};

__global__ void __launch_bounds__(64) k_wide_orient3d(const double* __restrict__ pts, const int32_t* __restrict__ idx,
                                                      int8_t* __restrict__ out, const int64_t* __restrict__ wq,
                                                      int64_t first, int64_t count, uint64_t* arena,
                                                      int64_t arena_limbs, uint32_t* status) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t q = wq[first + k];
    const int4 t = *reinterpret_cast<const int4*>(idx + 4 * q);
    Arena A{arena + k * arena_limbs, arena_limbs, 0, false};
    const int s = Orient3dWide{&A, status}(load_pt(pts, t.x), load_pt(pts, t.y), load_pt(pts, t.z),
                                           load_pt(pts, t.w));
    if (A.overflow) report(status, ST_EXACT_CAPACITY);
    out[q] = int8_t(s);
}

__global__ void __launch_bounds__(64) k_wide_in_sphere(const double* __restrict__ pts, const int32_t* __restrict__ idx,
                                                       int8_t* __restrict__ out, const int64_t* __restrict__ wq,
                                                       int64_t first, int64_t count, int perturbed, uint64_t* arena,
                                                       int64_t arena_limbs, uint32_t* status) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t q = wq[first + k];
    const int32_t* t = idx + 5 * q;
    const Pt a = load_pt(pts, t[0]), b = load_pt(pts, t[1]), c = load_pt(pts, t[2]), d = load_pt(pts, t[3]),
             e = load_pt(pts, t[4]);
    Arena A{arena + k * arena_limbs, arena_limbs, 0, false};
    Span s;
    s.add(a.x); s.add(a.y); s.add(a.z); s.add(b.x); s.add(b.y); s.add(b.z);
    s.add(c.x); s.add(c.y); s.add(c.z); s.add(d.x); s.add(d.y); s.add(d.z);
    s.add(e.x); s.add(e.y); s.add(e.z);
    const int L = limbs_for(5 * (s.bits() + 1) + 7);
    int sign = in_sphere_num<WideG>(a, b, c, d, e, NumFrom<WideG>{s.emin, L, &A});
    if (!A.overflow) A.used = 0;
    if (sign == 0 && perturbed)
        sign = in_sphere_perturb_by(Orient3dWide{&A, status}, a, b, c, d, e, t[0], t[1], t[2], t[3], t[4]);
    if (A.overflow) report(status, ST_EXACT_CAPACITY);
    out[q] = int8_t(sign);
}

__global__ void __launch_bounds__(128) k_coplanar(const double* __restrict__ pts, int64_t npts,
                                                  const int32_t* __restrict__ idx, int64_t nq,
                                                  int kind, int8_t* __restrict__ out,
                                                  unsigned long long* nexact, uint32_t* status) {
    const int k = (kind == D3G_COPLANAR_ORIENTATION3 || kind == D3G_COLLINEAR) ? 3 : 4;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nq;
         q += int64_t(gridDim.x) * blockDim.x) {
        const int32_t* t = idx + k * q;
        bool ok = true;
        for (int j = 0; j < k; ++j) ok = ok && idx_ok(t[j], npts);
        if (!ok) {
            out[q] = 0;
            report(status, ST_INTERNAL);
            continue;
        }
        const Pt p0 = load_pt(pts, t[0]), p1 = load_pt(pts, t[1]), p2 = load_pt(pts, t[2]);
        int s = 0;
        switch (kind) {
            case D3G_COPLANAR_ORIENTATION3: s = coplanar_orientation3(p0, p1, p2, status); break;
            case D3G_COLLINEAR: s = collinear(p0, p1, p2, status) ? 1 : 0; break;
            case D3G_COPLANAR_ORIENTATION4:
                s = coplanar_orientation4(p0, p1, p2, load_pt(pts, t[3]), status);
                break;
            default: {
                const Pt p3 = load_pt(pts, t[3]);
                const InCircleFilter f = in_circle_filter(p0, p1, p2, p3);
                if (f.certain) {
                    s = sign_of(f.det);
                } else {
                    atomicAdd(nexact, 1ull);
                    s = in_circle_degenerate(p0.x, p0.y, p0.z, p1.x, p1.y, p1.z, p2.x, p2.y, p2.z, p3.x, p3.y,
                                             p3.z, t[0], t[1], t[2], t[3], f.det,
                                             kind == D3G_COPLANAR_IN_CIRCLE ? 1 : 0, status);
                }
            }
        }
        out[q] = int8_t(s);
    }
}

__global__ void k_orient2d(const double* __restrict__ six, int64_t nq, int8_t* __restrict__ out,
                           uint32_t* status) {
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nq;
         q += int64_t(gridDim.x) * blockDim.x) {
        const double* s = six + 6 * q;
        out[q] = int8_t(orient2d(s[0], s[1], s[2], s[3], s[4], s[5], status));
    }
}

}  // namespace

int predicates_device(const double* d_pts, int64_t n_pts, const int32_t* d_idx, int64_t nq, int kind,
                      int8_t* d_out, cudaStream_t stream, d3g_predicate_stats* stats) {
    if (nq < 0 || n_pts < 0 || d3g_predicate_arity(kind) == 0) {
        set_error("d3g_predicates: bad size or kind");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    if (nq == 0) {
        if (stats) *stats = d3g_predicate_stats{0, 0};
        return D3G_OK;
    }
    D3G_TRY(prepare_device());
    if (!d_pts || !d_idx || !d_out) {
        set_error("d3g_predicates: null pointer");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    if (kind == D3G_ORIENT3D && (reinterpret_cast<uintptr_t>(d_idx) & 15u) != 0) {
        set_error("d3g_predicates: orient3d index array must be 16-byte aligned");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    // Scratch: status word, queue counter, wide-queue counter, and the queues
    // of the exact stage and of its wide tier.
    DevBuf<unsigned long long> counters;
    D3G_TRY(counters.alloc(3, stream));
    D3G_CUDA(cudaMemsetAsync(counters.p, 0, 3 * sizeof(unsigned long long), stream));
    uint32_t* status = reinterpret_cast<uint32_t*>(counters.p);
    unsigned long long* qcount = counters.p + 1;
    unsigned long long* wcount = counters.p + 2;
    DevBuf<int64_t> queue, wqueue;
    const int64_t wcap = std::min<int64_t>(nq, kWideQueueCap);
    const int blk = 256;
    const bool queued = kind == D3G_ORIENT3D || kind == D3G_IN_SPHERE || kind == D3G_IN_SPHERE_UNPERTURBED;
    if (queued) {
        D3G_TRY(queue.alloc(size_t(nq), stream));
        D3G_TRY(wqueue.alloc(size_t(wcap), stream));
        const unsigned g = grid_for(nq, blk, int64_t(kNumSMs) * 16);
        if (kind == D3G_ORIENT3D) {
            k_filter_orient3d<<<g, blk, 0, stream>>>(d_pts, n_pts, d_idx, nq, d_out, queue.p, qcount,
                                                     status);
            k_exact_orient3d<<<kNumSMs * 4, 256, 0, stream>>>(d_pts, d_idx, d_out, queue.p, qcount, wqueue.p,
                                                             wcount, wcap, status);
        } else {
            k_filter_in_sphere<<<g, blk, 0, stream>>>(d_pts, n_pts, d_idx, nq, d_out, queue.p,
                                                      qcount, status);
            k_exact_in_sphere<<<kNumSMs * 8, 128, 0, stream>>>(d_pts, d_idx, d_out, queue.p, qcount,
                                                               kind == D3G_IN_SPHERE ? 1 : 0, wqueue.p, wcount,
                                                               wcap, status);
        }
    } else {
        k_coplanar<<<grid_for(nq, 128), 128, 0, stream>>>(d_pts, n_pts, d_idx, nq, kind, d_out,
                                                          qcount, status);
    }
    D3G_CUDA(cudaGetLastError());
    unsigned long long host_counters[3] = {0, 0, 0};
    D3G_CUDA(cudaMemcpyAsync(host_counters, counters.p, sizeof host_counters, cudaMemcpyDeviceToHost,
                             stream));
    queue.release();
    D3G_CUDA(cudaStreamSynchronize(stream));
    // The wide tier, for the calls queued: kWideSlots at a time, each thread
    // with its own piece of the arena.
    const int64_t nwide = std::min<int64_t>(int64_t(host_counters[2]), wcap);
    if (queued && nwide > 0 && (uint32_t(host_counters[0]) & ST_INTERNAL) == 0) {
        DevBuf<uint64_t> arena;
        const int64_t slots = std::min<int64_t>(nwide, kWideSlots);
        D3G_TRY(arena.alloc(size_t(slots) * size_t(kWideArenaLimbs), stream));
        for (int64_t first = 0; first < nwide; first += slots) {
            const int64_t cnt = std::min<int64_t>(slots, nwide - first);
            if (kind == D3G_ORIENT3D)
                k_wide_orient3d<<<unsigned((cnt + 63) / 64), 64, 0, stream>>>(d_pts, d_idx, d_out, wqueue.p, first,
                                                                           cnt, arena.p, kWideArenaLimbs, status);
            else
                k_wide_in_sphere<<<unsigned((cnt + 63) / 64), 64, 0, stream>>>(
                    d_pts, d_idx, d_out, wqueue.p, first, cnt, kind == D3G_IN_SPHERE ? 1 : 0, arena.p,
                    kWideArenaLimbs, status);
            D3G_CUDA(cudaGetLastError());
        }
        D3G_CUDA(cudaMemcpyAsync(host_counters, counters.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 stream));
        D3G_CUDA(cudaStreamSynchronize(stream));
    }
    wqueue.release();
    counters.release();
    if (stats) *stats = d3g_predicate_stats{nq, int64_t(host_counters[1])};
    const uint32_t bits = uint32_t(host_counters[0]);
    if (bits & ST_INTERNAL) {
        set_error("d3g_predicates: point index out of range");
        return D3G_ERR_INVALID_INPUT;
    }
    return status_from_bits(bits);
}

int orient2d_device(const double* d_six, int64_t nq, int8_t* d_out, cudaStream_t stream) {
    DevBuf<uint32_t> st;
    D3G_TRY(st.alloc(1, stream));
    D3G_CUDA(cudaMemsetAsync(st.p, 0, sizeof(uint32_t), stream));
    if (nq > 0) k_orient2d<<<grid_for(nq, 128), 128, 0, stream>>>(d_six, nq, d_out, st.p);
    D3G_CUDA(cudaGetLastError());
    uint32_t bits = 0;
    D3G_CUDA(cudaMemcpyAsync(&bits, st.p, sizeof bits, cudaMemcpyDeviceToHost, stream));
    st.release();
    D3G_CUDA(cudaStreamSynchronize(stream));
    return status_from_bits(bits);
}

// ---- the entry point that allocates nothing ---------------------------------
//
// Some callers cannot allocate device memory when they evaluate predicates: a
// framework whose caching allocator has reserved the whole device, or a code
// path where an allocation's implicit synchronisation or possible failure is not
// acceptable.  d3g_predicates_noalloc_device serves them: its exact-stage queue
// and counters live in the fixed array below instead of stream-ordered
// allocations.  The array exists once per device that loads this library and is
// held until the process exits.

namespace {

struct NoAllocScratch {
    unsigned long long counters[2];            // [0] status bits, [1] exact-stage queue length
    int64_t queue[D3G_NOALLOC_MAX_QUERIES];     // indices of the queries the filter left uncertain
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

/// Identity of the calling thread's current CUDA context (driver entry points
/// reached through the runtime, so no link to the driver library is needed);
/// false if it cannot be had.
bool current_context_id(unsigned long long* id) {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

/// The device address of g_noalloc_scratch on the current device.  In host
/// code the symbol is a host-side stand-in, not a device address, so it is
/// looked up with the device current (cudaGetSymbolAddress) on the first call
/// in each context of a device and cached.  The cache is keyed on the context's
/// identity as well as the device ordinal: after a cudaDeviceReset the module
/// is loaded again into a new context, where the array may sit elsewhere, and
/// the first call there looks it up anew.  Without a context identity (no
/// driver entry point) the address is looked up on every call.
int noalloc_scratch(NoAllocScratch** out) {
    static std::mutex mu;
    static NoAllocScratch* addr[64] = {};
    static unsigned long long ctx_of[64] = {};
    int dev = 0;
    const cudaError_t ge = cudaGetDevice(&dev);
    if (ge != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        set_error("d3g_predicates_noalloc_device: no usable current device");
        return D3G_ERR_NO_DEVICE;
    }
    unsigned long long ctx = 0;
    bool have_ctx = current_context_id(&ctx);
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev] || !have_ctx || ctx_of[dev] != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return D3G_ERR_CUDA;
        }
        // The lookup makes the device's primary context current if none was:
        // record the identity of the context the address belongs to.
        if (!have_ctx) have_ctx = current_context_id(&ctx);
        addr[dev] = static_cast<NoAllocScratch*>(p);
        ctx_of[dev] = have_ctx ? ctx : 0;
    }
    *out = addr[dev];
    return D3G_OK;
}

}  // namespace

int predicates_noalloc_device(const double* d_pts, int64_t n_pts, const int32_t* d_idx, int64_t nq,
                              int kind, int8_t* d_out, cudaStream_t stream,
                              d3g_predicate_stats* stats) {
    if (nq < 0 || n_pts < 0 || d3g_predicate_arity(kind) == 0) {
        set_error("d3g_predicates_noalloc_device: bad size or kind");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    if (nq > D3G_NOALLOC_MAX_QUERIES) {
        set_error("d3g_predicates_noalloc_device: at most D3G_NOALLOC_MAX_QUERIES (1048576) "
                  "queries per call");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    if (nq == 0) {
        if (stats) *stats = d3g_predicate_stats{0, 0};
        return D3G_OK;
    }
    if (!d_pts || !d_idx || !d_out) {
        set_error("d3g_predicates_noalloc_device: null pointer");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    if (kind == D3G_ORIENT3D && (reinterpret_cast<uintptr_t>(d_idx) & 15u) != 0) {
        set_error("d3g_predicates_noalloc_device: orient3d index array must be 16-byte aligned");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    NoAllocScratch* sc = nullptr;
    D3G_TRY(noalloc_scratch(&sc));
    // The array keeps the previous call's contents: the counters must start at zero.
    D3G_CUDA(cudaMemsetAsync(sc->counters, 0, sizeof sc->counters, stream));
    uint32_t* status = reinterpret_cast<uint32_t*>(&sc->counters[0]);
    unsigned long long* qcount = &sc->counters[1];
    const int blk = 256;
    if (kind == D3G_ORIENT3D || kind == D3G_IN_SPHERE || kind == D3G_IN_SPHERE_UNPERTURBED) {
        const unsigned g = grid_for(nq, blk, int64_t(kNumSMs) * 16);
        if (kind == D3G_ORIENT3D) {
            k_filter_orient3d<<<g, blk, 0, stream>>>(d_pts, n_pts, d_idx, nq, d_out, sc->queue, qcount,
                                                     status);
            k_exact_orient3d<<<kNumSMs * 4, 256, 0, stream>>>(d_pts, d_idx, d_out, sc->queue, qcount,
                                                             nullptr, nullptr, 0, status);
        } else {
            k_filter_in_sphere<<<g, blk, 0, stream>>>(d_pts, n_pts, d_idx, nq, d_out, sc->queue,
                                                      qcount, status);
            k_exact_in_sphere<<<kNumSMs * 8, 128, 0, stream>>>(
                d_pts, d_idx, d_out, sc->queue, qcount, kind == D3G_IN_SPHERE ? 1 : 0, nullptr, nullptr, 0,
                status);
        }
    } else {
        k_coplanar<<<grid_for(nq, 128), 128, 0, stream>>>(d_pts, n_pts, d_idx, nq, kind, d_out,
                                                          qcount, status);
    }
    D3G_CUDA(cudaGetLastError());
    unsigned long long host_counters[2] = {0, 0};
    D3G_CUDA(cudaMemcpyAsync(host_counters, sc->counters, sizeof host_counters,
                             cudaMemcpyDeviceToHost, stream));
    D3G_CUDA(cudaStreamSynchronize(stream));
    if (stats) *stats = d3g_predicate_stats{nq, int64_t(host_counters[1])};
    const uint32_t bits = uint32_t(host_counters[0]);
    if (bits & ST_INTERNAL) {
        set_error("d3g_predicates_noalloc_device: point index out of range");
        return D3G_ERR_INVALID_INPUT;
    }
    return status_from_bits(bits);
}

}  // namespace d3g

extern "C" int d3g_predicates_noalloc_device(const double* d_pts, int64_t n_pts, const int32_t* d_idx,
                                             int64_t n_queries, int kind, int8_t* d_sign_out,
                                             void* stream, d3g_predicate_stats* stats) {
    return d3g::predicates_noalloc_device(d_pts, n_pts, d_idx, n_queries, kind, d_sign_out,
                                          static_cast<cudaStream_t>(stream), stats);
}
