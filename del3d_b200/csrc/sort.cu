// Device insertion order: the reference's spatial_sort (src/spatial_sort.cpp,
// src/rand48.h), rebuilt as data-parallel passes.
//
// 1. Shuffle.  The reference runs a forward Fisher-Yates loop whose k-th step
//    swaps a[k] with a[j_k], j_k uniform in [0,k] drawn from a 48-bit LCG with
//    bucket-and-reject reduction (rand48.h:113-153).  Here:
//      * every LCG output is computed in parallel by affine jump-ahead;
//      * a draw can only be rejected if it lies in the top n values of the
//        31-bit range, so only those few "candidate" draws are compacted and
//        scanned in order by one thread, which fixes which draws are rejected
//        (and so which draw each step consumes);
//      * the permutation follows from the j_k without replaying the swaps: the
//        value that ends at position p is the last step m > p with j_m = p,
//        else what step p moved there - the predecessor of p among the steps
//        targeting j_p, or recursively what j_p held.  Each chain strictly
//        decreases, so a thread per position resolves it.
// 2. Multiscale split into levels [floor(n/8^(k+1)), floor(n/8^k)) while a
//    range holds at least 64 points (spatial_sort.cpp:130-137).
// 3. Within each level the points are ordered along a space-filling curve.
#include "device_util.cuh"

namespace d3g {
namespace {

constexpr uint64_t kA = 0x5DEECE66DULL;
constexpr uint64_t kC = 0xBULL;
constexpr uint64_t kMask = (1ULL << 48) - 1;
constexpr uint64_t kSeedState = (1ULL << 16) | 0x330EULL;   // Rand48() = seed(1)

struct Affine {
    uint64_t a, c;   // x -> a*x + c (mod 2^48)
};

__host__ __device__ inline Affine compose(const Affine& f, const Affine& g) {   // f after g
    return Affine{(f.a * g.a) & kMask, (f.a * g.c + f.c) & kMask};
}

struct JumpTable {
    Affine step[48];   // the LCG applied 2^i times
};

/// outs[t] = the (t+1)-th output of the reference engine, t in [0, T).
__global__ void k_draws(JumpTable jt, int64_t T, uint32_t* __restrict__ outs, int per_thread) {
    const int64_t t0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) * per_thread;
    if (t0 >= T) return;
    Affine f{1, 0};
    for (int i = 0; i < 48; ++i)
        if ((uint64_t(t0) >> i) & 1) f = compose(jt.step[i], f);
    uint64_t x = (f.a * kSeedState + f.c) & kMask;     // state after t0 steps
    const int64_t t1 = t0 + per_thread < T ? t0 + per_thread : T;
    for (int64_t t = t0; t < t1; ++t) {
        x = (kA * x + kC) & kMask;
        outs[t] = uint32_t(x >> 17);
    }
}

/// Flags the draws that could be rejected for some step k <= n-1.
__global__ void k_candidates(const uint32_t* __restrict__ outs, int64_t T, uint32_t threshold,
                             int32_t* __restrict__ cand, unsigned long long* ncand) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T;
         t += int64_t(gridDim.x) * blockDim.x) {
        if (outs[t] >= threshold) {
            const unsigned long long k = atomicAdd(ncand, 1ull);
            cand[k] = int32_t(t);
        }
    }
}

/// One thread: walks the (sorted) candidate draws in order and decides which
/// are rejected.  Draw t is consumed by step t + 1 - (rejections before t).
__global__ void k_reject_scan(const uint32_t* __restrict__ outs, const int32_t* __restrict__ cand,
                              const unsigned long long* ncand, int64_t n,
                              uint8_t* __restrict__ rejected, int64_t* nrej) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int64_t s = 0;
    const int64_t nc = int64_t(*ncand);
    for (int64_t i = 0; i < nc; ++i) {
        const int64_t t = cand[i];
        const int64_t k = t + 1 - s;
        if (k > n - 1) break;
        const uint64_t bucket = (uint64_t(1) << 31) / uint64_t(k + 1);
        if (uint64_t(outs[t]) / bucket > uint64_t(k)) {
            rejected[t] = 1;
            ++s;
        }
    }
    *nrej = s;
}

__global__ void k_accept_flags(const uint8_t* __restrict__ rejected, int64_t T,
                               int32_t* __restrict__ acc) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T;
         t += int64_t(gridDim.x) * blockDim.x)
        acc[t] = rejected[t] ? 0 : 1;
}

/// j[k] for k in [1, n): the k-th accepted draw reduced into [0, k].
__global__ void k_steps(const uint32_t* __restrict__ outs, const uint8_t* __restrict__ rejected,
                        const int32_t* __restrict__ accpos, int64_t T, int64_t n,
                        int32_t* __restrict__ j) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < T;
         t += int64_t(gridDim.x) * blockDim.x) {
        if (rejected[t]) continue;
        const int64_t k = int64_t(accpos[t]) + 1;
        if (k > n - 1) continue;
        const uint64_t bucket = (uint64_t(1) << 31) / uint64_t(k + 1);
        j[k] = int32_t(uint64_t(outs[t]) / bucket);
    }
}

__global__ void k_iota(int32_t* __restrict__ a, int64_t n, int32_t base) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        a[i] = int32_t(i) + base;
}

/// From the steps sorted by target (sj ascending, sm ascending within a
/// target): pred[m] = previous step with the same target, last[q] = final step
/// targeting q.
__global__ void k_lists(const int32_t* __restrict__ sj, const int32_t* __restrict__ sm, int64_t cnt,
                        int32_t* __restrict__ pred, int32_t* __restrict__ last) {
    for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < cnt;
         s += int64_t(gridDim.x) * blockDim.x) {
        const int32_t q = sj[s], m = sm[s];
        pred[m] = (s > 0 && sj[s - 1] == q) ? sm[s - 1] : -1;
        if (s + 1 == cnt || sj[s + 1] != q) last[q] = m;
    }
}

__global__ void k_final(const int32_t* __restrict__ j, const int32_t* __restrict__ pred,
                        const int32_t* __restrict__ last, int64_t n, int32_t* __restrict__ order) {
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        const int32_t l = last[p];
        if (l > p) {
            order[p] = l;
            continue;
        }
        int64_t x = p;
        int32_t v = 0;
        while (x > 0) {
            const int32_t q = j[x];
            if (q == x) { v = int32_t(x); break; }
            const int32_t pm = pred[x];
            if (pm > q) { v = pm; break; }
            x = q;
        }
        order[p] = v;
    }
}

// ---- placeholder in-level curve order: Morton keys inside BRIO levels ---------

__global__ void k_bbox(const double* __restrict__ xyz, int64_t n, unsigned long long* bb) {
    unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0, 0, 0};
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            const unsigned long long k = dbl_order_key(xyz[3 * i + a]);
            lo[a] = k < lo[a] ? k : lo[a];
            hi[a] = k > hi[a] ? k : hi[a];
        }
    for (int a = 0; a < 3; ++a) {
        atomicMin(bb + a, lo[a]);
        atomicMax(bb + 3 + a, hi[a]);
    }
}

__device__ __forceinline__ uint64_t spread3(uint64_t x) {   // 16 bits -> every third bit
    x &= 0xFFFF;
    x = (x | (x << 32)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 16)) & 0x00FF0000FF0000FFull;
    x = (x | (x << 8)) & 0xF00F00F00F00F00Full;
    x = (x | (x << 4)) & 0x30C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x9249249249249249ull;
    return x;
}

__global__ void k_level_morton(const double* __restrict__ xyz, const int32_t* __restrict__ order,
                               int64_t n, const unsigned long long* bb, const int64_t* bounds,
                               int nlev, uint64_t* __restrict__ keys) {
    double lo[3], ext[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = dbl_from_order_key(bb[a]);
        const double hi = dbl_from_order_key(bb[3 + a]);
        ext[a] = hi > lo[a] ? hi - lo[a] : 1.0;
    }
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        // Level: bounds[0] = n > bounds[1] > ... ; position p is in level k if
        // bounds[k+1] <= p < bounds[k]; the coarsest (highest k) goes first.
        int lvl = 0;
        while (lvl + 1 < nlev && p < bounds[lvl + 1]) ++lvl;
        const int64_t i = order[p];
        uint64_t m = 0;
        for (int a = 0; a < 3; ++a) {
            double u = (xyz[3 * i + a] - lo[a]) / ext[a];
            u = u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u);
            const uint64_t c = uint64_t(u * 65535.0);
            m |= spread3(c) << a;
        }
        keys[p] = (uint64_t(nlev - 1 - lvl) << 48) | m;
    }
}

}  // namespace

/// The reference's shuffled sequence (rand48.h:146-153 applied to 0..n-1).
int shuffle_device(int64_t n, int32_t* d_order, cudaStream_t s) {
    if (n <= 0) return D3G_OK;
    if (n == 1) {
        k_iota<<<1, 32, 0, s>>>(d_order, 1, 0);
        D3G_CUDA(cudaGetLastError());
        return D3G_OK;
    }
    JumpTable jt;
    jt.step[0] = Affine{kA, kC};
    for (int i = 1; i < 48; ++i) jt.step[i] = compose(jt.step[i - 1], jt.step[i - 1]);

    // Expected rejections ~ n^2 / 2^32; draw with a generous margin, retry if short.
    int64_t margin = 1024 + 4 * (int64_t)((double(n) * double(n)) / 4294967296.0);
    for (int attempt = 0; attempt < 6; ++attempt, margin *= 4) {
        const int64_t T = (n - 1) + margin;
        DevBuf<uint32_t> outs;
        DevBuf<int32_t> cand, acc, j, keys2, vals, vals2, pred, last;
        DevBuf<uint8_t> rej;
        DevBuf<unsigned long long> ncand;
        DevBuf<int64_t> nrej;
        D3G_TRY(outs.alloc(size_t(T), s));
        D3G_TRY(rej.alloc(size_t(T), s));
        D3G_TRY(ncand.alloc(1, s));
        D3G_TRY(nrej.alloc(1, s));
        D3G_CUDA(cudaMemsetAsync(rej.p, 0, size_t(T), s));
        D3G_CUDA(cudaMemsetAsync(ncand.p, 0, sizeof(unsigned long long), s));
        const int per = 64;
        k_draws<<<grid_for((T + per - 1) / per, 256, 1 << 30), 256, 0, s>>>(jt, T, outs.p, per);
        // A draw r can be rejected for step k only if r >= 2^31 - (k+1) > 2^31 - n - 1.
        const uint32_t threshold = uint32_t((uint64_t(1) << 31) - uint64_t(n) - 1);
        D3G_TRY(cand.alloc(size_t(T), s));
        k_candidates<<<grid_for(T, 256), 256, 0, s>>>(outs.p, T, threshold, cand.p, ncand.p);
        unsigned long long nc = 0;
        D3G_CUDA(cudaMemcpyAsync(&nc, ncand.p, sizeof nc, cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaStreamSynchronize(s));
        if (nc > 1) {   // order the candidates by draw index
            DevBuf<int32_t> sorted;
            D3G_TRY(sorted.alloc(size_t(nc), s));
            size_t bytes = 0;
            D3G_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, bytes, cand.p, sorted.p, int64_t(nc), 0,
                                                    bits_for(uint64_t(T)), s));
            DevBuf<char> tmp;
            D3G_TRY(tmp.alloc(bytes, s));
            D3G_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, bytes, cand.p, sorted.p, int64_t(nc), 0,
                                                    bits_for(uint64_t(T)), s));
            D3G_CUDA(cudaMemcpyAsync(cand.p, sorted.p, sizeof(int32_t) * nc, cudaMemcpyDeviceToDevice, s));
        }
        k_reject_scan<<<1, 32, 0, s>>>(outs.p, cand.p, ncand.p, n, rej.p, nrej.p);
        int64_t R = 0;
        D3G_CUDA(cudaMemcpyAsync(&R, nrej.p, sizeof R, cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaStreamSynchronize(s));
        if (T - R < n - 1) continue;   // not enough accepted draws: widen the margin

        D3G_TRY(acc.alloc(size_t(T), s));
        k_accept_flags<<<grid_for(T, 256), 256, 0, s>>>(rej.p, T, acc.p);
        D3G_TRY(exclusive_scan(acc.p, acc.p, T, s));
        D3G_TRY(j.alloc(size_t(n), s));
        k_steps<<<grid_for(T, 256), 256, 0, s>>>(outs.p, rej.p, acc.p, T, n, j.p);
        outs.release();
        rej.release();
        acc.release();
        cand.release();

        // Steps m = 1..n-1 sorted by target j_m (stable: m ascending within a target).
        const int64_t cnt = n - 1;
        D3G_TRY(keys2.alloc(size_t(cnt), s));
        D3G_TRY(vals.alloc(size_t(cnt), s));
        D3G_TRY(vals2.alloc(size_t(cnt), s));
        k_iota<<<grid_for(cnt, 256), 256, 0, s>>>(vals.p, cnt, 1);
        D3G_TRY(sort_pairs(j.p + 1, keys2.p, vals.p, vals2.p, cnt, 0, bits_for(uint64_t(n)), s));
        D3G_TRY(pred.alloc(size_t(n), s));
        D3G_TRY(last.alloc(size_t(n), s));
        D3G_CUDA(cudaMemsetAsync(last.p, 0xFF, sizeof(int32_t) * size_t(n), s));
        k_lists<<<grid_for(cnt, 256), 256, 0, s>>>(keys2.p, vals2.p, cnt, pred.p, last.p);
        k_final<<<grid_for(n, 256), 256, 0, s>>>(j.p, pred.p, last.p, n, d_order);
        D3G_CUDA(cudaGetLastError());
        return D3G_OK;
    }
    set_error("shuffle: rejection margin exhausted");
    return D3G_ERR_INTERNAL;
}

/// Level boundaries of the multiscale pass: b[0] = n, b[k+1] = floor(b[k]/8)
/// while b[k] >= 64 (spatial_sort.cpp:130-137; the ratio 0.125 is exact).
int multiscale_bounds(int64_t n, int64_t* b, int cap) {
    int k = 0;
    b[k++] = n;
    while (k < cap && b[k - 1] >= 64) {
        b[k] = int64_t(double(b[k - 1]) * 0.125);
        ++k;
    }
    return k;   // levels: [b[k+1], b[k]) for k < count-1, plus [0, b[count-1])
}

int spatial_order_device(const double* d_xyz, int64_t n, int32_t* d_order, cudaStream_t s) {
    if (n <= 0) return D3G_OK;
    D3G_TRY(shuffle_device(n, d_order, s));
    if (n < 2) return D3G_OK;
    int64_t hb[64];
    const int nb = multiscale_bounds(n, hb, 63);
    DevBuf<int64_t> bounds;
    DevBuf<unsigned long long> bb;
    DevBuf<uint64_t> keys, keys2;
    DevBuf<int32_t> tmp;
    D3G_TRY(bounds.alloc(size_t(nb), s));
    D3G_TRY(bb.alloc(6, s));
    D3G_CUDA(cudaMemcpyAsync(bounds.p, hb, sizeof(int64_t) * nb, cudaMemcpyHostToDevice, s));
    const unsigned long long init[6] = {~0ull, ~0ull, ~0ull, 0, 0, 0};
    D3G_CUDA(cudaMemcpyAsync(bb.p, init, sizeof init, cudaMemcpyHostToDevice, s));
    k_bbox<<<grid_for(n, 256, kNumSMs * 4), 256, 0, s>>>(d_xyz, n, bb.p);
    D3G_TRY(keys.alloc(size_t(n), s));
    D3G_TRY(keys2.alloc(size_t(n), s));
    D3G_TRY(tmp.alloc(size_t(n), s));
    k_level_morton<<<grid_for(n, 256), 256, 0, s>>>(d_xyz, d_order, n, bb.p, bounds.p, nb, keys.p);
    D3G_TRY(sort_pairs(keys.p, keys2.p, d_order, tmp.p, n, 0, 48 + bits_for(uint64_t(nb)), s));
    D3G_CUDA(cudaMemcpyAsync(d_order, tmp.p, sizeof(int32_t) * size_t(n), cudaMemcpyDeviceToDevice, s));
    D3G_CUDA(cudaGetLastError());
    return D3G_OK;
}

}  // namespace d3g

using namespace d3g;

extern "C" {

/// The shuffled index sequence alone (the first stage of spatial_sort); exposed
/// for testing the rand48 emulation.
int d3g_shuffle_device(int64_t n, int32_t* d_order, void* stream) {
    if (n < 0 || (n > 0 && !d_order)) return D3G_ERR_INVALID_ARGUMENT;
    const int st = shuffle_device(n, d_order, static_cast<cudaStream_t>(stream));
    if (st != D3G_OK) return st;
    if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) return D3G_ERR_CUDA;
    return D3G_OK;
}

int d3g_spatial_sort_device(const double* d_xyz, int64_t n, int32_t* d_order, void* stream) {
    if (n < 0 || (n > 0 && (!d_xyz || !d_order))) return D3G_ERR_INVALID_ARGUMENT;
    const int st = spatial_order_device(d_xyz, n, d_order, static_cast<cudaStream_t>(stream));
    if (st != D3G_OK) return st;
    if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) return D3G_ERR_CUDA;
    return D3G_OK;
}

int d3g_spatial_sort(const double* xyz, int64_t n, int32_t* order) {
    if (n < 0 || (n > 0 && (!xyz || !order))) return D3G_ERR_INVALID_ARGUMENT;
    if (n == 0) return D3G_OK;
    D3G_TRY(ensure_device());
    cudaStream_t s = nullptr;
    DevBuf<double> dx;
    DevBuf<int32_t> dord;
    D3G_TRY(dx.alloc(size_t(3 * n), s));
    D3G_TRY(dord.alloc(size_t(n), s));
    D3G_CUDA(cudaMemcpyAsync(dx.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    D3G_TRY(spatial_order_device(dx.p, n, dord.p, s));
    D3G_CUDA(cudaMemcpyAsync(order, dord.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    D3G_CUDA(cudaStreamSynchronize(s));
    return D3G_OK;
}

}  // extern "C"
