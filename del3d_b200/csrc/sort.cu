// Device insertion order: the reference's spatial_sort (src/spatial_sort.cpp,
// src/rand48.h), rebuilt as data-parallel passes.
//
// 1. Shuffle.  The reference runs a forward Fisher-Yates loop whose k-th step
//    swaps a[k] with a[j_k], j_k uniform in [0,k] drawn from a 48-bit LCG with
//    bucket-and-reject reduction (rand48.h:113-153).  Here:
//      * every LCG output is computed in parallel by affine jump-ahead;
//      * a draw can only be rejected if it lies in the top n values of the
//        31-bit range, so only those few "candidate" draws are compacted and
//        scanned in order by one thread (from tiles a block stages in shared
//        memory), which fixes which draws are rejected (and so which draw each
//        step consumes);
//      * the permutation follows from the j_k without replaying the swaps: the
//        value that ends at position p is the last step m > p with j_m = p,
//        else what step p moved there - the predecessor of p among the steps
//        targeting j_p, or recursively what j_p held.  Each chain strictly
//        decreases, so a thread per position resolves it.
// 2. Multiscale split into levels [floor(n/8^(k+1)), floor(n/8^k)) while a
//    range holds at least 64 points (spatial_sort.cpp:130-137).
// 3. Each level is ordered by the reference's Hilbert median splits, bit for bit
//    (see k_select / k_small_sort below).
#include "device_util.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

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

/// Walks the (sorted) candidate draws in order and decides which are rejected:
/// draw t is consumed by step k = t + 1 - (rejections before t) and rejected if
/// r / (2^31 / (k + 1)) > k (rand48.h:115-127).  The decisions chain through the
/// rejection count, so one thread makes them; the block first stages a tile of
/// candidates and their draws in shared memory, so that the thread's loop waits
/// on no global load.  A draw below 2^31 - k is accepted without the division:
/// the rejected range, 2^31 mod (k + 1) values at the top, holds at most k.
constexpr int kRejectTile = 4096;
__global__ void __launch_bounds__(1024) k_reject_scan(const uint32_t* __restrict__ outs,
                                                      const int32_t* __restrict__ cand,
                                                      const unsigned long long* ncand, int64_t n,
                                                      uint8_t* __restrict__ rejected, int64_t* nrej) {
    __shared__ uint32_t val[kRejectTile];
    __shared__ int32_t pos[kRejectTile];
    __shared__ long long s_total;
    __shared__ int stop;
    const int64_t nc = int64_t(*ncand);
    if (threadIdx.x == 0) {
        s_total = 0;
        stop = 0;
    }
    __syncthreads();
    for (int64_t base = 0; base < nc && !stop; base += kRejectTile) {
        const int cnt = int(nc - base < kRejectTile ? nc - base : kRejectTile);
        for (int i = int(threadIdx.x); i < cnt; i += blockDim.x) {
            const int32_t t = cand[base + i];
            pos[i] = t;
            val[i] = outs[t];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t s = s_total;
            for (int i = 0; i < cnt; ++i) {
                const int64_t t = pos[i];
                const int64_t k = t + 1 - s;
                if (k > n - 1) {
                    stop = 1;
                    break;
                }
                const uint32_t r = val[i];
                if (r < (1u << 31) - uint32_t(k)) continue;
                const uint64_t bucket = (uint64_t(1) << 31) / uint64_t(k + 1);
                if (uint64_t(r) / bucket > uint64_t(k)) {
                    rejected[t] = 1;
                    ++s;
                }
            }
            s_total = s;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *nrej = s_total;
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

/// Index of the set holding global position g: offsets[s] <= g < offsets[s+1].
__device__ __forceinline__ int set_of(const int64_t* __restrict__ off, int nsets, int64_t g) {
    int lo = 0, hi = nsets - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

/// First and last position of each target in the steps sorted by target.
__global__ void k_target_ranges(const int32_t* __restrict__ sj, int64_t cnt, int32_t* __restrict__ tfirst,
                                int32_t* __restrict__ tlast) {
    for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < cnt;
         s += int64_t(gridDim.x) * blockDim.x) {
        const int32_t q = sj[s];
        if (s == 0 || sj[s - 1] != q) tfirst[q] = int32_t(s);
        if (s + 1 == cnt || sj[s + 1] != q) tlast[q] = int32_t(s);
    }
}

/// The shuffled sequence of every set at once.  All sets consume the same
/// prefix of the one engine stream (seeded to 1 for each spatial_sort call),
/// so the step targets j are shared; a set of n points stops at step n-1, which
/// only changes which steps count as "later".
__global__ void k_final_sets(const int32_t* __restrict__ j, const int32_t* __restrict__ pred,
                             const int32_t* __restrict__ sm, const int32_t* __restrict__ tfirst,
                             const int32_t* __restrict__ tlast, const int64_t* __restrict__ off,
                             int nsets, int64_t total, int32_t* __restrict__ order) {
    for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int s = set_of(off, nsets, g);
        const int64_t p = g - off[s];
        const int64_t n = off[s + 1] - off[s];
        // The last step m < n that targets p.
        int32_t l = -1;
        int lo = tfirst[p], hi = tlast[p];
        if (lo >= 0) {
            while (lo <= hi) {
                const int mid = (lo + hi) >> 1;
                if (sm[mid] < n) {
                    l = sm[mid];
                    lo = mid + 1;
                } else {
                    hi = mid - 1;
                }
            }
        }
        if (l > p) {
            order[g] = l;
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
        order[g] = v;
    }
}

/// Sets of at most this many points are shuffled by the reference's loop itself,
/// one thread per set over the set's sequence in shared memory: for a few
/// thousand points that is far quicker than the parallel machinery above,
/// whose fixed cost is several kernels and host round trips.
constexpr int kSerialShuffleMax = 8192;

/// rand48.h:146-153 with the engine seeded to 1, verbatim: element k (1..n-1)
/// swapped with element j drawn uniformly from [0, k] by the bucket reduction of
/// rand48.h:115-127 (draw r, j = r / (2^31 / (k+1)), redrawn while j > k).
__global__ void k_shuffle_serial(const int64_t* __restrict__ off, int32_t* __restrict__ order) {
    __shared__ int32_t a[kSerialShuffleMax];
    const int s = blockIdx.x;
    const int64_t base = off[s];
    const int n = int(off[s + 1] - base);
    for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = i;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t x = kSeedState;
        for (int k = 1; k < n; ++k) {
            const uint32_t bucket = uint32_t((uint64_t(1) << 31) / uint64_t(k + 1));
            uint32_t j;
            do {
                x = (kA * x + kC) & kMask;
                j = uint32_t(x >> 17) / bucket;
            } while (j > uint32_t(k));
            const int32_t t = a[k];
            a[k] = a[j];
            a[j] = t;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) order[base + i] = a[i];
}

// ---- the Hilbert median splits (spatial_sort.cpp:40-117) -------------------------
//
// Every split position is begin + (end - begin) / 2 whatever the data, so the
// host knows the whole recursion tree in advance and only the permutations need
// the device.  Ranges of more than kSmall points are split by k_select, one
// block per quickselect task; smaller ranges finish their whole recursion in
// shared memory (k_small_sort).

constexpr int kSelThreads = 512;
constexpr int kSmall = 1024;

/// The points being ordered: index plus coordinates, structure of arrays.
struct Elems {
    int32_t* idx;
    double* x;
    double* y;
    double* z;
};

__device__ __forceinline__ double coord(const Elems& E, int axis, int j) {
    return axis == 0 ? E.x[j] : (axis == 1 ? E.y[j] : E.z[j]);
}

__device__ __forceinline__ void move(const Elems& from, int i, const Elems& to, int j) {
    to.idx[j] = from.idx[i];
    to.x[j] = from.x[i];
    to.y[j] = from.y[i];
    to.z[j] = from.z[i];
}

/// The reference's Cmp (spatial_sort.cpp:25-36) called as cmp(element, pivot).
__device__ __forceinline__ bool before_pivot(double c, double p, int up) {
    return up ? (p < c) : (c < p);
}

struct SelTask {
    int left, end, nth, axis, up;   // nth_element_deterministic on [left, end)
};

/// One block per task: the reference's middle-pivot quickselect
/// (spatial_sort.cpp:60-71), each Lomuto partition (:40-51) done in parallel.
/// A Lomuto pass moves the elements that compare before the pivot to the front
/// in their original order; the others end up rotated: the element that lands
/// on a "not before" slot q is the one scanned at q if that one was not before
/// the pivot, and otherwise - the before-element at q having been swapped out to
/// its rank position - whatever landed there, recursively.  Those chains are
/// disjoint and strictly decreasing, and each thread follows its own.
__global__ void __launch_bounds__(kSelThreads) k_select(const SelTask* __restrict__ tasks, Elems E,
                                                         Elems B, int32_t* __restrict__ rk) {
    typedef cub::BlockScan<int, kSelThreads> BlockScan;
    __shared__ typename BlockScan::TempStorage scan_tmp;
    const SelTask t = tasks[blockIdx.x];
    if (t.end - t.left < 2) return;
    int left = t.left, right = t.end - 1;
    for (;;) {
        const int pm = left + (right - left) / 2;
        __syncthreads();
        if (threadIdx.x == 0 && pm != right) {
            move(E, pm, B, right);          // B as a one-element temporary
            move(E, right, E, pm);
            move(B, right, E, right);
        }
        __syncthreads();
        const double P = coord(E, t.axis, right);
        int running = 0;
        for (int base = left; base < right; base += kSelThreads) {
            const int j = base + int(threadIdx.x);
            int less = 0;
            if (j < right) less = before_pivot(coord(E, t.axis, j), P, t.up) ? 1 : 0;
            int excl = 0, total = 0;
            BlockScan(scan_tmp).ExclusiveSum(less, excl, total);
            __syncthreads();
            if (j < right) {
                rk[j] = less ? running + excl : -1;
                if (less) move(E, j, B, left + running + excl);
            }
            running += total;
        }
        const int L = running;
        __syncthreads();
        for (int q = left + L + int(threadIdx.x); q < right; q += kSelThreads) {
            int x = q;
            while (rk[x] >= 0) x = left + rk[x];
            move(E, x, B, q == left + L ? right : q);
        }
        if (threadIdx.x == 0) move(E, right, B, left + L);
        __syncthreads();
        for (int j = left + int(threadIdx.x); j <= right; j += kSelThreads) move(B, j, E, j);
        const int np = left + L;
        if (np == t.nth) break;
        if (t.nth < np) right = np - 1;
        else left = np + 1;
    }
}

// ---- the same quickselect across the whole GPU, for tasks too big for a block ----
//
// While a phase has tasks longer than kBlockSelectMax, each Lomuto pass of every
// such task is spread over tiles of kTile elements: count the elements before
// the pivot per tile, scan the counts, scatter them stably, resolve the rotated
// rest by the same chains as k_select, copy back, update the range.  Tasks that
// have shrunk below the limit are finished by k_select.

constexpr int kTile = 1024;
constexpr int kTileThreads = 256;
constexpr int kBlockSelectMax = 1 << 16;

struct TaskState {
    int left, right, nth, axis, up, done;
    double pivot;
    int tile0, ntiles, L;
};

__device__ __forceinline__ int task_of_tile(const TaskState* __restrict__ ts, int ntask, int tile) {
    int lo = 0, hi = ntask - 1;
    while (lo < hi) {   // last task whose first tile <= tile
        const int mid = (lo + hi + 1) >> 1;
        if (ts[mid].tile0 <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

/// One block: pivot swap of every active task, tile counts and first tiles.
__global__ void __launch_bounds__(1024) k_plan(TaskState* ts, int ntask, Elems E, Elems B, int* total) {
    typedef cub::BlockScan<int, 1024> BlockScan;
    __shared__ typename BlockScan::TempStorage tmp;
    int running = 0;
    for (int base = 0; base < ntask; base += 1024) {
        const int t = base + int(threadIdx.x);
        int tiles = 0;
        if (t < ntask && !ts[t].done) {
            TaskState& k = ts[t];
            const int pm = k.left + (k.right - k.left) / 2;
            if (pm != k.right) {
                move(E, pm, B, k.right);
                move(E, k.right, E, pm);
                move(B, k.right, E, k.right);
            }
            k.pivot = coord(E, k.axis, k.right);
            tiles = (k.right - k.left + kTile - 1) / kTile;
        }
        int excl = 0, sum = 0;
        BlockScan(tmp).ExclusiveSum(tiles, excl, sum);
        __syncthreads();
        if (t < ntask) {
            ts[t].tile0 = running + excl;
            ts[t].ntiles = tiles;
        }
        running += sum;
    }
    if (threadIdx.x == 0) *total = running;
}

__global__ void __launch_bounds__(kTileThreads) k_tile_count(const TaskState* __restrict__ ts, int ntask,
                                                             Elems E, const int* total,
                                                             int* __restrict__ tile_less) {
    typedef cub::BlockReduce<int, kTileThreads> BlockReduce;
    __shared__ typename BlockReduce::TempStorage tmp;
    const int T = *total;
    for (int tile = blockIdx.x; tile < T; tile += gridDim.x) {
        const TaskState& k = ts[task_of_tile(ts, ntask, tile)];
        const int b = k.left + (tile - k.tile0) * kTile;
        const int e = min(b + kTile, k.right);
        int c = 0;
        for (int j = b + int(threadIdx.x); j < e; j += kTileThreads)
            c += before_pivot(coord(E, k.axis, j), k.pivot, k.up) ? 1 : 0;
        const int sum = BlockReduce(tmp).Sum(c);
        if (threadIdx.x == 0) tile_less[tile] = sum;
        __syncthreads();
    }
}

/// One block: exclusive scan of the tile counts; each task's L.
__global__ void __launch_bounds__(1024) k_tile_scan(TaskState* ts, int ntask, const int* total,
                                                    int* tile_less) {
    typedef cub::BlockScan<int, 1024> BlockScan;
    __shared__ typename BlockScan::TempStorage tmp;
    const int T = *total;
    int running = 0;
    for (int base = 0; base < T; base += 1024) {
        const int i = base + int(threadIdx.x);
        const int v = i < T ? tile_less[i] : 0;
        int excl = 0, sum = 0;
        BlockScan(tmp).ExclusiveSum(v, excl, sum);
        __syncthreads();
        if (i < T) tile_less[i] = running + excl;   // now: elements before the pivot ahead of the tile
        running += sum;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < ntask; t += 1024) {
        TaskState& k = ts[t];
        if (k.done) continue;
        const int first = k.tile0, last = k.tile0 + k.ntiles;    // tiles [first, last)
        const int end_off = last < T ? tile_less[last] : running;
        k.L = end_off - tile_less[first];
    }
}

__global__ void __launch_bounds__(kTileThreads) k_tile_scatter(const TaskState* __restrict__ ts, int ntask,
                                                               Elems E, Elems B, const int* total,
                                                               const int* __restrict__ tile_off,
                                                               int32_t* __restrict__ rk) {
    typedef cub::BlockScan<int, kTileThreads> BlockScan;
    __shared__ typename BlockScan::TempStorage tmp;
    const int T = *total;
    for (int tile = blockIdx.x; tile < T; tile += gridDim.x) {
        const TaskState& k = ts[task_of_tile(ts, ntask, tile)];
        const int b = k.left + (tile - k.tile0) * kTile;
        const int e = min(b + kTile, k.right);
        int running = tile_off[tile] - tile_off[k.tile0];
        for (int base = b; base < e; base += kTileThreads) {
            const int j = base + int(threadIdx.x);
            int less = 0;
            if (j < e) less = before_pivot(coord(E, k.axis, j), k.pivot, k.up) ? 1 : 0;
            int excl = 0, sum = 0;
            BlockScan(tmp).ExclusiveSum(less, excl, sum);
            __syncthreads();
            if (j < e) {
                rk[j] = less ? running + excl : -1;
                if (less) move(E, j, B, k.left + running + excl);
            }
            running += sum;
        }
    }
}

__global__ void __launch_bounds__(kTileThreads) k_tile_place(const TaskState* __restrict__ ts, int ntask,
                                                             Elems E, Elems B, const int* total,
                                                             const int32_t* __restrict__ rk) {
    const int T = *total;
    for (int tile = blockIdx.x; tile < T; tile += gridDim.x) {
        const TaskState& k = ts[task_of_tile(ts, ntask, tile)];
        const int b = k.left + (tile - k.tile0) * kTile;
        const int e = min(b + kTile, k.right);
        const int first_ge = k.left + k.L;
        for (int q = max(b, first_ge) + int(threadIdx.x); q < e; q += kTileThreads) {
            int x = q;
            while (rk[x] >= 0) x = k.left + rk[x];
            move(E, x, B, q == first_ge ? k.right : q);
        }
    }
}

__global__ void k_tile_pivot(const TaskState* __restrict__ ts, int ntask, Elems E, Elems B) {
    for (int t = int(blockIdx.x) * blockDim.x + threadIdx.x; t < ntask; t += gridDim.x * blockDim.x)
        if (!ts[t].done) move(E, ts[t].right, B, ts[t].left + ts[t].L);
}

__global__ void __launch_bounds__(kTileThreads) k_tile_copy(const TaskState* __restrict__ ts, int ntask,
                                                            Elems E, Elems B, const int* total) {
    const int T = *total;
    for (int tile = blockIdx.x; tile < T; tile += gridDim.x) {
        const TaskState& k = ts[task_of_tile(ts, ntask, tile)];
        const int b = k.left + (tile - k.tile0) * kTile;
        const int e = min(b + kTile, k.right);
        for (int j = b + int(threadIdx.x); j < e; j += kTileThreads) move(B, j, E, j);
    }
}

/// Per task: the pivot slot, the new range; counts the tasks still too big.
__global__ void k_tile_update(TaskState* ts, int ntask, Elems E, Elems B, int* big_left) {
    for (int t = int(blockIdx.x) * blockDim.x + threadIdx.x; t < ntask; t += gridDim.x * blockDim.x) {
        TaskState& k = ts[t];
        if (k.done) continue;
        move(B, k.right, E, k.right);
        const int np = k.left + k.L;
        if (np == k.nth) k.done = 1;
        else if (k.nth < np) k.right = np - 1;
        else k.left = np + 1;
        if (!k.done && k.left == k.right) k.done = 1;
        if (!k.done && k.right - k.left + 1 > kBlockSelectMax) atomicAdd(big_left, 1);
    }
}

__global__ void k_to_seltask(const TaskState* __restrict__ ts, int ntask, SelTask* out) {
    for (int t = int(blockIdx.x) * blockDim.x + threadIdx.x; t < ntask; t += gridDim.x * blockDim.x) {
        const TaskState& k = ts[t];
        out[t] = SelTask{k.left, k.done ? k.left : k.right + 1, k.nth, k.axis, k.up};
    }
}

struct Seg {
    int begin, end, x, ux, uy, uz;   // recursive_sort(begin, end, x, upx, upy, upz)
};

/// A range of at most kSmall points in shared memory: coordinates and indices
/// stay where they were loaded; the splits permute `perm`, the range's order
/// (position -> loaded slot).
struct Local {
    const double* c[3];
    uint16_t* perm;
};

__device__ __forceinline__ double local_coord(const Local& L, int axis, int j) {
    return L.c[axis][L.perm[j]];
}

__device__ __forceinline__ void local_swap(Local& L, int i, int j) {
    const uint16_t t = L.perm[i];
    L.perm[i] = L.perm[j];
    L.perm[j] = t;
}

/// spatial_sort.cpp:40-79, verbatim in shared memory by one lane; [begin, end).
__device__ int local_split(Local& L, int begin, int end, int axis, int up) {
    if (begin >= end) return begin;
    const int middle = begin + (end - begin) / 2;
    int left = begin, right = end - 1;
    if (left == right) return middle;
    for (;;) {
        const int pm = left + (right - left) / 2;
        local_swap(L, pm, right);
        const double P = local_coord(L, axis, right);
        int result = left;
        for (int it = left; it != right; ++it) {
            if (before_pivot(local_coord(L, axis, it), P, up)) {
                local_swap(L, result, it);
                ++result;
            }
        }
        local_swap(L, right, result);
        if (result == middle) return middle;
        if (middle < result) right = result - 1;
        else left = result + 1;
    }
}

/// The same split by the whole warp: each Lomuto pass as in k_select (the
/// elements before the pivot compacted in order by a ballot scan, the rest
/// placed by following their chains), through `tmp` and the ranks `rk`.
/// Every lane returns the split position.
__device__ int warp_split(Local& L, uint16_t* tmp, int16_t* rk, int begin, int end, int axis, int up) {
    const int lane = int(threadIdx.x & 31u);
    const unsigned lt = (1u << lane) - 1u;
    if (begin >= end) return begin;
    const int middle = begin + (end - begin) / 2;
    int left = begin, right = end - 1;
    if (left == right) return middle;
    for (;;) {
        const int pm = left + (right - left) / 2;
        if (lane == 0) local_swap(L, pm, right);
        __syncwarp();
        const double P = local_coord(L, axis, right);
        int running = 0;
        for (int base = left; base < right; base += 32) {
            const int j = base + lane;
            const bool less = j < right && before_pivot(local_coord(L, axis, j), P, up);
            const unsigned m = __ballot_sync(0xffffffffu, less);
            if (j < right) {
                const int r = running + __popc(m & lt);
                rk[j] = less ? int16_t(r) : int16_t(-1);
                if (less) tmp[left + r] = L.perm[j];
            }
            running += __popc(m);
        }
        const int nl = running;
        __syncwarp();
        for (int q = left + nl + lane; q < right; q += 32) {
            int x = q;
            while (rk[x] >= 0) x = left + rk[x];
            tmp[q == left + nl ? right : q] = L.perm[x];
        }
        if (lane == 0) tmp[left + nl] = L.perm[right];
        __syncwarp();
        for (int q = left + lane; q <= right; q += 32) L.perm[q] = tmp[q];
        __syncwarp();
        const int np = left + nl;
        if (np == middle) return middle;
        if (middle < np) right = np - 1;
        else left = np + 1;
    }
}

/// A node of the recursion inside a range of at most kSmall points, packed in
/// 32 bits: begin and end (11 bits each), the axis (2 bits), the three
/// directions (1 bit each).
__device__ __forceinline__ uint32_t pack_node(int b, int e, int x, int ux, int uy, int uz) {
    return uint32_t(b) | uint32_t(e) << 11 | uint32_t(x) << 22 | uint32_t(ux) << 24 | uint32_t(uy) << 25 |
           uint32_t(uz) << 26;
}

/// A level holding at most this many nodes is split node by node by the whole
/// warp; a fuller level, one node per lane.
constexpr int kWarpSplitNodes = 8;

/// One warp per range of at most kSmall points: the whole remaining recursion
/// (spatial_sort.cpp:95-117) in shared memory.  The recursion's nodes cover
/// disjoint index ranges and each one's splits read and permute only its own
/// range, so once a node is split its eight children are independent of each
/// other: the tree is processed level by level.  The first levels (a few large
/// nodes) are split by the whole warp, node after node; the later ones by the
/// lanes taking the nodes of the level in turn, each node's seven splits done
/// by one lane exactly as the reference does them.  The result is the
/// reference's depth-first order, bit for bit.
__global__ void __launch_bounds__(32) k_small_sort(const Seg* __restrict__ segs, Elems E) {
    __shared__ int32_t sidx[kSmall];
    __shared__ double sc[3][kSmall];
    __shared__ uint16_t perm[kSmall], tmp[kSmall];
    __shared__ int16_t rk[kSmall];
    // Nodes of more than 8 points at one level: fewer than kSmall / 9 + 1.
    constexpr int kNodes = kSmall / 9 + 1;
    __shared__ uint32_t nodes[2][kNodes];
    __shared__ int nnodes[2];
    const Seg g = segs[blockIdx.x];
    const int m = g.end - g.begin;
    for (int j = threadIdx.x; j < m; j += 32) {
        sidx[j] = E.idx[g.begin + j];
        sc[0][j] = E.x[g.begin + j];
        sc[1][j] = E.y[g.begin + j];
        sc[2][j] = E.z[g.begin + j];
        perm[j] = uint16_t(j);
    }
    if (threadIdx.x == 0) {
        nodes[0][0] = pack_node(0, m, g.x, g.ux, g.uy, g.uz);
        nnodes[0] = m > 8 ? 1 : 0;
        nnodes[1] = 0;
    }
    __syncwarp();
    Local L{{sc[0], sc[1], sc[2]}, perm};
    for (int cur = 0; nnodes[cur] > 0; cur ^= 1) {
        const int nxt = cur ^ 1;
        const int count = nnodes[cur];
        const bool whole_warp = count <= kWarpSplitNodes;
        for (int k = whole_warp ? 0 : int(threadIdx.x); k < count; k += whole_warp ? 1 : 32) {
            const uint32_t f = nodes[cur][k];
            const int m0 = int(f & 0x7FFu), m8 = int((f >> 11) & 0x7FFu), x = int((f >> 22) & 3u);
            const int ux = int((f >> 24) & 1u), uy = int((f >> 25) & 1u), uz = int((f >> 26) & 1u);
            const int y = (x + 1) % 3, z = (x + 2) % 3;
            int m1, m2, m3, m4, m5, m6, m7;
            if (whole_warp) {
                m4 = warp_split(L, tmp, rk, m0, m8, x, ux);
                m2 = warp_split(L, tmp, rk, m0, m4, y, uy);
                m1 = warp_split(L, tmp, rk, m0, m2, z, uz);
                m3 = warp_split(L, tmp, rk, m2, m4, z, !uz);
                m6 = warp_split(L, tmp, rk, m4, m8, y, !uy);
                m5 = warp_split(L, tmp, rk, m4, m6, z, uz);
                m7 = warp_split(L, tmp, rk, m6, m8, z, !uz);
            } else {
                m4 = local_split(L, m0, m8, x, ux);
                m2 = local_split(L, m0, m4, y, uy);
                m1 = local_split(L, m0, m2, z, uz);
                m3 = local_split(L, m2, m4, z, !uz);
                m6 = local_split(L, m4, m8, y, !uy);
                m5 = local_split(L, m4, m6, z, uz);
                m7 = local_split(L, m6, m8, z, !uz);
            }
            if (!whole_warp || threadIdx.x == 0) {
                const uint32_t ch[8] = {pack_node(m0, m1, z, uz, ux, uy),   pack_node(m1, m2, y, uy, uz, ux),
                                        pack_node(m2, m3, y, uy, uz, ux),   pack_node(m3, m4, x, ux, !uy, !uz),
                                        pack_node(m4, m5, x, ux, !uy, !uz), pack_node(m5, m6, y, !uy, uz, !ux),
                                        pack_node(m6, m7, y, !uy, uz, !ux), pack_node(m7, m8, z, !uz, !ux, uy)};
                const int lo[8] = {m0, m1, m2, m3, m4, m5, m6, m7}, hi[8] = {m1, m2, m3, m4, m5, m6, m7, m8};
                for (int c = 0; c < 8; ++c)
                    if (hi[c] - lo[c] > 8) nodes[nxt][atomicAdd(&nnodes[nxt], 1)] = ch[c];
            }
            if (whole_warp) __syncwarp();
        }
        __syncwarp();
        if (threadIdx.x == 0) nnodes[cur] = 0;
        __syncwarp();
    }
    for (int j = threadIdx.x; j < m; j += 32) E.idx[g.begin + j] = sidx[perm[j]];
}

__global__ void k_gather_xyz(const double* __restrict__ xyz, const int32_t* __restrict__ order, int64_t n,
                             const int64_t* __restrict__ off, int nsets,
                             double* __restrict__ x, double* __restrict__ y, double* __restrict__ z) {
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = off[set_of(off, nsets, p)] + order[p];
        x[p] = xyz[3 * i];
        y[p] = xyz[3 * i + 1];
        z[p] = xyz[3 * i + 2];
    }
}

}  // namespace

/// The reference's shuffled sequence (rand48.h:146-153 applied to 0..n-1) for
/// every set: order[off[s] + p] is the local index at position p of set s.
/// `h_off` / `d_off`: the same nsets+1 offsets on the host and on the device.
int shuffle_sets_device(const int64_t* h_off, const int64_t* d_off, int nsets, int32_t* d_order,
                        cudaStream_t s) {
    int64_t n = 0;
    for (int i = 0; i < nsets; ++i) n = std::max<int64_t>(n, h_off[i + 1] - h_off[i]);
    const int64_t total = h_off[nsets] - h_off[0];
    if (total <= 0) return D3G_OK;
    if (n <= kSerialShuffleMax) {
        k_shuffle_serial<<<unsigned(nsets), 128, 0, s>>>(d_off, d_order);
        D3G_CUDA(cudaGetLastError());
        return D3G_OK;
    }
    JumpTable jt;
    jt.step[0] = Affine{kA, kC};
    for (int i = 1; i < 48; ++i) jt.step[i] = compose(jt.step[i - 1], jt.step[i - 1]);

    // Expected rejections ~ n^2 / 2^32; draw with a generous margin, retry if short.
    int64_t margin = 1024 + 4 * (int64_t)((double(n) * double(n)) / 4294967296.0);
    for (int attempt = 0; attempt < 6; ++attempt, margin *= 4) {
        const int64_t T = std::max<int64_t>(n - 1, 0) + margin;
        DevBuf<uint32_t> outs;
        DevBuf<int32_t> cand, acc, j, keys2, vals, vals2, pred, tfirst, tlast;
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
        k_reject_scan<<<1, 1024, 0, s>>>(outs.p, cand.p, ncand.p, n, rej.p, nrej.p);
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
        D3G_TRY(pred.alloc(size_t(n), s));
        D3G_TRY(tfirst.alloc(size_t(n), s));
        D3G_TRY(tlast.alloc(size_t(n), s));
        D3G_CUDA(cudaMemsetAsync(tfirst.p, 0xFF, sizeof(int32_t) * size_t(n), s));
        D3G_CUDA(cudaMemsetAsync(tlast.p, 0xFF, sizeof(int32_t) * size_t(n), s));
        if (cnt > 0) {
            D3G_TRY(keys2.alloc(size_t(cnt), s));
            D3G_TRY(vals.alloc(size_t(cnt), s));
            D3G_TRY(vals2.alloc(size_t(cnt), s));
            k_iota<<<grid_for(cnt, 256), 256, 0, s>>>(vals.p, cnt, 1);
            D3G_TRY(sort_pairs(j.p + 1, keys2.p, vals.p, vals2.p, cnt, 0, bits_for(uint64_t(n)), s));
            DevBuf<int32_t> last_unused;
            D3G_TRY(last_unused.alloc(size_t(n), s));
            k_lists<<<grid_for(cnt, 256), 256, 0, s>>>(keys2.p, vals2.p, cnt, pred.p, last_unused.p);
            k_target_ranges<<<grid_for(cnt, 256), 256, 0, s>>>(keys2.p, cnt, tfirst.p, tlast.p);
        }
        k_final_sets<<<grid_for(total, 256), 256, 0, s>>>(j.p, pred.p, vals2.p, tfirst.p, tlast.p, d_off,
                                                          nsets, total, d_order);
        D3G_CUDA(cudaGetLastError());
        return D3G_OK;
    }
    set_error("shuffle: rejection margin exhausted");
    return D3G_ERR_INTERNAL;
}

int shuffle_device(int64_t n, int32_t* d_order, cudaStream_t s) {
    if (n <= 0) return D3G_OK;
    const int64_t h_off[2] = {0, n};
    DevBuf<int64_t> d_off;
    D3G_TRY(d_off.alloc(2, s));
    D3G_CUDA(cudaMemcpyAsync(d_off.p, h_off, sizeof h_off, cudaMemcpyHostToDevice, s));
    return shuffle_sets_device(h_off, d_off.p, 1, d_order, s);
}

/// Level boundaries of the multiscale pass: b[0] = n, b[k+1] = floor(b[k]/8)
/// while b[k] >= 64 (spatial_sort.cpp:130-137; the ratio 0.125 is exact).  A
/// build may ask for another ratio (1/2 ... 1/7) for its own insertion order.
int multiscale_bounds(int64_t n, int64_t* b, int cap, double ratio = 0.125) {
    int k = 0;
    b[k++] = n;
    while (k < cap && b[k - 1] >= 64) {
        b[k] = int64_t(double(b[k - 1]) * ratio);
        ++k;
    }
    return k;   // levels: [b[k+1], b[k]) for k < count-1, plus [0, b[count-1])
}

namespace {

template <class T>
int upload(const std::vector<T>& v, DevBuf<T>& d, cudaStream_t s) {
    D3G_TRY(d.alloc(v.size(), s));
    if (!v.empty())
        D3G_CUDA(cudaMemcpyAsync(d.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
    return D3G_OK;
}

}  // namespace

/// spatial_sort of every set: d_order[off[s] + p] is the local index of the
/// point at position p of set s's insertion order.  `level_ratio` is the
/// multiscale ratio: the reference's 1/8, or another a build asks for.
int spatial_order_sets_device(const double* d_xyz, const int64_t* h_off, const int64_t* d_off, int nsets,
                              int32_t* d_order, cudaStream_t s, double level_ratio = 0.125) {
    const int64_t n = h_off[nsets] - h_off[0];
    if (n <= 0) return D3G_OK;
    const bool trace = getenv("D3G_TRACE") != nullptr;
    cudaEvent_t tev[4];
    if (trace) {
        for (auto& e : tev) cudaEventCreate(&e);
        cudaEventRecord(tev[0], s);
    }
    D3G_TRY(shuffle_sets_device(h_off, d_off, nsets, d_order, s));
    if (trace) cudaEventRecord(tev[1], s);
    DevBuf<double> ex, ey, ez, bx, by, bz;
    DevBuf<int32_t> bidx, rk;
    D3G_TRY(ex.alloc(size_t(n), s));
    D3G_TRY(ey.alloc(size_t(n), s));
    D3G_TRY(ez.alloc(size_t(n), s));
    k_gather_xyz<<<grid_for(n, 256), 256, 0, s>>>(d_xyz, d_order, n, d_off, nsets, ex.p, ey.p, ez.p);
    const Elems E{d_order, ex.p, ey.p, ez.p};

    // Roots: each set's multiscale levels (spatial_sort.cpp:130-137), each
    // Hilbert-sorted from axis x with every direction "down".
    std::vector<Seg> big, small;
    auto classify = [&](const Seg& g) {
        const int len = g.end - g.begin;
        if (len <= 8) return;
        if (len <= kSmall) small.push_back(g);
        else big.push_back(g);
    };
    for (int st = 0; st < nsets; ++st) {
        const int64_t base = h_off[st], ns = h_off[st + 1] - h_off[st];
        if (ns < 2) continue;
        int64_t hb[64];
        const int nb = multiscale_bounds(ns, hb, 63, level_ratio);
        for (int k = 0; k < nb; ++k) {
            const int64_t lo = k + 1 < nb ? hb[k + 1] : 0;
            classify(Seg{int(base + lo), int(base + hb[k]), 0, 0, 0, 0});
        }
    }
    if (!big.empty()) {
        D3G_TRY(bidx.alloc(size_t(n), s));
        D3G_TRY(bx.alloc(size_t(n), s));
        D3G_TRY(by.alloc(size_t(n), s));
        D3G_TRY(bz.alloc(size_t(n), s));
        D3G_TRY(rk.alloc(size_t(n), s));
    }
    const Elems B{bidx.p, bx.p, by.p, bz.p};
    auto mid = [](int b, int e) { return b + (e - b) / 2; };
    while (!big.empty()) {
        std::vector<SelTask> ta, tb, tc;
        std::vector<Seg> next;
        auto task = [](std::vector<SelTask>& v, int b, int e, int axis, int up) {
            if (e - b >= 2) v.push_back(SelTask{b, e, b + (e - b) / 2, axis, up});
        };
        for (const Seg& g : big) {
            const int x = g.x, y = (x + 1) % 3, z = (x + 2) % 3;
            const int m0 = g.begin, m8 = g.end, m4 = mid(m0, m8);
            const int m2 = mid(m0, m4), m6 = mid(m4, m8);
            const int m1 = mid(m0, m2), m3 = mid(m2, m4), m5 = mid(m4, m6), m7 = mid(m6, m8);
            task(ta, m0, m8, x, g.ux);
            task(tb, m0, m4, y, g.uy);
            task(tb, m4, m8, y, !g.uy);
            task(tc, m0, m2, z, g.uz);
            task(tc, m2, m4, z, !g.uz);
            task(tc, m4, m6, z, g.uz);
            task(tc, m6, m8, z, !g.uz);
            const Seg kids[8] = {{m0, m1, z, g.uz, g.ux, g.uy},   {m1, m2, y, g.uy, g.uz, g.ux},
                                 {m2, m3, y, g.uy, g.uz, g.ux},   {m3, m4, x, g.ux, !g.uy, !g.uz},
                                 {m4, m5, x, g.ux, !g.uy, !g.uz}, {m5, m6, y, !g.uy, g.uz, !g.ux},
                                 {m6, m7, y, !g.uy, g.uz, !g.ux}, {m7, m8, z, !g.uz, !g.ux, g.uy}};
            for (const Seg& k : kids) {
                const int len = k.end - k.begin;
                if (len <= 8) continue;
                if (len <= kSmall) small.push_back(k);
                else next.push_back(k);
            }
        }
        for (const std::vector<SelTask>* phase : {&ta, &tb, &tc}) {
            if (phase->empty()) continue;
            DevBuf<SelTask> dt;
            D3G_TRY(upload(*phase, dt, s));
            int longest = 0;
            for (const SelTask& t : *phase) longest = std::max(longest, t.end - t.left);
            if (longest > kBlockSelectMax) {
                // Whole-GPU passes until every task fits a block.
                const int nt = int(phase->size());
                std::vector<TaskState> hs(static_cast<size_t>(nt));
                for (int i = 0; i < nt; ++i) {
                    const SelTask& t = (*phase)[size_t(i)];
                    hs[size_t(i)] = TaskState{t.left, t.end - 1, t.nth, t.axis, t.up, t.end - t.left < 2 ? 1 : 0,
                                              0.0, 0, 0, 0};
                }
                DevBuf<TaskState> dts;
                DevBuf<int> ctrl, tiles;
                D3G_TRY(upload(hs, dts, s));
                D3G_TRY(ctrl.alloc(2, s));
                D3G_TRY(tiles.alloc(size_t(n / kTile + nt + 1), s));
                const unsigned tg = unsigned(kNumSMs * 8);
                for (int iter = 0;; ++iter) {
                    D3G_CUDA(cudaMemsetAsync(ctrl.p, 0, 2 * sizeof(int), s));
                    k_plan<<<1, 1024, 0, s>>>(dts.p, nt, E, B, ctrl.p);
                    k_tile_count<<<tg, kTileThreads, 0, s>>>(dts.p, nt, E, ctrl.p, tiles.p);
                    k_tile_scan<<<1, 1024, 0, s>>>(dts.p, nt, ctrl.p, tiles.p);
                    k_tile_scatter<<<tg, kTileThreads, 0, s>>>(dts.p, nt, E, B, ctrl.p, tiles.p, rk.p);
                    k_tile_place<<<tg, kTileThreads, 0, s>>>(dts.p, nt, E, B, ctrl.p, rk.p);
                    k_tile_pivot<<<grid_for(nt, 128), 128, 0, s>>>(dts.p, nt, E, B);
                    k_tile_copy<<<tg, kTileThreads, 0, s>>>(dts.p, nt, E, B, ctrl.p);
                    k_tile_update<<<grid_for(nt, 128), 128, 0, s>>>(dts.p, nt, E, B, ctrl.p + 1);
                    D3G_CUDA(cudaGetLastError());
                    int big_left = 0;
                    D3G_CUDA(cudaMemcpyAsync(&big_left, ctrl.p + 1, sizeof big_left, cudaMemcpyDeviceToHost, s));
                    D3G_CUDA(cudaStreamSynchronize(s));
                    if (big_left == 0) break;
                    if (iter > (1 << 26)) {
                        set_error("spatial sort: quickselect did not converge");
                        return D3G_ERR_INTERNAL;
                    }
                }
                k_to_seltask<<<grid_for(nt, 128), 128, 0, s>>>(dts.p, nt, dt.p);
            }
            k_select<<<unsigned(phase->size()), kSelThreads, 0, s>>>(dt.p, E, B, rk.p);
            D3G_CUDA(cudaGetLastError());
        }
        big.swap(next);
    }
    if (trace) cudaEventRecord(tev[2], s);
    if (!small.empty()) {
        DevBuf<Seg> ds;
        D3G_TRY(upload(small, ds, s));
        k_small_sort<<<unsigned(small.size()), 32, 0, s>>>(ds.p, E);
        D3G_CUDA(cudaGetLastError());
    }
    if (trace) {
        cudaEventRecord(tev[3], s);
        cudaEventSynchronize(tev[3]);
        float a = 0, b = 0, c = 0;
        cudaEventElapsedTime(&a, tev[0], tev[1]);
        cudaEventElapsedTime(&b, tev[1], tev[2]);
        cudaEventElapsedTime(&c, tev[2], tev[3]);
        fprintf(stderr, "d3g sort: shuffle %.2f ms, big splits %.2f ms, small ranges %.2f ms (%zu)\n", a, b, c,
                small.size());
        for (auto& e : tev) cudaEventDestroy(e);
    }
    return D3G_OK;
}

int spatial_order_device(const double* d_xyz, int64_t n, int32_t* d_order, cudaStream_t s) {
    if (n <= 0) return D3G_OK;
    const int64_t h_off[2] = {0, n};
    DevBuf<int64_t> d_off;
    D3G_TRY(d_off.alloc(2, s));
    D3G_CUDA(cudaMemcpyAsync(d_off.p, h_off, sizeof h_off, cudaMemcpyHostToDevice, s));
    return spatial_order_sets_device(d_xyz, h_off, d_off.p, 1, d_order, s);
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
