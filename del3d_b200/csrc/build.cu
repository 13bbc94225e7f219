// The Delaunay build on the device: del3d::Delaunay::build
// (src/triangulation.cpp:65-120, 702-769, 932-968) as parallel insertion rounds.
//
// Why a parallel build can return the reference's tets: in_sphere never
// returns ZERO (symbolic perturbation, src/predicates.cpp:206-232) and the hull
// conflict rule is fixed (src/triangulation.cpp:588-602), so the set of finite
// cells is a function of the point set alone, whatever the insertion order.
// The device therefore inserts many points at once, in rounds:
//
//   * Points are ordered by the spatial sort (sort.cu) and grouped into BRIO
//     levels; each level is cut into chunks, one per worker.  A worker inserts
//     its chunk's points one per round, so the points in flight in a round are
//     spread along the Hilbert curve, i.e. far apart.
//   * k_cavity   each worker walks from the last vertex it inserted to the tet
//                its point conflicts with (visibility walk, exact orient3d),
//                then grows the conflict region breadth-first with the
//                reference's in_conflict rule, claiming every region tet and
//                every tet across its boundary with a 64-bit atomicMin of
//                (round, point rank) - the earliest point in insertion order
//                wins ties.  A worker that meets a claim of an earlier point
//                stops at once: it would lose anyway.
//   * k_check    a worker wins if it still holds every claim.  Winners' regions
//                and their one-ring of outside tets are pairwise disjoint, so
//                winners can re-star concurrently without locks.
//   * k_restar   each winner re-stars its region (one new tet per boundary
//                facet, src/tds.h:160-221), reusing its region's slots, and
//                advances to its next point.  The earliest pending point always
//                wins, so every round makes progress.
//
// The output is canonicalised (even rotation, lexicographic sort), so it is
// identical across runs whatever order the rounds happened to take.
#include "build_api.cuh"

#include <cuda/atomic>
#include "device_util.cuh"

#include <algorithm>
#include <mutex>
#include <numeric>
#include <optional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace d3g {

int spatial_order_device(const double* d_xyz, int64_t n, int32_t* d_order, cudaStream_t s);
int spatial_order_sets_device(const double* d_xyz, const int64_t* h_off, const int64_t* d_off, int nsets,
                              int32_t* d_order, cudaStream_t s, double level_ratio = 0.125);
int multiscale_bounds(int64_t n, int64_t* b, int cap, double ratio = 0.125);

namespace {

constexpr int kInf = -1;
constexpr int kWalkLimit = 1 << 20;
constexpr int kRotateLimit = 1 << 16;
constexpr int kRoundsPerBatch = 16;
// Scratch of a worker in a normal round, and of each of the kBigSlots workers
// served at a time in a big round.
constexpr int kCavCap = 256;                     // boundary facets: twice the tets
constexpr int kBigSlots = 64, kBigCav = 16384;   // boundary facets: twice the tets

enum : int { WS_DONE = 0, WS_CAND = 1, WS_LOST = 2, WS_WIN = 3, WS_PARKED = 4, WS_FAIL = 5 };

__device__ __forceinline__ Pt vpt(const double* __restrict__ vx, int v) {
    const double* p = vx + 3 * int64_t(v);
    return Pt{p[0], p[1], p[2]};
}

__device__ __forceinline__ int at(const int4& t, int i) {
    return i == 0 ? t.x : (i == 1 ? t.y : (i == 2 ? t.z : t.w));
}
__device__ __forceinline__ void set_at(int4& t, int i, int v) {
    if (i == 0) t.x = v;
    else if (i == 1) t.y = v;
    else if (i == 2) t.z = v;
    else t.w = v;
}
__device__ __forceinline__ int inf_pos(const int4& t) {
    return t.x == kInf ? 0 : (t.y == kInf ? 1 : (t.z == kInf ? 2 : (t.w == kInf ? 3 : -1)));
}
__device__ __forceinline__ int pos_of(const int4& t, int v) {
    return t.x == v ? 0 : (t.y == v ? 1 : (t.z == v ? 2 : 3));
}

struct Tables {
    int4* tv;                  // vertices (kInf = the infinite vertex)
    int4* tn;                  // neighbours: tet * 4 + the facet of that tet facing back
    unsigned long long* claim; // per-round ownership claims
    uint8_t* alive;
    int* fnew;                 // per tet facet: the new tet built on it (restar scratch)
    int* vert_tet;             // one live tet incident to each inserted vertex
    int* tet_count;
    int cap;
    int walk_limit;            // steps of a lockstep walk before ST_WALK_LIMIT
    const int32_t* vset;       // the point set of each vertex (batched builds share the tables)
};

struct Workers {
    const int* list;  // big mode: the workers served (warp i serves list[i]); null otherwise
    int* parked;  // 1 while the worker's point needs the big scratch
    int* cur;     // current point (vertex id) of each worker
    int* beg;     // start of its chunk
    int* end;     // end of its chunk
    int* pos;     // next position to visit, relative to beg (chunks are walked cyclically)
    int* left;    // positions still to visit after the current point
    int* nwon;    // points this worker inserted in the current level
    int* last;    // last vertex it inserted (-1: none yet)
    int* guide;   // an inserted vertex near its chunk, for the first walk
    int* state;
    int* ncav;
    int* nfac;
    int* cav;     // worker-major scratch: cav_cap region tets per worker
    int* fac;     // fac_cap boundary facets (tet * 4 + facet) per worker
    int4* st_v;   // fac_cap staged new tets per worker (vertices) ...
    int4* st_n;   // ... and neighbours
    int* wset;        // set of each worker
    const int4* skips; // per set: its first tet's vertices (inserted before the rounds)
    const uint8_t* set_exact;  // per set: 1 if its coordinates make the filters exact
    int cav_cap;
    int fac_cap;
    int n;
};

struct Round {
    const unsigned* round;    // current round number (device), set by k_round_begin
    int* counters;            // [0] active workers, [1] parked workers, [2] winners,
                              // [3] workers parked this round
    unsigned long long* sums; // [0] region tets, [1] boundary facets of the winners
    unsigned long long* totals; // [0] winners, [1] attempts, [2] rounds with work,
                                // [3] parked workers, [4] stalled round seen, [5] active
    unsigned long long* steps;  // timing runs only (else null): [0] walk steps,
                                // [1] breadth-first steps, over all attempts
    uint32_t* status;
    unsigned long long* pstats; // [0] conflict tests, [1] of which the filter left uncertain,
                                // [2] of which exactly degenerate (tie-break), [3] largest
                                // conflict region inserted (tets)
};

/// A thread's conflict-test counters, added to Round::pstats once at the end
/// of a launch (flush_counters).  `flags` holds the uncertain count in its low
/// 20 bits and the tie count above: a thread makes far fewer than 2^20 tests in
/// one launch (a warp inserts a few hundred points per launch, a few tests per
/// lane each).  The insertion kernels keep them in shared memory, one slot per
/// thread, so that they take no registers from the loops they count in.
constexpr int kCounterThreads = 128;   // the insertion kernels' block size

struct SharedCounters {
    unsigned* tests;
    unsigned* flags;
    int* max_region;
    __device__ void count(int r) const {
        tests[threadIdx.x] += 1;
        flags[threadIdx.x] += ((r >> 1) & 1) + (((r >> 2) & 1) << 20);
    }
    __device__ void region(int c) const { max_region[threadIdx.x] = max(max_region[threadIdx.x], c); }
};

#define D3G_SHARED_COUNTERS(name)                                                   \
    __shared__ unsigned name##_t[kCounterThreads], name##_f[kCounterThreads];     \
    __shared__ int name##_m[kCounterThreads];                                       \
    name##_t[threadIdx.x] = 0;                                                      \
    name##_f[threadIdx.x] = 0;                                                      \
    name##_m[threadIdx.x] = 0;                                                      \
    const SharedCounters name{name##_t, name##_f, name##_m}

/// Sums the warp's counters into R.pstats (one atomic per counter per warp).
__device__ void flush_counters(const SharedCounters& c, const Round& R) {
    unsigned long long t = c.tests[threadIdx.x], u = c.flags[threadIdx.x] & 0xFFFFFu,
                       z = c.flags[threadIdx.x] >> 20;
    int m = c.max_region[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t += __shfl_xor_sync(0xffffffffu, t, o);
        u += __shfl_xor_sync(0xffffffffu, u, o);
        z += __shfl_xor_sync(0xffffffffu, z, o);
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (t) atomicAdd(R.pstats, t);
        if (u) atomicAdd(R.pstats + 1, u);
        if (z) atomicAdd(R.pstats + 2, z);
        if (m) atomicMax(R.pstats + 3, (unsigned long long)m);
    }
}

/// Claim key of point v this round: (~round) << 32 makes every newer round win
/// against stale claims; the point rank breaks ties (earliest wins).
__device__ __forceinline__ unsigned long long claim_key(const Round& R, int v) {
    return ((unsigned long long)(0xFFFFFFFFu - *R.round) << 32) |
           (unsigned long long)(uint32_t(v)) << 1;
}

__global__ void k_round_begin(Round R) {
    unsigned* r = const_cast<unsigned*>(R.round);
    *r += 1;
    R.counters[0] = R.counters[1] = R.counters[2] = R.counters[3] = 0;
}

/// Folds one round's counters into the running totals; flags a round in which
/// workers were active but nobody won (the earliest pending point must win).
__global__ void k_round_end(Round R) {
    const int active = R.counters[0], parked = R.counters[1], won = R.counters[2];
    R.totals[0] += (unsigned long long)won;
    R.totals[1] += (unsigned long long)(active + won);
    if (active + won > 0) R.totals[2] += 1;
    R.totals[3] = (unsigned long long)parked;
    // A worker parked this round may have claimed tets of every other candidate.
    if (active > 0 && won == 0 && R.counters[3] == 0) R.totals[4] = 1;
    R.totals[5] = (unsigned long long)active;
}

/// orient3d of tet (q0,q1,q2,q3) with vertex i replaced by p (one call site);
/// `ex`: the set's coordinates make the filter exact.
__device__ __forceinline__ int orient_replaced(const Pt* q, int i, const Pt& p, bool ex, uint32_t* st) {
    const Pt& A = i == 0 ? p : q[0];
    const Pt& B = i == 1 ? p : q[1];
    const Pt& C = i == 2 ? p : q[2];
    const Pt& D = i == 3 ? p : q[3];
    return orient3d_x(A, B, C, D, ex, st);
}

/// coplanar_in_circle for the hull case of the conflict test (rare: the point
/// lies in the plane of a hull facet), out of line so that its code stays out
/// of the hot path's instruction stream.
__device__ __noinline__ int hull_in_circle(double ax, double ay, double az, double bx, double by, double bz,
                                           double dx, double dy, double dz, double px, double py, double pz,
                                           int ia, int ib, int id_, int ip, uint32_t* st) {
    const int64_t id[4] = {ia, ib, id_, ip};
    return coplanar_in_circle(Pt{ax, ay, az}, Pt{bx, by, bz}, Pt{dx, dy, dz}, Pt{px, py, pz}, id, st);
}

/// Outcome bits of a conflict test: in conflict; the floating-point filter
/// could not certify the sign (the set's exact filter value, the exact stage or
/// a tie-break decided it); the exact value was zero (decided by the symbolic
/// perturbation, or the hull in-circle test); and, for the fast variant only,
/// undecided (left to the full variant).
enum : int { CT_IN = 1, CT_UNCERTAIN = 2, CT_TIE = 4, CT_UNDECIDED = 8 };

/// in_sphere's exact sign for a set whose filter is not exact and, when it is
/// zero, the reference's tie-break (src/predicates.cpp:206-232): the sign, plus
/// 4 if the tie-break gave it.  Out of line.
__device__ __noinline__ int in_sphere_exact_tie(double ax, double ay, double az, double bx, double by, double bz,
                                                double cx, double cy, double cz, double dx, double dy, double dz,
                                                double ex, double ey, double ez, int id0, int id1, int id2, int id3,
                                                int id4, double fdet, uint32_t* st) {
    const int s = in_sphere_degenerate(ax, ay, az, bx, by, bz, cx, cy, cz, dx, dy, dz, ex, ey, ez, id0, id1, id2, id3,
                                       id4, fdet, 0, st);
    if (s != 0) return s;
    return 4 + in_sphere_perturb(Pt{ax, ay, az}, Pt{bx, by, bz}, Pt{cx, cy, cz}, Pt{dx, dy, dz}, Pt{ex, ey, ez},
                                 id0, id1, id2, id3, id4, st);
}

/// The reference's conflict test, src/triangulation.cpp:588-602, with its
/// outcome bits (CT_*).  `ex`: the point set's coordinates span few enough bits
/// that the orient3d and in_sphere filters compute their determinants exactly.
__device__ int conflict_test(const int4 t, const Pt& p, int pid, const double* __restrict__ vx, bool ex,
                             uint32_t* st) {
    const int ip = inf_pos(t);
    if (ip >= 0) {
        // For each slot of the infinite vertex, the three finite vertices in
        // the order that makes orient3d(a, b, d, p) the half-space test.
        const int o0 = ip == 0 ? 2 : (ip == 1 ? 2 : (ip == 2 ? 1 : 0));
        const int o1 = ip == 0 ? 1 : (ip == 1 ? 3 : (ip == 2 ? 0 : 1));
        const int o2 = ip == 0 ? 3 : (ip == 1 ? 0 : (ip == 2 ? 3 : 2));
        const int va = at(t, o0), vb = at(t, o1), vd = at(t, o2);
        const Pt a = vpt(vx, va), b = vpt(vx, vb), d = vpt(vx, vd);
        const Orient3dFilter f = orient3d_filter(a, b, d, p);
        const int unc = f.certain ? 0 : CT_UNCERTAIN;
        const int s = (f.certain || ex) ? -sign_of(f.det) : orient3d_exact(a, b, d, p, f.det, st);
        if (s != 0) return (s > 0 ? CT_IN : 0) | unc;
        return (hull_in_circle(a.x, a.y, a.z, b.x, b.y, b.z, d.x, d.y, d.z, p.x, p.y, p.z, va, vb, vd, pid, st) > 0
                    ? CT_IN : 0) | unc | CT_TIE;
    }
    const Pt a = vpt(vx, t.x), b = vpt(vx, t.y), c = vpt(vx, t.z), d = vpt(vx, t.w);
    const InSphereFilter f = in_sphere_filter(a, b, c, d, p);
    if (f.certain) return f.det < 0.0 ? CT_IN : 0;   // in_sphere = -sign(det)
    if (ex && f.det != 0.0) return (f.det < 0.0 ? CT_IN : 0) | CT_UNCERTAIN;
    if (ex)
        return (in_sphere_tiebreak_exact(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, d.x, d.y, d.z, p.x, p.y, p.z,
                                         t.x, t.y, t.z, t.w, pid, st) > 0 ? CT_IN : 0) | CT_UNCERTAIN | CT_TIE;
    const int r = in_sphere_exact_tie(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, d.x, d.y, d.z, p.x, p.y, p.z, t.x,
                                      t.y, t.z, t.w, pid, f.det, st);
    const bool tie = r > 1;
    return ((tie ? r - 4 : r) > 0 ? CT_IN : 0) | CT_UNCERTAIN | (tie ? CT_TIE : 0);
}

/// conflict_test out of line, for the once-per-insertion seed check (one inline
/// copy, in the breadth-first growth, is enough).
__device__ __noinline__ int conflict_test_seed(int4 t, double px, double py, double pz, int pid,
                                               const double* __restrict__ vx, bool ex, uint32_t* st) {
    return conflict_test(t, Pt{px, py, pz}, pid, vx, ex, st);
}

constexpr unsigned kFull = 0xffffffffu;

/// Advances worker w to the next point of its chunk (walked cyclically),
/// skipping its set's first-tet vertices; -1 when the chunk is done.
__device__ int next_point(const Workers& W, int w) {
    const int b = W.beg[w], len = W.end[w] - b;
    const int4 sk = W.skips[W.wset[w]];
    int pos = W.pos[w], left = W.left[w];
    int v = -1;
    while (left > 0) {
        const int c = b + pos;
        pos = pos + 1 == len ? 0 : pos + 1;
        --left;
        if (c != sk.x && c != sk.y && c != sk.z && c != sk.w) {
            v = c;
            break;
        }
    }
    W.pos[w] = pos;
    W.left[w] = left;
    W.cur[w] = v;
    return v;
}

// ---- the insertion kernels ---------------------------------------------------
//
// A worker is served by a group of G lanes (G = 32, 16, 8 or 4), so one warp
// serves 32 / G workers side by side.  Few workers: G = 32 shortens each
// worker's chain of dependent memory accesses (8 region tets per step).  Many
// workers (more than the GPU keeps resident as warps): a small G packs them into
// fewer warps, so the whole round fits the resident warps and its time is one
// chain instead of several waves of chains.  Control flow stays uniform over
// the warp - every loop runs until all of its groups are done - so the groups'
// memory accesses are issued together and warp votes cover all 32 lanes; a
// group reads its own bits of each vote.

template <int G>
struct Lanes {
    int lane, sub, gbase;
    unsigned gm;   // the group's bits in a warp-wide vote
    __device__ Lanes() {
        lane = threadIdx.x & 31;
        sub = lane & (G - 1);
        gbase = lane - sub;
        gm = G == 32 ? kFull : (((1u << G) - 1u) << gbase);
    }
    /// The group's bits of a warp-wide vote, lane 0 of the group at bit 0.
    __device__ unsigned own(unsigned vote) const { return G == 32 ? vote : (vote & gm) >> gbase; }
};

/// Visibility walk from each live group's start tet to a tet in conflict with
/// its point p: the finite tet containing p, or the infinite tet beyond the hull
/// facet the walk crosses.  Lanes 0-3 of a group test the four facets of a step;
/// the first negative one in a pseudo-random cyclic order is crossed (never the
/// facet just crossed).  Returns the tet (same in every lane of the group), or
/// -1 for a group that is not live or hit the walk limit.
template <int G>
__device__ int walk_g(bool live, int t, const Pt& p, int pid, const Tables& T, const double* __restrict__ vx,
                      bool ex, uint32_t* st, const Lanes<G>& L, int* nsteps) {
    int4 tv = make_int4(0, 0, 0, 0);
    if (live) {
        tv = T.tv[t];
        const int ip = inf_pos(tv);
        if (ip >= 0) {
            t = at(T.tn[t], ip) >> 2;
            tv = T.tv[t];
        }
    }
    int prev = -1, found = -1;
    uint32_t h = uint32_t(pid) * 2654435761u + 12345u;
    bool walking = live;
    for (int step = 0; __any_sync(kFull, walking); ++step) {
        int4 tn = make_int4(0, 0, 0, 0);
        bool neg = false;
        if (walking) {
            tn = T.tn[t];
            h = h * 1664525u + 1013904223u;
            if (L.sub < 4 && (at(tn, L.sub) >> 2) != prev) {
                const Pt q[4] = {vpt(vx, tv.x), vpt(vx, tv.y), vpt(vx, tv.z), vpt(vx, tv.w)};
                neg = orient_replaced(q, L.sub, p, ex, st) < 0;
            }
        }
        const unsigned m = L.own(__ballot_sync(kFull, neg)) & 0xFu;
        if (walking) {
            *nsteps = step + 1;
            if (m == 0) {
                found = t;
                walking = false;
            } else {
                const int s0 = int(h >> 30);
                const unsigned rot = ((m >> s0) | (m << (4 - s0))) & 0xFu;
                const int i = (s0 + __ffs(int(rot)) - 1) & 3;
                const int next = at(tn, i) >> 2;
                const int4 nv = T.tv[next];
                if (inf_pos(nv) >= 0) {
                    found = next;
                    walking = false;
                } else {
                    prev = t;
                    t = next;
                    tv = nv;
                    if (step + 1 >= T.walk_limit) {
                        report(st, ST_WALK_LIMIT);
                        walking = false;
                    }
                }
            }
        }
    }
    return found;
}

/// One group of G lanes per worker: locate the worker's point, then grow its
/// conflict region breadth-first, G/4 region tets (G facets) per step, claiming
/// every region tet (key) and every tet across the region boundary (key|1).
template <int G>
__global__ void __launch_bounds__(128, 8) k_cavity(Tables T, Workers W, Round R, const double* __restrict__ vx,
                                                int first) {
    const Lanes<G> L;
    D3G_SHARED_COUNTERS(ctr);
    const int slot = first + int((blockIdx.x * blockDim.x + threadIdx.x) / G);
    bool live = slot < W.n;
    int w = 0, v = -1;
    if (live) {
        w = W.list ? W.list[slot] : slot;
        v = W.cur[w];
        // Normal rounds leave parked workers alone; big rounds serve only those.
        if (v < 0 || (W.parked[w] != 0) != (W.list != nullptr)) {
            if (L.sub == 0) W.state[w] = v < 0 ? WS_DONE : WS_PARKED;
            live = false;
        }
    }
    if (!__any_sync(kFull, live)) return;
    const Pt p = live ? vpt(vx, v) : Pt{0.0, 0.0, 0.0};
    const bool ex = live && W.set_exact[W.wset[w]] != 0;
    int start = 0;
    if (live) start = T.vert_tet[W.last[w] >= 0 ? W.last[w] : W.guide[w]];
    int wsteps = 0;
    const int seed = walk_g<G>(live, start, p, v, T, vx, ex, R.status, L, &wsteps);
    if (R.steps && live && L.sub == 0) atomicAdd(R.steps, (unsigned long long)wsteps);
    if (live && seed < 0) {
        if (L.sub == 0) W.state[w] = WS_FAIL;
        live = false;
    }
    const unsigned long long key = live ? claim_key(R, v) : 0ull;
    const unsigned long long mine = key >> 1;
    int* cav = W.cav + int64_t(live ? slot : 0) * W.cav_cap;
    int* fac = W.fac + int64_t(live ? slot : 0) * W.fac_cap;
    int lost = 0;
    if (live && L.sub == 0) {
        const unsigned long long old = atomicMin(T.claim + seed, key);
        lost = (old >> 1) < mine;
        cav[0] = seed;
    }
    lost = __shfl_sync(kFull, lost, L.gbase);
    if (live && lost) {
        if (L.sub == 0) W.state[w] = WS_LOST;
        live = false;
    }
    __syncwarp();
    const unsigned lt = (1u << L.lane) - 1u;
    int ncav = 1, nfac = 0, head = 0;
    bool growing = live;
    while (__any_sync(kFull, growing)) {
        if (R.steps && growing && L.sub == 0) atomicAdd(R.steps + 1, 1ull);
        const int nproc = growing ? min(ncav - head, G / 4) : 0;
        const bool valid = (L.sub >> 2) < nproc;
        const int i = L.sub & 3;
        int c = 0, nb = 0;
        int kind = 0;   // 0: nothing, 1: boundary facet, 2: new region tet, 3: re-check
        bool abort = false;
        if (valid) {
            c = cav[head + (L.sub >> 2)];
            nb = at(T.tn[c], i) >> 2;
            const unsigned long long old = atomicMin(T.claim + nb, key | 1ull);
            if (old == key) {
                kind = 0;                               // already in the region
            } else if (old == (key | 1ull)) {
                kind = 3;                               // seen by us: decided below
            } else if ((old >> 1) < mine) {
                abort = true;                           // an earlier point holds it
            } else {
                const int r = conflict_test(T.tv[nb], p, v, vx, ex, R.status);
                ctr.count(r);
                if (r & CT_IN) {
                    const unsigned long long o2 = atomicMin(T.claim + nb, key);
                    if ((o2 >> 1) < mine) abort = true;
                    else kind = 2;
                } else {
                    kind = 1;
                }
            }
        }
        const unsigned ab0 = L.own(__ballot_sync(kFull, abort));
        if (growing && ab0) {
            if (L.sub == 0) W.state[w] = WS_LOST;
            growing = false;
        }
        __syncwarp();
        if (growing && kind == 3) {
            // Another lane of this step may have just turned it into a region tet.
            const unsigned long long now = __ldcg(T.claim + nb);
            if (now == key) kind = 0;
            else if ((now >> 1) < mine) abort = true;
            else kind = 1;
        }
        const unsigned ab = L.own(__ballot_sync(kFull, growing && abort));
        if (growing && ab) {
            if (L.sub == 0) W.state[w] = WS_LOST;
            growing = false;
        }
        const unsigned mc = __ballot_sync(kFull, growing && kind == 2) & L.gm;
        const unsigned mf = __ballot_sync(kFull, growing && kind == 1) & L.gm;
        if (growing && (ncav + __popc(mc) > W.cav_cap || nfac + __popc(mf) > W.fac_cap)) {
            if (L.sub == 0) {
                // Too big for this scratch: park the worker until a big round
                // (or, in a big round, report that even that was not enough).
                W.state[w] = WS_PARKED;
                if (W.list) report(R.status, ST_CAVITY_CAPACITY);
                else W.parked[w] = 1;
                atomicAdd(R.counters + 3, 1);   // its claims may have blocked others
            }
            growing = false;
        }
        if (growing) {
            if (kind == 2) cav[ncav + __popc(mc & lt)] = nb;
            if (kind == 1) fac[nfac + __popc(mf & lt)] = c * 4 + i;
            ncav += __popc(mc);
            nfac += __popc(mf);
            head += nproc;
            if (head >= ncav) {
                if (L.sub == 0) {
                    W.ncav[w] = ncav;
                    W.nfac[w] = nfac;
                    W.state[w] = WS_CAND;
                }
                growing = false;
            }
        }
        __syncwarp();
    }
    flush_counters(ctr, R);
}

/// One group per candidate: it wins if it still holds every claim it made.
template <int G>
__global__ void __launch_bounds__(128, 8) k_check(Tables T, Workers W, Round R, int first) {
    const Lanes<G> L;
    const int slot = first + int((blockIdx.x * blockDim.x + threadIdx.x) / G);
    bool live = slot < W.n;
    int w = 0;
    if (live) {
        w = W.list ? W.list[slot] : slot;
        live = W.state[w] == WS_CAND;
    }
    if (!__any_sync(kFull, live)) return;
    bool ok = true;
    if (live) {
        const int v = W.cur[w];
        const unsigned long long key = claim_key(R, v);
        const int* cav = W.cav + int64_t(slot) * W.cav_cap;
        const int* fac = W.fac + int64_t(slot) * W.fac_cap;
        const int ncav = W.ncav[w], nfac = W.nfac[w];
        for (int k = L.sub; k < ncav; k += G) ok = ok && T.claim[cav[k]] == key;
        for (int k = L.sub; k < nfac; k += G) {
            const int f = fac[k];
            ok = ok && T.claim[at(T.tn[f >> 2], f & 3) >> 2] == (key | 1ull);
        }
    }
    const bool win = L.own(__ballot_sync(kFull, !ok)) == 0;
    if (live && L.sub == 0) {
        W.state[w] = win ? WS_WIN : WS_LOST;
        if (win) atomicMax(R.pstats + 3, (unsigned long long)W.ncav[w]);
    }
}

/// Neighbour of new tet facet j (the new tet replaces facet i of region tet c):
/// facet j is {v} + edge (va, vb), and its neighbour is the new tet on the other
/// boundary facet through that edge, reached by turning around the edge inside
/// the region (reference src/tds.h:160-221).  Returns the encoded neighbour
/// (tet * 4 + facet), or -1 if the region is inconsistent.
__device__ int restar_neighbour(const Tables& T, int c, const int4& cv, int i, int j,
                                unsigned long long key) {
    int a = -1, b = -1;
    for (int m = 0; m < 4; ++m)
        if (m != i && m != j) {
            if (a < 0) a = m;
            else b = m;
        }
    const int va = at(cv, a), vb = at(cv, b);
    int cur = c, f = j, steps = 0;
    for (;;) {
        const int enc = at(T.tn[cur], f);
        const int nb = enc >> 2;
        if (T.claim[nb] != key) {   // (cur, f) is a boundary facet
            const int4 tc = T.tv[cur];
            const int wpos = 6 - f - pos_of(tc, va) - pos_of(tc, vb);
            if (wpos < 0 || wpos > 3 || wpos == f) return -1;
            return T.fnew[cur * 4 + f] * 4 + wpos;
        }
        const int4 tb = T.tv[nb];
        const int g = enc & 3;
        f = 6 - g - pos_of(tb, va) - pos_of(tb, vb);
        cur = nb;
        if (f < 0 || f > 3 || f == g || ++steps > kRotateLimit) return -1;
    }
}

/// One group per winner: re-star its region, one boundary facet per lane.
template <int G>
__global__ void __launch_bounds__(128, 8) k_restar(Tables T, Workers W, Round R, int first) {
    __shared__ int sh_count[3];
    const Lanes<G> L;
    const int slot = first + int((blockIdx.x * blockDim.x + threadIdx.x) / G);
    if (threadIdx.x < 3) sh_count[threadIdx.x] = 0;
    __syncthreads();
    const bool exists = slot < W.n;
    const int w = exists ? (W.list ? W.list[slot] : slot) : 0;
    const int state = exists ? W.state[w] : WS_DONE;
    const int v = exists ? W.cur[w] : -1;
    const bool winner = state == WS_WIN;
    bool advanced = false;
    if (__any_sync(kFull, winner)) {
        const unsigned long long key = winner ? claim_key(R, v) : 0ull;
        const int64_t sl = winner ? slot : 0;
        const int* cav = W.cav + sl * W.cav_cap;
        const int* fac = W.fac + sl * W.fac_cap;
        int4* sv = W.st_v + sl * W.fac_cap;
        int4* sn = W.st_n + sl * W.fac_cap;
        const int C = winner ? W.ncav[w] : 0, F = winner ? W.nfac[w] : 0;
        const int extra = F > C ? F - C : 0;
        int base = 0, ok = winner ? 1 : 0;
        if (winner && L.sub == 0 && extra > 0) {
            base = atomicAdd(T.tet_count, extra);
            if (base + extra > T.cap) {
                report(R.status, ST_TET_CAPACITY);
                ok = 0;
            }
        }
        base = __shfl_sync(kFull, base, L.gbase);
        ok = __shfl_sync(kFull, ok, L.gbase);
        // 1a: the new tet of each boundary facet.
        if (ok)
            for (int k = L.sub; k < F; k += G) T.fnew[fac[k]] = k < C ? cav[k] : base + (k - C);
        __syncwarp();
        // 1b: vertices and neighbours, from the region as it was.
        bool bad = false;
        for (int k0 = 0; __any_sync(kFull, ok && k0 < F); k0 += G) {
            const int k = k0 + L.sub;
            if (ok && k < F) {
                const int c = fac[k] >> 2, i = fac[k] & 3;
                const int4 cv = T.tv[c];
                const int4 cn = T.tn[c];
                int4 nv = cv, nn = cn;
                set_at(nv, i, v);
                for (int j = 0; j < 4 && !bad; ++j) {
                    if (j == i) continue;
                    const int e = restar_neighbour(T, c, cv, i, j, key);
                    if (e < 0) bad = true;
                    else set_at(nn, j, e);
                }
                sv[k] = nv;
                sn[k] = nn;
            }
        }
        if (L.own(__ballot_sync(kFull, bad))) {
            if (L.sub == 0) report(R.status, ST_INTERNAL);
            ok = 0;
        }
        __syncwarp();
        if (ok) {
            // 2: write the new tets and re-point the outside neighbours.
            for (int k = L.sub; k < F; k += G) {
                const int id = k < C ? cav[k] : base + (k - C);
                const int4 nv = sv[k], nn = sn[k];
                const int i = fac[k] & 3;
                T.tv[id] = nv;
                T.tn[id] = nn;
                T.alive[id] = 1;
                const int enc = at(nn, i);
                reinterpret_cast<int*>(T.tn)[(enc >> 2) * 4 + (enc & 3)] = id * 4 + i;
                if (nv.x != kInf) T.vert_tet[nv.x] = id;
                if (nv.y != kInf) T.vert_tet[nv.y] = id;
                if (nv.z != kInf) T.vert_tet[nv.z] = id;
                if (nv.w != kInf) T.vert_tet[nv.w] = id;
            }
            for (int k = F + L.sub; k < C; k += G) T.alive[cav[k]] = 0;
            advanced = true;
            if (L.sub == 0) {
                atomicAdd(R.sums, (unsigned long long)C);
                atomicAdd(R.sums + 1, (unsigned long long)F);
            }
        }
    }
    if (L.sub == 0 && exists) {
        int cur = v;
        if (advanced) {
            W.last[w] = v;
            W.parked[w] = 0;
            W.nwon[w] += 1;
            cur = next_point(W, w);
        }
        if (cur >= 0 && W.parked[w]) atomicAdd(sh_count + 1, 1);     // waits for a big round
        else if (state != WS_DONE && cur >= 0) atomicAdd(sh_count, 1);
        if (advanced) atomicAdd(sh_count + 2, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (sh_count[0]) atomicAdd(R.counters, sh_count[0]);
        if (sh_count[1]) atomicAdd(R.counters + 1, sh_count[1]);
        if (sh_count[2]) atomicAdd(R.counters + 2, sh_count[2]);
    }
}

// ---- asynchronous insertion --------------------------------------------------
//
// The rounds above insert in lockstep: every round waits for its slowest
// worker.  k_insert_async lets every warp run at its own pace instead.  A
// persistent grid of warps takes the level's chunks from a queue and inserts
// their points one after another.  An insertion try-locks every tet it reads
// to decide its conflict region - the region tets and the tets across the
// region boundary - and holds the locks until its new tets are written, so
// insertions whose locks succeed touch disjoint tets and commute: the result
// is that of some sequential order, hence (the tet set does not depend on the
// insertion order) the canonical set.  A lock held by another warp makes the
// insertion give back its locks and try again after a back-off; after a few
// failures, and for a conflict region too large for the warp's scratch, the
// point is left for the rounds, which finish it.  No warp ever waits while it
// holds a lock, and every loop is bounded.
//
// Lock word of a tet: 0 free, else (owner << 1) | ring, owner = warp slot + 1;
// ring = 1 for a tet across the region boundary, 0 for a region tet.  Locks are
// taken with acquire and released with release ordering, and every read of
// tet data that other warps write goes to L2 (__ldcg), not the SM's L1.

constexpr int kAsyncRetries = 6;
// Passes of the full variant over a level's left points before the rounds.
constexpr int kLeftPasses = 8;
// BRIO level growth of the build's own order when a set's filters are exact,
// or when the whole build has fewer than kSmallBuildPoints points.
constexpr int kExactSetGrowth = 4;
constexpr int64_t kSmallBuildPoints = 65536;
constexpr int kAsyncWalkLimit = 1 << 14;
// The neighbour records of a warp's first kHandedTn region tets, read under
// their locks together with their vertices, are kept in shared memory for the
// growth step that expands them (instead of being read from L2 again there).
constexpr int kHandedTn = 64;

struct AsyncCtx {
    int* lock;                      // per tet lock word
    int* next;                      // chunk queue head
    int* leftover;                  // points left for the rounds
    int* n_leftover;
    int64_t stride;                 // entry q of the queue is worker (q * stride) % nw
    int nw;
    unsigned long long* ekey;       // per warp slot: 3 edge keys per boundary facet (re-star)
    unsigned long long* stats;      // [0] lock conflicts, [1] walk restarts, [2] invalid seeds,
                                    // [3] regions too big, [4] points left, [5] first points left,
                                    // [6] points deferred by the fast variant
};

using LockRef = cuda::atomic_ref<int, cuda::thread_scope_device>;

__device__ __forceinline__ bool try_lock(int* lock, int t, int value, int* seen) {
    int expected = 0;
    const bool ok = LockRef(lock[t]).compare_exchange_strong(expected, value, cuda::memory_order_acquire,
                                                             cuda::memory_order_relaxed);
    *seen = ok ? 0 : expected;
    return ok;
}

/// Releases tet t if `value` still holds it (a ring tet may be listed twice).
__device__ __forceinline__ void unlock_if(int* lock, int t, int value) {
    int expected = value;
    LockRef(lock[t]).compare_exchange_strong(expected, 0, cuda::memory_order_release, cuda::memory_order_relaxed);
}

__device__ __forceinline__ int4 ld4(const int4* p) { return __ldcg(p); }

/// orient3d of tet (a, b, c, d) with vertex `i` replaced by p, from the filter
/// alone: the sign when the filter decides it (or `ex`: the set's coordinates
/// make the filter's value exact), else 2.  Selects, no calls and no local
/// arrays, so that it adds nothing to the caller's live state.
__device__ __forceinline__ int orient_replaced_filter(const Pt& a, const Pt& b, const Pt& c, const Pt& d, int i,
                                                      const Pt& p, bool ex) {
    const Pt A = i == 0 ? p : a, B = i == 1 ? p : b, C = i == 2 ? p : c, D = i == 3 ? p : d;
    const Orient3dFilter f = orient3d_filter(A, B, C, D);
    if (f.certain || ex) return -sign_of(f.det);
    return 2;
}

/// Visibility walk on a mesh other warps are changing: reads go to L2 and may
/// be stale, so the tet it returns is only a candidate, checked under its lock.
/// Returns -1 after kAsyncWalkLimit steps (or the build's walk limit, if lower).
/// kFast: orientations come from the filter alone, and a step the filter cannot
/// decide ends the walk with -2 (the point is left to the other variant, which
/// runs the exact stage).
template <bool kFast>
__device__ int walk_async(int t, const Pt& p, int pid, const Tables& T, const double* __restrict__ vx,
                          bool ex, uint32_t* st, int lane) {
    int4 tv = ld4(T.tv + t);
    {
        const int ip = inf_pos(tv);
        if (ip >= 0) {
            t = at(ld4(T.tn + t), ip) >> 2;
            tv = ld4(T.tv + t);
        }
    }
    int4 tn = ld4(T.tn + t);
    int prev = -1;
    uint32_t h = uint32_t(pid) * 2654435761u + 12345u;
    const int limit = min(kAsyncWalkLimit, T.walk_limit);
    for (int step = 0; step < limit; ++step) {
        // While lanes 0-3 test the four facets, lanes 4-7 fetch the four
        // neighbours' vertices and lanes 8-11 their neighbours: the step to
        // the chosen neighbour then waits for no further memory read.
        int4 pre = make_int4(0, 0, 0, 0);
        if (lane >= 4 && lane < 12) {
            const int nbr = at(tn, lane & 3) >> 2;
            pre = lane < 8 ? ld4(T.tv + nbr) : ld4(T.tn + nbr);
        }
        h = h * 1664525u + 1013904223u;
        const int s0 = int(h >> 30);
        bool neg = false, undecided = false;
        if (lane < 4 && (at(tn, lane) >> 2) != prev && tv.x != kInf && tv.y != kInf && tv.z != kInf &&
            tv.w != kInf) {
            const Pt a = vpt(vx, tv.x), b = vpt(vx, tv.y), c = vpt(vx, tv.z), d = vpt(vx, tv.w);
            int o = orient_replaced_filter(a, b, c, d, lane, p, ex);
            if (o == 2) {
                if (kFast) {
                    undecided = true;
                    o = 0;
                } else {
                    const Pt A = lane == 0 ? p : a, B = lane == 1 ? p : b, C = lane == 2 ? p : c,
                             D = lane == 3 ? p : d;
                    o = orient3d(A, B, C, D, st);
                }
            }
            neg = o < 0;
        }
        if (kFast && __any_sync(kFull, undecided)) return -2;
        const unsigned m = __ballot_sync(kFull, neg) & 0xFu;
        if (m == 0) return t;
        const unsigned rot = ((m >> s0) | (m << (4 - s0))) & 0xFu;
        const int i = (s0 + __ffs(int(rot)) - 1) & 3;
        const int next = at(tn, i) >> 2;
        const int4 nv = make_int4(__shfl_sync(kFull, pre.x, 4 + i), __shfl_sync(kFull, pre.y, 4 + i),
                                  __shfl_sync(kFull, pre.z, 4 + i), __shfl_sync(kFull, pre.w, 4 + i));
        const int4 nn = make_int4(__shfl_sync(kFull, pre.x, 8 + i), __shfl_sync(kFull, pre.y, 8 + i),
                                  __shfl_sync(kFull, pre.z, 8 + i), __shfl_sync(kFull, pre.w, 8 + i));
        if (inf_pos(nv) >= 0) return next;
        prev = t;
        t = next;
        tv = nv;
        tn = nn;
    }
    return -1;
}

/// A vertex coordinate read again from memory (the read-only path), as a
/// volatile load so that the compiler does not keep an earlier read of it
/// alive in registers across the code in between.
__device__ __forceinline__ double ld_coord(const double* p) {
    double v;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ Pt ld_vertex(const double* __restrict__ vx, int v) {
    const double* q = vx + 3 * int64_t(v);
    return Pt{ld_coord(q), ld_coord(q + 1), ld_coord(q + 2)};
}

/// The symbolic perturbation of an exactly cospherical in_sphere(a, b, c, d, p)
/// (reference src/predicates.cpp:206-232) for the conflict test of tet t and
/// vertex pid, when the set's coordinates make the orient3d filter exact.  The
/// five points are distinct vertices, so their lexicographic order is strict:
/// walking down it from the largest, the largest is p -> NEGATIVE; else the
/// orient3d with that point's slot replaced by p decides if it is not zero;
/// else the next largest, once more; else NEGATIVE.  Points are read again
/// from memory each time they are needed, so the tie-break adds no live state
/// to the loop around it.
__device__ __forceinline__ int in_sphere_tiebreak_ex(const int4 t, int pid, const double* __restrict__ vx) {
    int skip = -1;
#pragma unroll 1
    for (int r = 0; r < 2; ++r) {
        int best = -1;
        Pt bp{0.0, 0.0, 0.0};
#pragma unroll 1
        for (int k = 0; k < 5; ++k) {
            if (k == skip) continue;
            const Pt q = ld_vertex(vx, k < 4 ? at(t, k) : pid);
            if (best < 0 || lexico_less(bp, q)) {
                best = k;
                bp = q;
            }
        }
        if (best == 4) return -1;
        const Pt pp = ld_vertex(vx, pid);
        const Pt A = best == 0 ? pp : ld_vertex(vx, t.x), B = best == 1 ? pp : ld_vertex(vx, t.y),
                 C = best == 2 ? pp : ld_vertex(vx, t.z), D = best == 3 ? pp : ld_vertex(vx, t.w);
        const int o = -sign_of(orient3d_filter(A, B, C, D).det);
        if (o != 0) return o;
        skip = best;
    }
    return -1;
}

/// in_sphere_filter's arithmetic, operation for operation (so its value and
/// its decision are bit-identical), in an order that retires values early:
/// lifts right after the differences, each product pair folded at once into
/// its minor and its permanent pair sum (|x*y| = |x|*|y| exactly).
__device__ __forceinline__ InSphereFilter in_sphere_filter_lean(const Pt& a, const Pt& b, const Pt& c, const Pt& d,
                                                                const Pt& e) {
    const double aex = fsub(a.x, e.x), aey = fsub(a.y, e.y), aez = fsub(a.z, e.z);
    const double bex = fsub(b.x, e.x), bey = fsub(b.y, e.y), bez = fsub(b.z, e.z);
    const double cex = fsub(c.x, e.x), cey = fsub(c.y, e.y), cez = fsub(c.z, e.z);
    const double dex = fsub(d.x, e.x), dey = fsub(d.y, e.y), dez = fsub(d.z, e.z);
    const double alift = fadd(fadd(fmul(aex, aex), fmul(aey, aey)), fmul(aez, aez));
    const double blift = fadd(fadd(fmul(bex, bex), fmul(bey, bey)), fmul(bez, bez));
    const double clift = fadd(fadd(fmul(cex, cex), fmul(cey, cey)), fmul(cez, cez));
    const double dlift = fadd(fadd(fmul(dex, dex), fmul(dey, dey)), fmul(dez, dez));
    double ab, bc, cd, da, ac, bd, sab, sbc, scd, sda, sac, sbd;
    {
        const double p = fmul(aex, bey), q = fmul(bex, aey);
        ab = fsub(p, q);
        sab = fadd(fabs_(p), fabs_(q));
    }
    {
        const double p = fmul(bex, cey), q = fmul(cex, bey);
        bc = fsub(p, q);
        sbc = fadd(fabs_(p), fabs_(q));
    }
    {
        const double p = fmul(cex, dey), q = fmul(dex, cey);
        cd = fsub(p, q);
        scd = fadd(fabs_(p), fabs_(q));
    }
    {
        const double p = fmul(dex, aey), q = fmul(aex, dey);
        da = fsub(p, q);
        sda = fadd(fabs_(p), fabs_(q));
    }
    {
        const double p = fmul(aex, cey), q = fmul(cex, aey);
        ac = fsub(p, q);
        sac = fadd(fabs_(p), fabs_(q));
    }
    {
        const double p = fmul(bex, dey), q = fmul(dex, bey);
        bd = fsub(p, q);
        sbd = fadd(fabs_(p), fabs_(q));
    }
    const double abc = fadd(fsub(fmul(aez, bc), fmul(bez, ac)), fmul(cez, ab));
    const double bcd = fadd(fsub(fmul(bez, cd), fmul(cez, bd)), fmul(dez, bc));
    const double cda = fadd(fadd(fmul(cez, da), fmul(dez, ac)), fmul(aez, cd));
    const double dab = fadd(fadd(fmul(dez, ab), fmul(aez, bd)), fmul(bez, da));
    const double det = fadd(fsub(fmul(dlift, abc), fmul(clift, dab)), fsub(fmul(blift, cda), fmul(alift, bcd)));
    const double aezp = fabs_(aez), bezp = fabs_(bez), cezp = fabs_(cez), dezp = fabs_(dez);
    const double pa = fadd(fadd(fmul(scd, bezp), fmul(sbd, cezp)), fmul(sbc, dezp));
    const double pb = fadd(fadd(fmul(sda, cezp), fmul(sac, dezp)), fmul(scd, aezp));
    const double pc = fadd(fadd(fmul(sab, dezp), fmul(sbd, aezp)), fmul(sda, bezp));
    const double pd = fadd(fadd(fmul(sbc, aezp), fmul(sac, bezp)), fmul(sab, cezp));
    const double permanent = fadd(fadd(fadd(fmul(pa, alift), fmul(pb, blift)), fmul(pc, clift)), fmul(pd, dlift));
    const double errbound = fmul(kInSphereBound, permanent);
    InSphereFilter r;
    r.det = det;
    r.certain = (det > errbound) || (-det > errbound);
    return r;
}

/// coplanar_orientation3 (the first non-zero orient2d of the xy, yz and xz
/// projections) for a set whose coordinates make the orient2d determinants
/// exact in double: each is the sign of its determinant.
__device__ __forceinline__ int coplanar_orientation3_ex(const Pt& p, const Pt& q, const Pt& r) {
    int o = sign_of(fsub(fmul(fsub(q.x, p.x), fsub(r.y, p.y)), fmul(fsub(q.y, p.y), fsub(r.x, p.x))));
    if (o != 0) return o;
    o = sign_of(fsub(fmul(fsub(q.y, p.y), fsub(r.z, p.z)), fmul(fsub(q.z, p.z), fsub(r.y, p.y))));
    if (o != 0) return o;
    return sign_of(fsub(fmul(fsub(q.x, p.x), fsub(r.z, p.z)), fmul(fsub(q.z, p.z), fsub(r.x, p.x))));
}

/// The cocircular tie-break (reference src/predicates2.cpp:241-258) of four
/// distinct vertices va, vb, vd, pid of such a set: walking down their
/// lexicographic order from the largest, the first that is pid gives NEGATIVE;
/// the first other one whose replacement by pid gives a non-zero coplanar
/// orientation gives it times the orientation of (va, vb, vd); else the
/// opposite of that orientation.  Points are read again from memory, as in
/// in_sphere_tiebreak_ex.
__device__ __forceinline__ int in_circle_tiebreak_ex(int va, int vb, int vd, int pid,
                                                     const double* __restrict__ vx) {
    const int local = coplanar_orientation3_ex(ld_vertex(vx, va), ld_vertex(vx, vb), ld_vertex(vx, vd));
    unsigned excluded = 0;
#pragma unroll 1
    for (int r = 0; r < 3; ++r) {
        int best = -1;
        Pt bp{0.0, 0.0, 0.0};
#pragma unroll 1
        for (int k = 0; k < 4; ++k) {
            if (excluded & (1u << k)) continue;
            const Pt q = ld_vertex(vx, k == 0 ? va : (k == 1 ? vb : (k == 2 ? vd : pid)));
            if (best < 0 || !lexico_less(q, bp)) {   // a later slot wins ties
                best = k;
                bp = q;
            }
        }
        excluded |= 1u << best;
        if (best == 3) return -1;
        const Pt pp = ld_vertex(vx, pid);
        const Pt A = best == 0 ? pp : ld_vertex(vx, va), B = best == 1 ? pp : ld_vertex(vx, vb),
                 C = best == 2 ? pp : ld_vertex(vx, vd);
        const int o = coplanar_orientation3_ex(A, B, C);
        if (o != 0) return o * local;
    }
    return -local;
}

/// The hull in-circle test (reference src/triangulation.cpp:588-602, a point
/// in the plane of the hull facet (va, vb, vd) of infinite tet `tet`: in
/// conflict iff inside the facet's circumcircle, a tie by the cocircular
/// perturbation) for a set whose coordinates make the filters exact, without
/// the in-circle determinant: the sphere through va, vb, vd and the apex x of
/// the finite tet across the facet cuts the facet's plane in the facet's
/// circumcircle, and a point of that plane has the same power with respect
/// to both, so sign in_circle(va, vb, vd, p) = sign det_in_sphere(va, vb, vd,
/// x, p) * sign det_orient3d(va, vb, vd, x), both exact here.  The caller
/// holds the lock of `tet`, so the finite tet across its facet is not being
/// rewritten.  Returns 1 (inside), -1 (outside), or 0 if the apex is unusable
/// (the caller then leaves the test undecided).
__device__ __forceinline__ int hull_in_circle_ex(const Tables& T, int tet, int ip, int va, int vb, int vd, int pid,
                                                 const double* __restrict__ vx) {
    const int f = at(ld4(T.tn + tet), ip) >> 2;
    const int4 fv = ld4(T.tv + f);
    int x = -1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int w = at(fv, k);
        if (w != va && w != vb && w != vd) x = w;
    }
    if (x < 0) return 0;   // kInf is negative
    const Pt a = ld_vertex(vx, va), b = ld_vertex(vx, vb), d = ld_vertex(vx, vd), xp = ld_vertex(vx, x);
    const int so = sign_of(orient3d_filter(a, b, d, xp).det);
    if (so == 0) return 0;
    const int ss = sign_of(in_sphere_filter_lean(a, b, d, xp, ld_vertex(vx, pid)).det);
    if (ss != 0) return ss * so;
    return in_circle_tiebreak_ex(va, vb, vd, pid, vx);
}

/// The conflict test of the fast variant (reference src/triangulation.cpp:588-602,
/// as conflict_test) of tet `tet` = t, with its outcome bits; CT_UNDECIDED when
/// the filter cannot decide and the exact stage is needed, or the point lies in
/// the plane of a hull facet (the coplanar in-circle test) of a set whose
/// filters are not exact.  Call-free: on a set whose coordinates make the
/// filters exact, an exactly cospherical call gets its tie-break inline, and
/// a point in the plane of a hull facet its in-circle test.
__device__ __forceinline__ int in_conflict_fast(const Tables& T, int tet, const int4 t, const Pt& p, int pid,
                                                const double* __restrict__ vx, bool ex) {
    const int ip = inf_pos(t);
    if (ip >= 0) {
        const int o0 = ip == 0 ? 2 : (ip == 1 ? 2 : (ip == 2 ? 1 : 0));
        const int o1 = ip == 0 ? 1 : (ip == 1 ? 3 : (ip == 2 ? 0 : 1));
        const int o2 = ip == 0 ? 3 : (ip == 1 ? 0 : (ip == 2 ? 3 : 2));
        const Pt a = vpt(vx, at(t, o0)), b = vpt(vx, at(t, o1)), d = vpt(vx, at(t, o2));
        const Orient3dFilter f = orient3d_filter(a, b, d, p);
        if (f.certain) return f.det < 0.0 ? CT_IN : 0;   // orient3d = -sign(det)
        if (ex && f.det != 0.0) return (f.det < 0.0 ? CT_IN : 0) | CT_UNCERTAIN;
        if (ex) {
            const int h = hull_in_circle_ex(T, tet, ip, at(t, o0), at(t, o1), at(t, o2), pid, vx);
            if (h != 0) return (h > 0 ? CT_IN : 0) | CT_UNCERTAIN | CT_TIE;
        }
        return CT_UNDECIDED;
    }
    const Pt a = vpt(vx, t.x), b = vpt(vx, t.y), c = vpt(vx, t.z), d = vpt(vx, t.w);
    const InSphereFilter f = in_sphere_filter_lean(a, b, c, d, p);
    if (f.certain) return f.det < 0.0 ? CT_IN : 0;   // in_sphere = -sign(det)
    if (ex && f.det != 0.0) return (f.det < 0.0 ? CT_IN : 0) | CT_UNCERTAIN;
    if (ex) return (in_sphere_tiebreak_ex(t, pid, vx) > 0 ? CT_IN : 0) | CT_UNCERTAIN | CT_TIE;
    return CT_UNDECIDED;
}

enum : int { AI_DONE = 0, AI_RETRY = 1, AI_LEAVE = 2, AI_DEFER = 3 };

/// Key of the edge (a, b), either order.
__device__ __forceinline__ unsigned long long edge_key(int a, int b) {
    const unsigned ua = unsigned(a + 1), ub = unsigned(b + 1);
    return ua < ub ? ((unsigned long long)ua << 32) | ub : ((unsigned long long)ub << 32) | ua;
}

/// Edge keys of facets p0 < p1 < p2 (the positions other than i) of a tet with
/// vertices c: facet j's edge joins the two positions other than i and j.
__device__ __forceinline__ void facet_edge_keys(const int4 c, int i, unsigned long long& e0,
                                                unsigned long long& e1, unsigned long long& e2) {
    const int p0 = i == 0 ? 1 : 0, p1 = i <= 1 ? 2 : 1, p2 = i <= 2 ? 3 : 2;
    const int a0 = at(c, p0), a1 = at(c, p1), a2 = at(c, p2);
    e0 = edge_key(a1, a2);
    e1 = edge_key(a0, a2);
    e2 = edge_key(a0, a1);
}

/// One insertion of point v by the whole warp, starting the walk at tet t0.
/// AI_DONE: inserted; AI_RETRY: a lock was taken by another warp (nothing
/// changed, every lock given back); AI_LEAVE: leave it for the rounds;
/// AI_DEFER (kFast only): a test the filter could not decide, nothing changed,
/// leave it for the other variant.
///
/// kFast = true is the variant for the bulk of the points: its walk and
/// conflict tests use the filters alone and make no calls.  A call anywhere in
/// the insertion loop - even one the uniform case never takes - makes the
/// compiler keep the loop's state in local memory around it; without calls the
/// state stays in registers.  kFast = false runs the exact stage, the hull
/// in-circle test and the tie-breaks, out of line, for the points the fast
/// variant deferred.
template <bool kFast>
__device__ int insert_async(int v, int t0, const Tables& T, const Workers& W, const AsyncCtx& A,
                            const double* __restrict__ vx, bool ex, uint32_t* st, int slot, int lane,
                            unsigned long long* nC, unsigned long long* nF, const SharedCounters& ctr,
                            int4* htn) {
    const int owner = slot + 1;
    const int region = owner << 1, ring = region | 1;
    const Pt p = vpt(vx, v);
    const int seed = walk_async<kFast>(t0, p, v, T, vx, ex, st, lane);
    if (kFast && seed == -2) {
        if (lane == 0) atomicAdd(A.stats + 6, 1ull);
        return AI_DEFER;
    }
    if (seed < 0) {
        if (lane == 0) atomicAdd(A.stats + 1, 1ull);
        return AI_RETRY;
    }
    int* cav = W.cav + int64_t(slot) * W.cav_cap;
    int* fac = W.fac + int64_t(slot) * W.fac_cap;
    // Seed: lock it, then check under the lock that it is alive and in conflict.
    int res = 0;   // 0 ok, 1 lock held by another, 2 not a valid seed, 3 undecided (kFast)

    if (lane == 0) {
        int seen = 0;
        if (!try_lock(A.lock, seed, region, &seen)) {
            res = 1;
        } else {
            // The walk read tets other warps were rewriting: a tet read half
            // written (vertices new, neighbours not yet) can send it on through a
            // slot not yet filled in - into another set's tets in a batched
            // build.  Only a live tet of v's own set can seed the region.
            int r = 0;
            const int4 stv = ld4(T.tv + seed);
            htn[0] = ld4(T.tn + seed);
            if (__ldcg(T.alive + seed) && T.vset[stv.x != kInf ? stv.x : stv.y] == T.vset[v]) {
                if (kFast) r = in_conflict_fast(T, seed, stv, p, v, vx, ex);
                else r = conflict_test_seed(stv, p.x, p.y, p.z, v, vx, ex, st);
                ctr.count(r);
            }
            if (r & CT_IN) {
                cav[0] = seed;
            } else {
                unlock_if(A.lock, seed, region);
                res = (r & CT_UNDECIDED) ? 3 : 2;
            }
        }
    }
    res = __shfl_sync(kFull, res, 0);
    if (res != 0) {
        if (lane == 0) atomicAdd(A.stats + (res == 1 ? 0 : (res == 2 ? 2 : 6)), 1ull);
        return res == 3 ? AI_DEFER : AI_RETRY;
    }
    __syncwarp();
    const unsigned lt = (1u << lane) - 1u;
    int ncav = 1, nfac = 0, head = 0;
    int outcome = AI_DONE;
    while (head < ncav) {
        const int nproc = min(ncav - head, 8);
        const bool valid = (lane >> 2) < nproc;
        const int i = lane & 3;
        int c = 0, nb = 0, kind = 0, got = -1;   // got: a tet this lane locked in this step
        bool abort = false, undecided = false;
        int4 found_tn = make_int4(0, 0, 0, 0);
        if (valid) {
            const int pidx = head + (lane >> 2);
            c = cav[pidx];
            nb = at(pidx < kHandedTn ? htn[pidx] : ld4(T.tn + c), i) >> 2;
            int seen = 0;
            if (try_lock(A.lock, nb, ring, &seen)) {
                got = nb;
                int r;
                const int4 ntv = ld4(T.tv + nb);
                found_tn = ld4(T.tn + nb);
                if (kFast) r = in_conflict_fast(T, nb, ntv, p, v, vx, ex);
                else r = conflict_test(ntv, p, v, vx, ex, st);
                ctr.count(r);
                if (r & CT_IN) {
                    LockRef(A.lock[nb]).store(region, cuda::memory_order_relaxed);
                    kind = 2;
                } else {
                    kind = 1;                             // undecided: held as ring
                    undecided = (r & CT_UNDECIDED) != 0;
                }
            } else if (seen == region) {
                kind = 0;                                 // already in the region
            } else if (seen == ring) {
                kind = 3;                                 // locked by us this step: decided below
            } else {
                abort = true;                             // another warp holds it
            }
        }
        __syncwarp();
        if (kind == 3) kind = __ldcg(A.lock + nb) == region ? 0 : 1;
        const bool ab = __any_sync(kFull, abort);
        const bool und = kFast && __any_sync(kFull, undecided);
        const unsigned mc = __ballot_sync(kFull, kind == 2);
        const unsigned mf = __ballot_sync(kFull, kind == 1);
        const bool full = ncav + __popc(mc) > W.cav_cap || nfac + __popc(mf) > W.fac_cap;
        if (ab || full || und) {
            // Give everything back: this step's new locks, the region, the ring.
            if (got >= 0) unlock_if(A.lock, got, kind == 2 ? region : ring);
            __syncwarp();
            for (int k = lane; k < nfac; k += 32) {
                const int f = fac[k];
                unlock_if(A.lock, at(ld4(T.tn + (f >> 2)), f & 3) >> 2, ring);
            }
            __syncwarp();
            for (int k = lane; k < ncav; k += 32) unlock_if(A.lock, cav[k], region);
            if (lane == 0) atomicAdd(A.stats + (ab ? 0 : (und ? 6 : 3)), 1ull);
            outcome = ab ? AI_RETRY : (und ? AI_DEFER : AI_LEAVE);
            break;
        }
        if (kind == 2) cav[ncav + __popc(mc & lt)] = nb;
        if (kind == 1) fac[nfac + __popc(mf & lt)] = c * 4 + i;
        if (kind == 2 && ncav + __popc(mc & lt) < kHandedTn) htn[ncav + __popc(mc & lt)] = found_tn;
        ncav += __popc(mc);
        nfac += __popc(mf);
        head += nproc;
        __syncwarp();
    }
    if (outcome != AI_DONE) return outcome;

    // Re-star (as k_restar), reading the locked region through L2.
    const int C = ncav, F = nfac;
    const int extra = F > C ? F - C : 0;
    int base = 0, ok = 1;
    if (lane == 0 && extra > 0) {
        base = atomicAdd(T.tet_count, extra);
        if (base + extra > T.cap) {
            report(st, ST_TET_CAPACITY);
            ok = 0;
        }
    }
    base = __shfl_sync(kFull, base, 0);
    ok = __shfl_sync(kFull, ok, 0);
    int4* sv = W.st_v + int64_t(slot) * W.fac_cap;
    int4* sn = W.st_n + int64_t(slot) * W.fac_cap;
    // Fresh slots are locked too, so that whoever locks one later reads it only
    // after this warp's release.  A stale walk of another warp may hold one for
    // a moment (it finds it not alive and lets go): wait for that, bounded.
    bool locked_fresh = true;
    if (ok) {
        for (int k = C + lane; k < F; k += 32) {
            int seen = 0;
            bool got = false;
            for (int it = 0; it < (1 << 16) && !got; ++it) {
                got = try_lock(A.lock, base + (k - C), region, &seen);
                if (!got) __nanosleep(128);
            }
            locked_fresh = locked_fresh && got;
        }
        if (!__all_sync(kFull, locked_fresh)) {
            for (int k = C + lane; k < F; k += 32) unlock_if(A.lock, base + (k - C), region);
            if (lane == 0) report(st, ST_INTERNAL);
            ok = 0;
        }
    }
    if (ok) {
        // New tet k (on boundary facet (c, i), vertex i of c replaced by v) keeps
        // c's outside neighbour across facet i.  Its facet j != i is v plus the
        // edge of c's vertices at the other two positions; that edge lies on
        // exactly one other boundary facet k2, where it is the edge of some
        // facet j2 of new tet k2: the two new tets meet there, k2 facing back
        // through j2.  Matching edge keys gives the same adjacency as turning
        // round the edge inside the region (reference src/tds.h:160-221)
        // without reading the mesh again.  The keys go through the warp's key
        // scratch, which stays in L1 (a shared-memory hash table per warp was
        // slower: the shared memory it takes comes out of L1).
        unsigned long long* keys = A.ekey + int64_t(slot) * 3 * W.fac_cap;
        for (int k = lane; k < F; k += 32) {
            const int c = fac[k] >> 2, i = fac[k] & 3;
            const int4 cv = ld4(T.tv + c);
            int4 nv = cv;
            set_at(nv, i, v);
            sv[k] = nv;
            sn[k] = ld4(T.tn + c);
            facet_edge_keys(cv, i, keys[3 * k], keys[3 * k + 1], keys[3 * k + 2]);
        }
        __syncwarp();
        bool bad = false;
        for (int k = lane; k < F; k += 32) {
            // One pass over the keys of every other facet finds the partners of
            // all three edges (key m of facet k2 is its edge m: each edge key
            // must occur on exactly one other facet).  The lanes walk the keys
            // in step, so every load is a broadcast.
            const unsigned long long e0 = keys[3 * k], e1 = keys[3 * k + 1], e2 = keys[3 * k + 2];
            int f0 = -1, f1 = -1, f2 = -1, n0 = 0, n1 = 0, n2 = 0;
            for (int o = 0; o < F; ++o) {
                const bool other = o != k;
#pragma unroll
                for (int m2 = 0; m2 < 3; ++m2) {
                    const unsigned long long key = keys[3 * o + m2];
                    const int q = 3 * o + m2;
                    if (other && key == e0) { f0 = q; ++n0; }
                    if (other && key == e1) { f1 = q; ++n1; }
                    if (other && key == e2) { f2 = q; ++n2; }
                }
            }
            const int i = fac[k] & 3;
            int4 nn = sn[k];
            // Facet j of new tet k (j != i, increasing) carries edge key m = 0, 1, 2.
            auto link = [&](int j, int found, int count) {
                if (count != 1) {
                    bad = true;
                    return;
                }
                const int k2 = found / 3, m2 = found - 3 * k2, i2 = fac[k2] & 3;
                const int j2 = m2 + (m2 >= i2 ? 1 : 0);
                set_at(nn, j, (k2 < C ? cav[k2] : base + (k2 - C)) * 4 + j2);
            };
            link(i == 0 ? 1 : 0, f0, n0);
            link(i <= 1 ? 2 : 1, f1, n1);
            link(i <= 2 ? 3 : 2, f2, n2);
            sn[k] = nn;
        }
        if (__any_sync(kFull, bad)) {
            if (lane == 0) report(st, ST_INTERNAL);
            ok = 0;
        }
        __syncwarp();
    }
    if (ok) {
        for (int k = lane; k < F; k += 32) {
            const int id = k < C ? cav[k] : base + (k - C);
            const int4 nv = sv[k], nn = sn[k];
            const int i = fac[k] & 3;
            T.tv[id] = nv;
            T.tn[id] = nn;
            T.alive[id] = 1;
            const int enc = at(nn, i);
            reinterpret_cast<int*>(T.tn)[(enc >> 2) * 4 + (enc & 3)] = id * 4 + i;
            if (nv.x != kInf) T.vert_tet[nv.x] = id;
            if (nv.y != kInf) T.vert_tet[nv.y] = id;
            if (nv.z != kInf) T.vert_tet[nv.z] = id;
            if (nv.w != kInf) T.vert_tet[nv.w] = id;
        }
        for (int k = F + lane; k < C; k += 32) T.alive[cav[k]] = 0;
    }
    // Publish, then give the locks back (ring tets first: their neighbour
    // entries now point at the new tets).
    __threadfence();
    __syncwarp();
    for (int k = lane; k < F; k += 32) {
        const int f = fac[k];
        const int c = f >> 2, i = f & 3;
        // The outside tet across facet (c, i): read from the staged neighbours,
        // since slot c may now hold a new tet.
        const int outside = ok ? (at(sn[k], i) >> 2) : (at(ld4(T.tn + c), i) >> 2);
        unlock_if(A.lock, outside, ring);
    }
    __syncwarp();
    for (int k = lane; k < C; k += 32) unlock_if(A.lock, cav[k], region);
    if (ok)
        for (int k = C + lane; k < F; k += 32) unlock_if(A.lock, base + (k - C), region);
    if (lane == 0) {
        *nC += (unsigned long long)C;
        *nF += (unsigned long long)F;
    }
    if (ok && lane == 0) ctr.region(C);
    return ok ? AI_DONE : AI_LEAVE;
}

/// Persistent warps over a level's chunks (set up by k_setup_level), or over
/// the points a pass left, one worker each (k_setup_list).  kFast: the call-free
/// variant; a point it cannot decide goes to A.leftover for the other variant.
template <bool kFast>
__global__ void __launch_bounds__(128, 8) k_insert_async(Tables T, Workers W, AsyncCtx A, Round R,
                                                      const double* __restrict__ vx, int nslots) {
    const int lane = threadIdx.x & 31;
    const int slot = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (slot >= nslots) return;   // the grid is rounded up to whole blocks; scratch has nslots slots
    unsigned long long won = 0, tries = 0, nC = 0, nF = 0;
    D3G_SHARED_COUNTERS(ctr);
    __shared__ int4 handed_tn[4][kHandedTn];   // per warp of the block
    for (;;) {
        int q = 0;
        if (lane == 0) q = atomicAdd(A.next, 1);
        q = __shfl_sync(kFull, q, 0);
        if (q >= A.nw) break;
        const int w = int((int64_t(q) * A.stride) % A.nw);
        const bool ex = W.set_exact[W.wset[w]] != 0;
        const int b = W.beg[w], len = W.end[w] - b;
        const int4 sk = W.skips[W.wset[w]];
        int pos = W.pos[w], left = W.left[w];
        int v = W.cur[w];
        int last = -1;
        const int guide = W.guide[w];
        while (v >= 0) {
            int outcome = AI_RETRY;
            for (int attempt = 0; attempt < kAsyncRetries && outcome == AI_RETRY; ++attempt) {
                if (attempt > 0) __nanosleep(200u << min(attempt, 6));
                const int t0 = __ldcg(T.vert_tet + (last >= 0 ? last : guide));
                outcome = insert_async<kFast>(v, t0, T, W, A, vx, ex, R.status, slot, lane, &nC, &nF, ctr,
                                              handed_tn[threadIdx.x >> 5]);
                ++tries;
                if (__ldcg(R.status) != 0) outcome = AI_LEAVE;
            }
            if (outcome == AI_DONE) {
                ++won;
                last = v;
            } else if (lane == 0) {
                A.leftover[atomicAdd(A.n_leftover, 1)] = v;
                atomicAdd(A.stats + 4, 1ull);
                if (last < 0) atomicAdd(A.stats + 5, 1ull);
            }
            if (__ldcg(R.status) != 0) break;
            // next point of the chunk (as next_point)
            v = -1;
            while (left > 0) {
                const int c = b + pos;
                pos = pos + 1 == len ? 0 : pos + 1;
                --left;
                if (c != sk.x && c != sk.y && c != sk.z && c != sk.w) {
                    v = c;
                    break;
                }
            }
        }
        if (__ldcg(R.status) != 0) break;
    }
    if (lane == 0) {
        atomicAdd(R.totals, won);
        atomicAdd(R.totals + 1, tries);
        atomicAdd(R.sums, nC);
        atomicAdd(R.sums + 1, nF);
    }
    flush_counters(ctr, R);
}

// ---- structural self-check (the reference's Tds::validate, src/tds.h:483-530) ----

/// Codes of the first broken invariant k_validate finds.
enum : int {
    VF_VERTEX = 1,      // a vertex out of range, or repeated in a tet, or two infinite
    VF_NEIGHBOUR = 2,   // a neighbour out of range or dead
    VF_BACK = 3,        // a neighbour that does not point back through the same facet
    VF_FACET = 4,       // two neighbours whose shared facets have different vertices
    VF_LOCK = 5,        // a tet still locked after the asynchronous passes
    VF_VERT_TET = 6,    // an inserted vertex whose tet is dead or does not contain it
    VF_SET = 7,         // a tet whose vertices belong to different point sets
};

/// One thread per tet slot, then one per vertex: checks what the reference's
/// validate() checks - distinct vertices, live neighbours that point back, no
/// mark left behind (here: no lock held), every vertex's cached tet alive and
/// containing it - and, beyond it, that each pair of neighbours shares the
/// same three vertices.  Every index is range-checked before it is followed.
/// The first failure (lowest code, then lowest slot) is recorded in `fail` =
/// code << 60 | tet or vertex << 30 | detail, and ST_INTERNAL is reported;
/// nothing traps.
__global__ void k_validate(Tables T, const int* __restrict__ lock, int ntet, int nv, uint32_t* status,
                           unsigned long long* fail) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    int code = 0, where = 0, detail = 0;
    if (i < ntet) {
        const int c = int(i);
        if (T.alive[c]) {
            const int4 tv = T.tv[c], tn = T.tn[c];
            int ninf = 0;
            for (int k = 0; k < 4 && !code; ++k) {
                const int v = at(tv, k);
                if (v < -1 || v >= nv) code = VF_VERTEX;
                ninf += v == kInf;
                for (int m = k + 1; m < 4; ++m)
                    if (v == at(tv, m)) code = VF_VERTEX;
                detail = k;
            }
            if (!code && ninf > 1) code = VF_VERTEX;
            if (!code) {
                const int s0 = T.vset[tv.x != kInf ? tv.x : tv.y];
                for (int k = 0; k < 4; ++k)
                    if (at(tv, k) != kInf && T.vset[at(tv, k)] != s0) code = VF_SET;
            }
            for (int k = 0; k < 4 && !code; ++k) {
                detail = k;
                const int e = at(tn, k);
                const int n = e >> 2, f = e & 3;
                if (e < 0 || n >= ntet || !T.alive[n]) {
                    code = VF_NEIGHBOUR;
                    break;
                }
                if (at(T.tn[n], f) != c * 4 + k) {
                    code = VF_BACK;
                    break;
                }
                // The facet of c opposite k and the facet of n opposite f: the same
                // three vertices (in any order).
                const int4 nvx = T.tv[n];
                for (int m = 0; m < 4 && !code; ++m) {
                    if (m == k) continue;
                    const int v = at(tv, m);
                    bool found = false;
                    for (int q = 0; q < 4; ++q) found = found || (q != f && at(nvx, q) == v);
                    if (!found) code = VF_FACET;
                }
            }
            if (!code && lock && lock[c] != 0) {
                code = VF_LOCK;
                detail = lock[c];
            }
        }
        where = c;
    } else if (i < int64_t(ntet) + nv) {
        const int v = int(i - ntet);
        const int c = T.vert_tet[v];
        if (c >= 0) {   // -1: not inserted yet
            if (c >= ntet || !T.alive[c]) code = VF_VERT_TET;
            else if (pos_of(T.tv[c], v) == 3 && T.tv[c].w != v) code = VF_VERT_TET;
            detail = c;
        }
        where = v;
    }
    if (code) {
        report(status, ST_INTERNAL);
        const unsigned long long rec = (unsigned long long)(uint32_t(code)) << 60 |
                                       (unsigned long long)(uint32_t(where) & 0x3FFFFFFFu) << 30 |
                                       (unsigned long long)(uint32_t(detail) & 0x3FFFFFFFu);
        atomicMin(fail, rec);
    }
}

/// Workers for the points the asynchronous pass left: one point each, its walk
/// starting from the nearest earlier inserted vertex of its set.
__global__ void k_setup_list(Workers W, const int* __restrict__ list, int n, const int32_t* __restrict__ vset,
                             const int32_t* __restrict__ voff, const int* __restrict__ vert_tet) {
    const int w = int(blockIdx.x) * blockDim.x + threadIdx.x;
    if (w >= n) return;
    const int v = list[w];
    const int set = vset[v];
    W.beg[w] = v;
    W.end[w] = v + 1;
    W.pos[w] = 0;
    W.left[w] = 1;
    W.nwon[w] = 0;
    W.parked[w] = 0;
    W.last[w] = -1;
    W.wset[w] = set;
    next_point(W, w);
    int g = W.skips[set].x;
    for (int u = v - 1, k = 0; u >= voff[set] && k < 4096; --u, ++k)
        if (__ldcg(vert_tet + u) >= 0) {
            g = u;
            break;
        }
    W.guide[w] = g;
    W.state[w] = WS_DONE;
}

/// Per set, the exponent span of its vertex coordinates (Span: lowest set bit,
/// just above the highest), reduced over runs of vertices of one set.
__global__ void k_set_span(const double* __restrict__ vx, int nv, const int32_t* __restrict__ vset,
                           int* __restrict__ smin, int* __restrict__ stop) {
    constexpr int kRun = 64;
    const int64_t first = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) * kRun;
    if (first >= nv) return;
    const int last = int(min(int64_t(nv), first + kRun));
    int set = vset[first];
    Span sp;
    for (int v = int(first); v <= last; ++v) {
        if (v == last || vset[v] != set) {
            if (!sp.empty()) {
                atomicMin(smin + set, sp.emin);
                atomicMax(stop + set, sp.top);
            }
            if (v == last) break;
            set = vset[v];
            sp = Span();
        }
        sp.add(vx[3 * int64_t(v)]);
        sp.add(vx[3 * int64_t(v) + 1]);
        sp.add(vx[3 * int64_t(v) + 2]);
    }
}

/// A set whose span makes the orient3d and in_sphere filters exact.
__global__ void k_set_exact(const int* __restrict__ smin, const int* __restrict__ stop, int nsets,
                            uint8_t* __restrict__ ex) {
    const int s = int(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= nsets) return;
    Span sp;
    sp.emin = smin[s];
    sp.top = stop[s];
    ex[s] = (sp.exact_in_double(5, 7) && sp.exact_in_double(3, 3)) ? 1 : 0;
}

/// Launches one insertion kernel (0: k_cavity, 1: k_check, 2: k_restar) over
/// `n` worker slots with G lanes per worker.
template <int G>
void launch_insertion_t(int which, const Tables& T, const Workers& W, const Round& R, const double* vx, int n,
                        cudaStream_t s) {
    const unsigned grid = unsigned((int64_t(n) * G + 127) / 128);
    if (which == 0) k_cavity<G><<<grid, 128, 0, s>>>(T, W, R, vx, 0);
    else if (which == 1) k_check<G><<<grid, 128, 0, s>>>(T, W, R, 0);
    else k_restar<G><<<grid, 128, 0, s>>>(T, W, R, 0);
}

void launch_insertion(int lanes, int which, const Tables& T, const Workers& W, const Round& R, const double* vx,
                      cudaStream_t s) {
    switch (lanes) {
        case 4: launch_insertion_t<4>(which, T, W, R, vx, W.n, s); break;
        case 8: launch_insertion_t<8>(which, T, W, R, vx, W.n, s); break;
        case 16: launch_insertion_t<16>(which, T, W, R, vx, W.n, s); break;
        default: launch_insertion_t<32>(which, T, W, R, vx, W.n, s); break;
    }
}


/// Lists the parked workers (for the big rounds).
__global__ void k_collect_parked(Workers W, int* list, int* count) {
    const int w = int(blockIdx.x) * blockDim.x + threadIdx.x;
    if (w >= W.n) return;
    if (W.parked[w] && W.cur[w] >= 0) list[atomicAdd(count, 1)] = w;
}

/// One set's share of a level: vertices [lb, le) (global ids) inserted by
/// workers [w0, w0 + count) with chunks of `chunk`; [plb, ple) is the set's
/// previous level.
struct LevelDesc {
    int set, lb, le, chunk, plb, ple, w0;
};

/// Workers of one level, one chunk each.  Each starts at a scattered offset
/// inside its chunk: chunks that are neighbours along the curve are mirror
/// images of each other, and workers walking them in step would reach their
/// common boundary together and keep colliding.
__global__ void k_setup_level(Workers W, const LevelDesc* __restrict__ ds, int nds) {
    const int w = int(blockIdx.x) * blockDim.x + threadIdx.x;
    if (w >= W.n) return;
    int lo = 0, hi = nds - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ds[mid].w0 <= w) lo = mid;
        else hi = mid - 1;
    }
    const LevelDesc d = ds[lo];
    const int lw = w - d.w0;
    const int b = d.lb + lw * d.chunk;
    const int e = min(d.le, b + d.chunk);
    const int len = e - b;
    const int off = len > 0 ? int((uint32_t(lw) * 2654435761u >> 7) % uint32_t(len)) : 0;
    W.beg[w] = b;
    W.end[w] = e;
    W.pos[w] = off;
    W.left[w] = len;
    W.nwon[w] = 0;
    W.parked[w] = 0;
    W.last[w] = -1;
    W.wset[w] = d.set;
    next_point(W, w);
    // The previous level is ordered along the same curve: the same fraction
    // along it lands near this worker's first point.
    int g = W.skips[d.set].x;
    if (d.ple > d.plb) {
        const double frac = (double(lw) * d.chunk + off) / double(d.le - d.lb);
        g = d.plb + int(frac * double(d.ple - d.plb));
        if (g >= d.ple) g = d.ple - 1;
    }
    W.guide[w] = g;
    W.state[w] = WS_DONE;
}

// ---- growing the worker pool within a level ------------------------------------------
//
// A level's workers are sized for the points its set had when the level began;
// by its end the set has 8 times as many.  Once a set's inserted points call
// for twice its current workers, every worker of that set with enough of its
// chunk left hands the second half of what remains to a new worker.

struct SplitState {
    int* set_p0;     // per set: points inserted before the level
    int* set_ins;    // per set: points inserted so far in the level
    int* set_w;      // per set: current workers
    int* set_split;  // per set: split this time
    int* nworkers;   // the pool size (device copy of W.n)
    int cap;         // worker slots allocated
};

__global__ void k_count_wins(Workers W, SplitState S) {
    const int w = int(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool ok = w < W.n;
    const int set = ok ? W.wset[w] : -1;
    const int c = ok ? W.nwon[w] : 0;
    // Lanes of one set add once per warp.
    const unsigned m = __match_any_sync(__activemask(), set);
    const int sum = int(__reduce_add_sync(m, unsigned(c)));
    if (ok && (threadIdx.x & 31) == __ffs(int(m)) - 1 && sum) atomicAdd(S.set_ins + set, sum);
}

__global__ void k_plan_split(SplitState S, int nsets, double alpha) {
    for (int s = int(blockIdx.x) * blockDim.x + threadIdx.x; s < nsets; s += gridDim.x * blockDim.x) {
        const double p = double(S.set_p0[s]) + double(S.set_ins[s]);
        S.set_split[s] = (S.set_w[s] > 0 && p / alpha >= 2.0 * S.set_w[s]) ? 1 : 0;
        S.set_ins[s] = 0;
    }
}

__global__ void k_split(Workers W, SplitState S, int n_before) {
    const int w = int(blockIdx.x) * blockDim.x + threadIdx.x;
    if (w >= n_before) return;
    const int set = W.wset[w];
    if (!S.set_split[set] || W.cur[w] < 0 || W.parked[w] || W.left[w] < 2 * 16) return;
    const int slot = atomicAdd(S.nworkers, 1);
    if (slot >= S.cap) return;
    const int len = W.end[w] - W.beg[w];
    const int left = W.left[w];
    const int give = left - left / 2;
    W.beg[slot] = W.beg[w];
    W.end[slot] = W.end[w];
    W.pos[slot] = (W.pos[w] + left / 2) % len;
    W.left[slot] = give;
    W.left[w] = left / 2;
    W.nwon[slot] = 0;
    W.parked[slot] = 0;
    W.last[slot] = W.last[w];
    W.guide[slot] = W.guide[w];
    W.wset[slot] = set;
    W.state[slot] = WS_DONE;
    next_point(W, slot);
    atomicAdd(S.set_w + set, 1);
}

// ---- set-up: validation, duplicates, initial tet ----------------------------------

__global__ void k_check_finite(const double* __restrict__ xyz, int64_t n3, uint32_t* bad) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n3;
         i += int64_t(gridDim.x) * blockDim.x)
        if (!isfinite(xyz[i])) atomicOr(bad, 1u);
}

/// The set holding position g: off[s] <= g < off[s+1].
__device__ __forceinline__ int set_of(const int64_t* __restrict__ off, int nsets, int64_t g) {
    int lo = 0, hi = nsets - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

/// Per set, the exponent span of its input coordinates, before any ordering
/// (as k_set_span; duplicates do not change it).
__global__ void k_raw_span(const double* __restrict__ xyz, const int64_t* __restrict__ off, int nsets, int64_t n,
                           int* __restrict__ smin, int* __restrict__ stop) {
    constexpr int kRun = 64;
    const int64_t first = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) * kRun;
    if (first >= n) return;
    const int64_t last = min(n, first + kRun);
    int set = set_of(off, nsets, first);
    Span sp;
    for (int64_t p = first; p <= last; ++p) {
        if (p == last || p >= off[set + 1]) {
            if (!sp.empty()) {
                atomicMin(smin + set, sp.emin);
                atomicMax(stop + set, sp.top);
            }
            if (p == last) break;
            while (p >= off[set + 1]) ++set;
            sp = Span();
        }
        sp.add(xyz[3 * p]);
        sp.add(xyz[3 * p + 1]);
        sp.add(xyz[3 * p + 2]);
    }
}

/// Global index of the input point at rank r (position r of its set's order).
__device__ __forceinline__ int64_t point_at(const int32_t* __restrict__ order, const int64_t* __restrict__ off,
                                            int nsets, int64_t r) {
    return off[set_of(off, nsets, r)] + order[r];
}

/// Coordinate bit patterns (with -0.0 folded onto +0.0, which compare equal)
/// of the point at each rank, for the duplicate grouping; axis 3 = the set.
__global__ void k_coord_keys(const double* __restrict__ xyz, const int32_t* __restrict__ order,
                             const int64_t* __restrict__ off, int nsets, int64_t n, int axis,
                             unsigned long long* __restrict__ keys, const int32_t* __restrict__ ranks) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        if (axis == 3) {
            keys[i] = (unsigned long long)set_of(off, nsets, ranks[i]);
            continue;
        }
        const double x = xyz[3 * point_at(order, off, nsets, ranks[i]) + axis];
        keys[i] = x == 0.0 ? 0ull : (unsigned long long)__double_as_longlong(x);
    }
}

__device__ __forceinline__ bool same_point(const double* xyz, int64_t i, int64_t j) {
    const double* a = xyz + 3 * i;
    const double* b = xyz + 3 * j;
    return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
}

/// Over ranks sorted by (set, coordinates), ties by rank: flags the first rank
/// of each group of equal points of one set and records the group's
/// representative, the point with the LAST rank (src/triangulation.cpp:77-81),
/// as an index local to its set.
__global__ void k_groups(const double* __restrict__ xyz, const int32_t* __restrict__ order,
                         const int64_t* __restrict__ off, int nsets, const int32_t* __restrict__ sranks,
                         int64_t n, int32_t* __restrict__ first, int32_t* __restrict__ rep_at_first,
                         int* ndup) {
    for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < n;
         s += int64_t(gridDim.x) * blockDim.x) {
        const int32_t r = sranks[s];
        const int set = set_of(off, nsets, r);
        const int64_t pr = off[set] + order[r];
        auto same = [&](int64_t t) {
            const int32_t rt = sranks[t];
            const int st = set_of(off, nsets, rt);
            return st == set && same_point(xyz, off[st] + order[rt], pr);
        };
        if (s > 0 && same(s - 1)) {
            first[r] = 0;
            atomicAdd(ndup, 1);
            continue;
        }
        int64_t e = s;
        while (e + 1 < n && same(e + 1)) ++e;
        first[r] = 1;
        rep_at_first[r] = order[sranks[e]];
    }
}

/// Vertex records: coordinates, the input index (local to the set) the vertex
/// stands for, and its set.
__global__ void k_vertices(const double* __restrict__ xyz, const int32_t* __restrict__ order,
                           const int64_t* __restrict__ off, int nsets,
                           const int32_t* __restrict__ first, const int32_t* __restrict__ vid_of_rank,
                           const int32_t* __restrict__ rep_at_first, int64_t n, bool dups,
                           double* __restrict__ vx, int32_t* __restrict__ vert_point,
                           int32_t* __restrict__ vset) {
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
         r += int64_t(gridDim.x) * blockDim.x) {
        if (dups && !first[r]) continue;
        const int32_t v = dups ? vid_of_rank[r] : int32_t(r);
        const int set = set_of(off, nsets, r);
        const int64_t i = off[set] + order[r];
        vx[3 * int64_t(v)] = xyz[3 * i];
        vx[3 * int64_t(v) + 1] = xyz[3 * i + 1];
        vx[3 * int64_t(v) + 2] = xyz[3 * i + 2];
        vert_point[v] = dups ? rep_at_first[r] : order[r];
        vset[v] = set;
    }
}

/// Per set: the first vertex (in insertion order) not collinear with its first
/// two, and then the first not coplanar with those three.
__global__ void k_find_noncollinear(const double* __restrict__ vx, int nv, const int32_t* __restrict__ vset,
                                    const int32_t* __restrict__ voff, int* found, uint32_t* st) {
    for (int v = int(blockIdx.x) * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const int set = vset[v], base = voff[set];
        if (v - base < 2 || v > found[set]) continue;
        if (!collinear(vpt(vx, base), vpt(vx, base + 1), vpt(vx, v), st)) atomicMin(found + set, v);
    }
}

__global__ void k_find_noncoplanar(const double* __restrict__ vx, int nv, const int32_t* __restrict__ vset,
                                   const int32_t* __restrict__ voff, const int* found2, int* found3,
                                   uint32_t* st) {
    for (int v = int(blockIdx.x) * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const int set = vset[v], base = voff[set], v2 = found2[set];
        if (v2 >= voff[set + 1] || v - base < 2 || v == v2 || v > found3[set]) continue;
        if (orient3d(vpt(vx, base), vpt(vx, base + 1), vpt(vx, v2), vpt(vx, v), st) != 0)
            atomicMin(found3 + set, v);
    }
}

/// Per set: its first four vertices (or -1s when the set is flat: no cells,
/// src/triangulation.cpp:943-949).
__global__ void k_set_skips(const int32_t* __restrict__ voff, const int* found2, const int* found3,
                            int nsets, int4* __restrict__ skips) {
    for (int s = int(blockIdx.x) * blockDim.x + threadIdx.x; s < nsets; s += gridDim.x * blockDim.x) {
        const int base = voff[s], end = voff[s + 1];
        if (end - base >= 4 && found2[s] < end && found3[s] < end)
            skips[s] = make_int4(base, base + 1, found2[s], found3[s]);
        else
            skips[s] = make_int4(-1, -1, -1, -1);
    }
}

/// One thread per set: the first tet and its four infinite neighbours, in
/// slots 5s .. 5s+4.
__global__ void k_init_tets(Tables T, const double* __restrict__ vx, const int4* __restrict__ skips,
                            int nsets, uint32_t* st) {
    for (int set = int(blockIdx.x) * blockDim.x + threadIdx.x; set < nsets; set += gridDim.x * blockDim.x) {
        const int4 sk = skips[set];
        if (sk.x < 0) continue;
        int v0 = sk.x, v1 = sk.y;
        const int v2 = sk.z, v3 = sk.w;
        if (orient3d(vpt(vx, v0), vpt(vx, v1), vpt(vx, v2), vpt(vx, v3), st) < 0) {
            const int t = v0;
            v0 = v1;
            v1 = t;
        }
        int4 tv[5];
        tv[0] = make_int4(v0, v1, v2, v3);
        for (int i = 0; i < 4; ++i) {
            // Facet i of the first tet, capped by the infinite vertex in slot i
            // and two other slots swapped, so the cap is positively oriented.
            int4 c = tv[0];
            set_at(c, i, kInf);
            const int a = (i + 1) & 3, b = (i + 2) & 3;
            const int x = at(c, a);
            set_at(c, a, at(c, b));
            set_at(c, b, x);
            tv[1 + i] = c;
        }
        const int base = 5 * set;
        int4 tn[5];
        for (int t = 0; t < 5; ++t)
            for (int f = 0; f < 4; ++f) {
                int fv[3], w = 0;
                for (int m = 0; m < 4; ++m)
                    if (m != f) fv[w++] = at(tv[t], m);
                for (int u = 0; u < 5; ++u) {
                    if (u == t) continue;
                    for (int g = 0; g < 4; ++g) {
                        int hits = 0;
                        for (int m = 0; m < 4; ++m) {
                            if (m == g) continue;
                            const int x = at(tv[u], m);
                            hits += (x == fv[0]) + (x == fv[1]) + (x == fv[2]);
                        }
                        if (hits == 3) set_at(tn[t], f, (base + u) * 4 + g);
                    }
                }
            }
        for (int t = 0; t < 5; ++t) {
            T.tv[base + t] = tv[t];
            T.tn[base + t] = tn[t];
            T.alive[base + t] = 1;
        }
        T.vert_tet[v0] = base;
        T.vert_tet[v1] = base;
        T.vert_tet[v2] = base;
        T.vert_tet[v3] = base;
    }
}

// ---- output -----------------------------------------------------------------------

/// Even permutation bringing the smallest index to slot 0, then the cyclic
/// rotation of the other three that puts their smallest first.
__device__ __forceinline__ int4 canonical(int4 t) {
    int m = 0;
    int mv = t.x;
    if (t.y < mv) { m = 1; mv = t.y; }
    if (t.z < mv) { m = 2; mv = t.z; }
    if (t.w < mv) { m = 3; mv = t.w; }
    if (m == 1) t = make_int4(t.y, t.x, t.w, t.z);
    else if (m == 2) t = make_int4(t.z, t.w, t.x, t.y);
    else if (m == 3) t = make_int4(t.w, t.z, t.y, t.x);
    if (t.z < t.y && t.z < t.w) t = make_int4(t.x, t.z, t.w, t.y);
    else if (t.w < t.y && t.w < t.z) t = make_int4(t.x, t.w, t.y, t.z);
    return t;
}

__global__ void k_cell_flags(const int4* __restrict__ tv, const uint8_t* __restrict__ alive, int ntet,
                             bool with_infinite, int32_t* __restrict__ flag) {
    for (int t = int(blockIdx.x) * blockDim.x + threadIdx.x; t < ntet; t += gridDim.x * blockDim.x) {
        const int4 c = tv[t];
        flag[t] = alive[t] && (with_infinite || inf_pos(c) < 0) ? 1 : 0;
    }
}

/// Writes the flagged tets, mapped to input point indices and canonicalised,
/// plus (khi given) their sort keys (shifted by one so the infinite vertex, -1,
/// is 0).
__global__ void k_cells_out(const int4* __restrict__ tv, const int32_t* __restrict__ flag,
                            const int32_t* __restrict__ pos, int ntet,
                            const int32_t* __restrict__ vert_point, const int32_t* __restrict__ vset,
                            int kbits, int4* __restrict__ cells,
                            unsigned long long* __restrict__ khi, unsigned long long* __restrict__ klo,
                            int32_t* __restrict__ idx, int32_t* __restrict__ cset) {
    for (int t = int(blockIdx.x) * blockDim.x + threadIdx.x; t < ntet; t += gridDim.x * blockDim.x) {
        if (!flag[t]) continue;
        const int4 c = tv[t];
        if (cset) cset[pos[t]] = vset[c.x != kInf ? c.x : c.y];
        int4 q;
        q.x = c.x == kInf ? -1 : vert_point[c.x];
        q.y = c.y == kInf ? -1 : vert_point[c.y];
        q.z = c.z == kInf ? -1 : vert_point[c.z];
        q.w = c.w == kInf ? -1 : vert_point[c.w];
        q = canonical(q);
        const int o = pos[t];
        cells[o] = q;
        if (khi) {
            khi[o] = ((unsigned long long)(uint32_t(q.x + 1)) << kbits) | uint32_t(q.y + 1);
            klo[o] = ((unsigned long long)(uint32_t(q.z + 1)) << kbits) | uint32_t(q.w + 1);
            idx[o] = o;
        }
    }
}

// ---- canonical order of the finite cells by buckets ---------------------------------
//
// A canonical cell leads with its smallest vertex, so the lexicographic order
// is: by that vertex, then by the other three.  The cells are bucketed by the
// global index of their first vertex (set offset + local index; the sets are
// contiguous, so this also orders them by set) with a counting sort, then each
// bucket - the few cells whose smallest vertex is that point - is sorted by its
// other three vertices.

/// One thread sorts a bucket of up to kBucketThread cells, one block one of up
/// to kBucketBlock; a larger bucket leaves the whole output to the radix sort.
constexpr int kBucketThread = 32;
constexpr int kBucketBlock = 2048;

__device__ __forceinline__ int cell_bucket(const int4& q, const int32_t* __restrict__ cset,
                                           const int64_t* __restrict__ off, int64_t o) {
    return int(cset ? off[cset[o]] : 0) + q.x;
}

__global__ void k_bucket_count(const int4* __restrict__ cells, const int32_t* __restrict__ cset,
                               const int64_t* __restrict__ off, int64_t n, int* __restrict__ count) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        atomicAdd(count + cell_bucket(cells[i], cset, off, i), 1);
}

__global__ void k_bucket_place(const int4* __restrict__ cells, const int32_t* __restrict__ cset,
                               const int64_t* __restrict__ off, int64_t n, const int* __restrict__ start,
                               int* __restrict__ fill, int4* __restrict__ out) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const int4 q = cells[i];
        const int b = cell_bucket(q, cset, off, i);
        out[start[b] + atomicAdd(fill + b, 1)] = q;
    }
}

__device__ __forceinline__ bool cell_tail_less(const int4& a, const int4& b) {
    if (a.y != b.y) return a.y < b.y;
    if (a.z != b.z) return a.z < b.z;
    return a.w < b.w;
}

/// One thread per bucket: insertion sort by the last three vertices.  A
/// bucket of more than kBucketThread cells is listed in `mid` for
/// k_bucket_sort_block, one of more than kBucketBlock only raises `big`.
__global__ void k_bucket_sort(int4* __restrict__ cells, const int* __restrict__ start, int nb,
                              int* __restrict__ mid, int* __restrict__ nmid, int* __restrict__ big) {
    for (int b = int(blockIdx.x) * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int lo = start[b], hi = start[b + 1];
        if (hi - lo > kBucketBlock) {
            *big = 1;
            continue;
        }
        if (hi - lo > kBucketThread) {
            mid[atomicAdd(nmid, 1)] = b;
            continue;
        }
        for (int i = lo + 1; i < hi; ++i) {
            const int4 x = cells[i];
            int j = i - 1;
            while (j >= lo && cell_tail_less(x, cells[j])) {
                cells[j + 1] = cells[j];
                --j;
            }
            cells[j + 1] = x;
        }
    }
}

/// One block per listed bucket: a bitonic sort by the last three vertices in
/// shared memory (padded to a power of two with cells that sort last).
__global__ void __launch_bounds__(512) k_bucket_sort_block(int4* __restrict__ cells, const int* __restrict__ start,
                                                           const int* __restrict__ mid) {
    __shared__ int4 sh[kBucketBlock];
    const int b = mid[blockIdx.x];
    const int lo = start[b], n = start[b + 1] - lo;
    int m = 1;
    while (m < n) m <<= 1;
    const int4 pad = make_int4(INT_MAX, INT_MAX, INT_MAX, INT_MAX);
    for (int i = int(threadIdx.x); i < m; i += blockDim.x) sh[i] = i < n ? cells[lo + i] : pad;
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = int(threadIdx.x); i < m; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const int4 a = sh[i], c = sh[l];
                    if (cell_tail_less(c, a) == up) {
                        sh[i] = c;
                        sh[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = int(threadIdx.x); i < n; i += blockDim.x) cells[lo + i] = sh[i];
}

/// cell_off[s] = the first bucket of set s.
__global__ void k_cell_off(const int* __restrict__ start, const int64_t* __restrict__ off, int nsets,
                           int64_t* __restrict__ cell_off) {
    for (int s = int(blockIdx.x) * blockDim.x + threadIdx.x; s <= nsets; s += gridDim.x * blockDim.x)
        cell_off[s] = start[off[s]];
}

__global__ void k_gather_cells(const int4* __restrict__ in, const int32_t* __restrict__ idx, int64_t n,
                               int4* __restrict__ out) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        out[i] = in[idx[i]];
}

__global__ void k_incident_pairs(const int4* __restrict__ cells, int64_t nc, int32_t* __restrict__ pt,
                                 int32_t* __restrict__ cell, int32_t* __restrict__ count) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nc;
         i += int64_t(gridDim.x) * blockDim.x) {
        const int4 c = cells[i];
        const int v[4] = {c.x, c.y, c.z, c.w};
        for (int k = 0; k < 4; ++k) {
            pt[4 * i + k] = v[k];
            cell[4 * i + k] = int32_t(i);
            atomicAdd(count + v[k], 1);
        }
    }
}

__global__ void k_set_int(int* p, int v) { *p = v; }

__global__ void k_gather_u64(const unsigned long long* __restrict__ in, const int32_t* __restrict__ ix,
                             int64_t m, unsigned long long* __restrict__ o) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += int64_t(gridDim.x) * blockDim.x)
        o[i] = in[ix[i]];
}

__global__ void k_gather_i32(const int32_t* __restrict__ in, const int32_t* __restrict__ ix, int64_t m,
                             int32_t* __restrict__ o) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += int64_t(gridDim.x) * blockDim.x)
        o[i] = in[ix[i]];
}

__global__ void k_iota32(int32_t* __restrict__ a, int64_t m) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += int64_t(gridDim.x) * blockDim.x)
        a[i] = int32_t(i);
}

__global__ void k_widen(const int32_t* __restrict__ a, int64_t m, int64_t* __restrict__ o) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += int64_t(gridDim.x) * blockDim.x)
        o[i] = a[i];
}

}  // namespace

namespace {

__global__ void k_voff(const int64_t* __restrict__ off, int nsets, const int32_t* __restrict__ vid, bool dups,
                       int64_t n, int nv, int32_t* __restrict__ voff) {
    for (int s = int(blockIdx.x) * blockDim.x + threadIdx.x; s <= nsets; s += gridDim.x * blockDim.x) {
        const int64_t o = off[s];
        voff[s] = o >= n ? nv : (dups ? vid[o] : int32_t(o));
    }
}

/// Sorts `n` canonical cells lexicographically - by set first when `cset` is
/// given - into `out` (keys prepared by k_cells_out).
int sort_cells(DevBuf<int4>& cells, DevBuf<unsigned long long>& khi, DevBuf<unsigned long long>& klo,
               DevBuf<int32_t>& idx, const int32_t* cset, int nsets, int64_t n, int kbits,
               DevBuf<int4>& out, cudaStream_t s) {
    D3G_TRY(out.alloc(size_t(n), s));
    if (n == 0) return D3G_OK;
    DevBuf<unsigned long long> k2, kg;
    DevBuf<int32_t> i2;
    D3G_TRY(k2.alloc(size_t(n), s));
    D3G_TRY(kg.alloc(size_t(n), s));
    D3G_TRY(i2.alloc(size_t(n), s));
    // LSD: low half, then the high half, then (several sets) the set - each stable.
    D3G_TRY(sort_pairs(klo.p, k2.p, idx.p, i2.p, n, 0, 2 * kbits, s));
    k_gather_u64<<<grid_for(n, 256), 256, 0, s>>>(khi.p, i2.p, n, kg.p);
    D3G_TRY(sort_pairs(kg.p, k2.p, i2.p, idx.p, n, 0, 2 * kbits, s));
    if (cset) {
        DevBuf<int32_t> sk, sk2;
        D3G_TRY(sk.alloc(size_t(n), s));
        D3G_TRY(sk2.alloc(size_t(n), s));
        k_gather_i32<<<grid_for(n, 256), 256, 0, s>>>(cset, idx.p, n, sk.p);
        D3G_TRY(sort_pairs(sk.p, sk2.p, idx.p, i2.p, n, 0, bits_for(uint64_t(nsets)), s));
        idx.swap(i2);
    }
    k_gather_cells<<<grid_for(n, 256), 256, 0, s>>>(cells.p, idx.p, n, out.p);
    D3G_CUDA(cudaGetLastError());
    return D3G_OK;
}

}  // namespace

int build_sets_impl(const double* d_xyz, const int64_t* h_off, int nsets, const d3g_options& opt,
                    cudaStream_t s, DeviceResult& R);

/// A non-blocking stream of the calling thread for the current device; it lives
/// as long as the thread, so buffers bound to it can be freed at any later time.
cudaStream_t internal_stream() {
    thread_local cudaStream_t streams[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    if (!streams[dev] && cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking) != cudaSuccess)
        streams[dev] = nullptr;
    return streams[dev];
}

/// Runs the build on `s`, or - for the legacy default stream, which cannot be
/// captured into a graph - on the thread's internal stream, after the legacy
/// stream's prior work (the build synchronises its stream before returning).
int build_on_stream(const double* d_xyz, const int64_t* h_off, int nsets, const d3g_options& opt,
                    cudaStream_t s, DeviceResult& R) {
    D3G_TRY(prepare_device());
    if (s != nullptr && s != cudaStreamLegacy) return build_sets_impl(d_xyz, h_off, nsets, opt, s, R);
    cudaStream_t own = internal_stream();
    if (!own) {
        set_error("d3g_build: could not create a stream");
        return D3G_ERR_CUDA;
    }
    cudaEvent_t ev;
    D3G_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaEventRecord(ev, cudaStreamLegacy);
    cudaStreamWaitEvent(own, ev, 0);
    cudaEventDestroy(ev);
    return build_sets_impl(d_xyz, h_off, nsets, opt, own, R);
}

int build_on_stream(const double* d_xyz, int64_t n, const d3g_options& opt, cudaStream_t s,
                    DeviceResult& R) {
    const int64_t h_off[2] = {0, n};
    return build_on_stream(d_xyz, h_off, 1, opt, s, R);
}

int build_sets_impl(const double* d_xyz, const int64_t* h_off, int nsets, const d3g_options& opt,
                    cudaStream_t s, DeviceResult& R) {
    R.reset();
    const int64_t n = h_off[nsets];
    int64_t max_n = 0;
    for (int i = 0; i < nsets; ++i) {
        if (h_off[i + 1] < h_off[i]) {
            set_error("d3g_build: set offsets must not decrease");
            return D3G_ERR_INVALID_ARGUMENT;
        }
        max_n = std::max<int64_t>(max_n, h_off[i + 1] - h_off[i]);
    }
    R.cell_off.assign(size_t(nsets) + 1, 0);
    R.set_nv.assign(size_t(nsets), 0);
    if (n == 0) return D3G_OK;
    if (n > (int64_t(1) << 27) || h_off[0] != 0) {
        set_error("d3g_build: at most 2^27 points per call, offsets starting at 0");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    if (opt.level_growth != 0 && (opt.level_growth < 2 || opt.level_growth > 8)) {
        set_error("d3g_build: level_growth must be 0 or 2-8");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    const bool single = nsets == 1;
    const int N = int(n);
    DevBuf<uint32_t> status;
    DevBuf<int64_t> d_off;
    D3G_TRY(status.alloc(4, s));
    D3G_TRY(d_off.alloc(size_t(nsets) + 1, s));
    D3G_CUDA(cudaMemsetAsync(status.p, 0, 4 * sizeof(uint32_t), s));
    D3G_CUDA(cudaMemcpyAsync(d_off.p, h_off, sizeof(int64_t) * (size_t(nsets) + 1), cudaMemcpyHostToDevice, s));
    k_check_finite<<<grid_for(3 * n, 256), 256, 0, s>>>(d_xyz, 3 * n, status.p + 1);

    cudaEvent_t ph[4];
    for (auto& e : ph) cudaEventCreate(&e);
    struct PhGuard {
        cudaEvent_t* e;
        ~PhGuard() {
            for (int i = 0; i < 4; ++i) cudaEventDestroy(e[i]);
        }
    } ph_guard{ph};
    cudaEventRecord(ph[0], s);
    NvtxRange nvtx_build("d3g.build");
    std::optional<NvtxRange> nvtx_phase;
    nvtx_phase.emplace("d3g.order");
    // ---- insertion order and duplicate groups ----
    // BRIO levels of the build's own insertion order: each level `growth` times
    // the points before it.  Any order gives the same cells, so the build may
    // take more and shorter levels than the reference's 8, as it does by default
    // when a set's coordinates make the filters exact (lattices and coarse grids,
    // whose long levels collide most) and for a build too small to fill the GPU
    // (whose levels are inserted chunk by chunk, so shorter ones finish sooner).  The one thing the reference's order
    // decides is which copy of a repeated point keeps its index (the last one in
    // that order), so input with repeated points is ordered again by it.
    int growth = opt.level_growth;
    if (growth == 0) {
        DevBuf<int> span;
        DevBuf<uint8_t> ex;
        D3G_TRY(span.alloc(size_t(2) * size_t(nsets), s));
        D3G_TRY(ex.alloc(size_t(nsets), s));
        std::vector<int> init(size_t(2) * size_t(nsets));
        for (int i = 0; i < nsets; ++i) {
            init[size_t(i)] = 1 << 20;
            init[size_t(nsets) + size_t(i)] = -(1 << 20);
        }
        D3G_CUDA(cudaMemcpyAsync(span.p, init.data(), sizeof(int) * init.size(), cudaMemcpyHostToDevice, s));
        k_raw_span<<<grid_for((n + 63) / 64, 128, 1 << 30), 128, 0, s>>>(d_xyz, d_off.p, nsets, n, span.p,
                                                                         span.p + nsets);
        k_set_exact<<<grid_for(nsets, 128), 128, 0, s>>>(span.p, span.p + nsets, nsets, ex.p);
        std::vector<uint8_t> hex(static_cast<size_t>(nsets));
        D3G_CUDA(cudaMemcpyAsync(hex.data(), ex.p, size_t(nsets), cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaStreamSynchronize(s));   // `init` must outlive the copy
        growth = n < kSmallBuildPoints ? kExactSetGrowth : 8;
        for (const uint8_t e : hex) growth = e ? kExactSetGrowth : growth;
    }
    DevBuf<int32_t> order;
    D3G_TRY(order.alloc(size_t(N), s));

    DevBuf<double> vx;
    DevBuf<int32_t> vert_point, vset, voff;
    int nv = N;
    D3G_TRY(voff.alloc(size_t(nsets) + 1, s));
    for (;;) {
        D3G_TRY(spatial_order_sets_device(d_xyz, h_off, d_off.p, nsets, order.p, s, 1.0 / double(growth)));
        DevBuf<int32_t> ranks, sranks, first, rep, vid;
        DevBuf<unsigned long long> keys, keys2;
        DevBuf<int> ndup;
        D3G_TRY(ranks.alloc(size_t(N), s));
        D3G_TRY(sranks.alloc(size_t(N), s));
        D3G_TRY(keys.alloc(size_t(N), s));
        D3G_TRY(keys2.alloc(size_t(N), s));
        D3G_TRY(ndup.alloc(1, s));
        D3G_CUDA(cudaMemsetAsync(ndup.p, 0, sizeof(int), s));
        k_iota32<<<grid_for(n, 256), 256, 0, s>>>(ranks.p, n);
        // LSD over z, y, x (and the set): ranks sorted by (set, coordinates),
        // ties kept in rank order.
        for (int axis = 2; axis >= (single ? 0 : -1); --axis) {
            const int key_axis = axis < 0 ? 3 : axis;
            k_coord_keys<<<grid_for(n, 256), 256, 0, s>>>(d_xyz, order.p, d_off.p, nsets, n, key_axis, keys.p,
                                                          ranks.p);
            D3G_TRY(sort_pairs(keys.p, keys2.p, ranks.p, sranks.p, n, 0,
                               key_axis == 3 ? bits_for(uint64_t(nsets)) : 64, s));
            ranks.swap(sranks);
        }
        D3G_TRY(first.alloc(size_t(N), s));
        D3G_TRY(rep.alloc(size_t(N), s));
        k_groups<<<grid_for(n, 256), 256, 0, s>>>(d_xyz, order.p, d_off.p, nsets, ranks.p, n, first.p, rep.p,
                                                  ndup.p);
        int hdup = 0;
        D3G_CUDA(cudaMemcpyAsync(&hdup, ndup.p, sizeof hdup, cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaStreamSynchronize(s));
        if (hdup > 0 && growth != 8) {
            growth = 8;
            continue;
        }
        nv = N - hdup;
        D3G_TRY(vx.alloc(size_t(3) * nv, s));
        D3G_TRY(vert_point.alloc(size_t(nv), s));
        D3G_TRY(vset.alloc(size_t(nv), s));
        if (hdup > 0) {
            D3G_TRY(vid.alloc(size_t(N), s));
            D3G_TRY(exclusive_scan(first.p, vid.p, n, s));
        }
        k_vertices<<<grid_for(n, 256), 256, 0, s>>>(d_xyz, order.p, d_off.p, nsets, first.p, vid.p, rep.p, n,
                                                    hdup > 0, vx.p, vert_point.p, vset.p);
        k_voff<<<grid_for(nsets + 1, 128), 128, 0, s>>>(d_off.p, nsets, vid.p, hdup > 0, n, nv, voff.p);
        D3G_CUDA(cudaGetLastError());
        break;
    }
    const double level_ratio = 1.0 / double(growth);
    order.release();
    R.n_vertices = nv;
    std::vector<int32_t> hvoff(size_t(nsets) + 1);
    D3G_CUDA(cudaMemcpyAsync(hvoff.data(), voff.p, sizeof(int32_t) * hvoff.size(), cudaMemcpyDeviceToHost, s));

    uint32_t hst[2] = {0, 0};
    D3G_CUDA(cudaMemcpyAsync(hst, status.p, sizeof hst, cudaMemcpyDeviceToHost, s));
    D3G_CUDA(cudaStreamSynchronize(s));
    if (hst[1]) {
        set_error("d3g_build: non-finite coordinate");
        return D3G_ERR_INVALID_INPUT;
    }
    for (int i = 0; i < nsets; ++i) R.set_nv[size_t(i)] = hvoff[size_t(i) + 1] - hvoff[size_t(i)];

    cudaEventRecord(ph[1], s);
    nvtx_phase.reset();
    nvtx_phase.emplace("d3g.insert");
    // ---- each set's first tet: its first four affinely independent vertices ----
    DevBuf<int> found;
    DevBuf<int4> skips;
    D3G_TRY(found.alloc(2 * size_t(nsets), s));
    D3G_TRY(skips.alloc(size_t(nsets), s));
    D3G_CUDA(cudaMemsetAsync(found.p, 0x7F, 2 * sizeof(int) * size_t(nsets), s));
    k_find_noncollinear<<<grid_for(nv, 256), 256, 0, s>>>(vx.p, nv, vset.p, voff.p, found.p, status.p);
    k_find_noncoplanar<<<grid_for(nv, 256), 256, 0, s>>>(vx.p, nv, vset.p, voff.p, found.p, found.p + nsets,
                                                         status.p);
    k_set_skips<<<grid_for(nsets, 128), 128, 0, s>>>(voff.p, found.p, found.p + nsets, nsets, skips.p);
    std::vector<int4> hskips(static_cast<size_t>(nsets));
    D3G_CUDA(cudaMemcpyAsync(hskips.data(), skips.p, sizeof(int4) * size_t(nsets), cudaMemcpyDeviceToHost, s));
    D3G_CUDA(cudaMemcpyAsync(hst, status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    D3G_CUDA(cudaStreamSynchronize(s));
    {
        const int st = status_from_bits(hst[0]);
        if (st != D3G_OK) return st;
    }
    bool any_cells = false;
    for (const int4& k : hskips) any_cells = any_cells || k.x >= 0;
    if (!any_cells) {
        // Every set collinear or coplanar: no cells (src/triangulation.cpp:943-949).
        if (single && opt.want_incident) {
            D3G_TRY(R.inc_off.alloc(size_t(N) + 1, s));
            D3G_CUDA(cudaMemsetAsync(R.inc_off.p, 0, sizeof(int64_t) * (size_t(N) + 1), s));
        }
        D3G_CUDA(cudaStreamSynchronize(s));
        return D3G_OK;
    }

    // ---- tables ----
    Tables T;
    const int tets_per_vertex = opt.tet_capacity > 0 ? opt.tet_capacity : 8;
    int64_t cap64 = int64_t(nv) * tets_per_vertex + 5 * int64_t(nsets) + 4096;
    if (cap64 > (int64_t(1) << 29)) cap64 = int64_t(1) << 29;
    T.cap = int(cap64);
    T.walk_limit = opt.walk_limit > 0 ? opt.walk_limit : kWalkLimit;
    DevBuf<int4> tv, tn;
    DevBuf<unsigned long long> claim;
    DevBuf<uint8_t> alive;
    DevBuf<int> fnew, vert_tet, tet_count;
    D3G_TRY(tv.alloc(size_t(T.cap), s));
    D3G_TRY(tn.alloc(size_t(T.cap), s));
    D3G_TRY(claim.alloc(size_t(T.cap), s));
    D3G_TRY(alive.alloc(size_t(T.cap), s));
    D3G_TRY(fnew.alloc(size_t(T.cap) * 4, s));
    D3G_TRY(vert_tet.alloc(size_t(nv), s));
    D3G_TRY(tet_count.alloc(1, s));
    D3G_CUDA(cudaMemsetAsync(claim.p, 0xFF, sizeof(unsigned long long) * size_t(T.cap), s));
    D3G_CUDA(cudaMemsetAsync(alive.p, 0, size_t(T.cap), s));
    // Every slot holds in-range indices from the start (the asynchronous walk
    // may read a slot before its tet is written), and a vertex not inserted yet
    // has no tet.
    D3G_CUDA(cudaMemsetAsync(tv.p, 0, sizeof(int4) * size_t(T.cap), s));
    D3G_CUDA(cudaMemsetAsync(tn.p, 0, sizeof(int4) * size_t(T.cap), s));
    D3G_CUDA(cudaMemsetAsync(vert_tet.p, 0xFF, sizeof(int) * size_t(nv), s));
    T.tv = tv.p;
    T.tn = tn.p;
    T.claim = claim.p;
    T.alive = alive.p;
    T.fnew = fnew.p;
    T.vert_tet = vert_tet.p;
    T.tet_count = tet_count.p;
    T.vset = vset.p;
    k_set_int<<<1, 1, 0, s>>>(tet_count.p, 5 * nsets);
    k_init_tets<<<grid_for(nsets, 64), 64, 0, s>>>(T, vx.p, skips.p, nsets, status.p);
    // Sets whose coordinates span few bits (integer lattices, coarse grids):
    // their filters are exact, so their degenerate queries skip the exact stage.
    DevBuf<int> set_span;
    DevBuf<uint8_t> set_exact;
    D3G_TRY(set_span.alloc(size_t(2) * size_t(nsets), s));
    D3G_TRY(set_exact.alloc(size_t(nsets), s));
    {
        std::vector<int> init(size_t(2) * size_t(nsets));
        for (int i = 0; i < nsets; ++i) {
            init[size_t(i)] = 1 << 20;                   // emin of an empty span
            init[size_t(nsets) + size_t(i)] = -(1 << 20); // top of an empty span
        }
        D3G_CUDA(cudaMemcpyAsync(set_span.p, init.data(), sizeof(int) * init.size(), cudaMemcpyHostToDevice, s));
        if (nv > 0)
            k_set_span<<<grid_for((int64_t(nv) + 63) / 64, 128, 1 << 30), 128, 0, s>>>(vx.p, nv, vset.p, set_span.p,
                                                                                 set_span.p + nsets);
        k_set_exact<<<grid_for(nsets, 128), 128, 0, s>>>(set_span.p, set_span.p + nsets, nsets, set_exact.p);
        D3G_CUDA(cudaStreamSynchronize(s));   // `init` must outlive the copy
    }

    // ---- workers ----
    // A level of s points goes into a triangulation of p earlier points.  Two
    // insertions collide when their regions (about 20 tets and their ring)
    // meet, so the useful number of simultaneous insertions grows with p, not
    // with s: each level gets about p / alpha workers (a fixed chunk if the
    // caller asks for one), each with a chunk of at least kMinChunk points.
    // Several sets: their levels are aligned from the coarsest, and a round
    // serves the workers of every set at once.
    const int alpha = opt.chunk < 0 ? -opt.chunk : 48;
    constexpr int kMinChunk = 16;
    // Below one latency wave of the GPU (about 4K resident warps), a round costs
    // the same whatever its size: then a denser pool (down to one worker per
    // kAlphaSmall earlier points) trades more collisions for far fewer rounds.
    constexpr double kWaveWorkers = 4096.0;
    const double kAlphaSmall = opt.alpha_small > 0 ? double(opt.alpha_small) : double(alpha);
    auto level_chunk = [&](int64_t lb, int64_t le, double alpha_eff) -> int {
        if (opt.chunk > 0) return opt.chunk;
        const int64_t s_ = le - lb;
        int64_t w_ = std::max<int64_t>(1, int64_t(double(lb) / alpha_eff));
        w_ = std::min<int64_t>(w_, (s_ + kMinChunk - 1) / kMinChunk);
        return int((s_ + w_ - 1) / w_);
    };
    // levels[set] = bounds from the coarsest: [lev[k], lev[k+1]) local vertex ids.
    std::vector<std::vector<int>> levels(static_cast<size_t>(nsets));
    int nlev = 0;
    for (int st = 0; st < nsets; ++st) {
        if (hskips[size_t(st)].x < 0) continue;
        int64_t hb[64];
        const int nb = multiscale_bounds(R.set_nv[size_t(st)], hb, 63, level_ratio);
        std::vector<int>& L = levels[size_t(st)];
        L.push_back(0);
        for (int k = nb - 1; k >= 0; --k) L.push_back(int(hb[k]));
        nlev = std::max(nlev, int(L.size()) - 1);
    }
    // The effective alpha of a level: alpha, lowered (to kAlphaSmall at most)
    // while the whole pool would stay below one latency wave.
    auto level_alpha = [&](int lev) -> double {
        double w0 = 0;
        for (int st = 0; st < nsets; ++st) {
            const std::vector<int>& L = levels[size_t(st)];
            if (int(L.size()) - 1 <= lev) continue;
            w0 += std::max(1.0, double(L[size_t(lev)]) / alpha);
        }
        const double m = std::min(std::max(kWaveWorkers / std::max(w0, 1.0), 1.0), alpha / kAlphaSmall);
        return alpha / m;
    };
    auto level_descs = [&](int lev, double alpha_eff, std::vector<LevelDesc>& out) -> int {
        out.clear();
        int w = 0;
        for (int st = 0; st < nsets; ++st) {
            const std::vector<int>& L = levels[size_t(st)];
            if (int(L.size()) - 1 <= lev) continue;
            const int lb = L[size_t(lev)], le = L[size_t(lev) + 1];
            if (le <= lb) continue;
            const int plb = lev > 0 ? L[size_t(lev) - 1] : 0, ple = lb;
            const int ch = level_chunk(lb, le, alpha_eff);
            const int base = hvoff[size_t(st)];
            out.push_back(LevelDesc{st, base + lb, base + le, ch, base + plb, base + ple, w});
            w += (le - lb + ch - 1) / ch;
        }
        return w;
    };
    int maxw = 1;
    {
        std::vector<LevelDesc> tmp;
        for (int lev = 0; lev < nlev; ++lev) maxw = std::max(maxw, level_descs(lev, level_alpha(lev), tmp));
    }
    // Room for the pool to grow within levels (at most one worker per 16 points).
    const bool grow = opt.chunk <= 0 && opt.split != 0;
    if (grow) maxw = std::max<int>(maxw, int(std::min<int64_t>(int64_t(nv) / 16, int64_t(1) << 18)));
    // Asynchronous passes (see k_insert_async): a persistent grid of at most
    // kAsyncWarps warps per level, the fast variant over the level's chunks,
    // the full variant over what that leaves; the rounds finish the rest.
    const bool use_async = opt.schedule != 1 && !grow;
    constexpr int kAsyncWarps = kNumSMs * 32;   // resident at 64 registers a thread
    // The passes over left points take all of them at once, one worker per
    // point: the workers' own records are sized for that (wcap), the
    // per-slot scratch (conflict region, boundary facets, staged tets) for the
    // warps of a pass and the workers of a round, whichever is more (wslots).
    const int wcap = use_async ? std::max<int>(maxw, int(std::min<int64_t>(nv, int64_t(1) << 20))) : maxw;
    const int wslots = std::max(maxw, std::min(wcap, kAsyncWarps));
    Workers W;
    // Conflict-region scratch per worker (normal rounds and asynchronous
    // passes) and per big-round slot; a caller's cavity_capacity lowers both.
    const int cav_normal = opt.cavity_capacity > 0 ? std::min(kCavCap, int(opt.cavity_capacity)) : kCavCap;
    const int cav_big = opt.cavity_capacity > 0 ? std::min(kBigCav, int(opt.cavity_capacity)) : kBigCav;
    W.cav_cap = cav_normal;
    W.fac_cap = 2 * cav_normal;
    W.n = maxw;
    DevBuf<int> wcur, wbeg, wend, wpos, wleft, wnwon, wlast, wguide, wstate, wncav, wnfac, wcav, wfac, counters;
    DevBuf<int> set_p0, set_ins, set_w, set_split, nworkers;
    DevBuf<int> wparked, wset, blist, bcount, bcav, bfac;
    DevBuf<int4> bsv, bsn;
    DevBuf<int4> wsv, wsn;
    D3G_TRY(wcur.alloc(size_t(wcap), s));
    D3G_TRY(wend.alloc(size_t(wcap), s));
    D3G_TRY(wbeg.alloc(size_t(wcap), s));
    D3G_TRY(wparked.alloc(size_t(wcap), s));
    D3G_TRY(wset.alloc(size_t(wcap), s));
    D3G_TRY(wpos.alloc(size_t(wcap), s));
    D3G_TRY(wleft.alloc(size_t(wcap), s));
    D3G_TRY(wnwon.alloc(size_t(wcap), s));
    D3G_TRY(set_p0.alloc(size_t(nsets), s));
    D3G_TRY(set_ins.alloc(size_t(nsets), s));
    D3G_TRY(set_w.alloc(size_t(nsets), s));
    D3G_TRY(set_split.alloc(size_t(nsets), s));
    D3G_TRY(nworkers.alloc(1, s));
    D3G_CUDA(cudaMemsetAsync(set_ins.p, 0, sizeof(int) * size_t(nsets), s));
    SplitState SS{set_p0.p, set_ins.p, set_w.p, set_split.p, nworkers.p, maxw};
    D3G_TRY(wlast.alloc(size_t(wcap), s));
    D3G_TRY(wguide.alloc(size_t(wcap), s));
    D3G_TRY(wstate.alloc(size_t(wcap), s));
    D3G_TRY(wncav.alloc(size_t(wcap), s));
    D3G_TRY(wnfac.alloc(size_t(wcap), s));
    D3G_TRY(wcav.alloc(size_t(wslots) * W.cav_cap, s));
    D3G_TRY(wfac.alloc(size_t(wslots) * W.fac_cap, s));
    D3G_TRY(wsv.alloc(size_t(wslots) * W.fac_cap, s));
    D3G_TRY(wsn.alloc(size_t(wslots) * W.fac_cap, s));
    D3G_TRY(counters.alloc(4, s));
    DevBuf<unsigned long long> sums, totals, steps;
    DevBuf<unsigned> dround;
    D3G_TRY(sums.alloc(2, s));
    D3G_TRY(steps.alloc(2, s));
    D3G_CUDA(cudaMemsetAsync(steps.p, 0, 2 * sizeof(unsigned long long), s));
    D3G_TRY(totals.alloc(6, s));
    D3G_TRY(dround.alloc(1, s));
    D3G_CUDA(cudaMemsetAsync(sums.p, 0, 2 * sizeof(unsigned long long), s));
    D3G_CUDA(cudaMemsetAsync(totals.p, 0, 6 * sizeof(unsigned long long), s));
    D3G_CUDA(cudaMemsetAsync(dround.p, 0, sizeof(unsigned), s));
    W.cur = wcur.p;
    W.end = wend.p;
    W.beg = wbeg.p;
    W.list = nullptr;
    W.parked = wparked.p;
    W.wset = wset.p;
    W.skips = skips.p;
    W.set_exact = set_exact.p;
    W.pos = wpos.p;
    W.left = wleft.p;
    W.nwon = wnwon.p;
    W.last = wlast.p;
    W.guide = wguide.p;
    W.state = wstate.p;
    W.ncav = wncav.p;
    W.nfac = wnfac.p;
    W.cav = wcav.p;
    W.fac = wfac.p;
    W.st_v = wsv.p;
    W.st_n = wsn.p;

    Round Rd;
    Rd.counters = counters.p;
    Rd.sums = sums.p;
    Rd.totals = totals.p;
    Rd.steps = opt.timing ? steps.p : nullptr;
    Rd.round = dround.p;
    Rd.status = status.p;
    DevBuf<unsigned long long> pstats;
    D3G_TRY(pstats.alloc(4, s));
    D3G_CUDA(cudaMemsetAsync(pstats.p, 0, 4 * sizeof(unsigned long long), s));
    Rd.pstats = pstats.p;
    const int max_rounds = opt.max_rounds > 0 ? opt.max_rounds : (1 << 20);
    int round = 0;
    DevBuf<int> alock, anext, aleft, aleft2, anleft;
    DevBuf<unsigned long long> astats, aekey;
    if (use_async) {
        D3G_TRY(aekey.alloc(size_t(std::min(wslots, kAsyncWarps)) * 3 * size_t(W.fac_cap), s));
        D3G_TRY(alock.alloc(size_t(T.cap), s));
        D3G_TRY(anext.alloc(1, s));
        D3G_TRY(aleft.alloc(size_t(nv), s));
        D3G_TRY(aleft2.alloc(size_t(nv), s));
        D3G_TRY(anleft.alloc(2, s));
        D3G_TRY(astats.alloc(7, s));
        D3G_CUDA(cudaMemsetAsync(alock.p, 0, sizeof(int) * size_t(T.cap), s));
        D3G_CUDA(cudaMemsetAsync(astats.p, 0, 7 * sizeof(unsigned long long), s));
    }
    // Structural self-check after each level (opt.validate): k_validate over
    // every tet slot and vertex; the first broken invariant ends the build.
    DevBuf<unsigned long long> vfail;
    auto validate_tables = [&](const char* when, int lev) -> int {
        if (!vfail.p) D3G_TRY(vfail.alloc(1, s));
        D3G_CUDA(cudaMemsetAsync(vfail.p, 0xFF, sizeof(unsigned long long), s));
        int ntet_now = 0;
        D3G_CUDA(cudaMemcpyAsync(&ntet_now, tet_count.p, sizeof ntet_now, cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaStreamSynchronize(s));
        const int64_t threads = int64_t(ntet_now) + nv;
        k_validate<<<grid_for(threads, 256, 1 << 30), 256, 0, s>>>(T, use_async ? alock.p : nullptr, ntet_now, nv,
                                                                   status.p, vfail.p);
        D3G_CUDA(cudaGetLastError());
        unsigned long long rec = ~0ull;
        D3G_CUDA(cudaMemcpyAsync(&rec, vfail.p, sizeof rec, cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaStreamSynchronize(s));
        if (rec == ~0ull) return D3G_OK;
        static const char* what[] = {"", "bad vertex", "bad neighbour", "neighbour does not point back",
                                     "neighbours' shared facets differ", "lock held", "vertex's tet",
                                     "vertices of different sets"};
        const int code = int(rec >> 60);
        char msg[200];
        std::snprintf(msg, sizeof msg, "d3g_build: validate %s level %d: %s (%s %lld, %lld)", when, lev,
                      what[code > 0 && code < 8 ? code : 0], code == VF_VERT_TET ? "vertex" : "tet",
                      (long long)((rec >> 30) & 0x3FFFFFFFull), (long long)(rec & 0x3FFFFFFFull));
        set_error(msg);
        return D3G_ERR_INTERNAL;
    };
    const bool trace = getenv("D3G_TRACE") != nullptr;
    cudaEvent_t kev[4] = {nullptr, nullptr, nullptr, nullptr};
    if (opt.timing)
        for (auto& e : kev) cudaEventCreate(&e);
    struct EvGuard {
        cudaEvent_t* e;
        ~EvGuard() {
            for (int i = 0; i < 4; ++i)
                if (e[i]) cudaEventDestroy(e[i]);
        }
    } ev_guard{kev};
    // Big rounds: workers whose conflict region outgrew the normal scratch.
    Workers WB = W;
    auto big_rounds = [&]() -> int {
        if (!blist.p) {
            D3G_TRY(blist.alloc(size_t(maxw), s));
            D3G_TRY(bcount.alloc(1, s));
            D3G_TRY(bcav.alloc(size_t(kBigSlots) * cav_big, s));
            D3G_TRY(bfac.alloc(size_t(kBigSlots) * 2 * cav_big, s));
            D3G_TRY(bsv.alloc(size_t(kBigSlots) * 2 * cav_big, s));
            D3G_TRY(bsn.alloc(size_t(kBigSlots) * 2 * cav_big, s));
        }
        for (;;) {
            D3G_CUDA(cudaMemsetAsync(bcount.p, 0, sizeof(int), s));
            k_collect_parked<<<grid_for(W.n, 128, 1 << 30), 128, 0, s>>>(W, blist.p, bcount.p);
            int nparked = 0;
            D3G_CUDA(cudaMemcpyAsync(&nparked, bcount.p, sizeof nparked, cudaMemcpyDeviceToHost, s));
            D3G_CUDA(cudaStreamSynchronize(s));
            if (nparked == 0) return D3G_OK;
            WB = W;
            WB.list = blist.p;
            WB.n = std::min(nparked, kBigSlots);
            WB.cav = bcav.p;
            WB.fac = bfac.p;
            WB.st_v = bsv.p;
            WB.st_n = bsn.p;
            WB.cav_cap = cav_big;
            WB.fac_cap = 2 * cav_big;
            for (;;) {
                if (++round > max_rounds) {
                    set_error("d3g_build: insertion round limit reached");
                    return D3G_ERR_ROUND_LIMIT;
                }
                unsigned long long before = 0;
                D3G_CUDA(cudaMemcpyAsync(&before, totals.p, sizeof before, cudaMemcpyDeviceToHost, s));
                k_round_begin<<<1, 1, 0, s>>>(Rd);
                launch_insertion(32, 0, T, WB, Rd, vx.p, s);
                launch_insertion(32, 1, T, WB, Rd, vx.p, s);
                launch_insertion(32, 2, T, WB, Rd, vx.p, s);
                k_round_end<<<1, 1, 0, s>>>(Rd);
                unsigned long long ht[6];
                uint32_t hs = 0;
                D3G_CUDA(cudaMemcpyAsync(ht, totals.p, sizeof ht, cudaMemcpyDeviceToHost, s));
                D3G_CUDA(cudaMemcpyAsync(&hs, status.p, sizeof hs, cudaMemcpyDeviceToHost, s));
                D3G_CUDA(cudaStreamSynchronize(s));
                if (hs != 0) {
                    const int st = status_from_bits(hs);
                    if (st == D3G_ERR_CAVITY_CAPACITY)
                        set_error("d3g_build: a conflict region exceeded the big-round scratch");
                    return st;
                }
                if (ht[3] == 0) break;           // every listed worker got its point in
                if (ht[0] == before) {           // the earliest parked point must win
                    set_error("d3g_build: a big round made no progress");
                    return D3G_ERR_INTERNAL;
                }
            }
        }
    };
    std::vector<LevelDesc> descs;
    std::vector<int> hp0(static_cast<size_t>(nsets)), hw(static_cast<size_t>(nsets));
    for (int lev = 0; lev < nlev; ++lev) {
        const double alpha_eff = level_alpha(lev);
        W.n = level_descs(lev, alpha_eff, descs);
        if (W.n == 0) continue;
        char level_name[32];
        std::snprintf(level_name, sizeof level_name, "d3g.level %d", lev);
        NvtxRange nvtx_level(level_name);
        std::fill(hp0.begin(), hp0.end(), 0);
        std::fill(hw.begin(), hw.end(), 0);
        for (size_t i = 0; i < descs.size(); ++i) {
            const LevelDesc& d = descs[i];
            hp0[size_t(d.set)] = d.lb - hvoff[size_t(d.set)];
            hw[size_t(d.set)] = (i + 1 < descs.size() ? descs[i + 1].w0 : W.n) - d.w0;
        }
        D3G_CUDA(cudaMemcpyAsync(set_p0.p, hp0.data(), sizeof(int) * size_t(nsets), cudaMemcpyHostToDevice, s));
        D3G_CUDA(cudaMemcpyAsync(set_w.p, hw.data(), sizeof(int) * size_t(nsets), cudaMemcpyHostToDevice, s));
        k_set_int<<<1, 1, 0, s>>>(nworkers.p, W.n);
        const int round0 = round;
        long long won = 0, attempts = 0;
        long long won_before = 0, att_before = 0;
        {
            unsigned long long ht0[2];
            D3G_CUDA(cudaMemcpyAsync(ht0, totals.p, sizeof ht0, cudaMemcpyDeviceToHost, s));
            D3G_CUDA(cudaStreamSynchronize(s));
            won_before = (long long)ht0[0];
            att_before = (long long)ht0[1];
        }
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        if (trace) {
            cudaEventCreate(&ev0);
            cudaEventCreate(&ev1);
            cudaEventRecord(ev0, s);
        }
        DevBuf<LevelDesc> ddesc;
        D3G_TRY(ddesc.alloc(descs.size(), s));
        D3G_CUDA(cudaMemcpyAsync(ddesc.p, descs.data(), sizeof(LevelDesc) * descs.size(), cudaMemcpyHostToDevice, s));
        k_setup_level<<<grid_for(W.n, 128, 1 << 30), 128, 0, s>>>(W, ddesc.p, int(descs.size()));
        int lanes = opt.lanes > 0 ? opt.lanes : 32;
        auto one_round = [&](bool timed) {
            k_round_begin<<<1, 1, 0, s>>>(Rd);
            if (timed) cudaEventRecord(kev[0], s);
            launch_insertion(lanes, 0, T, W, Rd, vx.p, s);
            if (timed) cudaEventRecord(kev[1], s);
            launch_insertion(lanes, 1, T, W, Rd, vx.p, s);
            if (timed) cudaEventRecord(kev[2], s);
            launch_insertion(lanes, 2, T, W, Rd, vx.p, s);
            if (timed) cudaEventRecord(kev[3], s);
            k_round_end<<<1, 1, 0, s>>>(Rd);
        };
        // Rounds go out in batches captured as one CUDA graph; the host looks at
        // the counters once per batch.  Rounds after the level is done find no
        // active worker and return at once.
        cudaGraphExec_t gexec = nullptr;
        struct GraphGuard {
            cudaGraphExec_t* g;
            ~GraphGuard() {
                if (*g) cudaGraphExecDestroy(*g);
            }
        } graph_guard{&gexec};
        auto capture = [&]() -> int {
            if (gexec) cudaGraphExecDestroy(gexec);
            gexec = nullptr;
            if (opt.timing) return D3G_OK;
            cudaGraph_t graph = nullptr;
            D3G_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            for (int r = 0; r < kRoundsPerBatch; ++r) one_round(false);
            D3G_CUDA(cudaStreamEndCapture(s, &graph));
            const cudaError_t ge = cudaGraphInstantiate(&gexec, graph, 0);
            cudaGraphDestroy(graph);
            if (ge != cudaSuccess) {
                set_error(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ge));
                return D3G_ERR_CUDA;
            }
            return D3G_OK;
        };
        auto run_rounds = [&]() -> int {
        D3G_TRY(capture());
        for (;;) {
            const int batch = opt.timing ? 1 : kRoundsPerBatch;
            round += batch;
            if (round > max_rounds) {
                set_error("d3g_build: insertion round limit reached");
                return D3G_ERR_ROUND_LIMIT;
            }
            if (opt.timing) one_round(true);
            else D3G_CUDA(cudaGraphLaunch(gexec, s));
            if (grow) {
                D3G_CUDA(cudaMemsetAsync(set_ins.p, 0, sizeof(int) * size_t(nsets), s));
                k_count_wins<<<grid_for(W.n, 128, 1 << 30), 128, 0, s>>>(W, SS);
                k_plan_split<<<grid_for(nsets, 128), 128, 0, s>>>(SS, nsets, alpha_eff);
                k_split<<<grid_for(W.n, 128, 1 << 30), 128, 0, s>>>(W, SS, W.n);
            }
            unsigned long long ht[6];
            uint32_t hs = 0;
            int hn = W.n;
            D3G_CUDA(cudaMemcpyAsync(ht, totals.p, sizeof ht, cudaMemcpyDeviceToHost, s));
            D3G_CUDA(cudaMemcpyAsync(&hs, status.p, sizeof hs, cudaMemcpyDeviceToHost, s));
            if (grow) D3G_CUDA(cudaMemcpyAsync(&hn, nworkers.p, sizeof hn, cudaMemcpyDeviceToHost, s));
            D3G_CUDA(cudaStreamSynchronize(s));
            hn = std::min(hn, maxw);
            if (hn != W.n) {
                // The pool grew: the next batches serve the new workers too.
                W.n = hn;
                k_set_int<<<1, 1, 0, s>>>(nworkers.p, W.n);
                D3G_TRY(capture());
            }
            if (hs != 0) {
                const int st = status_from_bits(hs);
                if (st == D3G_ERR_OOM) set_error("d3g_build: tet table full");
                return st;
            }
            if (ht[4]) {
                set_error("d3g_build: an insertion round made no progress");
                return D3G_ERR_INTERNAL;
            }
            if (opt.timing) {
                float a = 0.f, b2 = 0.f, c = 0.f;
                cudaEventElapsedTime(&a, kev[0], kev[1]);
                cudaEventElapsedTime(&b2, kev[1], kev[2]);
                cudaEventElapsedTime(&c, kev[2], kev[3]);
                R.stats.ms_cavity += a;
                R.stats.ms_check += b2;
                R.stats.ms_restar += c;
                R.stats.launches_cavity += 1;
            }
            won = (long long)ht[0] - won_before;
            attempts = (long long)ht[1] - att_before;
            if (ht[5] != 0) continue;
            if (ht[3] == 0) break;
            // Only parked workers are left: serve them in big rounds, up to
            // kBigSlots at a time, each until its point is in.
            D3G_TRY(big_rounds());
        }
        return D3G_OK;
        };
        long long async_left = -1, deferred = -1;
        if (use_async) {
            // One asynchronous pass: a persistent grid over the workers W
            // (level chunks, or one leftover point each), writing the points it
            // leaves to `left` / `nleft_d`; their count goes to *nleft_out.
            auto async_pass = [&](bool fast, int nw, int* left, int* nleft_d,
                                  int* nleft_out) -> int {
                // The chunks go out in a scattered order (stride coprime with the
                // chunk count, near the golden ratio of it), so that chunks taken
                // at the same time lie far apart along the curve.
                int64_t stride = std::max<int64_t>(1, int64_t(double(nw) * 0.6180339887));
                while (std::gcd(stride, int64_t(nw)) != 1) ++stride;
                D3G_CUDA(cudaMemsetAsync(anext.p, 0, sizeof(int), s));
                AsyncCtx A{alock.p, anext.p, left, nleft_d, stride, nw, aekey.p, astats.p};
                const int warps = std::min(nw, kAsyncWarps);
                if (warps > wslots) {
                    set_error("d3g_build: asynchronous pass wider than its scratch");
                    return D3G_ERR_INTERNAL;
                }
                const unsigned grid = unsigned((int64_t(warps) * 32 + 127) / 128);
                unsigned long long won0 = 0;
                D3G_CUDA(cudaMemcpyAsync(&won0, totals.p, sizeof won0, cudaMemcpyDeviceToHost, s));
                if (opt.timing) cudaEventRecord(kev[0], s);
                if (fast) k_insert_async<true><<<grid, 128, 0, s>>>(T, W, A, Rd, vx.p, warps);
                else k_insert_async<false><<<grid, 128, 0, s>>>(T, W, A, Rd, vx.p, warps);
                D3G_CUDA(cudaGetLastError());
                if (opt.timing) cudaEventRecord(kev[1], s);
                uint32_t hs = 0;
                unsigned long long won1 = 0;
                D3G_CUDA(cudaMemcpyAsync(nleft_out, nleft_d, sizeof(int), cudaMemcpyDeviceToHost, s));
                D3G_CUDA(cudaMemcpyAsync(&hs, status.p, sizeof hs, cudaMemcpyDeviceToHost, s));
                D3G_CUDA(cudaMemcpyAsync(&won1, totals.p, sizeof won1, cudaMemcpyDeviceToHost, s));
                D3G_CUDA(cudaStreamSynchronize(s));
                R.stats.launches_async += 1;
                R.stats.async_inserted += int64_t(won1 - won0);
                if (trace)
                    fprintf(stderr, "d3g level %d async pass %s chunks-or-points %d inserted %llu left %d\n", lev,
                            fast ? "fast" : "full", nw, won1 - won0, *nleft_out);
                if (opt.timing) {
                    float am = 0.f;
                    cudaEventElapsedTime(&am, kev[0], kev[1]);
                    R.stats.ms_async += am;
                }
                if (hs != 0) {
                    const int st = status_from_bits(hs);
                    if (st == D3G_ERR_OOM) set_error("d3g_build: tet table full");
                    return st;
                }
                return D3G_OK;
            };
            // The level's chunks through the fast variant; what it deferred or
            // left (undecided tests, lock conflicts, regions too big) through
            // the full variant, one worker per point, all of them at once,
            // again while a pass inserts at least a quarter of its points; what
            // that leaves through the rounds, maxw points at a time.
            int nleft = 0;
            D3G_CUDA(cudaMemsetAsync(anleft.p, 0, 2 * sizeof(int), s));
            D3G_TRY(async_pass(true, W.n, aleft.p, anleft.p, &nleft));
            deferred = nleft;
            int* cur = aleft.p;
            int* nxt = aleft2.p;
            int ncur = nleft;
            for (int pass = 0; ncur > 0 && pass < kLeftPasses; ++pass) {
                int nnext = 0;
                D3G_CUDA(cudaMemsetAsync(anleft.p + 1, 0, sizeof(int), s));
                for (int off = 0; off < ncur; off += wcap) {
                    W.n = std::min(wcap, ncur - off);
                    k_setup_list<<<grid_for(W.n, 128, 1 << 30), 128, 0, s>>>(W, cur + off, W.n, vset.p, voff.p,
                                                                            T.vert_tet);
                    D3G_TRY(async_pass(false, W.n, nxt, anleft.p + 1, &nnext));
                }
                const bool slow = int64_t(ncur - nnext) * 4 < int64_t(ncur);
                std::swap(cur, nxt);
                ncur = nnext;
                if (slow) break;
            }
            async_left = ncur;
            for (int off = 0; off < ncur; off += maxw) {
                W.n = std::min(maxw, ncur - off);
                k_setup_list<<<grid_for(W.n, 128, 1 << 30), 128, 0, s>>>(W, cur + off, W.n, vset.p, voff.p,
                                                                        T.vert_tet);
                D3G_TRY(run_rounds());
            }
        } else {
            D3G_TRY(run_rounds());
        }
        if (opt.validate) D3G_TRY(validate_tables("after", lev));
        if (trace) {
            cudaEventRecord(ev1, s);
            cudaEventSynchronize(ev1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev0, ev1);
            {
                unsigned long long ht1[2];
                cudaMemcpy(ht1, totals.p, sizeof ht1, cudaMemcpyDeviceToHost);
                won = (long long)ht1[0] - won_before;
                attempts = (long long)ht1[1] - att_before;
            }
            unsigned long long as[7] = {0, 0, 0, 0, 0, 0, 0};
            if (use_async) cudaMemcpy(as, astats.p, sizeof as, cudaMemcpyDeviceToHost);
            fprintf(stderr, "d3g level %d sets %zu workers %d rounds %d inserted %lld attempts %lld "
                    "left-by-fast-pass %lld left-by-async %lld ms %.2f | async totals: lock-conflicts %llu "
                    "walk-restarts %llu bad-seeds %llu too-big %llu left %llu first-left %llu deferred %llu\n",
                    lev, descs.size(), W.n, round - round0, won, attempts, deferred, async_left, ms, as[0],
                    as[1], as[2], as[3], as[4], as[5], as[6]);
            cudaEventDestroy(ev0);
            cudaEventDestroy(ev1);
        }
    }
    {
        unsigned long long hs2[2] = {0, 0}, ht[6], hst[2] = {0, 0}, hp[4] = {0, 0, 0, 0}, ha[7] = {};
        D3G_CUDA(cudaMemcpyAsync(hp, pstats.p, sizeof hp, cudaMemcpyDeviceToHost, s));
        if (use_async) D3G_CUDA(cudaMemcpyAsync(ha, astats.p, sizeof ha, cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaMemcpyAsync(hs2, sums.p, sizeof hs2, cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaMemcpyAsync(hst, steps.p, sizeof hst, cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaMemcpyAsync(ht, totals.p, sizeof ht, cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaStreamSynchronize(s));
        R.stats.region_tets = int64_t(hs2[0]);
        R.stats.boundary_facets = int64_t(hs2[1]);
        R.stats.rounds = int(ht[2]);
        R.stats.attempts = int64_t(ht[1]);
        R.stats.walk_steps = int64_t(hst[0]);
        R.stats.bfs_steps = int64_t(hst[1]);
        R.stats.conflict_tests = int64_t(hp[0]);
        R.stats.uncertain_tests = int64_t(hp[1]);
        R.stats.tie_breaks = int64_t(hp[2]);
        R.stats.max_region_tets = int64_t(hp[3]);
        R.stats.deferred_points = int64_t(ha[6]);
    }
    // Release round scratch before the output stage.
    wcav.release();
    wfac.release();
    wsv.release();
    wsn.release();
    claim.release();
    fnew.release();

    cudaEventRecord(ph[2], s);
    nvtx_phase.reset();
    nvtx_phase.emplace("d3g.output");
    // ---- output: canonical cells ----
    int ntet = 0;
    D3G_CUDA(cudaMemcpyAsync(&ntet, tet_count.p, sizeof ntet, cudaMemcpyDeviceToHost, s));
    D3G_CUDA(cudaStreamSynchronize(s));
    const int kbits = bits_for(uint64_t(max_n) + 1);
    for (int pass = 0; pass < (single && opt.want_all_cells ? 2 : 1); ++pass) {
        const bool with_inf = pass == 1;
        DevBuf<int32_t> flag, pos, idx, cset;
        D3G_TRY(flag.alloc(size_t(ntet), s));
        D3G_TRY(pos.alloc(size_t(ntet), s));
        k_cell_flags<<<grid_for(ntet, 256), 256, 0, s>>>(tv.p, alive.p, ntet, with_inf, flag.p);
        D3G_TRY(exclusive_scan(flag.p, pos.p, ntet, s));
        int last_pos = 0, last_flag = 0;
        D3G_CUDA(cudaMemcpyAsync(&last_pos, pos.p + ntet - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaMemcpyAsync(&last_flag, flag.p + ntet - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        D3G_CUDA(cudaStreamSynchronize(s));
        const int64_t nc = int64_t(last_pos) + last_flag;
        DevBuf<int4> raw;
        DevBuf<unsigned long long> khi, klo;
        D3G_TRY(raw.alloc(size_t(nc), s));
        D3G_TRY(khi.alloc(size_t(nc), s));
        D3G_TRY(klo.alloc(size_t(nc), s));
        D3G_TRY(idx.alloc(size_t(nc), s));
        if (!single) D3G_TRY(cset.alloc(size_t(nc), s));
        if (!with_inf) {
            // Buckets by first vertex; the radix sort of every cell only if a
            // bucket is too large for one thread.
            k_cells_out<<<grid_for(ntet, 256), 256, 0, s>>>(tv.p, flag.p, pos.p, ntet, vert_point.p, vset.p,
                                                            kbits, raw.p, nullptr, nullptr, nullptr,
                                                            single ? nullptr : cset.p);
            DevBuf<int> bstart, bfill, big, mid;
            D3G_TRY(bstart.alloc(size_t(N) + 1, s));
            D3G_TRY(bfill.alloc(size_t(N) + 1, s));
            D3G_TRY(big.alloc(2, s));
            D3G_TRY(mid.alloc(size_t(nc / (kBucketThread + 1)) + 1, s));
            D3G_TRY(R.cells.alloc(size_t(nc), s));
            D3G_CUDA(cudaMemsetAsync(bfill.p, 0, sizeof(int) * (size_t(N) + 1), s));
            D3G_CUDA(cudaMemsetAsync(big.p, 0, 2 * sizeof(int), s));
            if (nc > 0) {
                k_bucket_count<<<grid_for(nc, 256), 256, 0, s>>>(raw.p, single ? nullptr : cset.p, d_off.p, nc,
                                                                 bfill.p);
            }
            D3G_TRY(exclusive_scan(bfill.p, bstart.p, int64_t(N) + 1, s));
            D3G_CUDA(cudaMemsetAsync(bfill.p, 0, sizeof(int) * (size_t(N) + 1), s));
            if (nc > 0) {
                k_bucket_place<<<grid_for(nc, 256), 256, 0, s>>>(raw.p, single ? nullptr : cset.p, d_off.p, nc,
                                                                 bstart.p, bfill.p, R.cells.p);
                k_bucket_sort<<<grid_for(N, 128), 128, 0, s>>>(R.cells.p, bstart.p, N, mid.p, big.p + 1, big.p);
            }
            int hbig[2] = {0, 0};
            D3G_CUDA(cudaMemcpyAsync(hbig, big.p, sizeof hbig, cudaMemcpyDeviceToHost, s));
            if (!single) {
                DevBuf<int64_t> coff;
                D3G_TRY(coff.alloc(size_t(nsets) + 1, s));
                k_cell_off<<<grid_for(nsets + 1, 128), 128, 0, s>>>(bstart.p, d_off.p, nsets, coff.p);
                D3G_CUDA(cudaMemcpyAsync(R.cell_off.data(), coff.p, sizeof(int64_t) * (size_t(nsets) + 1),
                                         cudaMemcpyDeviceToHost, s));
            }
            D3G_CUDA(cudaStreamSynchronize(s));
            R.n_cells = nc;
            if (single) R.cell_off[1] = nc;
            if (!hbig[0] && hbig[1] > 0)
                k_bucket_sort_block<<<unsigned(hbig[1]), 512, 0, s>>>(R.cells.p, bstart.p, mid.p);
            if (hbig[0]) {
                k_cells_out<<<grid_for(ntet, 256), 256, 0, s>>>(tv.p, flag.p, pos.p, ntet, vert_point.p, vset.p,
                                                                kbits, raw.p, khi.p, klo.p, idx.p,
                                                                single ? nullptr : cset.p);
                D3G_TRY(sort_cells(raw, khi, klo, idx, single ? nullptr : cset.p, nsets, nc, kbits, R.cells, s));
            }
        } else {
            k_cells_out<<<grid_for(ntet, 256), 256, 0, s>>>(tv.p, flag.p, pos.p, ntet, vert_point.p, vset.p,
                                                            kbits, raw.p, khi.p, klo.p, idx.p, nullptr);
            D3G_TRY(sort_cells(raw, khi, klo, idx, nullptr, 1, nc, kbits, R.all, s));
            R.n_all = nc;
        }
    }
    if (single && opt.want_incident) {
        const int64_t m = 4 * R.n_cells;
        DevBuf<int32_t> pt, cell, pt2, cnt;
        D3G_TRY(R.inc_off.alloc(size_t(N) + 1, s));
        D3G_TRY(R.inc.alloc(size_t(m > 0 ? m : 1), s));
        D3G_TRY(cnt.alloc(size_t(N) + 1, s));
        D3G_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (size_t(N) + 1), s));
        if (m > 0) {
            D3G_TRY(pt.alloc(size_t(m), s));
            D3G_TRY(cell.alloc(size_t(m), s));
            D3G_TRY(pt2.alloc(size_t(m), s));
            k_incident_pairs<<<grid_for(R.n_cells, 256), 256, 0, s>>>(R.cells.p, R.n_cells, pt.p, cell.p,
                                                                     cnt.p);
            D3G_TRY(sort_pairs(pt.p, pt2.p, cell.p, R.inc.p, m, 0, bits_for(uint64_t(N)), s));
        }
        DevBuf<int64_t> cnt64;
        D3G_TRY(cnt64.alloc(size_t(N) + 1, s));
        k_widen<<<grid_for(n + 1, 256), 256, 0, s>>>(cnt.p, n + 1, cnt64.p);
        D3G_TRY(exclusive_scan(cnt64.p, R.inc_off.p, n + 1, s));
        R.n_inc = m;
    }
    D3G_CUDA(cudaGetLastError());
    cudaEventRecord(ph[3], s);
    D3G_CUDA(cudaMemcpyAsync(hst, status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    D3G_CUDA(cudaStreamSynchronize(s));
    {
        float a = 0.f, b = 0.f, c = 0.f;
        cudaEventElapsedTime(&a, ph[0], ph[1]);
        cudaEventElapsedTime(&b, ph[1], ph[2]);
        cudaEventElapsedTime(&c, ph[2], ph[3]);
        R.stats.ms_order = a;
        R.stats.ms_rounds = b;
        R.stats.ms_output = c;
    }
    return status_from_bits(hst[0]);
}

}  // namespace d3g

using namespace d3g;

namespace d3g {
namespace {

// The settings d3g_autotune_device chose, per device (d3g_options_default
// hands them out).
constexpr int kMaxTunedDevices = 64;
std::mutex g_tuning_mu;
d3g_tuning g_tuning[kMaxTunedDevices];
bool g_tuned[kMaxTunedDevices] = {};

bool current_tuning(d3g_tuning* out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxTunedDevices) {
        cudaGetLastError();
        return false;
    }
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    if (!g_tuned[dev]) return false;
    *out = g_tuning[dev];
    return true;
}

}  // namespace
}  // namespace d3g

extern "C" {

void d3g_options_default(d3g_options* o) {
    if (!o) return;
    o->want_all_cells = 1;
    o->want_incident = 1;
    o->chunk = 0;
    o->max_rounds = 0;
    o->timing = 0;
    o->alpha_small = 24;
    o->lanes = 0;
    o->schedule = 0;
    o->split = 0;
    o->tet_capacity = 0;
    o->walk_limit = 0;
    o->cavity_capacity = 0;
    o->level_growth = 0;
    // D3G_VALIDATE=1 in the environment turns the device self-check on for every
    // build that takes the defaults (as the reference's DEL3D_VALIDATE builds do).
    const char* val = getenv("D3G_VALIDATE");
    o->validate = (val && val[0] && val[0] != '0') ? 1 : 0;
    d3g_tuning t;
    if (current_tuning(&t)) {
        o->schedule = t.schedule;
        o->chunk = t.chunk;
        o->alpha_small = t.alpha_small;
        o->lanes = t.lanes;
    }
}

int d3g_get_tuning(d3g_tuning* out) {
    if (!out) return D3G_ERR_INVALID_ARGUMENT;
    if (!current_tuning(out)) {
        d3g_options o;
        d3g_options_default(&o);
        *out = d3g_tuning{o.schedule, o.chunk, o.alpha_small, o.lanes, 0.0, 0};
    }
    return D3G_OK;
}

int d3g_reset_tuning(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxTunedDevices) {
        cudaGetLastError();
        return D3G_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    g_tuned[dev] = false;
    return D3G_OK;
}

int d3g_autotune_device(const double* d_xyz, const int64_t* set_offsets, int32_t n_sets, void* stream,
                        d3g_tuning* best) {
    if (n_sets < 1 || !set_offsets || set_offsets[0] != 0 || set_offsets[n_sets] < 0 ||
        (set_offsets[n_sets] > 0 && !d_xyz))
        return D3G_ERR_INVALID_ARGUMENT;
    D3G_TRY(ensure_device());
    int dev = 0;
    D3G_CUDA(cudaGetDevice(&dev));
    if (dev >= kMaxTunedDevices) return D3G_ERR_NO_DEVICE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Candidates: the schedule, the worker density (one worker per `alpha`
    // earlier points, denser below one wave: `alpha_small`) and, for the
    // lockstep rounds, the lanes per worker.  Every setting gives the same
    // cells; only the time differs.
    struct Cand { int schedule, alpha, alpha_small, lanes; };
    std::vector<Cand> cands;
    for (int a : {24, 48, 96})
        for (int as : {12, 24}) cands.push_back({0, a, as, 0});
    for (int a : {24, 48})
        for (int l : {32, 16}) cands.push_back({1, a, 24, l});
    cudaEvent_t e0, e1;
    D3G_CUDA(cudaEventCreate(&e0));
    D3G_CUDA(cudaEventCreate(&e1));
    d3g_tuning win{0, 0, 24, 0, 1e30, 0};
    int st = D3G_OK;
    for (const Cand& c : cands) {
        d3g_options o;
        d3g_options_default(&o);
        o.want_all_cells = 0;
        o.want_incident = 0;
        o.schedule = c.schedule;
        o.chunk = -c.alpha;
        o.alpha_small = c.alpha_small;
        o.lanes = c.lanes;
        float best_ms = 1e30f;
        for (int rep = 0; rep < 2 && st == D3G_OK; ++rep) {   // first run warms the pool
            DeviceResult R;
            cudaEventRecord(e0, s == nullptr ? cudaStreamLegacy : s);
            st = build_on_stream(d_xyz, set_offsets, n_sets, o, s, R);
            cudaEventRecord(e1, s == nullptr ? cudaStreamLegacy : s);
            R.reset();
            if (st != D3G_OK) break;
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                st = D3G_ERR_CUDA;
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) best_ms = ms;
        }
        if (st != D3G_OK) break;
        win.candidates += 1;
        if (best_ms < win.ms) win = d3g_tuning{c.schedule, -c.alpha, c.alpha_small, c.lanes, best_ms, win.candidates};
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != D3G_OK) return st;
    {
        std::lock_guard<std::mutex> lock(g_tuning_mu);
        g_tuning[dev] = win;
        g_tuned[dev] = true;
    }
    if (best) *best = win;
    return D3G_OK;
}

void d3g_result_free(d3g_result* r) {
    if (!r) return;
    host_result_free(r->cells);
    host_result_free(r->all_cells);
    host_result_free(r->incident_offsets);
    host_result_free(r->incident);
    *r = d3g_result{};
}

int d3g_build(const double* xyz, int64_t n, const d3g_options* opts, d3g_result* out) {
    if (!out || n < 0 || (n > 0 && !xyz)) return D3G_ERR_INVALID_ARGUMENT;
    *out = d3g_result{};
    d3g_options o;
    d3g_options_default(&o);
    if (opts) o = *opts;
    out->n_points = n;
    if (n == 0) {
        out->incident_offsets = static_cast<int64_t*>(calloc(1, sizeof(int64_t)));
        return D3G_OK;
    }
    D3G_TRY(ensure_device());
    cudaStream_t s = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st;
    DeviceResult R;
    {
        DevBuf<double> dx;
        D3G_TRY(dx.alloc(size_t(3 * n), s));
        D3G_CUDA(cudaMemcpyAsync(dx.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
        cudaEventRecord(e0, s);
        st = build_on_stream(dx.p, n, o, s, R);
        cudaEventRecord(e1, s);
    }
    if (st == D3G_OK) {
        out->n_vertices = R.n_vertices;
        out->n_cells = R.n_cells;
        out->n_all = R.n_all;
        out->stats = R.stats;
        out->cells = static_cast<int32_t*>(host_result_alloc(sizeof(int32_t) * 4 * size_t(R.n_cells > 0 ? R.n_cells : 1)));
        if (R.n_cells > 0)
            cudaMemcpyAsync(out->cells, R.cells.p, sizeof(int4) * R.n_cells, cudaMemcpyDeviceToHost, s);
        if (o.want_all_cells) {
            out->all_cells = static_cast<int32_t*>(host_result_alloc(sizeof(int32_t) * 4 * size_t(R.n_all > 0 ? R.n_all : 1)));
            if (R.n_all > 0)
                cudaMemcpyAsync(out->all_cells, R.all.p, sizeof(int4) * R.n_all, cudaMemcpyDeviceToHost, s);
        }
        if (o.want_incident) {
            out->incident_offsets = static_cast<int64_t*>(host_result_alloc(sizeof(int64_t) * (size_t(n) + 1)));
            out->incident = static_cast<int32_t*>(host_result_alloc(sizeof(int32_t) * size_t(R.n_inc > 0 ? R.n_inc : 1)));
            cudaMemcpyAsync(out->incident_offsets, R.inc_off.p, sizeof(int64_t) * (n + 1),
                            cudaMemcpyDeviceToHost, s);
            if (R.n_inc > 0)
                cudaMemcpyAsync(out->incident, R.inc.p, sizeof(int32_t) * R.n_inc, cudaMemcpyDeviceToHost, s);
        }
        const cudaError_t e = cudaStreamSynchronize(s);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        out->device_ms = ms;
        if (e != cudaSuccess) {
            set_error(std::string("d3g_build: ") + cudaGetErrorString(e));
            st = D3G_ERR_CUDA;
        }
    }
    R.reset();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != D3G_OK) d3g_result_free(out);
    return st;
}

int d3g_build_device(const double* d_xyz, int64_t n, const d3g_options* opts, int32_t* d_cells,
                     int64_t cap_cells, int64_t* n_cells_out, int64_t* n_vertices_out, void* stream,
                     d3g_build_stats* stats) {
    if (n < 0 || (n > 0 && !d_xyz) || cap_cells < 0) return D3G_ERR_INVALID_ARGUMENT;
    d3g_options o;
    d3g_options_default(&o);
    if (opts) o = *opts;
    o.want_all_cells = 0;
    o.want_incident = 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DeviceResult R;
    const int st = build_on_stream(d_xyz, n, o, s, R);
    if (st != D3G_OK) return st;
    if (n_cells_out) *n_cells_out = R.n_cells;
    if (n_vertices_out) *n_vertices_out = R.n_vertices;
    if (stats) *stats = R.stats;
    if (R.n_cells > cap_cells) {
        set_error("d3g_build_device: output capacity too small");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    if (R.n_cells > 0) {
        if (!d_cells) return D3G_ERR_INVALID_ARGUMENT;
        D3G_CUDA(cudaMemcpyAsync(d_cells, R.cells.p, sizeof(int4) * R.n_cells, cudaMemcpyDeviceToDevice, s));
    }
    R.reset();
    D3G_CUDA(cudaStreamSynchronize(s));
    return D3G_OK;
}

}  // extern "C"

extern "C" {

void d3g_batch_result_free(d3g_batch_result* r) {
    if (!r) return;
    host_result_free(r->cell_offsets);
    host_result_free(r->cells);
    host_result_free(r->n_vertices);
    *r = d3g_batch_result{};
}

int d3g_build_batch(const double* xyz, const int64_t* set_offsets, int32_t n_sets, const d3g_options* opts,
                    d3g_batch_result* out) {
    if (!out || n_sets < 1 || !set_offsets) return D3G_ERR_INVALID_ARGUMENT;
    *out = d3g_batch_result{};
    const int64_t n = set_offsets[n_sets];
    if (set_offsets[0] != 0 || n < 0 || (n > 0 && !xyz)) return D3G_ERR_INVALID_ARGUMENT;
    d3g_options o;
    d3g_options_default(&o);
    if (opts) o = *opts;
    D3G_TRY(ensure_device());
    cudaStream_t s = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st;
    DeviceResult R;
    {
        DevBuf<double> dx;
        D3G_TRY(dx.alloc(size_t(3 * (n > 0 ? n : 1)), s));
        if (n > 0) D3G_CUDA(cudaMemcpyAsync(dx.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
        cudaEventRecord(e0, s);
        st = build_on_stream(dx.p, set_offsets, n_sets, o, s, R);
        cudaEventRecord(e1, s);
    }
    if (st == D3G_OK) {
        out->n_sets = n_sets;
        out->stats = R.stats;
        out->cell_offsets = static_cast<int64_t*>(host_result_alloc(sizeof(int64_t) * (size_t(n_sets) + 1)));
        out->n_vertices = static_cast<int64_t*>(host_result_alloc(sizeof(int64_t) * size_t(n_sets)));
        out->cells = static_cast<int32_t*>(host_result_alloc(sizeof(int32_t) * 4 * size_t(R.n_cells > 0 ? R.n_cells : 1)));
        for (int i = 0; i <= n_sets; ++i) out->cell_offsets[i] = R.cell_off[size_t(i)];
        for (int i = 0; i < n_sets; ++i) out->n_vertices[i] = R.set_nv[size_t(i)];
        if (R.n_cells > 0)
            cudaMemcpyAsync(out->cells, R.cells.p, sizeof(int4) * R.n_cells, cudaMemcpyDeviceToHost, s);
        const cudaError_t e = cudaStreamSynchronize(s);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        out->device_ms = ms;
        if (e != cudaSuccess) {
            set_error(std::string("d3g_build_batch: ") + cudaGetErrorString(e));
            st = D3G_ERR_CUDA;
        }
    }
    R.reset();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != D3G_OK) d3g_batch_result_free(out);
    return st;
}

int d3g_build_batch_device(const double* d_xyz, const int64_t* set_offsets, int32_t n_sets,
                           const d3g_options* opts, int32_t* d_cells, int64_t cap_cells,
                           int64_t* cell_offsets, int64_t* n_vertices, void* stream, d3g_build_stats* stats) {
    if (n_sets < 1 || !set_offsets || cap_cells < 0) return D3G_ERR_INVALID_ARGUMENT;
    if (set_offsets[0] != 0 || set_offsets[n_sets] < 0 || (set_offsets[n_sets] > 0 && !d_xyz))
        return D3G_ERR_INVALID_ARGUMENT;
    d3g_options o;
    d3g_options_default(&o);
    if (opts) o = *opts;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DeviceResult R;
    const int st = build_on_stream(d_xyz, set_offsets, n_sets, o, s, R);
    if (st != D3G_OK) return st;
    if (cell_offsets)
        for (int i = 0; i <= n_sets; ++i) cell_offsets[i] = R.cell_off[size_t(i)];
    if (n_vertices)
        for (int i = 0; i < n_sets; ++i) n_vertices[i] = R.set_nv[size_t(i)];
    if (stats) *stats = R.stats;
    if (R.n_cells > cap_cells) {
        set_error("d3g_build_batch_device: output capacity too small");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    if (R.n_cells > 0) {
        if (!d_cells) return D3G_ERR_INVALID_ARGUMENT;
        D3G_CUDA(cudaMemcpyAsync(d_cells, R.cells.p, sizeof(int4) * R.n_cells, cudaMemcpyDeviceToDevice, s));
    }
    R.reset();
    D3G_CUDA(cudaStreamSynchronize(s));
    return D3G_OK;
}

}  // extern "C"
