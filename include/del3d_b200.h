/*
 * del3d_b200 - C ABI of the B200 (sm_100a) implementation of del3d's
 * Delaunay::build hot path.
 *
 * Plain pointers and sizes only.  Every entry point returns a d3g_status; none
 * aborts.  Entry points whose name ends in _device take device pointers and a
 * cudaStream_t (passed as void*; NULL = the legacy default stream) and run
 * asynchronously on that stream unless stated otherwise; the others take host
 * pointers, copy in and out, and return when the result is on the host.
 *
 * Reference interfaces replaced (paths inside the del3d source tree):
 *   del3d::orient3d / in_sphere / in_sphere_unperturbed  include/del3d/predicates.h:28,52,57
 *   del3d::orient2d / coplanar_orientation (x2) / collinear /
 *     coplanar_in_circle(_unperturbed)                    include/del3d/predicates2.h:27-70
 *   del3d::spatial_sort                                    include/del3d/spatial_sort.h:37
 *   del3d::Delaunay::build / finite_cells / all_cells /
 *     incident_cells / number_of_vertices                  include/del3d/delaunay.h:68-85
 *   meshio::load / weld / drop_non_finite (viewer reader)  viewer/mesh_io.h:26-60
 *
 * Documented difference from the reference: finite_cells() comes back in a
 * canonical order instead of the reference's cell-allocation order.  Each tet
 * is rotated by an even permutation (orientation preserved) so that its
 * smallest point index comes first and the other three follow in the cyclic
 * order that starts with their smallest; tets are then sorted
 * lexicographically.  The SET of tets is identical to the reference's.
 */
#ifndef DEL3D_B200_H
#define DEL3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum d3g_status {
    D3G_OK = 0,
    D3G_ERR_INVALID_ARGUMENT = 1, /* null pointer, negative size, unknown kind   */
    D3G_ERR_INVALID_INPUT = 2,    /* non-finite coordinate or out-of-range index */
    D3G_ERR_OOM = 3,              /* a device allocation failed                  */
    D3G_ERR_EXACT_CAPACITY = 4,   /* exponent span too wide for the exact stage  */
    D3G_ERR_CAVITY_CAPACITY = 5,  /* a conflict region outgrew its scratch space */
    D3G_ERR_WALK_LIMIT = 6,       /* a point-location walk hit its step limit    */
    D3G_ERR_ROUND_LIMIT = 7,      /* insertion rounds hit their limit            */
    D3G_ERR_CUDA = 8,             /* a CUDA runtime call failed                  */
    D3G_ERR_INTERNAL = 9,         /* an internal invariant did not hold          */
    D3G_ERR_NO_DEVICE = 10,       /* no CUDA device could be used                */
    D3G_ERR_NOT_READY = 11        /* d3g_server_wait: not complete within timeout */
} d3g_status;

/* Human-readable name of a status; never NULL. */
const char* d3g_status_string(int status);
/* Detail of the last error on the calling thread ("" if none). */
const char* d3g_last_error(void);

/* The library keeps device memory it frees for later calls (builds allocate
 * gigabytes per call): blocks of 1 MiB and more in its own cache, which hands a
 * block to a later request of about its size on any stream (idle blocks up to
 * half the device memory), the rest in the current device's stream-ordered
 * pool.  Host result arrays come from a cache of pinned blocks (freed results'
 * blocks serve later ones, up to 16 GiB).  This returns all of them to the
 * CUDA driver; it synchronises the device. */
int d3g_release_cached_memory(void);

/* ---- predicates ------------------------------------------------------------
 * Batch evaluation over index tuples into a point table `pts` (3 doubles per
 * point, x y z).  `idx` holds k int32 indices per query, k given by the kind;
 * `sign_out` receives one int8 per query: -1, 0, +1 (collinear: 1 true, 0 false).
 * Signs equal the reference functions named below on the same points, with
 * "the same point" meaning the same index (the reference compares pointers).
 */
typedef enum d3g_predicate {
    D3G_ORIENT3D = 0,                      /* k=4  del3d::orient3d(a,b,c,d)                */
    D3G_IN_SPHERE = 1,                     /* k=5  del3d::in_sphere(a,b,c,d,e)             */
    D3G_IN_SPHERE_UNPERTURBED = 2,         /* k=5  del3d::in_sphere_unperturbed            */
    D3G_COPLANAR_ORIENTATION3 = 3,         /* k=3  del3d::coplanar_orientation(p,q,r)      */
    D3G_COPLANAR_ORIENTATION4 = 4,         /* k=4  del3d::coplanar_orientation(p,q,r,s)    */
    D3G_COPLANAR_IN_CIRCLE = 5,            /* k=4  del3d::coplanar_in_circle(p0,p1,p2,p)   */
    D3G_COPLANAR_IN_CIRCLE_UNPERTURBED = 6,/* k=4  del3d::coplanar_in_circle_unperturbed   */
    D3G_COLLINEAR = 7                      /* k=3  del3d::collinear(p,q,r)                 */
} d3g_predicate;

/* Queries per kind (k above); 0 for an unknown kind. */
int d3g_predicate_arity(int kind);

typedef struct d3g_predicate_stats {
    int64_t n_queries;     /* queries evaluated                              */
    int64_t n_exact;       /* of which the filter left uncertain (exact stage) */
} d3g_predicate_stats;

/* Host pointers; synchronous.  `stats` may be NULL. */
int d3g_predicates(const double* pts, int64_t n_pts, const int32_t* idx, int64_t n_queries,
                   int kind, int8_t* sign_out, d3g_predicate_stats* stats);

/* Device pointers on `stream`.  Reads the status back, so it synchronises
 * `stream` before returning.  `stats` (host pointer) may be NULL. */
int d3g_predicates_device(const double* d_pts, int64_t n_pts, const int32_t* d_idx,
                          int64_t n_queries, int kind, int8_t* d_sign_out, void* stream,
                          d3g_predicate_stats* stats);

/* The same as d3g_predicates_device, for callers that cannot allocate device
 * memory (a framework whose caching allocator has reserved the device, or a path
 * where an allocation's implicit synchronisation or failure is unacceptable).
 * No counterpart in the reference, which has no device code.
 *   - Allocates nothing: the exact-stage queue and counters live in a fixed
 *     array of this library (8 MiB per device that loads it, held until exit).
 *   - At most D3G_NOALLOC_MAX_QUERIES queries per call; more returns
 *     D3G_ERR_INVALID_ARGUMENT without touching the device.
 *   - The first call on a device looks up the array's device address; make that
 *     first call before any stream capture.  A cudaDeviceReset gives the device a
 *     new context, where the first call looks the address up again (and so
 *     should come before any capture there too).
 *   - Every call reuses the same array (the counters are cleared per call):
 *     calls that overlap on the GPU, on any streams, race with each other.
 * Synchronises `stream`. */
#define D3G_NOALLOC_MAX_QUERIES (1 << 20)
int d3g_predicates_noalloc_device(const double* d_pts, int64_t n_pts, const int32_t* d_idx,
                                  int64_t n_queries, int kind, int8_t* d_sign_out, void* stream,
                                  d3g_predicate_stats* stats);

/* del3d::orient2d(px,py,qx,qy,rx,ry) over `six` (6 doubles per query); host pointers. */
int d3g_orient2d(const double* six, int64_t n_queries, int8_t* sign_out);

/* ---- circumcentres ---------------------------------------------------------
 * lazy = 0: del3d::circumcenter (reference include/del3d/delaunay.h:29,
 * src/triangulation.cpp:805-852); lazy = 1: del3d::circumcenter_lazy
 * (delaunay.h:48, triangulation.cpp:873-930).  `tets`: 4 indices into `pts` per
 * tet; `out`: x y z per tet.  A coplanar tet gives its first vertex, as in the
 * reference.  The lazy form is the reference's value bit for bit where its
 * interval pass decides a coordinate; a coordinate that needs the exact
 * fallback, and every coordinate of the exact form, is the reference's value
 * within 4 ulp of the quotient nx/den plus 1 ulp of the result (bit-identical
 * whenever the reference's expansion sum is the nearest double).
 * stats->n_exact: tets that needed exact arithmetic (all of them for lazy = 0).
 * Returns D3G_ERR_INVALID_INPUT for an index out of range. */
int d3g_circumcenters(const double* pts, int64_t n_pts, const int32_t* tets, int64_t n_tets, int lazy,
                      double* out, d3g_predicate_stats* stats);
/* Device pointers on `stream`; synchronises `stream`. */
int d3g_circumcenters_device(const double* d_pts, int64_t n_pts, const int32_t* d_tets, int64_t n_tets,
                             int lazy, double* d_out, void* stream, d3g_predicate_stats* stats);

/* ---- spatial sort ----------------------------------------------------------
 * The reference insertion order (rand48 shuffle, multiscale split, Hilbert
 * median splits), bit for bit: order[k] = index of the k-th point. */
int d3g_spatial_sort(const double* xyz, int64_t n, int32_t* order);
int d3g_spatial_sort_device(const double* d_xyz, int64_t n, int32_t* d_order, void* stream);
/* The first stage alone: the rand48 Fisher-Yates shuffle of 0..n-1
 * (reference src/rand48.h:146-153 with the engine seeded to 1). */
int d3g_shuffle_device(int64_t n, int32_t* d_order, void* stream);

/* ---- the build ---------------------------------------------------------------
 * A d3g_result holds one triangulation on the host.  It owns its arrays; free
 * it with d3g_result_free.  Fields are valid until then. */
typedef struct d3g_options {
    int32_t want_all_cells;  /* also produce all_cells                           */
    int32_t want_incident;   /* also produce incident_cells                      */
    int32_t chunk;           /* > 0: points per worker chunk; < 0: -alpha, one   */
                             /* worker per alpha earlier points; 0 = default    */
    int32_t max_rounds;      /* 0 = default                                      */
    int32_t timing;          /* time each insertion kernel with CUDA events      */
    int32_t alpha_small;     /* > 0: densest worker pool (one per alpha_small    */
                             /* earlier points) while a round's pool stays below */
                             /* one latency wave of the GPU; 0 = never denser;   */
                             /* default 24                                       */
    int32_t split;           /* grow the worker pool within a level as points go */
                             /* in (0 = off)                                     */
    int32_t lanes;           /* lanes per worker in the lockstep insertion       */
                             /* kernels: 32, 16, 8 or 4; 0 = 32 (default)        */
    int32_t schedule;        /* 0 = asynchronous insertion with rounds for what  */
                             /* it leaves (default); 1 = lockstep rounds only    */
    /* Capacities and step limits (0 = the built-in value).  Lowering one makes
     * its failure path reachable on small input, for testing: the build then
     * stops with the status named, returns no cells, and the device stays
     * usable for the next call. */
    int32_t tet_capacity;    /* tet-table slots per vertex (built-in 8);         */
                             /* too few: D3G_ERR_OOM ("tet table full")          */
    int32_t walk_limit;      /* steps of a point-location walk (built-in 2^20    */
                             /* in the rounds, 2^14 per asynchronous attempt);   */
                             /* exceeded: D3G_ERR_WALK_LIMIT                     */
    int32_t cavity_capacity; /* conflict-region tets a worker may hold: caps the */
                             /* normal scratch (256) and the big-round scratch   */
                             /* (16384), boundary facets at twice it; exceeded   */
                             /* in a big round: D3G_ERR_CAVITY_CAPACITY          */
    int32_t validate;        /* debug: after each BRIO level, check the device   */
                             /* tet table's invariants (the reference's          */
                             /* Tds::validate(), src/tds.h:483-530): distinct    */
                             /* vertices, live neighbours pointing back through  */
                             /* the same facet, no lock left, every vertex's     */
                             /* cached tet containing it; the first violation    */
                             /* ends the build with D3G_ERR_INTERNAL and its     */
                             /* description in d3g_last_error()                  */
    int32_t level_growth;    /* points of a BRIO level over the points before it */
    /* in the build's own insertion order: 8 (the reference's multiscale ratio  */
    /* 1/8) or 2-7 (more, shorter levels); 0 = default: 4 when a set's          */
    /* coordinates make the filters exact (lattices, coarse grids) or the build */
    /* has fewer than 65536 points, else 8.                                     */
    /* Input with repeated points is always ordered with 8, since the           */
    /* reference's order decides which copy keeps its index.  The cells do not */
    /* depend on it.                                                            */
} d3g_options;

/* What a build did (filled by d3g_build and d3g_build_device). */
typedef struct d3g_build_stats {
    int32_t rounds;          /* insertion rounds                                 */
    int64_t attempts;        /* insertion attempts, winners and losers           */
    int64_t region_tets;     /* sum over insertions of conflict-region tets      */
    int64_t boundary_facets; /* sum over insertions of region boundary facets    */
    double ms_order;         /* spatial order + duplicate grouping               */
    double ms_rounds;        /* insertion rounds                                 */
    double ms_output;        /* canonical output                                 */
    /* with d3g_options.timing: device time of each insertion kernel, summed */
    double ms_cavity, ms_check, ms_restar;
    int64_t launches_cavity;
    int64_t walk_steps;      /* with timing: point-location steps over all attempts  */
    int64_t bfs_steps;       /* with timing: conflict-region growth steps (8 tets each) */
    double ms_async;         /* with timing: device time of the asynchronous passes  */
    int64_t launches_async;  /* asynchronous passes: per level the fast variant,    */
                             /* then the full one over what it deferred or left,    */
                             /* repeated while it inserts                           */
    int64_t async_inserted;  /* points the asynchronous passes inserted              */
    /* Conflict tests (in_sphere, or orient3d against a hull facet) the insertion
     * kernels evaluated, attempts that gave way included; of these, the ones the
     * floating-point filter could not certify (decided by a set's exact filter
     * value, the exact stage or a tie-break), and the ones whose exact value was
     * zero (decided by the symbolic perturbation or the hull in-circle test). */
    int64_t conflict_tests;
    int64_t uncertain_tests;
    int64_t tie_breaks;
    int64_t max_region_tets;  /* the largest conflict region inserted (tets)         */
    int64_t deferred_points;  /* points the fast asynchronous variant left to the    */
                              /* full one (a test its filters could not decide)     */
} d3g_build_stats;

typedef struct d3g_result {
    int64_t n_points;        /* input size                                       */
    int64_t n_vertices;      /* distinct points (number_of_vertices())           */
    int64_t n_cells;         /* finite tets                                      */
    int32_t* cells;          /* n_cells x 4, canonical order (finite_cells())    */
    int64_t n_all;           /* all tets, infinite ones included                 */
    int32_t* all_cells;      /* n_all x 4, -1 = the infinite vertex, canonical   */
    int64_t* incident_offsets; /* n_points + 1 (CSR of incident_cells())         */
    int32_t* incident;       /* incident_offsets[n_points] finite-cell indices   */
    /* build statistics */
    double device_ms;        /* device time of the build (CUDA events)           */
    d3g_build_stats stats;
} d3g_result;

/* Fills `opts` with the defaults (all outputs on). */
void d3g_options_default(d3g_options* opts);

/* del3d::Delaunay::build over host points (3 doubles per point).  `opts` may be
 * NULL.  On success *out owns the result (free with d3g_result_free); on error
 * *out is left zeroed. */
int d3g_build(const double* xyz, int64_t n, const d3g_options* opts, d3g_result* out);
void d3g_result_free(d3g_result* r);

/* The same build over device-resident points, writing the canonical finite
 * cells into a caller-supplied device array of `cap_cells` x 4 int32 on
 * `stream`.  *n_cells_out receives the cell count (also when it exceeds
 * cap_cells, in which case nothing is written and D3G_ERR_INVALID_ARGUMENT is
 * returned).  `stats` may be NULL.  Synchronises `stream`. */
int d3g_build_device(const double* d_xyz, int64_t n, const d3g_options* opts, int32_t* d_cells,
                     int64_t cap_cells, int64_t* n_cells_out, int64_t* n_vertices_out,
                     void* stream, d3g_build_stats* stats);

/* ---- batched builds ------------------------------------------------------------
 * Many independent point sets in one call (no reference counterpart: the
 * reference builds one set per Delaunay::build call).  Set s is the points
 * [set_offsets[s], set_offsets[s+1]) of `xyz`; set_offsets has n_sets + 1
 * entries starting at 0.  Each set's cells are exactly what d3g_build returns
 * for that set alone (same canonical order, indices local to the set). */
typedef struct d3g_batch_result {
    int32_t n_sets;
    int64_t* cell_offsets;   /* n_sets + 1: set s owns cells [cell_offsets[s], cell_offsets[s+1]) */
    int32_t* cells;          /* cell_offsets[n_sets] x 4                                          */
    int64_t* n_vertices;     /* n_sets: distinct points per set                                  */
    double device_ms;        /* device time of the build (CUDA events)                           */
    d3g_build_stats stats;
} d3g_batch_result;

int d3g_build_batch(const double* xyz, const int64_t* set_offsets, int32_t n_sets, const d3g_options* opts,
                    d3g_batch_result* out);
void d3g_batch_result_free(d3g_batch_result* r);

/* Device-resident points; set_offsets, cell_offsets (n_sets + 1) and n_vertices
 * (n_sets) are host arrays; the cells of all sets go to d_cells (cap_cells x 4).
 * Synchronises `stream`. */
int d3g_build_batch_device(const double* d_xyz, const int64_t* set_offsets, int32_t n_sets,
                           const d3g_options* opts, int32_t* d_cells, int64_t cap_cells,
                           int64_t* cell_offsets, int64_t* n_vertices, void* stream,
                           d3g_build_stats* stats);

/* ---- synthetic inputs (host) -------------------------------------------------
 * Deterministic generators (std::mt19937 with u01 = word * 2^-32, written out). */
void d3g_gen_uniform(int64_t n, uint32_t seed, double lo, double hi, double* xyz);
/* Sphere of radius r (z and angle uniform), coordinates snapped to 1/q (q a power of two). */
void d3g_gen_sphere(int64_t n, uint32_t seed, double r, int32_t q, double* xyz);
/* k Gaussian clusters of standard deviation sigma, centres uniform in [0.1,0.9]^3. */
void d3g_gen_clusters(int64_t n, uint32_t seed, int32_t k, double sigma, double* xyz);
/* The first n points of the integer lattice of side ceil(n^(1/3)), lexicographic. */
void d3g_gen_lattice(int64_t n, double* xyz);

/* ---- serving ----------------------------------------------------------------
 * A request server on one GPU with continuous batching.  No counterpart in the
 * reference (one single-threaded build per call); each request's cells are
 * exactly what d3g_build returns for its points alone.
 *   - `slots` worker threads, each with its own CUDA stream: up to `slots`
 *     batches run on the device at once.
 *   - A free slot takes the request at the head of the queue and, behind it,
 *     requests of a similar size (within a factor 4) while they fit: at most
 *     max_batch_sets requests and max_batch_points points per batch, and the
 *     estimated device memory of all in-flight batches within hbm_budget_bytes
 *     (a request larger than the budget runs alone once nothing else is in
 *     flight).  Requests arriving while batches run are admitted as soon as a
 *     slot and memory free up.
 *   - Points and tets stay on the device for the whole build; each request's
 *     cells are copied to a host buffer of its own.
 * Thread-safe: submit and wait may be called from any threads. */
typedef struct d3g_server d3g_server;

typedef struct d3g_server_options {
    int32_t slots;             /* batches in flight at once (default 4)                       */
    int64_t hbm_budget_bytes;  /* device memory for in-flight batches; 0 = half the free
                                  memory at creation (default 0)                             */
    int32_t max_batch_sets;    /* requests per batch (default 1024)                           */
    int64_t max_batch_points;  /* points per batch (default 8 Mi)                             */
    int32_t device;            /* CUDA device; -1 = the current one (default -1)              */
} d3g_server_options;

typedef struct d3g_request_result {
    int32_t status;            /* D3G_OK or the build's status for this request              */
    int64_t n_points, n_vertices, n_cells;
    int32_t* cells;            /* n_cells x 4 int32, canonical order, indices into the
                                  request's points; free with d3g_request_result_free        */
    double t_submit, t_admit, t_done;  /* seconds since the server was created              */
    int32_t batch_sets;        /* requests in the batch it was built in                      */
} d3g_request_result;

typedef struct d3g_server_stats {
    int64_t submitted, completed, queued, batches, batched_requests;
    int64_t bytes_in_use, peak_bytes_in_use, hbm_budget_bytes;  /* admission estimates */
    int64_t peak_in_flight_requests;
    int32_t slots;
} d3g_server_stats;

void d3g_server_options_default(d3g_server_options* o);
int d3g_server_create(const d3g_server_options* o, d3g_server** out);
/* Queues a request of n points (3 doubles each, host memory; pinned memory
 * copies fastest).  `xyz` is borrowed until the request completes. */
int d3g_server_submit(d3g_server* s, const double* xyz, int64_t n, int64_t* ticket);
/* Waits for request `ticket` (timeout_s < 0: no limit) and hands over its
 * result, once; returns the request's status, or D3G_ERR_NOT_READY on timeout
 * (the ticket stays valid). */
int d3g_server_wait(d3g_server* s, int64_t ticket, double timeout_s, d3g_request_result* out);
void d3g_request_result_free(d3g_request_result* r);
int d3g_server_get_stats(d3g_server* s, d3g_server_stats* out);
/* Completes every queued and in-flight request, then frees the server and any
 * results not collected. */
int d3g_server_destroy(d3g_server* s);

/* The current device's stream-ordered pool: bytes in use (the library's
 * cached blocks included) and the high-water mark since the last reset
 * (reset_high != 0 resets it). */
int d3g_pool_usage(int64_t* used, int64_t* used_high, int reset_high);

/* ---- autotuning -----------------------------------------------------------------
 * Times builds of the given (device-resident) sets under candidate settings of
 * the options that only change speed - schedule, worker density (chunk as
 * -alpha, alpha_small) and lanes per worker - and makes the fastest the default
 * that d3g_options_default returns on this device from then on.  Every setting
 * gives the same cells.  Runs 2 builds per candidate (10 candidates); pass a
 * sample of the workload.  No counterpart in the reference. */
typedef struct d3g_tuning {
    int32_t schedule, chunk, alpha_small, lanes;  /* the chosen option values        */
    double ms;                                   /* its build time on the sample     */
    int32_t candidates;                          /* settings timed                   */
} d3g_tuning;
int d3g_autotune_device(const double* d_xyz, const int64_t* set_offsets, int32_t n_sets, void* stream,
                        d3g_tuning* best);
/* The current device's tuned settings (the built-in defaults if never tuned). */
int d3g_get_tuning(d3g_tuning* out);
/* Forgets the current device's tuning. */
int d3g_reset_tuning(void);

/* ---- measurement aid ------------------------------------------------------------
 * FP64 throughput of the current device with the filters' arithmetic: separate
 * DADD/DMUL operations per second (the filters are built without contraction)
 * and, for comparison, DFMA instructions per second; `iters` steps of 8
 * independent chains per thread.  No counterpart in the reference. */
int d3g_microbench_fp64(int64_t iters, double* addmul_ops_per_s, double* fma_per_s, void* stream);

/* ---- checking a result (host) ---------------------------------------------------
 * The output-side counterpart of the reference's Tds::validate() (src/tds.h:483-530)
 * for all_cells() (infinite vertex = -1; any cell order, any even rotation): every
 * cell has four distinct vertices in [-1, n_points) (n_points <= 0: no upper bound)
 * with at most one infinite; every triangular facet is shared by exactly two cells
 * inducing opposite orientations on it; the Euler characteristic V - E + F - T is 0.
 * Necessary conditions only (closed, consistently oriented, chi 0: a triangulation
 * closed through the infinite vertex meets them, as does any closed oriented
 * 3-manifold complex); no coordinates are read, so a complex flipped throughout or
 * not Delaunay passes.  Returns D3G_OK, or D3G_ERR_INVALID_INPUT with the first
 * violation in d3g_last_error().  No device is needed. */
int d3g_validate_cells(const int32_t* all_cells, int64_t n_cells, int64_t n_points);

/* ---- input readers (host) -------------------------------------------------------
 * The point and mesh formats of the reference's viewer reader (replaces
 * meshio::load / weld / drop_non_finite / supported_formats,
 * viewer/mesh_io.h:26-60): chosen by extension - .obj (Wavefront, polygons as
 * fans, v/vt/vn and negative indices), .off (OFF/COFF/NOFF), .ply (ASCII and
 * binary little-endian), .stl (ASCII and binary, welded), .xyz .txt .pts or no
 * extension ("x y z" per line).  Vertices, faces and error texts equal the
 * reference reader's on the same bytes.  No device is needed. */
typedef struct d3g_mesh {
    double* vertices;       /* n_vertices x 3 (x y z) */
    int32_t* faces;         /* n_faces x 3 vertex indices (empty for a point set) */
    int64_t n_vertices;
    int64_t n_faces;
} d3g_mesh;

/* Loads `path`.  On a reader error returns D3G_ERR_INVALID_INPUT with the
 * reference's text in d3g_last_error(); `out` then holds what was read before
 * the error, as the reference's Mesh does.  Free with d3g_mesh_free. */
int d3g_mesh_load(const char* path, d3g_mesh* out);
/* examples/simple.cpp:17-23: "x y z" triples, whitespace-separated, until the
 * first that does not parse. */
int d3g_read_xyz(const char* path, d3g_mesh* out);
/* In place: merges vertices with equal coordinates (the first kept, faces
 * remapped, faces whose corners merged removed); nothing changes when no two
 * vertices are equal.  A vertex with a NaN coordinate never merges. */
int d3g_mesh_weld(d3g_mesh* m);
/* In place: removes vertices with a non-finite coordinate and every face that
 * touches one; `dropped` (may be NULL) receives how many vertices went. */
int d3g_mesh_drop_non_finite(d3g_mesh* m, int64_t* dropped);
void d3g_mesh_free(d3g_mesh* m);
/* "obj, off, ply, stl, xyz". */
const char* d3g_mesh_supported_formats(void);

/* Many files as point sets for d3g_build_batch: every file is read (as
 * d3g_mesh_load) on `threads` host threads (<= 0: one per core), its faces
 * ignored and its non-finite vertices dropped (the build needs finite input),
 * and the vertices packed back to back into pinned host memory.  A file that
 * fails to read fails the call (D3G_ERR_INVALID_INPUT, "path: text"). */
typedef struct d3g_point_sets {
    double* xyz;            /* 3 doubles per point, set s at [set_offsets[s], set_offsets[s+1]) */
    int64_t* set_offsets;   /* n_sets + 1 */
    int64_t* dropped;       /* per set: non-finite vertices removed */
    int n_sets;
} d3g_point_sets;
int d3g_load_point_sets(const char* const* paths, int n_paths, int threads, d3g_point_sets* out);
void d3g_point_sets_free(d3g_point_sets* s);

#ifdef __cplusplus
}
#endif

#endif /* DEL3D_B200_H */
