// C-ABI wrapper around the reference del3d library, compiled together with the
// reference's own sources (see oracle/Makefile) into oracle/_ref/libdel3d_ref.so.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product links or loads this file:
// it exists so that the parity tests, the CPU baseline leg of bench.py and
// `bench.py --impl reference` can call the real reference implementation
// through plain pointers.
//
// Three groups of entry points:
//   * ref_*    - the reference library itself (include/del3d/*.h), unmodified;
//   * exact_*  - the reference's independent integer oracle (tests/exact.h);
//   * ps_*     - the reference's test point-set generators (tests/pointsets.h),
//                so golden inputs are produced by the reference's own code.
#include "del3d/delaunay.h"
#include "del3d/predicates.h"
#include "del3d/predicates2.h"
#include "del3d/spatial_sort.h"

#include "exact.h"
#include "pointsets.h"

#include <cstdint>
#include <cstring>
#include <vector>

namespace {

inline const double* P(const double* pts, int32_t i) { return pts + 3 * int64_t(i); }

struct BuildResult {
    std::vector<del3d::Delaunay::Tet> cells;
    std::vector<del3d::Delaunay::Tet> all;
    std::vector<std::vector<int>> incident;
    int64_t n_vertices = 0;
};

std::vector<del3d::Point3> to_points(const double* xyz, int64_t n) {
    std::vector<del3d::Point3> pts(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) pts[i] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    return pts;
}

int64_t copy_pts(const std::vector<pointsets::Pt>& v, double* out) {
    if (out)
        for (size_t i = 0; i < v.size(); ++i)
            for (int k = 0; k < 3; ++k) out[3 * i + k] = v[i][k];
    return int64_t(v.size());
}

}  // namespace

extern "C" {

// ---- predicates: the reference library ------------------------------------
// Query layout: `idx` holds k point indices per query (k = 4 for orient3d,
// 5 for in_sphere, 3/4 for the coplanar family); `out` receives one sign.

void ref_orient3d(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 4 * q;
        out[q] = int8_t(del3d::orient3d(P(pts, t[0]), P(pts, t[1]), P(pts, t[2]), P(pts, t[3])));
    }
}

void ref_in_sphere(const double* pts, const int32_t* idx, int64_t nq, int perturbed, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 5 * q;
        const double *a = P(pts, t[0]), *b = P(pts, t[1]), *c = P(pts, t[2]), *d = P(pts, t[3]),
                     *e = P(pts, t[4]);
        out[q] = int8_t(perturbed ? del3d::in_sphere(a, b, c, d, e)
                                  : del3d::in_sphere_unperturbed(a, b, c, d, e));
    }
}

void ref_orient2d(const double* six, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const double* s = six + 6 * q;
        out[q] = int8_t(del3d::orient2d(s[0], s[1], s[2], s[3], s[4], s[5]));
    }
}

void ref_coplanar_orientation3(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 3 * q;
        out[q] = int8_t(del3d::coplanar_orientation(P(pts, t[0]), P(pts, t[1]), P(pts, t[2])));
    }
}

void ref_coplanar_orientation4(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 4 * q;
        out[q] = int8_t(del3d::coplanar_orientation(P(pts, t[0]), P(pts, t[1]), P(pts, t[2]),
                                                    P(pts, t[3])));
    }
}

void ref_coplanar_in_circle(const double* pts, const int32_t* idx, int64_t nq, int perturbed,
                            int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 4 * q;
        const double *a = P(pts, t[0]), *b = P(pts, t[1]), *c = P(pts, t[2]), *d = P(pts, t[3]);
        out[q] = int8_t(perturbed ? del3d::coplanar_in_circle(a, b, c, d)
                                  : del3d::coplanar_in_circle_unperturbed(a, b, c, d));
    }
}

void ref_collinear(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 3 * q;
        out[q] = int8_t(del3d::collinear(P(pts, t[0]), P(pts, t[1]), P(pts, t[2])) ? 1 : 0);
    }
}

// ---- predicates: the reference's integer oracle (tests/exact.h) ------------

void exact_orient3d(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 4 * q;
        out[q] = int8_t(exact::orient3d(P(pts, t[0]), P(pts, t[1]), P(pts, t[2]), P(pts, t[3])));
    }
}

void exact_in_sphere(const double* pts, const int32_t* idx, int64_t nq, int perturbed, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 5 * q;
        const double *a = P(pts, t[0]), *b = P(pts, t[1]), *c = P(pts, t[2]), *d = P(pts, t[3]),
                     *e = P(pts, t[4]);
        out[q] = int8_t(perturbed ? exact::in_sphere(a, b, c, d, e)
                                  : exact::in_sphere_raw(a, b, c, d, e));
    }
}

void exact_coplanar_in_circle(const double* pts, const int32_t* idx, int64_t nq, int perturbed,
                              int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 4 * q;
        const double *a = P(pts, t[0]), *b = P(pts, t[1]), *c = P(pts, t[2]), *d = P(pts, t[3]);
        out[q] = int8_t(perturbed ? exact::coplanar_in_circle(a, b, c, d)
                                  : exact::coplanar_in_circle_raw(a, b, c, d));
    }
}

void exact_coplanar_orientation3(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 3 * q;
        out[q] = int8_t(exact::coplanar_orientation(P(pts, t[0]), P(pts, t[1]), P(pts, t[2])));
    }
}

void exact_coplanar_orientation4(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 4 * q;
        out[q] = int8_t(exact::coplanar_orientation(P(pts, t[0]), P(pts, t[1]), P(pts, t[2]),
                                                    P(pts, t[3])));
    }
}

void exact_collinear(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 3 * q;
        out[q] = int8_t(exact::collinear(P(pts, t[0]), P(pts, t[1]), P(pts, t[2])) ? 1 : 0);
    }
}

// ---- spatial sort ----------------------------------------------------------

void ref_spatial_sort(const double* xyz, int64_t n, int32_t* order) {
    const std::vector<del3d::Point3> pts = to_points(xyz, n);
    std::vector<int> o(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) o[i] = int(i);
    del3d::spatial_sort(pts, o);
    for (int64_t i = 0; i < n; ++i) order[i] = o[i];
}

// ---- the build ---------------------------------------------------------------

void* ref_build(const double* xyz, int64_t n) {
    const std::vector<del3d::Point3> pts = to_points(xyz, n);
    del3d::Delaunay d;
    d.build(pts);
    BuildResult* r = new BuildResult;
    r->cells = d.finite_cells();
    r->all = d.all_cells();
    r->incident = d.incident_cells();
    r->n_vertices = int64_t(d.number_of_vertices());
    return r;
}

int64_t ref_build_ncells(void* h) { return int64_t(static_cast<BuildResult*>(h)->cells.size()); }
int64_t ref_build_nall(void* h) { return int64_t(static_cast<BuildResult*>(h)->all.size()); }
int64_t ref_build_nvertices(void* h) { return static_cast<BuildResult*>(h)->n_vertices; }

void ref_build_cells(void* h, int32_t* out) {
    const auto& c = static_cast<BuildResult*>(h)->cells;
    for (size_t i = 0; i < c.size(); ++i)
        for (int k = 0; k < 4; ++k) out[4 * i + k] = c[i][k];
}

void ref_build_all(void* h, int32_t* out) {
    const auto& c = static_cast<BuildResult*>(h)->all;
    for (size_t i = 0; i < c.size(); ++i)
        for (int k = 0; k < 4; ++k) out[4 * i + k] = c[i][k];
}

/// CSR form of incident_cells(): offsets[n+1], then data[offsets[n]].
int64_t ref_build_incident(void* h, int64_t* offsets, int32_t* data) {
    const auto& inc = static_cast<BuildResult*>(h)->incident;
    int64_t k = 0;
    for (size_t i = 0; i < inc.size(); ++i) {
        if (offsets) offsets[i] = k;
        for (int c : inc[i]) {
            if (data) data[k] = c;
            ++k;
        }
    }
    if (offsets) offsets[inc.size()] = k;
    return k;
}

void ref_build_free(void* h) { delete static_cast<BuildResult*>(h); }

/// Times one build of n points: returns seconds of wall time around build().
double ref_build_time(const double* xyz, int64_t n, int64_t* ncells_out);

// ---- circumcentres -----------------------------------------------------------

void ref_circumcenter(const double* pts, const int32_t* tets, int64_t nt, int lazy, double* out) {
    for (int64_t t = 0; t < nt; ++t) {
        const int32_t* q = tets + 4 * t;
        const double *a = P(pts, q[0]), *b = P(pts, q[1]), *c = P(pts, q[2]), *d = P(pts, q[3]);
        const del3d::Point3 A{a[0], a[1], a[2]}, B{b[0], b[1], b[2]}, C{c[0], c[1], c[2]},
            D{d[0], d[1], d[2]};
        const del3d::Point3 r = lazy ? del3d::circumcenter_lazy(A, B, C, D)
                                     : del3d::circumcenter(A, B, C, D);
        out[3 * t] = r.x;
        out[3 * t + 1] = r.y;
        out[3 * t + 2] = r.z;
    }
}

// ---- the reference's test point sets (tests/pointsets.h) ---------------------
// Each returns the number of points; `out` (3 doubles per point) may be null to
// query the size first.

int64_t ps_cylinder(int64_t n, int q, unsigned seed, double* out) {
    return copy_pts(pointsets::cylinder(size_t(n), q, seed), out);
}
int64_t ps_sphere(int64_t n, int q, unsigned seed, double* out) {
    return copy_pts(pointsets::sphere(size_t(n), q, seed), out);
}
int64_t ps_torus(int64_t n, int q, unsigned seed, double* out) {
    return copy_pts(pointsets::torus(size_t(n), q, seed), out);
}
int64_t ps_box_shell(int m, double* out) { return copy_pts(pointsets::box_shell(m), out); }
int64_t ps_lattice(int nx, int ny, int nz, double* out) {
    return copy_pts(pointsets::lattice(nx, ny, nz), out);
}
int64_t ps_random_cube(int64_t n, unsigned seed, double* out) {
    return copy_pts(pointsets::random_cube(size_t(n), seed), out);
}

/// pointsets::Rng(seed).below(m), drawn `count` times: the index stream the
/// reference's predicate tests use to pick 5-tuples.
void ps_rng_below(unsigned seed, int64_t m, int64_t count, int64_t* out) {
    pointsets::Rng rng(seed);
    for (int64_t i = 0; i < count; ++i) out[i] = int64_t(rng.below(size_t(m)));
}

}  // extern "C"

#include <chrono>

extern "C" double ref_build_time(const double* xyz, int64_t n, int64_t* ncells_out) {
    const std::vector<del3d::Point3> pts = to_points(xyz, n);
    del3d::Delaunay d;
    const auto t0 = std::chrono::steady_clock::now();
    d.build(pts);
    const auto t1 = std::chrono::steady_clock::now();
    if (ncells_out) *ncells_out = int64_t(d.finite_cells().size());
    return std::chrono::duration<double>(t1 - t0).count();
}
