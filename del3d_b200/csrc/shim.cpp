// The reference's C++ interface (include/del3d/delaunay.h, predicates.h,
// predicates2.h, spatial_sort.h) implemented over this library's C ABI, so that
// code written against the reference builds unchanged and runs on the GPU.
//
// Reference functions replaced: Delaunay::build (src/triangulation.cpp:932-968),
// circumcenter / circumcenter_lazy (:805-930), spatial_sort
// (src/spatial_sort.cpp:141-151), the predicates (src/predicates.cpp:125-232,
// src/predicates2.cpp:111-259).  The reference reports no errors; here a failed
// device call throws std::runtime_error instead of returning a wrong answer.
#include "del3d/delaunay.h"
#include "del3d/predicates2.h"
#include "del3d_b200.h"

#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <stdexcept>
#include <string>

namespace del3d {
namespace {

static_assert(sizeof(Point3) == 3 * sizeof(double), "Point3 must be three packed doubles");
static_assert(sizeof(Delaunay::Tet) == 4 * sizeof(int32_t), "Tet must be four packed ints");

void check(int status, const char* where) {
    if (status != D3G_OK)
        throw std::runtime_error(std::string("del3d: ") + where + ": " + d3g_status_string(status) +
                                 " (" + d3g_last_error() + ")");
}

/// One predicate query.  The arguments become a small point table in which an
/// argument passed by the same pointer as an earlier one gets that one's index,
/// so "the same point" keeps the reference's pointer identity (its symbolic
/// perturbation tells points apart by address).
Sign predicate(int kind, std::initializer_list<const double*> args, const char* where) {
    double table[5 * 3];
    const double* seen[5];
    alignas(16) int32_t idx[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int n = 0, k = 0;
    for (const double* p : args) {
        int j = 0;
        while (j < n && seen[j] != p) ++j;
        if (j == n) {
            seen[n] = p;
            table[3 * n] = p[0];
            table[3 * n + 1] = p[1];
            table[3 * n + 2] = p[2];
            ++n;
        }
        idx[k++] = j;
    }
    int8_t out = 0;
    check(d3g_predicates(table, n, idx, 1, kind, &out, nullptr), where);
    return static_cast<Sign>(out);
}

Point3 circumcenter_of(const Point3& a, const Point3& b, const Point3& c, const Point3& d, int lazy) {
    const Point3 pts[4] = {a, b, c, d};
    const int32_t tet[4] = {0, 1, 2, 3};
    double out[3];
    check(d3g_circumcenters(&pts[0].x, 4, tet, 1, lazy, out, nullptr),
          lazy ? "circumcenter_lazy" : "circumcenter");
    return Point3{out[0], out[1], out[2]};
}

}  // namespace

// ---- predicates ----------------------------------------------------------------

Sign orient3d(const double* a, const double* b, const double* c, const double* d) {
    return predicate(D3G_ORIENT3D, {a, b, c, d}, "orient3d");
}

Sign in_sphere(const double* a, const double* b, const double* c, const double* d, const double* e) {
    return predicate(D3G_IN_SPHERE, {a, b, c, d, e}, "in_sphere");
}

Sign in_sphere_unperturbed(const double* a, const double* b, const double* c, const double* d,
                           const double* e) {
    return predicate(D3G_IN_SPHERE_UNPERTURBED, {a, b, c, d, e}, "in_sphere_unperturbed");
}

Sign orient2d(double px, double py, double qx, double qy, double rx, double ry) {
    const double six[6] = {px, py, qx, qy, rx, ry};
    int8_t out = 0;
    check(d3g_orient2d(six, 1, &out), "orient2d");
    return static_cast<Sign>(out);
}

Sign coplanar_orientation(const double* p, const double* q, const double* r) {
    return predicate(D3G_COPLANAR_ORIENTATION3, {p, q, r}, "coplanar_orientation");
}

Sign coplanar_orientation(const double* p, const double* q, const double* r, const double* s) {
    return predicate(D3G_COPLANAR_ORIENTATION4, {p, q, r, s}, "coplanar_orientation");
}

bool collinear(const double* p, const double* q, const double* r) {
    return predicate(D3G_COLLINEAR, {p, q, r}, "collinear") != ZERO;
}

Sign coplanar_in_circle(const double* p0, const double* p1, const double* p2, const double* p) {
    return predicate(D3G_COPLANAR_IN_CIRCLE, {p0, p1, p2, p}, "coplanar_in_circle");
}

Sign coplanar_in_circle_unperturbed(const double* p0, const double* p1, const double* p2,
                                    const double* p) {
    return predicate(D3G_COPLANAR_IN_CIRCLE_UNPERTURBED, {p0, p1, p2, p},
                     "coplanar_in_circle_unperturbed");
}

// Coordinate comparisons only (no arithmetic, nothing to round): the
// reference's definitions, src/predicates2.cpp:158-180.
bool equal(const double* p, const double* q) { return p[0] == q[0] && p[1] == q[1] && p[2] == q[2]; }

CollinearPosition collinear_position(const double* p, const double* q, const double* r) {
    if (equal(q, p)) return CP_SOURCE;
    if (equal(q, r)) return CP_TARGET;
    // Along the line, order on the first coordinate in which p and r differ.
    const int k = (p[0] != r[0]) ? 0 : (p[1] != r[1]) ? 1 : 2;
    const double a = p[k], b = q[k], c = r[k];
    const bool up = a < c;
    if (up ? b < a : b > a) return CP_BEFORE;
    if (up ? b > c : b < c) return CP_AFTER;
    return CP_MIDDLE;
}

// ---- circumcentres -----------------------------------------------------------

Point3 circumcenter(const Point3& p0, const Point3& p1, const Point3& p2, const Point3& p3) {
    return circumcenter_of(p0, p1, p2, p3, 0);
}

Point3 circumcenter_lazy(const Point3& p, const Point3& q, const Point3& r, const Point3& s) {
    return circumcenter_of(p, q, r, s, 1);
}

// ---- spatial sort --------------------------------------------------------------

void spatial_sort(const std::vector<Point3>& points, std::vector<int>& order) {
    const size_t m = order.size();
    if (m < 2) return;
    // The reference permutes the entries of `order` and compares only the
    // coordinates they point at, so sorting the gathered points and mapping
    // the resulting positions back through `order` gives its sequence.
    std::vector<double> xyz(3 * m);
    for (size_t k = 0; k < m; ++k) {
        const Point3& p = points.at(static_cast<size_t>(order[k]));
        xyz[3 * k] = p.x;
        xyz[3 * k + 1] = p.y;
        xyz[3 * k + 2] = p.z;
    }
    std::vector<int32_t> perm(m);
    check(d3g_spatial_sort(xyz.data(), static_cast<int64_t>(m), perm.data()), "spatial_sort");
    std::vector<int> out(m);
    for (size_t k = 0; k < m; ++k) out[k] = order[static_cast<size_t>(perm[k])];
    order.swap(out);
}

// ---- the build -------------------------------------------------------------------

void Delaunay::build(const std::vector<Point3>& points) {
    cells_.clear();
    all_cells_.clear();
    incident_.assign(points.size(), {});
    n_vertices_ = 0;
    if (points.empty()) return;
    d3g_options opts;
    d3g_options_default(&opts);
    opts.want_all_cells = 1;
    opts.want_incident = 1;
    d3g_result r;
    std::memset(&r, 0, sizeof r);
    check(d3g_build(&points[0].x, static_cast<int64_t>(points.size()), &opts, &r), "Delaunay::build");
    struct Release {
        d3g_result* r;
        ~Release() { d3g_result_free(r); }
    } release{&r};
    cells_.resize(static_cast<size_t>(r.n_cells));
    if (r.n_cells) std::memcpy(cells_.data(), r.cells, sizeof(Tet) * static_cast<size_t>(r.n_cells));
    all_cells_.resize(static_cast<size_t>(r.n_all));
    if (r.n_all) std::memcpy(all_cells_.data(), r.all_cells, sizeof(Tet) * static_cast<size_t>(r.n_all));
    if (r.incident_offsets) {
        for (size_t i = 0; i < points.size(); ++i)
            incident_[i].assign(r.incident + r.incident_offsets[i], r.incident + r.incident_offsets[i + 1]);
    }
    n_vertices_ = static_cast<size_t>(r.n_vertices);
}

}  // namespace del3d
