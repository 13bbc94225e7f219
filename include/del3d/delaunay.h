// del3d drop-in (del3d_b200): 3D Delaunay triangulation built on a B200.
//
// Same declarations as the reference's include/del3d/delaunay.h, so code
// written against the reference compiles unchanged and links against
// libdel3d_b200.so instead.  The implementation (del3d_b200/csrc/shim.cpp)
// calls the library's C ABI (del3d_b200.h); every computation runs on the GPU.
//
// One documented difference: finite_cells() and all_cells() come back in a
// canonical order - each tet rotated by an even permutation so that its
// smallest index leads and the other three follow in smallest-first cyclic
// order, tets sorted lexicographically - instead of the reference's
// cell-allocation order.  The set of tets is the reference's, bit for bit, and
// the order is the same on every run.  Errors (no device, out of memory,
// non-finite input) throw std::runtime_error; the reference has no error channel.
#ifndef DEL3D_DELAUNAY_H
#define DEL3D_DELAUNAY_H

#include "del3d/spatial_sort.h"   // Point3

#include <array>
#include <cstddef>
#include <vector>

namespace del3d {

/// Circumcentre of the tetrahedron (p0, p1, p2, p3): numerator and denominator
/// exact, each rounded once, then one double quotient.  Returns p0 when the
/// four points are coplanar.
Point3 circumcenter(const Point3& p0, const Point3& p1,
                    const Point3& p2, const Point3& p3);

/// The circumcentre as the reference's lazy evaluation produces it: an
/// upward-rounded interval evaluation whose midpoint is taken per coordinate
/// when accurate to 1e-5 relative, else the exact value above.
Point3 circumcenter_lazy(const Point3& p, const Point3& q,
                         const Point3& r, const Point3& s);

class Delaunay {
public:
    /// A finite tetrahedron: four indices into the points given to build().
    using Tet = std::array<int, 4>;

    /// Builds the triangulation on the GPU.  Points equal to an earlier point
    /// are ignored (the copy last in spatial-sort order represents them).
    void build(const std::vector<Point3>& points);

    /// The finite tetrahedra, canonical order.
    const std::vector<Tet>& finite_cells() const { return cells_; }

    /// Every tetrahedron, infinite ones included (-1 = the infinite vertex),
    /// canonical order.
    const std::vector<Tet>& all_cells() const { return all_cells_; }

    /// Per input point, the ascending indices into finite_cells() of its
    /// tetrahedra; empty for a point that duplicated another.
    const std::vector<std::vector<int>>& incident_cells() const { return incident_; }

    /// Distinct vertices inserted (duplicates excluded).
    std::size_t number_of_vertices() const { return n_vertices_; }

private:
    std::vector<Tet>              cells_;
    std::vector<Tet>              all_cells_;
    std::vector<std::vector<int>> incident_;
    std::size_t                   n_vertices_ = 0;
};

} // namespace del3d

#endif // DEL3D_DELAUNAY_H
