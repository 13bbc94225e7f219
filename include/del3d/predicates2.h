// del3d drop-in (del3d_b200): lower-dimensional predicates.
//
// Same declarations as the reference's include/del3d/predicates2.h.  The sign
// predicates run on the GPU one query per call (batch them with
// d3g_predicates() for throughput); `equal` and `collinear_position` compare
// coordinates only.  Throws std::runtime_error if a device call fails.
#ifndef DEL3D_PREDICATES2_H
#define DEL3D_PREDICATES2_H

#include "del3d/predicates.h"

namespace del3d {

/// Sign of |q-p, r-p| in the plane.
Sign orient2d(double px, double py, double qx, double qy, double rx, double ry);

/// Orientation of three coplanar points in the first of the xy, yz, xz
/// projections where they are not collinear (they must not be collinear).
Sign coplanar_orientation(const double* p, const double* q, const double* r);

/// Orientation of s against the directed line (p, q), measured in the
/// projection that the triple (p, q, r) selects, so that its sign compares
/// with coplanar_orientation(p, q, r).
Sign coplanar_orientation(const double* p, const double* q,
                          const double* r, const double* s);

/// True iff p, q, r are exactly collinear.
bool collinear(const double* p, const double* q, const double* r);

/// True iff p and q have equal coordinates.
bool equal(const double* p, const double* q);

enum CollinearPosition { CP_BEFORE, CP_SOURCE, CP_MIDDLE, CP_TARGET, CP_AFTER };

/// Where q lies on the line from p to r (the three collinear).
CollinearPosition collinear_position(const double* p, const double* q, const double* r);

/// POSITIVE iff p is strictly inside the circle through the coplanar points
/// p0, p1, p2 (coplanar_orientation(p0,p1,p2) must not be ZERO).  Never ZERO:
/// exact ties are decided by the reference's symbolic perturbation.
Sign coplanar_in_circle(const double* p0, const double* p1,
                        const double* p2, const double* p);

/// The raw in-circle sign: ZERO when the four points are cocircular.
Sign coplanar_in_circle_unperturbed(const double* p0, const double* p1,
                                    const double* p2, const double* p);

} // namespace del3d

#endif // DEL3D_PREDICATES2_H
