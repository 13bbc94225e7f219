// del3d drop-in (del3d_b200): exact 3D predicates.
//
// Same declarations as the reference's include/del3d/predicates.h.  Each call
// is one query evaluated on the GPU (filter, then exact stage and symbolic
// perturbation); for throughput, batch queries with d3g_predicates()
// (del3d_b200.h).  Points passed by the same pointer are the same point, as in
// the reference.  Throws std::runtime_error if the device call fails.
#ifndef DEL3D_PREDICATES_H
#define DEL3D_PREDICATES_H

namespace del3d {

enum Sign { NEGATIVE = -1, ZERO = 0, POSITIVE = 1 };

/// Sign of the determinant |b-a, c-a, d-a|: POSITIVE when d lies on the
/// positive side of the oriented plane (a, b, c).
Sign orient3d(const double* a, const double* b, const double* c, const double* d);

/// POSITIVE iff e is strictly inside the sphere through a, b, c, d
/// (orient3d(a,b,c,d) must be POSITIVE).  Never ZERO: exact ties are decided by
/// the reference's lexicographic symbolic perturbation.
Sign in_sphere(const double* a, const double* b, const double* c,
               const double* d, const double* e);

/// The raw in-sphere sign: ZERO when the five points are cospherical.
Sign in_sphere_unperturbed(const double* a, const double* b, const double* c,
                           const double* d, const double* e);

} // namespace del3d

#endif // DEL3D_PREDICATES_H
