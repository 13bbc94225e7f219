// CPU restatement of the reference del3d `Delaunay::build` path.
//
// TEST INFRASTRUCTURE ONLY: the parity tests, smoke() and bench.py's
// cpu_baseline leg use it as a checker.  The product (del3d_b200) never links,
// loads or calls it.
//
// Parity pin: every function here is checked against the reference compiled
// from its own sources (oracle/_ref/libdel3d_ref.so) and against the golden
// hashes held in the reference's own tests (tests/golden/), see
// tests/test_oracle.py.
#ifndef DEL3D_ORACLE_H
#define DEL3D_ORACLE_H

#include <cstdint>

extern "C" {

// Predicates over index tuples into `pts` (3 doubles per point); same layout as
// the reference wrapper: k indices per query, one int8 sign out.
void orc_orient3d(const double* pts, const int32_t* idx, int64_t nq, int8_t* out);
void orc_in_sphere(const double* pts, const int32_t* idx, int64_t nq, int perturbed, int8_t* out);
void orc_orient2d(const double* six, int64_t nq, int8_t* out);
void orc_coplanar_orientation3(const double* pts, const int32_t* idx, int64_t nq, int8_t* out);
void orc_coplanar_orientation4(const double* pts, const int32_t* idx, int64_t nq, int8_t* out);
void orc_coplanar_in_circle(const double* pts, const int32_t* idx, int64_t nq, int perturbed,
                            int8_t* out);
void orc_collinear(const double* pts, const int32_t* idx, int64_t nq, int8_t* out);

// The rand48 Fisher-Yates shuffle of 0..n-1 alone (rand48.h:146-153, seed 1).
void orc_shuffle(int64_t n, int32_t* order);

// The insertion order (spatial_sort.cpp:141-151).
void orc_spatial_sort(const double* xyz, int64_t n, int32_t* order);

// The build.  Returns a handle; cells come out in the canonical order (each tet
// rotated by an even permutation so its smallest index is first and the other
// three follow in their smallest-first cyclic order; tets sorted
// lexicographically).  Returns null on non-finite input.
void* orc_build(const double* xyz, int64_t n);
int64_t orc_build_ncells(void* h);
int64_t orc_build_nall(void* h);
int64_t orc_build_nvertices(void* h);
void orc_build_cells(void* h, int32_t* out);
void orc_build_all(void* h, int32_t* out);
void orc_build_free(void* h);

// Canonicalises tets in place (rotation only; no sorting): even permutation that
// puts the smallest index first, then the remaining triple rotated cyclically so
// that its smallest index leads.
void orc_canonical_rotate(int32_t* tets, int64_t nt);

}  // extern "C"

#endif
