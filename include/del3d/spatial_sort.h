// del3d drop-in (del3d_b200): the insertion order of the incremental build.
//
// Same declarations as the reference's include/del3d/spatial_sort.h; the
// implementation (del3d_b200/csrc/shim.cpp) runs the bit-exact device spatial
// sort: rand48 Fisher-Yates shuffle, multiscale 12.5% prefix split while a range
// holds at least 64 points, Hilbert median splits down to 8 points.
#ifndef DEL3D_SPATIAL_SORT_H
#define DEL3D_SPATIAL_SORT_H

#include <cstddef>
#include <vector>

namespace del3d {

struct Point3 { double x, y, z; };

/// Reorders `order` (indices into `points`, normally 0..n-1) into the
/// reference's spatial-sort sequence.  `points` is not modified.  Throws
/// std::runtime_error if the device call fails.
void spatial_sort(const std::vector<Point3>& points, std::vector<int>& order);

} // namespace del3d

#endif // DEL3D_SPATIAL_SORT_H
