// The reference viewer's mesh reader interface (viewer/mesh_io.h), implemented
// by libdel3d_b200.so: a program written against it links this library instead
// of compiling viewer/mesh_io.cpp.  The declarations are the reference's, so
// that such code builds unchanged; the implementation is del3d_b200's own
// (del3d_b200/csrc/meshio.cpp) and reads the same vertices and faces, with the
// same error texts, from the same bytes.
#ifndef DEL3D_VIEWER_MESH_IO_H
#define DEL3D_VIEWER_MESH_IO_H

#include <array>
#include <cstddef>
#include <string>
#include <vector>

namespace meshio {

struct Mesh {
    std::vector<std::array<double, 3>> vertices;
    std::vector<std::array<int, 3>>    faces;    // empty for a plain point set
    bool empty() const { return vertices.empty(); }
};

/// Reads `path`, the format chosen by extension: .obj, .off, .ply (ASCII and
/// binary little-endian), .stl (ASCII and binary, welded), and .xyz / .txt /
/// .pts or none for "x y z" lines.  On failure `error` is set and the mesh
/// holds what was read before it.
Mesh load(const std::string& path, std::string& error);

/// Merges vertices with equal coordinates and rewrites the faces to match.
void weld(Mesh& m);

/// Removes vertices with a non-finite coordinate and the faces touching them;
/// returns how many vertices went.
std::size_t drop_non_finite(Mesh& m);

/// The readable formats as a list for display.
const char* supported_formats();

} // namespace meshio

#endif // DEL3D_VIEWER_MESH_IO_H
