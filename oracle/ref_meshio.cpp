// TEST INFRASTRUCTURE ONLY.  A C wrapper around the reference viewer's mesh
// reader (viewer/mesh_io.h, compiled from viewer/mesh_io.cpp where it lies by
// oracle/Makefile into oracle/_ref/libmeshio_ref.so), so that the tests can
// compare del3d_b200's readers with it on the same files.
#include "mesh_io.h"

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>

extern "C" {

struct RefMesh {
    double* v;       // nv x 3
    int32_t* f;      // nf x 3
    int64_t nv, nf;
    char err[512];
};

static void to_c(const meshio::Mesh& m, RefMesh* out) {
    out->nv = int64_t(m.vertices.size());
    out->nf = int64_t(m.faces.size());
    out->v = static_cast<double*>(std::malloc((m.vertices.size() * 3 + 1) * sizeof(double)));
    out->f = static_cast<int32_t*>(std::malloc((m.faces.size() * 3 + 1) * sizeof(int32_t)));
    for (size_t i = 0; i < m.vertices.size(); ++i)
        for (int k = 0; k < 3; ++k) out->v[3 * i + k] = m.vertices[i][k];
    for (size_t i = 0; i < m.faces.size(); ++i)
        for (int k = 0; k < 3; ++k) out->f[3 * i + k] = m.faces[i][k];
}

static meshio::Mesh from_arrays(const double* v, int64_t nv, const int32_t* f, int64_t nf) {
    meshio::Mesh m;
    m.vertices.resize(size_t(nv));
    m.faces.resize(size_t(nf));
    for (int64_t i = 0; i < nv; ++i)
        for (int k = 0; k < 3; ++k) m.vertices[size_t(i)][k] = v[3 * i + k];
    for (int64_t i = 0; i < nf; ++i)
        for (int k = 0; k < 3; ++k) m.faces[size_t(i)][k] = f[3 * i + k];
    return m;
}

void ref_mesh_free(RefMesh* m) {
    std::free(m->v);
    std::free(m->f);
    m->v = nullptr;
    m->f = nullptr;
    m->nv = m->nf = 0;
}

static thread_local std::string g_err;

/// meshio::load; returns 1 when it set an error (full text from
/// ref_mesh_error, the first 511 bytes also in out->err), 2 when it threw (the
/// reference aborts a program on such a file, e.g. a count it cannot reserve).
int ref_mesh_load(const char* path, RefMesh* out) {
    int rc = 0;
    meshio::Mesh m;
    try {
        g_err.clear();
        m = meshio::load(path, g_err);
        rc = g_err.empty() ? 0 : 1;
    } catch (const std::exception& e) {
        g_err = std::string("threw: ") + e.what();
        rc = 2;
    }
    to_c(m, out);
    std::strncpy(out->err, g_err.c_str(), sizeof out->err - 1);
    out->err[sizeof out->err - 1] = '\0';
    return rc;
}

const char* ref_mesh_error() { return g_err.c_str(); }

/// meshio::weld of the given arrays, result in `out`.
void ref_mesh_weld(const double* v, int64_t nv, const int32_t* f, int64_t nf, RefMesh* out) {
    meshio::Mesh m = from_arrays(v, nv, f, nf);
    meshio::weld(m);
    to_c(m, out);
}

/// meshio::drop_non_finite of the given arrays, result in `out`; returns the count.
int64_t ref_mesh_drop_non_finite(const double* v, int64_t nv, const int32_t* f, int64_t nf, RefMesh* out) {
    meshio::Mesh m = from_arrays(v, nv, f, nf);
    const size_t d = meshio::drop_non_finite(m);
    to_c(m, out);
    return int64_t(d);
}

const char* ref_mesh_formats() { return meshio::supported_formats(); }

}  // extern "C"
