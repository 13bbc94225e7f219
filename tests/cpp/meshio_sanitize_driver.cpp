// Loads every file named on the command line through the reader's C entry
// points (load, weld, drop_non_finite, read_xyz, then all of them as point
// sets on 4 threads); built with sanitizers by tests/test_meshio_sanitizers.py.
// The library-side hooks the reader calls are stubbed: no CUDA is involved.
#include "del3d_b200.h"

#include <cstdio>
#include <cstdlib>
#include <string>

namespace d3g {
void set_error(const std::string&) {}
void* host_result_alloc(size_t b) { return std::malloc(b); }
void host_result_free(void* p) { std::free(p); }
}  // namespace d3g

int main(int argc, char** argv) {
    long total = 0;
    for (int i = 1; i < argc; ++i) {
        d3g_mesh m{};
        const int st = d3g_mesh_load(argv[i], &m);
        if (st == D3G_OK || st == D3G_ERR_INVALID_INPUT) {
            d3g_mesh_weld(&m);
            int64_t dropped = 0;
            d3g_mesh_drop_non_finite(&m, &dropped);
        }
        total += m.n_vertices + m.n_faces;
        d3g_mesh_free(&m);
        d3g_mesh r{};
        d3g_read_xyz(argv[i], &r);
        d3g_mesh_free(&r);
    }
    d3g_point_sets ps{};
    d3g_load_point_sets(const_cast<const char* const*>(argv + 1), argc - 1, 4, &ps);
    d3g_point_sets_free(&ps);
    std::printf("ok %ld\n", total);
    return 0;
}
