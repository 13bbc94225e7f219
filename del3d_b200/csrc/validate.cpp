// Host-side check of a triangulation's cells: the output-side counterpart of
// the reference's Tds::validate() (src/tds.h:483-530), for all_cells() (the
// infinite vertex as -1).  Valid means: every cell has four distinct vertices,
// in range and at most one of them infinite; every triangular facet is shared
// by exactly two cells, which induce opposite orientations on it (the complex
// closes up and is consistently oriented, as the reference keeps it); and the
// Euler characteristic V - E + F - T of the complex is 0.  These are necessary
// conditions only: a triangulation of the points closed through the infinite
// vertex is a 3-sphere and meets them, but so does any closed, consistently
// oriented 3-manifold complex, and no geometry is looked at (a complex whose
// orientation is flipped throughout, or that is not Delaunay, passes).  The
// cells may come in any order and any even rotation.
#include "../../include/del3d_b200.h"

#include <algorithm>
#include <cstdint>
#include <exception>
#include <string>
#include <utility>
#include <vector>

namespace d3g {
void set_error(const std::string& msg);
}

namespace {

struct Facet {
    int32_t a, b, c;   // sorted vertices
    int32_t parity;    // induced orientation relative to the sorted order
    int64_t cell;
    bool operator<(const Facet& o) const {
        if (a != o.a) return a < o.a;
        if (b != o.b) return b < o.b;
        if (c != o.c) return c < o.c;
        return parity < o.parity;
    }
    bool same_triple(const Facet& o) const { return a == o.a && b == o.b && c == o.c; }
};

/// Sorts three values; returns the permutation's parity (0 even, 1 odd).
int sort3(int32_t& x, int32_t& y, int32_t& z) {
    int p = 0;
    if (x > y) std::swap(x, y), p ^= 1;
    if (y > z) std::swap(y, z), p ^= 1;
    if (x > y) std::swap(x, y), p ^= 1;
    return p;
}

int fail(const std::string& msg) {
    d3g::set_error("d3g_validate_cells: " + msg);
    return D3G_ERR_INVALID_INPUT;
}

int validate(const int32_t* t, int64_t n, int64_t n_points) {
    std::vector<Facet> facets;
    facets.reserve(size_t(n) * 4);
    std::vector<std::pair<int32_t, int32_t>> edges;
    edges.reserve(size_t(n) * 6);
    std::vector<int32_t> verts;
    verts.reserve(size_t(n) * 4);
    for (int64_t k = 0; k < n; ++k) {
        const int32_t* v = t + 4 * k;
        int infinite = 0;
        for (int i = 0; i < 4; ++i) {
            if (v[i] < -1 || (n_points > 0 && v[i] >= n_points))
                return fail("cell " + std::to_string(k) + " has vertex " + std::to_string(v[i]) + " out of range");
            infinite += v[i] == -1;
            for (int j = i + 1; j < 4; ++j)
                if (v[i] == v[j])
                    return fail("cell " + std::to_string(k) + " repeats vertex " + std::to_string(v[i]));
            verts.push_back(v[i]);
        }
        if (infinite > 1) return fail("cell " + std::to_string(k) + " has more than one infinite vertex");
        // The boundary of (v0 v1 v2 v3) is the sum over i of (-1)^i times the
        // facet without v_i, in its remaining order.
        for (int i = 0; i < 4; ++i) {
            int32_t f[3];
            for (int j = 0, m = 0; j < 4; ++j)
                if (j != i) f[m++] = v[j];
            const int p = sort3(f[0], f[1], f[2]) ^ (i & 1);
            facets.push_back(Facet{f[0], f[1], f[2], p, k});
        }
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j) edges.emplace_back(std::min(v[i], v[j]), std::max(v[i], v[j]));
    }
    std::sort(facets.begin(), facets.end());
    size_t nf = 0;
    for (size_t i = 0; i < facets.size();) {
        size_t j = i;
        while (j < facets.size() && facets[j].same_triple(facets[i])) ++j;
        const Facet& f = facets[i];
        const std::string name = "facet (" + std::to_string(f.a) + ", " + std::to_string(f.b) + ", " +
                                 std::to_string(f.c) + ")";
        if (j - i != 2)
            return fail(name + " belongs to " + std::to_string(j - i) + " cells (cell " + std::to_string(f.cell) +
                        "), not 2");
        if (facets[i].parity == facets[i + 1].parity)
            return fail(name + ": cells " + std::to_string(facets[i].cell) + " and " +
                        std::to_string(facets[i + 1].cell) + " are not consistently oriented");
        ++nf;
        i = j;
    }
    std::sort(edges.begin(), edges.end());
    const size_t ne = size_t(std::unique(edges.begin(), edges.end()) - edges.begin());
    std::sort(verts.begin(), verts.end());
    const size_t nv = size_t(std::unique(verts.begin(), verts.end()) - verts.begin());
    const int64_t chi = int64_t(nv) - int64_t(ne) + int64_t(nf) - n;
    if (n > 0 && chi != 0)
        return fail("Euler characteristic " + std::to_string(chi) + " (vertices " + std::to_string(nv) + ", edges " +
                    std::to_string(ne) + ", facets " + std::to_string(nf) + ", cells " + std::to_string(n) +
                    "), not 0");
    return D3G_OK;
}

}  // namespace

extern "C" int d3g_validate_cells(const int32_t* cells, int64_t n_cells, int64_t n_points) {
    if (n_cells < 0 || (n_cells > 0 && !cells)) {
        d3g::set_error("d3g_validate_cells: bad argument");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    try {
        return validate(cells, n_cells, n_points);
    } catch (const std::exception& e) {
        d3g::set_error(std::string("d3g_validate_cells: ") + e.what());
        return D3G_ERR_OOM;
    }
}
