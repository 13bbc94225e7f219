// Drives the del3d C++ interface (include/del3d/*.h, implemented by
// libdel3d_b200.so) the way a caller of the reference does, and writes what it
// got to files for tests/test_dropin_gpu.py to compare with the Python API and
// the reference:
//   dropin_check <n> <seed> <out_dir>
// Points: n uniform in [0,1)^3 from std::mt19937(seed), u01 = word * 2^-32.
#include <del3d/delaunay.h>
#include <del3d/predicates2.h>

#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

template <class T>
static void dump(const std::string& path, const T* data, size_t count) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) std::exit(3);
    if (count) std::fwrite(data, sizeof(T), count, f);
    std::fclose(f);
}

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    const size_t n = std::strtoull(argv[1], nullptr, 10);
    const unsigned seed = unsigned(std::strtoul(argv[2], nullptr, 10));
    const std::string dir = argv[3];
    std::mt19937 g(seed);
    std::vector<del3d::Point3> pts(n);
    for (auto& p : pts) {
        p.x = g() * 0x1p-32;
        p.y = g() * 0x1p-32;
        p.z = g() * 0x1p-32;
    }

    del3d::Delaunay d;
    d.build(pts);
    const auto& cells = d.finite_cells();
    dump(dir + "/cells.i32", cells.data(), cells.size());
    const auto& all = d.all_cells();
    dump(dir + "/all.i32", all.data(), all.size());
    std::vector<int> inc_sizes;
    for (const auto& v : d.incident_cells()) inc_sizes.push_back(int(v.size()));
    dump(dir + "/incident_sizes.i32", inc_sizes.data(), inc_sizes.size());
    const long long nv = (long long)d.number_of_vertices();
    dump(dir + "/nvertices.i64", &nv, 1);

    // Circumcentres and predicates of the first few cells, one call each.
    std::vector<double> cc, ccl;
    std::vector<int> signs;
    for (size_t i = 0; i < cells.size() && i < 64; ++i) {
        const auto& t = cells[i];
        const del3d::Point3 &a = pts[t[0]], &b = pts[t[1]], &c = pts[t[2]], &e = pts[t[3]];
        const del3d::Point3 x = del3d::circumcenter(a, b, c, e);
        const del3d::Point3 y = del3d::circumcenter_lazy(a, b, c, e);
        cc.insert(cc.end(), {x.x, x.y, x.z});
        ccl.insert(ccl.end(), {y.x, y.y, y.z});
        signs.push_back(del3d::orient3d(&a.x, &b.x, &c.x, &e.x));
        // A point of the tet against its own circumsphere: the perturbation decides.
        signs.push_back(del3d::in_sphere(&a.x, &b.x, &c.x, &e.x, &pts[t[0]].x));
        signs.push_back(del3d::in_sphere_unperturbed(&a.x, &b.x, &c.x, &e.x, &pts[(i * 7) % n].x));
    }
    dump(dir + "/cc.f64", cc.data(), cc.size());
    dump(dir + "/ccl.f64", ccl.data(), ccl.size());
    dump(dir + "/signs.i32", signs.data(), signs.size());

    std::vector<int> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = int(i);
    del3d::spatial_sort(pts, order);
    dump(dir + "/order.i32", order.data(), order.size());
    std::printf("ok %zu cells\n", cells.size());
    return 0;
}
