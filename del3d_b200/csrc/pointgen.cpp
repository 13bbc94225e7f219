// Deterministic synthetic point sets for the benchmarks and tests.
//
// The words come from a Mersenne Twister MT19937 (Matsumoto & Nishimura 1998,
// the generator std::mt19937 specifies), and are mapped to doubles as
// u01 = word * 2^-32, the same explicit mapping the reference's test point sets
// use, so a seed gives the same doubles on every platform.
#include "../../include/del3d_b200.h"

#include <cmath>
#include <cstdint>

namespace {

class MT19937 {
public:
    explicit MT19937(uint32_t seed) {
        s_[0] = seed;
        for (int i = 1; i < 624; ++i) s_[i] = 1812433253u * (s_[i - 1] ^ (s_[i - 1] >> 30)) + uint32_t(i);
        i_ = 624;
    }
    uint32_t next() {
        if (i_ >= 624) twist();
        uint32_t y = s_[i_++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9D2C5680u;
        y ^= (y << 15) & 0xEFC60000u;
        y ^= y >> 18;
        return y;
    }
    double u01() { return double(next()) * (1.0 / 4294967296.0); }
    double range(double lo, double hi) { return lo + (hi - lo) * u01(); }

private:
    void twist() {
        for (int k = 0; k < 624; ++k) {
            const uint32_t y = (s_[k] & 0x80000000u) | (s_[(k + 1) % 624] & 0x7FFFFFFFu);
            uint32_t v = s_[(k + 397) % 624] ^ (y >> 1);
            if (y & 1u) v ^= 0x9908B0DFu;
            s_[k] = v;
        }
        i_ = 0;
    }
    uint32_t s_[624];
    int i_;
};

}  // namespace

extern "C" {

void d3g_gen_uniform(int64_t n, uint32_t seed, double lo, double hi, double* xyz) {
    MT19937 g(seed);
    for (int64_t i = 0; i < 3 * n; ++i) xyz[i] = g.range(lo, hi);
}

/// Unit-sphere samples (z uniform in [-1,1), angle uniform), radius `r`, each
/// coordinate snapped to a multiple of 1/q (q a power of two, so exact).
void d3g_gen_sphere(int64_t n, uint32_t seed, double r, int32_t q, double* xyz) {
    MT19937 g(seed);
    const double two_pi = 6.283185307179586;
    for (int64_t i = 0; i < n; ++i) {
        const double z = g.range(-1.0, 1.0);
        const double rr = std::sqrt(1.0 - z * z);
        const double t = two_pi * g.u01();
        const double p[3] = {r * rr * std::cos(t), r * rr * std::sin(t), r * z};
        for (int k = 0; k < 3; ++k)
            xyz[3 * i + k] = q > 0 ? std::floor(p[k] * q + 0.5) / q : p[k];
    }
}

/// `k` Gaussian clusters (centres uniform in [0.1, 0.9]^3, standard deviation
/// `sigma`), points assigned round-robin; normals by the Box-Muller transform.
void d3g_gen_clusters(int64_t n, uint32_t seed, int32_t k, double sigma, double* xyz) {
    MT19937 g(seed);
    double c[64][3];
    if (k < 1) k = 1;
    if (k > 64) k = 64;
    for (int j = 0; j < k; ++j)
        for (int a = 0; a < 3; ++a) c[j][a] = g.range(0.1, 0.9);
    const double two_pi = 6.283185307179586;
    for (int64_t i = 0; i < n; ++i) {
        const int j = int(i % k);
        for (int a = 0; a < 3; ++a) {
            const double u1 = 1.0 - g.u01();     // (0, 1]
            const double u2 = g.u01();
            const double nrm = std::sqrt(-2.0 * std::log(u1)) * std::cos(two_pi * u2);
            xyz[3 * i + a] = c[j][a] + sigma * nrm;
        }
    }
}

/// The first n points of the integer lattice of side ceil(n^(1/3)), in
/// lexicographic (i, j, k) order.
void d3g_gen_lattice(int64_t n, double* xyz) {
    int64_t s = 1;
    while (s * s * s < n) ++s;
    int64_t w = 0;
    for (int64_t i = 0; i < s && w < n; ++i)
        for (int64_t j = 0; j < s && w < n; ++j)
            for (int64_t k = 0; k < s && w < n; ++k, ++w) {
                xyz[3 * w] = double(i);
                xyz[3 * w + 1] = double(j);
                xyz[3 * w + 2] = double(k);
            }
}

}  // extern "C"
