// Exact integers wider than the exact stage's 16 limbs, for the rare predicate
// calls whose coordinates span more than about 200 binades.
//
// The reference evaluates these with floating-point expansions that grow on the
// heap (src/expansion.h:137-175).  Here the integers of one call live in an
// arena of global memory that the host hands to the thread evaluating it (sized
// for the widest span finite doubles allow: 2^-1074 to 2^1024), so that no call
// is left without a sign.  Every value of one evaluation has the same number
// of limbs, chosen from the call's exponent span exactly as for the narrower
// tiers (exact_int.cuh), and the same polynomial code (in_sphere_num,
// orient3d_num) runs over it.
#pragma once

#include "exact_int.cuh"

namespace d3g {

/// Limbs of the widest exact value any call can need: in_sphere's degree-5
/// determinant of coordinates spanning 2098 bits (5 * 2099 + 7 bits + sign).
constexpr int kWideMaxLimbs = 165;
/// Values an evaluation keeps at once, at most (in_sphere_num allocates about
/// 100 of its width; multiplication borrows two more and gives them back).
constexpr int kWideValues = 112;
/// Arena limbs one evaluation needs at the widest.
constexpr int64_t kWideArenaLimbs = int64_t(kWideValues) * kWideMaxLimbs;

/// A bump allocator over one thread's piece of the arena.
struct Arena {
    uint64_t* base;
    int64_t cap;
    int64_t used;
    bool overflow;
    D3G_HD uint64_t* take(int n) {
        if (used + n > cap) {   // cannot happen for widths up to kWideMaxLimbs; flagged, never silent
            overflow = true;
            return base;
        }
        uint64_t* p = base + used;
        used += n;
        return p;
    }
};

/// An integer of n limbs (two's complement) in an arena.
struct WideG {
    uint64_t* w;
    int n;
    Arena* a;
};

D3G_NOINLINE_HD WideG wg_add(const WideG& x, const WideG& y) {
    WideG r{x.a->take(x.n), x.n, x.a};
    limbs_add(x.w, y.w, r.w, x.n);
    return r;
}
D3G_NOINLINE_HD WideG wg_sub(const WideG& x, const WideG& y) {
    WideG r{x.a->take(x.n), x.n, x.a};
    limbs_sub(x.w, y.w, r.w, x.n);
    return r;
}
/// Product truncated to n limbs (the width is chosen so that nothing is lost).
D3G_NOINLINE_HD WideG wg_mul(const WideG& x, const WideG& y) {
    const int n = x.n;
    WideG r{x.a->take(n), n, x.a};
    uint64_t* ta = x.a->take(n);
    uint64_t* tb = x.a->take(n);
    for (int i = 0; i < n; ++i) {
        ta[i] = x.w[i];
        tb[i] = y.w[i];
    }
    const bool na = limbs_is_neg(ta, n), nb = limbs_is_neg(tb, n);
    if (na) limbs_neg(ta, n);
    if (nb) limbs_neg(tb, n);
    limbs_mul_mag(ta, tb, r.w, n);
    if (na != nb) limbs_neg(r.w, n);
    if (!x.a->overflow) x.a->used -= 2 * int64_t(n);   // the two copies go back
    return r;
}
D3G_HD WideG operator+(const WideG& a, const WideG& b) { return wg_add(a, b); }
D3G_HD WideG operator-(const WideG& a, const WideG& b) { return wg_sub(a, b); }
D3G_HD WideG operator*(const WideG& a, const WideG& b) { return wg_mul(a, b); }
D3G_HD int num_sign(const WideG& a) { return limbs_sign(a.w, a.n); }

template <>
struct NumFrom<WideG> {
    int emin;
    int n;
    Arena* a;
    D3G_HD WideG operator()(double x) const {
        WideG r{a->take(n), n, a};
        limbs_from(x, emin, r.w, n);
        return r;
    }
};

}  // namespace d3g
