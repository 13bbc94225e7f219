// Device predicates of the del3d build path: orient3d, in_sphere (raw and
// symbolically perturbed), orient2d, the coplanar family and collinear.
//
// Two stages, as in the reference (src/predicates.cpp, src/predicates2.cpp):
//
//   1. Filter.  The reference's own expression, evaluated in the same
//      association order with explicit round-to-nearest intrinsics
//      (__dadd_rn/__dsub_rn/__dmul_rn never contract into FMAs), together with
//      the reference's permanent-based error bound.  Every filter decision
//      therefore matches the reference bit for bit, including wherever its
//      static bound is not rigorous.
//   2. Exact stage, for the calls the filter leaves uncertain.  If the
//      coordinates' exponent span is small enough that the filter's arithmetic
//      could not have rounded, the filter value itself is exact and is used
//      directly (integer lattices, coarse quantisations).  Otherwise the
//      determinant is recomputed in fixed-width integers (exact_int.cuh).
//
// Symbolic perturbation follows src/predicates.cpp:206-232 and
// src/predicates2.cpp:236-259 step for step; "the same point" is decided by the
// caller-supplied identity (point index), which is what the reference's pointer
// comparisons amount to for points taken from one array.
#pragma once

#include "exact_int.cuh"

#include <cstdint>

#if defined(__CUDACC__)
#define D3G_NOINLINE static __host__ __device__ __noinline__
#else
#define D3G_NOINLINE static inline
#endif

namespace d3g {

/// Status bits reported by device code (OR-ed into a status word).
enum : uint32_t {
    ST_EXACT_CAPACITY = 1u << 0,   // exponent span too wide for the exact stage
    ST_CAVITY_CAPACITY = 1u << 1,  // a conflict region outgrew its scratch space
    ST_WALK_LIMIT = 1u << 2,       // a point-location walk exceeded its step limit
    ST_TET_CAPACITY = 1u << 3,     // the tet table is full
    ST_ROUND_LIMIT = 1u << 4,      // insertion rounds exceeded their limit
    ST_INTERNAL = 1u << 5,         // an invariant did not hold
};

struct Pt {
    double x, y, z;
};

D3G_HD double fadd(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
D3G_HD double fsub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
D3G_HD double fmul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
D3G_HD double fabs_(double a) { return a < 0.0 ? -a : a; }
D3G_HD int sign_of(double d) { return d > 0.0 ? 1 : (d < 0.0 ? -1 : 0); }

D3G_HD void report(uint32_t* status, uint32_t bit) {
    if (!status) return;
#if defined(__CUDA_ARCH__)
    atomicOr(status, bit);
#else
    *status |= bit;
#endif
}

// First-stage bounds: src/predicates.cpp:23-27 and src/predicates2.cpp:22-27.
constexpr double kEps = 1.1102230246251565e-16;
constexpr double kOrient3dBound = (7.0 + 56.0 * kEps) * kEps;
constexpr double kInSphereBound = (16.0 + 224.0 * kEps) * kEps;
constexpr double kOrient2dBound = (3.0 + 16.0 * kEps) * kEps;
constexpr double kInCircleBound = (16.0 + 224.0 * kEps) * kEps;

/// Limb count for an exact value of `bits` magnitude bits plus a sign bit.
D3G_HD int limbs_for(int bits) { return (bits + 1 + 63) / 64; }

// =============================================================================
// orient3d: filter src/predicates.cpp:125-147, exact :46-63.
// Sign of |b-a, c-a, d-a|; evaluated as -sign|a-d, b-d, c-d|.
// =============================================================================

struct Orient3dFilter {
    double det;
    bool certain;
};

D3G_HD Orient3dFilter orient3d_filter(const Pt& a, const Pt& b, const Pt& c, const Pt& d) {
    const double adx = fsub(a.x, d.x), bdx = fsub(b.x, d.x), cdx = fsub(c.x, d.x);
    const double ady = fsub(a.y, d.y), bdy = fsub(b.y, d.y), cdy = fsub(c.y, d.y);
    const double adz = fsub(a.z, d.z), bdz = fsub(b.z, d.z), cdz = fsub(c.z, d.z);
    const double bdxcdy = fmul(bdx, cdy), cdxbdy = fmul(cdx, bdy);
    const double cdxady = fmul(cdx, ady), adxcdy = fmul(adx, cdy);
    const double adxbdy = fmul(adx, bdy), bdxady = fmul(bdx, ady);
    const double det = fadd(fadd(fmul(adz, fsub(bdxcdy, cdxbdy)), fmul(bdz, fsub(cdxady, adxcdy))),
                            fmul(cdz, fsub(adxbdy, bdxady)));
    const double permanent =
        fadd(fadd(fmul(fadd(fabs_(bdxcdy), fabs_(cdxbdy)), fabs_(adz)),
                  fmul(fadd(fabs_(cdxady), fabs_(adxcdy)), fabs_(bdz))),
             fmul(fadd(fabs_(adxbdy), fabs_(bdxady)), fabs_(cdz)));
    const double errbound = fmul(kOrient3dBound, permanent);
    Orient3dFilter r;
    r.det = det;
    r.certain = (det > errbound) || (-det > errbound);
    return r;
}

template <class N>
D3G_HD int orient3d_num(const Pt& a, const Pt& b, const Pt& c, const Pt& d, const NumFrom<N>& f) {
    const N dx = f(d.x), dy = f(d.y), dz = f(d.z);
    const N adx = f(a.x) - dx, ady = f(a.y) - dy, adz = f(a.z) - dz;
    const N bdx = f(b.x) - dx, bdy = f(b.y) - dy, bdz = f(b.z) - dz;
    const N cdx = f(c.x) - dx, cdy = f(c.y) - dy, cdz = f(c.z) - dz;
    const N t1 = bdx * cdy - cdx * bdy;
    const N t2 = cdx * ady - adx * cdy;
    const N t3 = adx * bdy - bdx * ady;
    const N det = adz * t1 + bdz * t2 + cdz * t3;
    return -num_sign(det);
}

/// Exact orient3d of a call the filter left uncertain.  Out of line and shared
/// by every call site (one copy of the degenerate-case code keeps the kernels'
/// instruction footprint small when many lanes take it), with scalar arguments
/// so that nothing needs an address in local memory.  `fdet` is the filter's
/// value, exact - and used - when the exponent span is small (integer lattices,
/// coarse grids); otherwise fixed-width integers.
D3G_NOINLINE int orient3d_degenerate(double ax, double ay, double az, double bx, double by, double bz,
                                     double cx, double cy, double cz, double dx, double dy, double dz,
                                     double fdet, uint32_t* status) {
    const Pt a{ax, ay, az}, b{bx, by, bz}, c{cx, cy, cz}, d{dx, dy, dz};
    Span s;
    s.add(ax); s.add(ay); s.add(az); s.add(bx); s.add(by); s.add(bz);
    s.add(cx); s.add(cy); s.add(cz); s.add(dx); s.add(dy); s.add(dz);
    if (s.exact_in_double(3, 3)) return -sign_of(fdet);
    const int L = limbs_for(3 * (s.bits() + 1) + 3);
    if (L <= 2) return orient3d_num<WideS<2>>(a, b, c, d, NumFrom<WideS<2>>{s.emin});
    if (L <= 4) return orient3d_num<WideS<4>>(a, b, c, d, NumFrom<WideS<4>>{s.emin});
    if (L <= kMaxLimbs) return orient3d_num<WideV>(a, b, c, d, NumFrom<WideV>{s.emin, L});
    report(status, ST_EXACT_CAPACITY);
    return 0;
}

D3G_HD int orient3d_exact(const Pt& a, const Pt& b, const Pt& c, const Pt& d, double fdet, uint32_t* status) {
    return orient3d_degenerate(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, d.x, d.y, d.z, fdet, status);
}

D3G_HD int orient3d(const Pt& a, const Pt& b, const Pt& c, const Pt& d, uint32_t* status) {
    const Orient3dFilter f = orient3d_filter(a, b, c, d);
    if (f.certain) return -sign_of(f.det);
    return orient3d_exact(a, b, c, d, f.det, status);
}

/// orient3d where the caller knows the filter's arithmetic is exact for these
/// points when `exact` is set (a point set whose coordinates span few bits):
/// then the filter value is the determinant and no exact stage is needed.
D3G_HD int orient3d_x(const Pt& a, const Pt& b, const Pt& c, const Pt& d, bool exact, uint32_t* status) {
    const Orient3dFilter f = orient3d_filter(a, b, c, d);
    if (f.certain || exact) return -sign_of(f.det);
    return orient3d_exact(a, b, c, d, f.det, status);
}

// =============================================================================
// in_sphere: filter src/predicates.cpp:149-204, exact :76-113, perturbation
// :206-232.  POSITIVE iff e is strictly inside the sphere through a,b,c,d
// (for positively oriented a,b,c,d).
// =============================================================================

struct InSphereFilter {
    double det;
    bool certain;
};

D3G_HD InSphereFilter in_sphere_filter(const Pt& a, const Pt& b, const Pt& c, const Pt& d,
                                       const Pt& e) {
    const double aex = fsub(a.x, e.x), aey = fsub(a.y, e.y), aez = fsub(a.z, e.z);
    const double bex = fsub(b.x, e.x), bey = fsub(b.y, e.y), bez = fsub(b.z, e.z);
    const double cex = fsub(c.x, e.x), cey = fsub(c.y, e.y), cez = fsub(c.z, e.z);
    const double dex = fsub(d.x, e.x), dey = fsub(d.y, e.y), dez = fsub(d.z, e.z);

    const double aexbey = fmul(aex, bey), bexaey = fmul(bex, aey);
    const double bexcey = fmul(bex, cey), cexbey = fmul(cex, bey);
    const double cexdey = fmul(cex, dey), dexcey = fmul(dex, cey);
    const double dexaey = fmul(dex, aey), aexdey = fmul(aex, dey);
    const double aexcey = fmul(aex, cey), cexaey = fmul(cex, aey);
    const double bexdey = fmul(bex, dey), dexbey = fmul(dex, bey);

    const double ab = fsub(aexbey, bexaey);
    const double bc = fsub(bexcey, cexbey);
    const double cd = fsub(cexdey, dexcey);
    const double da = fsub(dexaey, aexdey);
    const double ac = fsub(aexcey, cexaey);
    const double bd = fsub(bexdey, dexbey);

    const double abc = fadd(fsub(fmul(aez, bc), fmul(bez, ac)), fmul(cez, ab));
    const double bcd = fadd(fsub(fmul(bez, cd), fmul(cez, bd)), fmul(dez, bc));
    const double cda = fadd(fadd(fmul(cez, da), fmul(dez, ac)), fmul(aez, cd));
    const double dab = fadd(fadd(fmul(dez, ab), fmul(aez, bd)), fmul(bez, da));

    const double alift = fadd(fadd(fmul(aex, aex), fmul(aey, aey)), fmul(aez, aez));
    const double blift = fadd(fadd(fmul(bex, bex), fmul(bey, bey)), fmul(bez, bez));
    const double clift = fadd(fadd(fmul(cex, cex), fmul(cey, cey)), fmul(cez, cez));
    const double dlift = fadd(fadd(fmul(dex, dex), fmul(dey, dey)), fmul(dez, dez));

    const double det = fadd(fsub(fmul(dlift, abc), fmul(clift, dab)),
                            fsub(fmul(blift, cda), fmul(alift, bcd)));

    const double aezp = fabs_(aez), bezp = fabs_(bez), cezp = fabs_(cez), dezp = fabs_(dez);
    const double aexbeyp = fabs_(aexbey), bexaeyp = fabs_(bexaey);
    const double bexceyp = fabs_(bexcey), cexbeyp = fabs_(cexbey);
    const double cexdeyp = fabs_(cexdey), dexceyp = fabs_(dexcey);
    const double dexaeyp = fabs_(dexaey), aexdeyp = fabs_(aexdey);
    const double aexceyp = fabs_(aexcey), cexaeyp = fabs_(cexaey);
    const double bexdeyp = fabs_(bexdey), dexbeyp = fabs_(dexbey);

    const double pa = fadd(fadd(fmul(fadd(cexdeyp, dexceyp), bezp), fmul(fadd(dexbeyp, bexdeyp), cezp)),
                           fmul(fadd(bexceyp, cexbeyp), dezp));
    const double pb = fadd(fadd(fmul(fadd(dexaeyp, aexdeyp), cezp), fmul(fadd(aexceyp, cexaeyp), dezp)),
                           fmul(fadd(cexdeyp, dexceyp), aezp));
    const double pc = fadd(fadd(fmul(fadd(aexbeyp, bexaeyp), dezp), fmul(fadd(bexdeyp, dexbeyp), aezp)),
                           fmul(fadd(dexaeyp, aexdeyp), bezp));
    const double pd = fadd(fadd(fmul(fadd(bexceyp, cexbeyp), aezp), fmul(fadd(cexaeyp, aexceyp), bezp)),
                           fmul(fadd(aexbeyp, bexaeyp), cezp));
    const double permanent =
        fadd(fadd(fadd(fmul(pa, alift), fmul(pb, blift)), fmul(pc, clift)), fmul(pd, dlift));
    const double errbound = fmul(kInSphereBound, permanent);
    InSphereFilter r;
    r.det = det;
    r.certain = (det > errbound) || (-det > errbound);
    return r;
}

template <class N>
D3G_HD int in_sphere_num(const Pt& a, const Pt& b, const Pt& c, const Pt& d, const Pt& e,
                         const NumFrom<N>& f) {
    const N ex = f(e.x), ey = f(e.y), ez = f(e.z);
    const N aex = f(a.x) - ex, aey = f(a.y) - ey, aez = f(a.z) - ez;
    const N bex = f(b.x) - ex, bey = f(b.y) - ey, bez = f(b.z) - ez;
    const N cex = f(c.x) - ex, cey = f(c.y) - ey, cez = f(c.z) - ez;
    const N dex = f(d.x) - ex, dey = f(d.y) - ey, dez = f(d.z) - ez;
    const N ab = aex * bey - bex * aey;
    const N bc = bex * cey - cex * bey;
    const N cd = cex * dey - dex * cey;
    const N da = dex * aey - aex * dey;
    const N ac = aex * cey - cex * aey;
    const N bd = bex * dey - dex * bey;
    const N abc = aez * bc - bez * ac + cez * ab;
    const N bcd = bez * cd - cez * bd + dez * bc;
    const N cda = cez * da + dez * ac + aez * cd;
    const N dab = dez * ab + aez * bd + bez * da;
    const N alift = aex * aex + aey * aey + aez * aez;
    const N blift = bex * bex + bey * bey + bez * bez;
    const N clift = cex * cex + cey * cey + cez * cez;
    const N dlift = dex * dex + dey * dey + dez * dez;
    const N det = (dlift * abc - clift * dab) + (blift * cda - alift * bcd);
    return -num_sign(det);
}

D3G_NOINLINE int in_sphere_degenerate(double ax, double ay, double az, double bx, double by, double bz,
                                      double cx, double cy, double cz, double dx, double dy, double dz,
                                      double ex, double ey, double ez, int64_t id0, int64_t id1, int64_t id2,
                                      int64_t id3, int64_t id4, double fdet, int perturbed, uint32_t* status);

D3G_HD int in_sphere_exact(const Pt& a, const Pt& b, const Pt& c, const Pt& d, const Pt& e, double fdet,
                           uint32_t* status) {
    return in_sphere_degenerate(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, d.x, d.y, d.z, e.x, e.y, e.z, 0, 1,
                                2, 3, 4, fdet, 0, status);
}

D3G_HD int in_sphere_unperturbed(const Pt& a, const Pt& b, const Pt& c, const Pt& d, const Pt& e,
                                 uint32_t* status) {
    const InSphereFilter f = in_sphere_filter(a, b, c, d, e);
    if (f.certain) return -sign_of(f.det);
    return in_sphere_exact(a, b, c, d, e, f.det, status);
}

D3G_HD bool lexico_less(const Pt& p, const Pt& q) {
    if (p.x != q.x) return p.x < q.x;
    if (p.y != q.y) return p.y < q.y;
    return p.z < q.z;
}

/// The cospherical tie-break (src/predicates.cpp:211-231).  `id` holds the
/// identities of a,b,c,d,e; slot order (a,b,c,d,e) is kept among equal points,
/// as the reference's std::sort of five elements (an insertion sort) keeps it.
/// The slot (0-4) of (a, b, c, d, e) that comes last when the five points are
/// sorted lexicographically with equal points kept in slot order (a stable
/// sort, as the reference's insertion-sort std::sort of five elements is),
/// leaving out slot `skip` (-1: none).  Registers only.
D3G_HD int lexico_last(const Pt& a, const Pt& b, const Pt& c, const Pt& d, const Pt& e, int skip) {
    int best = skip == 0 ? 1 : 0;
    Pt bp = skip == 0 ? b : a;
#pragma unroll
    for (int k = 1; k < 5; ++k) {
        if (k == skip || k == best) continue;
        const Pt& q = k == 1 ? b : (k == 2 ? c : (k == 3 ? d : e));
        if (!lexico_less(q, bp)) {   // a later slot wins ties
            best = k;
            bp = q;
        }
    }
    return best;
}

/// The cospherical tie-break (src/predicates.cpp:211-231): walking down the
/// lexicographic order from the largest point, the first point that is e
/// gives NEGATIVE; the first other point whose replacement by e gives a
/// non-zero orient3d gives that sign.  `id0..id4` are the identities of a..e
/// (the reference compares pointers, so equal identities are the same point).
template <class Orient>
D3G_HD int in_sphere_perturb_by(const Orient& orient, const Pt& a, const Pt& b, const Pt& c, const Pt& d,
                                const Pt& e, int64_t id0, int64_t id1, int64_t id2, int64_t id3, int64_t id4) {
    int skip = -1;
#pragma unroll 1
    for (int r = 0; r < 2; ++r) {
        const int k = lexico_last(a, b, c, d, e, skip);
        skip = k;
        const int64_t idk = k == 0 ? id0 : (k == 1 ? id1 : (k == 2 ? id2 : (k == 3 ? id3 : id4)));
        if (idk == id4) return -1;
        // The reference tests d, c, b, a in this order; each replaces that slot by e.
#pragma unroll 1
        for (int j = 3; j >= 0; --j) {
            const int64_t idj = j == 0 ? id0 : (j == 1 ? id1 : (j == 2 ? id2 : id3));
            if (idk != idj) continue;
            const Pt& A = j == 0 ? e : a;
            const Pt& B = j == 1 ? e : b;
            const Pt& C = j == 2 ? e : c;
            const Pt& D = j == 3 ? e : d;
            const int o = orient(A, B, C, D);
            if (o != 0) return o;
        }
    }
    return -1;
}

/// orient3d_x as a function object (the orientation the tie-break uses).
template <bool EX>
struct Orient3dX {
    uint32_t* status;
    D3G_HD int operator()(const Pt& A, const Pt& B, const Pt& C, const Pt& D) const {
        return orient3d_x(A, B, C, D, EX, status);
    }
};

template <bool EX = false>
D3G_HD int in_sphere_perturb(const Pt& a, const Pt& b, const Pt& c, const Pt& d, const Pt& e, int64_t id0,
                             int64_t id1, int64_t id2, int64_t id3, int64_t id4, uint32_t* status) {
    return in_sphere_perturb_by(Orient3dX<EX>{status}, a, b, c, d, e, id0, id1, id2, id3, id4);
}

/// Exact sign of in_sphere (and, with `perturbed`, the tie-break) for a call the
/// filter left uncertain; shared and out of line like orient3d_degenerate.
D3G_NOINLINE int in_sphere_degenerate(double ax, double ay, double az, double bx, double by, double bz,
                                      double cx, double cy, double cz, double dx, double dy, double dz,
                                      double ex, double ey, double ez, int64_t id0, int64_t id1, int64_t id2,
                                      int64_t id3, int64_t id4, double fdet, int perturbed, uint32_t* status) {
    const Pt a{ax, ay, az}, b{bx, by, bz}, c{cx, cy, cz}, d{dx, dy, dz}, e{ex, ey, ez};
    Span s;
    s.add(ax); s.add(ay); s.add(az); s.add(bx); s.add(by); s.add(bz);
    s.add(cx); s.add(cy); s.add(cz); s.add(dx); s.add(dy); s.add(dz);
    s.add(ex); s.add(ey); s.add(ez);
    int sign;
    if (s.exact_in_double(5, 7)) {
        sign = -sign_of(fdet);
    } else {
        const int L = limbs_for(5 * (s.bits() + 1) + 7);
        if (L <= 2) sign = in_sphere_num<WideS<2>>(a, b, c, d, e, NumFrom<WideS<2>>{s.emin});
        else if (L <= 4) sign = in_sphere_num<WideS<4>>(a, b, c, d, e, NumFrom<WideS<4>>{s.emin});
        else if (L <= kMaxLimbs) sign = in_sphere_num<WideV>(a, b, c, d, e, NumFrom<WideV>{s.emin, L});
        else {
            report(status, ST_EXACT_CAPACITY);
            return 0;
        }
    }
    if (sign != 0 || !perturbed) return sign;
    return in_sphere_perturb(a, b, c, d, e, id0, id1, id2, id3, id4, status);
}

/// The tie-break of an exactly cospherical in_sphere call for points whose
/// filter arithmetic is exact (shared and out of line).
D3G_NOINLINE int in_sphere_tiebreak_exact(double ax, double ay, double az, double bx, double by, double bz,
                                          double cx, double cy, double cz, double dx, double dy, double dz,
                                          double ex, double ey, double ez, int64_t id0, int64_t id1,
                                          int64_t id2, int64_t id3, int64_t id4, uint32_t* status) {
    const Pt a{ax, ay, az}, b{bx, by, bz}, c{cx, cy, cz}, d{dx, dy, dz}, e{ex, ey, ez};
    return in_sphere_perturb<true>(a, b, c, d, e, id0, id1, id2, id3, id4, status);
}

D3G_HD int in_sphere(const Pt& a, const Pt& b, const Pt& c, const Pt& d, const Pt& e,
                     const int64_t* id, uint32_t* status) {
    const InSphereFilter f = in_sphere_filter(a, b, c, d, e);
    if (f.certain) return -sign_of(f.det);
    return in_sphere_degenerate(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, d.x, d.y, d.z, e.x, e.y, e.z, id[0],
                                id[1], id[2], id[3], id[4], f.det, 1, status);
}

// =============================================================================
// orient2d and the coplanar family: src/predicates2.cpp:111-259.
// =============================================================================

template <class N>
D3G_HD int orient2d_num(double px, double py, double qx, double qy, double rx, double ry,
                        const NumFrom<N>& f) {
    const N PX = f(px), PY = f(py);
    const N qpx = f(qx) - PX, qpy = f(qy) - PY;
    const N rpx = f(rx) - PX, rpy = f(ry) - PY;
    return num_sign(qpx * rpy - qpy * rpx);
}

D3G_NOINLINE int orient2d_exact(double px, double py, double qx, double qy, double rx, double ry,
                                double fdet, uint32_t* status) {
    Span s;
    s.add(px); s.add(py); s.add(qx); s.add(qy); s.add(rx); s.add(ry);
    if (s.exact_in_double(2, 1)) return sign_of(fdet);
    const int L = limbs_for(2 * (s.bits() + 1) + 1);
    if (L <= 2) return orient2d_num<WideS<2>>(px, py, qx, qy, rx, ry, NumFrom<WideS<2>>{s.emin});
    if (L <= kMaxLimbs) return orient2d_num<WideV>(px, py, qx, qy, rx, ry, NumFrom<WideV>{s.emin, L});
    report(status, ST_EXACT_CAPACITY);
    return 0;
}

D3G_HD int orient2d(double px, double py, double qx, double qy, double rx, double ry,
                    uint32_t* status) {
    const double qpx = fsub(qx, px), qpy = fsub(qy, py);
    const double rpx = fsub(rx, px), rpy = fsub(ry, py);
    const double a = fmul(qpx, rpy), b = fmul(qpy, rpx);
    const double det = fsub(a, b);
    const double permanent = fadd(fabs_(a), fabs_(b));
    const double errbound = fmul(kOrient2dBound, permanent);
    if (det > errbound || -det > errbound) return sign_of(det);
    return orient2d_exact(px, py, qx, qy, rx, ry, det, status);
}

D3G_HD int coplanar_orientation3(const Pt& p, const Pt& q, const Pt& r, uint32_t* st) {
    const int oxy = orient2d(p.x, p.y, q.x, q.y, r.x, r.y, st);
    if (oxy != 0) return oxy;
    const int oyz = orient2d(p.y, p.z, q.y, q.z, r.y, r.z, st);
    if (oyz != 0) return oyz;
    return orient2d(p.x, p.z, q.x, q.z, r.x, r.z, st);
}

D3G_HD int coplanar_orientation4(const Pt& p, const Pt& q, const Pt& r, const Pt& s, uint32_t* st) {
    const int oxy = orient2d(p.x, p.y, q.x, q.y, r.x, r.y, st);
    if (oxy != 0) return oxy * orient2d(p.x, p.y, q.x, q.y, s.x, s.y, st);
    const int oyz = orient2d(p.y, p.z, q.y, q.z, r.y, r.z, st);
    if (oyz != 0) return oyz * orient2d(p.y, p.z, q.y, q.z, s.y, s.z, st);
    const int oxz = orient2d(p.x, p.z, q.x, q.z, r.x, r.z, st);
    return oxz * orient2d(p.x, p.z, q.x, q.z, s.x, s.z, st);
}

D3G_HD bool collinear(const Pt& p, const Pt& q, const Pt& r, uint32_t* st) {
    if (orient2d(r.x, r.y, p.x, p.y, q.x, q.y, st) != 0) return false;
    if (orient2d(r.x, r.z, p.x, p.z, q.x, q.z, st) != 0) return false;
    return orient2d(r.y, r.z, p.y, p.z, q.y, q.z, st) == 0;
}

struct InCircleFilter {
    double det;
    bool certain;
};

/// The filtered in-circle determinant of src/predicates2.cpp:182-231: rows
/// (pt, rt, qt, v) with v the plane normal, minors m01 = a10*a01 - a00*a11.
D3G_HD InCircleFilter in_circle_filter(const Pt& p0, const Pt& p1, const Pt& p2, const Pt& p) {
    const double ptx = fsub(p0.x, p.x), pty = fsub(p0.y, p.y), ptz = fsub(p0.z, p.z);
    const double qtx = fsub(p1.x, p.x), qty = fsub(p1.y, p.y), qtz = fsub(p1.z, p.z);
    const double rtx = fsub(p2.x, p.x), rty = fsub(p2.y, p.y), rtz = fsub(p2.z, p.z);
    const double pt2 = fadd(fadd(fmul(ptx, ptx), fmul(pty, pty)), fmul(ptz, ptz));
    const double qt2 = fadd(fadd(fmul(qtx, qtx), fmul(qty, qty)), fmul(qtz, qtz));
    const double rt2 = fadd(fadd(fmul(rtx, rtx), fmul(rty, rty)), fmul(rtz, rtz));
    const double pqx = fsub(p1.x, p0.x), pqy = fsub(p1.y, p0.y), pqz = fsub(p1.z, p0.z);
    const double prx = fsub(p2.x, p0.x), pry = fsub(p2.y, p0.y), prz = fsub(p2.z, p0.z);
    const double vx = fsub(fmul(pqy, prz), fmul(pqz, pry));
    const double vy = fsub(fmul(pqz, prx), fmul(pqx, prz));
    const double vz = fsub(fmul(pqx, pry), fmul(pqy, prx));
    const double v2 = fadd(fadd(fmul(vx, vx), fmul(vy, vy)), fmul(vz, vz));
    const double a00 = ptx, a01 = pty, a02 = ptz, a03 = pt2;
    const double a10 = rtx, a11 = rty, a12 = rtz, a13 = rt2;
    const double a20 = qtx, a21 = qty, a22 = qtz, a23 = qt2;
    const double a30 = vx, a31 = vy, a32 = vz, a33 = v2;
    const double m01 = fsub(fmul(a10, a01), fmul(a00, a11));
    const double m02 = fsub(fmul(a20, a01), fmul(a00, a21));
    const double m03 = fsub(fmul(a30, a01), fmul(a00, a31));
    const double m12 = fsub(fmul(a20, a11), fmul(a10, a21));
    const double m13 = fsub(fmul(a30, a11), fmul(a10, a31));
    const double m23 = fsub(fmul(a30, a21), fmul(a20, a31));
    const double m012 = fadd(fsub(fmul(m12, a02), fmul(m02, a12)), fmul(m01, a22));
    const double m013 = fadd(fsub(fmul(m13, a02), fmul(m03, a12)), fmul(m01, a32));
    const double m023 = fadd(fsub(fmul(m23, a02), fmul(m03, a22)), fmul(m02, a32));
    const double m123 = fadd(fsub(fmul(m23, a12), fmul(m13, a22)), fmul(m12, a32));
    const double det = fsub(fadd(fsub(fmul(m123, a03), fmul(m023, a13)), fmul(m013, a23)),
                            fmul(m012, a33));
    const double rows[4][4] = {{a00, a01, a02, a03}, {a10, a11, a12, a13},
                               {a20, a21, a22, a23}, {a30, a31, a32, a33}};
    double mag = 0.0;
    for (int i = 0; i < 4; ++i) {
        double row = 0.0;
        for (int j = 0; j < 4; ++j) row = fadd(row, fabs_(rows[i][j]));
        mag = (mag == 0.0) ? row : fmul(mag, row);
    }
    const double errbound = fmul(kInCircleBound, mag);
    InCircleFilter r;
    r.det = det;
    r.certain = (det > errbound) || (-det > errbound);
    return r;
}

template <class N>
D3G_HD int in_circle_num(const Pt& p, const Pt& q, const Pt& r, const Pt& t, const NumFrom<N>& f) {
    const N tx = f(t.x), ty = f(t.y), tz = f(t.z);
    const N px = f(p.x), py = f(p.y), pz = f(p.z);
    const N qx = f(q.x), qy = f(q.y), qz = f(q.z);
    const N rx = f(r.x), ry = f(r.y), rz = f(r.z);
    const N ptx = px - tx, pty = py - ty, ptz = pz - tz;
    const N qtx = qx - tx, qty = qy - ty, qtz = qz - tz;
    const N rtx = rx - tx, rty = ry - ty, rtz = rz - tz;
    const N pt2 = ptx * ptx + pty * pty + ptz * ptz;
    const N qt2 = qtx * qtx + qty * qty + qtz * qtz;
    const N rt2 = rtx * rtx + rty * rty + rtz * rtz;
    const N pqx = qx - px, pqy = qy - py, pqz = qz - pz;
    const N prx = rx - px, pry = ry - py, prz = rz - pz;
    const N vx = pqy * prz - pqz * pry;
    const N vy = pqz * prx - pqx * prz;
    const N vz = pqx * pry - pqy * prx;
    const N v2 = vx * vx + vy * vy + vz * vz;
    // Rows (pt, rt, qt, v); minors m01 = a10*a01 - a00*a11 (src/predicates2.cpp:84-101).
    const N m01 = rtx * pty - ptx * rty;
    const N m02 = qtx * pty - ptx * qty;
    const N m03 = vx * pty - ptx * vy;
    const N m12 = qtx * rty - rtx * qty;
    const N m13 = vx * rty - rtx * vy;
    const N m23 = vx * qty - qtx * vy;
    const N m012 = m12 * ptz - m02 * rtz + m01 * qtz;
    const N m013 = m13 * ptz - m03 * rtz + m01 * vz;
    const N m023 = m23 * ptz - m03 * qtz + m02 * vz;
    const N m123 = m23 * rtz - m13 * qtz + m12 * vz;
    const N det = m123 * pt2 - m023 * rt2 + m013 * qt2 - m012 * v2;
    return num_sign(det);
}

/// The slot (0-3) of (p0, p1, p2, p) last in lexicographic order with equal
/// points kept in slot order, among the slots not in `excluded` (bit mask).
D3G_HD int lexico_last4(const Pt& p0, const Pt& p1, const Pt& p2, const Pt& p, unsigned excluded) {
    int best = -1;
    Pt bp = p0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (excluded & (1u << k)) continue;
        const Pt& q = k == 0 ? p0 : (k == 1 ? p1 : (k == 2 ? p2 : p));
        if (best < 0 || !lexico_less(q, bp)) {
            best = k;
            bp = q;
        }
    }
    return best;
}

/// The cocircular tie-break (src/predicates2.cpp:241-258): walking down the
/// lexicographic order of (p0, p1, p2, p) from the largest, the first point
/// that is p gives NEGATIVE; the first other point whose replacement by p
/// gives a non-zero coplanar orientation gives it times the orientation of
/// (p0, p1, p2).  `id0..id3` are the identities of p0, p1, p2, p.
D3G_HD int in_circle_perturb(const Pt& p0, const Pt& p1, const Pt& p2, const Pt& p, int64_t id0, int64_t id1,
                             int64_t id2, int64_t id3, uint32_t* status) {
    const int local = coplanar_orientation3(p0, p1, p2, status);
    unsigned excluded = 0;
#pragma unroll 1
    for (int r = 0; r < 3; ++r) {
        const int k = lexico_last4(p0, p1, p2, p, excluded);
        excluded |= 1u << k;
        const int64_t idk = k == 0 ? id0 : (k == 1 ? id1 : (k == 2 ? id2 : id3));
        if (idk == id3) return -1;
#pragma unroll 1
        for (int j = 2; j >= 0; --j) {
            const int64_t idj = j == 0 ? id0 : (j == 1 ? id1 : id2);
            if (idk != idj) continue;
            const Pt& A = j == 0 ? p : p0;
            const Pt& B = j == 1 ? p : p1;
            const Pt& C = j == 2 ? p : p2;
            const int o = coplanar_orientation3(A, B, C, status);
            if (o != 0) return o * local;
        }
    }
    return -local;
}

/// Exact in-circle sign (and, with `perturbed`, the tie-break) for a call the
/// filter left uncertain; shared and out of line like orient3d_degenerate.
D3G_NOINLINE int in_circle_degenerate(double ax, double ay, double az, double bx, double by, double bz,
                                      double cx, double cy, double cz, double px, double py, double pz,
                                      int64_t id0, int64_t id1, int64_t id2, int64_t id3, double fdet,
                                      int perturbed, uint32_t* status) {
    const Pt p0{ax, ay, az}, p1{bx, by, bz}, p2{cx, cy, cz}, p{px, py, pz};
    Span s;
    s.add(ax); s.add(ay); s.add(az); s.add(bx); s.add(by); s.add(bz);
    s.add(cx); s.add(cy); s.add(cz); s.add(px); s.add(py); s.add(pz);
    int sign;
    if (s.exact_in_double(7, 9)) {
        sign = sign_of(fdet);
    } else {
        const int L = limbs_for(7 * (s.bits() + 1) + 9);
        if (L <= 4) sign = in_circle_num<WideS<4>>(p0, p1, p2, p, NumFrom<WideS<4>>{s.emin});
        else if (L <= kMaxLimbs) sign = in_circle_num<WideV>(p0, p1, p2, p, NumFrom<WideV>{s.emin, L});
        else {
            report(status, ST_EXACT_CAPACITY);
            return 0;
        }
    }
    if (sign != 0 || !perturbed) return sign;
    return in_circle_perturb(p0, p1, p2, p, id0, id1, id2, id3, status);
}

D3G_HD int coplanar_in_circle_unperturbed(const Pt& p0, const Pt& p1, const Pt& p2, const Pt& p,
                                          uint32_t* status) {
    const InCircleFilter f = in_circle_filter(p0, p1, p2, p);
    if (f.certain) return sign_of(f.det);
    return in_circle_degenerate(p0.x, p0.y, p0.z, p1.x, p1.y, p1.z, p2.x, p2.y, p2.z, p.x, p.y, p.z, 0, 1, 2, 3,
                                f.det, 0, status);
}

D3G_HD int coplanar_in_circle(const Pt& p0, const Pt& p1, const Pt& p2, const Pt& p,
                              const int64_t* id, uint32_t* status) {
    const InCircleFilter f = in_circle_filter(p0, p1, p2, p);
    if (f.certain) return sign_of(f.det);
    return in_circle_degenerate(p0.x, p0.y, p0.z, p1.x, p1.y, p1.z, p2.x, p2.y, p2.z, p.x, p.y, p.z, id[0], id[1],
                                id[2], id[3], f.det, 1, status);
}

}  // namespace d3g
