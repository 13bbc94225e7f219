// CPU restatement of the reference del3d `Delaunay::build` path.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h).  Written for obviousness, not speed.
//
// Reference files cited below are paths inside the del3d source tree.
//
// Compile with -ffp-contract=off: the first (filtered) stage of each predicate
// must round exactly as the reference's does, so the same expressions are
// evaluated in the same association order with no fused multiply-adds.
#include "oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

namespace {

// =============================================================================
// Exact integers on a common binary scale.
//
// Every finite double is M * 2^E with M an integer.  For one predicate call all
// coordinates are rewritten as integers times 2^emin (emin the smallest E in the
// call), which scales every determinant by a positive power of two and leaves
// its sign alone.  The determinant is then evaluated with no rounding at all.
// This replaces the reference's expansion arithmetic (src/expansion.h) for the
// exact stage: the exact sign is unique, so any exact evaluation agrees.
// =============================================================================
class Big {
public:
    Big() = default;
    static Big from_u64(uint64_t m, int shift, bool neg) {
        Big r;
        if (m == 0) return r;
        const int words = shift / 32, rest = shift % 32;
        r.mag_.assign(size_t(words), 0u);
        unsigned __int128 v = (unsigned __int128)m << rest;
        while (v) { r.mag_.push_back(uint32_t(v)); v >>= 32; }
        r.neg_ = neg;
        r.trim();
        return r;
    }
    int sign() const { return mag_.empty() ? 0 : (neg_ ? -1 : 1); }
    Big operator-() const { Big r = *this; if (!r.mag_.empty()) r.neg_ = !r.neg_; return r; }
    friend Big operator+(const Big& a, const Big& b) {
        if (a.mag_.empty()) return b;
        if (b.mag_.empty()) return a;
        Big r;
        if (a.neg_ == b.neg_) { r.mag_ = add(a.mag_, b.mag_); r.neg_ = a.neg_; }
        else {
            const int c = cmp(a.mag_, b.mag_);
            if (c == 0) return Big();
            if (c > 0) { r.mag_ = sub(a.mag_, b.mag_); r.neg_ = a.neg_; }
            else       { r.mag_ = sub(b.mag_, a.mag_); r.neg_ = b.neg_; }
        }
        r.trim();
        return r;
    }
    friend Big operator-(const Big& a, const Big& b) { return a + (-b); }
    friend Big operator*(const Big& a, const Big& b) {
        Big r;
        if (a.mag_.empty() || b.mag_.empty()) return r;
        r.mag_.assign(a.mag_.size() + b.mag_.size(), 0u);
        for (size_t i = 0; i < a.mag_.size(); ++i) {
            uint64_t carry = 0;
            for (size_t j = 0; j < b.mag_.size(); ++j) {
                const uint64_t cur = uint64_t(r.mag_[i + j]) + uint64_t(a.mag_[i]) * b.mag_[j] + carry;
                r.mag_[i + j] = uint32_t(cur);
                carry = cur >> 32;
            }
            r.mag_[i + b.mag_.size()] = uint32_t(carry);
        }
        r.neg_ = a.neg_ != b.neg_;
        r.trim();
        return r;
    }

private:
    std::vector<uint32_t> mag_;
    bool neg_ = false;
    void trim() { while (!mag_.empty() && mag_.back() == 0) mag_.pop_back(); if (mag_.empty()) neg_ = false; }
    static int cmp(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {
        if (a.size() != b.size()) return a.size() < b.size() ? -1 : 1;
        for (size_t i = a.size(); i-- > 0;) if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
        return 0;
    }
    static std::vector<uint32_t> add(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {
        std::vector<uint32_t> r(std::max(a.size(), b.size()) + 1, 0u);
        uint64_t c = 0;
        for (size_t i = 0; i < r.size(); ++i) {
            const uint64_t s = c + (i < a.size() ? a[i] : 0u) + (i < b.size() ? b[i] : 0u);
            r[i] = uint32_t(s);
            c = s >> 32;
        }
        return r;
    }
    static std::vector<uint32_t> sub(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {
        std::vector<uint32_t> r(a.size(), 0u);
        int64_t br = 0;
        for (size_t i = 0; i < a.size(); ++i) {
            int64_t s = int64_t(a[i]) - (i < b.size() ? int64_t(b[i]) : 0) - br;
            br = s < 0;
            if (s < 0) s += (int64_t(1) << 32);
            r[i] = uint32_t(s);
        }
        return r;
    }
};

/// Splits a finite nonzero double into an odd-or-not integer mantissa and exponent:
/// x = m * 2^e, |m| < 2^53.
void split_double(double x, uint64_t& m, int& e, bool& neg) {
    int be = 0;
    const double f = std::frexp(std::fabs(x), &be);       // |x| = f * 2^be, 0.5 <= f < 1
    m = uint64_t(std::ldexp(f, 53));
    e = be - 53;
    neg = x < 0;
}

/// The common scale of a group of doubles.
struct Scale {
    int emin = 0;
    bool any = false;
    void add(double x) {
        if (x == 0.0) return;
        uint64_t m; int e; bool n;
        split_double(x, m, e, n);
        if (!any || e < emin) { emin = e; any = true; }
    }
    Big operator()(double x) const {
        if (x == 0.0) return Big();
        uint64_t m; int e; bool n;
        split_double(x, m, e, n);
        return Big::from_u64(m, e - emin, n);
    }
};

inline int sgn(double d) { return d > 0.0 ? 1 : (d < 0.0 ? -1 : 0); }

// 2^-53 and the first-stage bounds: src/predicates.cpp:23-27, src/predicates2.cpp:22-27.
constexpr double kEps = 1.1102230246251565e-16;
constexpr double kOrient3dBound = (7.0 + 56.0 * kEps) * kEps;
constexpr double kInSphereBound = (16.0 + 224.0 * kEps) * kEps;
constexpr double kOrient2dBound = (3.0 + 16.0 * kEps) * kEps;
constexpr double kInCircleBound = (16.0 + 224.0 * kEps) * kEps;

// ---- orient3d: src/predicates.cpp:46-63 (exact) and :125-147 (filter) --------

int orient3d_exact(const double* a, const double* b, const double* c, const double* d) {
    Scale s;
    for (const double* p : {a, b, c, d}) for (int k = 0; k < 3; ++k) s.add(p[k]);
    const Big adx = s(a[0]) - s(d[0]), ady = s(a[1]) - s(d[1]), adz = s(a[2]) - s(d[2]);
    const Big bdx = s(b[0]) - s(d[0]), bdy = s(b[1]) - s(d[1]), bdz = s(b[2]) - s(d[2]);
    const Big cdx = s(c[0]) - s(d[0]), cdy = s(c[1]) - s(d[1]), cdz = s(c[2]) - s(d[2]);
    const Big det = adz * (bdx * cdy - cdx * bdy) + bdz * (cdx * ady - adx * cdy) +
                    cdz * (adx * bdy - bdx * ady);
    return -det.sign();   // |a-d,b-d,c-d| is an odd permutation of |b-a,c-a,d-a|
}

int orient3d(const double* a, const double* b, const double* c, const double* d) {
    const double adx = a[0] - d[0], bdx = b[0] - d[0], cdx = c[0] - d[0];
    const double ady = a[1] - d[1], bdy = b[1] - d[1], cdy = c[1] - d[1];
    const double adz = a[2] - d[2], bdz = b[2] - d[2], cdz = c[2] - d[2];
    const double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    const double cdxady = cdx * ady, adxcdy = adx * cdy;
    const double adxbdy = adx * bdy, bdxady = bdx * ady;
    const double det = adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy) + cdz * (adxbdy - bdxady);
    const double permanent = (std::fabs(bdxcdy) + std::fabs(cdxbdy)) * std::fabs(adz) +
                             (std::fabs(cdxady) + std::fabs(adxcdy)) * std::fabs(bdz) +
                             (std::fabs(adxbdy) + std::fabs(bdxady)) * std::fabs(cdz);
    const double errbound = kOrient3dBound * permanent;
    if (det > errbound || -det > errbound) return -sgn(det);
    return orient3d_exact(a, b, c, d);
}

// ---- in_sphere: src/predicates.cpp:76-113 (exact), :149-204 (filter), :206-232 --

int in_sphere_exact(const double* a, const double* b, const double* c, const double* d,
                    const double* e) {
    Scale s;
    for (const double* p : {a, b, c, d, e}) for (int k = 0; k < 3; ++k) s.add(p[k]);
    const Big ex = s(e[0]), ey = s(e[1]), ez = s(e[2]);
    const Big aex = s(a[0]) - ex, aey = s(a[1]) - ey, aez = s(a[2]) - ez;
    const Big bex = s(b[0]) - ex, bey = s(b[1]) - ey, bez = s(b[2]) - ez;
    const Big cex = s(c[0]) - ex, cey = s(c[1]) - ey, cez = s(c[2]) - ez;
    const Big dex = s(d[0]) - ex, dey = s(d[1]) - ey, dez = s(d[2]) - ez;
    const Big alift = aex * aex + aey * aey + aez * aez;
    const Big blift = bex * bex + bey * bey + bez * bez;
    const Big clift = cex * cex + cey * cey + cez * cez;
    const Big dlift = dex * dex + dey * dey + dez * dez;
    const Big ab = aex * bey - bex * aey, bc = bex * cey - cex * bey;
    const Big cd = cex * dey - dex * cey, da = dex * aey - aex * dey;
    const Big ac = aex * cey - cex * aey, bd = bex * dey - dex * bey;
    const Big abc = aez * bc - bez * ac + cez * ab;
    const Big bcd = bez * cd - cez * bd + dez * bc;
    const Big cda = cez * da + dez * ac + aez * cd;
    const Big dab = dez * ab + aez * bd + bez * da;
    const Big det = (dlift * abc - clift * dab) + (blift * cda - alift * bcd);
    return -det.sign();
}

int in_sphere_unperturbed(const double* a, const double* b, const double* c, const double* d,
                          const double* e) {
    const double aex = a[0] - e[0], aey = a[1] - e[1], aez = a[2] - e[2];
    const double bex = b[0] - e[0], bey = b[1] - e[1], bez = b[2] - e[2];
    const double cex = c[0] - e[0], cey = c[1] - e[1], cez = c[2] - e[2];
    const double dex = d[0] - e[0], dey = d[1] - e[1], dez = d[2] - e[2];
    const double ab = aex * bey - bex * aey;
    const double bc = bex * cey - cex * bey;
    const double cd = cex * dey - dex * cey;
    const double da = dex * aey - aex * dey;
    const double ac = aex * cey - cex * aey;
    const double bd = bex * dey - dex * bey;
    const double abc = aez * bc - bez * ac + cez * ab;
    const double bcd = bez * cd - cez * bd + dez * bc;
    const double cda = cez * da + dez * ac + aez * cd;
    const double dab = dez * ab + aez * bd + bez * da;
    const double alift = aex * aex + aey * aey + aez * aez;
    const double blift = bex * bex + bey * bey + bez * bez;
    const double clift = cex * cex + cey * cey + cez * cez;
    const double dlift = dex * dex + dey * dey + dez * dez;
    const double det = (dlift * abc - clift * dab) + (blift * cda - alift * bcd);
    const double aezplus = std::fabs(aez), bezplus = std::fabs(bez);
    const double cezplus = std::fabs(cez), dezplus = std::fabs(dez);
    const double aexbeyplus = std::fabs(aex * bey), bexaeyplus = std::fabs(bex * aey);
    const double bexceyplus = std::fabs(bex * cey), cexbeyplus = std::fabs(cex * bey);
    const double cexdeyplus = std::fabs(cex * dey), dexceyplus = std::fabs(dex * cey);
    const double dexaeyplus = std::fabs(dex * aey), aexdeyplus = std::fabs(aex * dey);
    const double aexceyplus = std::fabs(aex * cey), cexaeyplus = std::fabs(cex * aey);
    const double bexdeyplus = std::fabs(bex * dey), dexbeyplus = std::fabs(dex * bey);
    const double permanent =
        ((cexdeyplus + dexceyplus) * bezplus + (dexbeyplus + bexdeyplus) * cezplus +
         (bexceyplus + cexbeyplus) * dezplus) * alift +
        ((dexaeyplus + aexdeyplus) * cezplus + (aexceyplus + cexaeyplus) * dezplus +
         (cexdeyplus + dexceyplus) * aezplus) * blift +
        ((aexbeyplus + bexaeyplus) * dezplus + (bexdeyplus + dexbeyplus) * aezplus +
         (dexaeyplus + aexdeyplus) * bezplus) * clift +
        ((bexceyplus + cexbeyplus) * aezplus + (cexaeyplus + aexceyplus) * bezplus +
         (aexbeyplus + bexaeyplus) * cezplus) * dlift;
    const double errbound = kInSphereBound * permanent;
    if (det > errbound || -det > errbound) return -sgn(det);
    return in_sphere_exact(a, b, c, d, e);
}

bool lexico_less(const double* p, const double* q) {
    if (p[0] != q[0]) return p[0] < q[0];
    if (p[1] != q[1]) return p[1] < q[1];
    return p[2] < q[2];
}

/// Sorts pointers by lexico_less keeping ties in their original order, which is
/// what the reference's std::sort does on arrays this short (insertion sort).
template <int N>
void stable_lexico_sort(const double* (&p)[N]) {
    for (int i = 1; i < N; ++i) {
        const double* v = p[i];
        int j = i;
        while (j > 0 && lexico_less(v, p[j - 1])) { p[j] = p[j - 1]; --j; }
        p[j] = v;
    }
}

int in_sphere(const double* a, const double* b, const double* c, const double* d, const double* e) {
    const int s = in_sphere_unperturbed(a, b, c, d, e);
    if (s != 0) return s;
    const double* p[5] = {a, b, c, d, e};
    stable_lexico_sort<5>(p);
    for (int i = 4; i > 2; --i) {
        if (p[i] == e) return -1;
        int o;
        if (p[i] == d && (o = orient3d(a, b, c, e)) != 0) return o;
        if (p[i] == c && (o = orient3d(a, b, e, d)) != 0) return o;
        if (p[i] == b && (o = orient3d(a, e, c, d)) != 0) return o;
        if (p[i] == a && (o = orient3d(e, b, c, d)) != 0) return o;
    }
    return -1;
}

// ---- coplanar family: src/predicates2.cpp ---------------------------------------

int orient2d_exact(double px, double py, double qx, double qy, double rx, double ry) {
    Scale s;
    for (double v : {px, py, qx, qy, rx, ry}) s.add(v);
    const Big qpx = s(qx) - s(px), qpy = s(qy) - s(py), rpx = s(rx) - s(px), rpy = s(ry) - s(py);
    return (qpx * rpy - qpy * rpx).sign();
}

int orient2d(double px, double py, double qx, double qy, double rx, double ry) {   // :111-120
    const double qpx = qx - px, qpy = qy - py;
    const double rpx = rx - px, rpy = ry - py;
    const double a = qpx * rpy, b = qpy * rpx;
    const double det = a - b;
    const double permanent = std::fabs(a) + std::fabs(b);
    const double errbound = kOrient2dBound * permanent;
    if (det > errbound || -det > errbound) return sgn(det);
    return orient2d_exact(px, py, qx, qy, rx, ry);
}

int coplanar_orientation3(const double* p, const double* q, const double* r) {   // :122-132
    const int oxy = orient2d(p[0], p[1], q[0], q[1], r[0], r[1]);
    if (oxy != 0) return oxy;
    const int oyz = orient2d(p[1], p[2], q[1], q[2], r[1], r[2]);
    if (oyz != 0) return oyz;
    return orient2d(p[0], p[2], q[0], q[2], r[0], r[2]);
}

int coplanar_orientation4(const double* p, const double* q, const double* r, const double* s) {   // :134-146
    const int oxy = orient2d(p[0], p[1], q[0], q[1], r[0], r[1]);
    if (oxy != 0) return oxy * orient2d(p[0], p[1], q[0], q[1], s[0], s[1]);
    const int oyz = orient2d(p[1], p[2], q[1], q[2], r[1], r[2]);
    if (oyz != 0) return oyz * orient2d(p[1], p[2], q[1], q[2], s[1], s[2]);
    const int oxz = orient2d(p[0], p[2], q[0], q[2], r[0], r[2]);
    return oxz * orient2d(p[0], p[2], q[0], q[2], s[0], s[2]);
}

bool collinear(const double* p, const double* q, const double* r) {   // :148-156
    if (orient2d(r[0], r[1], p[0], p[1], q[0], q[1]) != 0) return false;
    if (orient2d(r[0], r[2], p[0], p[2], q[0], q[2]) != 0) return false;
    return orient2d(r[1], r[2], p[1], p[2], q[1], q[2]) == 0;
}

int in_circle_exact(const double* p, const double* q, const double* r, const double* t) {   // :60-101
    Scale s;
    for (const double* x : {p, q, r, t}) for (int k = 0; k < 3; ++k) s.add(x[k]);
    auto D = [&](double a, double b) { return s(a) - s(b); };
    const Big ptx = D(p[0], t[0]), pty = D(p[1], t[1]), ptz = D(p[2], t[2]);
    const Big qtx = D(q[0], t[0]), qty = D(q[1], t[1]), qtz = D(q[2], t[2]);
    const Big rtx = D(r[0], t[0]), rty = D(r[1], t[1]), rtz = D(r[2], t[2]);
    const Big pt2 = ptx * ptx + pty * pty + ptz * ptz;
    const Big qt2 = qtx * qtx + qty * qty + qtz * qtz;
    const Big rt2 = rtx * rtx + rty * rty + rtz * rtz;
    const Big pqx = D(q[0], p[0]), pqy = D(q[1], p[1]), pqz = D(q[2], p[2]);
    const Big prx = D(r[0], p[0]), pry = D(r[1], p[1]), prz = D(r[2], p[2]);
    const Big vx = pqy * prz - pqz * pry;
    const Big vy = pqz * prx - pqx * prz;
    const Big vz = pqx * pry - pqy * prx;
    const Big v2 = vx * vx + vy * vy + vz * vz;
    // Rows (pt, rt, qt, v) and the m01 = a10*a01 - a00*a11 minor convention.
    const Big &a00 = ptx, &a01 = pty, &a02 = ptz, &a03 = pt2;
    const Big &a10 = rtx, &a11 = rty, &a12 = rtz, &a13 = rt2;
    const Big &a20 = qtx, &a21 = qty, &a22 = qtz, &a23 = qt2;
    const Big &a30 = vx, &a31 = vy, &a32 = vz, &a33 = v2;
    const Big m01 = a10 * a01 - a00 * a11, m02 = a20 * a01 - a00 * a21;
    const Big m03 = a30 * a01 - a00 * a31, m12 = a20 * a11 - a10 * a21;
    const Big m13 = a30 * a11 - a10 * a31, m23 = a30 * a21 - a20 * a31;
    const Big m012 = m12 * a02 - m02 * a12 + m01 * a22;
    const Big m013 = m13 * a02 - m03 * a12 + m01 * a32;
    const Big m023 = m23 * a02 - m03 * a22 + m02 * a32;
    const Big m123 = m23 * a12 - m13 * a22 + m12 * a32;
    return (m123 * a03 - m023 * a13 + m013 * a23 - m012 * a33).sign();
}

int coplanar_in_circle_unperturbed(const double* p0, const double* p1, const double* p2,
                                   const double* p) {   // :182-234
    const double ptx = p0[0] - p[0], pty = p0[1] - p[1], ptz = p0[2] - p[2];
    const double qtx = p1[0] - p[0], qty = p1[1] - p[1], qtz = p1[2] - p[2];
    const double rtx = p2[0] - p[0], rty = p2[1] - p[1], rtz = p2[2] - p[2];
    const double pt2 = ptx * ptx + pty * pty + ptz * ptz;
    const double qt2 = qtx * qtx + qty * qty + qtz * qtz;
    const double rt2 = rtx * rtx + rty * rty + rtz * rtz;
    const double pqx = p1[0] - p0[0], pqy = p1[1] - p0[1], pqz = p1[2] - p0[2];
    const double prx = p2[0] - p0[0], pry = p2[1] - p0[1], prz = p2[2] - p0[2];
    const double vx = pqy * prz - pqz * pry;
    const double vy = pqz * prx - pqx * prz;
    const double vz = pqx * pry - pqy * prx;
    const double v2 = vx * vx + vy * vy + vz * vz;
    const double a00 = ptx, a01 = pty, a02 = ptz, a03 = pt2;
    const double a10 = rtx, a11 = rty, a12 = rtz, a13 = rt2;
    const double a20 = qtx, a21 = qty, a22 = qtz, a23 = qt2;
    const double a30 = vx, a31 = vy, a32 = vz, a33 = v2;
    const double m01 = a10 * a01 - a00 * a11;
    const double m02 = a20 * a01 - a00 * a21;
    const double m03 = a30 * a01 - a00 * a31;
    const double m12 = a20 * a11 - a10 * a21;
    const double m13 = a30 * a11 - a10 * a31;
    const double m23 = a30 * a21 - a20 * a31;
    const double m012 = m12 * a02 - m02 * a12 + m01 * a22;
    const double m013 = m13 * a02 - m03 * a12 + m01 * a32;
    const double m023 = m23 * a02 - m03 * a22 + m02 * a32;
    const double m123 = m23 * a12 - m13 * a22 + m12 * a32;
    const double det = m123 * a03 - m023 * a13 + m013 * a23 - m012 * a33;
    const double rows[4][4] = {{a00, a01, a02, a03}, {a10, a11, a12, a13},
                               {a20, a21, a22, a23}, {a30, a31, a32, a33}};
    double mag = 0.0;
    for (int i = 0; i < 4; ++i) {
        double row = 0.0;
        for (int j = 0; j < 4; ++j) row += std::fabs(rows[i][j]);
        mag = (mag == 0.0) ? row : mag * row;
    }
    const double errbound = kInCircleBound * mag;
    if (det > errbound || -det > errbound) return sgn(det);
    return in_circle_exact(p0, p1, p2, p);
}

int coplanar_in_circle(const double* p0, const double* p1, const double* p2, const double* p) {   // :236-259
    const int bs = coplanar_in_circle_unperturbed(p0, p1, p2, p);
    if (bs != 0) return bs;
    const double* pts[4] = {p0, p1, p2, p};
    stable_lexico_sort<4>(pts);
    const int local = coplanar_orientation3(p0, p1, p2);
    for (int i = 3; i > 0; --i) {
        if (pts[i] == p) return -1;
        int o;
        if (pts[i] == p2 && (o = coplanar_orientation3(p0, p1, p)) != 0) return o * local;
        if (pts[i] == p1 && (o = coplanar_orientation3(p0, p, p2)) != 0) return o * local;
        if (pts[i] == p0 && (o = coplanar_orientation3(p, p1, p2)) != 0) return o * local;
    }
    return -local;
}

// =============================================================================
// The insertion order: src/rand48.h and src/spatial_sort.cpp.
// =============================================================================

/// x <- (0x5DEECE66D x + 0xB) mod 2^48, output x >> 17 (src/rand48.h:26-50).
struct Rand48 {
    uint64_t x = ((uint64_t(1) << 16) | 0x330Eu);
    uint32_t next() {
        x = (0x5DEECE66Dull * x + 0xBull) & ((uint64_t(1) << 48) - 1);
        return uint32_t(x >> 17);
    }
};

/// Uniform integer in [0, k]: the bucket-and-reject branch of
/// generate_uniform_int (src/rand48.h:113-127), the only one Rand48 reaches.
uint32_t uniform_0_k(Rand48& g, uint64_t k) {
    const uint64_t brange = 0x7FFFFFFFull;
    const uint64_t bucket = (brange + 1) / (k + 1);
    for (;;) {
        const uint64_t r = uint64_t(g.next()) / bucket;
        if (r <= k) return uint32_t(r);
    }
}

struct SortCtx {
    const double* xyz;
    double coord(int i, int axis) const { return xyz[3 * int64_t(i) + axis]; }
};

/// Lomuto partition, src/spatial_sort.cpp:40-51; `right` is the last element.
int partition_lomuto(int* a, int left, int right, int pivot, const SortCtx& s, int axis, bool up) {
    std::swap(a[pivot], a[right]);
    const double pv = s.coord(a[right], axis);
    int result = left;
    for (int it = left; it != right; ++it) {
        const double cv = s.coord(a[it], axis);
        const bool less = up ? (pv < cv) : (cv < pv);
        if (less) { std::swap(a[result], a[it]); ++result; }
    }
    std::swap(a[right], a[result]);
    return result;
}

/// Middle-pivot quickselect, src/spatial_sort.cpp:60-71; [left, right).
void nth_select(int* a, int left, int nth, int right, const SortCtx& s, int axis, bool up) {
    if (left == right) return;
    --right;
    if (left == right) return;
    for (;;) {
        const int pivot = left + (right - left) / 2;
        const int np = partition_lomuto(a, left, right, pivot, s, axis, up);
        if (np == nth) return;
        if (nth < np) right = np - 1;
        else left = np + 1;
    }
}

int hilbert_split(int* a, int begin, int end, const SortCtx& s, int axis, bool up) {   // :74-79
    if (begin >= end) return begin;
    const int middle = begin + (end - begin) / 2;
    nth_select(a, begin, middle, end, s, axis, up);
    return middle;
}

void hilbert_rec(int* a, int begin, int end, const SortCtx& s, int x, bool ux, bool uy, bool uz) {   // :95-117
    const int y = (x + 1) % 3, z = (x + 2) % 3;
    if (end - begin <= 8) return;
    const int m0 = begin, m8 = end;
    const int m4 = hilbert_split(a, m0, m8, s, x, ux);
    const int m2 = hilbert_split(a, m0, m4, s, y, uy);
    const int m1 = hilbert_split(a, m0, m2, s, z, uz);
    const int m3 = hilbert_split(a, m2, m4, s, z, !uz);
    const int m6 = hilbert_split(a, m4, m8, s, y, !uy);
    const int m5 = hilbert_split(a, m4, m6, s, z, uz);
    const int m7 = hilbert_split(a, m6, m8, s, z, !uz);
    hilbert_rec(a, m0, m1, s, z, uz, ux, uy);
    hilbert_rec(a, m1, m2, s, y, uy, uz, ux);
    hilbert_rec(a, m2, m3, s, y, uy, uz, ux);
    hilbert_rec(a, m3, m4, s, x, ux, !uy, !uz);
    hilbert_rec(a, m4, m5, s, x, ux, !uy, !uz);
    hilbert_rec(a, m5, m6, s, y, !uy, uz, !ux);
    hilbert_rec(a, m6, m7, s, y, !uy, uz, !ux);
    hilbert_rec(a, m7, m8, s, z, !uz, !ux, uy);
}

void multiscale(int* a, int begin, int end, const SortCtx& s) {   // :130-137
    int middle = begin;
    if (end - begin >= 64) {
        middle = begin + int(double(end - begin) * 0.125);
        multiscale(a, begin, middle, s);
    }
    hilbert_rec(a, middle, end, s, 0, false, false, false);
}

void spatial_sort(const double* xyz, int n, int* order) {   // :141-151
    for (int i = 0; i < n; ++i) order[i] = i;
    if (n < 2) return;
    Rand48 g;
    for (int k = 1; k < n; ++k) std::swap(order[k], order[uniform_0_k(g, uint64_t(k))]);
    SortCtx s{xyz};
    multiscale(order, 0, n, s);
}

// =============================================================================
// The build: sequential Bowyer-Watson over the perturbed predicates.
//
// The reference inserts points in spatial-sort order through a dimension ladder
// (src/triangulation.cpp:65-120, 161-269) and re-stars each conflict region
// (src/tds.h:160-221, 634-683).  Because in_sphere never returns ZERO and the
// hull rule is fixed (src/triangulation.cpp:588-602), the set of finite cells
// does not depend on insertion order, so this restatement starts from any four
// affinely independent points and inserts the rest.  Duplicates keep the index
// of the copy that comes last in spatial-sort order (src/triangulation.cpp:77-81).
// =============================================================================

constexpr int kInf = -1;

struct TetRec {
    int v[4];
    int n[4];   // neighbour tet * 4 + its facet index facing back
    bool alive;
};

struct Builder {
    const double* pts;             // vertex coordinates, by vertex id
    std::vector<TetRec> tets;
    std::vector<int> free_slots;
    std::vector<int> vtet;         // one incident tet per vertex id

    const double* P(int v) const { return pts + 3 * int64_t(v); }

    int alloc() {
        if (!free_slots.empty()) { int t = free_slots.back(); free_slots.pop_back(); return t; }
        tets.push_back(TetRec{});
        return int(tets.size()) - 1;
    }

    bool has_inf(int t) const {
        const TetRec& c = tets[size_t(t)];
        return c.v[0] == kInf || c.v[1] == kInf || c.v[2] == kInf || c.v[3] == kInf;
    }

    /// src/triangulation.cpp:588-602.
    bool in_conflict(int t, const double* p) const {
        const TetRec& c = tets[size_t(t)];
        static const int kOrder[4][3] = {{2, 1, 3}, {2, 3, 0}, {1, 0, 3}, {0, 1, 2}};
        for (int i = 0; i < 4; ++i) {
            if (c.v[i] != kInf) continue;
            const double* a = P(c.v[kOrder[i][0]]);
            const double* b = P(c.v[kOrder[i][1]]);
            const double* d = P(c.v[kOrder[i][2]]);
            const int s = orient3d(a, b, d, p);
            if (s != 0) return s > 0;
            return coplanar_in_circle(a, b, d, p) > 0;
        }
        return in_sphere(P(c.v[0]), P(c.v[1]), P(c.v[2]), P(c.v[3]), p) > 0;
    }

    /// Visibility walk from tet `t` towards p; returns a tet in conflict with p
    /// (the finite tet containing it, or the infinite tet beyond the hull facet
    /// it crossed).
    int locate(int t, const double* p) const {
        if (has_inf(t)) {
            const TetRec& c = tets[size_t(t)];
            for (int i = 0; i < 4; ++i) if (c.v[i] == kInf) { t = c.n[i] >> 2; break; }
        }
        int prev = -1;
        uint32_t rng = 12345u;
        for (long step = 0;; ++step) {
            const TetRec& c = tets[size_t(t)];
            rng = rng * 1103515245u + 12345u;
            const int start = int((rng >> 16) & 3u);
            bool moved = false;
            for (int j = 0; j < 4 && !moved; ++j) {
                const int i = (start + j) & 3;
                const int nb = c.n[i] >> 2;
                if (nb == prev) continue;
                const double* q[4] = {P(c.v[0]), P(c.v[1]), P(c.v[2]), P(c.v[3])};
                q[i] = p;
                if (orient3d(q[0], q[1], q[2], q[3]) < 0) {
                    if (has_inf(nb)) return nb;
                    prev = t;
                    t = nb;
                    moved = true;
                }
            }
            if (!moved) return t;
        }
    }

    void link(int t0, int f0, int t1, int f1) {
        tets[size_t(t0)].n[f0] = t1 * 4 + f1;
        tets[size_t(t1)].n[f1] = t0 * 4 + f0;
    }

    void insert(int v, int seed) {
        const double* p = P(v);
        std::vector<int> cav{seed};
        std::vector<std::pair<int, int>> facets;   // (cavity tet, facet index)
        std::map<int, bool> seen{{seed, true}};
        for (size_t k = 0; k < cav.size(); ++k) {
            const int c = cav[k];
            for (int i = 0; i < 4; ++i) {
                const int nb = tets[size_t(c)].n[i] >> 2;
                auto it = seen.find(nb);
                bool conflict;
                if (it == seen.end()) {
                    conflict = in_conflict(nb, p);
                    seen[nb] = conflict;
                    if (conflict) cav.push_back(nb);
                } else {
                    conflict = it->second;
                }
                if (!conflict) facets.push_back({c, i});
            }
        }
        // One new tet per boundary facet: the cavity tet with vertex i replaced.
        std::vector<int> nt(facets.size());
        std::map<std::pair<int, int>, std::pair<int, int>> edge_face;   // edge -> (tet, facet)
        std::vector<std::array<int, 4>> verts(facets.size());
        std::vector<int> outer(facets.size());
        for (size_t k = 0; k < facets.size(); ++k) {
            const TetRec& c = tets[size_t(facets[k].first)];
            for (int j = 0; j < 4; ++j) verts[k][size_t(j)] = c.v[j];
            verts[k][size_t(facets[k].second)] = v;
            outer[k] = c.n[facets[k].second];
        }
        for (int c : cav) { tets[size_t(c)].alive = false; free_slots.push_back(c); }
        for (size_t k = 0; k < facets.size(); ++k) {
            nt[k] = alloc();
            TetRec& r = tets[size_t(nt[k])];
            for (int j = 0; j < 4; ++j) r.v[j] = verts[k][size_t(j)];
            r.alive = true;
        }
        for (size_t k = 0; k < facets.size(); ++k) {
            const int fi = facets[k].second;
            link(nt[k], fi, outer[k] >> 2, outer[k] & 3);
            for (int j = 0; j < 4; ++j) {
                if (j == fi) continue;
                int e[2], w = 0;
                for (int m = 0; m < 4; ++m) if (m != fi && m != j) e[w++] = verts[k][size_t(m)];
                const std::pair<int, int> key{std::min(e[0], e[1]), std::max(e[0], e[1])};
                auto it = edge_face.find(key);
                if (it == edge_face.end()) edge_face[key] = {nt[k], j};
                else { link(nt[k], j, it->second.first, it->second.second); edge_face.erase(it); }
            }
            for (int j = 0; j < 4; ++j) if (verts[k][size_t(j)] != kInf) vtet[size_t(verts[k][size_t(j)])] = nt[k];
        }
    }
};

struct Result {
    std::vector<std::array<int, 4>> cells, all;
    int64_t n_vertices = 0;
};

std::array<int, 4> canonical(std::array<int, 4> t) {
    // Even permutation bringing the minimum to slot 0 ...
    int m = 0;
    for (int i = 1; i < 4; ++i) if (t[size_t(i)] < t[size_t(m)]) m = i;
    switch (m) {
        case 1: t = {t[1], t[0], t[3], t[2]}; break;
        case 2: t = {t[2], t[3], t[0], t[1]}; break;
        case 3: t = {t[3], t[2], t[1], t[0]}; break;
        default: break;
    }
    // ... then a cyclic rotation of the remaining triple putting its minimum first.
    int r = 1;
    for (int i = 2; i < 4; ++i) if (t[size_t(i)] < t[size_t(r)]) r = i;
    if (r == 2) t = {t[0], t[2], t[3], t[1]};
    else if (r == 3) t = {t[0], t[3], t[1], t[2]};
    return t;
}

Result build(const double* xyz, int n) {
    Result res;
    if (n == 0) return res;
    std::vector<int> order(static_cast<size_t>(n));
    spatial_sort(xyz, n, order.data());
    std::vector<int> rank(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) rank[size_t(order[size_t(i)])] = i;

    // Duplicate groups (exact coordinate equality; -0.0 == 0.0 as in the reference).
    auto key = [&](int i) {
        std::array<double, 3> k{};
        for (int a = 0; a < 3; ++a) { double v = xyz[3 * int64_t(i) + a]; k[size_t(a)] = (v == 0.0) ? 0.0 : v; }
        return k;
    };
    std::map<std::array<double, 3>, int> group_of;   // coordinates -> vertex id
    std::vector<int> vert_point;                     // vertex id -> representative point index
    std::vector<double> vxyz;
    for (int r = 0; r < n; ++r) {
        const int i = order[size_t(r)];
        auto it = group_of.find(key(i));
        if (it == group_of.end()) {
            const int v = int(vert_point.size());
            group_of[key(i)] = v;
            vert_point.push_back(i);
            for (int a = 0; a < 3; ++a) vxyz.push_back(xyz[3 * int64_t(i) + a]);
        } else {
            vert_point[size_t(it->second)] = i;     // the later copy wins
        }
    }
    const int nv = int(vert_point.size());
    res.n_vertices = nv;

    Builder b;
    b.pts = vxyz.data();
    b.vtet.assign(size_t(nv), -1);
    const double* V0 = b.P(0);
    int i1 = -1, i2 = -1, i3 = -1;
    if (nv >= 2) i1 = 1;
    for (int k = 2; k < nv && i2 < 0; ++k) if (!collinear(V0, b.P(i1), b.P(k))) i2 = k;
    if (i2 >= 0)
        for (int k = 2; k < nv && i3 < 0; ++k)
            if (k != i2 && orient3d(V0, b.P(i1), b.P(i2), b.P(k)) != 0) i3 = k;
    if (i3 < 0) return res;   // collinear or coplanar: no cells

    int s0 = 0, s1 = i1;
    if (orient3d(b.P(s0), b.P(s1), b.P(i2), b.P(i3)) < 0) std::swap(s0, s1);
    const int T0v[4] = {s0, s1, i2, i3};
    // Tet 0 finite; tet 1+i infinite, opposite face i: vertex i replaced by the
    // infinite vertex and two finite slots swapped so it is positively oriented.
    for (int i = 0; i < 5; ++i) { b.alloc(); b.tets[size_t(i)].alive = true; }
    for (int j = 0; j < 4; ++j) b.tets[0].v[j] = T0v[j];
    for (int i = 0; i < 4; ++i) {
        int v4[4] = {T0v[0], T0v[1], T0v[2], T0v[3]};
        v4[i] = kInf;
        const int a = (i + 1) & 3, c = (i + 2) & 3;
        std::swap(v4[a], v4[c]);
        for (int j = 0; j < 4; ++j) b.tets[size_t(1 + i)].v[j] = v4[j];
    }
    // Glue the five tets by matching facets.
    for (int t = 0; t < 5; ++t)
        for (int f = 0; f < 4; ++f) {
            std::array<int, 3> ft{};
            for (int m = 0, w = 0; m < 4; ++m) if (m != f) ft[size_t(w++)] = b.tets[size_t(t)].v[m];
            std::sort(ft.begin(), ft.end());
            for (int u = 0; u < 5; ++u) {
                if (u == t) continue;
                for (int g = 0; g < 4; ++g) {
                    std::array<int, 3> fu{};
                    for (int m = 0, w = 0; m < 4; ++m) if (m != g) fu[size_t(w++)] = b.tets[size_t(u)].v[m];
                    std::sort(fu.begin(), fu.end());
                    if (fu == ft) b.tets[size_t(t)].n[f] = u * 4 + g;
                }
            }
        }
    for (int j = 0; j < 4; ++j) b.vtet[size_t(T0v[j])] = 0;

    int last = T0v[0];
    for (int v = 1; v < nv; ++v) {
        if (v == i1 || v == i2 || v == i3) continue;
        const int seed = b.locate(b.vtet[size_t(last)], b.P(v));
        b.insert(v, seed);
        last = v;
    }

    for (const TetRec& t : b.tets) {
        if (!t.alive) continue;
        std::array<int, 4> q{};
        bool inf = false;
        for (int j = 0; j < 4; ++j) {
            if (t.v[j] == kInf) { q[size_t(j)] = -1; inf = true; }
            else q[size_t(j)] = vert_point[size_t(t.v[j])];
        }
        res.all.push_back(canonical(q));
        if (!inf) res.cells.push_back(canonical(q));
    }
    std::sort(res.cells.begin(), res.cells.end());
    std::sort(res.all.begin(), res.all.end());
    return res;
}

bool all_finite(const double* xyz, int64_t n) {
    for (int64_t i = 0; i < 3 * n; ++i) if (!std::isfinite(xyz[i])) return false;
    return true;
}

inline const double* Q(const double* pts, int32_t i) { return pts + 3 * int64_t(i); }

}  // namespace

extern "C" {

void orc_orient3d(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 4 * q;
        out[q] = int8_t(orient3d(Q(pts, t[0]), Q(pts, t[1]), Q(pts, t[2]), Q(pts, t[3])));
    }
}

void orc_in_sphere(const double* pts, const int32_t* idx, int64_t nq, int perturbed, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 5 * q;
        const double *a = Q(pts, t[0]), *b = Q(pts, t[1]), *c = Q(pts, t[2]), *d = Q(pts, t[3]),
                     *e = Q(pts, t[4]);
        out[q] = int8_t(perturbed ? in_sphere(a, b, c, d, e) : in_sphere_unperturbed(a, b, c, d, e));
    }
}

void orc_orient2d(const double* six, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const double* s = six + 6 * q;
        out[q] = int8_t(orient2d(s[0], s[1], s[2], s[3], s[4], s[5]));
    }
}

void orc_coplanar_orientation3(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 3 * q;
        out[q] = int8_t(coplanar_orientation3(Q(pts, t[0]), Q(pts, t[1]), Q(pts, t[2])));
    }
}

void orc_coplanar_orientation4(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 4 * q;
        out[q] = int8_t(coplanar_orientation4(Q(pts, t[0]), Q(pts, t[1]), Q(pts, t[2]), Q(pts, t[3])));
    }
}

void orc_coplanar_in_circle(const double* pts, const int32_t* idx, int64_t nq, int perturbed,
                            int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 4 * q;
        const double *a = Q(pts, t[0]), *b = Q(pts, t[1]), *c = Q(pts, t[2]), *d = Q(pts, t[3]);
        out[q] = int8_t(perturbed ? coplanar_in_circle(a, b, c, d)
                                  : coplanar_in_circle_unperturbed(a, b, c, d));
    }
}

void orc_collinear(const double* pts, const int32_t* idx, int64_t nq, int8_t* out) {
    for (int64_t q = 0; q < nq; ++q) {
        const int32_t* t = idx + 3 * q;
        out[q] = int8_t(collinear(Q(pts, t[0]), Q(pts, t[1]), Q(pts, t[2])) ? 1 : 0);
    }
}

void orc_shuffle(int64_t n, int32_t* order) {
    for (int64_t i = 0; i < n; ++i) order[i] = int32_t(i);
    Rand48 g;
    for (int64_t k = 1; k < n; ++k) std::swap(order[k], order[uniform_0_k(g, uint64_t(k))]);
}

void orc_spatial_sort(const double* xyz, int64_t n, int32_t* order) {
    std::vector<int> o(static_cast<size_t>(n));
    spatial_sort(xyz, int(n), o.data());
    for (int64_t i = 0; i < n; ++i) order[i] = o[size_t(i)];
}

void* orc_build(const double* xyz, int64_t n) {
    if (!all_finite(xyz, n)) return nullptr;
    return new Result(build(xyz, int(n)));
}

int64_t orc_build_ncells(void* h) { return int64_t(static_cast<Result*>(h)->cells.size()); }
int64_t orc_build_nall(void* h) { return int64_t(static_cast<Result*>(h)->all.size()); }
int64_t orc_build_nvertices(void* h) { return static_cast<Result*>(h)->n_vertices; }

void orc_build_cells(void* h, int32_t* out) {
    const auto& c = static_cast<Result*>(h)->cells;
    for (size_t i = 0; i < c.size(); ++i) for (int k = 0; k < 4; ++k) out[4 * i + size_t(k)] = c[i][size_t(k)];
}

void orc_build_all(void* h, int32_t* out) {
    const auto& c = static_cast<Result*>(h)->all;
    for (size_t i = 0; i < c.size(); ++i) for (int k = 0; k < 4; ++k) out[4 * i + size_t(k)] = c[i][size_t(k)];
}

void orc_build_free(void* h) { delete static_cast<Result*>(h); }

void orc_canonical_rotate(int32_t* tets, int64_t nt) {
    for (int64_t i = 0; i < nt; ++i) {
        std::array<int, 4> t{tets[4 * i], tets[4 * i + 1], tets[4 * i + 2], tets[4 * i + 3]};
        t = canonical(t);
        for (int k = 0; k < 4; ++k) tets[4 * i + k] = t[size_t(k)];
    }
}

}  // extern "C"
