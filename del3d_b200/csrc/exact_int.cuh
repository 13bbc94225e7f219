// Fixed-width exact integer arithmetic for the exact stage of the predicates.
//
// Every finite double is M * 2^E with M a 53-bit integer.  For one predicate
// call, all coordinates involved are rewritten as integers times a common
// 2^emin (emin = the smallest E among them); that scales each determinant by a
// positive power of two and does not change its sign.  The determinant is then
// evaluated in two's-complement integers of L 64-bit limbs, with L chosen from
// the exponent span of the call so that no intermediate value can overflow.
//
// The reference evaluates its exact stage with floating-point expansions
// (src/expansion.h); the sign of an exact value is unique, so any exact
// evaluation returns the same sign.  Integers need no dynamic allocation and
// have a size known before the evaluation starts, which is what a GPU thread
// wants.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define D3G_HD __host__ __device__ __forceinline__
#define D3G_NOINLINE_HD static __host__ __device__ __noinline__
#else
#define D3G_HD inline
#define D3G_NOINLINE_HD static inline
#endif

namespace d3g {

D3G_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return uint64_t((unsigned __int128)a * b >> 64);
#endif
}

/// Integers of a fixed number L of 64-bit limbs, two's complement.  The limb
/// loops are unrolled; used for the common narrow cases (L = 2, 4).
template <int L>
struct WideS {
    uint64_t w[L];
};

/// Integers of a runtime number n <= 16 of limbs; the loops are not unrolled
/// and the operations are out-of-line, so one copy of the code serves every
/// width.  Used for wide exponent spans, which are rare.
constexpr int kMaxLimbs = 16;
struct WideV {
    uint64_t w[kMaxLimbs];
    int n;
};

// ---- limb kernels over raw arrays -------------------------------------------

D3G_HD void limbs_neg(uint64_t* a, int n) {
    uint64_t carry = 1;
    for (int i = 0; i < n; ++i) {
        const uint64_t v = ~a[i] + carry;
        carry = (carry && v == 0) ? 1 : 0;
        a[i] = v;
    }
}

D3G_HD void limbs_add(const uint64_t* a, const uint64_t* b, uint64_t* r, int n) {
    uint64_t carry = 0;
    for (int i = 0; i < n; ++i) {
        const uint64_t s = a[i] + b[i];
        const uint64_t c1 = s < a[i];
        const uint64_t t = s + carry;
        const uint64_t c2 = t < s;
        r[i] = t;
        carry = c1 | c2;
    }
}

D3G_HD void limbs_sub(const uint64_t* a, const uint64_t* b, uint64_t* r, int n) {
    uint64_t borrow = 0;
    for (int i = 0; i < n; ++i) {
        const uint64_t d = a[i] - b[i];
        const uint64_t b1 = a[i] < b[i];
        const uint64_t t = d - borrow;
        const uint64_t b2 = d < borrow;
        r[i] = t;
        borrow = b1 | b2;
    }
}

/// Unsigned product of magnitudes, truncated to n limbs (r must not alias).
D3G_HD void limbs_mul_mag(const uint64_t* a, const uint64_t* b, uint64_t* r, int n) {
    for (int i = 0; i < n; ++i) r[i] = 0;
    for (int i = 0; i < n; ++i) {
        if (a[i] == 0) continue;
        uint64_t carry = 0;
        for (int j = 0; i + j < n; ++j) {
            const uint64_t lo = a[i] * b[j];
            const uint64_t hi = mulhi64(a[i], b[j]);
            const uint64_t s = r[i + j] + lo;
            uint64_t c = s < lo;
            const uint64_t s2 = s + carry;
            c += s2 < s;
            r[i + j] = s2;
            carry = hi + c;     // a*b + r + carry < 2^128: cannot overflow
        }
    }
}

D3G_HD bool limbs_is_neg(const uint64_t* a, int n) { return (a[n - 1] >> 63) != 0; }

D3G_HD int limbs_sign(const uint64_t* a, int n) {
    if (limbs_is_neg(a, n)) return -1;
    uint64_t o = 0;
    for (int i = 0; i < n; ++i) o |= a[i];
    return o ? 1 : 0;
}

D3G_HD void limbs_mul(const uint64_t* a0, const uint64_t* b0, uint64_t* r, int n) {
    uint64_t a[kMaxLimbs], b[kMaxLimbs];
    for (int i = 0; i < n; ++i) { a[i] = a0[i]; b[i] = b0[i]; }
    const bool na = limbs_is_neg(a, n), nb = limbs_is_neg(b, n);
    if (na) limbs_neg(a, n);
    if (nb) limbs_neg(b, n);
    limbs_mul_mag(a, b, r, n);
    if (na != nb) limbs_neg(r, n);
}

// ---- fixed width: unrolled ----------------------------------------------------

template <int L>
D3G_HD WideS<L> operator+(const WideS<L>& a, const WideS<L>& b) {
    WideS<L> r;
    uint64_t carry = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        const uint64_t s = a.w[i] + b.w[i];
        const uint64_t c1 = s < a.w[i];
        const uint64_t t = s + carry;
        const uint64_t c2 = t < s;
        r.w[i] = t;
        carry = c1 | c2;
    }
    return r;
}

template <int L>
D3G_HD WideS<L> operator-(const WideS<L>& a, const WideS<L>& b) {
    WideS<L> r;
    uint64_t borrow = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        const uint64_t d = a.w[i] - b.w[i];
        const uint64_t b1 = a.w[i] < b.w[i];
        const uint64_t t = d - borrow;
        const uint64_t b2 = d < borrow;
        r.w[i] = t;
        borrow = b1 | b2;
    }
    return r;
}

template <int L>
D3G_HD void ws_neg(WideS<L>& a) {
    uint64_t carry = 1;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        const uint64_t v = ~a.w[i] + carry;
        carry = (carry && v == 0) ? 1 : 0;
        a.w[i] = v;
    }
}

template <int L>
D3G_HD WideS<L> operator*(WideS<L> a, WideS<L> b) {
    const bool na = (a.w[L - 1] >> 63) != 0, nb = (b.w[L - 1] >> 63) != 0;
    if (na) ws_neg(a);
    if (nb) ws_neg(b);
    WideS<L> r;
#pragma unroll
    for (int i = 0; i < L; ++i) r.w[i] = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        uint64_t carry = 0;
#pragma unroll
        for (int j = 0; i + j < L; ++j) {
            const uint64_t lo = a.w[i] * b.w[j];
            const uint64_t hi = mulhi64(a.w[i], b.w[j]);
            const uint64_t s = r.w[i + j] + lo;
            uint64_t c = s < lo;
            const uint64_t s2 = s + carry;
            c += s2 < s;
            r.w[i + j] = s2;
            carry = hi + c;
        }
    }
    if (na != nb) ws_neg(r);
    return r;
}

template <int L>
D3G_HD int num_sign(const WideS<L>& a) {
    if ((a.w[L - 1] >> 63) != 0) return -1;
    uint64_t o = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) o |= a.w[i];
    return o ? 1 : 0;
}

// ---- runtime width: out of line -------------------------------------------------

D3G_NOINLINE_HD WideV wv_add(const WideV& a, const WideV& b) {
    WideV r;
    r.n = a.n;
    limbs_add(a.w, b.w, r.w, a.n);
    return r;
}
D3G_NOINLINE_HD WideV wv_sub(const WideV& a, const WideV& b) {
    WideV r;
    r.n = a.n;
    limbs_sub(a.w, b.w, r.w, a.n);
    return r;
}
D3G_NOINLINE_HD WideV wv_mul(const WideV& a, const WideV& b) {
    WideV r;
    r.n = a.n;
    limbs_mul(a.w, b.w, r.w, a.n);
    return r;
}
D3G_HD WideV operator+(const WideV& a, const WideV& b) { return wv_add(a, b); }
D3G_HD WideV operator-(const WideV& a, const WideV& b) { return wv_sub(a, b); }
D3G_HD WideV operator*(const WideV& a, const WideV& b) { return wv_mul(a, b); }
D3G_HD int num_sign(const WideV& a) { return limbs_sign(a.w, a.n); }

/// Decomposition of a double: |x| = m * 2^e with m < 2^53 (m = 0 for x = 0).
struct Decomp {
    uint64_t m;
    int e;
    bool neg;
};

D3G_HD Decomp decompose(double x) {
    uint64_t bits;
#if defined(__CUDA_ARCH__)
    bits = uint64_t(__double_as_longlong(x));
#else
    __builtin_memcpy(&bits, &x, 8);
#endif
    Decomp d;
    d.neg = (bits >> 63) != 0;
    const int be = int((bits >> 52) & 0x7FF);
    const uint64_t frac = bits & ((uint64_t(1) << 52) - 1);
    if (be == 0) {                    // zero or subnormal
        d.m = frac;
        d.e = -1074;
    } else {
        d.m = frac | (uint64_t(1) << 52);
        d.e = be - 1075;
    }
    return d;
}

D3G_HD int ctz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __ffsll((long long)x) - 1;
#else
    return __builtin_ctzll(x);
#endif
}

D3G_HD int clz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

/// Exponent span of a group of coordinates: `emin` is the exponent of the
/// lowest set bit over all nonzero values, `top` the exponent just above the
/// highest set bit.  Every value is then an integer multiple of 2^emin of
/// magnitude below 2^top, i.e. an integer of at most `top - emin` bits.
struct Span {
    int emin = 1 << 20;
    int top = -(1 << 20);
    D3G_HD void add(double x) {
        if (x == 0.0) return;
        const Decomp d = decompose(x);
        const int lo = d.e + ctz64(d.m);
        const int hi = d.e + 64 - clz64(d.m);
        if (lo < emin) emin = lo;
        if (hi > top) top = hi;
    }
    D3G_HD bool empty() const { return top < emin; }
    D3G_HD int bits() const { return empty() ? 0 : top - emin; }
    /// True if a polynomial of the given degree in coordinate differences,
    /// whose exact value needs at most `degree * (bits + 1) + extra` bits, is
    /// computed without any rounding (and without underflow or overflow) by
    /// plain double arithmetic: then the filter's own value is exact.
    D3G_HD bool exact_in_double(int degree, int extra) const {
        if (empty()) return true;
        return degree * (bits() + 1) + extra <= 53 && degree * emin >= -1000 &&
               degree * (top + 1) + extra <= 1000;
    }
};

/// Writes x / 2^emin (an integer: emin is at most x's lowest set bit) into n
/// limbs, two's complement.
D3G_HD void limbs_from(double x, int emin, uint64_t* r, int n) {
    for (int i = 0; i < n; ++i) r[i] = 0;
    if (x == 0.0) return;
    const Decomp d = decompose(x);
    const int tz = ctz64(d.m);
    const uint64_t m = d.m >> tz;
    const int shift = d.e + tz - emin;        // >= 0 by construction of emin
    const int limb = shift >> 6, bit = shift & 63;
    if (limb < n) r[limb] = m << bit;
    if (bit != 0 && limb + 1 < n) r[limb + 1] = m >> (64 - bit);
    if (d.neg) limbs_neg(r, n);
}

/// Conversion of a coordinate into the number type N of an exact evaluation.
template <class N>
struct NumFrom;

template <int L>
struct NumFrom<WideS<L>> {
    int emin;
    D3G_HD WideS<L> operator()(double x) const {
        WideS<L> r;
        limbs_from(x, emin, r.w, L);
        return r;
    }
};

template <>
struct NumFrom<WideV> {
    int emin;
    int n;
    D3G_HD WideV operator()(double x) const {
        WideV r;
        r.n = n;
        limbs_from(x, emin, r.w, n);
        return r;
    }
};

}  // namespace d3g
