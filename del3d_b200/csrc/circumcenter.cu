// Circumcentres of tetrahedra on the device: the reference's `circumcenter`
// (exact numerator and denominator, one rounding each, then a double quotient)
// and `circumcenter_lazy` (directed-rounding interval evaluation, midpoint
// accepted at 1e-5 relative, exact fallback per coordinate).
//
// Reference: src/triangulation.cpp:805-852 (circumcenter), :854-930
// (circumcenter_lazy, det3), src/interval.h:56-202 (Interval).
//
// Exact form.  The reference forms nx, ny, nz and den = 2 a.(b x c) in
// floating-point expansions and rounds each with Expansion::to_double
// (src/expansion.h:95-99, a smallest-first sum of the components).  Here the
// same polynomials are evaluated in fixed-width integers on the common binary
// scale of the four points (exact_int.cuh) and each is rounded to the nearest
// double (ties to even); the quotient and the translation back by p0 are the
// same two double operations as the reference's.  Where the expansion sum is
// the nearest double - every case met in the tests - the result is bit-identical;
// a smallest-first expansion sum can differ from the nearest double by one
// unit in the last place, which bounds the difference at 4 ulp of the quotient
// plus 1 ulp of the result per coordinate.
//
// Lazy form.  The reference switches the FPU to round-upward and evaluates
// intervals stored as (-inf, sup); every operation here is the same double
// operation with an explicit round-upward intrinsic (__dadd_ru, __dmul_ru,
// __ddiv_ru), the branches of the interval product, quotient and square are
// the reference's, and the accept-or-refine test and midpoint are computed the
// same way - so the lazy result is bit-identical whenever no coordinate needs
// the exact fallback.
#include "common.cuh"
#include "exact_int.cuh"

#include <cuda_runtime.h>

namespace d3g {
namespace {

// ---- exact numerator / denominator -------------------------------------------

/// Bits [pos, pos + 64) of the magnitude w[0..n) (bits outside the array are 0).
__device__ __forceinline__ uint64_t window64(const uint64_t* w, int n, int pos) {
    if (pos <= -64) return 0;
    if (pos < 0) return w[0] << (-pos);
    const int li = pos >> 6, sh = pos & 63;
    const uint64_t lo = li < n ? (w[li] >> sh) : 0;
    const uint64_t hi = (sh != 0 && li + 1 < n) ? (w[li + 1] << (64 - sh)) : 0;
    return lo | hi;
}

/// Nearest double (ties to even) to the two's-complement integer w[0..n) times
/// 2^e2, including the subnormal range and overflow to infinity.
__device__ double limbs_to_double(const uint64_t* w_in, int n, int e2) {
    uint64_t w[kMaxLimbs];
    for (int i = 0; i < n; ++i) w[i] = w_in[i];
    const bool neg = limbs_is_neg(w, n);
    if (neg) limbs_neg(w, n);
    int top = -1;
    for (int i = n - 1; i >= 0; --i)
        if (w[i]) {
            top = 64 * i + 63 - clz64(w[i]);
            break;
        }
    if (top < 0) return 0.0;
    const int E = top + e2;                          // |value| in [2^E, 2^(E+1))
    const int keep = E < -1022 ? 53 - (-1022 - E) : 53;   // significant bits kept (<= 0: below
                                                     // half the smallest subnormal or just at it)
    const int low = top - keep + 1;                  // lowest kept bit position
    uint64_t m = keep > 0 ? (window64(w, n, low) & ((uint64_t(1) << keep) - 1)) : 0;
    const int g = low - 1;                           // guard bit position
    const uint64_t guard = (g >= 0 && g < 64 * n) ? ((w[g >> 6] >> (g & 63)) & 1u) : 0;
    bool sticky = false;
    if (g > 0) {
        const int li = g >> 6, sh = g & 63;
        if (li < n) sticky = (w[li] & ((uint64_t(1) << sh) - 1)) != 0;
        for (int i = 0; i < li && i < n && !sticky; ++i) sticky = w[i] != 0;
    }
    if (guard && (sticky || (m & 1u))) m += 1;
    const double r = ldexp(double(m), low + e2);    // exact: at most 2^53 times a power of two
    return neg ? -r : r;
}

template <int L>
__device__ __forceinline__ int num_limbs(const WideS<L>&) { return L; }
__device__ __forceinline__ int num_limbs(const WideV& a) { return a.n; }
template <int L>
__device__ __forceinline__ const uint64_t* limb_ptr(const WideS<L>& a) { return a.w; }
__device__ __forceinline__ const uint64_t* limb_ptr(const WideV& a) { return a.w; }

struct ExactCenter {
    double nx, ny, nz, den;   // each the nearest double to the exact value
    bool coplanar;
    bool capacity;
};

/// nx, ny, nz, den of the reference's closed form, exact then rounded.
/// N: WideS<L> or WideV.  `emin`: the common scale of the coordinates.
template <class N>
__device__ ExactCenter exact_center(const double* p0, const double* p1, const double* p2,
                                    const double* p3, const NumFrom<N>& from, int emin) {
    const N x0 = from(p0[0]), y0 = from(p0[1]), z0 = from(p0[2]);
    const N ax = from(p1[0]) - x0, ay = from(p1[1]) - y0, az = from(p1[2]) - z0;
    const N bx = from(p2[0]) - x0, by = from(p2[1]) - y0, bz = from(p2[2]) - z0;
    const N cx = from(p3[0]) - x0, cy = from(p3[1]) - y0, cz = from(p3[2]) - z0;
    const N bcx = by * cz - bz * cy, bcy = bz * cx - bx * cz, bcz = bx * cy - by * cx;
    const N cax = cy * az - cz * ay, cay = cz * ax - cx * az, caz = cx * ay - cy * ax;
    const N abx = ay * bz - az * by, aby = az * bx - ax * bz, abz = ax * by - ay * bx;
    const N a2 = ax * ax + ay * ay + az * az;
    const N b2 = bx * bx + by * by + bz * bz;
    const N c2 = cx * cx + cy * cy + cz * cz;
    const N nx = a2 * bcx + b2 * cax + c2 * abx;
    const N ny = a2 * bcy + b2 * cay + c2 * aby;
    const N nz = a2 * bcz + b2 * caz + c2 * abz;
    const N vol = ax * bcx + ay * bcy + az * bcz;
    ExactCenter r;
    r.capacity = false;
    r.coplanar = num_sign(vol) == 0;
    const int n = num_limbs(nx);
    r.nx = limbs_to_double(limb_ptr(nx), n, 4 * emin);
    r.ny = limbs_to_double(limb_ptr(ny), n, 4 * emin);
    r.nz = limbs_to_double(limb_ptr(nz), n, 4 * emin);
    r.den = limbs_to_double(limb_ptr(vol), n, 3 * emin + 1);   // 2 * vol
    return r;
}

/// The exact numerator and denominator for the four points, in the narrowest
/// integer width their exponent span allows.  A span needing more than 16
/// limbs reports capacity.
__device__ ExactCenter exact_center_any(const double* p0, const double* p1, const double* p2,
                                        const double* p3) {
    Span sp;
    for (int k = 0; k < 3; ++k) {
        sp.add(p0[k]);
        sp.add(p1[k]);
        sp.add(p2[k]);
        sp.add(p3[k]);
    }
    ExactCenter r;
    if (sp.empty()) {                      // all coordinates zero: coplanar
        r.coplanar = true;
        r.capacity = false;
        r.nx = r.ny = r.nz = r.den = 0.0;
        return r;
    }
    // Differences need bits+1 bits; the numerators are degree 4 in them with
    // at most 2^5 terms of equal sign, plus a sign bit.
    const int need = 4 * (sp.bits() + 1) + 6 + 1;
    if (need <= 128) return exact_center<WideS<2>>(p0, p1, p2, p3, NumFrom<WideS<2>>{sp.emin}, sp.emin);
    if (need <= 256) return exact_center<WideS<4>>(p0, p1, p2, p3, NumFrom<WideS<4>>{sp.emin}, sp.emin);
    const int limbs = (need + 63) / 64;
    if (limbs > kMaxLimbs) {
        r.capacity = true;
        r.coplanar = false;
        r.nx = r.ny = r.nz = r.den = 0.0;
        return r;
    }
    return exact_center<WideV>(p0, p1, p2, p3, NumFrom<WideV>{sp.emin, limbs}, sp.emin);
}

/// del3d::circumcenter (src/triangulation.cpp:805-852).  Returns false on
/// exact-stage capacity.
__device__ bool circumcenter_exact(const double* p0, const double* p1, const double* p2,
                                   const double* p3, double out[3]) {
    const ExactCenter e = exact_center_any(p0, p1, p2, p3);
    if (e.capacity) return false;
    if (e.coplanar) {
        out[0] = p0[0];
        out[1] = p0[1];
        out[2] = p0[2];
        return true;
    }
    out[0] = __dadd_rn(p0[0], __ddiv_rn(e.nx, e.den));
    out[1] = __dadd_rn(p0[1], __ddiv_rn(e.ny, e.den));
    out[2] = __dadd_rn(p0[2], __ddiv_rn(e.nz, e.den));
    return true;
}

// ---- intervals with upward rounding (src/interval.h) ----------------------------

/// [inf, sup] stored as (ni = -inf, s = sup); every bound is one upward-rounded
/// operation.
struct Iv {
    double ni, s;
    __device__ double inf() const { return -ni; }
    __device__ double sup() const { return s; }
};

__device__ __forceinline__ Iv iv_point(double d) { return Iv{-d, d}; }
__device__ __forceinline__ Iv iv_make(double i, double s) { return Iv{-i, s}; }
__device__ __forceinline__ double ru_mul(double a, double b) { return __dmul_ru(a, b); }
__device__ __forceinline__ double ru_div(double a, double b) { return __ddiv_ru(a, b); }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }   // std::max

__device__ Iv iv_add(const Iv& a, const Iv& b) {
    return iv_make(-__dadd_ru(-a.inf(), -b.inf()), __dadd_ru(a.sup(), b.sup()));
}
__device__ Iv iv_sub(const Iv& a, const Iv& b) {
    return iv_make(-__dadd_ru(-a.inf(), b.sup()), __dadd_ru(a.sup(), -b.inf()));
}

/// Interval product: the sign case analysis of interval.h:88-120.
__device__ Iv iv_mul(const Iv& a, const Iv& b) {
    if (a.inf() >= 0.0) {
        double aa = a.inf(), bb = a.sup();
        if (bb <= 0.0) return iv_point(0.0);
        if (b.inf() < 0.0) {
            aa = bb;
            if (b.sup() < 0.0) bb = a.inf();
        }
        const double r = (b.sup() == 0) ? 0.0 : ru_mul(bb, b.sup());
        return iv_make(-ru_mul(aa, -b.inf()), r);
    }
    if (a.sup() <= 0.0) {
        double aa = a.sup(), bb = a.inf();
        if (b.inf() < 0.0) {
            aa = bb;
            if (b.sup() <= 0.0) bb = a.sup();
        } else if (b.sup() <= 0) {
            return iv_point(0.0);
        }
        return iv_make(-ru_mul(-bb, b.sup()), ru_mul(-aa, -b.inf()));
    }
    if (b.inf() >= 0.0) {
        if (b.sup() <= 0.0) return iv_point(0.0);
        return iv_make(-ru_mul(-a.inf(), b.sup()), ru_mul(a.sup(), b.sup()));
    }
    if (b.sup() <= 0.0) return iv_make(-ru_mul(a.sup(), -b.inf()), ru_mul(-a.inf(), -b.inf()));
    const double t1 = ru_mul(-a.inf(), b.sup());
    const double t2 = ru_mul(a.sup(), -b.inf());
    const double t3 = ru_mul(-a.inf(), -b.inf());
    const double t4 = ru_mul(a.sup(), b.sup());
    return iv_make(-dmax(t1, t2), dmax(t3, t4));
}

/// Interval quotient (interval.h:124-142); a divisor containing 0 gives the
/// whole line.
__device__ Iv iv_div(const Iv& a, const Iv& b) {
    if (b.inf() > 0.0) {
        double aa = b.sup(), bb = b.inf();
        if (a.inf() < 0.0) {
            aa = bb;
            if (a.sup() < 0.0) bb = b.sup();
        }
        return iv_make(-ru_div(-a.inf(), aa), ru_div(a.sup(), bb));
    }
    if (b.sup() < 0.0) {
        double aa = b.sup(), bb = b.inf();
        if (a.inf() < 0.0) {
            bb = aa;
            if (a.sup() < 0.0) aa = b.inf();
        }
        return iv_make(-ru_div(a.sup(), -aa), ru_div(a.inf(), bb));
    }
    const double inf = __longlong_as_double(0x7FF0000000000000LL);
    return iv_make(-inf, inf);
}

/// Square (interval.h:149-154): lower bound 0 for an interval straddling 0.
__device__ Iv iv_square(const Iv& d) {
    if (d.inf() >= 0.0) return iv_make(-ru_mul(-d.inf(), d.inf()), ru_mul(d.sup(), d.sup()));
    if (d.sup() <= 0.0) return iv_make(-ru_mul(d.sup(), -d.sup()), ru_mul(-d.inf(), -d.inf()));
    const double m = dmax(-d.inf(), d.sup());
    return iv_make(0.0, ru_mul(m, m));
}

/// 3x3 determinant with the reference's fixed association (triangulation.cpp:861-871).
__device__ Iv iv_det3(const Iv& a00, const Iv& a01, const Iv& a02, const Iv& a10, const Iv& a11,
                      const Iv& a12, const Iv& a20, const Iv& a21, const Iv& a22) {
    const Iv m01 = iv_sub(iv_mul(a00, a11), iv_mul(a10, a01));
    const Iv m02 = iv_sub(iv_mul(a00, a21), iv_mul(a20, a01));
    const Iv m12 = iv_sub(iv_mul(a10, a21), iv_mul(a20, a11));
    return iv_add(iv_sub(iv_mul(m01, a22), iv_mul(m02, a12)), iv_mul(m12, a02));
}

/// Interval -> double decision of circumcenter_lazy (triangulation.cpp:908-917):
/// 0 = the bound (a point interval), 1 = the midpoint, 2 = exact needed.
__device__ int iv_pick(const Iv& v, double* out) {
    const double lo = v.inf(), hi = v.sup();
    if (hi == lo) {
        *out = lo;
        return 0;
    }
    const double mag = dmax(fabs(lo), fabs(hi));
    const double width = __dadd_ru(hi, -lo);
    const double radius = __ddiv_ru(width, 2.0);
    const double kPrec = 0.00001;
    if (mag == 0 || radius < __dmul_ru(kPrec, mag)) {
        *out = __dmul_ru(__dadd_ru(hi, lo), 0.5);
        return 1;
    }
    return 2;
}

/// del3d::circumcenter_lazy.  Returns false on exact-stage capacity; sets
/// *refined when a coordinate needed the exact fallback.
__device__ bool circumcenter_lazy(const double* p, const double* q, const double* r, const double* s,
                                  double out[3], bool* refined) {
    const Iv px = iv_point(p[0]), py = iv_point(p[1]), pz = iv_point(p[2]);
    const Iv qpx = iv_sub(iv_point(q[0]), px), qpy = iv_sub(iv_point(q[1]), py),
             qpz = iv_sub(iv_point(q[2]), pz);
    const Iv qp2 = iv_add(iv_add(iv_square(qpx), iv_square(qpy)), iv_square(qpz));
    const Iv rpx = iv_sub(iv_point(r[0]), px), rpy = iv_sub(iv_point(r[1]), py),
             rpz = iv_sub(iv_point(r[2]), pz);
    const Iv rp2 = iv_add(iv_add(iv_square(rpx), iv_square(rpy)), iv_square(rpz));
    const Iv spx = iv_sub(iv_point(s[0]), px), spy = iv_sub(iv_point(s[1]), py),
             spz = iv_sub(iv_point(s[2]), pz);
    const Iv sp2 = iv_add(iv_add(iv_square(spx), iv_square(spy)), iv_square(spz));

    const Iv num_x = iv_det3(qpy, qpz, qp2, rpy, rpz, rp2, spy, spz, sp2);
    const Iv num_y = iv_det3(qpx, qpz, qp2, rpx, rpz, rp2, spx, spz, sp2);
    const Iv num_z = iv_det3(qpx, qpy, qp2, rpx, rpy, rp2, spx, spy, sp2);
    const Iv den = iv_det3(qpx, qpy, qpz, rpx, rpy, rpz, spx, spy, spz);

    const Iv inv = iv_div(iv_point(1.0), iv_mul(iv_point(2.0), den));
    const Iv cx = iv_add(px, iv_mul(num_x, inv));
    const Iv cy = iv_sub(py, iv_mul(num_y, inv));
    const Iv cz = iv_add(pz, iv_mul(num_z, inv));

    const int kx = iv_pick(cx, &out[0]);
    const int ky = iv_pick(cy, &out[1]);
    const int kz = iv_pick(cz, &out[2]);
    *refined = false;
    if (kx == 2 || ky == 2 || kz == 2) {
        *refined = true;
        double ex[3];
        if (!circumcenter_exact(p, q, r, s, ex)) return false;
        if (kx == 2) out[0] = ex[0];
        if (ky == 2) out[1] = ex[1];
        if (kz == 2) out[2] = ex[2];
    }
    return true;
}

__global__ void __launch_bounds__(128) k_circumcenters(const double* __restrict__ pts, int64_t npts,
                                                       const int32_t* __restrict__ tets, int64_t nt,
                                                       int lazy, double* __restrict__ out,
                                                       unsigned long long* __restrict__ counters) {
    // counters[0]: status bits, counters[1]: tets that needed exact arithmetic
    unsigned long long n_exact = 0;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nt;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int32_t i0 = tets[4 * t], i1 = tets[4 * t + 1], i2 = tets[4 * t + 2], i3 = tets[4 * t + 3];
        double r[3];
        if (i0 < 0 || i1 < 0 || i2 < 0 || i3 < 0 || i0 >= npts || i1 >= npts || i2 >= npts ||
            i3 >= npts) {
            atomicOr(&counters[0], (unsigned long long)ST_INTERNAL);
            const double nan = __longlong_as_double(0x7FF8000000000000LL);
            out[3 * t] = out[3 * t + 1] = out[3 * t + 2] = nan;
            continue;
        }
        const double *a = pts + 3 * int64_t(i0), *b = pts + 3 * int64_t(i1), *c = pts + 3 * int64_t(i2),
                     *d = pts + 3 * int64_t(i3);
        bool ok, refined = true;
        if (lazy)
            ok = circumcenter_lazy(a, b, c, d, r, &refined);
        else
            ok = circumcenter_exact(a, b, c, d, r);
        if (!ok) {
            atomicOr(&counters[0], (unsigned long long)ST_EXACT_CAPACITY);
            const double nan = __longlong_as_double(0x7FF8000000000000LL);
            r[0] = r[1] = r[2] = nan;
        }
        n_exact += refined ? 1 : 0;
        out[3 * t] = r[0];
        out[3 * t + 1] = r[1];
        out[3 * t + 2] = r[2];
    }
    if (n_exact) atomicAdd(&counters[1], n_exact);
}

}  // namespace

int circumcenters_device(const double* d_pts, int64_t n_pts, const int32_t* d_tets, int64_t n_tets,
                         int lazy, double* d_out, cudaStream_t stream, d3g_predicate_stats* stats) {
    if (n_tets < 0 || n_pts < 0) {
        set_error("d3g_circumcenters: negative size");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    if (n_tets == 0) {
        if (stats) *stats = d3g_predicate_stats{0, 0};
        return D3G_OK;
    }
    if (!d_pts || !d_tets || !d_out) {
        set_error("d3g_circumcenters: null pointer");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    D3G_TRY(prepare_device());
    DevBuf<unsigned long long> counters;
    D3G_TRY(counters.alloc(2, stream));
    D3G_CUDA(cudaMemsetAsync(counters.p, 0, 2 * sizeof(unsigned long long), stream));
    k_circumcenters<<<grid_for(n_tets, 128, int64_t(kNumSMs) * 16), 128, 0, stream>>>(
        d_pts, n_pts, d_tets, n_tets, lazy ? 1 : 0, d_out, counters.p);
    D3G_CUDA(cudaGetLastError());
    unsigned long long host[2] = {0, 0};
    D3G_CUDA(cudaMemcpyAsync(host, counters.p, sizeof host, cudaMemcpyDeviceToHost, stream));
    counters.release();
    D3G_CUDA(cudaStreamSynchronize(stream));
    if (stats) *stats = d3g_predicate_stats{n_tets, int64_t(host[1])};
    const uint32_t bits = uint32_t(host[0]);
    if (bits & ST_INTERNAL) {
        set_error("d3g_circumcenters: point index out of range");
        return D3G_ERR_INVALID_INPUT;
    }
    return status_from_bits(bits);
}

}  // namespace d3g

using namespace d3g;

extern "C" {

int d3g_circumcenters_device(const double* d_pts, int64_t n_pts, const int32_t* d_tets, int64_t n_tets,
                             int lazy, double* d_out, void* stream, d3g_predicate_stats* stats) {
    return circumcenters_device(d_pts, n_pts, d_tets, n_tets, lazy, d_out,
                                static_cast<cudaStream_t>(stream), stats);
}

int d3g_circumcenters(const double* pts, int64_t n_pts, const int32_t* tets, int64_t n_tets, int lazy,
                      double* out, d3g_predicate_stats* stats) {
    if (n_pts < 0 || n_tets < 0) return D3G_ERR_INVALID_ARGUMENT;
    if (n_tets == 0) {
        if (stats) *stats = d3g_predicate_stats{0, 0};
        return D3G_OK;
    }
    if (!pts || !tets || !out) return D3G_ERR_INVALID_ARGUMENT;
    D3G_TRY(ensure_device());
    cudaStream_t s = nullptr;
    DevBuf<double> dp, dout;
    DevBuf<int32_t> dt;
    D3G_TRY(dp.alloc(size_t(3 * n_pts > 0 ? 3 * n_pts : 1), s));
    D3G_TRY(dt.alloc(size_t(4 * n_tets), s));
    D3G_TRY(dout.alloc(size_t(3 * n_tets), s));
    if (n_pts > 0)
        D3G_CUDA(cudaMemcpyAsync(dp.p, pts, sizeof(double) * 3 * n_pts, cudaMemcpyHostToDevice, s));
    D3G_CUDA(cudaMemcpyAsync(dt.p, tets, sizeof(int32_t) * 4 * n_tets, cudaMemcpyHostToDevice, s));
    const int st = circumcenters_device(dp.p, n_pts, dt.p, n_tets, lazy, dout.p, s, stats);
    if (st != D3G_OK) return st;
    D3G_CUDA(cudaMemcpyAsync(out, dout.p, sizeof(double) * 3 * n_tets, cudaMemcpyDeviceToHost, s));
    D3G_CUDA(cudaStreamSynchronize(s));
    return D3G_OK;
}

}  // extern "C"
