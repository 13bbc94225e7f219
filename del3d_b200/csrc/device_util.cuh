// Small device utilities shared by the sort and the build: scans and radix
// sorts (CUB, compiled into this library), bounding boxes, key helpers.
#pragma once

#include "common.cuh"

#include <cub/cub.cuh>

namespace d3g {

/// Exclusive prefix sum of n ints (in place allowed), on `s`.
template <class T>
int exclusive_scan(const T* in, T* out, int64_t n, cudaStream_t s) {
    if (n <= 0) return D3G_OK;
    size_t bytes = 0;
    D3G_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    DevBuf<char> tmp;
    D3G_TRY(tmp.alloc(bytes, s));
    D3G_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, in, out, n, s));
    return D3G_OK;
}

/// Stable radix sort of (key, value) pairs over bits [begin_bit, end_bit).
template <class K, class V>
int sort_pairs(const K* kin, K* kout, const V* vin, V* vout, int64_t n, int begin_bit, int end_bit,
               cudaStream_t s) {
    if (n <= 0) return D3G_OK;
    size_t bytes = 0;
    D3G_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, begin_bit,
                                             end_bit, s));
    DevBuf<char> tmp;
    D3G_TRY(tmp.alloc(bytes, s));
    D3G_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, kin, kout, vin, vout, n, begin_bit,
                                             end_bit, s));
    return D3G_OK;
}

/// Bits needed to represent values in [0, v].
inline int bits_for(uint64_t v) {
    int b = 1;
    while (b < 64 && (v >> b) != 0) ++b;
    return b;
}

/// Ordered-integer image of a double (monotone: a < b <=> key(a) < key(b)).
__device__ __forceinline__ unsigned long long dbl_order_key(double x) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dbl_from_order_key(unsigned long long k) {
    const unsigned long long b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    return __longlong_as_double((long long)b);
}

}  // namespace d3g
