// x^(1/4) rounded as the C library's powf(x, 0.25f) rounds it, on the device
// (and on the host, for the exhaustive check of this function).
//
// The reference's 2D solvers raise smoke to the power 0.25f with std::pow,
// which is the C library's powf. That powf is not correctly rounded: for about
// 0.07% of inputs it returns the float one ulp away from the correctly
// rounded x^(1/4). The device computes the correctly rounded value (two IEEE
// double square roots, one rounding to float; the double result is within
// 1.5 double ulps of the exact root, far inside the float rounding margin
// except at those same near-midpoint inputs) and then applies the library's
// differences from powf_quarter_table.inc (generated by gen_powf_quarter.cpp
// from powf itself): one table per period of four binades, where x * 16 maps
// to 2 x^(1/4) exactly, plus the 32 inputs that break the period.
// +0 and -0 give +0, as powf does; infinity gives infinity. Negative inputs
// give a NaN (payload unspecified).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define VB_POWQ_TABLE static __device__ const
#define VB_POWQ_FN __device__ __forceinline__
#else
#define VB_POWQ_TABLE static const
#define VB_POWQ_FN inline
#endif

namespace vb {
namespace powq {

#include "powf_quarter_table.inc"

#ifdef __CUDACC__
VB_POWQ_FN uint32_t bits_of(float x) { return __float_as_uint(x); }
VB_POWQ_FN float float_of(uint32_t b) { return __uint_as_float(b); }
#else
inline uint32_t bits_of(float x) {
    uint32_t b;
    std::memcpy(&b, &x, 4);
    return b;
}
inline float float_of(uint32_t b) {
    float x;
    std::memcpy(&x, &b, 4);
    return x;
}
#endif

// (unbiased exponent mod 4) << 23 | mantissa of a positive finite float.
VB_POWQ_FN uint32_t period_class(uint32_t b) {
    int e = int(b >> 23);
    uint32_t m = b & 0x7FFFFFu;
    if (e == 0) {  // subnormal: normalise (m != 0)
        while (!(m & 0x800000u)) {
            m <<= 1;
            --e;
        }
        m &= 0x7FFFFFu;
        e += 1;
    }
    return (uint32_t((e - 127) & 3) << 23) | m;
}

// Index of the first entry >= key in a sorted array, or count.
VB_POWQ_FN int lower_bound(const uint32_t* a, int count, uint32_t key) {
    int lo = 0, hi = count;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

}  // namespace powq

// powf(x, 0.25f) of the C library, bit for bit, for x >= 0 (and +-0, inf).
VB_POWQ_FN float powf_quarter(float x) {
    if (x == 0.f) return 0.f;
    const float rounded = float(sqrt(sqrt(double(x))));
    const uint32_t b = powq::bits_of(x);
    if (b >= 0x7F800000u) return rounded;  // +inf, NaN, negative
    const int e = powq::lower_bound(powq::kQuarterExactIn, powq::kQuarterExactCount, b);
    if (e < powq::kQuarterExactCount && powq::kQuarterExactIn[e] == b) return powq::float_of(powq::kQuarterExactOut[e]);
    const uint32_t key = powq::period_class(b) << 1;
    const int k = powq::lower_bound(powq::kQuarterPeriodic, powq::kQuarterPeriodicCount, key);
    if (k < powq::kQuarterPeriodicCount && (powq::kQuarterPeriodic[k] >> 1) == (key >> 1)) {
        // one ulp up or down; the result is a positive normal float
        const uint32_t r = powq::bits_of(rounded);
        return powq::float_of((powq::kQuarterPeriodic[k] & 1u) ? r + 1u : r - 1u);
    }
    return rounded;
}

}  // namespace vb
