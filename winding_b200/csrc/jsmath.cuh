// The JavaScript number arithmetic the reference's capture readers use
// (src/scene/splats.js, src/render/hdr.js), restated for the device and the
// host with one fixed result for every input:
//
//   exp_js      Math.exp as the double nearest the real exponential. The
//               reference leaves it to the engine (V8's is within an ulp);
//               the nearest double is what every engine approximates. It is
//               evaluated in double-double arithmetic (about 104 bits):
//               x = k ln 2 + r, |r| <= ln 2 / 2, exp(r) by its Taylor series
//               in Horner form 1 + r (1 + r/2 (1 + r/3 (...))) to 25 terms,
//               then scaled by 2^k with exact multiplications by powers of
//               two (a result below 2^-1022, x < -708.39, is rounded to a
//               double first and then to the subnormal grid: no reader's
//               byte or f32 output can tell). Double-double operations are the error-free
//               transformations of Dekker and Knuth (two-sum, Dekker's
//               split and two-product), so no fused multiply-add is needed
//               and the result does not depend on the compiler contracting.
//   js_round    Math.round: the nearest integer, halves towards +infinity.
//   js_byte     byte() of the readers: max(0, min(255, round(v * 255))), and
//               0 for NaN (ToInt32 of NaN, where the reader packs the bytes).
//   half_bits   halfBits (render/hdr.js:152-163): the nearest half float of
//               a positive value, halves rounded up, 0x7bff from 65504 on,
//               0 below 2^-24; floor(log2 v) taken exactly from the exponent
//               (the reference's log2 can be an ulp off only next to a power
//               of two, where its own correction gives the same bits).
//   signed_half signedHalf (scene/splats.js:50-52).
//   from_half   fromHalf (scene/splats.js:219-225), exact.
//
// Compiled with contraction off on both sides (nvcc -fmad=false, host
// -ffp-contract=off), every + - * / below is one IEEE double operation.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define JS_HD __host__ __device__ __forceinline__
#else
#define JS_HD inline
#endif

namespace jsmath {

struct dd {
    double hi, lo;
};

JS_HD dd two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}

JS_HD dd quick_two_sum(double a, double b) {
    const double s = a + b;
    return {s, b - (s - a)};
}

JS_HD void split(double a, double* hi, double* lo) {
    const double c = 134217729.0 * a;   // 2^27 + 1
    const double t = c - a;
    *hi = c - t;
    *lo = a - *hi;
}

JS_HD dd two_prod(double a, double b) {
    const double p = a * b;
    double ah, al, bh, bl;
    split(a, &ah, &al);
    split(b, &bh, &bl);
    const double e = (((ah * bh - p) + ah * bl) + al * bh) + al * bl;
    return {p, e};
}

JS_HD dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    const dd t = two_sum(a.lo, b.lo);
    s.lo = s.lo + t.hi;
    s = quick_two_sum(s.hi, s.lo);
    s.lo = s.lo + t.lo;
    return quick_two_sum(s.hi, s.lo);
}

JS_HD dd dd_mul(dd a, dd b) {
    dd p = two_prod(a.hi, b.hi);
    p.lo = p.lo + (a.hi * b.lo + a.lo * b.hi);
    return quick_two_sum(p.hi, p.lo);
}

JS_HD dd dd_div(dd a, double b) {
    const double q1 = a.hi / b;
    const dd p = two_prod(q1, b);
    dd r = two_sum(a.hi, -p.hi);
    r.lo = r.lo - p.lo;
    r.lo = r.lo + a.lo;
    const double q2 = (r.hi + r.lo) / b;
    return quick_two_sum(q1, q2);
}

JS_HD double pow2(int e) {   // e in [-1022, 1023]
    const uint64_t bits = (uint64_t)(e + 1023) << 52;
    double d;
    memcpy(&d, &bits, 8);
    return d;
}

JS_HD double exp_js(double x) {
    if (x != x) return x;
    if (x > 1000.0) return INFINITY;
    if (x < -1000.0) return 0.0;
    const double k = rint(x * 1.4426950408889634);   // nearest, ties to even
    // ln 2 as a double-double: 0x3FE62E42FEFA39EF + 0x3C7ABC9E3B39803F.
    dd kl = two_prod(k, 6.93147180559945286227e-01);
    kl.lo = kl.lo + k * 2.31904681384629955842e-17;
    const dd r = dd_add(dd{x, 0.0}, dd{-kl.hi, -kl.lo});
    dd s{1.0, 0.0};
    for (int n = 25; n >= 1; --n) s = dd_add(dd{1.0, 0.0}, dd_div(dd_mul(r, s), (double)n));
    // 2^k in two exact steps and one rounding (|k| <= 1443 here).
    double y = s.hi;
    int ki = (int)k;
    if (ki > 1023) {
        y = y * pow2(ki - 1023);
        ki = 1023;
    } else if (ki < -1022) {
        y = y * pow2(ki + 1022);
        ki = -1022;
    }
    return y * pow2(ki);
}

JS_HD double js_round(double x) {
    if (!(x == x) || x == INFINITY || x == -INFINITY) return x;
    const double f = std::floor(x);
    return (x - f >= 0.5) ? f + 1.0 : f;
}

JS_HD uint32_t js_byte(double v) {
    const double r = js_round(v * 255.0);
    if (r != r) return 0u;
    return (uint32_t)(r < 0.0 ? 0.0 : (r > 255.0 ? 255.0 : r));
}

JS_HD uint32_t half_bits(double value) {
    if (!(value > 0.0)) return 0u;
    if (value >= 65504.0) return 0x7bffu;
    if (value < 5.9604644775390625e-08) return 0u;                 // 2^-24
    if (value < 6.103515625e-05) return (uint32_t)js_round(value * 16777216.0);   // 2^-14, / 2^-24
    int e;
    std::frexp(value, &e);
    int exponent = e - 1;
    uint32_t mantissa = (uint32_t)js_round((value * pow2(-exponent) - 1.0) * 1024.0);
    if (mantissa == 1024u) {
        mantissa = 0u;
        ++exponent;
    }
    return ((uint32_t)(exponent + 15) << 10) | mantissa;
}

JS_HD uint32_t signed_half(double v) { return v < 0.0 ? (0x8000u | half_bits(-v)) : half_bits(v); }

JS_HD double from_half(uint32_t h) {
    const double sign = (h & 0x8000u) ? -1.0 : 1.0;
    const int exponent = (int)((h >> 10) & 31u);
    const uint32_t mantissa = h & 1023u;
    if (exponent == 31) return mantissa ? NAN : sign * INFINITY;
    return sign * (exponent == 0 ? (double)mantissa * 5.9604644775390625e-08
                                 : (1.0 + (double)mantissa / 1024.0) * pow2(exponent - 15));
}

}  // namespace jsmath
