// put() of the reference's capture readers (src/scene/splats.js:335-369) on
// the device: the covariance M M^T with M = R(q / |q|) diag(scale), in FP64
// with separately rounded IEEE ops in the reference's evaluation order,
// rounded to f32 at the end. |q| is Math.hypot as V8 computes it (the
// largest magnitude factored out, the squares of the quotients summed with
// Kahan compensation), then `|| 1`.
#pragma once

#include <cstdint>

namespace wsort {

__device__ __forceinline__ double v8_hypot4(double a, double b, double c, double d) {
    const double v[4] = {fabs(a), fabs(b), fabs(c), fabs(d)};
    // ECMAScript: any infinite argument gives +Infinity, else any NaN NaN.
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (isinf(v[k])) return INFINITY;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (isnan(v[k])) return NAN;
    double m = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (v[k] > m) m = v[k];
    if (m == 0.0) return 0.0;
    double sum = 0.0, comp = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double n = __ddiv_rn(v[k], m);
        const double summand = __dsub_rn(__dmul_rn(n, n), comp);
        const double prelim = __dadd_rn(sum, summand);
        comp = __dsub_rn(__dsub_rn(prelim, sum), summand);
        sum = prelim;
    }
    return __dmul_rn(__dsqrt_rn(sum), m);
}

#define DM(a, b) __dmul_rn((a), (b))
#define DA(a, b) __dadd_rn((a), (b))
#define DS(a, b) __dsub_rn((a), (b))

// put() (src/scene/splats.js:335-369) from its FP64 inputs: the covariance
// M M^T, M = R(q / |q|) diag(s), rounded to f32 at the end.
__device__ __forceinline__ void covariance_d(double sx, double sy, double sz, double qw, double qx, double qy,
                                             double qz, float out[6]) {
    double length = v8_hypot4(qw, qx, qy, qz);
    if (!(length != 0.0)) length = 1.0;   // `|| 1` (0 and NaN are falsy)
    const double w = __ddiv_rn(qw, length), u = __ddiv_rn(qx, length);
    const double v = __ddiv_rn(qy, length), t = __ddiv_rn(qz, length);
    const double r00 = DS(1.0, DM(2.0, DA(DM(v, v), DM(t, t))));
    const double r01 = DM(2.0, DS(DM(u, v), DM(w, t)));
    const double r02 = DM(2.0, DA(DM(u, t), DM(w, v)));
    const double r10 = DM(2.0, DA(DM(u, v), DM(w, t)));
    const double r11 = DS(1.0, DM(2.0, DA(DM(u, u), DM(t, t))));
    const double r12 = DM(2.0, DS(DM(v, t), DM(w, u)));
    const double r20 = DM(2.0, DS(DM(u, t), DM(w, v)));
    const double r21 = DM(2.0, DA(DM(v, t), DM(w, u)));
    const double r22 = DS(1.0, DM(2.0, DA(DM(u, u), DM(v, v))));
    const double m00 = DM(r00, sx), m01 = DM(r01, sy), m02 = DM(r02, sz);
    const double m10 = DM(r10, sx), m11 = DM(r11, sy), m12 = DM(r12, sz);
    const double m20 = DM(r20, sx), m21 = DM(r21, sy), m22 = DM(r22, sz);
    out[0] = __double2float_rn(DA(DA(DM(m00, m00), DM(m01, m01)), DM(m02, m02)));
    out[1] = __double2float_rn(DA(DA(DM(m00, m10), DM(m01, m11)), DM(m02, m12)));
    out[2] = __double2float_rn(DA(DA(DM(m00, m20), DM(m01, m21)), DM(m02, m22)));
    out[3] = __double2float_rn(DA(DA(DM(m10, m10), DM(m11, m11)), DM(m12, m12)));
    out[4] = __double2float_rn(DA(DA(DM(m10, m20), DM(m11, m21)), DM(m12, m22)));
    out[5] = __double2float_rn(DA(DA(DM(m20, m20), DM(m21, m21)), DM(m22, m22)));
}

#undef DM
#undef DA
#undef DS

}  // namespace wsort
