// Decoding .splat records into a resident cloud.
//
// Restates put() and parseSplatFile (src/scene/splats.js:335-388 of the
// reference) on the device: centre, colour word, and the covariance
// M M^T with M = R(q / |q|) diag(scale), all in FP64 with separately rounded
// IEEE ops in the reference's evaluation order, rounded to f32 at the end.
// |q| is Math.hypot as V8 computes it (the largest magnitude factored out,
// the squares of the quotients summed with Kahan compensation), then `|| 1`.
// The box around the centres and the index of the first non-finite position
// are reduced with atomics on order-preserving integer images of the floats.
#include "wsort_dev.cuh"

namespace wsort {

__device__ __forceinline__ uint32_t ordered(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ double v8_hypot4(double a, double b, double c, double d) {
    const double v[4] = {fabs(a), fabs(b), fabs(c), fabs(d)};
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

__device__ __forceinline__ void covariance(float fsx, float fsy, float fsz, uint32_t rot, float out[6]) {
    const double sx = fsx, sy = fsy, sz = fsz;
    const double qw = __ddiv_rn(double((int)(rot & 255u) - 128), 128.0);
    const double qx = __ddiv_rn(double((int)((rot >> 8) & 255u) - 128), 128.0);
    const double qy = __ddiv_rn(double((int)((rot >> 16) & 255u) - 128), 128.0);
    const double qz = __ddiv_rn(double((int)(rot >> 24) - 128), 128.0);
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

// bounds: 3 ordered minima then 3 ordered maxima (initialised by the host to
// 0xFFFFFFFF and 0), then the ordered maximum of |covariance entry| over the
// cloud (initialised to 0); bad: first non-finite index (initialised to
// 0xFFFFFFFF).
__global__ void __launch_bounds__(256) decode_kernel(const uint4* __restrict__ rec, uint32_t n,
                                                     float4* __restrict__ centers, float2* __restrict__ cov,
                                                     int8_t* __restrict__ sexp, uint32_t* __restrict__ bounds,
                                                     uint32_t* __restrict__ bad) {
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
    uint32_t hi[3] = {0u, 0u, 0u};
    uint32_t smax = 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint4 a = __ldcs(&rec[2 * (size_t)i]);
        const uint4 b = __ldcs(&rec[2 * (size_t)i + 1]);
        const float x = __uint_as_float(a.x), y = __uint_as_float(a.y), z = __uint_as_float(a.z);
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) {
            atomicMin(bad, i);
            continue;
        }
        centers[i] = make_float4(x, y, z, __uint_as_float(b.z));
        float c[6];
        covariance(__uint_as_float(a.w), __uint_as_float(b.x), __uint_as_float(b.y), b.w, c);
        cov[3 * (size_t)i] = make_float2(c[0], c[1]);
        cov[3 * (size_t)i + 1] = make_float2(c[2], c[3]);
        cov[3 * (size_t)i + 2] = make_float2(c[4], c[5]);
        float m = 0.0f;
#pragma unroll
        for (int k = 0; k < 6; ++k) m = fmaxf(m, fabsf(c[k]));
        bool finite = true;
#pragma unroll
        for (int k = 0; k < 6; ++k) finite = finite && isfinite(c[k]);
        // The least e with max |entry| <= 2^e (frexp: m = f 2^e, f in [.5, 1)),
        // clamped to [-100, 127]; 127 for a non-finite entry.
        int e = -100;
        if (!finite) {
            e = 127;
        } else if (m > 0.0f) {
            frexpf(m, &e);
            e = e < -100 ? -100 : (e > 127 ? 127 : e);
        }
        sexp[i] = (int8_t)e;
#pragma unroll
        for (int k = 0; k < 6; ++k) smax = max(smax, ordered(fabsf(c[k])));
        const uint32_t o[3] = {ordered(x), ordered(y), ordered(z)};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = min(lo[k], o[k]);
            hi[k] = max(hi[k], o[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
            hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) smax = max(smax, __shfl_xor_sync(0xffffffffu, smax, off));
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (lo[k] != 0xFFFFFFFFu) atomicMin(&bounds[k], lo[k]);
            if (hi[k] != 0u) atomicMax(&bounds[3 + k], hi[k]);
        }
        if (smax != 0u) atomicMax(&bounds[6], smax);
    }
}

cudaError_t launch_decode(const void* records, uint32_t n, float4* centers, float2* cov, int8_t* sexp,
                          uint32_t* bounds, uint32_t* bad, int sms, cudaStream_t stream) {
    const uint32_t want = (n + 255) / 256;
    const uint32_t grid = want < (uint32_t)sms * 8u ? (want ? want : 1u) : (uint32_t)sms * 8u;
    decode_kernel<<<grid, 256, 0, stream>>>(static_cast<const uint4*>(records), n, centers, cov, sexp, bounds, bad);
    return cudaGetLastError();
}

}  // namespace wsort
