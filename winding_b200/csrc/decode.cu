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
#include "put.cuh"
#include "wsort_dev.cuh"

namespace wsort {

__device__ __forceinline__ uint32_t ordered(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// A .splat record's covariance: f32 scales, rotation bytes (b - 128) / 128.
__device__ __forceinline__ void covariance(float fsx, float fsy, float fsz, uint32_t rot, float out[6]) {
    const double qw = __ddiv_rn(double((int)(rot & 255u) - 128), 128.0);
    const double qx = __ddiv_rn(double((int)((rot >> 8) & 255u) - 128), 128.0);
    const double qy = __ddiv_rn(double((int)((rot >> 16) & 255u) - 128), 128.0);
    const double qz = __ddiv_rn(double((int)(rot >> 24) - 128), 128.0);
    covariance_d(fsx, fsy, fsz, qw, qx, qy, qz, out);
}

// bounds: 3 ordered minima then 3 ordered maxima (initialised by the host to
// 0xFFFFFFFF and 0); bad: first non-finite index (initialised to 0xFFFFFFFF).
__global__ void __launch_bounds__(256) decode_kernel(const uint4* __restrict__ rec, uint32_t n,
                                                     float4* __restrict__ centers, float2* __restrict__ cov,
                                                     int8_t* __restrict__ sexp, uint32_t* __restrict__ bounds,
                                                     uint32_t* __restrict__ bad, uint32_t first) {
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
    uint32_t hi[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint4 a = __ldcs(&rec[2 * (size_t)i]);
        const uint4 b = __ldcs(&rec[2 * (size_t)i + 1]);
        const float x = __uint_as_float(a.x), y = __uint_as_float(a.y), z = __uint_as_float(a.z);
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) {
            atomicMin(bad, first + i);
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
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (lo[k] != 0xFFFFFFFFu) atomicMin(&bounds[k], lo[k]);
            if (hi[k] != 0u) atomicMax(&bounds[3 + k], hi[k]);
        }
    }
}

// Decodes records [0, n) into splats first .. first + n - 1 of the cloud's
// arrays (centers, cov and sexp point at splat 0); bad receives the least
// cloud index of a record whose position is not finite.
cudaError_t launch_decode(const void* records, uint32_t n, float4* centers, float2* cov, int8_t* sexp,
                          uint32_t* bounds, uint32_t* bad, int sms, cudaStream_t stream, uint32_t first) {
    const uint32_t want = (n + 255) / 256;
    const uint32_t grid = want < (uint32_t)sms * 8u ? (want ? want : 1u) : (uint32_t)sms * 8u;
    decode_kernel<<<grid, 256, 0, stream>>>(static_cast<const uint4*>(records), n, centers + first,
                                            cov + 3 * (size_t)first, sexp + first, bounds, bad, first);
    return cudaGetLastError();
}

}  // namespace wsort
