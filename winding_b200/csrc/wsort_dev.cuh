// Device-side definitions shared by the decode and sort kernels.
//
// The key arithmetic here follows makeKeys and footprint of the reference
// (src/render/splats.js:102-124, :155-186) with one pinned evaluation order:
// every f32 operation is a separately rounded IEEE op (__fmul_rn, __fadd_rn,
// __fdiv_rn, __fsqrt_rn; the library is also built with -fmad=false),
// sums run left to right in the order the WGSL source writes them, and a
// matrix-vector product is the column sum col0*v0 + col1*v1 + col2*v2 + col3*v3.
// The per-cloud depth range (src/render/splats.js:561-582) is computed in
// FP64 with __dmul_rn / __dadd_rn / __ddiv_rn, as the reference's JavaScript
// computes it in doubles before storing f32.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace wsort {

constexpr uint32_t kBuckets = 65536u;     // render/splats.js:64
constexpr uint32_t kCulled = 0xFFFFFFFFu;
constexpr int kThreads = 256;             // threads per CTA of every sort kernel
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kPadSplats = 4096;     // resident clouds are padded to this multiple

// Look-back status word: 2 flag bits over a 30-bit count.
constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1;

// Error codes a kernel leaves in LaunchCtl::error.
constexpr uint32_t kErrWaitPhase = 1;     // a phase dependency never completed
constexpr uint32_t kErrWaitLookback = 2;  // a predecessor tile never published
constexpr uint32_t kErrBounds = 3;        // a scatter position fell outside the output

// One (cloud, view) to sort, as the persistent kernel reads it.
struct alignas(16) JobDesc {
    // cloud (resident)
    const float4* centers;      // x, y, z, colour word bits; padded to kPadSplats
    const float2* cov;          // 6 f32 a splat as 3 float2; padded likewise
    double bmin[3], bmax[3];    // box around the centres
    uint32_t n;
    uint32_t tiles1, tiles2, tiles3;
    // view: the values the reference writes into its Cloud uniform
    float mv[16];
    float proj[16];
    float viewport[2];
    float cull;
    uint32_t pad0;
    // outputs
    uint32_t* order;            // >= n
    uint32_t* keys;             // >= n, or null
    uint32_t* count;            // 1
    // scratch
    uint16_t* k16;              // per splat key (survivors) ; n_pad
    uint32_t* mask;             // survivor bits, one word per 32 splats
    uint16_t* key_b;            // low-digit pass output: keys
    uint32_t* idx_b;            // low-digit pass output: splat indices
    uint32_t* status;           // look-back words: (tiles2 + tiles3) * 256
    uint32_t* ctl;              // JobCtl
};

// Per-job counters, zeroed before a launch.
struct JobCtl {
    uint32_t hist[2][256];      // survivor digit histograms: low byte, high byte
    uint32_t p1_done;           // key tiles whose writes are visible
    uint32_t p2_done;           // low-digit tiles whose writes are visible
    uint32_t pad[14];
};
static_assert(sizeof(JobCtl) % 64 == 0, "JobCtl size");

// Per-launch counters, zeroed before a launch.
struct LaunchCtl {
    uint32_t ticket;            // next work item
    uint32_t error;             // first error code
    uint32_t error_item;        // the item that raised it
    uint32_t exited;            // CTAs that left the loop
    uint32_t pad[12];
};

// Work item: x = job, y = phase << 30 | tile.
constexpr uint32_t kPhaseKeys = 0, kPhaseLow = 1, kPhaseHigh = 2;

// ---------------------------------------------------------------- f32 ops
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
// WGSL clamp(e, low, high) = min(max(e, low), high); fmaxf/fminf return the
// non-NaN operand.
__device__ __forceinline__ float fclamp(float e, float lo, float hi) { return fminf(fmaxf(e, lo), hi); }

// Per-view constants of one job, computed once per work item. Each is the
// same IEEE operation on the same operands the per-splat WGSL evaluates, so
// hoisting them changes no bit.
struct ViewConsts {
    float mv[16];
    float proj[16];
    float fx, fy;               // p[0][0] * viewport.x * 0.5, p[1][1] * viewport.y * 0.5
    float xlo, xhi, ylo, yhi;   // -1.3 / p[0][0], 1.3 / p[0][0], and for p[1][1]
    float cull;
    float depth_min, depth_scale;
    int persp;                  // p[3][3] == 0
    int visible;                // far > 0
};

// The depth range in FP64 (render/splats.js:561-582).
__device__ __forceinline__ void depth_range(const JobDesc& J, float* depth_min, float* depth_scale,
                                            int* visible) {
    const double m2 = J.mv[2], m6 = J.mv[6], m10 = J.mv[10], m14 = J.mv[14];
    double nearv = __longlong_as_double(0x7ff0000000000000ll);   // +inf
    double farv = -nearv;
    for (int k = 0; k < 8; ++k) {
        const double x = (k & 1) ? J.bmax[0] : J.bmin[0];
        const double y = (k & 2) ? J.bmax[1] : J.bmin[1];
        const double z = (k & 4) ? J.bmax[2] : J.bmin[2];
        const double s = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m2, x), __dmul_rn(m6, y)), __dmul_rn(m10, z)), m14);
        const double depth = -s;
        if (depth < nearv) nearv = depth;
        if (depth > farv) farv = depth;
    }
    *visible = farv > 0.0;
    nearv = nearv > 0.0 ? nearv : 0.0;
    const double span = __dsub_rn(farv, nearv);
    *depth_min = __double2float_rn(nearv);
    *depth_scale = __double2float_rn(__ddiv_rn(65535.0, span > 1e-6 ? span : 1e-6));
}

__device__ __forceinline__ void make_consts(const JobDesc& J, ViewConsts& c) {
    for (int k = 0; k < 16; ++k) {
        c.mv[k] = J.mv[k];
        c.proj[k] = J.proj[k];
    }
    const float p0 = J.proj[0], p5 = J.proj[5];
    c.fx = fmul(fmul(p0, J.viewport[0]), 0.5f);
    c.fy = fmul(fmul(p5, J.viewport[1]), 0.5f);
    c.xlo = fdiv(-1.3f, p0);
    c.xhi = fdiv(1.3f, p0);
    c.ylo = fdiv(-1.3f, p5);
    c.yhi = fdiv(1.3f, p5);
    c.cull = J.cull;
    c.persp = J.proj[15] == 0.0f;
    depth_range(J, &c.depth_min, &c.depth_scale, &c.visible);
}

// view = modelView * (x, y, z, 1) and clip = projection * view.
__device__ __forceinline__ void transform(const ViewConsts& c, float x, float y, float z, float view[4],
                                          float clip[4]) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
        view[j] = fadd(fadd(fadd(fmul(c.mv[j], x), fmul(c.mv[4 + j], y)), fmul(c.mv[8 + j], z)),
                       fmul(c.mv[12 + j], 1.0f));
#pragma unroll
    for (int j = 0; j < 4; ++j)
        clip[j] = fadd(fadd(fadd(fmul(c.proj[j], view[0]), fmul(c.proj[4 + j], view[1])),
                            fmul(c.proj[8 + j], view[2])),
                       fmul(c.proj[12 + j], view[3]));
}

// Frustum and faintness tests (render/splats.js:163-170). Returns alpha, or a
// negative value when culled.
__device__ __forceinline__ float frustum_alpha(const float view[4], const float clip[4], uint32_t word) {
    const float w = clip[3];
    if (view[2] >= 0.0f || clip[2] > w || fabsf(clip[0]) > fmul(1.3f, w) || fabsf(clip[1]) > fmul(1.3f, w))
        return -1.0f;
    const float alpha = fdiv(float(word >> 24), 255.0f);   // unpack4x8unorm(..).a
    if (fmul(alpha, 255.0f) <= 1.0f) return -1.0f;
    return alpha;
}

// The footprint cull (render/splats.js:172-178 with footprint :102-124).
// Returns true when the splat is kept. s[6] is its covariance.
__device__ __forceinline__ bool footprint_keeps(const ViewConsts& c, const float view[4], const float s[6],
                                                float alpha) {
    float J00 = c.fx, J11 = c.fy, J02 = 0.0f, J12 = 0.0f;
    if (c.persp) {
        const float d = -view[2];
        const float x = fmul(fclamp(fdiv(view[0], d), c.xlo, c.xhi), d);
        const float y = fmul(fclamp(fdiv(view[1], d), c.ylo, c.yhi), d);
        const float dd = fmul(d, d);
        J00 = fdiv(c.fx, d);
        J11 = fdiv(c.fy, d);
        J02 = fdiv(fmul(c.fx, x), dd);
        J12 = fdiv(fmul(c.fy, y), dd);
    }
    // J = [[J00, 0, J02], [0, J11, J12], [0, 0, 0]];  W[r][col] = mv[col*4 + r].
    const float J[2][3] = {{J00, 0.0f, J02}, {0.0f, J11, J12}};
    const float S[3][3] = {{s[0], s[1], s[2]}, {s[1], s[3], s[4]}, {s[2], s[4], s[5]}};
    float T[2][3], U[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col)
            T[r][col] = fadd(fadd(fmul(J[r][0], c.mv[col * 4 + 0]), fmul(J[r][1], c.mv[col * 4 + 1])),
                             fmul(J[r][2], c.mv[col * 4 + 2]));
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col)
            U[r][col] = fadd(fadd(fmul(T[r][0], S[0][col]), fmul(T[r][1], S[1][col])), fmul(T[r][2], S[2][col]));
    const float fxx = fadd(fadd(fmul(U[0][0], T[0][0]), fmul(U[0][1], T[0][1])), fmul(U[0][2], T[0][2]));
    const float fxy = fadd(fadd(fmul(U[1][0], T[0][0]), fmul(U[1][1], T[0][1])), fmul(U[1][2], T[0][2]));
    const float fyy = fadd(fadd(fmul(U[1][0], T[1][0]), fmul(U[1][1], T[1][1])), fmul(U[1][2], T[1][2]));
    const float det = fsub(fmul(fadd(fxx, 0.3f), fadd(fyy, 0.3f)), fmul(fxy, fxy));
    const float area = fmul(6.2831853f, __fsqrt_rn(fmaxf(det, 0.0f)));
    return !(fmul(alpha, area) < c.cull);
}

// key = 65535 - bucket (render/splats.js:180-181).
__device__ __forceinline__ uint32_t depth_key(const ViewConsts& c, const float view[4]) {
    const float scaled = fmul(fsub(-view[2], c.depth_min), c.depth_scale);
    const uint32_t bucket = __float2uint_rz(fclamp(scaled, 0.0f, 65535.0f));
    return kBuckets - 1u - bucket;
}

// ---------------------------------------------------------------- memory ops
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace wsort
