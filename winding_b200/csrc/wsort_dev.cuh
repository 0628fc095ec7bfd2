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
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace wsort {

constexpr uint32_t kBuckets = 65536u;     // render/splats.js:64
constexpr uint32_t kCulled = 0xFFFFFFFFu;
constexpr uint32_t kPadSplats = 4096;     // resident clouds are padded to this multiple

// Error codes a kernel leaves in the context's error word.
constexpr uint32_t kErrWaitPhase = 1;     // a dependency (phase, look-back or copy) never completed
constexpr uint32_t kErrBounds = 3;        // a scatter position fell outside the output

// The sort of one job is three phases, each split into the same segments
// (contiguous splat ranges of the job, one work item each):
//   Keys   cull, 16-bit key, survivor bit; the segment's low-digit counts
//          (published for the look-back) and the job's totals of both digits
//   Low    after the job's keys: stable rank by the low key byte, scatter
//          (key, splat index) to the job's intermediate arrays
//   High   after the job's low pass: a proportional slice of the
//          intermediate arrays; its high-digit counts, a look-back over the
//          earlier slices, stable rank by the high byte, scatter the final
//          order and keys
constexpr uint32_t kPhaseKeys = 0, kPhaseLow = 1, kPhaseHigh = 2, kPhases = 3;
constexpr uint32_t kSegAlign = 256;       // segment boundaries are multiples of this (splats)
constexpr uint32_t kGroup = 16;           // segments per look-back group
constexpr int kKeysIPT = 4;               // splats per thread in one sub-tile of a keys item
constexpr int kDigitIPT = 8;              // elements per thread in one sub-tile of a digit pass
constexpr int kSubHist = 8;               // lane-interleaved sub-histograms for counting
// The sort's algorithms (ws_params.algorithm): the three phases over
// segments of every job (any size), or one CTA per job with the job in its
// shared memory (jobs of splats up to kOneMax), placed by two 8-bit passes
// or by one counting pass over all 65536 keys.
constexpr uint32_t kAlgoPhases = 0, kAlgoOneRadix = 1, kAlgoOneCount = 2;
constexpr uint32_t kOneMax = 16384;       // largest job the one-CTA sorts take
constexpr int kOneThreads = 1024;

// Per-view constants of one job, computed once (by the host for a sort, by
// make_consts for the draw). Each is the same IEEE operation on the same
// operands the per-splat WGSL evaluates, so hoisting them changes no bit.
struct ViewConsts {
    float mv[16];
    float proj[16];
    float keep_q;
    uint32_t keep_byte;
    int fast;
    float fx, fy;               // p[0][0] * viewport.x * 0.5, p[1][1] * viewport.y * 0.5
    float xlo, xhi, ylo, yhi;   // -1.3 / p[0][0], 1.3 / p[0][0], and for p[1][1]
    float cull;
    float depth_min, depth_scale;
    int persp;                  // p[3][3] == 0
    int visible;                // far > 0
    uint32_t faint_max;         // alpha bytes up to this are too faint: unpack(byte) * 255 <= 1
    // Upper bounds (rounded up) for the per-splat footprint bound of the keys
    // phase: |fx|, |fy|, the absolute row sums of the model-view's 3x3 (rows
    // 0, 1, 2), and |1.3 / p[0][0]|, |1.3 / p[1][1]|.
    float afx, afy, r0, r1, r2, xcap, ycap;
    uint32_t revz;              // fast, and P[8] = P[9] = P[10] = 0, P[11] = -1 (reverse-Z infinite)
    // The footprint cull as a threshold on det, per alpha byte b: makeKeys
    // keeps the splat exactly when det >= det_min[b] (the host's bisection
    // over f32 values of the monotone test !(alpha * (2 pi sqrt(max(det, 0)))
    // < cull), each operation rounded as the kernels round it; -inf: kept
    // whatever det).
    float det_min[256];
};

// One (cloud, view) to sort, as the kernel reads it.
struct alignas(16) JobDesc {
    // cloud (resident)
    const float4* centers;      // x, y, z, colour word bits; padded to kPadSplats
    const float2* cov;          // 6 f32 a splat as 3 float2; padded likewise
    const int8_t* sexp;         // per splat: max |covariance entry| <= 2^sexp; padded likewise
    double bmin[3], bmax[3];    // box around the centres
    uint32_t n;                 // elements
    uint32_t npad;              // n rounded up to kSegAlign: the range the segments cover
    // Per-view shortcuts the host proves exact (see keys_item):
    uint32_t fast_transform;    // affine model-view, reverse-Z perspective, no overflow possible
    uint32_t keep_byte;         // alpha bytes at or above this pass the footprint cull when ...
    float keep_q;               // ... keep_q 2^sexp <= 100 d^2 (+inf: never)
    uint32_t kind;              // kJobSplats, kJobParticles or kJobKeys
    uint32_t idx_base;          // added to every element index the order holds (a ring's first slot)
    // view: the values the reference writes into its Cloud uniform
    float mv[16];
    float proj[16];
    float viewport[2];
    float cull;
    ViewConsts vc;              // the view's constants, filled by the host
    // segments
    uint32_t seg0;              // the launch's index of the job's first segment
    uint32_t nseg;              // the job's segments
    uint32_t ngroups;           // look-back groups: ceil(nseg / kGroup)
    // outputs
    uint32_t* order;            // >= n
    uint32_t* keys;             // >= n, or null
    uint32_t* count;            // 1
    // scratch
    uint16_t* k16;              // per splat key (survivors)
    uint32_t* mask;             // survivor bits, one word per 32 splats
    uint16_t* key_b;            // low pass output: keys
    uint32_t* idx_b;            // low pass output: splat indices
    uint32_t* agg;              // 2 x nseg x 256: per segment, low-digit then high-digit counts
    uint32_t* ctl;              // JobCtl, then the look-back words (zeroed before a launch)
    // particles (kind == kJobParticles): one emitter's ring of the pool
    const float4* pool;         // the pool: two float4 a particle (position, age; velocity, lifetime)
    const float* thr;           // kParticleBuckets depth thresholds of the log-depth buckets
    float eye[4];               // particles: camera position (View.eye); splats: the eye in the
                                // cloud's space (Cloud.eye), for the harmonics
    float fwd[4];               // view direction (View.forward)
    // splats with harmonics: the shade pass, fused into the keys phase
    const uint32_t* sh;         // packed half-float coefficients, sh_words a splat; null: no shading
    uint32_t* shaded;           // per splat: its colour word as seen from the eye (survivors only)
    uint32_t sh_degree;         // 1, 2 or 3
    uint32_t sh_words;          // 32-bit words a splat: ceil(3 x coefficients / 2)
    // given keys (kind == kJobKeys): n 16-bit keys, every element a survivor
    const uint16_t* keys_in;
    uint32_t pad1[2];
};

constexpr uint32_t kJobSplats = 0, kJobParticles = 1, kJobKeys = 2;
// Depth buckets of an alpha emitter's sort (render/particles.js:44-48):
// 12 bits of log2 depth over [2^-10, 2^20].
constexpr uint32_t kParticleBuckets = 4096u;

// Per-job counters, zeroed before a launch. The look-back words follow:
// gsum[2][ngroups][256] (per group, the sum of its segments' counts: low,
// high), gdone[ngroups] (high-count items finished, per group) and
// flag[nseg] (a segment's high-digit counts are published).
struct JobCtl {
    uint32_t tot[2][256];       // survivors per digit value: low byte, high byte
    uint32_t keys_done;         // keys items finished
    uint32_t low_done;          // low items finished
    uint32_t high_done;         // high items finished (the job's outputs are final at nseg)
    uint32_t pad[13];
};
static_assert(sizeof(JobCtl) % 64 == 0, "JobCtl size");

// Bytes of a job's zeroed control region (JobCtl and its look-back words).
__host__ __device__ inline size_t job_ctl_bytes(uint32_t nseg) {
    const size_t ng = (nseg + kGroup - 1) / kGroup;
    const size_t b = sizeof(JobCtl) + (2 * ng * 256 + ng + nseg) * sizeof(uint32_t);
    return (b + 255) / 256 * 256;
}

// One job's share of a chunk of a batch: splats [a, b) of job `job`, its
// segment number `local` among the job's segments.
struct alignas(16) SegDesc {
    uint32_t job, a, b, local;
};

// Per-launch counters, zeroed before a launch.
struct LaunchCtl {
    uint32_t ticket[3];         // next work item of each phase's kernel
    uint32_t pad[13];
};

// What one launch sorts: three kernels (keys, low pass, high pass), each
// with one work item per segment, claimed in order. Segments come from
// `segs`, or, for a launch of one job (segs null), are the job's consecutive
// ranges of `chunk` splats.
struct LaunchDesc {
    const JobDesc* jobs;
    uint32_t njobs;
    const SegDesc* segs;
    uint32_t nseg;              // segments in the launch
    uint32_t chunk;             // one job: splats a segment covers
    uint32_t first_phase;       // phases before it are left out (the failure self-test)
    uint32_t spin_limit;        // polls a wait makes before it gives up
    struct LaunchCtl* lctl;
    uint32_t* err;              // code, work item
    struct TraceRec* trace;     // or null
};

// One work item's timeline, when tracing: globaltimer ns at the claim of its
// ticket, after its dependency wait, and at its end; and the SM it ran on.
struct TraceRec {
    uint64_t claim, start, end;
    uint32_t item, sm;
    uint64_t mark[3];           // phase-specific points inside the item (0: none)
};

// ---------------------------------------------------------------- f32 ops
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
// WGSL clamp(e, low, high) = min(max(e, low), high); fmaxf/fminf return the
// non-NaN operand.
__device__ __forceinline__ float fclamp(float e, float lo, float hi) { return fminf(fmaxf(e, lo), hi); }

// ------------------------------------------------------------- harmonics
//
// The shade pass (src/render/splats.js:315-382): a survivor's colour seen
// along d = normalize(centre - eye), the constant term (its colour bytes)
// plus the higher harmonics, clamped to [0, 1] and packed as four bytes. The
// pinned order: normalize is v / sqrt((x x + y y) + z z); every product and
// sum of harmonics() is separately rounded, left to right as written, each
// scalar factor chain (K x y, say) formed before it scales a coefficient;
// unpack4x8unorm is byte / 255 and pack4x8unorm floor(0.5 + 255 e), both
// correctly rounded f32; clamp returns the bound for NaN.

// Splat i's coefficient k as (r, g, b): three half floats from the two
// words they lie across (coefficient(), :338-344).
__device__ __forceinline__ float3 sh_coef(const uint32_t* sh, uint32_t words, uint32_t i, uint32_t k) {
    const size_t h = (size_t)i * words * 2 + k * 3;
    const uint32_t w0 = __ldg(&sh[h >> 1]), w1 = __ldg(&sh[(h >> 1) + 1]);
    const float a0 = __half2float(__ushort_as_half((unsigned short)(w0 & 0xFFFFu)));
    const float a1 = __half2float(__ushort_as_half((unsigned short)(w0 >> 16)));
    const float b0 = __half2float(__ushort_as_half((unsigned short)(w1 & 0xFFFFu)));
    const float b1 = __half2float(__ushort_as_half((unsigned short)(w1 >> 16)));
    return (h & 1) ? make_float3(a1, b0, b1) : make_float3(a0, a1, b0);
}

// s * v and the elementwise sum / difference, each separately rounded.
__device__ __forceinline__ float3 sv(float s, float3 v) { return make_float3(__fmul_rn(s, v.x), __fmul_rn(s, v.y), __fmul_rn(s, v.z)); }
__device__ __forceinline__ float3 vadd(float3 a, float3 b) { return make_float3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
__device__ __forceinline__ float3 vsub(float3 a, float3 b) { return make_float3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }

__device__ __forceinline__ uint32_t pack_unorm8(float e) {
    const float c = fminf(fmaxf(e, 0.0f), 1.0f);
    return (uint32_t)floorf(__fadd_rn(0.5f, __fmul_rn(255.0f, c)));
}

// The shaded colour word of splat i with centre (cx, cy, cz) and colour
// word `colour`, seen from `eye` (shade(), :371-381).
__device__ __forceinline__ uint32_t shade_splat(const uint32_t* sh, uint32_t words, uint32_t degree, uint32_t i,
                                                float cx, float cy, float cz, uint32_t colour, const float* eye) {
    const float vx = __fsub_rn(cx, eye[0]), vy = __fsub_rn(cy, eye[1]), vz = __fsub_rn(cz, eye[2]);
    const float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz)));
    const float x = __fdiv_rn(vx, len), y = __fdiv_rn(vy, len), z = __fdiv_rn(vz, len);
    // degree 1
    float3 c = sv(0.4886025119029199f, vsub(vadd(sv(-y, sh_coef(sh, words, i, 0)), sv(z, sh_coef(sh, words, i, 1))),
                                            sv(x, sh_coef(sh, words, i, 2))));
    if (degree >= 2) {
        const float xx = __fmul_rn(x, x), yy = __fmul_rn(y, y), zz = __fmul_rn(z, z);
        const float t1 = __fmul_rn(__fmul_rn(1.0925484305920792f, x), y);
        const float t2 = __fmul_rn(__fmul_rn(1.0925484305920792f, y), z);
        const float t3 = __fmul_rn(0.31539156525252005f, __fsub_rn(__fsub_rn(__fmul_rn(2.0f, zz), xx), yy));
        const float t4 = __fmul_rn(__fmul_rn(1.0925484305920792f, x), z);
        const float t5 = __fmul_rn(0.5462742152960396f, __fsub_rn(xx, yy));
        float3 e = vsub(sv(t1, sh_coef(sh, words, i, 3)), sv(t2, sh_coef(sh, words, i, 4)));
        e = vadd(e, sv(t3, sh_coef(sh, words, i, 5)));
        e = vsub(e, sv(t4, sh_coef(sh, words, i, 6)));
        e = vadd(e, sv(t5, sh_coef(sh, words, i, 7)));
        c = vadd(c, e);
        if (degree >= 3) {
            const float q = __fsub_rn(__fsub_rn(__fmul_rn(4.0f, zz), xx), yy);
            const float a = __fmul_rn(__fmul_rn(-0.5900435899266435f, y), __fsub_rn(__fmul_rn(3.0f, xx), yy));
            const float b = __fmul_rn(__fmul_rn(__fmul_rn(2.890611442640554f, x), y), z);
            const float cc = __fmul_rn(__fmul_rn(0.4570457994644658f, y), q);
            const float d = __fmul_rn(__fmul_rn(0.3731763325901154f, z),
                                      __fsub_rn(__fsub_rn(__fmul_rn(2.0f, zz), __fmul_rn(3.0f, xx)), __fmul_rn(3.0f, yy)));
            const float ee = __fmul_rn(__fmul_rn(0.4570457994644658f, x), q);
            const float f = __fmul_rn(__fmul_rn(1.445305721320277f, z), __fsub_rn(xx, yy));
            const float g = __fmul_rn(__fmul_rn(0.5900435899266435f, x), __fsub_rn(xx, __fmul_rn(3.0f, yy)));
            float3 h = vadd(sv(a, sh_coef(sh, words, i, 8)), sv(b, sh_coef(sh, words, i, 9)));
            h = vsub(h, sv(cc, sh_coef(sh, words, i, 10)));
            h = vadd(h, sv(d, sh_coef(sh, words, i, 11)));
            h = vsub(h, sv(ee, sh_coef(sh, words, i, 12)));
            h = vadd(h, sv(f, sh_coef(sh, words, i, 13)));
            h = vsub(h, sv(g, sh_coef(sh, words, i, 14)));
            c = vadd(c, h);
        }
    }
    const float r = __fdiv_rn((float)(colour & 255u), 255.0f);
    const float gr = __fdiv_rn((float)((colour >> 8) & 255u), 255.0f);
    const float bl = __fdiv_rn((float)((colour >> 16) & 255u), 255.0f);
    const float al = __fdiv_rn((float)(colour >> 24), 255.0f);
    return pack_unorm8(__fadd_rn(r, c.x)) | (pack_unorm8(__fadd_rn(gr, c.y)) << 8) |
           (pack_unorm8(__fadd_rn(bl, c.z)) << 16) | (pack_unorm8(al) << 24);
}

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
    c.keep_q = J.keep_q;
    c.keep_byte = J.keep_byte;
    c.fast = J.fast_transform != 0;
    depth_range(J, &c.depth_min, &c.depth_scale, &c.visible);
}

// view = modelView * (x, y, z, 1) (render/splats.js:160).
__device__ __forceinline__ void view_of(const ViewConsts& c, float x, float y, float z, float view[4]) {
    if (c.fast) {
        // modelView's last row is (0, 0, 0, 1): view.w is exactly 1, and
        // m[12 + j] * 1 is m[12 + j].
#pragma unroll
        for (int j = 0; j < 3; ++j)
            view[j] = fadd(fadd(fadd(fmul(c.mv[j], x), fmul(c.mv[4 + j], y)), fmul(c.mv[8 + j], z)), c.mv[12 + j]);
        view[3] = 1.0f;
        return;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
        view[j] = fadd(fadd(fadd(fmul(c.mv[j], x), fmul(c.mv[4 + j], y)), fmul(c.mv[8 + j], z)),
                       fmul(c.mv[12 + j], 1.0f));
}

// The frustum test (render/splats.js:161-167) on clip = projection * view.
// With the fast transform the projection's zero entries are left out: each
// dropped term is a zero times a finite number, which changes at most the
// sign of a zero, and the tests below compare, so they decide the same.
__device__ __forceinline__ bool in_frustum(const ViewConsts& c, const float view[4]) {
    const float* P = c.proj;
    float clip[4];
    if (c.fast) {
        clip[0] = fadd(fmul(P[0], view[0]), fmul(P[8], view[2]));
        clip[1] = fadd(fmul(P[5], view[1]), fmul(P[9], view[2]));
        clip[2] = fadd(fmul(P[10], view[2]), P[14]);
        clip[3] = fmul(P[11], view[2]);
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            clip[j] = fadd(fadd(fadd(fmul(P[j], view[0]), fmul(P[4 + j], view[1])), fmul(P[8 + j], view[2])),
                           fmul(P[12 + j], view[3]));
    }
    const float w = clip[3];
    return !(view[2] >= 0.0f || clip[2] > w || fabsf(clip[0]) > fmul(1.3f, w) || fabsf(clip[1]) > fmul(1.3f, w));
}

// footprint (render/splats.js:102-124): the 2D covariance (xx, xy, yy) in
// pixels, before the third of a pixel the draw adds. s[6] is the splat's
// covariance. J's entries J[0][1] and J[1][0] are zero in both of its forms,
// so their products with the (finite) model-view are zeros and are left out
// of T = J W.
__device__ __forceinline__ void footprint2d(const ViewConsts& c, const float view[4], const float s[6], float* pxx,
                                            float* pxy, float* pyy) {
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
    // W[r][col] = mv[col*4 + r].
    float T[2][3], U[2][3];
#pragma unroll
    for (int col = 0; col < 3; ++col) {
        T[0][col] = fadd(fmul(J00, c.mv[col * 4 + 0]), fmul(J02, c.mv[col * 4 + 2]));
        T[1][col] = fadd(fmul(J11, c.mv[col * 4 + 1]), fmul(J12, c.mv[col * 4 + 2]));
    }
    const float S[3][3] = {{s[0], s[1], s[2]}, {s[1], s[3], s[4]}, {s[2], s[4], s[5]}};
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col)
            U[r][col] = fadd(fadd(fmul(T[r][0], S[0][col]), fmul(T[r][1], S[1][col])), fmul(T[r][2], S[2][col]));
    const float fxx = fadd(fadd(fmul(U[0][0], T[0][0]), fmul(U[0][1], T[0][1])), fmul(U[0][2], T[0][2]));
    const float fxy = fadd(fadd(fmul(U[1][0], T[0][0]), fmul(U[1][1], T[0][1])), fmul(U[1][2], T[0][2]));
    const float fyy = fadd(fadd(fmul(U[1][0], T[1][0]), fmul(U[1][1], T[1][1])), fmul(U[1][2], T[1][2]));
    *pxx = fxx;
    *pxy = fxy;
    *pyy = fyy;
}

// The per-view constants the keys sweep needs on the fast transform, held in
// registers for a whole tile (the same values as ViewConsts; the functions
// below are view_of, in_frustum and depth_key's fast branches, op for op).
struct FastView {
    float m[12];                   // model-view entries 0-2, 4-6, 8-10, 12-14 (columns, rows 0-2)
    float p0, p5, p8, p9, p10, p11, p14;
    float depth_min, depth_scale;
};

__device__ __forceinline__ FastView fast_view_of(const ViewConsts& c) {
    FastView f;
#pragma unroll
    for (int col = 0; col < 4; ++col)
#pragma unroll
        for (int j = 0; j < 3; ++j) f.m[col * 3 + j] = c.mv[col * 4 + j];
    f.p0 = c.proj[0];
    f.p5 = c.proj[5];
    f.p8 = c.proj[8];
    f.p9 = c.proj[9];
    f.p10 = c.proj[10];
    f.p11 = c.proj[11];
    f.p14 = c.proj[14];
    f.depth_min = c.depth_min;
    f.depth_scale = c.depth_scale;
    return f;
}

__device__ __forceinline__ void fast_view(const FastView& f, float x, float y, float z, float view[4]) {
#pragma unroll
    for (int j = 0; j < 3; ++j)
        view[j] = fadd(fadd(fadd(fmul(f.m[j], x), fmul(f.m[3 + j], y)), fmul(f.m[6 + j], z)), f.m[9 + j]);
    view[3] = 1.0f;
}

__device__ __forceinline__ bool fast_in_frustum(const FastView& f, const float view[4]) {
    const float c0 = fadd(fmul(f.p0, view[0]), fmul(f.p8, view[2]));
    const float c1 = fadd(fmul(f.p5, view[1]), fmul(f.p9, view[2]));
    const float c2 = fadd(fmul(f.p10, view[2]), f.p14);
    const float w = fmul(f.p11, view[2]);
    return !(view[2] >= 0.0f || c2 > w || fabsf(c0) > fmul(1.3f, w) || fabsf(c1) > fmul(1.3f, w));
}

// fast_in_frustum for a projection with P[8] = P[9] = P[10] = 0 and P[11] = -1: the
// zero products add a signed zero, which changes no comparison (|c0|, |c1|;
// c2 is P[14] itself), and w = -1 view.z is -view.z exactly.
__device__ __forceinline__ bool fast_in_frustum_revz(const FastView& f, const float view[4]) {
    const float w = -view[2];
    const float c0 = fmul(f.p0, view[0]), c1 = fmul(f.p5, view[1]);
    return !(view[2] >= 0.0f || f.p14 > w || fabsf(c0) > fmul(1.3f, w) || fabsf(c1) > fmul(1.3f, w));
}

__device__ __forceinline__ uint32_t fast_depth_key(const FastView& f, const float view[4]) {
    const float scaled = fmul(fsub(-view[2], f.depth_min), f.depth_scale);
    const uint32_t bucket = __float2uint_rz(fclamp(scaled, 0.0f, 65535.0f));
    return kBuckets - 1u - bucket;
}

// The footprint cull's determinant (render/splats.js:172-178): the pinned 2D
// covariance's det = (xx + .3)(yy + .3) - xy^2; makeKeys keeps the splat when
// RN(alpha * 2 pi sqrt(max(det, 0))) >= cull, which the keys phase tests as
// det >= det_min[alpha byte].
__device__ __forceinline__ float footprint_det(const ViewConsts& c, const float view[4], const float s[6]) {
    float fxx, fxy, fyy;
    footprint2d(c, view, s, &fxx, &fxy, &fyy);
    return fsub(fmul(fadd(fxx, 0.3f), fadd(fyy, 0.3f)), fmul(fxy, fxy));
}

// key = 65535 - bucket (render/splats.js:180-181).
__device__ __forceinline__ uint32_t depth_key(const ViewConsts& c, const float view[4]) {
    const float scaled = fmul(fsub(-view[2], c.depth_min), c.depth_scale);
    const uint32_t bucket = __float2uint_rz(fclamp(scaled, 0.0f, 65535.0f));
    return kBuckets - 1u - bucket;
}

// ---------------------------------------------------------------- memory ops
// 16-byte asynchronous copies global -> shared (cp.async, cached in L2
// only), their commit, and the waits for a thread's committed groups.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most one of this thread's committed copy groups is pending.
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_none() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_release_add(uint32_t* p, uint32_t v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace wsort
