// Drawing sorted splats into a headless image: the reference's splat draw
// (vs / fs, src/render/splats.js:252-312) as CUDA, writing an RGBA f32
// buffer in device memory instead of a WebGPU colour target.
//
// What is drawn, pinned (the reference leaves rasterisation, varyings and
// transcendental precision to the GPU; this fixes one answer, and the CPU
// oracle computes the same one):
//   - per splat i = order[j], in order (far first): view and clip as the
//     keys phase computes them; the footprint (xx, xy, yy) + 0.3 on the
//     diagonal; the ellipse's axes from its eigen-decomposition as the vertex
//     shader writes it (mid, radius, major, minor; the axis normalised as
//     v / sqrt(x x + y y)); half-lengths min(sqrt(2 major), 1024) and
//     min(sqrt(2 minor), 1024); reach = log(255 a) from a table (the f32
//     nearest the real logarithm of each of the 256 possible 255 a); the
//     quad's extent sqrt(min(reach, 4)) in units of the axes. A splat with
//     minor <= 0 or reach <= 0 is not drawn, as the vertex shader leaves it
//     off screen.
//   - the quad covers the pixels whose centre (px + 0.5, py + 0.5) maps into
//     [-e, e]^2 under the quad's own inverse: offset = ((d . axis) (1 / la),
//     (d . perp) (1 / lc)), the reciprocals rounded once per splat, d the
//     centre's offset from the splat's centre in pixels (y up, as clip
//     space). That offset is the fragment's varying
//     (it varies linearly over the quad, as the reference interpolates it).
//     Pixels are only considered within the quad's bounding box widened by a
//     pixel, the same box on both sides. The library keeps, of that box, the
//     pixels whose centre lies within the quad's half-extents (hx, hy) of
//     its centre, plus a margin of 1/64 pixel and 2^-16 of the extent: a
//     covered pixel's offset has |ox|, |oy| <= qm, so its centre lies within
//     qm (la |ax| + lc |ay|) = hx across and hy down, and the margin is far
//     above the rounding of the coverage test (a few ulps of coordinates
//     below 4096). The cut leaves out no covered pixel (the oracle counts
//     them on the tests' clouds: none), so the image is the same, while the
//     tiles, pairs and fragments it saves are many (a small splat's box is
//     mostly its margins: at clusters-1M the cut keeps 26 % of the pixels).
//   - the fragment: alpha = min(0.99, exp(-dot(offset, offset)) a), dropped
//     below 1/255; colour = decodeSRGB(rgb bytes) from a table (the f32
//     nearest ((c + 0.055) / 1.055)^2.4 above 0.04045, c / 12.92 below, c
//     = byte / 255); blended premultiplied over what the image holds:
//     dst = src + dst (1 - alpha) for colour and alpha, as the reference's
//     blend state (one, one-minus-src-alpha). exp is the one in
//     fragment_alpha: Cody and Waite's reduction (ln 2 split as 355/512 -
//     2.12194440e-4, Software Manual for the Elementary Functions, 1980),
//     exp(r) by its Taylor polynomial to r^7 / 7! in Horner form, 2^k from
//     the exponent bits (in two steps below 2^-126).
//   - no fog and no depth test (a headless image has no opaque scene).
// Every f32 operation is separately rounded (-fmad=false).
//
// The B200 shape: a prepare kernel (one thread per drawn splat) writes each
// splat's quad and the 16 x 16-pixel tiles its box touches; an exclusive
// scan gives each splat its run of (tile, splat) pairs, emitted in splat
// order; the library's own stable sort orders the pairs by tile (a 16-bit
// key; same-tile pairs keep splat order); one CTA per tile then blends its
// splats in order, 256 pixels a CTA, splat records staged in shared memory,
// the tiles with the longest lists launched first; tiles with thousands of
// splats are blended first, by a kernel with four warps to a row pair.
#include "wsort.h"
#include "wsort_dev.cuh"
#include "wsort_host.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

namespace wsort {

int run_given_keys(ws_ctx* ctx, const uint16_t* keys, uint32_t n, uint32_t* order, uint32_t* sorted, uint32_t* count,
                   cudaStream_t stream);

namespace {

constexpr int kTilePx = 16;
constexpr uint32_t kMaxSide = 4096;   // tiles of one image fit the 16-bit sort key
constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;         // elements a scan thread covers
constexpr int kScanTile = kScanBlock * kScanItems;

// One drawn splat's quad, in pixels (x right, y down for the centre and the
// pixel box; the axes are in clip space's y-up pixel units).
struct alignas(16) Quad {
    float cx, cy;          // centre
    float ax, ay;          // unit major axis
    float ila, ilc;        // 1 / the half-lengths along the major and minor axes
    float qm;              // extent in units of the axes
    float a;               // alpha
    float r, g, b;         // decoded colour
    int x0, x1, y0, y1;    // candidate pixels (x0 > x1: nothing)
    float pad;
};

// The quad of instance j (order[j]), or an empty one. tables: srgb[256]
// then reach[256].
__global__ void __launch_bounds__(256) prepare_kernel(const JobDesc* __restrict__ jd, const uint32_t* __restrict__ order,
                                                      const uint32_t* __restrict__ count,
                                                      const uint32_t* __restrict__ shaded,
                                                      const float* __restrict__ tables, uint32_t n, uint32_t width,
                                                      uint32_t height, Quad* __restrict__ quads,
                                                      uint32_t* __restrict__ ntiles) {
    __shared__ ViewConsts c;
    if (threadIdx.x == 0) make_consts(*jd, c);
    __syncthreads();
    const JobDesc& J = *jd;
    const uint32_t drawn = min(*count, n);
    const float half_w = fmul(0.5f, (float)width), half_h = fmul(0.5f, (float)height);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        Quad q;
        q.x0 = 1;
        q.x1 = 0;
        q.y0 = 1;
        q.y1 = 0;
        uint32_t tiles = 0;
        if (j < drawn) {
            const uint32_t i = order[j];
            const float4 p = J.centers[i];
            float view[4];
            view_of(c, p.x, p.y, p.z, view);
            const float* P = c.proj;
            float clip[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                clip[k] = fadd(fadd(fadd(fmul(P[k], view[0]), fmul(P[4 + k], view[1])), fmul(P[8 + k], view[2])),
                               fmul(P[12 + k], view[3]));
            const float2 s0 = J.cov[3 * (size_t)i], s1 = J.cov[3 * (size_t)i + 1], s2 = J.cov[3 * (size_t)i + 2];
            const float s[6] = {s0.x, s0.y, s1.x, s1.y, s2.x, s2.y};
            float fxx, fxy, fyy;
            footprint2d(c, view, s, &fxx, &fxy, &fyy);
            const float a = fadd(fxx, 0.3f), b = fxy, cc = fadd(fyy, 0.3f);
            const float mid = fmul(0.5f, fadd(a, cc));
            const float hd = fmul(0.5f, fsub(a, cc));
            const float radius = __fsqrt_rn(fadd(fmul(hd, hd), fmul(b, b)));
            const float major = fadd(mid, radius), minor = fsub(mid, radius);
            const uint32_t word = shaded ? shaded[i] : __float_as_uint(p.w);
            const float reach = tables[256 + (word >> 24)];
            if (minor > 0.0f && reach > 0.0f) {
                float ax = 1.0f, ay = 0.0f;
                if (fabsf(b) > 1e-12f) {
                    const float ey = fsub(major, a);
                    const float len = __fsqrt_rn(fadd(fmul(b, b), fmul(ey, ey)));
                    ax = fdiv(b, len);
                    ay = fdiv(ey, len);
                } else if (cc > a) {
                    ax = 0.0f;
                    ay = 1.0f;
                }
                q.ax = ax;
                q.ay = ay;
                const float la = fminf(__fsqrt_rn(fmul(2.0f, major)), 1024.0f);
                const float lc = fminf(__fsqrt_rn(fmul(2.0f, minor)), 1024.0f);
                q.ila = fdiv(1.0f, la);
                q.ilc = fdiv(1.0f, lc);
                q.qm = __fsqrt_rn(fminf(reach, 4.0f));
                q.cx = fmul(fadd(fdiv(clip[0], clip[3]), 1.0f), half_w);
                q.cy = fmul(fsub(1.0f, fdiv(clip[1], clip[3])), half_h);
                const float hx = fmul(q.qm, fadd(fmul(la, fabsf(ax)), fmul(lc, fabsf(ay))));
                const float hy = fmul(q.qm, fadd(fmul(la, fabsf(ay)), fmul(lc, fabsf(ax))));
                q.a = fdiv((float)(word >> 24), 255.0f);
                q.r = tables[word & 255u];
                q.g = tables[(word >> 8) & 255u];
                q.b = tables[(word >> 16) & 255u];
                if (isfinite(q.cx) && isfinite(q.cy) && isfinite(hx) && isfinite(hy)) {
                    // The pinned box, cut to the pixels whose centre lies
                    // within (hx, hy) of the splat's centre plus a margin of
                    // 1/64 pixel and 2^-16 of the extent (see the head).
                    const float mx = fadd(fadd(hx, 0.015625f), fmul(hx, 1.0f / 65536.0f));
                    const float my = fadd(fadd(hy, 0.015625f), fmul(hy, 1.0f / 65536.0f));
                    const float fx0 = fmaxf(fmaxf(floorf(fsub(fsub(q.cx, hx), 1.5f)), 0.0f),
                                            ceilf(fsub(fsub(q.cx, mx), 0.5f)));
                    const float fx1 = fminf(fminf(ceilf(fadd(fadd(q.cx, hx), 0.5f)), (float)(width - 1)),
                                            floorf(fsub(fadd(q.cx, mx), 0.5f)));
                    const float fy0 = fmaxf(fmaxf(floorf(fsub(fsub(q.cy, hy), 1.5f)), 0.0f),
                                            ceilf(fsub(fsub(q.cy, my), 0.5f)));
                    const float fy1 = fminf(fminf(ceilf(fadd(fadd(q.cy, hy), 0.5f)), (float)(height - 1)),
                                            floorf(fsub(fadd(q.cy, my), 0.5f)));
                    if (fx0 <= fx1 && fy0 <= fy1) {
                        q.x0 = (int)fx0;
                        q.x1 = (int)fx1;
                        q.y0 = (int)fy0;
                        q.y1 = (int)fy1;
                        tiles = (uint32_t)((q.x1 / kTilePx - q.x0 / kTilePx + 1) * (q.y1 / kTilePx - q.y0 / kTilePx + 1));
                    }
                }
            }
        }
        quads[j] = q;
        ntiles[j] = tiles;
    }
}

// Exclusive scan of n words in three steps: per-4096 block scan with its
// block sum, a scan of the block sums (one CTA; also their 64-bit total),
// and the block offsets added.
__global__ void __launch_bounds__(kScanBlock) scan_blocks_kernel(const uint32_t* in, uint32_t* out, uint32_t n,
                                                                 uint32_t* sums) {
    __shared__ uint32_t warp_sums[kScanBlock / 32];
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems], local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0u;
        local += v[k];
    }
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t run = (warp ? warp_sums[warp - 1] : 0u) + x - local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = warp_sums[31];
}

__global__ void __launch_bounds__(kScanBlock) scan_sums_kernel(uint32_t* sums, uint32_t nb, unsigned long long* total) {
    __shared__ uint32_t warp_sums[kScanBlock / 32];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t c0 = 0; c0 < nb; c0 += kScanBlock) {
        const uint32_t k = c0 + threadIdx.x;
        const uint32_t v = k < nb ? sums[k] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = warp_sums[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= (uint32_t)o) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const unsigned long long before = carry;
        if (k < nb) sums[k] = (uint32_t)(before + (warp ? warp_sums[warp - 1] : 0u) + x - v);
        __syncthreads();
        if (threadIdx.x == 0) carry = before + warp_sums[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(256) add_offsets_kernel(uint32_t* out, uint32_t n, const uint32_t* sums) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        out[k] += sums[k / kScanTile];
}

// The (tile, splat) pairs of every drawn splat, in splat order.
__global__ void __launch_bounds__(256) emit_kernel(const Quad* __restrict__ quads, const uint32_t* __restrict__ ntiles,
                                                   const uint32_t* __restrict__ offsets, uint32_t n,
                                                   uint32_t tiles_x, uint16_t* __restrict__ keys,
                                                   uint32_t* __restrict__ owner) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        if (!ntiles[j]) continue;
        const Quad q = quads[j];
        uint32_t at = offsets[j];
        for (int ty = q.y0 / kTilePx; ty <= q.y1 / kTilePx; ++ty)
            for (int tx = q.x0 / kTilePx; tx <= q.x1 / kTilePx; ++tx) {
                keys[at] = (uint16_t)(ty * tiles_x + tx);
                owner[at] = j;
                ++at;
            }
    }
}

// Each tile's run [start, end) in the pairs sorted by tile.
__global__ void __launch_bounds__(256) ranges_kernel(const uint32_t* __restrict__ skeys, uint32_t npairs,
                                                     uint2* __restrict__ range) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < npairs; k += gridDim.x * blockDim.x) {
        const uint32_t t = skeys[k];
        if (k == 0 || skeys[k - 1] != t) range[t].x = k;
        if (k == npairs - 1 || skeys[k + 1] != t) range[t].y = k + 1;
    }
}

// The order the blend visits tiles in: longest splat lists first (by the
// list length's top two bits: lengths within a factor of 1.5 share a class,
// in no particular order), so that the crowded tiles start in the first
// wave, one to an SM, instead of wherever their index falls. One CTA; any
// order gives the same image, as each tile is blended on its own.
// It also counts the crowded tiles, those whose list holds crowd_min splats
// or more (a power of two, so that they are exactly the first classes; 0:
// none), which take the first places of the order.
constexpr int kOrderClasses = 66;   // 0: empty; then 2 classes an octave, longest last
__device__ __forceinline__ int length_class(uint32_t len) {
    if (len == 0) return 0;
    const int top = 31 - __clz(len);                                             // 0..31
    const int half = top > 0 ? (int)((len >> (top - 1)) & 1u) : 0;             // the bit below the top
    return 2 + 2 * top + half;
}

__global__ void __launch_bounds__(1024) order_tiles_kernel(const uint2* __restrict__ range, uint32_t tiles,
                                                           uint32_t crowd_min, uint32_t* __restrict__ tile_order,
                                                           uint32_t* __restrict__ n_crowded) {
    __shared__ uint32_t count[kOrderClasses], start[kOrderClasses];
    auto class_of = [](uint2 r) -> int { return length_class(r.y - r.x); };
    for (int c = threadIdx.x; c < kOrderClasses; c += blockDim.x) count[c] = 0;
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < tiles; t += blockDim.x) atomicAdd(&count[class_of(range[t])], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        const int crowd_class = crowd_min ? length_class(crowd_min) : kOrderClasses;
        uint32_t run = 0;
        for (int c = kOrderClasses - 1; c >= 0; --c) {
            start[c] = run;
            run += count[c];
            if (c == crowd_class) *n_crowded = run;
        }
        if (crowd_class >= kOrderClasses) *n_crowded = 0;
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < tiles; t += blockDim.x)
        tile_order[atomicAdd(&start[class_of(range[t])], 1u)] = t;
}

// The splat of each pair, in tile order: one indirection less for the blend.
__global__ void __launch_bounds__(256) gather_kernel(const uint32_t* __restrict__ owner,
                                                     const uint32_t* __restrict__ sorted, uint32_t npairs,
                                                     uint32_t* __restrict__ splat_of) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < npairs; k += gridDim.x * blockDim.x)
        splat_of[k] = owner[sorted[k]];
}

// The fragments of splats q[0..N), splat t at pixel (px[t], py[t]) whose
// centre is (fx[t], fy[t]): each one's alpha, or 0 when its quad does not cover the pixel or
// the fragment is dropped. Evaluated in lock-step, every stage for all N
// splats before the next, so the N independent chains overlap; without
// branches (every value computed, the answer selected). A covered fragment
// has |ox|, |oy| <= qm <= 2, so x = -d2 lies in [-8, 0] and k in [-12, 0]:
// exp is 2^k p(r) with 2^k a normal power of two, one multiply (the head's
// two-step scaling multiplies by 2^0 first there, which is exact, and its
// cases for x below -104 or NaN are never reached). An uncovered fragment's
// value is discarded, whatever these steps give for it.
template <int N, bool kInBox = false>   // kInBox: the caller knows every pixel lies in its splat's box
__device__ __forceinline__ void fragment_alphas_at(const Quad* const* q, const int* px, const int* py, const float* fx,
                                                   const float* fy, float* out) {
    float x[N], k[N], r[N], p[N];
    bool covered[N];
#pragma unroll
    for (int t = 0; t < N; ++t) {
        const bool in_box =
            kInBox || (px[t] >= q[t]->x0 && px[t] <= q[t]->x1 && py[t] >= q[t]->y0 && py[t] <= q[t]->y1);
        const float ex = fsub(fx[t], q[t]->cx), ey = fsub(q[t]->cy, fy[t]);
        const float ox = fmul(fadd(fmul(ex, q[t]->ax), fmul(ey, q[t]->ay)), q[t]->ila);
        const float oy = fmul(fsub(fmul(ex, q[t]->ay), fmul(ey, q[t]->ax)), q[t]->ilc);
        covered[t] = in_box && fabsf(ox) <= q[t]->qm && fabsf(oy) <= q[t]->qm;
        x[t] = -fadd(fmul(ox, ox), fmul(oy, oy));
    }
#pragma unroll
    for (int t = 0; t < N; ++t) {
        k[t] = rintf(fmul(x[t], 1.44269504f));
        r[t] = fsub(fsub(x[t], fmul(k[t], 0.693359375f)), fmul(k[t], -2.12194440e-4f));
        p[t] = 1.98412698e-4f;
    }
#pragma unroll
    for (int t = 0; t < N; ++t) p[t] = fadd(fmul(p[t], r[t]), 1.38888889e-3f);
#pragma unroll
    for (int t = 0; t < N; ++t) p[t] = fadd(fmul(p[t], r[t]), 8.33333333e-3f);
#pragma unroll
    for (int t = 0; t < N; ++t) p[t] = fadd(fmul(p[t], r[t]), 4.16666667e-2f);
#pragma unroll
    for (int t = 0; t < N; ++t) p[t] = fadd(fmul(p[t], r[t]), 1.66666667e-1f);
#pragma unroll
    for (int t = 0; t < N; ++t) p[t] = fadd(fmul(p[t], r[t]), 0.5f);
#pragma unroll
    for (int t = 0; t < N; ++t) p[t] = fadd(fmul(p[t], r[t]), 1.0f);
#pragma unroll
    for (int t = 0; t < N; ++t) p[t] = fadd(fmul(p[t], r[t]), 1.0f);
#pragma unroll
    for (int t = 0; t < N; ++t) {
        const uint32_t bits = ((uint32_t)__float2int_rn(k[t]) + 127u) << 23;
        const float e = fmul(p[t], __uint_as_float(bits));
        const float alpha = fminf(0.99f, fmul(e, q[t]->a));
        out[t] = (covered[t] && !(alpha < 1.0f / 255.0f)) ? alpha : 0.0f;
    }
}

// The same, every splat at the one pixel (px, py) whose centre is (fx, fy).
template <int N>
__device__ __forceinline__ void fragment_alphas(const Quad* const* q, int px, int py, float fx, float fy, float* out) {
    int pxs[N], pys[N];
    float fxs[N], fys[N];
#pragma unroll
    for (int t = 0; t < N; ++t) {
        pxs[t] = px;
        pys[t] = py;
        fxs[t] = fx;
        fys[t] = fy;
    }
    fragment_alphas_at<N>(q, pxs, pys, fxs, fys, out);
}

// One CTA a tile, one thread a pixel: the tile's splats in order, staged in
// shared memory 256 at a time (the next chunk copied with cp.async while
// this one is blended), blended over the image. Warp w holds the tile's
// pixel rows 2w and 2w + 1; for each chunk it marks (one ballot per 32
// splats) the splats whose pixel box reaches those rows and walks only the
// marked ones, four at a time: their fragments are evaluated independently,
// then blended in order. A pixel meets exactly the splats whose box holds
// it, in order, and a splat that leaves it untouched is skipped, as when
// every splat is tried one by one.
__global__ void __launch_bounds__(256) blend_kernel(const Quad* __restrict__ quads,
                                                    const uint32_t* __restrict__ splat_of,
                                                    const uint2* __restrict__ range,
                                                    const uint32_t* __restrict__ tile_order,
                                                    const uint32_t* __restrict__ n_crowded, uint32_t width,
                                                    uint32_t height, uint32_t tiles_x, float4* __restrict__ image) {
    __shared__ Quad staged[2][256];
    const uint32_t slot = *n_crowded + blockIdx.x;   // the grid is one CTA a tile; the crowded ones are done
    if (slot >= gridDim.x) return;
    const uint32_t tile = tile_order[slot];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int px = (int)((tile % tiles_x) * kTilePx + (threadIdx.x & 15));
    const int py = (int)((tile / tiles_x) * kTilePx + (threadIdx.x >> 4));
    const int row0 = (int)((tile / tiles_x) * kTilePx + 2 * warp), row1 = row0 + 1;
    const bool inside = px < (int)width && py < (int)height;
    float4 dst = inside ? image[(size_t)py * width + px] : make_float4(0, 0, 0, 0);
    const float fx = fadd((float)px, 0.5f), fy = fadd((float)py, 0.5f);
    const uint2 rg = range[tile];
    auto stage = [&](uint32_t c0, int b) {   // this thread's quad of the chunk at c0 into buffer b
        const uint32_t k = c0 + threadIdx.x;
        if (k < rg.y) {
            const Quad* src = &quads[splat_of[k]];
#pragma unroll
            for (int w = 0; w < 4; ++w) cp_async16(reinterpret_cast<float4*>(&staged[b][threadIdx.x]) + w,
                                                   reinterpret_cast<const float4*>(src) + w);
        }
        cp_async_commit();
    };
    if (rg.x < rg.y) stage(rg.x, 0);
    int b = 0;
    for (uint32_t c0 = rg.x; c0 < rg.y; c0 += 256, b ^= 1) {
        cp_async_wait_none();
        __syncthreads();   // chunk c0 is in staged[b]; staged[b ^ 1] is no longer read
        if (c0 + 256 < rg.y) stage(c0 + 256, b ^ 1);
        const uint32_t m = min(256u, rg.y - c0);
        uint32_t marks[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t e = j * 32 + lane;
            bool hit = false;
            if (e < m) {
                const Quad& q = staged[b][e];
                hit = q.y0 <= row1 && q.y1 >= row0;
            }
            marks[j] = __ballot_sync(0xffffffffu, hit);
        }
#pragma unroll 1
        for (int j = 0; j < 8; ++j) {
            uint32_t word = marks[j];
            while (word) {
                uint32_t e[4];
                int cnt = 0;
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    e[t] = 0;
                    if (word) {
                        e[t] = j * 32 + (__ffs(word) - 1);
                        word &= word - 1;
                        cnt = t + 1;
                    }
                }
                float al[4];
                const Quad* qs[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) qs[t] = &staged[b][e[t]];
                fragment_alphas<4>(qs, px, py, fx, fy, al);
#pragma unroll
                for (int t = 0; t < 4; ++t)
                    if (t >= cnt) al[t] = 0.0f;
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const float alpha = al[t];
                    if (alpha == 0.0f) continue;
                    const Quad& q = staged[b][e[t]];
                    const float om = fsub(1.0f, alpha);
                    dst.x = fadd(fmul(q.r, alpha), fmul(dst.x, om));
                    dst.y = fadd(fmul(q.g, alpha), fmul(dst.y, om));
                    dst.z = fadd(fmul(q.b, alpha), fmul(dst.z, om));
                    dst.w = fadd(alpha, fmul(dst.w, om));
                }
            }
        }
    }
    cp_async_wait_none();
    if (inside) image[(size_t)py * width + px] = dst;
}

// Crowded tiles are drawn in bands of kBandRows rows, each band by its own
// CTA (a tile's kBands bands on different SMs), from its own list: the
// splats of the tile's list whose box meets the band's rows, in list order.
// A pixel of the band gets the same splats, in the same order, as from the
// whole list (a splat whose box misses the band has no fragment in it).
constexpr int kBands = 4;
constexpr int kBandRows = kTilePx / kBands;

// One CTA of 1024 threads per crowded tile (persistent over them): the
// tile's kBands band lists, compacted in list order into band_list at
// kBands * range.x + b * length, their lengths into band_count[slot * kBands + b].
// Each chunk of 1024 list entries: every thread's band bits, a ballot per
// band, the warps' counts scanned by warp 0; the next chunk's entries and
// boxes are loaded while the current one is placed.
constexpr int kSplitThreads = 1024;
__global__ void __launch_bounds__(kSplitThreads) band_split_kernel(const Quad* __restrict__ quads,
                                                                   const uint32_t* __restrict__ splat_of,
                                                                   const uint2* __restrict__ range,
                                                                   const uint32_t* __restrict__ tile_order,
                                                                   const uint32_t* __restrict__ n_crowded,
                                                                   uint32_t tiles_x, uint32_t* __restrict__ band_list,
                                                                   uint32_t* __restrict__ band_count) {
    constexpr int W = kSplitThreads / 32;
    __shared__ uint32_t warp_n[kBands][W];     // a chunk's count per band and warp, then their exclusive scan
    __shared__ uint32_t run[kBands];           // placed so far, per band
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, lt = lanemask_lt();
    const uint32_t crowded = *n_crowded;
    for (uint32_t slot = blockIdx.x; slot < crowded; slot += gridDim.x) {
        const uint32_t tile = tile_order[slot];
        const int ty0 = (int)((tile / tiles_x) * kTilePx);
        const uint2 rg = range[tile];
        const uint32_t len = rg.y - rg.x;
        uint32_t* const out = band_list + (size_t)kBands * rg.x;
        if (threadIdx.x < kBands) run[threadIdx.x] = 0;
        auto fetch = [&](uint32_t c0, uint32_t& idx, int2& ys) {
            const uint32_t e = c0 + threadIdx.x;
            idx = 0;
            ys = make_int2(INT_MAX, INT_MIN);   // past the list: meets no band
            if (e < len) {
                idx = __ldg(&splat_of[rg.x + e]);
                ys = make_int2(__ldg(&quads[idx].y0), __ldg(&quads[idx].y1));   // 4-byte fields, 4-byte aligned
            }
        };
        uint32_t idx_n;
        int2 ys_n;
        fetch(0, idx_n, ys_n);
        for (uint32_t c0 = 0; c0 < len; c0 += kSplitThreads) {
            const uint32_t idx = idx_n;
            const int2 ys = ys_n;
            if (c0 + kSplitThreads < len) fetch(c0 + kSplitThreads, idx_n, ys_n);
            uint32_t bits = 0;
#pragma unroll
            for (int b = 0; b < kBands; ++b)
                if (ys.x <= ty0 + (b + 1) * kBandRows - 1 && ys.y >= ty0 + b * kBandRows) bits |= 1u << b;
            uint32_t ballots[kBands];
#pragma unroll
            for (int b = 0; b < kBands; ++b) {
                ballots[b] = __ballot_sync(0xffffffffu, (bits >> b) & 1u);
                if (lane == 0) warp_n[b][warp] = __popc(ballots[b]);
            }
            __syncthreads();
            if (warp == 0) {
#pragma unroll
                for (int b = 0; b < kBands; ++b) {
                    const uint32_t v = lane < (uint32_t)W ? warp_n[b][lane] : 0u;
                    uint32_t x = v;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                        if (lane >= (uint32_t)o) x += y;
                    }
                    if (lane < (uint32_t)W) warp_n[b][lane] = run[b] + x - v;
                    if (lane == 31) run[b] += x;   // W == 32: lane 31 holds the chunk's total
                }
            }
            __syncthreads();
#pragma unroll
            for (int b = 0; b < kBands; ++b)
                if ((bits >> b) & 1u) out[(size_t)b * len + warp_n[b][warp] + __popc(ballots[b] & lt)] = idx;
            __syncthreads();   // warp_n is rewritten by the next chunk
        }
        if (threadIdx.x < kBands) band_count[slot * kBands + threadIdx.x] = run[threadIdx.x];
        __syncthreads();
    }
}

// Crowded tiles: the same blend, band by band, with the fragments evaluated
// by 29 warps and blended by 2. A band's list goes by in chunks of 128
// splats, a stage each: one warp lists the boxes of chunk i + 1 (each
// splat's box within the band and where its pixels start in a flat list of
// items), the evaluating warps take chunk i's items, a lane an item, and
// write each nonzero alpha into a splat x pixel table in shared memory, and
// each of the band's 64 pixels walks its column of chunk i - 1's table in
// splat order, blends the nonzero entries and clears them, while chunks
// i + 2 and i + 3 are copied in. The values and the order of every
// operation on a pixel are blend_kernel's, so the image is the same to the
// bit. One CTA of 1024 threads an SM (its registers keep it alone there),
// claiming (tile, band) units, densest tiles first.
constexpr int kCrowdThreads = 1024;
constexpr uint32_t kCrowdChunk = 128;                    // splats a stage
constexpr uint32_t kBandPx = kTilePx * kBandRows;        // pixels of a band
constexpr uint32_t kCrowdBlenders = kBandPx;             // a thread a pixel of the band: warps 0..1
constexpr uint32_t kCrowdLister = kCrowdBlenders / 32;   // warp 2 lists the boxes
constexpr uint32_t kCrowdEvalWarps = kCrowdThreads / 32 - kCrowdLister - 1;   // warps 3..31
constexpr uint32_t kCrowdBatch = 2;                      // items a lane evaluates at once
constexpr uint32_t kCrowdRead = 8;                       // table entries a blending thread reads at once
struct CrowdSmem {
    Quad staged[5][kCrowdChunk];                         // chunk i in staged[i % 5]
    float alpha[2][kCrowdChunk][kBandPx];                // chunk i's alphas in alpha[i % 2]; 0 where none
    uint32_t start[2][kCrowdChunk + 1];                  // chunk i's items: splat e's start in start[i % 2][e]
    uint32_t box[2][kCrowdChunk];                        // and its box (crowd_box)
};

// A staged splat's box within its tile, packed for the item decode: first
// column and row relative to the tile (4 bits each), width - 1 (4 bits), and
// ceil(2^16 / width) (17 bits), with which (local * that) >> 16 is local /
// width exactly for every local < 256 (the error, below 256 / 2^16, never
// reaches the next multiple of 1 / width >= 1 / 16).
__device__ __forceinline__ uint32_t crowd_box(int bx, int by, int bw) {
    const uint32_t magic = (65536u + (uint32_t)bw - 1u) / (uint32_t)bw;
    return (uint32_t)bx | ((uint32_t)by << 4) | ((uint32_t)(bw - 1) << 8) | (magic << 12);
}

__global__ void __launch_bounds__(kCrowdThreads, 1) crowd_kernel(const Quad* __restrict__ quads,
                                                                 const uint32_t* __restrict__ band_list,
                                                                 const uint32_t* __restrict__ band_count,
                                                                 const uint2* __restrict__ range,
                                                                 const uint32_t* __restrict__ tile_order,
                                                                 const uint32_t* __restrict__ n_crowded,
                                                                 uint32_t* __restrict__ ticket,
                                                                 uint32_t width, uint32_t height, uint32_t tiles_x,
                                                                 float4* __restrict__ image) {
    extern __shared__ __align__(16) unsigned char crowd_raw[];
    __shared__ uint32_t next_unit;
    CrowdSmem& sm = *reinterpret_cast<CrowdSmem*>(crowd_raw);
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool blender = threadIdx.x < kCrowdBlenders, lister = warp == kCrowdLister;
    const uint32_t ew = warp - kCrowdLister - 1;         // evaluating warp index (others: unused)
    {
        float4* z = reinterpret_cast<float4*>(&sm.alpha[0][0][0]);
        for (uint32_t k = threadIdx.x; k < sizeof(sm.alpha) / 16; k += kCrowdThreads) z[k] = make_float4(0, 0, 0, 0);
    }
    const uint32_t units = *n_crowded * kBands;   // (crowded tile, band), densest tile's bands first
    // Units are claimed in order from one counter: a CTA that finishes a
    // short band takes the next unit, so the densest bands (claimed first)
    // bound the kernel, not a fixed share of units.
    for (;;) {
        __syncthreads();   // every thread has read next_unit
        if (threadIdx.x == 0) next_unit = atomicAdd(ticket, 1u);
        __syncthreads();
        const uint32_t unit = next_unit;
        if (unit >= units) break;
        const uint32_t tile = tile_order[unit / kBands], band = unit % kBands;
        const int tx0 = (int)((tile % tiles_x) * kTilePx), ty0 = (int)((tile / tiles_x) * kTilePx);
        const int by0 = ty0 + (int)band * kBandRows, by1 = by0 + kBandRows - 1;   // the band's rows
        // A blending thread's pixel: column t % 16, row t / 16 of the band.
        const int px = tx0 + (int)(threadIdx.x & 15), py = by0 + (int)((threadIdx.x >> 4) & 3);
        const bool inside = blender && px < (int)width && py < (int)height;
        float4 dst = make_float4(0, 0, 0, 0);
        if (inside) dst = image[(size_t)py * width + px];
        const uint2 rg = range[tile];
        const uint32_t* const list = band_list + (size_t)kBands * rg.x + (size_t)band * (rg.y - rg.x);
        const uint32_t count = band_count[unit];
        const uint32_t chunks = (count + kCrowdChunk - 1) / kCrowdChunk;
        auto chunk_len = [&](uint32_t c) { return min(kCrowdChunk, count - c * kCrowdChunk); };
        // Staging: threads 0..255 copy one 16-byte quarter of a quad each;
        // the splat index is read a chunk ahead, so its latency is hidden.
        auto index_of = [&](uint32_t c) -> uint32_t {
            const uint32_t k = c * kCrowdChunk + (threadIdx.x >> 2);
            return threadIdx.x < kCrowdChunk * 4 && c < chunks && k < count ? list[k] : 0xffffffffu;
        };
        auto stage = [&](uint32_t idx, uint32_t b) {
            if (idx != 0xffffffffu)
                cp_async16(reinterpret_cast<float4*>(&sm.staged[b][threadIdx.x >> 2]) + (threadIdx.x & 3),
                           reinterpret_cast<const float4*>(&quads[idx]) + (threadIdx.x & 3));
            cp_async_commit();
        };
        // The lister's part: chunk c's boxes within the band and their
        // items' starts (an inclusive scan of the box sizes; lane l holds
        // splats l, 32 + l, 64 + l and 96 + l).
        constexpr int kListed = (int)kCrowdChunk / 32;
        auto list_boxes = [&](uint32_t c) {
            const uint32_t m = chunk_len(c), b = c % 5;
            uint32_t* st = sm.start[c & 1];
            uint32_t* bt = sm.box[c & 1];
            uint32_t n[kListed];
#pragma unroll
            for (int j = 0; j < kListed; ++j) {
                const uint32_t e = j * 32 + lane;
                n[j] = 0;
                if (e < m) {
                    const Quad& q = sm.staged[b][e];
                    const int bx = max(q.x0, tx0), by = max(q.y0, by0);
                    const int bw = min(q.x1, tx0 + kTilePx - 1) - bx + 1, bh = min(q.y1, by1) - by + 1;
                    n[j] = (uint32_t)(bw * bh);
                    bt[e] = crowd_box(bx - tx0, by - by0, bw);
                }
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
                for (int j = 0; j < kListed; ++j) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, n[j], o);
                    if (lane >= (uint32_t)o) n[j] += y;
                }
            }
            uint32_t before = 0;
#pragma unroll
            for (int j = 0; j < kListed; ++j) {
                st[j * 32 + lane + 1] = n[j] + before;
                before += __shfl_sync(0xffffffffu, n[j], 31);
            }
            if (lane == 0) st[0] = 0;
        };
        __syncthreads();   // the previous tile's last reads of the tables are done
        // Every thread commits one copy group a stage (empty past the end),
        // so waiting until one group is pending leaves the latest chunk's
        // copy in flight: each chunk has two stages to arrive.
        stage(index_of(0), 0);
        stage(index_of(1), 1);
        stage(index_of(2), 2);
        uint32_t next = index_of(3);
        cp_async_wait_one();
        __syncthreads();   // chunks 0 and 1 are staged
        if (lister && chunks) list_boxes(0);
        for (uint32_t i = 0; i <= chunks; ++i) {
            cp_async_wait_one();
            __syncthreads();   // chunk i + 1 is staged and chunk i listed; chunk i - 2 is no longer read
            stage(next, (i + 3) % 5);
            next = index_of(i + 4);
            if (blender) {
                if (i == 0) continue;
                const uint32_t c = i - 1, b = c % 5, m = chunk_len(c);
                float* col = &sm.alpha[c & 1][0][threadIdx.x];
                // Entries past the chunk's end are 0 (never written), so
                // reading them in groups is harmless.
                for (uint32_t e0 = 0; e0 < m; e0 += kCrowdRead) {
                    float a[kCrowdRead];
#pragma unroll
                    for (uint32_t k = 0; k < kCrowdRead; ++k) a[k] = col[(e0 + k) * kBandPx];
#pragma unroll
                    for (uint32_t k = 0; k < kCrowdRead; ++k) {
                        const float alpha = a[k];
                        if (alpha == 0.0f) continue;
                        col[(e0 + k) * kBandPx] = 0.0f;
                        const Quad& q = sm.staged[b][e0 + k];
                        const float om = fsub(1.0f, alpha);
                        dst.x = fadd(fmul(q.r, alpha), fmul(dst.x, om));
                        dst.y = fadd(fmul(q.g, alpha), fmul(dst.y, om));
                        dst.z = fadd(fmul(q.b, alpha), fmul(dst.z, om));
                        dst.w = fadd(alpha, fmul(dst.w, om));
                    }
                }
            } else if (lister) {
                if (i + 1 < chunks) list_boxes(i + 1);
            } else if (i < chunks) {
                const uint32_t b = i % 5;
                const uint32_t* st = sm.start[i & 1];
                const uint32_t* bt = sm.box[i & 1];
                const uint32_t total = st[kCrowdChunk];
                float* table = &sm.alpha[i & 1][0][0];
                for (uint32_t g0 = ew * 32 + lane; g0 < total; g0 += kCrowdEvalWarps * 32 * kCrowdBatch) {
                    const Quad* qs[kCrowdBatch];
                    int ipx[kCrowdBatch], ipy[kCrowdBatch];
                    float ifx[kCrowdBatch], ify[kCrowdBatch];
                    uint32_t cell[kCrowdBatch];
                    bool live[kCrowdBatch];
#pragma unroll
                    for (int t = 0; t < (int)kCrowdBatch; ++t) {
                        const uint32_t g = g0 + t * kCrowdEvalWarps * 32;
                        live[t] = g < total;
                        const uint32_t gg = live[t] ? g : g0;
                        uint32_t e = 0;   // the splat of item gg: the last start <= gg (a splat with items)
#pragma unroll
                        for (uint32_t step = kCrowdChunk / 2; step; step >>= 1)
                            e += st[e + step] <= gg ? step : 0u;
                        const uint32_t bx = bt[e], local = gg - st[e];
                        const uint32_t w = ((bx >> 8) & 15u) + 1u;
                        const uint32_t dy = (local * (bx >> 12)) >> 16;
                        const uint32_t cx = (bx & 15u) + local - dy * w, cy = ((bx >> 4) & 15u) + dy;
                        ipx[t] = tx0 + (int)cx;
                        ipy[t] = by0 + (int)cy;
                        ifx[t] = fadd((float)ipx[t], 0.5f);
                        ify[t] = fadd((float)ipy[t], 0.5f);
                        qs[t] = &sm.staged[b][e];
                        cell[t] = e * kBandPx + cy * kTilePx + cx;
                    }
                    float al[kCrowdBatch];
                    fragment_alphas_at<kCrowdBatch, true>(qs, ipx, ipy, ifx, ify, al);
#pragma unroll
                    for (int t = 0; t < (int)kCrowdBatch; ++t)
                        if (live[t] && al[t] != 0.0f) table[cell[t]] = al[t];
                }
            }
        }
        if (inside) image[(size_t)py * width + px] = dst;
    }
}

// decodeSRGB of byte / 255 and log(255 byte / 255), as f32 (see the head).
const std::vector<float>& draw_tables() {
    static std::vector<float> t;
    static std::once_flag once;
    std::call_once(once, [] {
        t.assign(512, 0.0f);
        for (int b = 0; b < 256; ++b) {
            const float c = (float)b / 255.0f;
            if (c <= 0.04045f) {
                t[b] = c / 12.92f;
            } else {
                const float base = (c + 0.055f) / 1.055f;
                t[b] = (float)std::pow((double)base, 2.4);
            }
            const float x = 255.0f * c;
            t[256 + b] = (float)std::log((double)x);
        }
    });
    return t;
}

}  // namespace
}  // namespace wsort

using namespace wsort;

extern "C" int ws_draw_tables(float* srgb, float* reach) {
    if (!srgb || !reach) return WS_ERR_ARG;
    const std::vector<float>& t = draw_tables();
    std::memcpy(srgb, t.data(), 256 * sizeof(float));
    std::memcpy(reach, t.data() + 256, 256 * sizeof(float));
    return WS_OK;
}

extern "C" int ws_set_draw_crowded(ws_ctx* ctx, uint32_t min_splats) {
    if (!ctx) return WS_ERR_ARG;
    if (min_splats & (min_splats - 1))
        return set_error(ctx, WS_ERR_ARG, "ws_set_draw_crowded: %u is not a power of two (or 0)", min_splats);
    ctx->draw_crowd_min = min_splats;
    return WS_OK;
}

extern "C" int ws_draw(ws_ctx* ctx, const ws_cloud* cloud, const ws_view* view, const uint32_t* order,
                       const uint32_t* count, const uint32_t* shaded, float* image, uint32_t width, uint32_t height,
                       void* stream_p) {
    NvtxRange nvtx("ws_draw");
    if (!ctx) return WS_ERR_ARG;
    if (!cloud || cloud->magic != kCloudMagic) return set_error(ctx, WS_ERR_ARG, "ws_draw: not a cloud");
    if (!cloud->alive) return set_error(ctx, WS_ERR_UNLOADED, "addSplats: these splats were unloaded; remove the node first");
    if (!view || !order || !count || !image) return set_error(ctx, WS_ERR_ARG, "ws_draw: null argument");
    if (width == 0 || height == 0 || width > kMaxSide || height > kMaxSide)
        return set_error(ctx, WS_ERR_ARG, "ws_draw: an image of %u x %u; 1 to %u pixels a side", width, height, kMaxSide);
    if (view->viewport[0] != (float)width || view->viewport[1] != (float)height)
        return set_error(ctx, WS_ERR_ARG, "ws_draw: the view's viewport is %g x %g, the image %u x %u",
                         (double)view->viewport[0], (double)view->viewport[1], width, height);
    if (reinterpret_cast<uintptr_t>(image) % 16)
        return set_error(ctx, WS_ERR_ARG, "ws_draw: the image is not 16-byte aligned");
    cudaSetDevice(ctx->device);
    cudaStream_t stream = stream_p ? static_cast<cudaStream_t>(stream_p) : ctx->stream;
    const uint32_t n = cloud->n;
    const uint32_t tiles_x = (width + kTilePx - 1) / kTilePx, tiles_y = (height + kTilePx - 1) / kTilePx;
    const uint32_t tiles = tiles_x * tiles_y;
    const uint32_t nb = (n + kScanTile - 1) / kScanTile;
    cudaError_t e;
    // Scratch: the job table, tables, quads, per-splat tile counts and offsets,
    // block sums, 64-bit total, tile ranges, the blend's tile order, the
    // number of crowded tiles.
    auto up = [](size_t v) { return (v + 255) / 256 * 256; };
    const size_t o_job = 0, o_tab = up(sizeof(JobDesc)), o_quad = o_tab + up(512 * 4);
    const size_t o_cnt = o_quad + up((size_t)n * sizeof(Quad)), o_off = o_cnt + up((size_t)n * 4);
    const size_t o_sums = o_off + up((size_t)n * 4), o_tot = o_sums + up((size_t)nb * 4 + 4);
    const size_t o_rng = o_tot + 256, o_tord = o_rng + up((size_t)tiles * 8), o_ncr = o_tord + up((size_t)tiles * 4);
    const size_t fixed = o_ncr + 256;
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_error(ctx, e, "ws_draw");
    if ((e = ctx->draw_d.ensure(fixed)) != cudaSuccess) return cuda_error(ctx, e, "ws_draw scratch");
    char* base = static_cast<char*>(ctx->draw_d.p);
    JobDesc jd;
    std::memset(&jd, 0, sizeof(jd));
    jd.centers = cloud->centers;
    jd.cov = cloud->cov;
    for (int k = 0; k < 3; ++k) {
        jd.bmin[k] = cloud->bmin[k];
        jd.bmax[k] = cloud->bmax[k];
    }
    jd.n = n;
    std::memcpy(jd.mv, view->model_view, sizeof(jd.mv));
    std::memcpy(jd.proj, view->projection, sizeof(jd.proj));
    jd.viewport[0] = view->viewport[0];
    jd.viewport[1] = view->viewport[1];
    jd.cull = view->cull;
    const std::vector<float>& tab = draw_tables();
    if ((e = cudaMemcpyAsync(base + o_job, &jd, sizeof(jd), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(base + o_tab, tab.data(), 512 * 4, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(base + o_rng, 0, (size_t)tiles * 8, stream)) != cudaSuccess)
        return cuda_error(ctx, e, "ws_draw");
    Quad* quads = reinterpret_cast<Quad*>(base + o_quad);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(base + o_cnt);
    uint32_t* off = reinterpret_cast<uint32_t*>(base + o_off);
    uint32_t* sums = reinterpret_cast<uint32_t*>(base + o_sums);
    unsigned long long* total = reinterpret_cast<unsigned long long*>(base + o_tot);
    uint2* range = reinterpret_cast<uint2*>(base + o_rng);
    uint32_t* tile_order = reinterpret_cast<uint32_t*>(base + o_tord);
    uint32_t* n_crowded = reinterpret_cast<uint32_t*>(base + o_ncr);
    const uint32_t g = std::max(1u, std::min((n + 255) / 256, (uint32_t)ctx->sms * 8));
    prepare_kernel<<<g, 256, 0, stream>>>(reinterpret_cast<const JobDesc*>(base + o_job), order, count, shaded,
                                          reinterpret_cast<const float*>(base + o_tab), n, width, height, quads, cnt);
    scan_blocks_kernel<<<std::max(nb, 1u), kScanBlock, 0, stream>>>(cnt, off, n, sums);
    scan_sums_kernel<<<1, kScanBlock, 0, stream>>>(sums, std::max(nb, 1u), total);
    add_offsets_kernel<<<g, 256, 0, stream>>>(off, n, sums);
    unsigned long long pairs64 = 0;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(&pairs64, total, 8, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess)
        return cuda_error(ctx, e, "ws_draw");
    if (pairs64 == 0) return WS_OK;
    if (pairs64 > WS_MAX_SPLATS)
        return set_error(ctx, WS_ERR_CAPACITY, "ws_draw: %llu (tile, splat) pairs, more than %u", pairs64,
                         WS_MAX_SPLATS);
    const uint32_t pairs = (uint32_t)pairs64;
    // The pair arrays, in a buffer of their own (growing it keeps the first):
    // keys, owners, sorted order, sorted keys, splats in tile order, count.
    const size_t o_keys = 0, o_own = o_keys + up((size_t)pairs * 2), o_sorted = o_own + up((size_t)pairs * 4);
    const size_t o_skeys = o_sorted + up((size_t)pairs * 4), o_spl = o_skeys + up((size_t)pairs * 4);
    const size_t o_pc = o_spl + up((size_t)pairs * 4);
    // and the crowded tiles' band lists (room for every pair in every band)
    // and band lengths
    const size_t o_band = o_pc + 256, o_bcnt = o_band + up((size_t)pairs * 4 * kBands);
    const size_t pairs_bytes = ctx->draw_crowd_min ? o_bcnt + up((size_t)tiles * 4 * kBands) : o_pc + 256;
    if ((e = ctx->pairs_d.ensure(pairs_bytes)) != cudaSuccess) return cuda_error(ctx, e, "ws_draw scratch");
    char* pb = static_cast<char*>(ctx->pairs_d.p);
    uint16_t* keys = reinterpret_cast<uint16_t*>(pb + o_keys);
    uint32_t* owner = reinterpret_cast<uint32_t*>(pb + o_own);
    uint32_t* sorted = reinterpret_cast<uint32_t*>(pb + o_sorted);
    uint32_t* skeys = reinterpret_cast<uint32_t*>(pb + o_skeys);
    uint32_t* pcount = reinterpret_cast<uint32_t*>(pb + o_pc);
    uint32_t* splat_of = reinterpret_cast<uint32_t*>(pb + o_spl);
    emit_kernel<<<g, 256, 0, stream>>>(quads, cnt, off, n, tiles_x, keys, owner);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(ctx, e, "ws_draw");
    int rc = run_given_keys(ctx, keys, pairs, sorted, skeys, pcount, stream);
    if (rc) return rc;
    const uint32_t gp = std::max(1u, std::min((pairs + 255) / 256, (uint32_t)ctx->sms * 8));
    ranges_kernel<<<gp, 256, 0, stream>>>(skeys, pairs, range);
    gather_kernel<<<gp, 256, 0, stream>>>(owner, sorted, pairs, splat_of);
    order_tiles_kernel<<<1, 1024, 0, stream>>>(range, tiles, ctx->draw_crowd_min, tile_order, n_crowded);
    if (ctx->draw_crowd_min) {
        if ((e = cudaFuncSetAttribute(crowd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sizeof(CrowdSmem))) != cudaSuccess)
            return cuda_error(ctx, e, "ws_draw");
        uint32_t* band_list = reinterpret_cast<uint32_t*>(pb + o_band);
        uint32_t* band_count = reinterpret_cast<uint32_t*>(pb + o_bcnt);
        uint32_t* ticket = n_crowded + 1;   // the crowded kernel's unit counter (its 256-byte slot)
        if ((e = cudaMemsetAsync(ticket, 0, sizeof(uint32_t), stream)) != cudaSuccess) return cuda_error(ctx, e, "ws_draw");
        band_split_kernel<<<std::min(tiles, (uint32_t)ctx->sms * 2), kSplitThreads, 0, stream>>>(
            quads, splat_of, range, tile_order, n_crowded, tiles_x, band_list, band_count);
        crowd_kernel<<<std::min(tiles * kBands, (uint32_t)ctx->sms), kCrowdThreads, sizeof(CrowdSmem), stream>>>(
            quads, band_list, band_count, range, tile_order, n_crowded, ticket, width, height, tiles_x,
            reinterpret_cast<float4*>(image));
    }
    blend_kernel<<<tiles, 256, 0, stream>>>(quads, splat_of, range, tile_order, n_crowded, width, height, tiles_x,
                                            reinterpret_cast<float4*>(image));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(ctx, e, "ws_draw");
    return WS_OK;
}
