// The sort: every (cloud, view) job's keys, survivor compaction and stable
// two-digit radix sort, for any number of jobs, in one launch of three
// persistent kernels (keys, low digit, high digit), chained by programmatic
// dependent launch; and the one-CTA sorts for small jobs.
//
// Reference (src/render/splats.js): makeKeys :155-186 appends survivors
// through a global atomic and counts them into 65536 buckets; scanCounts
// :188-212 scans the buckets; place :214-219 scatters through per-bucket
// atomics. Here the same keys feed a deterministic, stable LSD radix sort of
// the 16-bit key in two 8-bit digits, which gives the order the reference's
// stable CPU sort gives (src/render/drawlist.js:186-229): survivors by
// (key, splat index).
//
// Work. A launch's jobs are laid end to end and cut into segments of about
// equal size (a job's share of one chunk: one work item per phase). A job is
// three phases over its segments: Keys (cull, key, survivor bit, the
// segment's low-digit counts and the job's totals of both digits), Low
// (stable rank by the low byte and scatter, once the job's keys are done)
// and High (a proportional slice of the low pass's output: its high-digit
// counts, then stable rank by the high byte and scatter). A work item walks
// its segment in sub-tiles, in order, carrying each digit's running offset
// from one sub-tile to the next, so the only cross-item sum is over the
// segments before it. That sum is a two-level decoupled look-back: every
// segment publishes its 256 counts, and every group of kGroup segments their
// sum (red.add) with a completion count; a segment adds the group sums of
// the groups before its own and the counts of its own group's earlier
// segments, waiting (bounded) only for those. The digit starts come from the
// totals the keys phase counted.
//
// Items are claimed in ticket order, one ticket counter per phase: every
// segment's keys, then every low pass, then every high pass, each phase a
// persistent kernel. Each kernel lets the next one launch as soon as all its
// CTAs run (griddepcontrol.launch_dependents at their start); the next
// kernel's CTAs take SMs as this one's leave, and none waits for a whole
// grid: an item waits only for its own job's previous phase (a completion
// count) and for its own phase's earlier segments (which publish their
// counts before they wait). All of those have smaller tickets, claimed by
// CTAs that are running (a kernel launches only once every CTA of the one
// before it runs), so the queue always drains, whatever else shares the
// GPU; and a batch's later jobs can be in their keys while its earlier jobs
// are in their digit passes. Every wait is bounded: after spin_limit polls
// the kernel records an error and every CTA drains the remaining items
// without work.
//
// Ranking: a warp ranks 32 elements a round, in element order. Lanes with
// the same digit find each other by an atomicOr of their lane bit into the
// warp's word for that digit in shared memory (measured on B200 at 540-800
// Gelem/s for the whole GPU, against 300 for eight ballots and 150-830 for
// __match_any_sync, which depends on the number of distinct digits); the
// highest lane of each group clears the word and advances the warp's 16-bit
// count of the digit.
//
// Keys staging: a keys item copies each sub-tile's centres (and covariance
// exponents) into shared memory with one bulk copy (cp.async.bulk, completed
// on an mbarrier), the next sub-tile's copy in flight while the current one
// is swept.
#include "wsort_dev.cuh"

namespace wsort {

// Shared memory of a keys CTA (NT threads).
template <int NT>
struct KeysSmem {
    static constexpr int TK = NT * kKeysIPT;     // splats of a keys sub-tile
    alignas(8) uint64_t bar[2];                  // the staging buffers' mbarriers
    ViewConsts vc;
    uint32_t next;                               // the ticket this CTA works on next
    uint32_t drain;
    uint32_t abort;
    uint32_t pending;                            // staging buffers with a copy in flight (bits)
    uint32_t qn;
    uint64_t mark[3];                            // tracing: timestamps inside an item
    uint32_t hist[kSubHist][512];                // low digit at [s][..256), high at [s][256..)
    uint32_t queue[2 * TK];                      // splats whose footprint must be evaluated
    alignas(128) float4 centers[2][TK];
    int8_t sexp[2][TK];
};

// The keys CTA's shared memory fits the 227 KB a block may opt into.
static_assert(sizeof(KeysSmem<768>) <= 232448, "keys shared memory");

// Shared memory of a digit-pass CTA (NT threads).
template <int NT>
struct DigitSmem {
    static constexpr int W = NT / 32;
    static constexpr int TD = NT * kDigitIPT;    // elements of a sub-tile
    uint32_t next;
    uint32_t drain;
    uint32_t abort;
    uint32_t total;                              // survivors of the item's job
    uint32_t tile_total;                         // elements of the current sub-tile
    uint32_t scan[W];
    uint64_t mark[3];
    uint32_t dstart[256];                        // start of each digit in the pass's output
    uint32_t gbase[256];                         // dstart plus the segments before this one
    uint32_t run[256];                           // placed by the item's earlier sub-tiles
    uint32_t gofs[256];                          // gbase + run - sub-tile start, per digit
    uint32_t lstart[256];                        // sub-tile start of each digit
    uint32_t part[NT / 256][256];                // partial sums of the look-back
    uint32_t wmask[W][256];                      // per warp and digit: lanes of the round
    uint16_t wcnt[W][256];                       // per warp and digit: count, then the warp's start
    uint16_t skey[TD];                           // the sub-tile staged in output order
    uint32_t sidx[TD];
    uint32_t hist[kSubHist][256];                // high pass: the segment's counts
};

// The index of digit d's counter in sub-histogram s: rotated by 4 s, so that
// lanes of different sub-histograms with the same digit meet different banks.
__device__ __forceinline__ uint32_t sub_slot(uint32_t s, uint32_t d) { return (d + 4u * s) & 255u; }

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t sm_id() {
    uint32_t s;
    asm("mov.u32 %0, %%smid;" : "=r"(s));
    return s;
}

__device__ __forceinline__ void raise_error(uint32_t* err, uint32_t code, uint32_t item) {
    if (atomicCAS(err, 0u, code) == 0u) err[1] = item;
}

__device__ __forceinline__ void red_add(uint32_t* p, uint32_t v) {
    asm volatile("red.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ------------------------------------------------------------- mbarrier / bulk copy
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// One bulk copy of `bytes` (a multiple of 16, both ends 16-byte aligned) from
// this GPU's global memory into this CTA's shared memory, completed on bar.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
// Orders this thread's earlier shared-memory accesses (and those it has
// synchronised with) before later bulk-copy writes.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Per-thread state of the keys staging that lives across items: the next
// buffer and each buffer's mbarrier parity.
struct KeysStage {
    uint32_t buf;
    uint32_t parity;   // bit b: the parity of buffer b's next completion
};

// Waits (bounded) for buffer b's copy. Every thread calls it and flips its
// own copy of the parity bit. False if the wait gave up.
template <int NT>
__device__ __forceinline__ bool stage_wait(KeysSmem<NT>& sm, KeysStage& ks, uint32_t b, const LaunchDesc& L,
                                           uint32_t item) {
    const uint32_t par = (ks.parity >> b) & 1u;
    uint32_t spins = 0;
    bool ok = true;
    while (!mbar_try_wait(&sm.bar[b], par)) {
        if (++spins > L.spin_limit) {
            raise_error(L.err, kErrWaitPhase, item);
            ok = false;
            break;
        }
    }
    ks.parity ^= 1u << b;
    return ok;
}

// Waits (thread 0, bounded) until *p >= need. Returns false, uniformly
// across the CTA, if the wait gave up (or another CTA raised an error).
template <class SM>
__device__ bool wait_count(const uint32_t* p, uint32_t need, SM& sm, const LaunchDesc& L, uint32_t item) {
    if (threadIdx.x == 0) {
        uint32_t spins = 0;
        sm.abort = 0;
        while (ld_acquire(p) < need) {
            if (++spins > L.spin_limit || *(volatile uint32_t*)L.err) {
                raise_error(L.err, kErrWaitPhase, item);
                sm.abort = 1;
                break;
            }
            __nanosleep(32);
        }
    }
    __syncthreads();
    return sm.abort == 0;
}

// The start of each digit in a pass's output: an exclusive scan of the job's
// 256 digit totals into sm.dstart, their sum into sm.total.
template <int NT>
__device__ void digit_starts(const uint32_t* tot, DigitSmem<NT>& sm) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t v = 0, x = 0;
    if (tid < 256) {
        v = __ldcg(&tot[tid]);
        x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) sm.scan[warp] = x;
    }
    __syncthreads();
    if (tid < 256) {
        uint32_t off = 0;
#pragma unroll
        for (uint32_t w = 0; w < 8; ++w) off += w < warp ? sm.scan[w] : 0u;
        sm.dstart[tid] = off + x - v;
    }
    if (tid == 0) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) t += sm.scan[w];
        sm.total = t;
    }
    __syncthreads();
}

// gbase[d] = dstart[d] + the counts of digit d in the job's segments before
// segment `ls` of group g: the group sums of groups 0 .. g-1 and the counts
// of segments g kGroup .. ls-1 (all published before this is called).
template <int NT>
__device__ void segment_prefix(const uint32_t* gsum, const uint32_t* agg, uint32_t g, uint32_t ls,
                               DigitSmem<NT>& sm) {
    constexpr uint32_t P = NT / 256;
    const uint32_t d = threadIdx.x & 255u, p = threadIdx.x >> 8;
    const uint32_t g0 = g * kGroup;
    const uint32_t terms = g + (ls - g0);
    uint32_t s = 0;
#pragma unroll 4
    for (uint32_t t = p; t < terms; t += P) {
        const uint32_t* row = t < g ? gsum + (size_t)t * 256 : agg + (size_t)(g0 + t - g) * 256;
        s += __ldcg(row + d);
    }
    sm.part[p][d] = s;
    __syncthreads();
    if (threadIdx.x < 256) {
        uint32_t v = sm.dstart[d];
#pragma unroll
        for (uint32_t q = 0; q < P; ++q) v += sm.part[q][d];
        sm.gbase[d] = v;
        sm.run[d] = 0;
    }
    __syncthreads();
}

// ---------------------------------------------------------------- keys
//
// Footprint shortcut (exact). makeKeys culls a splat when
// RN(alpha * area) < cull, area = 2 pi sqrt(max(det, 0)), det =
// (xx + .3)(yy + .3) - xy^2 of the pinned 2D covariance T Sigma T^T
// (render/splats.js:102-124, :174-178). For a perspective view, with
// d = -view.z: |J00| = |fx| / d, |J02| = |fx| |x'| / d where |x'| =
// min(|view.x| / d, 1.3 / |p00|) is the clamped slope, and likewise for row 1;
// so the absolute row sums of T = J W are at most A = |fx| / d (r0 + |x'| r2)
// and B = |fy| / d (r1 + |y'| r2), r_k the absolute row sums of the
// model-view's 3x3, and with every |Sigma_ij| <= m = 2^sexp, every entry of
// |T| |Sigma| |T|^T in row 0 is at most A^2 m and in row 1 at most B^2 m. The
// kernel evaluates these bounds with approximate operations and a 1.002
// margin (far above their few ulps, and the few ulps by which the pinned T
// exceeds the real one), giving ga, gb.
//  * Kept: if ga, gb <= 100, the pinned 2D covariance differs from a positive
//    semi-definite one by at most 7.1 u * 100 per entry, which moves det at
//    most 0.0025 below 0.09; so area >= 1.85 whatever the rounding, and every
//    alpha byte >= keep_byte (RN(alpha * 1.85) >= cull, proved by the host)
//    is kept without its footprint (or its covariance) being computed.
//  * Culled: each pinned entry is at most g (1 + 8.2u) and the pinned det at
//    most (ga (1 + 8.2u) + .3)(gb (1 + 8.2u) + .3)(1 + 3u); the kernel forms
//    that with a further 1.0001 (which covers its own few roundings) and
//    compares it with det_min[byte], the least det the cull keeps for the
//    splat's alpha byte (found exactly by the host); below it the splat is
//    culled, again without its footprint.
// Splats that neither test decides are queued for the pinned computation.

// Counts a survivor's two digits into the lane's sub-histograms.
__device__ __forceinline__ void count_key(uint32_t* hist, uint32_t key, uint32_t s) {
    atomicAdd(&hist[s * 512u + sub_slot(s, key & 255u)], 1u);
    atomicAdd(&hist[s * 512u + 256u + sub_slot(s, key >> 8)], 1u);
}

// The footprint shortcut above for one splat of a perspective view: keep_sc
// when its footprint surely passes the cull, cull_sc when it surely does not.
__device__ __forceinline__ void shortcut(const ViewConsts& c, const float view[4], uint32_t byte, int8_t sexp, float afx,
                                         float afy, float r0, float r1, float r2, float xcap, float ycap,
                                         uint32_t keep_byte, bool* keep_sc, bool* cull_sc) {
    const float d = -view[2];
    // The splat's covariance bound 2^sexp, exactly (sexp is in [-100, 127]).
    const float m = __int_as_float((int(sexp) + 127) << 23);
    // A, B and ga, gb of the shortcut above, from this splat's own position.
    const float rd = __fdividef(1.0f, d);
    const float ax = fminf(fabsf(view[0]) * rd, xcap), ay = fminf(fabsf(view[1]) * rd, ycap);
    const float A = afx * rd * (r0 + ax * r2), B = afy * rd * (r1 + ay * r2);
    const float ga = 1.002f * (A * A) * m, gb = 1.002f * (B * B) * m;
    *keep_sc = byte >= keep_byte && ga <= 100.0f && gb <= 100.0f;
    // det's pinned value is at most (ga (1 + 8.2u) + .3)(gb (1 + 8.2u) +
    // .3)(1 + 3u); below the byte's threshold, culled.
    *cull_sc = !*keep_sc && ((ga * 1.00001f + 0.3f) * (gb * 1.00001f + 0.3f)) * 1.0001f < c.det_min[byte];
}

// Sweep 1 of a keys sub-tile: tests, keys and the footprint shortcut. Every
// splat's key slot and survivor word are written now (the passes read only
// the slots whose survivor bit is set), with the digit counts of the splats
// already decided; the ones whose footprint must still be evaluated go to
// the queue. Every test is evaluated for every splat and combined as
// predicates, so a warp does not split on the data. kMode 1: the fast
// transform, the view's constants in registers (FastView); 2: that, with a
// reverse-Z infinite projection's frustum test (fast_in_frustum_revz).
template <int kMode, int NT>
__device__ __forceinline__ void keys_sweep(const ViewConsts& c, KeysSmem<NT>& sm, uint32_t buf, uint32_t base,
                                           uint32_t cnt, uint32_t n, bool fp, uint16_t* k16, uint32_t* mask) {
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const uint32_t s = lane & (kSubHist - 1);
    FastView fv;
    if constexpr (kMode > 0) fv = fast_view_of(c);
    const bool persp = c.persp;
    const float afx = c.afx, afy = c.afy, r0 = c.r0, r1 = c.r1, r2 = c.r2, xcap = c.xcap, ycap = c.ycap;
    const uint32_t keep_byte = c.keep_byte, faint_max = c.faint_max;
    const float4* centers = sm.centers[buf];
    const int8_t* sexp = sm.sexp[buf];
#pragma unroll 1
    for (int r = 0; r < kKeysIPT; ++r) {
        const uint32_t at = (uint32_t)r * NT + tid;
        if (at >= cnt) break;   // uniform across the warp: cnt is a multiple of 32
        const float4 p = centers[at];
        float view[4];
        bool inside;
        uint32_t key;
        if constexpr (kMode > 0) {
            fast_view(fv, p.x, p.y, p.z, view);
            inside = kMode == 2 ? fast_in_frustum_revz(fv, view) : fast_in_frustum(fv, view);
            key = fast_depth_key(fv, view);
        } else {
            view_of(c, p.x, p.y, p.z, view);
            inside = in_frustum(c, view);
            key = depth_key(c, view);
        }
        const uint32_t byte = __float_as_uint(p.w) >> 24;
        // too faint to reach 1/255 at or below faint_max
        bool kept = base + at < n && inside && byte > faint_max;
        bool pending = false;
        if (fp) {
            bool keep_sc = false, cull_sc = false;
            if (persp) shortcut(c, view, byte, sexp[at], afx, afy, r0, r1, r2, xcap, ycap, keep_byte, &keep_sc, &cull_sc);
            pending = kept && !keep_sc && !cull_sc;
            kept = kept && keep_sc;
        }
        k16[base + at] = (uint16_t)key;
        const uint32_t kb = __ballot_sync(0xffffffffu, kept);
        if (lane == 0) mask[(base + at) >> 5] = kb;
        if (kept) count_key(&sm.hist[0][0], key, s);
        const uint32_t pend = __ballot_sync(0xffffffffu, pending);
        if (pend) {
            uint32_t first = 0;
            if (lane == (uint32_t)(__ffs(pend) - 1)) first = atomicAdd(&sm.qn, (uint32_t)__popc(pend));
            first = __shfl_sync(0xffffffffu, first, __ffs(pend) - 1);
            if (pending) sm.queue[first + __popc(pend & lanemask_lt())] = base + at;
        }
    }
}

// Issues the bulk copies of one keys sub-tile into staging buffer b (thread 0).
template <int NT>
__device__ __forceinline__ void stage_issue(const JobDesc& J, KeysSmem<NT>& sm, uint32_t b, uint32_t base,
                                            uint32_t cnt, bool fp) {
    fence_proxy_async();
    const uint32_t bytes = cnt * 16u + (fp ? cnt : 0u);
    mbar_expect_tx(&sm.bar[b], bytes);
    bulk_copy(sm.centers[b], J.centers + base, cnt * 16u, &sm.bar[b]);
    if (fp) bulk_copy(sm.sexp[b], J.sexp + base, cnt, &sm.bar[b]);
    sm.pending |= 1u << b;
}

// Publishes a keys item's counts: the segment's low-digit counts (for the
// low pass's look-back), its group's sum, the job's totals of both digits;
// then the item's completion.
template <int NT>
__device__ void keys_publish(const JobDesc& J, uint32_t ls, KeysSmem<NT>& sm) {
    JobCtl* ctl = reinterpret_cast<JobCtl*>(J.ctl);
    // Every thread's keys and survivor words are visible on the GPU before
    // the item is counted done: the low pass reads them after acquiring the
    // job's count, with no grid-wide wait.
    __threadfence();
    __syncthreads();
    const uint32_t d = threadIdx.x;
    if (d < 256) {
        uint32_t lo = 0, hi = 0;
#pragma unroll
        for (uint32_t s = 0; s < (uint32_t)kSubHist; ++s) {
            lo += sm.hist[s][sub_slot(s, d)];
            hi += sm.hist[s][256u + sub_slot(s, d)];
        }
        J.agg[(size_t)ls * 256 + d] = lo;
        if (lo) {
            uint32_t* gsum = J.ctl + sizeof(JobCtl) / 4;
            red_add(&gsum[(size_t)(ls / kGroup) * 256 + d], lo);
            red_add(&ctl->tot[0][d], lo);
        }
        if (hi) red_add(&ctl->tot[1][d], hi);
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) red_release_add(&ctl->keys_done, 1u);
}

template <int NT>
__device__ void zero_keys_hist(KeysSmem<NT>& sm) {
    uint32_t* h = &sm.hist[0][0];
    for (uint32_t k = threadIdx.x; k < (uint32_t)kSubHist * 512u; k += NT) h[k] = 0;
}

// makeKeys' footprint cull of one splat (view coordinates `view`, covariance
// sg, threshold thr = det_min of its alpha byte): true when it keeps it.
__device__ __forceinline__ bool footprint_keep(const ViewConsts& c, const float view[4], const float sg[6], float thr) {
    // A filter first: det from the same inputs with fast arithmetic (fused
    // products, an approximate reciprocal), and a bound on how far the
    // pinned det can lie from it: every intermediate of both is within
    // about 30 ulps of its real value, relative to the magnitudes
    // |T| |Sigma| |T|^T (ga, gb below), so 2^-16 of
    // (ga + .3)(gb + .3) + ga gb bounds the difference with room to spare.
    // Outside that band of the threshold the decision is the pinned one's;
    // inside, the pinned det decides.
    float J00 = c.fx, J11 = c.fy, J02 = 0.0f, J12 = 0.0f;
    if (c.persp) {
        const float rd = __fdividef(1.0f, -view[2]);
        J00 = c.fx * rd;
        J11 = c.fy * rd;
        J02 = J00 * fminf(fmaxf(view[0] * rd, c.xlo), c.xhi);
        J12 = J11 * fminf(fmaxf(view[1] * rd, c.ylo), c.yhi);
    }
    float T0[3], T1[3], ta = 0.0f, tb = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        T0[k] = __fmaf_rn(J00, c.mv[k * 4 + 0], J02 * c.mv[k * 4 + 2]);
        T1[k] = __fmaf_rn(J11, c.mv[k * 4 + 1], J12 * c.mv[k * 4 + 2]);
        ta += fabsf(T0[k]);
        tb += fabsf(T1[k]);
    }
    const float S[3][3] = {{sg[0], sg[1], sg[2]}, {sg[1], sg[3], sg[4]}, {sg[2], sg[4], sg[5]}};
    float U0[3], U1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        U0[k] = __fmaf_rn(T0[0], S[0][k], __fmaf_rn(T0[1], S[1][k], T0[2] * S[2][k]));
        U1[k] = __fmaf_rn(T1[0], S[0][k], __fmaf_rn(T1[1], S[1][k], T1[2] * S[2][k]));
    }
    const float xx = __fmaf_rn(U0[0], T0[0], __fmaf_rn(U0[1], T0[1], U0[2] * T0[2]));
    const float xy = __fmaf_rn(U1[0], T0[0], __fmaf_rn(U1[1], T0[1], U1[2] * T0[2]));
    const float yy = __fmaf_rn(U1[0], T1[0], __fmaf_rn(U1[1], T1[1], U1[2] * T1[2]));
    const float det = __fmaf_rn(xx + 0.3f, yy + 0.3f, -(xy * xy));
    const float ms = fmaxf(fmaxf(fmaxf(fabsf(sg[0]), fabsf(sg[1])), fmaxf(fabsf(sg[2]), fabsf(sg[3]))),
                           fmaxf(fabsf(sg[4]), fabsf(sg[5])));
    const float ga = ta * ta * ms, gb = tb * tb * ms;
    const float err = 1.52587890625e-5f * __fmaf_rn(ga + 0.3f, gb + 0.3f, ga * gb);
    if (det - err >= thr) return true;
    if (det + err < thr) return false;
    return fmaxf(footprint_det(c, view, sg), 0.0f) >= thr;   // the max of makeKeys' sqrt(max(det, 0))
}

// The queued splats' footprints, densely (a warp evaluates 32 of them at
// once, whichever sub-tiles they came from): a kept splat sets its survivor
// bit and counts its digits (its key is already out). Each thread's next
// splat is fetched while it evaluates the current one, so the records'
// latency overlaps the arithmetic.
template <int NT>
__device__ void keys_footprints(const JobDesc& J, KeysSmem<NT>& sm) {
    const ViewConsts& c = sm.vc;
    const uint32_t qn = sm.qn;
    uint32_t e = threadIdx.x, i_n = 0;
    float4 p_n = make_float4(0.f, 0.f, 0.f, 0.f);
    float2 a_n = make_float2(0.f, 0.f), b_n = a_n, c_n = a_n;
    if (e < qn) {
        i_n = sm.queue[e];
        p_n = __ldg(&J.centers[i_n]);
        a_n = __ldcs(&J.cov[3 * (size_t)i_n]);
        b_n = __ldcs(&J.cov[3 * (size_t)i_n + 1]);
        c_n = __ldcs(&J.cov[3 * (size_t)i_n + 2]);
    }
    for (; e < qn; e += NT) {
        const uint32_t i = i_n;
        const float4 p = p_n;
        const float sg[6] = {a_n.x, a_n.y, b_n.x, b_n.y, c_n.x, c_n.y};
        if (e + NT < qn) {
            i_n = sm.queue[e + NT];
            p_n = __ldg(&J.centers[i_n]);
            a_n = __ldcs(&J.cov[3 * (size_t)i_n]);
            b_n = __ldcs(&J.cov[3 * (size_t)i_n + 1]);
            c_n = __ldcs(&J.cov[3 * (size_t)i_n + 2]);
        }
        float view[4];
        view_of(c, p.x, p.y, p.z, view);
        const bool keep = footprint_keep(c, view, sg, c.det_min[__float_as_uint(p.w) >> 24]);
        if (keep) {
            atomicOr(&J.mask[i >> 5], 1u << (i & 31u));
            count_key(&sm.hist[0][0], depth_key(c, view), threadIdx.x & (kSubHist - 1));
        }
    }
}

// Keys of one segment of splats, in sub-tiles of TK splats staged by bulk
// copies (double-buffered). Sweep 1 writes every splat's key slot and
// survivor word; splats whose footprint must be evaluated are queued and
// evaluated together when the queue fills or the segment ends.
template <int NT>
__device__ void keys_item(const JobDesc& J, const SegDesc& sd, KeysSmem<NT>& sm, KeysStage& ks, const LaunchDesc& L,
                          uint32_t item) {
    constexpr uint32_t TK = KeysSmem<NT>::TK;
    const uint32_t tid = threadIdx.x;
    const uint32_t a = sd.a, b = sd.b, n = J.n;
    // The first sub-tile's copy goes out before the view's constants are
    // staged (the staging buffers are free: the previous item ended with a
    // barrier after its last sweep).
    if (tid == 0 && J.vc.visible != 0 && a < b) stage_issue(J, sm, ks.buf, a, min(TK, b - a), J.vc.cull > 0.0f);
    static_assert(sizeof(ViewConsts) % 4 == 0, "copied in words");
    for (uint32_t k = tid; k < sizeof(ViewConsts) / 4; k += NT)
        reinterpret_cast<uint32_t*>(&sm.vc)[k] = reinterpret_cast<const uint32_t*>(&J.vc)[k];
    if (tid == 0) sm.qn = 0;
    zero_keys_hist(sm);
    __syncthreads();
    const ViewConsts& c = sm.vc;
    const bool any = c.visible != 0;
    const bool fp = c.cull > 0.0f;
    uint16_t* const k16 = J.k16;
    uint32_t* const mask = J.mask;
    for (uint32_t base = a; base < b; base += TK) {
        const uint32_t cnt = min(TK, b - base);
        const uint32_t buf = ks.buf;
        if (any) {
            if (tid == 0 && base + TK < b) stage_issue(J, sm, buf ^ 1u, base + TK, min(TK, b - base - TK), fp);
            const uint64_t w0 = L.trace && tid == 0 ? global_ns() : 0;
            if (!stage_wait(sm, ks, buf, L, item)) sm.drain = 1;
            if (tid == 0) {
                sm.pending &= ~(1u << buf);
                if (L.trace) sm.mark[0] += global_ns() - w0;   // time spent waiting for staged records
            }
            if (c.revz)
                keys_sweep<2>(c, sm, buf, base, cnt, n, fp, k16, mask);
            else if (c.fast)
                keys_sweep<1>(c, sm, buf, base, cnt, n, fp, k16, mask);
            else
                keys_sweep<0>(c, sm, buf, base, cnt, n, fp, k16, mask);
            ks.buf ^= 1u;
        } else {
            // Wholly behind the camera: no survivors.
            for (uint32_t w = tid; w < cnt / 32; w += NT) mask[(base >> 5) + w] = 0;
        }
        __syncthreads();   // the staging buffer is free again; the queue is complete
        if (tid == 0 && base == a) sm.mark[1] = global_ns();
        if (sm.qn > TK) {   // room for one more sub-tile's worth
            keys_footprints(J, sm);
            __syncthreads();
            if (tid == 0) sm.qn = 0;
            __syncthreads();
        }
    }
    if (sm.qn) keys_footprints(J, sm);
    __syncthreads();
    // The shade pass, fused: every survivor of the segment (its survivor bit
    // final) gets its colour as seen from the eye.
    if (J.sh) {
        for (uint32_t i = a + tid; i < b; i += NT) {
            if (!((__ldcg(&mask[i >> 5]) >> (i & 31u)) & 1u)) continue;
            const float4 p = __ldg(&J.centers[i]);
            J.shaded[i] = shade_splat(J.sh, J.sh_words, J.sh_degree, i, p.x, p.y, p.z, __float_as_uint(p.w), J.eye);
        }
    }
    if (tid == 0) sm.mark[2] = global_ns();
    keys_publish(J, sd.local, sm);
}

// Keys of one segment of an alpha emitter's ring (render/particles.js:197-209):
// a slot is live unless age >= lifetime; its depth is
// max(dot(position - eye, forward), 1e-6) (the dot product summed x, y, z in
// order, each product and sum separately rounded; max returns the non-NaN
// operand); its bucket is the one of 4096 log2-depth buckets the pinned
// bucket function of the host puts it in, found here by comparing the depth
// with that function's thresholds (thr[b] = the least depth of bucket b or
// above), starting from an estimate by log2f and correcting it; the key is
// 4095 - bucket, far first.
template <int NT>
__device__ void particle_keys_item(const JobDesc& J, const SegDesc& sd, KeysSmem<NT>& sm) {
    const uint32_t tid = threadIdx.x, lane = tid & 31u, s = lane & (kSubHist - 1);
    zero_keys_hist(sm);
    __syncthreads();
    const uint32_t n = J.n;
    const float ex = J.eye[0], ey = J.eye[1], ez = J.eye[2];
    const float fx = J.fwd[0], fy = J.fwd[1], fz = J.fwd[2];
    const float4* pool = J.pool + 2 * (size_t)J.idx_base;
    uint16_t* const k16 = J.k16;
    // Every element of the segment is visited by whole warps (its ends are
    // multiples of 32), so the survivor words are whole ballots.
    for (uint32_t i = sd.a + tid; i < sd.b; i += NT) {
        uint32_t key = 0;
        bool live = false;
        if (i < n) {
            const float4 a = __ldcs(&pool[2 * (size_t)i]);
            const float life = __ldcs(&pool[2 * (size_t)i + 1].w);
            live = !(a.w >= life);
            if (live) {
                const float dot = fadd(fadd(fmul(fsub(a.x, ex), fx), fmul(fsub(a.y, ey), fy)), fmul(fsub(a.z, ez), fz));
                const float d = fmaxf(dot, 1e-6f);
                int b = (int)fclamp(fmul(fadd(log2f(d), 10.0f), 136.5f), 0.0f, 4095.0f);
                // The estimate is within a bucket or two; the thresholds decide.
                while (b < (int)kParticleBuckets - 1 && d >= __ldg(&J.thr[b + 1])) ++b;
                while (b > 0 && d < __ldg(&J.thr[b])) --b;
                key = kParticleBuckets - 1u - (uint32_t)b;
            }
        }
        k16[i] = (uint16_t)key;
        const uint32_t kb = __ballot_sync(0xffffffffu, live);
        if (lane == 0) J.mask[i >> 5] = kb;
        if (live) count_key(&sm.hist[0][0], key, s);
    }
    keys_publish(J, sd.local, sm);
}

// Keys of one segment of a job whose keys are given (kind kJobKeys): every
// element survives with its key; the low pass reads the keys in place, so
// only the counts are made here.
template <int NT>
__device__ void given_keys_item(const JobDesc& J, const SegDesc& sd, KeysSmem<NT>& sm) {
    const uint32_t tid = threadIdx.x, s = (tid & 31u) & (kSubHist - 1);
    zero_keys_hist(sm);
    __syncthreads();
    const uint32_t end = min(sd.b, J.n);
    // 8 keys a 16-byte load where the keys are so aligned (the segment starts
    // on a multiple of 256), the rest one at a time.
    const uint16_t* const kin = J.keys_in;
    uint32_t a8 = sd.a;
    if ((reinterpret_cast<uintptr_t>(kin + sd.a) & 15u) == 0) {
        const uint32_t nv = end > sd.a ? (end - sd.a) / 8u : 0u;
        const uint4* kv = reinterpret_cast<const uint4*>(kin + sd.a);
#pragma unroll 2
        for (uint32_t k = tid; k < nv; k += NT) {
            const uint4 w = __ldg(&kv[k]);
            const uint32_t words[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                count_key(&sm.hist[0][0], words[q] & 0xFFFFu, s);
                count_key(&sm.hist[0][0], words[q] >> 16, s);
            }
        }
        a8 = sd.a + nv * 8u;
    }
    for (uint32_t i = a8 + tid; i < end; i += NT) count_key(&sm.hist[0][0], __ldg(&kin[i]), s);
    keys_publish(J, sd.local, sm);
}

// ---------------------------------------------------------------- digit passes

// One stable counting pass over 8 key bits for one segment (PASS 0: the low
// byte, over the segment's splats; PASS 1: the high byte, over its slice of
// the low pass's output).
template <int PASS, int NT>
__device__ void digit_item(const JobDesc& J, const SegDesc& sd, DigitSmem<NT>& sm, const LaunchDesc& L,
                           uint32_t item) {
    constexpr int W = DigitSmem<NT>::W;
    constexpr uint32_t IPT = kDigitIPT;
    constexpr uint32_t TD = DigitSmem<NT>::TD;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    JobCtl* ctl = reinterpret_cast<JobCtl*>(J.ctl);
    uint32_t* const look = J.ctl + sizeof(JobCtl) / 4;
    uint32_t* const gsum = look + (size_t)PASS * J.ngroups * 256;
    uint32_t* const gdone = look + (size_t)2 * J.ngroups * 256;
    uint32_t* const flag = gdone + J.ngroups;
    uint32_t* const agg = J.agg + (size_t)PASS * J.nseg * 256;
    const uint32_t ls = sd.local, g = ls / kGroup;

    // The job's previous phase, every segment of it (its items have smaller
    // tickets of the previous kernel, whose CTAs are all resident: the wait
    // ends, unless the launch left that phase out, as the failure self-test
    // does). A job's pass starts as soon as its own previous phase is done,
    // while other jobs may still be in theirs.
    if (!wait_count(PASS == 0 ? &ctl->keys_done : &ctl->low_done, J.nseg, sm, L, item)) return;
    digit_starts(ctl->tot[PASS], sm);
    const uint32_t S = sm.total;   // the job's survivors
    uint32_t lo, hi;
    if (PASS == 0) {
        lo = sd.a;
        hi = sd.b;
        if (ls == 0 && tid == 0) *J.count = S;
    } else {
        // A slice of the low pass's output in proportion to the segment's
        // share of the job's splats; neighbouring segments meet exactly.
        lo = J.npad ? (uint32_t)((uint64_t)sd.a * S / J.npad) : 0u;
        hi = J.npad ? (uint32_t)((uint64_t)sd.b * S / J.npad) : 0u;
        // The slice's high-digit counts, published for the later segments.
        uint32_t* h = &sm.hist[0][0];
        for (uint32_t k = tid; k < (uint32_t)kSubHist * 256u; k += NT) h[k] = 0;
        __syncthreads();
        const uint32_t s = lane & (kSubHist - 1);
        const uint16_t* kb = J.key_b;
        // The slice's keys 8 at a time (16-byte loads from its first 8-key
        // boundary; key_b is 256-byte aligned), the few before and after it
        // one at a time: many bytes in flight, so the count is not bound by
        // the loads' latency.
        const uint32_t a8 = min(hi, (lo + 7u) & ~7u), b8 = max(a8, hi & ~7u);
        for (uint32_t e = lo + tid; e < a8; e += NT) atomicAdd(&h[s * 256u + sub_slot(s, __ldcg(&kb[e]) >> 8)], 1u);
        for (uint32_t e = b8 + tid; e < hi; e += NT) atomicAdd(&h[s * 256u + sub_slot(s, __ldcg(&kb[e]) >> 8)], 1u);
        const uint4* kv = reinterpret_cast<const uint4*>(kb + a8);
#pragma unroll 2
        for (uint32_t k = tid; k < (b8 - a8) / 8u; k += NT) {
            const uint4 w = __ldcg(&kv[k]);
            const uint32_t words[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                atomicAdd(&h[s * 256u + sub_slot(s, (words[q] >> 8) & 255u)], 1u);
                atomicAdd(&h[s * 256u + sub_slot(s, words[q] >> 24)], 1u);
            }
        }
        __syncthreads();
        if (tid < 256) {
            uint32_t v = 0;
#pragma unroll
            for (uint32_t q = 0; q < (uint32_t)kSubHist; ++q) v += h[q * 256u + sub_slot(q, tid)];
            agg[(size_t)ls * 256 + tid] = v;
            if (v) red_add(&gsum[(size_t)g * 256 + tid], v);
            __threadfence();
        }
        __syncthreads();
        if (tid == 0) {
            st_release(&flag[ls], 1u);
            red_release_add(&gdone[g], 1u);
        }
        if (warp == 0) {
            // The look-back: every earlier group complete, every earlier
            // segment of this group published (all have smaller tickets).
            // Lane k polls the k-th of these words, so one round trip
            // covers 32 of them.
            const uint32_t nflags = ls - g * kGroup, targets = g + nflags;
            uint32_t spins = 0;
            bool fail = false;
            for (uint32_t t0 = 0; t0 < targets && !fail; t0 += 32) {
                const uint32_t t = t0 + lane;
                bool met = t >= targets;
                for (;;) {
                    if (!met) {
                        if (t < g)
                            met = ld_acquire(&gdone[t]) >= min(kGroup, J.nseg - t * kGroup);
                        else
                            met = ld_acquire(&flag[g * kGroup + (t - g)]) != 0;
                    }
                    if (__all_sync(0xffffffffu, met)) break;
                    if (++spins > L.spin_limit || *(volatile uint32_t*)L.err) {
                        fail = true;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            if (lane == 0) {
                sm.abort = fail;
                if (fail) raise_error(L.err, kErrWaitPhase, item);
            }
        }
        __syncthreads();
        if (sm.abort) return;
    }
    segment_prefix(gsum, agg, g, ls, sm);
    if (tid == 0) sm.mark[0] = global_ns();

    const bool given = PASS == 0 && J.kind == kJobKeys;
    const uint16_t* const kin = PASS == 0 ? (given ? J.keys_in : J.k16) : J.key_b;
    const uint32_t* const mask = J.mask;
    const uint32_t* const idx_in = J.idx_b;
    const uint32_t n = J.n, idx_base = J.idx_base;
    uint16_t* const key_b = J.key_b;
    uint32_t* const idx_b = J.idx_b;
    uint32_t* const order = J.order;
    uint32_t* const keys_out = J.keys;
    const uint32_t lt = lanemask_lt();
    uint32_t* const wm = sm.wmask[warp];
    uint16_t* const wc = sm.wcnt[warp];
    {
        uint32_t* z = &sm.wmask[0][0];
        for (uint32_t k = tid; k < (uint32_t)W * 256u; k += NT) z[k] = 0;
        uint32_t* zc = reinterpret_cast<uint32_t*>(&sm.wcnt[0][0]);
        for (uint32_t k = tid; k < (uint32_t)W * 128u; k += NT) zc[k] = 0;
    }
    __syncthreads();

    // Element e of a sub-tile at b0 goes to warp w = (e - b0) / (32 IPT),
    // round r, lane e % 32: warps, rounds and lanes follow the element order.
    // Each sub-tile's inputs are loaded one sub-tile ahead (nk, nx), so their
    // latency overlaps the previous sub-tile's ranks, staging and writes.
    uint32_t nk[IPT], nx[IPT];
#define WS_FETCH(b0)                                                                \
    _Pragma("unroll") for (uint32_t r = 0; r < IPT; ++r) {                        \
        const uint32_t e = (b0) + (warp * IPT + r) * 32u + lane;                  \
        nk[r] = 0xFFFFFFFFu;                                                        \
        nx[r] = 0;                                                                  \
        if (e < hi) {                                                               \
            if (PASS == 1) {                                                        \
                nk[r] = __ldcg(&kin[e]);                                            \
                nx[r] = __ldcg(&idx_in[e]);                                         \
            } else if (given) {                                                     \
                /* given keys are read only below n */                             \
                if (e < n) nk[r] = __ldcg(&kin[e]);                                 \
                nx[r] = 0xFFFFFFFFu;                                                \
            } else {                                                                \
                nk[r] = __ldcg(&kin[e]);                                            \
                nx[r] = __ldcg(&mask[e >> 5]);                                      \
            }                                                                       \
        }                                                                           \
    }
    if (lo < hi) {
        WS_FETCH(lo)
    }
    for (uint32_t base = lo; base < hi; base += TD) {
        // kr: the key in bits 0-15 and its rank within the warp's digit
        // above, or 0xFFFFFFFF for no element.
        uint32_t kr[IPT], ix[IPT];
#pragma unroll
        for (uint32_t r = 0; r < IPT; ++r) {
            const bool v = nk[r] != 0xFFFFFFFFu && (PASS == 1 || ((nx[r] >> lane) & 1u));
            kr[r] = v ? nk[r] : 0xFFFFFFFFu;
            ix[r] = nx[r];
        }
        if (base + TD < hi) {
            WS_FETCH(base + TD)
        }
        // Rank within the warp, round by round.
#pragma unroll
        for (uint32_t r = 0; r < IPT; ++r) {
            const bool v = kr[r] != 0xFFFFFFFFu;
            if (__any_sync(0xffffffffu, v)) {
                const uint32_t d = PASS == 0 ? (kr[r] & 255u) : ((kr[r] >> 8) & 255u);
                if (v) atomicOr(&wm[d], 1u << lane);
                __syncwarp();
                uint32_t peers = 0, prior = 0;
                if (v) {
                    peers = wm[d];
                    prior = wc[d];
                }
                __syncwarp();
                if (v && lane == 31u - __clz(peers)) {
                    wm[d] = 0;
                    wc[d] = (uint16_t)(prior + __popc(peers));
                }
                __syncwarp();
                if (v) kr[r] |= (prior + __popc(peers & lt)) << 16;
            }
        }
        __syncthreads();
        // Thread d: each warp's start within digit d, and the sub-tile's
        // count of d; then the sub-tile start of every digit.
        uint32_t tc = 0, x = 0;
        if (tid < 256) {
#pragma unroll 8
            for (int w = 0; w < W; ++w) {
                const uint32_t c = sm.wcnt[w][tid];
                sm.wcnt[w][tid] = (uint16_t)tc;
                tc += c;
            }
            x = tc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= (uint32_t)o) x += y;
            }
            if (lane == 31) sm.scan[warp] = x;
        }
        __syncthreads();
        if (tid < 256) {
            uint32_t off = 0;
#pragma unroll
            for (uint32_t w = 0; w < 8; ++w) off += w < warp ? sm.scan[w] : 0u;
            const uint32_t ls0 = off + x - tc;
            sm.lstart[tid] = ls0;
            sm.gofs[tid] = sm.gbase[tid] + sm.run[tid] - ls0;
            sm.run[tid] += tc;
            if (tid == 255) sm.tile_total = off + x;
        }
        __syncthreads();
        // Stage in sub-tile order (digit, then element order).
#pragma unroll
        for (uint32_t r = 0; r < IPT; ++r) {
            if (kr[r] == 0xFFFFFFFFu) continue;
            const uint32_t d = PASS == 0 ? (kr[r] & 255u) : ((kr[r] >> 8) & 255u);
            const uint32_t slot = sm.lstart[d] + wc[d] + (kr[r] >> 16);
            sm.skey[slot] = (uint16_t)kr[r];
            sm.sidx[slot] = PASS == 0 ? idx_base + base + (warp * IPT + r) * 32u + lane : ix[r];
        }
        if (tid == 0 && base == lo) sm.mark[1] = global_ns();
        __syncthreads();
        // Write out: consecutive threads take consecutive slots, so a digit's
        // run goes out as consecutive addresses. The warp counters are cleared
        // meanwhile (nothing reads them until the next sub-tile's ranks).
        const uint32_t tt = sm.tile_total;
        {
            uint32_t* zc = reinterpret_cast<uint32_t*>(&sm.wcnt[0][0]);
            for (uint32_t k = tid; k < (uint32_t)W * 128u; k += NT) zc[k] = 0;
        }
#pragma unroll 4
        for (uint32_t i = tid; i < tt; i += NT) {
            const uint32_t k = sm.skey[i];
            const uint32_t d = PASS == 0 ? (k & 255u) : (k >> 8);
            const uint32_t gp = sm.gofs[d] + i;
            if (gp >= S) {   // only reachable if counts disagree: record, do not write
                raise_error(L.err, kErrBounds, item);
                continue;
            }
            if (PASS == 0) {
                key_b[gp] = (uint16_t)k;
                idx_b[gp] = sm.sidx[i];
            } else {
                __stcs(&order[gp], sm.sidx[i]);
                if (keys_out) __stcs(&keys_out[gp], k);
            }
        }
        __syncthreads();
    }
#undef WS_FETCH
    if (tid == 0) sm.mark[2] = global_ns();
    // The item is counted done once every thread's writes are visible: the
    // high pass reads the low pass's output, and a host-output copy reads the
    // job's final order, after acquiring these counts.
    __threadfence();
    __syncthreads();
    if (tid == 0) red_release_add(PASS == 0 ? &ctl->low_done : &ctl->high_done, 1u);
}

// ---------------------------------------------------------------- the kernels

// Lets the stream's next kernel (launched with programmatic stream
// serialization) schedule its CTAs once every CTA here has called it or
// exited. A kernel that calls wait_prerequisites (griddepcontrol.wait) then
// waits until the grids before it have finished and their writes are
// visible; the digit passes do not, and order their reads by each job's
// completion counts instead (release by the writer, acquire by the reader).
__device__ __forceinline__ void allow_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void wait_prerequisites() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---------------------------------------------------------------- one-CTA sorts
//
// A job of at most kOneMax splats sorted by one CTA in its shared memory, in
// one kernel: every splat's key and survivor bit into shared memory, then
// the survivors placed in (key, index) order, straight into the outputs.
// kCounting: one counting pass over all 65536 keys (the counts of every key,
// their exclusive scan, then one warp walks the splats in index order and
// gives each the next slot of its key; a key's peers within the 32 are
// ranked by their lanes). Otherwise two stable 8-bit passes, low digit then
// high, all warps at once: each warp takes a contiguous run of the pass's
// input, its per-digit starts from the counts of the runs before it.

template <bool kCounting, int NT>
struct OneSmem {
    static constexpr int W = NT / 32;
    ViewConsts vc;
    uint32_t total;                              // survivors
    uint32_t scan[32];
    uint32_t live[kOneMax / 32];                 // survivor bits
    uint16_t key[kOneMax];                       // each splat's key
    // counting: the counts of all 65536 keys, two 16-bit halves a word; then
    // each key's next slot. radix: the low pass's output (keys and indices),
    // each warp's counts of its run per digit (then its next slot), and the
    // lanes of a round per warp and digit.
    union {
        uint32_t hist[kCounting ? 32768 : 1];
        struct {
            uint16_t key1[kOneMax];
            uint16_t idx1[kOneMax];
            uint32_t off[W][256];
            uint32_t wm[W][256];
            uint32_t tot[256];
        } r;
    } u;
};

// Exclusive scan of v over the CTA's NT threads (NT <= 1024); the CTA's
// total in *total. Every thread calls it.
template <int NT>
__device__ __forceinline__ uint32_t cta_exclusive_scan(uint32_t v, uint32_t* scan, uint32_t* total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) scan[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (uint32_t)(NT / 32) ? scan[lane] : 0u;
        const uint32_t w0 = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        if (lane < (uint32_t)(NT / 32)) scan[lane] = w - w0;
        if (lane == 31) *total = w;
    }
    __syncthreads();
    const uint32_t r = scan[warp] + x - v;
    __syncthreads();   // scan[] may be reused by the caller
    return r;
}

// One stable 8-bit pass of the one-CTA radix sort over m elements: input
// element e is (key(e), idx(e)) when valid(e); warp w takes the elements
// [w ch, (w + 1) ch). Each survivor goes to slot out(pos, key, idx).
template <int NT, class In, class Out>
__device__ __forceinline__ void one_pass(OneSmem<false, NT>& sm, uint32_t m, uint32_t shift, In in, Out out) {
    constexpr int W = NT / 32;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t ch = ((m + W - 1) / W + 31u) & ~31u;
    const uint32_t a = min(warp * ch, m), b = min(a + ch, m);
    for (uint32_t k = tid; k < (uint32_t)W * 256u; k += NT) {
        (&sm.u.r.off[0][0])[k] = 0;
        (&sm.u.r.wm[0][0])[k] = 0;
    }
    __syncthreads();
    uint32_t* const off = sm.u.r.off[warp];
    uint32_t* const wm = sm.u.r.wm[warp];
    for (uint32_t e = a + lane; e < b; e += 32) {
        uint32_t k, x;
        if (in(e, &k, &x)) atomicAdd(&off[(k >> shift) & 255u], 1u);
    }
    __syncthreads();
    // Digit-major starts: digit d's runs in warp order, the digits in order.
    if (tid < 256) {
        uint32_t run = 0;
        for (int w = 0; w < W; ++w) {
            const uint32_t c = sm.u.r.off[w][tid];
            sm.u.r.off[w][tid] = run;
            run += c;
        }
        sm.u.r.tot[tid] = run;
    }
    __syncthreads();
    const uint32_t t = tid < 256 ? sm.u.r.tot[tid] : 0u;
    const uint32_t start = cta_exclusive_scan<NT>(t, sm.scan, &sm.total);
    if (tid < 256)
        for (int w = 0; w < W; ++w) sm.u.r.off[w][tid] += start;
    __syncthreads();
    const uint32_t lt = lanemask_lt();
    for (uint32_t e0 = a; e0 < b; e0 += 32) {
        const uint32_t e = e0 + lane;
        uint32_t k = 0, x = 0;
        const bool v = e < b && in(e, &k, &x);
        const uint32_t d = (k >> shift) & 255u;
        if (v) atomicOr(&wm[d], 1u << lane);
        __syncwarp();
        uint32_t peers = 0, prior = 0;
        if (v) {
            peers = wm[d];
            prior = off[d];
        }
        __syncwarp();
        if (v && lane == 31u - __clz(peers)) {
            wm[d] = 0;
            off[d] = prior + __popc(peers);
        }
        __syncwarp();
        if (v) out(prior + __popc(peers & lt), k, x);
    }
    __syncthreads();
}

template <bool kCounting, int NT>
__global__ void __launch_bounds__(NT, 1) one_kernel(const __grid_constant__ LaunchDesc L) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    OneSmem<kCounting, NT>& sm = *reinterpret_cast<OneSmem<kCounting, NT>*>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    wait_prerequisites();   // the job table
    if (*(volatile uint32_t*)L.err) return;
    const JobDesc& J = L.jobs[blockIdx.x];
    static_assert(sizeof(ViewConsts) % 4 == 0, "copied in words");
    for (uint32_t k = tid; k < sizeof(ViewConsts) / 4; k += NT)
        reinterpret_cast<uint32_t*>(&sm.vc)[k] = reinterpret_cast<const uint32_t*>(&J.vc)[k];
    if (kCounting)
        for (uint32_t k = tid; k < 32768u; k += NT) sm.u.hist[k] = 0;
    __syncthreads();
    const ViewConsts& c = sm.vc;
    const uint32_t n = min(J.n, kOneMax);
    const bool fp = c.cull > 0.0f, any = c.visible != 0;
    // Keys and survivors, as the keys phase decides them.
    for (uint32_t e0 = 0; e0 < n; e0 += NT) {
        const uint32_t e = e0 + tid;
        bool kept = false;
        uint32_t key = 0;
        if (e < n && any) {
            const float4 p = __ldg(&J.centers[e]);
            float view[4];
            view_of(c, p.x, p.y, p.z, view);
            key = depth_key(c, view);
            const uint32_t byte = __float_as_uint(p.w) >> 24;
            kept = in_frustum(c, view) && byte > c.faint_max;
            if (kept && fp) {
                bool keep_sc = false, cull_sc = false;
                if (c.persp)
                    shortcut(c, view, byte, J.sexp[e], c.afx, c.afy, c.r0, c.r1, c.r2, c.xcap, c.ycap, c.keep_byte,
                             &keep_sc, &cull_sc);
                if (!keep_sc) {
                    kept = false;
                    if (!cull_sc) {
                        const float2 a = __ldg(&J.cov[3 * (size_t)e]), b = __ldg(&J.cov[3 * (size_t)e + 1]),
                                     q = __ldg(&J.cov[3 * (size_t)e + 2]);
                        const float sg[6] = {a.x, a.y, b.x, b.y, q.x, q.y};
                        kept = footprint_keep(c, view, sg, c.det_min[byte]);
                    }
                }
            }
        }
        if (e < n) sm.key[e] = (uint16_t)key;
        const uint32_t kb = __ballot_sync(0xffffffffu, kept);
        if (lane == 0 && e < n) sm.live[e >> 5] = kb;
        if (kCounting && kept) atomicAdd(&sm.u.hist[key >> 1], 1u << ((key & 1u) * 16u));
    }
    __syncthreads();
    // The shade pass, fused: every survivor's colour as seen from the eye.
    if (J.sh)
        for (uint32_t e = tid; e < n; e += NT)
            if ((sm.live[e >> 5] >> (e & 31u)) & 1u) {
                const float4 p = __ldg(&J.centers[e]);
                J.shaded[e] = shade_splat(J.sh, J.sh_words, J.sh_degree, e, p.x, p.y, p.z, __float_as_uint(p.w), J.eye);
            }
    const uint32_t idx_base = J.idx_base;
    uint32_t* const order = J.order;
    uint32_t* const keys_out = J.keys;
    if constexpr (kCounting) {
        // Each thread's 65536 / NT keys: their counts' sum, the CTA's scan,
        // then each key's first slot (below 2^16: n <= kOneMax).
        constexpr uint32_t KW = 32768u / NT;   // words a thread owns
        uint32_t* const h = &sm.u.hist[tid * KW];
        uint32_t sum = 0;
        for (uint32_t k = 0; k < KW; ++k) sum += (h[k] & 0xFFFFu) + (h[k] >> 16);
        uint32_t run = cta_exclusive_scan<NT>(sum, sm.scan, &sm.total);
        for (uint32_t k = 0; k < KW; ++k) {
            const uint32_t lo = h[k] & 0xFFFFu, hi = h[k] >> 16;
            h[k] = run | ((run + lo) << 16);
            run += lo + hi;
        }
        __syncthreads();
        if (tid == 0) *J.count = sm.total;
        if (warp == 0) {
            const uint32_t lt = lanemask_lt();
            for (uint32_t b0 = 0; b0 < n; b0 += 32) {
                const uint32_t e = b0 + lane;
                const bool v = e < n && ((sm.live[b0 >> 5] >> lane) & 1u);
                const uint32_t k = v ? (uint32_t)sm.key[e] : (0x10000u | lane);
                const uint32_t peers = __match_any_sync(0xffffffffu, k);
                const uint32_t sh = (k & 1u) * 16u;
                const uint32_t prior = v ? (sm.u.hist[k >> 1] >> sh) & 0xFFFFu : 0u;
                __syncwarp();
                if (v && lane == 31u - __clz(peers)) atomicAdd(&sm.u.hist[k >> 1], (uint32_t)__popc(peers) << sh);
                __syncwarp();
                if (v) {
                    const uint32_t r = prior + __popc(peers & lt);
                    order[r] = idx_base + e;
                    if (keys_out) keys_out[r] = k;
                }
            }
        }
    } else {
        // Low digit: the splats (survivors only) into key1 / idx1, compacted.
        one_pass<NT>(
            sm, n, 0u,
            [&](uint32_t e, uint32_t* k, uint32_t* x) {
                *k = sm.key[e];
                *x = e;
                return ((sm.live[e >> 5] >> (e & 31u)) & 1u) != 0u;
            },
            [&](uint32_t pos, uint32_t k, uint32_t x) {
                sm.u.r.key1[pos] = (uint16_t)k;
                sm.u.r.idx1[pos] = (uint16_t)x;
            });
        const uint32_t s = sm.total;
        if (tid == 0) *J.count = s;
        // High digit: straight into the outputs.
        one_pass<NT>(
            sm, s, 8u,
            [&](uint32_t e, uint32_t* k, uint32_t* x) {
                *k = sm.u.r.key1[e];
                *x = sm.u.r.idx1[e];
                return true;
            },
            [&](uint32_t pos, uint32_t k, uint32_t x) {
                order[pos] = idx_base + x;
                if (keys_out) keys_out[pos] = k;
            });
    }
    // The job's outputs are final: counted as all of its segments, for a
    // host-output copy that waits on them.
    __threadfence();
    __syncthreads();
    if (tid == 0) red_release_add(&reinterpret_cast<JobCtl*>(J.ctl)->high_done, J.nseg);
}

template <bool kCounting>
static cudaError_t launch_one_variant(const LaunchDesc& L, cudaStream_t stream) {
    static bool ready = false;   // the attribute is per function, set once per process
    constexpr size_t bytes = sizeof(OneSmem<kCounting, kOneThreads>);
    if (!ready) {
        const cudaError_t e =
            cudaFuncSetAttribute(one_kernel<kCounting, kOneThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        ready = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(L.njobs);
    cfg.blockDim = dim3(kOneThreads);
    cfg.dynamicSmemBytes = bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, one_kernel<kCounting, kOneThreads>, L);
}

// Host-side launcher of the one-CTA sorts: one CTA per job of L.jobs (every
// one a job of splats of at most kOneMax).
cudaError_t launch_one(const LaunchDesc& L, uint32_t algorithm, cudaStream_t stream) {
    if (L.njobs == 0) return cudaSuccess;
    return algorithm == kAlgoOneCount ? launch_one_variant<true>(L, stream) : launch_one_variant<false>(L, stream);
}


// Work item `seg` of the launch: from the segment table, or the lone job's
// consecutive chunks.
__device__ __forceinline__ SegDesc segment_of(const LaunchDesc& L, uint32_t seg) {
    if (L.segs) return L.segs[seg];
    SegDesc sd;
    const uint32_t npad = L.jobs[0].npad;
    sd.job = 0;
    sd.a = min(seg * L.chunk, npad);
    sd.b = min(sd.a + L.chunk, npad);
    sd.local = seg;
    return sd;
}

template <class SM>
__device__ __forceinline__ void claim_next(SM& sm, uint32_t* ticket, uint32_t* err) {
    if (threadIdx.x == 0) {
        sm.next = atomicAdd(ticket, 1u);
        sm.drain = *(volatile uint32_t*)err;
    }
}

__device__ __forceinline__ void trace_item(const LaunchDesc& L, uint32_t slot, uint32_t it, uint64_t claim,
                                           uint64_t start, const uint64_t* mark) {
    TraceRec r;
    r.claim = claim;
    r.start = start;
    r.end = global_ns();
    r.item = it;
    r.sm = sm_id();
    for (int q = 0; q < 3; ++q) r.mark[q] = mark[q];
    L.trace[slot] = r;
}

// The keys phase: one work item per segment.
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) keys_kernel(const __grid_constant__ LaunchDesc L) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    KeysSmem<NT>& sm = *reinterpret_cast<KeysSmem<NT>*>(smem_raw);
    const uint32_t tid = threadIdx.x;
    if (tid == 0) {
        sm.pending = 0;
        mbar_init(&sm.bar[0]);
        mbar_init(&sm.bar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_proxy_async();
    }
    wait_prerequisites();   // the job table and the zeroed counters
    // The low pass may launch now: its CTAs take the SMs this kernel's CTAs
    // leave, and its items wait for their own job's keys.
    allow_dependents();
    claim_next(sm, &L.lctl->ticket[kPhaseKeys], L.err);
    KeysStage ks{0u, 0u};
    uint64_t t_claim = 0, t_start = 0;
    if (L.trace && tid == 0) t_claim = global_ns();
    for (;;) {
        __syncthreads();   // the previous item's shared state is no longer read
        const uint32_t it = sm.next;
        if (it >= L.nseg) break;
        const SegDesc sd = segment_of(L, it);
        const JobDesc& J = L.jobs[sd.job];
        if (!sm.drain) {   // after an error: claim the remaining items, do no work
            if (L.trace && tid == 0) {
                t_start = global_ns();
                sm.mark[0] = sm.mark[1] = sm.mark[2] = 0;
            }
            if (J.kind == kJobParticles)
                particle_keys_item(J, sd, sm);
            else if (J.kind == kJobKeys)
                given_keys_item(J, sd, sm);
            else
                keys_item(J, sd, sm, ks, L, it);
            __syncthreads();
            if (L.trace && tid == 0) trace_item(L, it, it, t_claim, t_start, sm.mark);
        }
        claim_next(sm, &L.lctl->ticket[kPhaseKeys], L.err);
        if (L.trace && tid == 0) t_claim = global_ns();
    }
    // No bulk copy into this CTA's shared memory outlives it (one is only
    // left in flight if a wait gave up).
    if (tid == 0) {
        for (uint32_t b = 0; b < 2; ++b) {
            if (!((sm.pending >> b) & 1u)) continue;
            uint32_t spins = 0;
            while (!mbar_try_wait(&sm.bar[b], (ks.parity >> b) & 1u) && ++spins < L.spin_limit) {
            }
        }
    }
}

// A digit pass (PASS 0: low byte, 1: high byte): one work item per segment.
template <int PASS, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) digit_kernel(const __grid_constant__ LaunchDesc L) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    DigitSmem<NT>& sm = *reinterpret_cast<DigitSmem<NT>*>(smem_raw);
    const uint32_t tid = threadIdx.x;
    // No grid-wide wait for the previous kernel: each item waits for its own
    // job's previous phase (digit_item). The next pass may launch now.
    allow_dependents();
    claim_next(sm, &L.lctl->ticket[kPhaseLow + PASS], L.err);
    uint64_t t_claim = 0, t_start = 0;
    if (L.trace && tid == 0) t_claim = global_ns();
    for (;;) {
        __syncthreads();
        const uint32_t it = sm.next;
        if (it >= L.nseg) break;
        const SegDesc sd = segment_of(L, it);
        const JobDesc& J = L.jobs[sd.job];
        if (!sm.drain) {
            if (L.trace && tid == 0) {
                t_start = global_ns();
                sm.mark[0] = sm.mark[1] = sm.mark[2] = 0;
            }
            digit_item<PASS>(J, sd, sm, L, it);
            __syncthreads();
            if (L.trace && tid == 0) trace_item(L, (kPhaseLow + PASS) * L.nseg + it, it, t_claim, t_start, sm.mark);
        }
        claim_next(sm, &L.lctl->ticket[kPhaseLow + PASS], L.err);
        if (L.trace && tid == 0) t_claim = global_ns();
    }
}

// Keys CTAs: 768 threads, one an SM (up to 85 registers a thread).
constexpr int kKeysThreads = 768;

template <class K>
static cudaError_t set_smem(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// A launch that may begin while the stream's previous kernel finishes (its
// CTAs wait in griddepcontrol.wait).
template <class K>
static cudaError_t launch_dependent(K kernel, int grid, int threads, size_t smem, cudaStream_t stream,
                                    const LaunchDesc& L) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, L);
}

template <int NT, int MINB>
static cudaError_t prepare_digit() {
    static bool done = false;   // the attributes are per function, set once per process
    if (done) return cudaSuccess;
    cudaError_t e;
    if ((e = set_smem(digit_kernel<0, NT, MINB>, sizeof(DigitSmem<NT>))) != cudaSuccess) return e;
    if ((e = set_smem(digit_kernel<1, NT, MINB>, sizeof(DigitSmem<NT>))) != cudaSuccess) return e;
    done = true;
    return cudaSuccess;
}

static cudaError_t prepare_keys() {
    static bool done = false;
    if (done) return cudaSuccess;
    const cudaError_t e = set_smem(keys_kernel<kKeysThreads, 1>, sizeof(KeysSmem<kKeysThreads>));
    if (e == cudaSuccess) done = true;
    return e;
}

template <int NT, int MINB>
static cudaError_t launch_digits(const LaunchDesc& L, int grid, cudaStream_t stream) {
    cudaError_t e = prepare_digit<NT, MINB>();
    if (e != cudaSuccess) return e;
    if (L.first_phase <= kPhaseLow &&
        (e = launch_dependent(digit_kernel<0, NT, MINB>, grid, NT, sizeof(DigitSmem<NT>), stream, L)) != cudaSuccess)
        return e;
    return launch_dependent(digit_kernel<1, NT, MINB>, grid, NT, sizeof(DigitSmem<NT>), stream, L);
}

// Host-side launcher: the keys kernel (unless L.first_phase leaves it out),
// one CTA an SM, then the two digit passes, `grid` CTAs of `threads` threads:
// 1024 (one CTA an SM) or 512 (two).
cudaError_t launch_sort(const LaunchDesc& L, int threads, int grid, int sms, cudaStream_t stream) {
    cudaError_t e;
    if (L.first_phase == kPhaseKeys) {
        if ((e = prepare_keys()) != cudaSuccess) return e;
        const int kg = (int)min((uint32_t)sms, L.nseg);
        if ((e = launch_dependent(keys_kernel<kKeysThreads, 1>, kg, kKeysThreads, sizeof(KeysSmem<kKeysThreads>),
                                  stream, L)) != cudaSuccess)
            return e;
    }
    if (threads == 512) return launch_digits<512, 2>(L, grid, stream);
    return launch_digits<1024, 1>(L, grid, stream);
}

template <int NT, int MINB>
static int occupancy_digit() {
    int blocks = 0;
    if (prepare_digit<NT, MINB>() != cudaSuccess) return 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, digit_kernel<0, NT, MINB>, NT, sizeof(DigitSmem<NT>));
    return blocks;
}

// Resident digit-pass CTAs per SM of the variant with `threads` threads.
int sort_occupancy(int threads) {
    static int cached[2] = {0, 0};
    const int k = threads == 512 ? 1 : 0;
    if (!cached[k]) cached[k] = k ? occupancy_digit<512, 2>() : occupancy_digit<1024, 1>();
    return cached[k];
}

}  // namespace wsort
