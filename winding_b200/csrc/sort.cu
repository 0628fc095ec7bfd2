// The persistent sort kernel: every (cloud, view) job's keys, survivor
// compaction and stable two-digit radix sort, for any number of jobs, in one
// launch.
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
// Items are claimed in ticket order by a persistent grid: every segment's
// keys, then every low pass, then every high pass. An item waits only for
// items with smaller tickets (the job's earlier phase, or its own phase's
// earlier segments, which publish their counts before they wait), all
// claimed by running CTAs, so the queue always drains, whatever else shares
// the GPU. Every wait is bounded: after spin_limit polls the kernel records
// an error and every CTA drains the remaining items without work.
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

template <int NT>
struct SortSmem {
    static constexpr int W = NT / 32;
    static constexpr int TK = NT * kKeysIPT;     // splats of a keys sub-tile
    static constexpr int TD = NT * kDigitIPT;    // elements of a digit-pass sub-tile
    alignas(8) uint64_t bar[2];                  // the keys staging buffers' mbarriers
    float alpha[256];                            // unpack4x8unorm(..).a: byte / 255, correctly rounded
    ViewConsts vc;
    int vc_job;                                  // job whose constants vc holds
    uint32_t next;                               // the ticket this CTA works on next
    uint32_t drain;
    uint32_t abort;
    uint32_t total;                              // survivors of the item's job
    uint32_t tile_total;                         // elements of the current sub-tile
    uint32_t pending;                            // staging buffers with a copy in flight (bits)
    uint32_t scan[W];
    uint64_t mark[3];                            // tracing: timestamps inside an item
    uint32_t dstart[256];                        // start of each digit in the pass's output
    uint32_t gbase[256];                         // dstart plus the segments before this one
    uint32_t run[256];                           // placed by the item's earlier sub-tiles
    uint32_t gofs[256];                          // gbase + run - sub-tile start, per digit
    uint32_t lstart[256];                        // sub-tile start of each digit
    uint32_t part[NT / 256][256];                // partial sums of the look-back
    union alignas(128) U {
        struct K {
            float4 centers[2][TK];
            int8_t sexp[2][TK];
            uint32_t maskw[TK / 32];             // survivor bits of the sub-tile
            uint16_t queue[TK];                  // splats whose footprint must be evaluated
            uint32_t qn;
            uint32_t hist[kSubHist][512];        // low digit at [s][..256), high at [s][256..)
        } k;
        struct P {
            uint32_t wmask[W][256];              // per warp and digit: lanes of the round
            uint16_t wcnt[W][256];               // per warp and digit: count, then the warp's start
            uint16_t skey[TD];                   // the sub-tile staged in output order
            uint32_t sidx[TD];
            uint32_t hist[kSubHist][256];        // high pass: the segment's counts
        } p;
    } u;
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
__device__ __forceinline__ bool stage_wait(SortSmem<NT>& sm, KeysStage& ks, uint32_t b, const LaunchDesc& L,
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
template <int NT>
__device__ bool wait_count(const uint32_t* p, uint32_t need, SortSmem<NT>& sm, const LaunchDesc& L, uint32_t item) {
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
__device__ void digit_starts(const uint32_t* tot, SortSmem<NT>& sm) {
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
                               SortSmem<NT>& sm) {
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
// Footprint shortcut (exact): for a perspective view the host proves
// keep_q 2^sexp <= 100 d^2 implies every entry of |T| |Sigma| |T|^T is at most
// 100 (T = J W, d = -view.z, sexp the splat's covariance exponent bound), and
// then the pinned computation of the area cannot fall below 1.85, whatever
// the rounding: the 2D covariance differs from a positive semi-definite one
// by at most 7.1 u * 100 per entry, which moves (xx + .3)(yy + .3) - xy^2 at
// most 0.0025 below 0.09. So alpha * area >= RN(alpha * 1.85) >= cull for
// every alpha byte >= keep_byte, and such a splat is kept without its
// footprint (or its covariance) being computed. The same analysis bounds the
// pinned area from above for any G = the largest entry of |T| |Sigma| |T|^T
// (G <= 1.002 keep_q 2^sexp / d^2): every 2D entry is at most G (1 + 8.2u),
// so the area is at most 2 pi (1.00001 G + 0.3)(1 + 5u); a splat with alpha
// times that below cull is culled, again without its footprint.

// Counts a survivor's two digits into the lane's sub-histograms.
__device__ __forceinline__ void count_key(uint32_t* hist, uint32_t key, uint32_t s) {
    atomicAdd(&hist[s * 512u + sub_slot(s, key & 255u)], 1u);
    atomicAdd(&hist[s * 512u + 256u + sub_slot(s, key >> 8)], 1u);
}

// Sweep 1 of a keys sub-tile: tests, keys and the footprint shortcut. Every
// splat's key slot is written now (the passes read only the slots whose
// survivor bit is set), with the survivor bits and digit counts of the
// splats already decided; the ones whose footprint must still be evaluated
// go to a queue. kFast: the fast transform, the view's constants in
// registers (FastView).
template <bool kFast, int NT>
__device__ __forceinline__ void keys_sweep(const ViewConsts& c, SortSmem<NT>& sm, uint32_t buf, uint32_t base,
                                           uint32_t cnt, uint32_t n, bool fp, uint16_t* k16) {
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const uint32_t s = lane & (kSubHist - 1);
    FastView fv;
    if constexpr (kFast) fv = fast_view_of(c);
    const bool persp = c.persp;
    const float keep_q = c.keep_q, cull = c.cull;
    const uint32_t keep_byte = c.keep_byte;
    const float4* centers = sm.u.k.centers[buf];
    const int8_t* sexp = sm.u.k.sexp[buf];
#pragma unroll
    for (int r = 0; r < kKeysIPT; ++r) {
        const uint32_t at = (uint32_t)r * NT + tid;
        if (at >= cnt) break;   // uniform across the warp: cnt is a multiple of 32
        uint32_t key = 0;
        bool kept = false, pending = false;
        if (base + at < n) {
            const float4 p = centers[at];
            float view[4];
            bool inside;
            if constexpr (kFast) {
                fast_view(fv, p.x, p.y, p.z, view);
                inside = fast_in_frustum(fv, view);
            } else {
                view_of(c, p.x, p.y, p.z, view);
                inside = in_frustum(c, view);
            }
            if (inside) {
                const uint32_t byte = __float_as_uint(p.w) >> 24;
                const float alpha = sm.alpha[byte];
                if (!(fmul(alpha, 255.0f) <= 1.0f)) {   // else too faint to reach 1/255
                    if constexpr (kFast)
                        key = fast_depth_key(fv, view);
                    else
                        key = depth_key(c, view);
                    kept = true;
                    if (fp) {
                        bool decided = false;
                        if (persp) {
                            const float d = -view[2];
                            // keep_q 2^sexp, exactly: sexp is in [-100, 127] and
                            // keep_q >= 2^-20, so the product is a normal float
                            // (or +inf).
                            const float pow2 = __int_as_float((int(sexp[at]) + 127) << 23);
                            const float q = fmul(keep_q, pow2);
                            const float dd = fmul(d, d);
                            if (byte >= keep_byte && q <= fmul(100.0f, dd)) {
                                decided = true;   // kept
                            } else if (dd > 1e-30f && dd < 1e30f && q < 1e30f) {
                                // An upper bound of G: the approximate quotient is
                                // within a few ulps, far inside the 1.002 margin.
                                const float g = fmul(1.002f, __fdividef(q, dd));
                                const float top =
                                    fmul(fmul(fmul(alpha, 6.2832f), fadd(fmul(g, 1.00001f), 0.3f)), 1.0001f);
                                if (top < cull) {
                                    kept = false;
                                    decided = true;
                                }
                            }
                        }
                        if (!decided) {
                            kept = false;
                            pending = true;
                        }
                    }
                }
            }
        }
        k16[base + at] = (uint16_t)key;
        const uint32_t kb = __ballot_sync(0xffffffffu, kept);
        if (lane == 0) sm.u.k.maskw[at >> 5] = kb;
        if (kept) count_key(&sm.u.k.hist[0][0], key, s);
        const uint32_t pend = __ballot_sync(0xffffffffu, pending);
        if (pend) {
            uint32_t first = 0;
            if (lane == (uint32_t)(__ffs(pend) - 1)) first = atomicAdd(&sm.u.k.qn, (uint32_t)__popc(pend));
            first = __shfl_sync(0xffffffffu, first, __ffs(pend) - 1);
            if (pending) sm.u.k.queue[first + __popc(pend & lanemask_lt())] = (uint16_t)at;
        }
    }
}

// Issues the bulk copies of one keys sub-tile into staging buffer b (thread 0).
template <int NT>
__device__ __forceinline__ void stage_issue(const JobDesc& J, SortSmem<NT>& sm, uint32_t b, uint32_t base,
                                            uint32_t cnt, bool fp) {
    fence_proxy_async();
    const uint32_t bytes = cnt * 16u + (fp ? cnt : 0u);
    mbar_expect_tx(&sm.bar[b], bytes);
    bulk_copy(sm.u.k.centers[b], J.centers + base, cnt * 16u, &sm.bar[b]);
    if (fp) bulk_copy(sm.u.k.sexp[b], J.sexp + base, cnt, &sm.bar[b]);
    sm.pending |= 1u << b;
}

// Publishes a keys item's counts: the segment's low-digit counts (for the
// low pass's look-back), its group's sum, the job's totals of both digits;
// then the item's completion.
template <int NT>
__device__ void keys_publish(const JobDesc& J, uint32_t ls, SortSmem<NT>& sm) {
    JobCtl* ctl = reinterpret_cast<JobCtl*>(J.ctl);
    __syncthreads();
    const uint32_t d = threadIdx.x;
    if (d < 256) {
        uint32_t lo = 0, hi = 0;
#pragma unroll
        for (uint32_t s = 0; s < (uint32_t)kSubHist; ++s) {
            lo += sm.u.k.hist[s][sub_slot(s, d)];
            hi += sm.u.k.hist[s][256u + sub_slot(s, d)];
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
__device__ void zero_keys_hist(SortSmem<NT>& sm) {
    uint32_t* h = &sm.u.k.hist[0][0];
    for (uint32_t k = threadIdx.x; k < (uint32_t)kSubHist * 512u; k += NT) h[k] = 0;
}

// Keys of one segment of splats, in sub-tiles of TK splats staged by bulk
// copies (double-buffered).
template <int NT>
__device__ void keys_item(const JobDesc& J, int job, const SegDesc& sd, SortSmem<NT>& sm, KeysStage& ks,
                          const LaunchDesc& L, uint32_t item) {
    constexpr uint32_t TK = SortSmem<NT>::TK;
    const uint32_t tid = threadIdx.x;
    if (tid == 0) {
        if (sm.vc_job != job) {
            make_consts(J, sm.vc);
            sm.vc_job = job;
        }
        sm.u.k.qn = 0;
    }
    zero_keys_hist(sm);
    __syncthreads();
    const ViewConsts& c = sm.vc;
    const bool any = c.visible != 0;
    const bool fp = c.cull > 0.0f;
    const uint32_t a = sd.a, b = sd.b, n = J.n;
    uint16_t* const k16 = J.k16;
    if (any && a < b && tid == 0) stage_issue(J, sm, ks.buf, a, min(TK, b - a), fp);
    for (uint32_t base = a; base < b; base += TK) {
        const uint32_t cnt = min(TK, b - base);
        const uint32_t buf = ks.buf;
        if (any) {
            if (tid == 0 && base + TK < b) stage_issue(J, sm, buf ^ 1u, base + TK, min(TK, b - base - TK), fp);
            if (!stage_wait(sm, ks, buf, L, item)) sm.drain = 1;
            if (tid == 0) sm.pending &= ~(1u << buf);
            if (c.fast)
                keys_sweep<true>(c, sm, buf, base, cnt, n, fp, k16);
            else
                keys_sweep<false>(c, sm, buf, base, cnt, n, fp, k16);
        } else {
            // Wholly behind the camera: no survivors.
            for (uint32_t at = tid; at < cnt; at += NT) k16[base + at] = 0;
            for (uint32_t w = tid; w < cnt / 32; w += NT) sm.u.k.maskw[w] = 0;
        }
        __syncthreads();
        if (tid == 0 && base == a) sm.mark[1] = global_ns();
        // Sweep 2: the queued footprints, densely; a kept splat sets its bit
        // and counts its digits (its key is already out).
        const uint32_t qn = sm.u.k.qn;
        const float4* centers = sm.u.k.centers[buf];
        for (uint32_t e = tid; e < qn; e += NT) {
            const uint32_t at = sm.u.k.queue[e];
            const size_t i = base + at;
            const float4 p = centers[at];
            float view[4];
            view_of(c, p.x, p.y, p.z, view);
            const float2 a2 = __ldcs(&J.cov[3 * i]);
            const float2 b2 = __ldcs(&J.cov[3 * i + 1]);
            const float2 c2 = __ldcs(&J.cov[3 * i + 2]);
            const float sg[6] = {a2.x, a2.y, b2.x, b2.y, c2.x, c2.y};
            const float alpha = sm.alpha[__float_as_uint(p.w) >> 24];
            if (footprint_keeps(c, view, sg, alpha)) {
                atomicOr(&sm.u.k.maskw[at >> 5], 1u << (at & 31u));
                count_key(&sm.u.k.hist[0][0], depth_key(c, view), tid & (kSubHist - 1));
            }
        }
        __syncthreads();
        for (uint32_t w = tid; w < cnt / 32; w += NT) J.mask[(base >> 5) + w] = sm.u.k.maskw[w];
        // The shade pass, fused: every survivor of the sub-tile (its survivor
        // bit is final here, its centre still staged) gets its colour as seen
        // from the eye.
        if (J.sh) {
            for (uint32_t at = tid; at < cnt; at += NT) {
                if (!((sm.u.k.maskw[at >> 5] >> (at & 31u)) & 1u)) continue;
                const float4 p = centers[at];
                J.shaded[base + at] = shade_splat(J.sh, J.sh_words, J.sh_degree, base + at, p.x, p.y, p.z,
                                                  __float_as_uint(p.w), J.eye);
            }
        }
        if (tid == 0) sm.u.k.qn = 0;
        __syncthreads();   // the buffer, the survivor words and the queue are free again
        if (any) ks.buf ^= 1u;
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
__device__ void particle_keys_item(const JobDesc& J, const SegDesc& sd, SortSmem<NT>& sm) {
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
        if (live) count_key(&sm.u.k.hist[0][0], key, s);
    }
    keys_publish(J, sd.local, sm);
}

// Keys of one segment of a job whose keys are given (kind kJobKeys): every
// element survives with its key; the low pass reads the keys in place, so
// only the counts are made here.
template <int NT>
__device__ void given_keys_item(const JobDesc& J, const SegDesc& sd, SortSmem<NT>& sm) {
    const uint32_t tid = threadIdx.x, s = (tid & 31u) & (kSubHist - 1);
    zero_keys_hist(sm);
    __syncthreads();
    const uint32_t end = min(sd.b, J.n);
#pragma unroll 4
    for (uint32_t i = sd.a + tid; i < end; i += NT) count_key(&sm.u.k.hist[0][0], __ldg(&J.keys_in[i]), s);
    keys_publish(J, sd.local, sm);
}

// ---------------------------------------------------------------- digit passes

// One stable counting pass over 8 key bits for one segment (PASS 0: the low
// byte, over the segment's splats; PASS 1: the high byte, over its slice of
// the low pass's output).
template <int PASS, int NT>
__device__ void digit_item(const JobDesc& J, const SegDesc& sd, SortSmem<NT>& sm, const LaunchDesc& L,
                           uint32_t item) {
    constexpr int W = SortSmem<NT>::W;
    constexpr uint32_t IPT = kDigitIPT;
    constexpr uint32_t TD = SortSmem<NT>::TD;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    JobCtl* ctl = reinterpret_cast<JobCtl*>(J.ctl);
    uint32_t* const look = J.ctl + sizeof(JobCtl) / 4;
    uint32_t* const gsum = look + (size_t)PASS * J.ngroups * 256;
    uint32_t* const gdone = look + (size_t)2 * J.ngroups * 256;
    uint32_t* const flag = gdone + J.ngroups;
    uint32_t* const agg = J.agg + (size_t)PASS * J.nseg * 256;
    const uint32_t ls = sd.local, g = ls / kGroup;

    // The job's previous phase, every segment of it.
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
        uint32_t* h = &sm.u.p.hist[0][0];
        for (uint32_t k = tid; k < (uint32_t)kSubHist * 256u; k += NT) h[k] = 0;
        __syncthreads();
        const uint32_t s = lane & (kSubHist - 1);
        const uint16_t* kb = J.key_b;
#pragma unroll 4
        for (uint32_t e = lo + tid; e < hi; e += NT) {
            const uint32_t d = __ldcg(&kb[e]) >> 8;
            atomicAdd(&h[s * 256u + sub_slot(s, d)], 1u);
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
            // The look-back: every earlier group complete, every earlier
            // segment of this group published (all have smaller tickets).
            uint32_t spins = 0;
            sm.abort = 0;
            for (uint32_t q = 0; q < g && !sm.abort; ++q) {
                const uint32_t need = min(kGroup, J.nseg - q * kGroup);
                while (ld_acquire(&gdone[q]) < need) {
                    if (++spins > L.spin_limit || *(volatile uint32_t*)L.err) {
                        raise_error(L.err, kErrWaitPhase, item);
                        sm.abort = 1;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            for (uint32_t q = g * kGroup; q < ls && !sm.abort; ++q) {
                while (ld_acquire(&flag[q]) == 0) {
                    if (++spins > L.spin_limit || *(volatile uint32_t*)L.err) {
                        raise_error(L.err, kErrWaitPhase, item);
                        sm.abort = 1;
                        break;
                    }
                    __nanosleep(32);
                }
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
    uint32_t* const wm = sm.u.p.wmask[warp];
    uint16_t* const wc = sm.u.p.wcnt[warp];
    {
        uint32_t* z = &sm.u.p.wmask[0][0];
        for (uint32_t k = tid; k < (uint32_t)W * 256u; k += NT) z[k] = 0;
        uint32_t* zc = reinterpret_cast<uint32_t*>(&sm.u.p.wcnt[0][0]);
        for (uint32_t k = tid; k < (uint32_t)W * 128u; k += NT) zc[k] = 0;
    }
    __syncthreads();

    for (uint32_t base = lo; base < hi; base += TD) {
        // Load: warp w takes elements base + 32 (IPT w + r) + lane, rounds
        // r in order, so warps, rounds and lanes follow the element order.
        uint32_t key[IPT], idx[IPT], rk[IPT];
#pragma unroll
        for (uint32_t r = 0; r < IPT; ++r) {
            const uint32_t e = base + (warp * IPT + r) * 32u + lane;
            key[r] = 0xFFFFFFFFu;
            idx[r] = 0;
            if (e < hi) {
                if (PASS == 0) {
                    // Given keys are read only below n (the segments run to
                    // the next multiple of 256).
                    if (given ? e < n : ((__ldcg(&mask[e >> 5]) >> lane) & 1u)) key[r] = __ldcg(&kin[e]);
                    idx[r] = idx_base + e;
                } else {
                    key[r] = __ldcg(&kin[e]);
                    idx[r] = __ldcg(&idx_in[e]);
                }
            }
        }
        // Rank within the warp, round by round.
#pragma unroll
        for (uint32_t r = 0; r < IPT; ++r) {
            const bool v = key[r] != 0xFFFFFFFFu;
            rk[r] = 0;
            if (__any_sync(0xffffffffu, v)) {
                const uint32_t d = PASS == 0 ? (key[r] & 255u) : ((key[r] >> 8) & 255u);
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
                rk[r] = prior + __popc(peers & lt);
            }
        }
        __syncthreads();
        // Thread d: each warp's start within digit d, and the sub-tile's
        // count of d; then the sub-tile start of every digit.
        uint32_t tc = 0, x = 0;
        if (tid < 256) {
#pragma unroll 8
            for (int w = 0; w < W; ++w) {
                const uint32_t c = sm.u.p.wcnt[w][tid];
                sm.u.p.wcnt[w][tid] = (uint16_t)tc;
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
            if (key[r] == 0xFFFFFFFFu) continue;
            const uint32_t d = PASS == 0 ? (key[r] & 255u) : ((key[r] >> 8) & 255u);
            const uint32_t slot = sm.lstart[d] + wc[d] + rk[r];
            sm.u.p.skey[slot] = (uint16_t)key[r];
            sm.u.p.sidx[slot] = idx[r];
        }
        if (tid == 0 && base == lo) sm.mark[1] = global_ns();
        __syncthreads();
        // Write out: consecutive threads take consecutive slots, so a digit's
        // run goes out as consecutive addresses. The warp counters are cleared
        // meanwhile (nothing reads them until the next sub-tile's ranks).
        const uint32_t tt = sm.tile_total;
        {
            uint32_t* zc = reinterpret_cast<uint32_t*>(&sm.u.p.wcnt[0][0]);
            for (uint32_t k = tid; k < (uint32_t)W * 128u; k += NT) zc[k] = 0;
        }
#pragma unroll 4
        for (uint32_t i = tid; i < tt; i += NT) {
            const uint32_t k = sm.u.p.skey[i];
            const uint32_t d = PASS == 0 ? (k & 255u) : (k >> 8);
            const uint32_t gp = sm.gofs[d] + i;
            if (gp >= S) {   // only reachable if counts disagree: record, do not write
                raise_error(L.err, kErrBounds, item);
                continue;
            }
            if (PASS == 0) {
                key_b[gp] = (uint16_t)k;
                idx_b[gp] = sm.u.p.sidx[i];
            } else {
                __stcs(&order[gp], sm.u.p.sidx[i]);
                if (keys_out) __stcs(&keys_out[gp], k);
            }
        }
        __syncthreads();
    }
    if (tid == 0) sm.mark[2] = global_ns();
    if (PASS == 0) {
        __threadfence();
        __syncthreads();
        if (tid == 0) red_release_add(&ctl->low_done, 1u);
    }
}

// ---------------------------------------------------------------- the kernel

template <int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) sort_kernel(const __grid_constant__ LaunchDesc L) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    SortSmem<NT>& sm = *reinterpret_cast<SortSmem<NT>*>(smem_raw);
    const uint32_t tid = threadIdx.x;
    if (tid < 256) sm.alpha[tid] = fdiv(float(tid), 255.0f);
    if (tid == 0) {
        sm.vc_job = -1;
        sm.pending = 0;
        mbar_init(&sm.bar[0]);
        mbar_init(&sm.bar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_proxy_async();
        sm.next = atomicAdd(&L.lctl->ticket, 1u);
        sm.drain = *(volatile uint32_t*)L.err;
    }
    KeysStage ks{0u, 0u};
    const uint32_t n_items = (kPhases - L.first_phase) * L.nseg;
    uint64_t t_claim = 0, t_start = 0;
    if (L.trace && tid == 0) t_claim = global_ns();
    for (;;) {
        __syncthreads();   // the previous item's shared state is no longer read
        const uint32_t it = sm.next;
        if (it >= n_items) break;
        const uint32_t phase = L.first_phase + it / L.nseg;
        const uint32_t seg = it % L.nseg;
        SegDesc sd;
        if (L.segs) {
            sd = L.segs[seg];
        } else {
            const uint32_t npad = L.jobs[0].npad;
            sd.job = 0;
            sd.a = min(seg * L.chunk, npad);
            sd.b = min(sd.a + L.chunk, npad);
            sd.local = seg;
        }
        const JobDesc& J = L.jobs[sd.job];
        const bool work = !sm.drain;   // after an error: claim the remaining items, do no work
        if (work) {
            if (L.trace && tid == 0) {
                t_start = global_ns();
                sm.mark[0] = sm.mark[1] = sm.mark[2] = 0;
            }
            if (phase == kPhaseKeys) {
                if (J.kind == kJobParticles)
                    particle_keys_item(J, sd, sm);
                else if (J.kind == kJobKeys)
                    given_keys_item(J, sd, sm);
                else
                    keys_item(J, (int)sd.job, sd, sm, ks, L, it);
            } else if (phase == kPhaseLow) {
                digit_item<0>(J, sd, sm, L, it);
            } else {
                digit_item<1>(J, sd, sm, L, it);
            }
            __syncthreads();
        }
        if (tid == 0) {
            if (work && L.trace) {
                TraceRec r;
                r.claim = t_claim;
                r.start = t_start;
                r.end = global_ns();
                r.item = it;
                r.sm = sm_id();
                for (int q = 0; q < 3; ++q) r.mark[q] = sm.mark[q];
                L.trace[it] = r;
            }
            sm.next = atomicAdd(&L.lctl->ticket, 1u);
            sm.drain = *(volatile uint32_t*)L.err;
            if (L.trace) t_claim = global_ns();
        }
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
        atomicAdd(&L.lctl->exited, 1u);
    }
}

template <int NT>
static cudaError_t prepare_variant() {
    static bool done = false;   // the attribute is per function, set once per process
    if (done) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(sort_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)sizeof(SortSmem<NT>));
    if (e == cudaSuccess) done = true;
    return e;
}

template <int NT>
static cudaError_t launch_variant(const LaunchDesc& L, int grid, cudaStream_t stream) {
    cudaError_t e = prepare_variant<NT>();
    if (e != cudaSuccess) return e;
    sort_kernel<NT><<<grid, NT, sizeof(SortSmem<NT>), stream>>>(L);
    return cudaGetLastError();
}

// Host-side launcher: `threads` per CTA is 1024 (one CTA an SM) or 512 (two).
cudaError_t launch_sort(const LaunchDesc& L, int threads, int grid, cudaStream_t stream) {
    if (threads == 512) return launch_variant<512>(L, grid, stream);
    return launch_variant<1024>(L, grid, stream);
}

template <int NT>
static int occupancy_variant() {
    int blocks = 0;
    if (prepare_variant<NT>() != cudaSuccess) return 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, sort_kernel<NT>, NT, sizeof(SortSmem<NT>));
    return blocks;
}

// Resident CTAs per SM of the variant with `threads` threads.
int sort_occupancy(int threads) {
    static int cached[2] = {0, 0};
    const int k = threads == 512 ? 1 : 0;
    if (!cached[k]) cached[k] = k ? occupancy_variant<512>() : occupancy_variant<1024>();
    return cached[k];
}

}  // namespace wsort
