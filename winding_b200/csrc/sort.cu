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
// Each digit pass is reduce-then-scan: per-tile digit counts (stored digit
// major), a scan over tiles for each digit (ScanLo / ScanHi) that turns them
// into each tile's starting offset per digit, then a stable warp-ranked
// scatter. The low pass's counts come out of the key phase for free. A job
// alone in its launch, of up to kRedHiTiles tiles, gets the high pass's
// counts from the low pass's scatter as well (atomic adds into the count of
// the tile each element lands in), which takes the CountHi phase off its
// critical path. There is no serial chain between
// tiles, so a pass whose tiles all start at once (they do: each pass waits
// for the whole of the one before) costs no look-back latency.
//
// Work is a queue of items, each (job, phase, tile), claimed in order through
// one atomic ticket by a persistent grid of CTAs. An item only waits for the
// phase before it of the same job, whose items all have smaller tickets and
// were claimed by CTAs that are running, so the queue always drains. Every
// wait is bounded: after spin_limit polls the kernel records an error and
// every CTA drains the remaining items without work.
#include "wsort_dev.cuh"

namespace wsort {

template <int IPT>
struct SortSmem {
    static constexpr int kTile = kThreads * IPT;
    ViewConsts vc;
    float alpha[256];               // unpack4x8unorm(..).a: byte / 255, correctly rounded
    int vc_job;                     // job whose constants vc holds
    int gb_job, gb_pass;            // job and pass whose digit starts gbase holds
    uint32_t gtotal;                // that pass's survivor count
    uint32_t gbase[256];            // global start of each digit of that pass
    uint32_t next;                  // the ticket this CTA works on next
    uint32_t drain;
    uint32_t abort;
    int ready_job;                  // (job, phase) whose dependency this CTA has seen met
    uint32_t ready_phase;
    uint64_t mark[4];               // tracing: timestamps inside an item
    uint32_t scan[kWarps];
    uint32_t hist[256];             // a tile's digit counts
    union {
        struct {                    // Keys
            float4 centers[kTile];
            int8_t sexp[kTile];
            uint32_t maskw[kTile / 32];     // survivor bits
            uint16_t queue[kTile];          // splats whose footprint must be evaluated
            uint32_t qn;
        } k;
        struct {                    // Low, CountHi, High
            uint16_t in_key[2][kTile];      // inputs (CountHi uses both key buffers)
            uint32_t in_idx[kTile];
            uint32_t mask[kTile / 32];
            uint16_t wcnt[kWarps][256];     // per-warp digit counts, then warp prefixes
            uint32_t gofs[256];             // global position of tile slot 0 of each digit
            uint32_t lstart[256];           // tile-local start of each digit
            uint16_t stage_key[kTile];
            uint32_t stage_idx[kTile];
        } p;
    } u;
};

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Copies `bytes` (a multiple of 16, both ends 16-byte aligned) with the whole
// CTA; the caller waits and synchronises.
__device__ __forceinline__ void cta_copy(void* smem_dst, const void* gsrc, uint32_t bytes) {
    char* d = static_cast<char*>(smem_dst);
    const char* g = static_cast<const char*>(gsrc);
    for (uint32_t o = threadIdx.x * 16u; o < bytes; o += kThreads * 16u) cp_async16(d + o, g + o);
}

// Exclusive scan of one value per thread across the CTA. *total receives the
// sum. Contains __syncthreads; every thread must call it.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* scan, uint32_t* total) {
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    __syncthreads();   // scan[] may still be read by a previous call
    if (lane == 31) scan[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kWarps ? scan[lane] : 0;
#pragma unroll
        for (int o = 1; o < kWarps; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        if (lane < kWarps) scan[lane] = w;
    }
    __syncthreads();
    *total = scan[kWarps - 1];
    return (warp ? scan[warp - 1] : 0) + x - v;
}

__device__ __forceinline__ void raise_error(uint32_t* err, uint32_t code, uint32_t item) {
    if (atomicCAS(err, 0u, code) == 0u) err[1] = item;
}

// Waits (thread 0, bounded) until `need` items of the phase before this one
// are done. Returns false, uniformly across the CTA, if the wait gave up.
template <int IPT>
__device__ bool wait_phase(const uint32_t* done, uint32_t need, SortSmem<IPT>& sm, uint32_t* err, uint32_t item,
                           uint32_t spin_limit) {
    if (threadIdx.x == 0) {
        uint32_t spins = 0;
        sm.abort = 0;
        while (ld_acquire(done) < need) {
            if (++spins > spin_limit || *(volatile uint32_t*)err) {
                raise_error(err, kErrWaitPhase, item);
                sm.abort = 1;
                break;
            }
            __nanosleep(32);
        }
    }
    __syncthreads();
    return sm.abort == 0;
}

// The lanes of the warp whose `on` is set and whose 8-bit digit equals this
// lane's: one ballot per digit bit (faster than __match_any_sync here).
__device__ __forceinline__ uint32_t match_digit8(uint32_t d, bool on) {
    uint32_t m = __ballot_sync(0xffffffffu, on);
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const bool bit = (d >> b) & 1u;
        const uint32_t v = __ballot_sync(0xffffffffu, bit);
        m &= bit ? v : ~v;
    }
    return m;
}

// Keys: keys, survivor bits and low-digit counts for one tile of splats.
// The tile's centres are copied to shared memory at once. A first sweep
// applies the frustum and faintness tests and the footprint shortcut; the
// splats whose footprint must still be evaluated go to a queue that all
// threads then work through densely (a warp does the footprint arithmetic
// for 32 such splats, not for every warp that holds one), reading each one's
// covariance only then.
//
// Footprint shortcut (exact): for a perspective view the host proves
// keep_q 2^sexp <= 100 d^2 implies every entry of |T| |Sigma| |T|^T is at most
// 100 (T = J W, d = -view.z, sexp the splat's covariance exponent bound), and
// then the pinned computation of the area cannot
// fall below 1.85, whatever the rounding: the 2D covariance differs from a
// positive semi-definite one by at most 7.1 u * 100 per entry, which moves
// (xx + .3)(yy + .3) - xy^2 at most 0.0025 below 0.09. So alpha * area >=
// RN(alpha * 1.85) >= cull for every alpha byte >= keep_byte, and such a
// splat is kept without its footprint (or its covariance) being computed.
// The same analysis bounds the pinned area from above for any G = the
// largest entry of |T| |Sigma| |T|^T (G <= 1.002 keep_q 2^sexp / d^2): every
// 2D entry is at most G (1 + 8.2u), so the area is at most
// 2 pi (1.00001 G + 0.3)(1 + 5u); a splat with alpha times that below cull
// is culled, again without its footprint.

// Sweep 1 of the keys tile (see keys_tile). kFast: the fast transform, with
// the view's constants in registers (FastView) for the whole tile.
template <bool kFast, int IPT>
__device__ __forceinline__ void keys_sweep(const ViewConsts& c, SortSmem<IPT>& sm, uint32_t base, uint32_t n, bool any,
                                           bool fp, uint16_t* k16) {
    constexpr uint32_t T = SortSmem<IPT>::kTile;
    const int tid = threadIdx.x;
    const uint32_t lane = lane_id();
    FastView fv;
    if constexpr (kFast) fv = fast_view_of(c);
    const bool persp = c.persp;
    const float keep_q = c.keep_q, cull = c.cull;
    const uint32_t keep_byte = c.keep_byte;
    // Sweep 1: tests, keys and the footprint shortcut. Every splat's key slot
    // is written now (the passes read only the slots whose survivor bit is
    // set), with the survivor bits and digit counts of the splats already
    // decided; the ones whose footprint must still be evaluated go to a queue.
#pragma unroll 2
    for (uint32_t k = 0; k < T; k += kThreads) {
        if (k == T / 2 && any) cp_async_wait_none();   // this thread's second-half centres
        const uint32_t at = k + tid;
        uint32_t key = 0;
        bool kept = false, pending = false;
        if (any && base + at < n) {
            const float4 p = sm.u.k.centers[at];
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
                        // Decided without the footprint when the bounds allow
                        // (see above); else queued.
                        bool decided = false;
                        if (persp) {
                            const float d = -view[2];
                            // keep_q 2^sexp, exactly: sexp is in [-100, 127] and
                            // keep_q >= 2^-20, so the product is a normal float
                            // (or +inf).
                            const float pow2 = __int_as_float((int(sm.u.k.sexp[at]) + 127) << 23);
                            const float q = fmul(keep_q, pow2);
                            const float dd = fmul(d, d);
                            if (byte >= keep_byte && q <= fmul(100.0f, dd)) {
                                decided = true;   // kept
                            } else if (dd > 1e-30f && dd < 1e30f && q < 1e30f) {
                                // An upper bound of G: the approximate quotient is
                                // within a few ulps, far inside the 1.002 margin.
                                const float g = fmul(1.002f, __fdividef(q, dd));
                                const float top = fmul(fmul(fmul(alpha, 6.2832f), fadd(fmul(g, 1.00001f), 0.3f)), 1.0001f);
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
        const uint32_t i = base + at;
        if (i < n) k16[i] = (uint16_t)key;
        const uint32_t kb = __ballot_sync(0xffffffffu, kept);
        if (lane == 0) sm.u.k.maskw[at >> 5] = kb;
        if (kept) atomicAdd(&sm.hist[key & 255u], 1u);
        const uint32_t pend = __ballot_sync(0xffffffffu, pending);
        if (pend) {
            uint32_t first = 0;
            if (lane == (uint32_t)(__ffs(pend) - 1)) first = atomicAdd(&sm.u.k.qn, (uint32_t)__popc(pend));
            first = __shfl_sync(0xffffffffu, first, __ffs(pend) - 1);
            if (pending) sm.u.k.queue[first + __popc(pend & lanemask_lt())] = (uint16_t)at;
        }
    }
}

template <int IPT>
__device__ void keys_tile(const JobDesc& J, int job, uint32_t tile, SortSmem<IPT>& sm) {
    constexpr uint32_t T = SortSmem<IPT>::kTile;
    const int tid = threadIdx.x;
    const uint32_t lane = lane_id();
    if (tid == 0) {
        if (sm.vc_job != job) {
            make_consts(J, sm.vc);
            sm.vc_job = job;
        }
        sm.u.k.qn = 0;
    }
    sm.hist[tid] = 0;
    __syncthreads();
    const ViewConsts& c = sm.vc;
    const uint32_t base = tile * T;
    const bool any = c.visible != 0;
    const bool fp = c.cull > 0.0f;
    const uint32_t n = J.n;
    uint16_t* const k16 = J.k16;
    // Every centre of the tile in flight at once, in two groups: this thread
    // copies the ones it will read (the cloud is padded to a whole number of
    // tiles), the first half with the exponents, then the second half, which
    // is still arriving while the first is swept.
    if (any) {
#pragma unroll
        for (int r = 0; r < IPT / 2; ++r)
            cp_async16(&sm.u.k.centers[r * kThreads + tid], &J.centers[base + r * kThreads + tid]);
        if (fp) cta_copy(sm.u.k.sexp, J.sexp + base, T);
        cp_async_commit();
#pragma unroll
        for (int r = IPT / 2; r < IPT; ++r)
            cp_async16(&sm.u.k.centers[r * kThreads + tid], &J.centers[base + r * kThreads + tid]);
        cp_async_commit();
        cp_async_wait_one();
    }
    __syncthreads();   // the exponents were copied by other threads
    if (tid == 0) sm.mark[0] = global_ns();
    if (c.fast)
        keys_sweep<true>(c, sm, base, n, any, fp, k16);
    else
        keys_sweep<false>(c, sm, base, n, any, fp, k16);
    __syncthreads();
    if (tid == 0) sm.mark[1] = global_ns();
    // Sweep 2: the queued footprints, densely; a kept splat sets its bit and
    // counts its digit (its key is already out).
    const uint32_t qn = sm.u.k.qn;
    for (uint32_t e = tid; e < qn; e += kThreads) {
        const uint32_t at = sm.u.k.queue[e];
        const size_t i = base + at;
        const float4 p = sm.u.k.centers[at];
        float view[4];
        view_of(c, p.x, p.y, p.z, view);
        const float2 a = __ldcs(&J.cov[3 * i]);
        const float2 b2 = __ldcs(&J.cov[3 * i + 1]);
        const float2 c2 = __ldcs(&J.cov[3 * i + 2]);
        const float sg[6] = {a.x, a.y, b2.x, b2.y, c2.x, c2.y};
        const float alpha = sm.alpha[__float_as_uint(p.w) >> 24];
        if (footprint_keeps(c, view, sg, alpha)) {
            atomicOr(&sm.u.k.maskw[at >> 5], 1u << (at & 31u));
            atomicAdd(&sm.hist[depth_key(c, view) & 255u], 1u);
        }
    }
    __syncthreads();
    if (tid == 0) sm.mark[2] = global_ns();
    for (uint32_t w = tid; w < T / 32; w += kThreads)
        if (base + w * 32 < n) J.mask[(base >> 5) + w] = sm.u.k.maskw[w];
    J.cnt_lo[(size_t)tid * J.tiles + tile] = sm.hist[tid];
    // The shade pass, fused: every survivor of the tile (its survivor bit is
    // final here, its centre still in shared memory) gets its colour as seen
    // from the eye.
    if (J.sh) {
        for (uint32_t at = tid; at < T; at += kThreads) {
            if (!((sm.u.k.maskw[at >> 5] >> (at & 31u)) & 1u)) continue;
            const float4 p = sm.u.k.centers[at];
            J.shaded[base + at] = shade_splat(J.sh, J.sh_words, J.sh_degree, base + at, p.x, p.y, p.z,
                                              __float_as_uint(p.w), J.eye);
        }
    }
}

// Keys of one tile of an alpha emitter's ring (render/particles.js:197-209):
// a slot is live unless age >= lifetime; its depth is
// max(dot(position - eye, forward), 1e-6) (the dot product summed x, y, z in
// order, each product and sum separately rounded; max returns the non-NaN
// operand); its bucket is the one of 4096 log2-depth buckets the pinned
// bucket function of the host puts it in, found here by comparing the depth
// with that function's thresholds (thr[b] = the least depth of bucket b or
// above), starting from an estimate by log2f and correcting it; the key is
// 4095 - bucket, far first.
template <int IPT>
__device__ void particle_keys_tile(const JobDesc& J, uint32_t tile, SortSmem<IPT>& sm) {
    constexpr uint32_t T = SortSmem<IPT>::kTile;
    const int tid = threadIdx.x;
    const uint32_t lane = lane_id();
    sm.hist[tid] = 0;
    __syncthreads();
    const uint32_t base = tile * T;
    const uint32_t n = J.n;
    const float ex = J.eye[0], ey = J.eye[1], ez = J.eye[2];
    const float fx = J.fwd[0], fy = J.fwd[1], fz = J.fwd[2];
    // Every particle of the tile in flight at once: position and age (a
    // record's first 16 bytes) into shared memory, lifetimes into registers;
    // each thread reads back only its own.
    const float4* pool = J.pool + 2 * ((size_t)J.idx_base + base);
    float life[IPT];
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
        const uint32_t at = r * kThreads + tid;
        if (base + at < n) {
            cp_async16(&sm.u.k.centers[at], &pool[2 * (size_t)at]);
            life[r] = __ldcs(&pool[2 * (size_t)at + 1].w);
        }
    }
    cp_async_wait_all();
    uint16_t* const k16 = J.k16;
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
        const uint32_t at = r * kThreads + tid;
        const uint32_t i = base + at;
        uint32_t key = 0;
        bool live = false;
        if (i < n) {
            const float4 a = sm.u.k.centers[at];
            live = !(a.w >= life[r]);
            if (live) {
                const float dot = fadd(fadd(fmul(fsub(a.x, ex), fx), fmul(fsub(a.y, ey), fy)), fmul(fsub(a.z, ez), fz));
                const float d = fmaxf(dot, 1e-6f);
                int b = (int)fclamp(fmul(fadd(log2f(d), 10.0f), 136.5f), 0.0f, 4095.0f);
                // The estimate is within a bucket or two; the thresholds decide.
                while (b < (int)kParticleBuckets - 1 && d >= __ldg(&J.thr[b + 1])) ++b;
                while (b > 0 && d < __ldg(&J.thr[b])) --b;
                key = kParticleBuckets - 1u - (uint32_t)b;
            }
            k16[i] = (uint16_t)key;
        }
        const uint32_t kb = __ballot_sync(0xffffffffu, live);
        if (lane == 0) sm.u.k.maskw[at >> 5] = kb;
        if (live) atomicAdd(&sm.hist[key & 255u], 1u);
    }
    __syncthreads();
    for (uint32_t w = tid; w < T / 32; w += kThreads)
        if (base + w * 32 < n) J.mask[(base >> 5) + w] = sm.u.k.maskw[w];
    J.cnt_lo[(size_t)tid * J.tiles + tile] = sm.hist[tid];
}

// Keys of one tile of a job whose keys are given (kind kJobKeys): every
// element survives, its key as given.
template <int IPT>
__device__ void given_keys_tile(const JobDesc& J, uint32_t tile, SortSmem<IPT>& sm) {
    constexpr uint32_t T = SortSmem<IPT>::kTile;
    const int tid = threadIdx.x;
    const uint32_t lane = lane_id();
    sm.hist[tid] = 0;
    __syncthreads();
    const uint32_t base = tile * T;
    const uint32_t n = J.n;
#pragma unroll 4
    for (uint32_t k = 0; k < T; k += kThreads) {
        const uint32_t i = base + k + tid;
        const bool on = i < n;
        const uint32_t key = on ? J.keys_in[i] : 0u;
        if (on) J.k16[i] = (uint16_t)key;
        const uint32_t b = __ballot_sync(0xffffffffu, on);
        if (lane == 0 && on) J.mask[i >> 5] = b;
        if (on) atomicAdd(&sm.hist[key & 255u], 1u);
    }
    __syncthreads();
    J.cnt_lo[(size_t)tid * J.tiles + tile] = sm.hist[tid];
}

// The start of each digit in a pass's output (an exclusive scan of the
// pass's digit totals), cached per (job, pass) for the CTA's next items.
template <int IPT>
__device__ void digit_starts(const JobDesc& J, int job, int pass, SortSmem<IPT>& sm) {
    if (sm.gb_job == job && sm.gb_pass == pass) return;
    JobCtl* ctl = reinterpret_cast<JobCtl*>(J.ctl);
    uint32_t total;
    const uint32_t g = block_exclusive_scan(__ldcg(&ctl->tot[pass][threadIdx.x]), sm.scan, &total);
    sm.gbase[threadIdx.x] = g;
    __syncthreads();
    if (threadIdx.x == 0) {
        sm.gtotal = total;
        sm.gb_job = job;
        sm.gb_pass = pass;
    }
    __syncthreads();
}

// CountHi: high-digit counts of tiles 2g and 2g + 1 of the low pass's
// output. Both tiles' keys are copied at once, into the two key buffers of
// the digit passes.
template <int IPT>
__device__ void count_hi_item(const JobDesc& J, int job, uint32_t g, SortSmem<IPT>& sm) {
    constexpr uint32_t T = SortSmem<IPT>::kTile;
    const int tid = threadIdx.x;
    // The survivor count, which the low pass's first tile stored (the whole
    // low pass is done before this phase starts).
    const uint32_t s_total = __ldcg(J.count);
    uint16_t* area[kCountSpan] = {sm.u.p.in_key[0], sm.u.p.in_key[1]};
#pragma unroll
    for (uint32_t q = 0; q < kCountSpan; ++q) {
        const uint32_t tile = g * kCountSpan + q;
        if (tile < J.tiles && tile * T < s_total) cta_copy(area[q], J.key_b + tile * T, T * 2);
    }
    cp_async_wait_all();
    __syncthreads();
    if (tid == 0) sm.mark[0] = global_ns();
    // Counters: four per warp (one per 8 lanes, so at most 8 lanes of a warp
    // meet on one counter however few digits the tile holds), two 16-bit
    // digit counts to a word (a counter sees at most 8 x IPT keys), bumped
    // with shared-memory atomics; counter w's word for digit pair p is at
    // w * 128 + (p ^ w), so one digit's counters are in different banks.
    // They live past the two key buffers.
    constexpr int kSubs = kWarps * 4;
    static_assert(sizeof(sm.u) >= 4 * (size_t)T + kSubs * 128 * 4, "counters fit the phase union");
    uint32_t* wc = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(&sm.u) + 4 * (size_t)T);
    const uint32_t warp = tid >> 5, lane = tid & 31;
    const uint32_t sub = warp * 4 + (lane >> 3);
#pragma unroll 1
    for (uint32_t q = 0; q < kCountSpan; ++q) {
        const uint32_t tile = g * kCountSpan + q;
        if (tile >= J.tiles) break;
        for (int k = tid; k < kSubs * 128; k += kThreads) wc[k] = 0;
        __syncthreads();
        const uint32_t base = tile * T;
        if (base < s_total) {
#pragma unroll
            for (int r = 0; r < IPT; ++r) {
                const uint32_t at = warp * 32u * IPT + r * 32u + lane;
                if (base + at < s_total) {
                    const uint32_t d = (q ? sm.u.p.in_key[1][at] : sm.u.p.in_key[0][at]) >> 8;
                    atomicAdd(&wc[sub * 128 + ((d >> 1) ^ sub)], 1u << ((d & 1u) * 16));
                }
            }
        }
        __syncthreads();
        uint32_t total = 0;
#pragma unroll 8
        for (int w = 0; w < kSubs; ++w) total += (wc[w * 128 + ((tid >> 1) ^ w)] >> ((tid & 1) * 16)) & 0xFFFFu;
        J.cnt_hi[(size_t)tid * J.tiles + tile] = total;
        __syncthreads();   // the counters are cleared for the next tile
        if (tid == 0) sm.mark[1 + q] = global_ns();
    }
}

// ScanLo / ScanHi: for digit d, the exclusive prefix over tiles of its
// per-tile counts (a contiguous row of the digit-major count matrix), in
// place, and its total. Chunks of 4096 tiles go through shared memory:
// loaded and stored coalesced (word e of the chunk at e + e / 32, so a
// thread's run of 16 is read without bank conflicts), each thread scanning
// 16 consecutive words between.
template <int IPT>
__device__ void scan_digit(uint32_t* cnt, uint32_t tiles, uint32_t d, uint32_t* tot, SortSmem<IPT>& sm) {
    constexpr int V = 16;
    constexpr uint32_t kChunk = kThreads * V;
    static_assert(sizeof(sm.u) >= (kChunk + kChunk / 32) * 4, "chunk fits the phase union");
    uint32_t* buf = reinterpret_cast<uint32_t*>(&sm.u);
    const int tid = threadIdx.x;
    uint32_t* row = cnt + (size_t)d * tiles;
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < tiles; c0 += kChunk) {
        __syncthreads();   // the previous chunk's stores have read buf
#pragma unroll
        for (int q = 0; q < V; ++q) {
            const uint32_t e = q * kThreads + tid;
            buf[e + e / 32] = c0 + e < tiles ? __ldcg(&row[c0 + e]) : 0u;
        }
        __syncthreads();
        uint32_t local = 0;
#pragma unroll
        for (int q = 0; q < V; ++q) {
            const uint32_t e = tid * V + q;
            local += buf[e + e / 32];
        }
        uint32_t chunk_total;
        uint32_t run = carry + block_exclusive_scan(local, sm.scan, &chunk_total);
#pragma unroll
        for (int q = 0; q < V; ++q) {   // only this thread touches its run of 16
            const uint32_t e = tid * V + q;
            const uint32_t x = buf[e + e / 32];
            buf[e + e / 32] = run;
            run += x;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < V; ++q) {
            const uint32_t e = q * kThreads + tid;
            if (c0 + e < tiles) row[c0 + e] = buf[e + e / 32];
        }
        carry += chunk_total;
    }
    if (tid == 0) tot[d] = carry;
}

// ScanLo / ScanHi of a job of at most kSmallScanTiles tiles: item g scans the
// rows of digits 32g .. 32g + 31, which are one contiguous block of the
// digit-major count matrix (32 x tiles words). The block is read into shared
// memory with coalesced loads, each of warp 0's lanes scans one row there,
// and the block is written back the same way.
template <int IPT>
__device__ void scan_rows(uint32_t* cnt, uint32_t tiles, uint32_t* tot, uint32_t g, SortSmem<IPT>& sm) {
    constexpr uint32_t R = 256 / kSmallScanItems;   // rows an item scans
    static_assert(sizeof(sm.u) >= R * (kSmallScanTiles + 1) * 4, "the block fits the phase union");
    uint32_t* buf = reinterpret_cast<uint32_t*>(&sm.u);
    const uint32_t tid = threadIdx.x;
    const uint32_t P = tiles | 1u;                  // odd row stride: the row scans meet no bank conflict
    uint32_t* block = cnt + (size_t)g * R * tiles;
    const uint32_t words = R * tiles;
#pragma unroll 4
    for (uint32_t e = tid; e < words; e += kThreads) buf[(e / tiles) * P + e % tiles] = __ldcg(&block[e]);
    __syncthreads();
    if (tid < R) {
        uint32_t run = 0;
        uint32_t* row = buf + tid * P;
#pragma unroll 4
        for (uint32_t c = 0; c < tiles; ++c) {
            const uint32_t x = row[c];
            row[c] = run;
            run += x;
        }
        tot[g * R + tid] = run;
    }
    __syncthreads();
#pragma unroll 4
    for (uint32_t e = tid; e < words; e += kThreads) block[e] = buf[(e / tiles) * P + e % tiles];
}

// Low / High: one stable counting pass over 8 key bits for one tile. The
// tile's input is copied to shared memory first (cp.async, all at once);
// each warp ranks its 32 x IPT consecutive elements in rounds of 32, stably.
template <int PASS, int IPT>
__device__ void digit_tile(const JobDesc& J, int job, uint32_t tile, SortSmem<IPT>& sm, uint32_t* err,
                           uint32_t item) {
    constexpr uint32_t T = SortSmem<IPT>::kTile;
    const int tid = threadIdx.x;
    const uint32_t lane = lane_id(), warp = tid >> 5;

    // Where each digit starts in this pass's output.
    digit_starts(J, job, PASS, sm);
    const uint32_t total = sm.gtotal;
    const uint32_t gbase = sm.gbase[tid];
    if (PASS == 0 && tile == 0 && tid == 0) *J.count = total;
    const uint32_t n_in = PASS == 0 ? J.n : total;
    const uint32_t base = tile * T;
    if (base >= n_in) {   // an empty job's one tile: nothing to move, but counted
        if (PASS == 0 && J.red_hi && tid == 0)
            red_release_add(&reinterpret_cast<JobCtl*>(J.ctl)->done[kPhaseCountHi], 1u);
        return;
    }
    const uint32_t* cnt = PASS == 0 ? J.cnt_lo : J.cnt_hi;
    const uint32_t excl = __ldcg(&cnt[(size_t)tid * J.tiles + tile]);
    const uint32_t b = 0;
    if (PASS == 0) {
        cta_copy(sm.u.p.in_key[b], J.k16 + base, T * 2);
        cta_copy(sm.u.p.mask, J.mask + base / 32, T / 8);
    } else {
        cta_copy(sm.u.p.in_key[b], J.key_b + base, T * 2);
        cta_copy(sm.u.p.in_idx, J.idx_b + base, T * 4);
    }
    for (int k = tid; k < kWarps * 256; k += kThreads) (&sm.u.p.wcnt[0][0])[k] = 0;
    cp_async_wait_all();
    __syncthreads();
    if (tid == 0) sm.mark[0] = global_ns();

    // Stable rank within the warp.
    uint32_t packed[IPT];
    const uint32_t wlocal = warp * 32u * IPT;
    const uint32_t lt = lanemask_lt();
    // The rounds' matches are independent: all of them first, then the
    // counter updates, which must run in round order.
    uint32_t peersv[IPT];
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
        const uint32_t at = wlocal + r * 32u + lane;
        bool valid = base + at < n_in;
        if (PASS == 0) valid = valid && ((sm.u.p.mask[at >> 5] >> lane) & 1u);
        const uint32_t key = sm.u.p.in_key[b][at];
        const uint32_t d = PASS == 0 ? (key & 255u) : (key >> 8);
        peersv[r] = match_digit8(d, valid);   // every lane takes part in the ballots
        packed[r] = valid ? key : 0xFFFFFFFFu;
    }
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
        const bool valid = packed[r] != 0xFFFFFFFFu;
        const uint32_t key = packed[r] & 0xFFFFu;
        const uint32_t d = PASS == 0 ? (key & 255u) : (key >> 8);
        const uint32_t peers = peersv[r];
        uint32_t prior = 0;
        if (valid) prior = sm.u.p.wcnt[warp][d];
        __syncwarp();
        if (valid && lane == (uint32_t)(__ffs(peers) - 1)) sm.u.p.wcnt[warp][d] = (uint16_t)(prior + __popc(peers));
        __syncwarp();
        packed[r] = valid ? (key | ((prior + __popc(peers & lt)) << 16)) : 0xFFFFFFFFu;
    }
    __syncthreads();

    // Thread d: warp prefixes and the tile's count of digit d.
    uint32_t tc = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const uint32_t cnt_w = sm.u.p.wcnt[w][tid];
        sm.u.p.wcnt[w][tid] = (uint16_t)tc;
        tc += cnt_w;
    }
    if (tid == 0) sm.mark[1] = global_ns();
    uint32_t tile_total;
    const uint32_t ls = block_exclusive_scan(tc, sm.scan, &tile_total);
    sm.u.p.lstart[tid] = ls;
    sm.u.p.gofs[tid] = gbase + excl - ls;
    __syncthreads();

    // Stage in tile order (digit, then index), then write out runs.
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
        if (packed[r] == 0xFFFFFFFFu) continue;
        const uint32_t key = packed[r] & 0xFFFFu;
        const uint32_t d = PASS == 0 ? (key & 255u) : (key >> 8);
        const uint32_t slot = sm.u.p.lstart[d] + sm.u.p.wcnt[warp][d] + (packed[r] >> 16);
        const uint32_t at = wlocal + r * 32u + lane;
        sm.u.p.stage_key[slot] = (uint16_t)key;
        sm.u.p.stage_idx[slot] = PASS == 0 ? J.idx_base + base + at : sm.u.p.in_idx[at];
    }
    __syncthreads();
    if (tid == 0) sm.mark[2] = global_ns();
    // Write-out in chunks of four slots per thread: the chunk's staged
    // entries are read first, so their shared-memory loads overlap. The job's
    // output pointers and size are read once, into registers. A low pass
    // that counts the high digits adds each element to the count of its
    // digit in the high pass's tile it lands in (tile g / T of its output);
    // the keys phase zeroed those counts.
    constexpr int kChunk = 4;
    constexpr uint32_t kTileShift = __builtin_ctz(T);
    static_assert((1u << kTileShift) == T, "tiles are powers of two");
    const uint32_t n_out = J.n;
    uint16_t* const key_b = J.key_b;
    uint32_t* const idx_b = J.idx_b;
    uint32_t* const cnt_hi = J.cnt_hi;
    const size_t hi_row = J.tiles;
    const bool red_hi = PASS == 0 && J.red_hi;
    uint32_t* const order = J.order;
    uint32_t* const keys_out = J.keys;
#pragma unroll 1
    for (int r0 = 0; r0 < IPT && (uint32_t)r0 * kThreads < tile_total; r0 += kChunk) {
        uint32_t kk[kChunk], ix[kChunk];
#pragma unroll
        for (int q = 0; q < kChunk; ++q) {
            const uint32_t s = (uint32_t)(r0 + q) * kThreads + tid;
            const bool on = s < tile_total;
            kk[q] = on ? (uint32_t)sm.u.p.stage_key[s] : 0xFFFFFFFFu;
            ix[q] = on ? sm.u.p.stage_idx[s] : 0u;
        }
#pragma unroll
        for (int q = 0; q < kChunk; ++q) {
            if (kk[q] == 0xFFFFFFFFu) continue;
            const uint32_t s = (uint32_t)(r0 + q) * kThreads + tid;
            const uint32_t key = kk[q];
            const uint32_t d = PASS == 0 ? (key & 255u) : (key >> 8);
            const uint32_t g = sm.u.p.gofs[d] + s;
            if (g >= n_out) {   // only reachable if counts disagree: record, do not write
                raise_error(err, kErrBounds, item);
                continue;
            }
            if (PASS == 0) {
                key_b[g] = (uint16_t)key;
                idx_b[g] = ix[q];
            } else {
                __stcs(&order[g], ix[q]);
                if (keys_out) __stcs(&keys_out[g], key);
            }
        }
        if (red_hi) {
            // Lanes hold consecutive staged slots, so neighbours often land
            // in the same tile with the same high digit: the first lane of
            // each such run adds the run's length. (The job's choice is
            // uniform, so every lane of the warp is here.)
#pragma unroll
            for (int q = 0; q < kChunk; ++q) {
                const uint32_t s = (uint32_t)(r0 + q) * kThreads + tid;
                const uint32_t key = kk[q];
                const uint32_t g = key != 0xFFFFFFFFu ? sm.u.p.gofs[key & 255u] + s : n_out;
                const bool put = g < n_out;
                const uint32_t cell = put ? ((key >> 8) << 21) | (g >> kTileShift) : 0xFFFFFFFFu;
                const uint32_t before = __shfl_up_sync(0xffffffffu, cell, 1);
                const bool head = lane == 0 || cell != before;
                const uint32_t heads = __ballot_sync(0xffffffffu, head);
                if (put && head) {
                    const uint32_t later = heads & ~((2u << lane) - 1u);
                    const uint32_t end = later ? (uint32_t)__ffs(later) - 1u : 32u;
                    atomicAdd(&cnt_hi[(key >> 8) * hi_row + (g >> kTileShift)], end - lane);
                }
            }
        }
    }
    if (red_hi) {
        // Published as a CountHi item (the job has none), for ScanHi; the
        // item's own publication as a low-pass item follows as usual.
        __syncthreads();
        if (tid == 0) red_release_add(&reinterpret_cast<JobCtl*>(J.ctl)->done[kPhaseCountHi], 1u);
    }
}

__device__ __forceinline__ uint32_t sm_id() {
    uint32_t s;
    asm("mov.u32 %0, %%smid;" : "=r"(s));
    return s;
}

template <int IPT, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) sort_kernel(const JobDesc* __restrict__ jobs,
                                                        const uint2* __restrict__ items, uint32_t n_items,
                                                        LaunchCtl* __restrict__ lctl, uint32_t* __restrict__ err,
                                                        uint32_t spin_limit, TraceRec* __restrict__ trace) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<IPT>& sm = *reinterpret_cast<SortSmem<IPT>*>(smem_raw);
    const int tid = threadIdx.x;
    sm.alpha[tid] = fdiv(float(tid), 255.0f);
    if (tid == 0) {
        sm.vc_job = -1;
        sm.gb_job = -1;
        sm.gb_pass = -1;
    }
    if (tid == 0) {
        sm.next = atomicAdd(&lctl->ticket, 1u);
        sm.drain = *(volatile uint32_t*)err;
        sm.ready_job = -1;
    }
    uint64_t t_claim = 0, t_start = 0;
    if (trace && tid == 0) t_claim = global_ns();
    for (;;) {
        __syncthreads();   // the previous item's shared state is no longer read
        const uint32_t it = sm.next;
        if (it >= n_items) break;
        const uint2 item = items[it];
        const uint32_t phase = item.y >> kPhaseShift, tile = item.y & kTileMask;
        const int job = (int)item.x;
        const JobDesc& J = jobs[job];
        JobCtl* ctl = reinterpret_cast<JobCtl*>(J.ctl);
        bool work = !sm.drain;   // after an error: claim the remaining items, do no work
        if (work && phase != kPhaseKeys && !(sm.ready_job == job && sm.ready_phase == phase)) {
            // Items the phase before this one has: tiles, one per digit, or
            // for ScanHi the items that count the high digits (CountHi's, or
            // the low pass's when it counts them and publishes as CountHi).
            const uint32_t need = (phase == kPhaseLow || phase == kPhaseHigh) ? J.scan_items
                                  : phase == kPhaseScanHi ? J.hi_items
                                                          : J.tiles;
            work = wait_phase(&ctl->done[phase - 1], need, sm, err, it, spin_limit);
            if (work && tid == 0) {
                sm.ready_job = job;
                sm.ready_phase = phase;
            }
        }
        if (work) {
            if (trace && tid == 0) {
                t_start = global_ns();
                sm.mark[0] = sm.mark[1] = sm.mark[2] = 0;
            }
            switch (phase) {
                case kPhaseKeys:
                    if (J.kind == kJobParticles)
                        particle_keys_tile(J, tile, sm);
                    else if (J.kind == kJobKeys)
                        given_keys_tile(J, tile, sm);
                    else
                        keys_tile(J, job, tile, sm);
                    // This tile's column of the high-digit counts, which a
                    // red_hi job's low pass adds to.
                    if (J.red_hi) J.cnt_hi[(size_t)tid * J.tiles + tile] = 0;
                    break;
                case kPhaseScanLo:
                    if (J.scan_items == kSmallScanItems)
                        scan_rows(J.cnt_lo, J.tiles, ctl->tot[0], tile, sm);
                    else
                        scan_digit(J.cnt_lo, J.tiles, tile, ctl->tot[0], sm);
                    break;
                case kPhaseLow: digit_tile<0>(J, job, tile, sm, err, it); break;
                case kPhaseCountHi: count_hi_item(J, job, tile, sm); break;
                case kPhaseScanHi:
                    if (J.scan_items == kSmallScanItems)
                        scan_rows(J.cnt_hi, J.tiles, ctl->tot[1], tile, sm);
                    else
                        scan_digit(J.cnt_hi, J.tiles, tile, ctl->tot[1], sm);
                    break;
                default: digit_tile<1>(J, job, tile, sm, err, it); break;
            }
            __syncthreads();
        }
        if (tid == 0) {
            if (work) {
                // Published at once (after the barrier above, so every
                // thread's writes of the item are ordered before it).
                red_release_add(&ctl->done[phase], 1u);
                if (trace) {
                    TraceRec r;
                    r.claim = t_claim;
                    r.start = t_start;
                    r.end = global_ns();
                    r.item = it;
                    r.sm = sm_id();
                    for (int q = 0; q < 3; ++q) r.mark[q] = sm.mark[q];
                    trace[it] = r;
                }
            }
            sm.next = atomicAdd(&lctl->ticket, 1u);
            sm.drain = *(volatile uint32_t*)err;
            if (trace) t_claim = global_ns();
        }
    }
    cp_async_wait_all();   // no copy into this CTA's shared memory outlives it
    if (tid == 0) atomicAdd(&lctl->exited, 1u);
}

// The kernel variants: a tile of 256 * IPT elements, at least MINB resident
// CTAs per SM (which caps the registers a thread may use).
template <int IPT, int MINB>
static cudaError_t prepare_variant() {
    static bool done = false;   // the attribute is per function, set once per process
    if (done) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(sort_kernel<IPT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)sizeof(SortSmem<IPT>));
    if (e == cudaSuccess) done = true;
    return e;
}

template <int IPT, int MINB>
static cudaError_t launch_variant(const JobDesc* jobs, const uint2* items, uint32_t n_items, LaunchCtl* lctl,
                                  uint32_t* err, uint32_t spin_limit, int grid, cudaStream_t stream,
                                  TraceRec* trace) {
    cudaError_t e = prepare_variant<IPT, MINB>();
    if (e != cudaSuccess) return e;
    sort_kernel<IPT, MINB><<<grid, kThreads, sizeof(SortSmem<IPT>), stream>>>(jobs, items, n_items, lctl, err,
                                                                               spin_limit, trace);
    return cudaGetLastError();
}

template <int IPT>
static cudaError_t launch_ipt(int minb, const JobDesc* jobs, const uint2* items, uint32_t n_items, LaunchCtl* lctl,
                              uint32_t* err, uint32_t spin_limit, int grid, cudaStream_t stream, TraceRec* trace) {
    if constexpr (IPT == 4)
        if (minb == 6) return launch_variant<IPT, 6>(jobs, items, n_items, lctl, err, spin_limit, grid, stream, trace);
    switch (minb) {
        case 2: return launch_variant<IPT, 2>(jobs, items, n_items, lctl, err, spin_limit, grid, stream, trace);
        case 4: return launch_variant<IPT, 4>(jobs, items, n_items, lctl, err, spin_limit, grid, stream, trace);
        default: return launch_variant<IPT, 3>(jobs, items, n_items, lctl, err, spin_limit, grid, stream, trace);
    }
}

// Host-side launcher: the variant for a tile of `tile` elements and `minb`
// resident CTAs per SM (2, 3 or 4; also 6 for tiles of 1024, whose shared
// memory allows six).
cudaError_t launch_sort(const JobDesc* jobs, const uint2* items, uint32_t n_items, LaunchCtl* lctl,
                        uint32_t* err, uint32_t tile, int minb, uint32_t spin_limit, int grid, cudaStream_t stream,
                        TraceRec* trace) {
    switch (tile) {
        case 1024: return launch_ipt<4>(minb, jobs, items, n_items, lctl, err, spin_limit, grid, stream, trace);
        case 2048: return launch_ipt<8>(minb, jobs, items, n_items, lctl, err, spin_limit, grid, stream, trace);
        default: return launch_ipt<16>(minb, jobs, items, n_items, lctl, err, spin_limit, grid, stream, trace);
    }
}

template <int IPT, int MINB>
static int occupancy_variant() {
    int blocks = 0;
    if (prepare_variant<IPT, MINB>() != cudaSuccess) return 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, sort_kernel<IPT, MINB>, kThreads, sizeof(SortSmem<IPT>));
    return blocks;
}

template <int IPT>
static int occupancy_ipt(int minb) {
    if constexpr (IPT == 4)
        if (minb == 6) return occupancy_variant<IPT, 6>();
    switch (minb) {
        case 2: return occupancy_variant<IPT, 2>();
        case 4: return occupancy_variant<IPT, 4>();
        default: return occupancy_variant<IPT, 3>();
    }
}

int sort_occupancy(uint32_t tile, int minb) {
    switch (tile) {
        case 1024: return occupancy_ipt<4>(minb);
        case 2048: return occupancy_ipt<8>(minb);
        default: return occupancy_ipt<16>(minb);
    }
}

}  // namespace wsort
