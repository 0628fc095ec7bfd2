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
// Work is a queue of items, each (job, phase, tile), claimed in order through
// one atomic ticket by a persistent grid of CTAs:
//   phase 0, keys   a tile of splats: cull, key, survivor bit, both digit
//                   histograms (warp-aggregated with __match_any_sync)
//   phase 1, low    a tile of splats: rank survivors by the low key byte
//                   (stable warp ranking), decoupled look-back across tiles
//                   for each of the 256 digits, scatter (key, index)
//   phase 2, high   a tile of the low pass's output, same by the high byte,
//                   scattering the final order and keys
// An item only ever waits for items with smaller tickets (the phase before
// it of the same job, or the tiles before it in a look-back), which were
// claimed by CTAs that are running, so the queue always drains. Every wait
// is bounded: after spin_limit polls the kernel records an error and every
// CTA drains the remaining items without work.
#include "wsort_dev.cuh"

namespace wsort {

template <int IPT>
struct SortSmem {
    static constexpr int kTile = kThreads * IPT;
    uint32_t hist[2][256];          // key-phase histograms accumulated across items
    ViewConsts vc;
    int vc_job;                     // job whose constants vc holds
    int acc_job;                    // job whose key tiles hist accumulates, or -1
    uint32_t acc_tiles;
    uint32_t item;
    uint32_t drain;
    uint32_t abort;
    uint32_t scan[kWarps];
    uint32_t total;
    uint16_t wcnt[kWarps][256];     // per-warp digit counts, then warp prefixes
    uint32_t gbase[256];            // global start of each digit
    uint32_t gofs[256];             // global position of tile slot 0 of each digit
    uint32_t lstart[256];           // tile-local start of each digit
    uint16_t stage_key[kTile];
    uint32_t stage_idx[kTile];
};

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

template <int IPT>
__device__ void flush_hist(const JobDesc* jobs, SortSmem<IPT>& sm) {
    const int tid = threadIdx.x;
    JobCtl* ctl = reinterpret_cast<JobCtl*>(jobs[sm.acc_job].ctl);
    const uint32_t a = sm.hist[0][tid], b = sm.hist[1][tid];
    if (a) atomicAdd(&ctl->hist[0][tid], a);
    if (b) atomicAdd(&ctl->hist[1][tid], b);
    sm.hist[0][tid] = 0;
    sm.hist[1][tid] = 0;
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        atomicAdd(&ctl->p1_done, sm.acc_tiles);
        sm.acc_job = -1;
        sm.acc_tiles = 0;
    }
    __syncthreads();
}

// Phase 0: keys, survivor bits and digit histograms for one tile of splats.
template <int IPT>
__device__ void keys_tile(const JobDesc& J, int job, uint32_t tile, uint32_t t1, SortSmem<IPT>& sm) {
    const int tid = threadIdx.x;
    const uint32_t lane = lane_id();
    if (tid == 0) {
        if (sm.vc_job != job) {
            make_consts(J, sm.vc);
            sm.vc_job = job;
        }
        sm.acc_job = job;
        sm.acc_tiles += 1;
    }
    // Clear this tile's share of the job's look-back words; the digit passes
    // read them only after every key tile is done.
    {
        const uint32_t words = (J.tiles2 + J.tiles3) * 256u;
        const uint32_t per = (words + J.tiles1 - 1) / J.tiles1;
        const uint32_t b = tile * per;
        const uint32_t e = min(words, b + per);
        for (uint32_t k = b + tid; k < e; k += kThreads) J.status[k] = 0;
    }
    __syncthreads();
    const ViewConsts& c = sm.vc;
    const uint32_t base = tile * t1;
    const bool any = c.visible != 0;
    for (uint32_t k = 0; k < t1; k += kThreads) {
        const uint32_t i = base + k + tid;
        uint32_t key = kCulled;
        if (any && i < J.n) {
            const float4 p = __ldcs(&J.centers[i]);
            float view[4], clip[4];
            transform(c, p.x, p.y, p.z, view, clip);
            const float alpha = frustum_alpha(view, clip, __float_as_uint(p.w));
            bool keep = alpha > 0.0f;
            if (keep && c.cull > 0.0f) {
                const float2 s0 = __ldg(&J.cov[3 * (size_t)i]);
                const float2 s1 = __ldg(&J.cov[3 * (size_t)i + 1]);
                const float2 s2 = __ldg(&J.cov[3 * (size_t)i + 2]);
                const float s[6] = {s0.x, s0.y, s1.x, s1.y, s2.x, s2.y};
                keep = footprint_keeps(c, view, s, alpha);
            }
            if (keep) key = depth_key(c, view);
        }
        const bool surv = key != kCulled;
        const uint32_t ballot = __ballot_sync(0xffffffffu, surv);
        if (i < J.n) J.k16[i] = surv ? (uint16_t)key : (uint16_t)0;
        if (lane == 0 && i < J.n) J.mask[i >> 5] = ballot;
        const uint32_t lo = key & 255u, hi = (key >> 8) & 255u;
        uint32_t peers = __match_any_sync(0xffffffffu, surv ? lo : (0x100u | lane));
        if (surv && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&sm.hist[0][lo], (uint32_t)__popc(peers));
        peers = __match_any_sync(0xffffffffu, surv ? hi : (0x100u | lane));
        if (surv && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&sm.hist[1][hi], (uint32_t)__popc(peers));
    }
}

// Phases 1 and 2: one stable counting pass over 8 key bits for one tile.
template <int PASS, int IPT>
__device__ void digit_tile(const JobDesc& J, uint32_t tile, SortSmem<IPT>& sm, uint32_t* err, uint32_t item,
                           uint32_t spin_limit) {
    constexpr uint32_t T = SortSmem<IPT>::kTile;
    const int tid = threadIdx.x;
    const uint32_t lane = lane_id(), warp = tid >> 5;
    JobCtl* ctl = reinterpret_cast<JobCtl*>(J.ctl);

    // The phase this one reads must be complete.
    if (tid == 0) {
        const uint32_t* done = PASS == 0 ? &ctl->p1_done : &ctl->p2_done;
        const uint32_t need = PASS == 0 ? J.tiles1 : J.tiles2;
        uint32_t spins = 0;
        sm.abort = 0;
        while (ld_acquire(done) < need) {
            if (++spins > spin_limit || *(volatile uint32_t*)err) {
                raise_error(err, kErrWaitPhase, item);
                sm.abort = 1;
                break;
            }
            __nanosleep(64);
        }
    }
    __syncthreads();
    if (sm.abort) return;

    // Where each digit starts in this pass's output.
    uint32_t total;
    const uint32_t h = __ldcg(&ctl->hist[PASS][tid]);
    sm.gbase[tid] = block_exclusive_scan(h, sm.scan, &total);
    if (PASS == 0 && tile == 0 && tid == 0) *J.count = total;
    const uint32_t n_in = PASS == 0 ? J.n : total;
    const uint32_t base = tile * T;

    if (base < n_in) {
        for (int k = tid; k < kWarps * 256; k += kThreads) (&sm.wcnt[0][0])[k] = 0;
        __syncthreads();

        // Stable rank within the warp: rounds of 32 consecutive elements.
        uint32_t packed[IPT];
        uint32_t idxv[IPT];
        const uint32_t wbase = base + warp * 32u * IPT;
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const uint32_t first = wbase + r * 32u;
            const uint32_t pos = first + lane;
            bool valid = pos < n_in;
            uint32_t key = 0;
            if (PASS == 0) {
                const uint32_t m = first < n_in ? __ldcg(&J.mask[first >> 5]) : 0u;
                valid = valid && ((m >> lane) & 1u);
                if (valid) key = __ldcg(&J.k16[pos]);
                idxv[r] = pos;
            } else {
                idxv[r] = 0;
                if (valid) {
                    key = __ldcg(&J.key_b[pos]);
                    idxv[r] = __ldcg(&J.idx_b[pos]);
                }
            }
            const uint32_t d = PASS == 0 ? (key & 255u) : (key >> 8);
            const uint32_t peers = __match_any_sync(0xffffffffu, valid ? d : (0x100u | lane));
            uint32_t prior = 0;
            if (valid) prior = sm.wcnt[warp][d];
            __syncwarp();
            if (valid && lane == (uint32_t)(__ffs(peers) - 1)) sm.wcnt[warp][d] = (uint16_t)(prior + __popc(peers));
            __syncwarp();
            packed[r] = valid ? (key | ((prior + __popc(peers & lanemask_lt())) << 16)) : 0xFFFFFFFFu;
        }
        __syncthreads();

        // Thread d: warp prefixes and the tile's count of digit d.
        uint32_t tc = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t cnt = sm.wcnt[w][tid];
            sm.wcnt[w][tid] = (uint16_t)tc;
            tc += cnt;
        }

        // Decoupled look-back over this pass's tiles, one chain per digit.
        uint32_t* st = J.status + (PASS == 0 ? 0u : J.tiles2 * 256u);
        uint32_t excl = 0;
        if (tile == 0) {
            st_release(&st[tid], kFlagPrefix | tc);
        } else {
            st_release(&st[tile * 256u + tid], kFlagAggregate | tc);
            int j = (int)tile - 1;
            uint32_t spins = 0;
            while (j >= 0) {
                const uint32_t s = ld_acquire(&st[(uint32_t)j * 256u + tid]);
                if (s & (kFlagAggregate | kFlagPrefix)) {
                    excl += s & kCountMask;
                    if (s & kFlagPrefix) break;
                    --j;
                    spins = 0;
                    continue;
                }
                if (++spins > spin_limit || ((spins & 1023u) == 0 && *(volatile uint32_t*)err)) {
                    raise_error(err, kErrWaitLookback, item);
                    break;
                }
            }
            st_release(&st[tile * 256u + tid], kFlagPrefix | (excl + tc));
        }

        uint32_t tile_total;
        const uint32_t ls = block_exclusive_scan(tc, sm.scan, &tile_total);
        sm.lstart[tid] = ls;
        sm.gofs[tid] = sm.gbase[tid] + excl - ls;
        __syncthreads();

        // Stage in tile order (digit, then index), then write out runs.
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            if (packed[r] == 0xFFFFFFFFu) continue;
            const uint32_t key = packed[r] & 0xFFFFu;
            const uint32_t d = PASS == 0 ? (key & 255u) : (key >> 8);
            const uint32_t slot = sm.lstart[d] + sm.wcnt[warp][d] + (packed[r] >> 16);
            sm.stage_key[slot] = (uint16_t)key;
            sm.stage_idx[slot] = idxv[r];
        }
        __syncthreads();
        for (uint32_t s = tid; s < tile_total; s += kThreads) {
            const uint32_t key = sm.stage_key[s];
            const uint32_t d = PASS == 0 ? (key & 255u) : (key >> 8);
            const uint32_t g = sm.gofs[d] + s;
            if (g >= J.n) {   // only reachable if counts disagree: record, do not write
                raise_error(err, kErrBounds, item);
                continue;
            }
            if (PASS == 0) {
                J.key_b[g] = (uint16_t)key;
                J.idx_b[g] = sm.stage_idx[s];
            } else {
                __stcs(&J.order[g], sm.stage_idx[s]);
                if (J.keys) __stcs(&J.keys[g], key);
            }
        }
    }
    __threadfence();
    __syncthreads();
    if (PASS == 0 && tid == 0) atomicAdd(&ctl->p2_done, 1u);
}

template <int IPT>
__global__ void __launch_bounds__(kThreads) sort_kernel(const JobDesc* __restrict__ jobs,
                                                        const uint2* __restrict__ items, uint32_t n_items,
                                                        LaunchCtl* __restrict__ lctl, uint32_t* __restrict__ err,
                                                        uint32_t t1, uint32_t spin_limit) {
    __shared__ SortSmem<IPT> sm;
    const int tid = threadIdx.x;
    sm.hist[0][tid] = 0;
    sm.hist[1][tid] = 0;
    if (tid == 0) {
        sm.acc_job = -1;
        sm.acc_tiles = 0;
        sm.vc_job = -1;
    }
    __syncthreads();
    for (;;) {
        __syncthreads();   // the previous item's shared state is no longer read
        if (tid == 0) {
            sm.item = atomicAdd(&lctl->ticket, 1u);
            sm.drain = *(volatile uint32_t*)err;
        }
        __syncthreads();
        const uint32_t it = sm.item;
        const uint2 item = it < n_items ? items[it] : make_uint2(0xFFFFFFFFu, 0u);
        const uint32_t phase = item.y >> 30, tile = item.y & 0x3FFFFFFFu;
        const int job = it < n_items ? (int)item.x : -1;
        if (sm.acc_job >= 0 && !(phase == kPhaseKeys && job == sm.acc_job)) flush_hist(jobs, sm);
        if (it >= n_items) break;
        if (sm.drain) continue;   // after an error: claim the remaining items, do no work
        const JobDesc& J = jobs[job];
        if (phase == kPhaseKeys) {
            keys_tile(J, job, tile, t1, sm);
            __threadfence();
        } else if (phase == kPhaseLow) {
            digit_tile<0>(J, tile, sm, err, it, spin_limit);
        } else {
            digit_tile<1>(J, tile, sm, err, it, spin_limit);
        }
    }
    if (tid == 0) atomicAdd(&lctl->exited, 1u);
}

// Host-side launcher: the kernel variant for a digit-pass tile of
// pass_tile elements.
cudaError_t launch_sort(const JobDesc* jobs, const uint2* items, uint32_t n_items, LaunchCtl* lctl,
                        uint32_t* err, uint32_t t1, uint32_t pass_tile, uint32_t spin_limit, int grid,
                        cudaStream_t stream) {
    if (pass_tile == 2048) {
        sort_kernel<8><<<grid, kThreads, 0, stream>>>(jobs, items, n_items, lctl, err, t1, spin_limit);
    } else {
        sort_kernel<16><<<grid, kThreads, 0, stream>>>(jobs, items, n_items, lctl, err, t1, spin_limit);
    }
    return cudaGetLastError();
}

int sort_occupancy(uint32_t pass_tile) {
    int blocks = 0;
    if (pass_tile == 2048)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, sort_kernel<8>, kThreads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, sort_kernel<16>, kThreads, 0);
    return blocks;
}

}  // namespace wsort
