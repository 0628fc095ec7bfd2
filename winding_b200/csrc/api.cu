// The C ABI of libwsort.so (include/wsort.h): contexts, resident clouds,
// single and batched sorts, and graph-captured plans.
#include "wsort.h"
#include "wsort_dev.cuh"
#include "wsort_host.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <functional>
#include <string>
#include <vector>

namespace wsort {
cudaError_t launch_decode(const void* records, uint32_t n, float4* centers, float2* cov, int8_t* sexp,
                          uint32_t* bounds, uint32_t* bad, int sms, cudaStream_t stream, uint32_t first);
cudaError_t stream_splat_records(ws_ctx* ctx, const uint8_t* src, uint32_t n, float4* centers, float2* cov,
                                 int8_t* sexp, uint32_t* bounds, uint32_t* bad);

int set_error(ws_ctx* ctx, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    return code;
}

int cuda_error(ws_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation)
        return set_error(ctx, WS_ERR_NOMEM, "%s: out of device memory (%s)", what, cudaGetErrorString(e));
    return set_error(ctx, WS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Device allocations that are to fail as if the device were out of memory
// (ws_inject_alloc_failures): a test hook for the allocation-failure paths.
static std::atomic<int> g_alloc_failures{0};

extern "C" int ws_inject_alloc_failures(int count) {
    if (count < 0) return WS_ERR_ARG;
    g_alloc_failures.store(count);
    return WS_OK;
}

cudaError_t DevBuf::ensure(size_t n) {
    if (n <= bytes) return cudaSuccess;
    release();
    int pending = g_alloc_failures.load();
    while (pending > 0 && !g_alloc_failures.compare_exchange_weak(pending, pending - 1)) {
    }
    if (pending > 0) return cudaErrorMemoryAllocation;
    const cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        return e;
    }
    bytes = n;
    return cudaSuccess;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}
cudaError_t HostBuf::ensure(size_t n) {
    if (n <= bytes) return cudaSuccess;
    release();
    const cudaError_t e = cudaHostAlloc(&p, n, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        return e;
    }
    bytes = n;
    return cudaSuccess;
}
void HostBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

uint32_t pad_splats(uint32_t n) { return (uint32_t)align_up(n ? n : 1, kPadSplats); }

static uint32_t npad_of(uint32_t n) { return (uint32_t)align_up(n, kSegAlign); }

// Threads per CTA of the kernel variant p selects: 1024 (one CTA an SM) or
// 512 (two).
static int threads_of(const ws_params& p) { return p.ctas_per_sm == 2 ? 512 : 1024; }

// The segments: the jobs laid end to end (each padded to kSegAlign) are cut
// into chunks of `chunk` splats, about segs_per_cta per resident CTA and no
// smaller than p.tile; a segment is one job's part of one chunk. Then the
// scratch: the launch counters and every job's control region (zeroed
// before a launch), then per job its key, survivor-bit, intermediate and
// count arrays.
void shape_launch(const uint32_t* ns, int njobs, const ws_params& p, int sms, LaunchShape& S) {
    S.threads = threads_of(p);
    const int want = S.threads == 512 ? 2 : 1;
    const int occ = sort_occupancy(S.threads);
    S.grid = sms * std::max(1, std::min(want, occ));
    uint64_t total = 0;
    for (int j = 0; j < njobs; ++j) total += npad_of(ns[j]);
    const uint64_t target = (uint64_t)S.grid * std::max(1u, p.segs_per_cta);
    uint64_t chunk = (total + target - 1) / std::max<uint64_t>(target, 1);
    chunk = std::max<uint64_t>(chunk, p.tile ? p.tile : 2048);
    chunk = align_up(chunk, kSegAlign);
    S.chunk = (uint32_t)std::min<uint64_t>(chunk, 0x80000000ull);
    S.regular = njobs == 1;
    S.segs.clear();
    S.nseg.assign(njobs, 0);
    S.seg0.assign(njobs, 0);
    // Each job is cut into equal segments of at most a chunk (multiples of
    // kSegAlign), and the jobs are queued largest first (ties in their given
    // order): a phase's last items are then the small jobs' short segments,
    // so the grid's last wave ends evenly. A job's segments stay in order,
    // which is all the look-back needs.
    std::vector<int> by_size(njobs);
    for (int j = 0; j < njobs; ++j) by_size[j] = j;
    std::stable_sort(by_size.begin(), by_size.end(), [&](int a, int b) { return ns[a] > ns[b]; });
    for (const int j : by_size) {
        const uint32_t np = npad_of(ns[j]);
        const uint64_t k = std::max<uint64_t>(1, (np + (uint64_t)S.chunk - 1) / S.chunk);
        const uint32_t each = (uint32_t)align_up((np + k - 1) / k, kSegAlign);
        S.seg0[j] = (uint32_t)S.segs.size();
        uint32_t at = 0, local = 0;
        do {
            const uint32_t end = std::min(np, at + each);
            S.segs.push_back(SegDesc{(uint32_t)j, at, end, local++});
            at = end;
        } while (at < np);
        S.nseg[j] = local;
    }
    if (S.regular) {
        // The kernel's own cut of a lone job: consecutive chunks from 0.
        const uint32_t np = npad_of(ns[0]);
        const uint32_t k = np ? (np + S.chunk - 1) / S.chunk : 1;
        S.segs.clear();
        for (uint32_t q = 0; q < k; ++q)
            S.segs.push_back(SegDesc{0u, std::min(q * S.chunk, np), std::min(q * S.chunk + S.chunk, np), q});
        S.nseg[0] = k;
    }
    size_t off = 256;   // LaunchCtl
    S.ctl_off.resize(njobs);
    for (int j = 0; j < njobs; ++j) {
        S.ctl_off[j] = off;
        off += job_ctl_bytes(S.nseg[j]);
    }
    S.ctl_bytes = off;
    S.arr_off.resize(njobs);
    for (int j = 0; j < njobs; ++j) {
        S.arr_off[j] = off;
        const size_t np = std::max<size_t>(npad_of(ns[j]), kSegAlign);
        off += align_up(np * 2, 256);                       // k16
        off += align_up(np / 8, 256);                       // survivor bits
        off += align_up(np * 2, 256);                       // key_b
        off += align_up(np * 4, 256);                       // idx_b
        off += align_up((size_t)S.nseg[j] * 2 * 1024, 256); // per-segment counts, both digits
    }
    S.bytes = off;
}

void place_job(JobDesc& d, uint32_t n, int j, const LaunchShape& S, char* scratch) {
    d.n = n;
    d.npad = npad_of(n);
    d.seg0 = S.seg0[j];
    d.nseg = S.nseg[j];
    d.ngroups = (d.nseg + kGroup - 1) / kGroup;
    d.ctl = reinterpret_cast<uint32_t*>(scratch + S.ctl_off[j]);
    char* at = scratch + S.arr_off[j];
    const size_t np = std::max<size_t>(d.npad, kSegAlign);
    d.k16 = reinterpret_cast<uint16_t*>(at);
    at += align_up(np * 2, 256);
    d.mask = reinterpret_cast<uint32_t*>(at);
    at += align_up(np / 8, 256);
    d.key_b = reinterpret_cast<uint16_t*>(at);
    at += align_up(np * 2, 256);
    d.idx_b = reinterpret_cast<uint32_t*>(at);
    at += align_up(np * 4, 256);
    d.agg = reinterpret_cast<uint32_t*>(at);
}

size_t table_bytes(int njobs, const LaunchShape& S) {
    return (size_t)njobs * sizeof(JobDesc) + (S.regular ? 0 : S.segs.size() * sizeof(SegDesc));
}

void write_table(void* dst, const JobDesc* jobs, int njobs, const LaunchShape& S) {
    char* p = static_cast<char*>(dst);
    if (p != reinterpret_cast<const char*>(jobs)) std::memcpy(p, jobs, (size_t)njobs * sizeof(JobDesc));
    if (!S.regular)
        std::memcpy(p + (size_t)njobs * sizeof(JobDesc), S.segs.data(), S.segs.size() * sizeof(SegDesc));
}

LaunchDesc launch_desc(const void* d_table, int njobs, const LaunchShape& S, char* scratch, uint32_t* err,
                       uint32_t spin_limit, TraceRec* trace) {
    LaunchDesc L;
    std::memset(&L, 0, sizeof(L));
    L.jobs = static_cast<const JobDesc*>(d_table);
    L.njobs = (uint32_t)njobs;
    L.segs = S.regular ? nullptr
                       : reinterpret_cast<const SegDesc*>(static_cast<const char*>(d_table) +
                                                          (size_t)njobs * sizeof(JobDesc));
    L.nseg = (uint32_t)S.segs.size();
    L.chunk = S.chunk;
    L.first_phase = 0;
    L.spin_limit = spin_limit;
    L.lctl = reinterpret_cast<LaunchCtl*>(scratch);
    L.err = err;
    L.trace = trace;
    return L;
}

// Scratch bytes of a launch of njobs jobs of ns[j] elements.
size_t launch_scratch_bytes(const uint32_t* ns, int njobs, const ws_params& p, int sms) {
    LaunchShape S;
    shape_launch(ns, njobs, p, sms, S);
    return S.bytes;
}

// The per-view shortcuts the keys phase may take, proved here on the host:
//
// fast_transform: the model-view's last row is (0, 0, 0, 1) and the
// projection has the zero pattern of a perspective (entries 1, 2, 3, 4, 6,
// 7, 12, 13, 15 are zero), every entry is finite, and no view-space
// coordinate of the cloud can overflow (|view_j| <= sum_k |m_jk| R + |m_j3|
// well below FLT_MAX, R the largest box coordinate). Then view.w is exactly
// 1 and the dropped projection terms are zeros times finite numbers.
//
// keep_byte / keep_q: the footprint shortcut of the keys phase. With
// A = fx (|W row 0|_1 + |1.3 / p00| |W row 2|_1) and the same for y, and a
// splat's largest |covariance entry| at most 2^sexp, every entry of its
// |T| |Sigma| |T|^T is at most 1.02 max(A)^2 2^sexp / d^2 =: keep_q 2^sexp / d^2
// (keep_q is at least 2^-20, so keep_q 2^sexp stays a normal float).
// keep_byte is the least alpha byte with RN(alpha * 1.85) >= cull.
void view_shortcuts(const ws_view& v, const ws_cloud* c, uint32_t* fast, uint32_t* keep_byte, float* keep_q) {
    const float* M = v.model_view;
    const float* P = v.projection;
    bool finite = true;
    for (int k = 0; k < 16; ++k) finite = finite && std::isfinite(M[k]) && std::isfinite(P[k]);
    *fast = 0;
    if (finite && M[3] == 0.0f && M[7] == 0.0f && M[11] == 0.0f && M[15] == 1.0f && P[1] == 0.0f &&
        P[2] == 0.0f && P[3] == 0.0f && P[4] == 0.0f && P[6] == 0.0f && P[7] == 0.0f && P[12] == 0.0f &&
        P[13] == 0.0f && P[15] == 0.0f) {
        double R = 0.0;
        for (int k = 0; k < 3; ++k) R = std::fmax(R, std::fmax(std::fabs(c->bmin[k]), std::fabs(c->bmax[k])));
        double vmax = 0.0;
        for (int j = 0; j < 3; ++j)
            vmax = std::fmax(vmax, (std::fabs((double)M[j]) + std::fabs((double)M[4 + j]) + std::fabs((double)M[8 + j])) * R +
                                       std::fabs((double)M[12 + j]));
        if (std::isfinite(R) && vmax * 1.01 < 1e37) *fast = 1;
    }
    *keep_byte = 256;
    *keep_q = INFINITY;
    if (!(v.cull > 0.0f) || P[15] != 0.0f || !finite) return;
    const float fx = (P[0] * v.viewport[0]) * 0.5f;
    const float fy = (P[5] * v.viewport[1]) * 0.5f;
    const double xhi = std::fabs((double)(1.3f / P[0])), yhi = std::fabs((double)(1.3f / P[5]));
    const double r0 = std::fabs((double)M[0]) + std::fabs((double)M[4]) + std::fabs((double)M[8]);
    const double r1 = std::fabs((double)M[1]) + std::fabs((double)M[5]) + std::fabs((double)M[9]);
    const double r2 = std::fabs((double)M[2]) + std::fabs((double)M[6]) + std::fabs((double)M[10]);
    const double a0 = std::fabs((double)fx) * (r0 + xhi * r2);
    const double a1 = std::fabs((double)fy) * (r1 + yhi * r2);
    const double a = std::fmax(a0, a1);
    const double q = std::fmax(1.02 * a * a, std::ldexp(1.0, -20));
    if (!std::isfinite(q) || q > 1e30) return;
    float qf = (float)q;
    if ((double)qf < q) qf = std::nextafter(qf, INFINITY);
    for (uint32_t b = 0; b < 256; ++b) {
        const float alpha = (float)b / 255.0f;
        if (alpha * 1.85f >= v.cull && alpha * 255.0f > 1.0f) {
            *keep_byte = b;
            break;
        }
    }
    *keep_q = qf;
}

double host_depth_range(const float mv[16], const double bmin[3], const double bmax[3], int* visible,
                        float* depth_min, float* depth_scale);

// det_min[b]: the least f32 det that makeKeys keeps with alpha byte b under
// `cull`, found by bisection over the ordered non-negative f32 values (the
// test is monotone in det: max, the square root and the two products are);
// -inf when it keeps every det. The table depends on cull alone: the last few
// are kept, so a frame loop's calls (one cull) compute it once.
static void det_thresholds(float cull, float out[256]) {
    struct Entry {
        uint32_t bits;
        float t[256];
    };
    static std::mutex mu;
    static std::vector<Entry> cache;
    static size_t next = 0;
    uint32_t bits;
    std::memcpy(&bits, &cull, 4);
    std::lock_guard<std::mutex> lock(mu);
    for (const Entry& e : cache)
        if (e.bits == bits) {
            std::memcpy(out, e.t, sizeof(e.t));
            return;
        }
    Entry e;
    e.bits = bits;
    for (uint32_t b = 0; b < 256; ++b) {
        const float alpha = (float)b / 255.0f;
        auto kept = [&](float det) {
            const float area = 6.2831853f * std::sqrt(std::fmax(det, 0.0f));
            return !(alpha * area < cull);
        };
        if (kept(0.0f)) {
            e.t[b] = -INFINITY;
            continue;
        }
        uint32_t lo = 0, hi = 0x7f800000u;   // kept(lo) false, kept(+inf) true
        while (hi - lo > 1) {
            const uint32_t mid = lo + (hi - lo) / 2;
            float f;
            std::memcpy(&f, &mid, 4);
            if (kept(f))
                hi = mid;
            else
                lo = mid;
        }
        std::memcpy(&e.t[b], &hi, 4);
    }
    std::memcpy(out, e.t, sizeof(e.t));
    if (cache.size() < 8) {
        cache.push_back(e);
    } else {
        cache[next] = e;
        next = (next + 1) % cache.size();
    }
}

// The view's constants for the keys phase, computed here once per job with
// the same IEEE operations (f32 products and quotients, the FP64 depth range;
// built with -ffp-contract=off) as the device's make_consts.
void fill_view_consts(JobDesc& d) {
    ViewConsts& c = d.vc;
    std::memset(&c, 0, sizeof(c));
    for (int k = 0; k < 16; ++k) {
        c.mv[k] = d.mv[k];
        c.proj[k] = d.proj[k];
    }
    const float p0 = d.proj[0], p5 = d.proj[5];
    c.fx = (p0 * d.viewport[0]) * 0.5f;
    c.fy = (p5 * d.viewport[1]) * 0.5f;
    c.xlo = -1.3f / p0;
    c.xhi = 1.3f / p0;
    c.ylo = -1.3f / p5;
    c.yhi = 1.3f / p5;
    c.cull = d.cull;
    c.persp = d.proj[15] == 0.0f;
    c.keep_q = d.keep_q;
    c.keep_byte = d.keep_byte;
    c.fast = d.fast_transform != 0;
    c.revz = c.fast && d.proj[8] == 0.0f && d.proj[9] == 0.0f && d.proj[10] == 0.0f && d.proj[11] == -1.0f;
    host_depth_range(d.mv, d.bmin, d.bmax, &c.visible, &c.depth_min, &c.depth_scale);
    // makeKeys drops a splat when unpack4x8unorm(colour).a * 255 <= 1
    // (render/splats.js:169-170): alpha = byte / 255 rounded to f32, so the
    // test is monotone in the byte and is a threshold on it.
    c.faint_max = 0;
    for (uint32_t b = 0; b < 256; ++b) {
        const float alpha = (float)b / 255.0f;
        if (alpha * 255.0f <= 1.0f) c.faint_max = b;
    }
    // The footprint bound's constants, each rounded up by a relative 1e-4
    // (far more than the rounding of the few operations that form them).
    auto up = [](double v) {
        const float f = (float)(std::fabs(v) * 1.0001);
        return std::isfinite(f) ? f : INFINITY;
    };
    const float* M = d.mv;
    c.afx = up(c.fx);
    c.afy = up(c.fy);
    c.r0 = up(std::fabs((double)M[0]) + std::fabs((double)M[4]) + std::fabs((double)M[8]));
    c.r1 = up(std::fabs((double)M[1]) + std::fabs((double)M[5]) + std::fabs((double)M[9]));
    c.r2 = up(std::fabs((double)M[2]) + std::fabs((double)M[6]) + std::fabs((double)M[10]));
    c.xcap = up(c.xhi);
    c.ycap = up(c.yhi);
    det_thresholds(d.cull, c.det_min);
}

// Emitter jobs (ws_sort_particles): the ring, the view and the outputs.
static void layout_emitters(JobDesc* out, const ws_emitter* em, int njobs, const LaunchShape& S, char* scratch,
                            const float* thr) {
    for (int j = 0; j < njobs; ++j) {
        JobDesc& d = out[j];
        std::memset(&d, 0, sizeof(d));
        d.kind = kJobParticles;
        d.idx_base = em[j].offset;
        d.pool = static_cast<const float4*>(em[j].pool);
        d.thr = thr;
        for (int k = 0; k < 3; ++k) {
            d.eye[k] = em[j].eye[k];
            d.fwd[k] = em[j].forward[k];
        }
        d.order = em[j].order;
        d.keys = em[j].keys;
        d.count = em[j].count;
        place_job(d, em[j].capacity, j, S, scratch);
    }
}

void layout_jobs(JobDesc* out, const ws_job* jobs, int njobs, const LaunchShape& S, char* scratch) {
    for (int j = 0; j < njobs; ++j) {
        const ws_cloud* c = jobs[j].cloud;
        JobDesc& d = out[j];
        std::memset(&d, 0, sizeof(d));
        d.centers = c->centers;
        d.cov = c->cov;
        d.sexp = c->sexp;
        for (int k = 0; k < 3; ++k) {
            d.bmin[k] = c->bmin[k];
            d.bmax[k] = c->bmax[k];
        }
        std::memcpy(d.mv, jobs[j].view.model_view, sizeof(d.mv));
        std::memcpy(d.proj, jobs[j].view.projection, sizeof(d.proj));
        d.viewport[0] = jobs[j].view.viewport[0];
        d.viewport[1] = jobs[j].view.viewport[1];
        d.cull = jobs[j].view.cull;
        d.order = jobs[j].order;
        d.keys = jobs[j].keys;
        d.count = jobs[j].count;
        view_shortcuts(jobs[j].view, c, &d.fast_transform, &d.keep_byte, &d.keep_q);
        fill_view_consts(d);
        place_job(d, c->n, j, S, scratch);
    }
}

int check_view(ws_ctx* ctx, const ws_view* v) {
    if (!v) return set_error(ctx, WS_ERR_ARG, "ws_sort: view is null");
    const float cull = v->cull;
    if (!(cull >= 0.0f && std::isfinite(cull))) {
        // The reference prints the number as JavaScript would; %g is close.
        return set_error(ctx, WS_ERR_ARG, "splatCull must be 0 or more, got %g", (double)cull);
    }
    return WS_OK;
}

int check_cloud(ws_ctx* ctx, const ws_cloud* c) {
    if (!c) return set_error(ctx, WS_ERR_ARG, "ws_sort: cloud is null");
    if (c->magic != kCloudMagic) return set_error(ctx, WS_ERR_ARG, "ws_sort: not a cloud handle");
    if (!c->alive)
        return set_error(ctx, WS_ERR_UNLOADED, "addSplats: these splats were unloaded; remove the node first");
    if (c->ctx != ctx) return set_error(ctx, WS_ERR_ARG, "ws_sort: the cloud belongs to another context");
    return WS_OK;
}

// The parameters a launch of `splats` splats in total runs with.
const ws_params& params_for(const ws_ctx* ctx, uint64_t splats) {
    int b = 0;
    while (b < 63 && (splats >> (b + 1))) ++b;
    if (b < ctx->tuning_n && ctx->tuning[b].tile) return ctx->tuning[b];
    return ctx->params;
}

// The one-CTA sorts take a launch when every job is one of splats of at
// most kOneMax.
bool one_cta_takes(const JobDesc* jobs, int njobs) {
    for (int j = 0; j < njobs; ++j)
        if (jobs[j].kind != kJobSplats || jobs[j].n > kOneMax) return false;
    return true;
}

// A lone job's staging in one launch: its description (passed by value with
// the launch, so no host-to-device copy) into the job table, and the launch's
// and the job's counters zeroed.
__global__ void __launch_bounds__(1024) stage_kernel(const __grid_constant__ JobDesc job, JobDesc* __restrict__ dst,
                                                     uint32_t* __restrict__ ctl, uint32_t ctl_words) {
    static_assert(sizeof(JobDesc) % 16 == 0, "copied in words");
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&job);
    uint32_t* d = reinterpret_cast<uint32_t*>(dst);
    for (uint32_t k = threadIdx.x; k < sizeof(JobDesc) / 4; k += blockDim.x) d[k] = src[k];
    uint4* c4 = reinterpret_cast<uint4*>(ctl);
    for (uint32_t k = threadIdx.x; k < ctl_words / 4; k += blockDim.x) c4[k] = make_uint4(0, 0, 0, 0);
}

// One persistent launch over `njobs` jobs of ns[j] elements each; `fill`
// writes the job table (kind-specific fields and scratch) into pinned
// staging, given the launch's shape and the scratch base. The stream waits
// for the context's previous launch, so one scratch is never shared by two
// launches in flight.
// `tail`, when given, queues more kernels right after the sort's, before the
// launch's events (so that nothing but kernels lies between them and they
// may overlap the sort's last phase).
template <class Fill>
static int launch_jobs(ws_ctx* ctx, const std::vector<uint32_t>& ns, int njobs, Fill fill, cudaStream_t stream,
                       const std::function<cudaError_t(cudaStream_t)>* tail = nullptr) {
    cudaError_t e;
    uint64_t splats = 0;
    for (int j = 0; j < njobs; ++j) splats += ns[j];
    const ws_params& P = params_for(ctx, splats);
    const bool same = ctx->shape_valid && ctx->last_ns == ns && !std::memcmp(&ctx->last_params, &P, sizeof(P));
    if (!same) {
        shape_launch(ns.data(), njobs, P, ctx->sms, ctx->shape);
        ctx->last_ns = ns;
        ctx->last_params = P;
        ctx->shape_valid = true;
    }
    const LaunchShape& S = ctx->shape;
    if (S.bytes > ctx->scratch.bytes) {
        // The old scratch may still be read by a launch in flight.
        if ((e = cudaEventSynchronize(ctx->launched)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort");
        if ((e = ctx->scratch.ensure(S.bytes)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort scratch");
    }
    const size_t tb = table_bytes(njobs, S);
    if (tb > ctx->jobs_d.bytes) {
        if ((e = cudaEventSynchronize(ctx->launched)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort");
        if ((e = ctx->jobs_d.ensure(tb)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort job table");
    }
    char* scratch = static_cast<char*>(ctx->scratch.p);
    if (stream != ctx->stream) cudaStreamWaitEvent(stream, ctx->launched, 0);
    // The one-CTA sorts take launches of small jobs of splats (not traced).
    bool one_cta = P.algorithm != kAlgoPhases && !ctx->tracing;
    if (njobs == 1) {
        // A lone job's description travels with the staging kernel's launch:
        // no pinned buffer, so nothing to wait for before writing it.
        JobDesc one;
        fill(&one, S, scratch);
        one_cta = one_cta && one_cta_takes(&one, 1);
        stage_kernel<<<1, 1024, 0, stream>>>(one, static_cast<JobDesc*>(ctx->jobs_d.p),
                                             reinterpret_cast<uint32_t*>(scratch), (uint32_t)(S.ctl_bytes / 4));
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(ctx, e, "ws_sort staging");
        ctx->h2d_bytes += sizeof(JobDesc);
    } else {
        // Pinned staging is rewritten only after its previous upload finished.
        if ((e = cudaEventSynchronize(ctx->staged)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort");
        if ((e = ctx->jobs_h.ensure(tb)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort staging");
        JobDesc* hj = static_cast<JobDesc*>(ctx->jobs_h.p);
        fill(hj, S, scratch);
        one_cta = one_cta && one_cta_takes(hj, njobs);
        write_table(ctx->jobs_h.p, hj, njobs, S);
        if ((e = cudaMemcpyAsync(ctx->jobs_d.p, ctx->jobs_h.p, tb, cudaMemcpyHostToDevice, stream)) != cudaSuccess)
            return cuda_error(ctx, e, "ws_sort upload");
        ctx->h2d_bytes += tb;
        cudaEventRecord(ctx->staged, stream);
    }
    if (njobs != 1 && (e = cudaMemsetAsync(scratch, 0, S.ctl_bytes, stream)) != cudaSuccess)
        return cuda_error(ctx, e, "ws_sort reset");
    const size_t n_items = (size_t)kPhases * S.segs.size();
    cudaEvent_t t_stop = nullptr;
    if (ctx->timing) {
        if (ctx->timing_used == ctx->timing_events.size()) {
            cudaEvent_t a, b;
            if ((e = cudaEventCreate(&a)) != cudaSuccess) return cuda_error(ctx, e, "ws_timing");
            if ((e = cudaEventCreate(&b)) != cudaSuccess) return cuda_error(ctx, e, "ws_timing");
            ctx->timing_events.emplace_back(a, b);
        }
        cudaEventRecord(ctx->timing_events[ctx->timing_used].first, stream);
        t_stop = ctx->timing_events[ctx->timing_used].second;
        ++ctx->timing_used;
    }
    TraceRec* trace = nullptr;
    if (ctx->tracing) {
        if ((e = ctx->trace_d.ensure(n_items * sizeof(TraceRec))) != cudaSuccess) return cuda_error(ctx, e, "ws_trace");
        trace = static_cast<TraceRec*>(ctx->trace_d.p);
        ctx->trace_segs = S.segs;
        ctx->trace_first_phase = 0;
        ctx->trace_grid = (int)std::min<size_t>(S.grid, S.segs.size());
    }
    const LaunchDesc L = launch_desc(ctx->jobs_d.p, njobs, S, scratch, ctx->err_d, P.spin_limit, trace);
    e = one_cta ? launch_one(L, P.algorithm, stream)
                : launch_sort(L, S.threads, (int)std::min<size_t>(S.grid, S.segs.size()), ctx->sms, stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "ws_sort launch");
    if (tail && (e = (*tail)(stream)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort copy");
    if (t_stop) cudaEventRecord(t_stop, stream);
    cudaEventRecord(ctx->launched, stream);
    ++ctx->launches;
    ++ctx->timing_launches;
    return WS_OK;
}

// A stable sort of n given 16-bit keys (every element kept) in one launch:
// order[] receives element indices by (key, index), sorted[] the keys.
int run_given_keys(ws_ctx* ctx, const uint16_t* keys, uint32_t n, uint32_t* order, uint32_t* sorted, uint32_t* count,
                   cudaStream_t stream) {
    std::vector<uint32_t> ns(1, n);
    return launch_jobs(
        ctx, ns, 1,
        [&](JobDesc* hj, const LaunchShape& S, char* scratch) {
            JobDesc& d = hj[0];
            std::memset(&d, 0, sizeof(d));
            d.kind = kJobKeys;
            d.keys_in = keys;
            d.order = order;
            d.keys = sorted;
            d.count = count;
            place_job(d, n, 0, S, scratch);
        },
        stream);
}

int run_batch(ws_ctx* ctx, const ws_job* jobs, int njobs, cudaStream_t stream,
              const std::function<cudaError_t(cudaStream_t)>* tail = nullptr) {
    std::vector<uint32_t> ns(njobs);
    for (int j = 0; j < njobs; ++j) ns[j] = jobs[j].cloud->n;
    return launch_jobs(
        ctx, ns, njobs,
        [&](JobDesc* hj, const LaunchShape& S, char* scratch) { layout_jobs(hj, jobs, njobs, S, scratch); },
        stream, tail);
}

// Reads and clears the sticky device error words. Call after a sync.
int take_device_error(ws_ctx* ctx) {
    uint32_t words[2] = {0, 0};
    cudaError_t e = cudaMemcpy(words, ctx->err_d, sizeof(words), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(ctx, e, "ws_sync");
    if (words[0]) {
        cudaMemset(ctx->err_d, 0, 2 * sizeof(uint32_t));
        return set_error(ctx, WS_ERR_TIMEOUT,
                         "a device-side wait gave up (code %u at work item %u); the results of that launch "
                         "are invalid",
                         words[0], words[1]);
    }
    return WS_OK;
}

double host_depth_range(const float mv[16], const double bmin[3], const double bmax[3], int* visible,
                        float* depth_min, float* depth_scale) {
    double nearv = INFINITY, farv = -INFINITY;
    for (int k = 0; k < 8; ++k) {
        const double x = (k & 1) ? bmax[0] : bmin[0];
        const double y = (k & 2) ? bmax[1] : bmin[1];
        const double z = (k & 4) ? bmax[2] : bmin[2];
        const double depth = -(double(mv[2]) * x + double(mv[6]) * y + double(mv[10]) * z + double(mv[14]));
        if (depth < nearv) nearv = depth;
        if (depth > farv) farv = depth;
    }
    *visible = farv > 0.0;
    nearv = nearv > 0.0 ? nearv : 0.0;
    const double span = farv - nearv;
    *depth_min = (float)nearv;
    *depth_scale = (float)(65535.0 / (span > 1e-6 ? span : 1e-6));
    return nearv;
}

}  // namespace wsort

using namespace wsort;

// ------------------------------------------------------------------ context

extern "C" int ws_create(ws_ctx** out, int device) {
    if (!out) return WS_ERR_ARG;
    *out = nullptr;
    ws_ctx* ctx = new (std::nothrow) ws_ctx();
    if (!ctx) return WS_ERR_NOMEM;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete ctx;
        return WS_ERR_CUDA;
    }
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
    // A blocking stream: work a caller queued on the legacy default stream
    // (where torch puts it unless told otherwise) is ordered before a sort.
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamDefault)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->staged, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->launched, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->err_d, 4 * sizeof(uint32_t))) != cudaSuccess ||
        (e = ctx->count_h.ensure(64)) != cudaSuccess) {
        ws_destroy(ctx);
        return WS_ERR_CUDA;
    }
    cudaMemset(ctx->err_d, 0, 4 * sizeof(uint32_t));
    ctx->params.tile = 2048;
    ctx->params.ctas_per_sm = 1;
    ctx->params.spin_limit = 1u << 22;
    ctx->params.segs_per_cta = 1;
    *out = ctx;
    return WS_OK;
}

extern "C" int ws_destroy(ws_ctx* ctx) {
    if (!ctx) return WS_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaDeviceSynchronize();
    ctx->scratch.release();
    ctx->jobs_d.release();
    ctx->out_d.release();
    ctx->copy_d.release();
    ctx->copy_h.release();
    ctx->thr_d.release();
    ctx->draw_d.release();
    ctx->pairs_d.release();
    ctx->jobs_h.release();
    ctx->count_h.release();
    for (int b = 0; b < 2; ++b) {
        ctx->load_h[b].release();
        ctx->load_d[b].release();
        if (ctx->load_done[b]) cudaEventDestroy(ctx->load_done[b]);
    }
    if (ctx->err_d) cudaFree(ctx->err_d);
    if (ctx->staged) cudaEventDestroy(ctx->staged);
    if (ctx->launched) cudaEventDestroy(ctx->launched);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    for (auto& pr : ctx->timing_events) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    for (ws_cloud* c : ctx->freed) delete c;
    delete ctx;
    return WS_OK;
}

extern "C" const char* ws_last_error(const ws_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

extern "C" int ws_sync(ws_ctx* ctx) {
    if (!ctx) return WS_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_error(ctx, e, "ws_sync");
    return take_device_error(ctx);
}

extern "C" int ws_get_params(const ws_ctx* ctx, ws_params* out) {
    if (!ctx || !out) return WS_ERR_ARG;
    *out = ctx->params;
    return WS_OK;
}

// The kernel variants that exist: tile 1024, 2048 or 4096 with 2, 3 or 4
// resident CTAs per SM (0 picks 3), and tile 1024 with 6.
// The kernel variants that exist: 1024 threads a CTA (one CTA an SM) or 512
// (two); segments no smaller than `tile` splats, a multiple of 256.
static const char* params_problem(const ws_params* p) {
    if (p->algorithm > kAlgoOneCount) return "algorithm must be 0 (three phases), 1 (one-CTA radix) or 2 (one-CTA counting)";
    if (p->tile < kSegAlign || p->tile > (1u << 24) || p->tile % kSegAlign)
        return "tile must be a multiple of 256 from 256 to 2^24";
    if (p->spin_limit == 0) return "spin_limit must be positive";
    if (p->ctas_per_sm > 2) return "ctas_per_sm must be 0, 1 or 2";
    if (p->segs_per_cta > 64) return "segs_per_cta must be 0 to 64";
    return nullptr;
}

static int valid_params(ws_ctx* ctx, const ws_params* p) {
    const char* why = params_problem(p);
    return why ? set_error(ctx, WS_ERR_ARG, "%s", why) : WS_OK;
}

extern "C" int ws_set_tuning(ws_ctx* ctx, const ws_params* table, int n) {
    if (!ctx || n < 0 || n > 32 || (n && !table)) return WS_ERR_ARG;
    for (int b = 0; b < n; ++b)
        if (table[b].tile) {
            const int rc = valid_params(ctx, &table[b]);
            if (rc) return rc;
        }
    for (int b = 0; b < 32; ++b) ctx->tuning[b] = b < n ? table[b] : ws_params{};
    ctx->tuning_n = n;
    ctx->shape_valid = false;
    return WS_OK;
}

extern "C" int ws_set_params(ws_ctx* ctx, const ws_params* p) {
    if (!ctx || !p) return WS_ERR_ARG;
    if (const char* why = params_problem(p)) return set_error(ctx, WS_ERR_ARG, "ws_set_params: %s", why);
    ctx->params = *p;
    ctx->shape_valid = false;
    return WS_OK;
}

// ------------------------------------------------------------------ clouds

static int sniff(ws_ctx* ctx, const uint8_t* d, size_t nbytes) {
    // The order of parseSplats (src/scene/splats.js:60-76).
    if (nbytes >= 8 && d[0] == 0x4e && d[1] == 0x47 && d[2] == 0x53 && d[3] == 0x50) {
        uint32_t version;
        std::memcpy(&version, d + 4, 4);
        if (version >= 4)
            return set_error(ctx, WS_ERR_FORMAT,
                             "splats: a .spz of version 4, compressed with zstd, which browsers cannot unpack; "
                             "save it as version 3, or as a .ply or .splat");
    }
    if (nbytes >= 4 && d[0] == 0x70 && d[1] == 0x6c && d[2] == 0x79 && (d[3] == 0x0a || d[3] == 0x0d))
        return set_error(ctx, WS_ERR_FORMAT, "splats: a .ply is not read here: only .splat records are");
    if (nbytes >= 4 && d[0] == 0x50 && d[1] == 0x4b && d[2] == 0x03 && d[3] == 0x04)
        return set_error(ctx, WS_ERR_FORMAT, "splats: this is a zip: unpack it with readSplats, which reads a .sog");
    if (nbytes >= 2 && d[0] == 0x1f && d[1] == 0x8b)
        return set_error(ctx, WS_ERR_FORMAT, "splats: this is gzipped: unpack it with readSplats, which reads a .spz");
    if (nbytes == 0 || nbytes % 32 != 0)
        return set_error(ctx, WS_ERR_FORMAT,
                         "splats: not a .ply, and %zu bytes is not a whole number of 32-byte .splat records", nbytes);
    if (nbytes / 32 > WS_MAX_SPLATS)
        return set_error(ctx, WS_ERR_CAPACITY, "splats: %zu splats are more than this device holds in one buffer, %u",
                         nbytes / 32, WS_MAX_SPLATS);
    return WS_OK;
}

// A cloud from n .splat records: in host memory (streamed through the
// context's pinned chunks, each decoded while the next one is copied) or on
// the device (decoded in place).
static int decode_cloud(ws_ctx* ctx, const void* records, bool on_host, uint32_t n, ws_cloud** out) {
    cudaError_t e;
    ws_cloud* c = new (std::nothrow) ws_cloud();
    if (!c) return set_error(ctx, WS_ERR_NOMEM, "ws_cloud: out of host memory");
    c->ctx = ctx;
    c->n = n;
    const size_t np = pad_splats(n);
    if ((e = cudaMalloc(&c->centers, np * sizeof(float4))) != cudaSuccess ||
        (e = cudaMalloc(&c->cov, np * 3 * sizeof(float2))) != cudaSuccess ||
        (e = cudaMalloc(&c->sexp, np)) != cudaSuccess) {
        ws_cloud_free(c);
        return cuda_error(ctx, e, "ws_cloud");
    }
    uint32_t* words = nullptr;   // bounds[6], unused, bad
    if ((e = cudaMalloc(&words, 8 * sizeof(uint32_t))) != cudaSuccess) {
        ws_cloud_free(c);
        return cuda_error(ctx, e, "ws_cloud");
    }
    const uint32_t init[8] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u, 0u, 0xFFFFFFFFu};
    cudaMemcpyAsync(words, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream);
    cudaMemsetAsync(c->centers, 0, np * sizeof(float4), ctx->stream);
    cudaMemsetAsync(c->cov, 0, np * 3 * sizeof(float2), ctx->stream);
    cudaMemsetAsync(c->sexp, 0x7f, np, ctx->stream);   // padding: no shortcut
    e = on_host ? stream_splat_records(ctx, static_cast<const uint8_t*>(records), n, c->centers, c->cov, c->sexp, words,
                                       words + 7)
                : launch_decode(records, n, c->centers, c->cov, c->sexp, words, words + 7, ctx->sms, ctx->stream, 0);
    uint32_t back[8];
    if (e == cudaSuccess) e = cudaMemcpyAsync(back, words, sizeof(back), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(words);
    if (e != cudaSuccess) {
        ws_cloud_free(c);
        return cuda_error(ctx, e, "ws_cloud decode");
    }
    if (back[7] != 0xFFFFFFFFu) {
        ws_cloud_free(c);
        return set_error(ctx, WS_ERR_NAN, "splats: splat %u has a position that is not a number", back[7]);
    }
    for (int k = 0; k < 3; ++k) {
        uint32_t lo = back[k], hi = back[3 + k];
        lo = (lo & 0x80000000u) ? (lo & 0x7FFFFFFFu) : ~lo;
        hi = (hi & 0x80000000u) ? (hi & 0x7FFFFFFFu) : ~hi;
        float flo, fhi;
        std::memcpy(&flo, &lo, 4);
        std::memcpy(&fhi, &hi, 4);
        c->bmin[k] = flo;
        c->bmax[k] = fhi;
    }
    c->magic = kCloudMagic;
    c->alive = true;
    *out = c;
    return WS_OK;
}

extern "C" int ws_cloud_from_splat(ws_ctx* ctx, const uint8_t* bytes, size_t nbytes, ws_cloud** out) {
    if (!ctx || !out || (!bytes && nbytes)) return set_error(ctx, WS_ERR_ARG, "ws_cloud_from_splat: null argument");
    *out = nullptr;
    cudaSetDevice(ctx->device);
    int rc = sniff(ctx, bytes, nbytes);
    if (rc) return rc;
    return decode_cloud(ctx, bytes, true, (uint32_t)(nbytes / 32), out);
}

extern "C" int ws_cloud_from_device(ws_ctx* ctx, const void* dev, size_t nbytes, ws_cloud** out) {
    if (!ctx || !out || (!dev && nbytes)) return set_error(ctx, WS_ERR_ARG, "ws_cloud_from_device: null argument");
    *out = nullptr;
    cudaSetDevice(ctx->device);
    if (reinterpret_cast<uintptr_t>(dev) % 16)
        return set_error(ctx, WS_ERR_ARG, "ws_cloud_from_device: records must be 16-byte aligned");
    uint8_t head[8] = {0};
    if (nbytes) {
        cudaError_t e = cudaMemcpy(head, dev, nbytes < 8 ? nbytes : 8, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_error(ctx, e, "ws_cloud_from_device");
    }
    int rc = sniff(ctx, head, nbytes);
    if (rc) return rc;
    return decode_cloud(ctx, dev, false, (uint32_t)(nbytes / 32), out);
}

extern "C" int ws_cloud_info(const ws_cloud* c, uint32_t* count, double mn[3], double mx[3]) {
    if (!c || c->magic != kCloudMagic) return WS_ERR_ARG;
    if (!c->alive) return WS_ERR_UNLOADED;
    if (count) *count = c->n;
    for (int k = 0; k < 3; ++k) {
        if (mn) mn[k] = c->bmin[k];
        if (mx) mx[k] = c->bmax[k];
    }
    return WS_OK;
}

extern "C" int ws_cloud_download(const ws_cloud* c, float* centers, float* covariances) {
    if (!c || c->magic != kCloudMagic) return WS_ERR_ARG;
    if (!c->alive) return WS_ERR_UNLOADED;
    cudaSetDevice(c->ctx->device);
    cudaError_t e = cudaStreamSynchronize(c->ctx->stream);
    if (e == cudaSuccess && centers) e = cudaMemcpy(centers, c->centers, (size_t)c->n * 16, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && covariances)
        e = cudaMemcpy(covariances, c->cov, (size_t)c->n * 24, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? WS_OK : cuda_error(c->ctx, e, "ws_cloud_download");
}

extern "C" int ws_cloud_free(ws_cloud* c) {
    if (!c) return WS_ERR_ARG;
    if (c->magic != kCloudMagic) {   // a half-built cloud from a failed load
        if (c->centers) cudaFree(c->centers);
        if (c->cov) cudaFree(c->cov);
        if (c->sexp) cudaFree(c->sexp);
        if (c->sh) cudaFree(c->sh);
        delete c;
        return WS_OK;
    }
    if (!c->alive) return WS_ERR_UNLOADED;
    cudaSetDevice(c->ctx->device);
    // A sort in flight may still read the cloud.
    cudaDeviceSynchronize();
    if (c->centers) cudaFree(c->centers);
    if (c->cov) cudaFree(c->cov);
    if (c->sexp) cudaFree(c->sexp);
    if (c->sh) cudaFree(c->sh);
    c->centers = nullptr;
    c->cov = nullptr;
    c->sexp = nullptr;
    c->sh = nullptr;
    c->sh_degree = 0;
    // The handle stays valid (and refused by every call) until its context
    // is destroyed, so a sort of a freed cloud is an error, not a crash.
    c->alive = false;
    c->ctx->freed.push_back(c);
    return WS_OK;
}

extern "C" int ws_depth_range(const ws_cloud* c, const float mv[16], int* visible, float* dmin, float* dscale) {
    if (!c || !mv || !visible || !dmin || !dscale || c->magic != kCloudMagic) return WS_ERR_ARG;
    if (!c->alive) return WS_ERR_UNLOADED;
    host_depth_range(mv, c->bmin, c->bmax, visible, dmin, dscale);
    return WS_OK;
}

// ------------------------------------------------------------------ sorting

// The device address of pinned host memory (mapped under unified
// addressing), or null for any other pointer.
static uint32_t* mapped_alias(uint32_t* p) {
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
    return static_cast<uint32_t*>(a.devicePointer);
}

// The survivors' order (and keys) into mapped host memory, and the count and
// the error words into `words`: consecutive threads write consecutive words,
// so each warp's stores leave as whole 128-byte writes.
__global__ void __launch_bounds__(256) copy_out_kernel(const uint32_t* __restrict__ order,
                                                       const uint32_t* __restrict__ keys,
                                                       const uint32_t* __restrict__ count,
                                                       const uint32_t* __restrict__ err, uint32_t* horder,
                                                       uint32_t* hkeys, uint32_t* words, uint32_t cap) {
    const uint32_t c = *count;
    const uint32_t s = c < cap ? c : cap;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        words[0] = c;
        words[1] = err[0];
        words[2] = err[1];
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s; i += gridDim.x * blockDim.x) {
        horder[i] = order[i];
        if (hkeys) hkeys[i] = keys[i];
    }
}

extern "C" int ws_sort(ws_ctx* ctx, const ws_cloud* cloud, const ws_view* view, uint32_t* order, uint32_t* keys,
                       uint32_t* count, int flags, void* stream_p) {
    NvtxRange nvtx("ws_sort");
    if (!ctx) return WS_ERR_ARG;
    int rc;
    if ((rc = check_cloud(ctx, cloud)) || (rc = check_view(ctx, view))) return rc;
    if (!order || !count) return set_error(ctx, WS_ERR_ARG, "ws_sort: order and count are required");
    if (flags != WS_HOST_OUTPUT && flags != WS_DEVICE_OUTPUT) return set_error(ctx, WS_ERR_ARG, "ws_sort: bad flags");
    cudaSetDevice(ctx->device);
    cudaStream_t stream = stream_p ? static_cast<cudaStream_t>(stream_p) : ctx->stream;
    ws_job job;
    job.cloud = cloud;
    job.view = *view;
    if (flags == WS_DEVICE_OUTPUT) {
        job.order = order;
        job.keys = keys;
        job.count = count;
        return run_batch(ctx, &job, 1, stream);
    }
    // Host output: sort into the context's device buffers, then copy back
    // the survivors only.
    const size_t n = cloud->n;
    cudaError_t e;
    // Pinned (device-mapped) host outputs: a small kernel after the sort
    // reads the count on the device and writes the survivors straight into
    // them, and the count and error words into the context's pinned words;
    // one synchronisation instead of a count read-back and a second copy.
    uint32_t* order_dev = mapped_alias(order);
    uint32_t* keys_dev = keys ? mapped_alias(keys) : nullptr;
    uint32_t* words_dev = mapped_alias(static_cast<uint32_t*>(ctx->count_h.p));
    const bool direct = order_dev && words_dev && (!keys || keys_dev);
    if ((e = cudaEventSynchronize(ctx->launched)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort");
    if ((e = ctx->out_d.ensure(align_up((2 * n + 1) * sizeof(uint32_t), 256))) != cudaSuccess)
        return cuda_error(ctx, e, "ws_sort output");
    uint32_t* d = static_cast<uint32_t*>(ctx->out_d.p);
    job.order = d;
    job.keys = keys ? d + n : nullptr;
    job.count = d + 2 * n;
    if ((rc = run_batch(ctx, &job, 1, stream))) return rc;
    uint32_t* hc = static_cast<uint32_t*>(ctx->count_h.p);
    if (direct) {
        const uint32_t blocks = std::max(1u, std::min((uint32_t)((n + 1023) / 1024), (uint32_t)ctx->sms * 4));
        copy_out_kernel<<<blocks, 256, 0, stream>>>(job.order, job.keys, job.count, ctx->err_d, order_dev, keys_dev,
                                                    words_dev, (uint32_t)n);
        if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(stream)) != cudaSuccess)
            return cuda_error(ctx, e, "ws_sort");
        if (hc[1]) return take_device_error(ctx);
        *count = hc[0];
        ctx->d2h_bytes += 12 + (size_t)hc[0] * (keys ? 8 : 4);
        return WS_OK;
    }
    if ((e = cudaMemcpyAsync(hc, job.count, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hc + 1, ctx->err_d, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess)
        return cuda_error(ctx, e, "ws_sort");
    if (hc[1]) return take_device_error(ctx);
    const uint32_t s = hc[0];
    *count = s;
    ctx->d2h_bytes += 12 + (size_t)s * (keys ? 8 : 4);
    if (s) {
        if ((e = cudaMemcpyAsync(order, job.order, (size_t)s * 4, cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
            return cuda_error(ctx, e, "ws_sort download");
        if (keys && (e = cudaMemcpyAsync(keys, job.keys, (size_t)s * 4, cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
            return cuda_error(ctx, e, "ws_sort download");
        if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort download");
    }
    return WS_OK;
}

extern "C" int ws_sort_batch(ws_ctx* ctx, int njobs, const ws_job* jobs, void* stream_p) {
    NvtxRange nvtx("ws_sort_batch");
    if (!ctx) return WS_ERR_ARG;
    if (njobs < 0 || (njobs && !jobs)) return set_error(ctx, WS_ERR_ARG, "ws_sort_batch: bad job list");
    if (njobs == 0) return WS_OK;
    if (njobs > (1 << 20)) return set_error(ctx, WS_ERR_ARG, "ws_sort_batch: too many jobs");
    for (int j = 0; j < njobs; ++j) {
        int rc;
        if ((rc = check_cloud(ctx, jobs[j].cloud)) || (rc = check_view(ctx, &jobs[j].view))) return rc;
        if (!jobs[j].order || !jobs[j].count) return set_error(ctx, WS_ERR_ARG, "ws_sort_batch: job %d has no output", j);
    }
    cudaSetDevice(ctx->device);
    return run_batch(ctx, jobs, njobs, stream_p ? static_cast<cudaStream_t>(stream_p) : ctx->stream);
}

// One job's results on their way to host memory (ws_sort_batch_host): the
// device addresses of the caller's pinned buffers; the job's device outputs
// and its completion count are in its job description.
struct HostCopy {
    uint32_t* horder;
    uint32_t* hkeys;            // or null
    uint32_t* hcount;
    uint32_t n;                 // the job's splats: no count read back exceeds it
    uint32_t pad[1];
};

// Every job's survivors into mapped host memory: blockIdx.y is the job, the
// x blocks stride over its survivors; consecutive threads write consecutive
// words. It is launched right behind the sort's last pass and may start
// while that pass runs: a block first waits (bounded) until its job's high
// pass is complete, so early jobs cross PCIe while later ones are sorted.
// Block (0, j) writes the count.
__global__ void __launch_bounds__(256) copy_jobs_kernel(const JobDesc* __restrict__ jobs,
                                                        const HostCopy* __restrict__ hc, uint32_t* err,
                                                        uint32_t spin_limit) {
    __shared__ uint32_t ready;
    const JobDesc& J = jobs[blockIdx.y];
    if (threadIdx.x == 0) {
        const JobCtl* ctl = reinterpret_cast<const JobCtl*>(J.ctl);
        uint32_t spins = 0;
        ready = 1;
        while (ld_acquire(&ctl->high_done) < J.nseg) {
            if (*(volatile uint32_t*)err) {   // the sort failed: its error stands
                ready = 0;
                break;
            }
            if (++spins > spin_limit) {
                if (atomicCAS(err, 0u, kErrWaitPhase) == 0u) err[1] = 0xFFFFFFFFu;
                ready = 0;
                break;
            }
            __nanosleep(64);
        }
    }
    __syncthreads();
    if (!ready) return;
    const HostCopy H = hc[blockIdx.y];
    // After a device error a job's count may never have been written: the
    // copy stays inside the job's buffers whatever it holds.
    const uint32_t c = min(__ldcg(J.count), H.n);
    if (blockIdx.x == 0 && threadIdx.x == 0) *H.hcount = c;
    const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    // 16 bytes a thread where both sides are 16-byte aligned (the device
    // outputs always are; pinned host buffers usually), the rest a word at a time.
    uint32_t done = 0;
    const bool wide = ((reinterpret_cast<uintptr_t>(H.horder) | reinterpret_cast<uintptr_t>(J.order)) & 15u) == 0 &&
                      (!H.hkeys || ((reinterpret_cast<uintptr_t>(H.hkeys) | reinterpret_cast<uintptr_t>(J.keys)) & 15u) == 0);
    if (wide) {
        const uint32_t c4 = c / 4u;
        for (uint32_t i = t0; i < c4; i += stride) {
            reinterpret_cast<uint4*>(H.horder)[i] = __ldcg(reinterpret_cast<const uint4*>(J.order) + i);
            if (H.hkeys) reinterpret_cast<uint4*>(H.hkeys)[i] = __ldcg(reinterpret_cast<const uint4*>(J.keys) + i);
        }
        done = c4 * 4u;
    }
    for (uint32_t i = done + t0; i < c; i += stride) {
        H.horder[i] = __ldcg(&J.order[i]);
        if (H.hkeys) H.hkeys[i] = __ldcg(&J.keys[i]);
    }
}

extern "C" int ws_sort_batch_host(ws_ctx* ctx, int njobs, const ws_job* jobs, void* stream_p) {
    NvtxRange nvtx("ws_sort_batch_host");
    if (!ctx) return WS_ERR_ARG;
    if (njobs < 0 || (njobs && !jobs)) return set_error(ctx, WS_ERR_ARG, "ws_sort_batch_host: bad job list");
    if (njobs == 0) return WS_OK;
    // One copy grid row a job: at most 65535 (the grid's y limit).
    if (njobs > 65535) return set_error(ctx, WS_ERR_ARG, "ws_sort_batch_host: too many jobs (at most 65535)");
    for (int j = 0; j < njobs; ++j) {
        int rc;
        if ((rc = check_cloud(ctx, jobs[j].cloud)) || (rc = check_view(ctx, &jobs[j].view))) return rc;
        if (!jobs[j].order || !jobs[j].count)
            return set_error(ctx, WS_ERR_ARG, "ws_sort_batch_host: job %d has no output", j);
    }
    cudaSetDevice(ctx->device);
    cudaStream_t stream = stream_p ? static_cast<cudaStream_t>(stream_p) : ctx->stream;
    cudaError_t e;
    // Device outputs, one region per job: order, keys, count.
    std::vector<size_t> off(njobs);
    size_t words = 0;
    for (int j = 0; j < njobs; ++j) {
        off[j] = words;
        words += align_up(2 * (size_t)jobs[j].cloud->n + 1, 64);
    }
    if ((e = cudaEventSynchronize(ctx->launched)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort_batch_host");
    if ((e = ctx->out_d.ensure(words * sizeof(uint32_t) + 256)) != cudaSuccess)
        return cuda_error(ctx, e, "ws_sort_batch_host output");
    uint32_t* d = static_cast<uint32_t*>(ctx->out_d.p);
    std::vector<ws_job> dj(jobs, jobs + njobs);
    std::vector<HostCopy> hc(njobs);
    bool direct = true;
    for (int j = 0; j < njobs; ++j) {
        const size_t n = jobs[j].cloud->n;
        dj[j].order = d + off[j];
        dj[j].keys = jobs[j].keys ? d + off[j] + n : nullptr;
        dj[j].count = d + off[j] + 2 * n;
        HostCopy& h = hc[j];
        std::memset(&h, 0, sizeof(h));
        h.horder = mapped_alias(jobs[j].order);
        h.hkeys = jobs[j].keys ? mapped_alias(jobs[j].keys) : nullptr;
        h.hcount = mapped_alias(jobs[j].count);
        h.n = (uint32_t)n;
        direct = direct && h.horder && h.hcount && (!jobs[j].keys || h.hkeys);
    }
    if (direct) {
        // The copy table goes up before the sort, so that the copy kernel
        // follows the sort's last pass directly in the stream and overlaps
        // it. The table's pinned staging is free: every call ends with a
        // synchronisation.
        const size_t tb = (size_t)njobs * sizeof(HostCopy);
        if ((e = ctx->copy_h.ensure(tb)) != cudaSuccess || (e = ctx->copy_d.ensure(tb)) != cudaSuccess)
            return cuda_error(ctx, e, "ws_sort_batch_host staging");
        std::memcpy(ctx->copy_h.p, hc.data(), tb);
        if ((e = cudaMemcpyAsync(ctx->copy_d.p, ctx->copy_h.p, tb, cudaMemcpyHostToDevice, stream)) != cudaSuccess)
            return cuda_error(ctx, e, "ws_sort_batch_host upload");
        uint32_t max_n = 0;
        for (int j = 0; j < njobs; ++j) max_n = std::max(max_n, jobs[j].cloud->n);
        const uint32_t bx = std::max(1u, std::min((max_n + 2047) / 2048, 64u));
        const HostCopy* table = static_cast<const HostCopy*>(ctx->copy_d.p);
        const uint32_t spin = ctx->params.spin_limit;
        const std::function<cudaError_t(cudaStream_t)> tail = [&](cudaStream_t s) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(bx, (unsigned)njobs);
            cfg.blockDim = dim3(256);
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            return cudaLaunchKernelEx(&cfg, copy_jobs_kernel, static_cast<const JobDesc*>(ctx->jobs_d.p), table,
                                      ctx->err_d, spin);
        };
        int rc = run_batch(ctx, dj.data(), njobs, stream, &tail);
        if (rc) return rc;
        uint32_t* hw = static_cast<uint32_t*>(ctx->count_h.p);
        if ((e = cudaMemcpyAsync(hw, ctx->err_d, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess)
            return cuda_error(ctx, e, "ws_sort_batch_host");
        if (hw[0]) return take_device_error(ctx);
        ctx->h2d_bytes += tb;
        ctx->d2h_bytes += 8;
        for (int j = 0; j < njobs; ++j) ctx->d2h_bytes += 4 + (size_t)*jobs[j].count * (jobs[j].keys ? 8 : 4);
        return WS_OK;
    }
    int rc = run_batch(ctx, dj.data(), njobs, stream);
    if (rc) return rc;
    // Pageable outputs: the counts first, then each job's survivors.
    std::vector<uint32_t> counts(njobs);
    for (int j = 0; j < njobs; ++j)
        if ((e = cudaMemcpyAsync(&counts[j], dj[j].count, 4, cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
            return cuda_error(ctx, e, "ws_sort_batch_host");
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort_batch_host");
    if ((rc = take_device_error(ctx))) return rc;
    ctx->d2h_bytes += 8;
    for (int j = 0; j < njobs; ++j) {
        *jobs[j].count = counts[j];
        ctx->d2h_bytes += 4 + (size_t)counts[j] * (jobs[j].keys ? 8 : 4);
        if (!counts[j]) continue;
        if ((e = cudaMemcpyAsync(jobs[j].order, dj[j].order, (size_t)counts[j] * 4, cudaMemcpyDeviceToHost, stream)) !=
                cudaSuccess ||
            (jobs[j].keys && (e = cudaMemcpyAsync(jobs[j].keys, dj[j].keys, (size_t)counts[j] * 4,
                                                  cudaMemcpyDeviceToHost, stream)) != cudaSuccess))
            return cuda_error(ctx, e, "ws_sort_batch_host download");
    }
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_error(ctx, e, "ws_sort_batch_host download");
    return WS_OK;
}

// -------------------------------------------------------------- self-test

extern "C" int ws_selftest_wait(ws_ctx* ctx, uint32_t spin_limit) {
    if (!ctx) return WS_ERR_ARG;
    if (spin_limit == 0 || spin_limit > (1u << 20))
        return set_error(ctx, WS_ERR_ARG, "ws_selftest_wait: spin_limit must be 1 to 2^20");
    cudaSetDevice(ctx->device);
    cudaError_t e;
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_error(ctx, e, "ws_selftest_wait");
    // One job of 4096 given keys whose keys items are left out of the launch:
    // its low-pass items wait for a completion count that nothing raises.
    const uint32_t n = 4096;
    LaunchShape S;
    shape_launch(&n, 1, ctx->params, ctx->sms, S);
    ctx->shape_valid = false;   // the context's scratch is reused below
    const size_t keys_bytes = 16384, out_bytes = 3 * 4 * (size_t)n + 256;
    if ((e = ctx->scratch.ensure(S.bytes + keys_bytes + out_bytes)) != cudaSuccess)
        return cuda_error(ctx, e, "ws_selftest_wait scratch");
    char* base = static_cast<char*>(ctx->scratch.p);
    uint16_t* keys = reinterpret_cast<uint16_t*>(base + S.bytes);
    uint32_t* outs = reinterpret_cast<uint32_t*>(base + S.bytes + keys_bytes);
    JobDesc d;
    std::memset(&d, 0, sizeof(d));
    d.kind = kJobKeys;
    d.keys_in = keys;
    d.order = outs;
    d.keys = outs + n;
    d.count = outs + 2 * n;
    place_job(d, n, 0, S, base);
    if ((e = ctx->jobs_d.ensure(sizeof(JobDesc))) != cudaSuccess) return cuda_error(ctx, e, "ws_selftest_wait");
    if ((e = cudaMemcpy(ctx->jobs_d.p, &d, sizeof(d), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(base, 0, S.ctl_bytes)) != cudaSuccess || (e = cudaMemset(keys, 0, keys_bytes)) != cudaSuccess)
        return cuda_error(ctx, e, "ws_selftest_wait");
    LaunchDesc L = launch_desc(ctx->jobs_d.p, 1, S, base, ctx->err_d, spin_limit, nullptr);
    L.first_phase = kPhaseLow;
    e = launch_sort(L, S.threads, 2, ctx->sms, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "ws_selftest_wait launch");
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_error(ctx, e, "ws_selftest_wait");
    return take_device_error(ctx);
}

// -------------------------------------------------------------- harmonics

// 32-bit words one splat's harmonics of `degree` take (scene/splats.js:43-47).
static uint32_t sh_words_of(int degree) {
    static const uint32_t coefficients[4] = {0, 3, 8, 15};
    return (coefficients[degree] * 3 + 1) / 2;
}

extern "C" int ws_cloud_set_harmonics(ws_cloud* c, int degree, const uint32_t* words, size_t nwords, int on_device) {
    if (!c || c->magic != kCloudMagic) return WS_ERR_ARG;
    ws_ctx* ctx = c->ctx;
    if (!c->alive) return set_error(ctx, WS_ERR_UNLOADED, "these splats were unloaded");
    if (degree < 0 || degree > 3)
        return set_error(ctx, WS_ERR_ARG, "ws_cloud_set_harmonics: degree must be 0 to 3, got %d", degree);
    cudaSetDevice(ctx->device);
    cudaError_t e;
    if (c->sh) {
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) return cuda_error(ctx, e, "ws_cloud_set_harmonics");
        cudaFree(c->sh);
        c->sh = nullptr;
        c->sh_degree = c->sh_words = 0;
    }
    if (degree == 0) return WS_OK;
    const uint32_t per = sh_words_of(degree);
    const size_t need = (size_t)c->n * per;
    if (!words || nwords < need)
        return set_error(ctx, WS_ERR_ARG, "ws_cloud_set_harmonics: %zu words for %u splats of degree %d; %zu needed",
                         nwords, c->n, degree, need);
    void* p = nullptr;
    if ((e = cudaMalloc(&p, (need + 1) * 4)) != cudaSuccess) return cuda_error(ctx, e, "ws_cloud_set_harmonics");
    // One word over, so the two-word read of the last coefficient stays inside.
    if ((e = cudaMemset(static_cast<uint32_t*>(p) + need, 0, 4)) != cudaSuccess ||
        (e = cudaMemcpy(p, words, need * 4, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice)) !=
            cudaSuccess) {
        cudaFree(p);
        return cuda_error(ctx, e, "ws_cloud_set_harmonics");
    }
    c->sh = static_cast<uint32_t*>(p);
    c->sh_degree = (uint32_t)degree;
    c->sh_words = per;
    return WS_OK;
}

extern "C" int ws_sort_batch_shaded(ws_ctx* ctx, int njobs, const ws_job* jobs, const ws_shade* shades,
                                    void* stream_p) {
    NvtxRange nvtx("ws_sort_batch_shaded");
    if (!ctx) return WS_ERR_ARG;
    if (njobs < 0 || (njobs && (!jobs || !shades)))
        return set_error(ctx, WS_ERR_ARG, "ws_sort_batch_shaded: bad job list");
    if (njobs == 0) return WS_OK;
    if (njobs > (1 << 20)) return set_error(ctx, WS_ERR_ARG, "ws_sort_batch_shaded: too many jobs");
    for (int j = 0; j < njobs; ++j) {
        int rc;
        if ((rc = check_cloud(ctx, jobs[j].cloud)) || (rc = check_view(ctx, &jobs[j].view))) return rc;
        if (!jobs[j].order || !jobs[j].count)
            return set_error(ctx, WS_ERR_ARG, "ws_sort_batch_shaded: job %d has no output", j);
        if (jobs[j].cloud->sh && !shades[j].shaded)
            return set_error(ctx, WS_ERR_ARG, "ws_sort_batch_shaded: job %d has harmonics but no shaded output", j);
    }
    cudaSetDevice(ctx->device);
    std::vector<uint32_t> ns(njobs);
    for (int j = 0; j < njobs; ++j) ns[j] = jobs[j].cloud->n;
    return launch_jobs(
        ctx, ns, njobs,
        [&](JobDesc* hj, const LaunchShape& S, char* scratch) {
            layout_jobs(hj, jobs, njobs, S, scratch);
            for (int j = 0; j < njobs; ++j) {
                const ws_cloud* c = jobs[j].cloud;
                if (!c->sh) continue;
                hj[j].sh = c->sh;
                hj[j].sh_degree = c->sh_degree;
                hj[j].sh_words = c->sh_words;
                hj[j].shaded = shades[j].shaded;
                for (int k = 0; k < 3; ++k) hj[j].eye[k] = shades[j].eye[k];
            }
        },
        stream_p ? static_cast<cudaStream_t>(stream_p) : ctx->stream);
}

// -------------------------------------------------------------- particles

// The pinned bucket of a particle depth d >= 1e-6 (render/particles.js:204):
// u32(clamp((log2(d) - -10) * 4095 / 30, 0, 4095)), each f32 operation
// separately rounded and log2 the f32 nearest the real log2 (log2l, with a
// 64-bit significand, rounded once to f32). WGSL leaves log2's accuracy to
// the implementation; this is the choice that every conforming one
// approximates.
static uint32_t particle_bucket(float d) {
    const float l = (float)log2l((long double)d);
    const float t = l - -10.0f;
    const float u = t * 4095.0f;
    const float v = u / 30.0f;
    const float c = std::fmin(std::fmax(v, 0.0f), 4095.0f);
    return (uint32_t)c;
}

// thr[b]: the least f32 depth whose bucket is b or more (thr[0] = 0). The
// bucket never decreases as the depth grows, so a depth d is in bucket b
// exactly when thr[b] <= d < thr[b + 1]; the kernel finds b by comparisons.
static const std::vector<float>& particle_thresholds() {
    static std::vector<float> thr;
    static std::once_flag once;
    std::call_once(once, [] {
        thr.assign(kParticleBuckets, 0.0f);
        uint32_t lo_bits, hi_bits;
        const float lo = 1e-6f, hi = INFINITY;
        std::memcpy(&lo_bits, &lo, 4);
        std::memcpy(&hi_bits, &hi, 4);
        for (uint32_t b = 1; b < kParticleBuckets; ++b) {
            uint32_t a = lo_bits, z = hi_bits;   // bucket(a) < b <= bucket(z)
            while (z - a > 1) {
                const uint32_t m = a + (z - a) / 2;
                float f;
                std::memcpy(&f, &m, 4);
                if (particle_bucket(f) >= b)
                    z = m;
                else
                    a = m;
            }
            std::memcpy(&thr[b], &z, 4);
        }
    });
    return thr;
}

extern "C" int ws_particle_thresholds(float* out) {
    if (!out) return WS_ERR_ARG;
    const std::vector<float>& thr = particle_thresholds();
    std::memcpy(out, thr.data(), thr.size() * sizeof(float));
    return WS_OK;
}

extern "C" int ws_sort_particles(ws_ctx* ctx, int n, const ws_emitter* emitters, void* stream_p) {
    NvtxRange nvtx("ws_sort_particles");
    if (!ctx) return WS_ERR_ARG;
    if (n < 0 || (n && !emitters)) return set_error(ctx, WS_ERR_ARG, "ws_sort_particles: bad emitter list");
    if (n == 0) return WS_OK;
    if (n > (1 << 20)) return set_error(ctx, WS_ERR_ARG, "ws_sort_particles: too many emitters");
    for (int j = 0; j < n; ++j) {
        const ws_emitter& e = emitters[j];
        if (!e.pool || !e.order || !e.count)
            return set_error(ctx, WS_ERR_ARG, "ws_sort_particles: emitter %d needs a pool, an order and a count", j);
        if (reinterpret_cast<uintptr_t>(e.pool) % 16)
            return set_error(ctx, WS_ERR_ARG, "ws_sort_particles: emitter %d's pool is not 16-byte aligned", j);
        if (e.capacity > WS_MAX_SPLATS)
            return set_error(ctx, WS_ERR_CAPACITY, "ws_sort_particles: emitter %d has %u slots, more than %u", j,
                             e.capacity, WS_MAX_SPLATS);
        if ((uint64_t)e.offset + e.capacity > 0xFFFFFFFFull)
            return set_error(ctx, WS_ERR_ARG, "ws_sort_particles: emitter %d's ring runs past slot 2^32 - 1", j);
    }
    cudaSetDevice(ctx->device);
    cudaError_t e;
    if (!ctx->thr_d.p) {
        const std::vector<float>& thr = particle_thresholds();
        if ((e = ctx->thr_d.ensure(thr.size() * sizeof(float))) != cudaSuccess)
            return cuda_error(ctx, e, "ws_sort_particles thresholds");
        if ((e = cudaMemcpy(ctx->thr_d.p, thr.data(), thr.size() * sizeof(float), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return cuda_error(ctx, e, "ws_sort_particles thresholds");
    }
    std::vector<uint32_t> ns(n);
    for (int j = 0; j < n; ++j) ns[j] = emitters[j].capacity;
    const float* thr = static_cast<const float*>(ctx->thr_d.p);
    return launch_jobs(
        ctx, ns, n,
        [&](JobDesc* hj, const LaunchShape& S, char* scratch) { layout_emitters(hj, emitters, n, S, scratch, thr); },
        stream_p ? static_cast<cudaStream_t>(stream_p) : ctx->stream);
}

// ------------------------------------------------------------------ plans

struct ws_plan {
    ws_ctx* ctx;
    int njobs;
    std::vector<ws_job> jobs;
    DevBuf scratch, jobs_d;
    HostBuf jobs_h;
    LaunchShape shape;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done = nullptr;
    int grid;
    size_t table_bytes = 0;   // the job table (and segment table) in jobs_h / jobs_d
};

extern "C" int ws_plan_create(ws_ctx* ctx, int njobs, const ws_job* jobs, ws_plan** out) {
    if (!ctx || !out) return WS_ERR_ARG;
    *out = nullptr;
    if (njobs <= 0 || !jobs) return set_error(ctx, WS_ERR_ARG, "ws_plan_create: no jobs");
    for (int j = 0; j < njobs; ++j) {
        int rc;
        if ((rc = check_cloud(ctx, jobs[j].cloud)) || (rc = check_view(ctx, &jobs[j].view))) return rc;
        if (!jobs[j].order || !jobs[j].count) return set_error(ctx, WS_ERR_ARG, "ws_plan_create: job %d has no output", j);
    }
    cudaSetDevice(ctx->device);
    uint64_t splats = 0;
    for (int j = 0; j < njobs; ++j) splats += jobs[j].cloud->n;
    const ws_params& P = params_for(ctx, splats);
    ws_plan* p = new (std::nothrow) ws_plan();
    if (!p) return set_error(ctx, WS_ERR_NOMEM, "ws_plan_create: out of host memory");
    p->ctx = ctx;
    p->njobs = njobs;
    p->jobs.assign(jobs, jobs + njobs);
    std::vector<uint32_t> ns(njobs);
    for (int j = 0; j < njobs; ++j) ns[j] = jobs[j].cloud->n;
    cudaError_t e;
    LaunchShape& S = p->shape;
    shape_launch(ns.data(), njobs, P, ctx->sms, S);
    const size_t tb = table_bytes(njobs, S);
    if ((e = p->scratch.ensure(S.bytes)) != cudaSuccess || (e = p->jobs_d.ensure(tb)) != cudaSuccess ||
        (e = p->jobs_h.ensure(tb)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming)) != cudaSuccess) {
        ws_plan_destroy(p);
        return cuda_error(ctx, e, "ws_plan_create");
    }
    JobDesc* hj = static_cast<JobDesc*>(p->jobs_h.p);
    layout_jobs(hj, jobs, njobs, S, static_cast<char*>(p->scratch.p));
    write_table(p->jobs_h.p, hj, njobs, S);
    // The job table stays in device memory (uploaded here and by
    // ws_plan_set_views); the graph resets the counters and launches.
    cudaStream_t cs;
    if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess) {
        ws_plan_destroy(p);
        return cuda_error(ctx, e, "ws_plan_create");
    }
    if ((e = cudaMemcpyAsync(p->jobs_d.p, p->jobs_h.p, tb, cudaMemcpyHostToDevice, cs)) != cudaSuccess ||
        (e = cudaStreamSynchronize(cs)) != cudaSuccess) {
        cudaStreamDestroy(cs);
        ws_plan_destroy(p);
        return cuda_error(ctx, e, "ws_plan_create upload");
    }
    p->table_bytes = tb;
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaMemsetAsync(p->scratch.p, 0, S.ctl_bytes, cs);
        const LaunchDesc L = launch_desc(p->jobs_d.p, njobs, S, static_cast<char*>(p->scratch.p), ctx->err_d,
                                         P.spin_limit, nullptr);
        if (P.algorithm != kAlgoPhases && one_cta_takes(hj, njobs))
            launch_one(L, P.algorithm, cs);
        else
            launch_sort(L, S.threads, (int)std::min<size_t>(S.grid, S.segs.size()), ctx->sms, cs);
        e = cudaStreamEndCapture(cs, &p->graph);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        ws_plan_destroy(p);
        return cuda_error(ctx, e, "ws_plan_create capture");
    }
    *out = p;
    return WS_OK;
}

extern "C" int ws_plan_set_views(ws_plan* p, const ws_view* views) {
    if (!p || !views) return WS_ERR_ARG;
    for (int j = 0; j < p->njobs; ++j) {
        int rc = check_view(p->ctx, &views[j]);
        if (rc) return rc;
    }
    cudaSetDevice(p->ctx->device);
    cudaError_t e = cudaEventSynchronize(p->done);
    if (e != cudaSuccess) return cuda_error(p->ctx, e, "ws_plan_set_views");
    JobDesc* hj = static_cast<JobDesc*>(p->jobs_h.p);
    for (int j = 0; j < p->njobs; ++j) {
        std::memcpy(hj[j].mv, views[j].model_view, sizeof(hj[j].mv));
        std::memcpy(hj[j].proj, views[j].projection, sizeof(hj[j].proj));
        hj[j].viewport[0] = views[j].viewport[0];
        hj[j].viewport[1] = views[j].viewport[1];
        hj[j].cull = views[j].cull;
        // The culling shortcuts are proved for one view: prove them again.
        view_shortcuts(views[j], p->jobs[j].cloud, &hj[j].fast_transform, &hj[j].keep_byte, &hj[j].keep_q);
        fill_view_consts(hj[j]);
        p->jobs[j].view = views[j];
    }
    // The new views go up now; no launch of the plan is in flight.
    if ((e = cudaMemcpyAsync(p->jobs_d.p, p->jobs_h.p, p->table_bytes, cudaMemcpyHostToDevice, p->ctx->stream)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(p->ctx->stream)) != cudaSuccess)
        return cuda_error(p->ctx, e, "ws_plan_set_views");
    p->ctx->h2d_bytes += p->table_bytes;
    return WS_OK;
}

extern "C" int ws_plan_launch(ws_plan* p, void* stream_p) {
    NvtxRange nvtx("ws_plan_launch");
    if (!p) return WS_ERR_ARG;
    for (int j = 0; j < p->njobs; ++j) {
        int rc = check_cloud(p->ctx, p->jobs[j].cloud);
        if (rc) return rc;
    }
    cudaSetDevice(p->ctx->device);
    cudaStream_t stream = stream_p ? static_cast<cudaStream_t>(stream_p) : p->ctx->stream;
    // One launch of a plan at a time on the device: it owns one scratch.
    cudaStreamWaitEvent(stream, p->done, 0);
    cudaError_t e = cudaGraphLaunch(p->exec, stream);
    if (e != cudaSuccess) return cuda_error(p->ctx, e, "ws_plan_launch");
    cudaEventRecord(p->done, stream);
    return WS_OK;
}

extern "C" int ws_plan_destroy(ws_plan* p) {
    if (!p) return WS_ERR_ARG;
    cudaSetDevice(p->ctx->device);
    if (p->done) {
        cudaEventSynchronize(p->done);
        cudaEventDestroy(p->done);
    }
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    p->scratch.release();
    p->jobs_d.release();
    p->jobs_h.release();
    delete p;
    return WS_OK;
}

// ------------------------------------------------------------------ buffers

extern "C" int ws_device_alloc(ws_ctx* ctx, size_t bytes, void** out) {
    if (!ctx || !out) return WS_ERR_ARG;
    cudaSetDevice(ctx->device);
    *out = nullptr;
    cudaError_t e = cudaMalloc(out, bytes ? bytes : 4);
    if (e != cudaSuccess) {
        *out = nullptr;
        return cuda_error(ctx, e, "ws_device_alloc");
    }
    return WS_OK;
}

extern "C" int ws_device_free(ws_ctx* ctx, void* ptr) {
    if (!ctx) return WS_ERR_ARG;
    if (!ptr) return WS_OK;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaFree(ptr);
    return e == cudaSuccess ? WS_OK : cuda_error(ctx, e, "ws_device_free");
}

extern "C" int ws_device_download(ws_ctx* ctx, const void* src, void* dst, size_t bytes, void* stream_p) {
    if (!ctx || (bytes && (!src || !dst))) return WS_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess && stream_p) e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream_p));
    if (e == cudaSuccess && bytes) e = cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(ctx, e, "ws_device_download");
    return take_device_error(ctx);
}

// ------------------------------------------------------------------ timing

extern "C" int ws_timing(ws_ctx* ctx, int enable) {
    if (!ctx) return WS_ERR_ARG;
    ctx->timing = enable != 0;
    ctx->timing_used = 0;
    ctx->timing_launches = 0;
    return WS_OK;
}

extern "C" int ws_copy_stats(ws_ctx* ctx, uint64_t* h2d_bytes, uint64_t* d2h_bytes, int reset) {
    if (!ctx) return WS_ERR_ARG;
    if (h2d_bytes) *h2d_bytes = ctx->h2d_bytes;
    if (d2h_bytes) *d2h_bytes = ctx->d2h_bytes;
    if (reset) ctx->h2d_bytes = ctx->d2h_bytes = 0;
    return WS_OK;
}

extern "C" int ws_timing_read(ws_ctx* ctx, double* kernel_ms, uint64_t* launches) {
    if (!ctx) return WS_ERR_ARG;
    cudaSetDevice(ctx->device);
    double total = 0.0;
    for (size_t k = 0; k < ctx->timing_used; ++k) {
        cudaError_t e = cudaEventSynchronize(ctx->timing_events[k].second);
        if (e != cudaSuccess) return cuda_error(ctx, e, "ws_timing_read");
        float ms = 0.0f;
        e = cudaEventElapsedTime(&ms, ctx->timing_events[k].first, ctx->timing_events[k].second);
        if (e != cudaSuccess) return cuda_error(ctx, e, "ws_timing_read");
        total += ms;
    }
    if (kernel_ms) *kernel_ms = total;
    if (launches) *launches = ctx->timing_launches;
    ctx->timing_used = 0;
    ctx->timing_launches = 0;
    return WS_OK;
}

// ------------------------------------------------------------------ tracing

extern "C" int ws_trace(ws_ctx* ctx, int enable) {
    if (!ctx) return WS_ERR_ARG;
    ctx->tracing = enable != 0;
    return WS_OK;
}

extern "C" int ws_trace_read(ws_ctx* ctx, ws_trace_rec* out, size_t cap, size_t* n) {
    if (!ctx || !n) return WS_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(ctx->launched);
    if (e != cudaSuccess) return cuda_error(ctx, e, "ws_trace_read");
    const size_t nseg = ctx->trace_segs.size();
    const size_t items = (kPhases - ctx->trace_first_phase) * nseg;
    *n = items;
    if (!out || cap == 0 || !ctx->trace_d.p) return WS_OK;
    std::vector<TraceRec> recs(items);
    e = cudaMemcpy(recs.data(), ctx->trace_d.p, items * sizeof(TraceRec), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(ctx, e, "ws_trace_read");
    for (size_t k = 0; k < items && k < cap; ++k) {
        out[k].claim_ns = recs[k].claim;
        out[k].start_ns = recs[k].start;
        out[k].end_ns = recs[k].end;
        const SegDesc& sd = ctx->trace_segs[k % nseg];
        out[k].job = sd.job;
        out[k].phase = ctx->trace_first_phase + (uint32_t)(k / nseg);
        out[k].segment = (uint32_t)(k % nseg);
        out[k].sm = recs[k].sm;
        for (int q = 0; q < 3; ++q) out[k].mark_ns[q] = recs[k].mark[q];
    }
    return WS_OK;
}
