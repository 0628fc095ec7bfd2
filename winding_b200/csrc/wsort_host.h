// Host-side state behind the opaque handles of include/wsort.h.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "wsort.h"
#include "wsort_dev.cuh"

namespace wsort {

// A named range on the calling thread's NVTX timeline (what nsys shows
// around each call); without a tool attached, a check and nothing more.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t n);
    void release();
};

struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t n);
    void release();
};

constexpr uint32_t kCloudMagic = 0x57534F52u;   // "WSOR"

int set_error(ws_ctx* ctx, int code, const char* fmt, ...);
int cuda_error(ws_ctx* ctx, cudaError_t e, const char* what);

// How one launch's jobs are cut into segments, and where its scratch lies.
struct LaunchShape {
    int threads = 1024;                 // per CTA: 1024 (one CTA an SM) or 512 (two)
    int grid = 0;                       // CTAs launched
    uint32_t chunk = 0;                 // splats a chunk covers
    bool regular = false;               // one job: the kernel computes its segments
    std::vector<SegDesc> segs;          // every segment, in launch order
    std::vector<uint32_t> nseg, seg0;   // per job
    std::vector<size_t> ctl_off;        // per job: its control region, from the scratch base
    std::vector<size_t> arr_off;        // per job: its arrays, from the scratch base
    size_t ctl_bytes = 0;               // LaunchCtl and every control region: zeroed before a launch
    size_t bytes = 0;                   // the whole scratch
};

// The launch of `njobs` jobs of ns[j] elements with parameters p on a GPU
// of `sms` SMs.
void shape_launch(const uint32_t* ns, int njobs, const ws_params& p, int sms, LaunchShape& S);
// Job j's segment fields and scratch pointers (n elements) in `scratch`.
void place_job(JobDesc& d, uint32_t n, int j, const LaunchShape& S, char* scratch);
// Bytes of the table a launch reads: the jobs, then (unless regular) the segments.
size_t table_bytes(int njobs, const LaunchShape& S);
void write_table(void* dst, const JobDesc* jobs, int njobs, const LaunchShape& S);
LaunchDesc launch_desc(const void* d_table, int njobs, const LaunchShape& S, char* scratch, uint32_t* err,
                       uint32_t spin_limit, TraceRec* trace);
cudaError_t launch_sort(const LaunchDesc& L, int threads, int grid, int sms, cudaStream_t stream);
// Whether the one-CTA sorts take these jobs (all of splats, none above kOneMax).
bool one_cta_takes(const JobDesc* jobs, int njobs);
// The one-CTA sorts (kAlgoOneRadix or kAlgoOneCount): one CTA per job.
cudaError_t launch_one(const LaunchDesc& L, uint32_t algorithm, cudaStream_t stream);
int sort_occupancy(int threads);

}  // namespace wsort

struct ws_ctx {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t staged = nullptr;     // the last upload from pinned staging finished
    cudaEvent_t launched = nullptr;   // the last launch on this context's scratch finished
    std::string err;
    ws_params params{};
    ws_params tuning[32] = {};        // per floor(log2(splats)); tile 0: unset
    int tuning_n = 0;
    wsort::DevBuf scratch, jobs_d, items_d, out_d, copy_d;
    wsort::HostBuf copy_h;            // ws_sort_batch_host: the copy table, pinned
    wsort::HostBuf jobs_h, items_h, count_h;
    uint32_t* err_d = nullptr;        // sticky device error: code, work item
    wsort::LaunchShape shape;         // the last launch's shape, reused while ns and params repeat
    std::vector<uint32_t> last_ns;
    ws_params last_params{};
    bool shape_valid = false;
    uint64_t launches = 0;
    // host <-> device bytes the sort calls moved (ws_copy_stats): job tables
    // and launch parameters up, counts, error words and survivors down
    uint64_t h2d_bytes = 0, d2h_bytes = 0;
    // kernel timing (ws_timing): event pairs recorded around each launch
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timing_events;
    size_t timing_used = 0;
    uint64_t timing_launches = 0;
    // item tracing (ws_trace): the last traced launch's records and items
    bool tracing = false;
    wsort::DevBuf trace_d;
    std::vector<wsort::SegDesc> trace_segs;
    uint32_t trace_first_phase = 0;
    int trace_grid = 0;
    std::vector<struct ws_cloud*> freed;   // freed clouds, kept as refusable handles
    wsort::DevBuf thr_d;              // particle depth thresholds, uploaded on first use
    wsort::DevBuf draw_d, pairs_d;    // ws_draw: per-splat quads and scans; (tile, splat) pairs
    uint32_t draw_crowd_min = 256;    // ws_draw: lists this long or longer take the crowded-tile kernel
    // Capture loads: two chunks of a file on their way to the device (pinned
    // host, device), each free again once its event has passed.
    wsort::HostBuf load_h[2];
    wsort::DevBuf load_d[2];
    cudaEvent_t load_done[2] = {nullptr, nullptr};
};

struct ws_cloud {
    uint32_t magic = 0;
    bool alive = false;
    ws_ctx* ctx = nullptr;
    uint32_t n = 0;
    float4* centers = nullptr;
    float2* cov = nullptr;
    int8_t* sexp = nullptr;         // per splat: max |covariance entry| <= 2^sexp
    double bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
    uint32_t* sh = nullptr;         // harmonics: sh_words packed half-float words a splat, + 1
    uint32_t sh_degree = 0;         // 0: none
    uint32_t sh_words = 0;
};
