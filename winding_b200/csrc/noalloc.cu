// ws_sort_noalloc: the plain one-cloud sort for callers that cannot allocate
// device memory when they sort.
//
// Who needs it: a host whose device memory belongs to someone else -- a
// renderer or engine plugin that must draw from the host application's own
// pool, a real-time frame loop that may not stall on cudaMalloc/cudaFree
// (both can synchronise the device), or code queued while another component
// holds the device's allocator. ws_sort grows a per-context scratch buffer
// with cudaMalloc on first use and whenever a larger cloud arrives; this entry
// point never allocates. Its scratch is one file-scope __device__ array of a
// fixed size (WS_NOALLOC_MAX_SPLATS splats' worth), which every GPU that
// loads the library holds until the process exits.
//
// Set-up: the first call on a device (with that device current) takes the
// array's device address with cudaGetSymbolAddress and keeps it; make that
// first call before any stream capture. Every call then queues three kernels
// on the stream: one that writes the job description into the array and
// clears the counters that must start at zero, the sort kernels of ws_sort
// themselves (keys, low digit, high digit), and one that turns a device-side
// error into *count = 0xFFFFFFFF. All calls share the one array, which keeps the last call's
// contents: calls whose work overlaps on the GPU (other streams, other host
// threads) race on it and must be serialised by the caller.
#include "wsort.h"
#include "wsort_dev.cuh"
#include "wsort_host.h"

#include <cmath>
#include <cstring>
#include <mutex>

namespace wsort {

void layout_jobs(JobDesc* out, const ws_job* jobs, int njobs, const LaunchShape& S, char* scratch);

namespace {

// Fixed kernel parameters of this entry point (the library's defaults).
constexpr uint32_t kMinSegment = 2048;
constexpr uint32_t kSpinLimit = 1u << 22;

// Layout of the array: the sort's scratch for one job of up to
// WS_NOALLOC_MAX_SPLATS splats (checked against the launch's shape on every
// call), then the job description and the error words.
constexpr size_t kSortBytes = 10u << 20;
constexpr size_t kJobOffset = kSortBytes;
constexpr size_t kErrOffset = kJobOffset + ((sizeof(JobDesc) + 255) / 256) * 256;
constexpr size_t kScratchBytes = kErrOffset + 256;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Writes the job description into g_scratch and clears the launch's and the
// job's counters (the first clear_bytes of the array) and the error words.
__global__ void noalloc_setup_kernel(const __grid_constant__ JobDesc desc, uint32_t clear_bytes) {
    JobDesc* job = reinterpret_cast<JobDesc*>(g_scratch + kJobOffset);
    uint32_t* err = reinterpret_cast<uint32_t*>(g_scratch + kErrOffset);
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    if (tid == 0) *job = desc;
    if (tid < 4) err[tid] = 0;
    for (uint32_t k = tid; k < clear_bytes / 4; k += stride) reinterpret_cast<uint32_t*>(g_scratch)[k] = 0;
}

// A device-side wait that gave up leaves its code in the error words; the
// caller sees it as *count == 0xFFFFFFFF.
__global__ void noalloc_check_kernel(uint32_t* count) {
    const uint32_t* err = reinterpret_cast<const uint32_t*>(g_scratch + kErrOffset);
    if (err[0] != 0) *count = 0xFFFFFFFFu;
}

// The array's device address on the current device, taken once per device.
// The address is kept for the life of the process; a cudaDeviceReset on that
// device would make it stale (this library never resets a device).
int scratch_address(int device, char** out) {
    if (device < 0 || device >= kMaxDevices) return WS_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
        if (e != cudaSuccess || !ptr) {
            cudaGetLastError();
            return WS_ERR_CUDA;
        }
        g_scratch_addr[device] = ptr;
    }
    *out = static_cast<char*>(g_scratch_addr[device]);
    return WS_OK;
}

}  // namespace
}  // namespace wsort

using namespace wsort;

extern "C" int ws_sort_noalloc(const ws_cloud* cloud, const ws_view* view, uint32_t* order, uint32_t* keys,
                               uint32_t* count, void* stream_p) {
    if (!cloud || !view || !order || !count) return WS_ERR_ARG;
    if (cloud->magic != kCloudMagic) return WS_ERR_ARG;
    if (!cloud->alive) return WS_ERR_UNLOADED;
    if (!(view->cull >= 0.0f && std::isfinite(view->cull))) return WS_ERR_ARG;
    if (cloud->n > WS_NOALLOC_MAX_SPLATS) return WS_ERR_CAPACITY;

    ws_params p{};
    p.tile = kMinSegment;
    p.ctas_per_sm = 1;
    p.spin_limit = kSpinLimit;
    p.segs_per_cta = 1;
    const uint32_t n = cloud->n;
    const int device = cloud->ctx->device;
    if (cudaSetDevice(device) != cudaSuccess) return WS_ERR_CUDA;
    LaunchShape S;
    shape_launch(&n, 1, p, cloud->ctx->sms, S);
    if (S.bytes > kSortBytes) return WS_ERR_CAPACITY;
    char* base = nullptr;
    int rc = scratch_address(device, &base);
    if (rc) return rc;
    cudaStream_t stream = stream_p ? static_cast<cudaStream_t>(stream_p) : cloud->ctx->stream;

    ws_job job;
    job.cloud = cloud;
    job.view = *view;
    job.order = order;
    job.keys = keys;
    job.count = count;
    JobDesc desc;
    layout_jobs(&desc, &job, 1, S, base);

    noalloc_setup_kernel<<<8, 256, 0, stream>>>(desc, (uint32_t)S.ctl_bytes);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        const LaunchDesc L = launch_desc(base + kJobOffset, 1, S, base, reinterpret_cast<uint32_t*>(base + kErrOffset),
                                         kSpinLimit, nullptr);
        e = launch_sort(L, S.threads, (int)std::min<size_t>(S.grid, S.segs.size()), cloud->ctx->sms, stream);
    }
    if (e == cudaSuccess) {
        noalloc_check_kernel<<<1, 1, 0, stream>>>(count);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}

extern "C" int ws_selftest_noalloc_wait(ws_ctx* ctx, uint32_t spin_limit, uint32_t* count, void* stream_p) {
    if (!ctx || !count) return WS_ERR_ARG;
    if (spin_limit == 0 || spin_limit > (1u << 20)) return WS_ERR_ARG;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return WS_ERR_CUDA;
    char* base = nullptr;
    int rc = scratch_address(ctx->device, &base);
    if (rc) return rc;
    cudaStream_t stream = stream_p ? static_cast<cudaStream_t>(stream_p) : ctx->stream;

    // One job of 4096 given keys, laid out on the array as ws_sort_noalloc
    // lays out a cloud, its keys kernel left out of the launch: the low pass's
    // items wait for a completion count that nothing raises and give up after
    // spin_limit polls. The job's keys and outputs sit after its scratch.
    ws_params p{};
    p.tile = kMinSegment;
    p.ctas_per_sm = 1;
    p.spin_limit = spin_limit;
    p.segs_per_cta = 1;
    const uint32_t n = 4096;
    LaunchShape S;
    shape_launch(&n, 1, p, ctx->sms, S);
    const size_t keys_off = (S.bytes + 255) / 256 * 256, out_off = keys_off + 2 * (size_t)n;
    if (out_off + 2 * 4 * (size_t)n > kSortBytes) return WS_ERR_CAPACITY;
    JobDesc d;
    std::memset(&d, 0, sizeof(d));
    d.kind = kJobKeys;
    d.keys_in = reinterpret_cast<const uint16_t*>(base + keys_off);
    d.order = reinterpret_cast<uint32_t*>(base + out_off);
    d.keys = d.order + n;
    d.count = count;
    place_job(d, n, 0, S, base);

    noalloc_setup_kernel<<<8, 256, 0, stream>>>(d, (uint32_t)S.ctl_bytes);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        LaunchDesc L = launch_desc(base + kJobOffset, 1, S, base, reinterpret_cast<uint32_t*>(base + kErrOffset),
                                   spin_limit, nullptr);
        L.first_phase = kPhaseLow;
        e = launch_sort(L, S.threads, 2, ctx->sms, stream);
    }
    if (e == cudaSuccess) {
        noalloc_check_kernel<<<1, 1, 0, stream>>>(count);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}
