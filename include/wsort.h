/*
 * wsort: the Gaussian-splat depth-key + stable counting sort of the Winding
 * engine, as a C-ABI shared library (libwsort.so) running sm_100a CUDA.
 *
 * Inputs and outputs are the reference's: 32-byte .splat records in, and for
 * each view the survivor count, the u32 permutation of splat indices (back to
 * front) and the matching 16-bit keys out. Citations are to files of the
 * reference project (winding-engine 1.9.0).
 *
 * Conventions
 *   - Every function returns WS_OK (0) or a negative WS_ERR_* code; the text
 *     of the last failure on a context is ws_last_error(ctx). Messages that
 *     have a counterpart in the reference use its wording.
 *   - Plain pointers and sizes only. `stream` is a cudaStream_t passed as
 *     void* (NULL: the context's own stream, a blocking stream, so work on
 *     the legacy default stream is ordered before it).
 *   - One context per host thread; a context's calls are not synchronised.
 *     The server object (ws_server_*) is internally synchronised.
 *   - Clouds belong to the context that made them. Output buffers belong to
 *     the caller.
 *
 * Order contract. The reference appends survivors through atomics and
 * scatters ties through atomics (src/render/splats.js:182, :218), so its order
 * within a key varies run to run. This library returns the one deterministic
 * order that the reference's own stable CPU sort gives (DrawList.sort,
 * src/render/drawlist.js:186-229, with survivors pushed in index order):
 * survivors ordered by (key ascending, splat index ascending).
 */
#ifndef WSORT_H
#define WSORT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WS_VERSION 1

enum {
    WS_OK = 0,
    WS_ERR_ARG = -1,          /* an argument is invalid (null, negative cull, ...) */
    WS_ERR_FORMAT = -2,       /* the bytes are not .splat records */
    WS_ERR_NAN = -3,          /* a splat position is not a finite number */
    WS_ERR_CAPACITY = -4,     /* more splats than one cloud holds */
    WS_ERR_CUDA = -5,         /* a CUDA runtime call failed */
    WS_ERR_NOMEM = -6,        /* device memory (or the server's budget) exhausted */
    WS_ERR_TIMEOUT = -7,      /* a bounded device-side wait expired; results invalid */
    WS_ERR_UNLOADED = -8,     /* the cloud was freed */
    WS_ERR_BUSY = -9,         /* the server's queue is full, or it is stopping */
    WS_ERR_PENDING = -10      /* ws_server_wait timed out: the request is not done yet */
};

/* Most splats one cloud holds (look-back counts are 30-bit). */
#define WS_MAX_SPLATS ((uint32_t)1 << 30)
/* Number of distinct keys: render/splats.js:64 (BUCKETS). */
#define WS_BUCKETS 65536u

typedef struct ws_ctx ws_ctx;
typedef struct ws_cloud ws_cloud;
typedef struct ws_plan ws_plan;
typedef struct ws_server ws_server;

/*
 * One view of a cloud: exactly the f32 values the reference writes into its
 * Cloud uniform for a sort (src/render/splats.js:80-92, filled at :574-587).
 * Matrices are column-major. depthMin / depthScale are not passed: the
 * library computes them from the cloud's box in FP64 as prepare does
 * (:561-582). cull is Renderer.splatCull (src/render/renderer.js:340-344):
 * 0 keeps every splat the frustum and faintness tests keep.
 */
typedef struct ws_view {
    float model_view[16];
    float projection[16];
    float viewport[2];
    float cull;
} ws_view;

/* ------------------------------------------------------------ context */

/* Replaces SplatPass.create (src/render/splats.js:418-501): a context on
 * CUDA device `device`, with its stream and scratch. */
int ws_create(ws_ctx** out, int device);
/* Replaces SplatPass.destroy (src/render/splats.js:724-727). */
int ws_destroy(ws_ctx* ctx);
/* The message of the last failure on ctx ("" if none). */
const char* ws_last_error(const ws_ctx* ctx);
/* Waits for the context's stream and reports any device-side error raised by
 * sorts queued with WS_DEVICE_OUTPUT since the last check. */
int ws_sync(ws_ctx* ctx);

/* ------------------------------------------------------------ clouds */

/*
 * Replaces parseSplats / parseSplatFile (src/scene/splats.js:60-76, :373-388)
 * followed by new Splats (src/render/splats.js:389-409): the records are
 * copied to the device, decoded there (centres, colour word, and each
 * covariance R S S^T R^T in FP64 rounded to f32, as put() computes it at
 * src/scene/splats.js:335-369) and kept resident. Refusals mirror the
 * reference: a zip, gzip, zstd .spz or .ply header (a .ply is not read by
 * this library), a length that is zero or not a multiple of 32, a position
 * that is not finite, or more than WS_MAX_SPLATS splats.
 */
int ws_cloud_from_splat(ws_ctx* ctx, const uint8_t* bytes, size_t nbytes, ws_cloud** out);
/*
 * readSplats (src/scene/splats.js:78-90): a capture in any format the
 * reference reads without help -- a binary .ply as training writes it
 * (parsePly :398-468), a gzipped .spz of version 1 to 3 (parseSpz
 * :227-303, gunzipped here on the host) or .splat records -- decoded on the
 * device into a resident cloud, with the higher harmonics a .ply or .spz
 * carries (ws_cloud_harmonics). Refused with the reference's messages:
 * a .sog (it needs an image decoder for its WebP images), a zstd .spz of
 * version 4, and every malformed header the reference refuses.
 */
int ws_cloud_load(ws_ctx* ctx, const uint8_t* bytes, size_t nbytes, ws_cloud** out);

/* A decoded image: width x height pixels of 4 bytes (red, green, blue,
 * alpha), row by row, exactly as stored -- never premultiplied, never
 * colour-managed -- what the reference's decodeImage returns. */
typedef struct ws_image {
    uint32_t width, height;
    const uint8_t* rgba;   /* width x height x 4 bytes */
} ws_image;
/* The caller's image decoder (decodeImage(bytes) -> {width, height, rgba},
 * src/scene/splats.js:81-84): decodes one image file of a bundle (a .sog's
 * lossless WebP) into *out and returns 0, or returns nonzero if it cannot.
 * The pixels must stay readable until the next call or until ws_cloud_read
 * returns. */
typedef int (*ws_decode_image)(void* user, const uint8_t* bytes, size_t nbytes, ws_image* out);
/*
 * readSplats(bytes, {decodeImage}) (src/scene/splats.js:85-92): as
 * ws_cloud_load, and a .sog -- a zip (stored or deflated entries, not zip64)
 * of meta.json (version 2) and images, readSog :127-200 -- is unzipped and
 * read on the host, its images decoded by `decode` (called with `user`),
 * and its splats decoded on the device: log-encoded positions, smallest-three
 * rotations, colour and scale codebooks, and the harmonics palette. With
 * decode NULL a .sog is refused as the reference refuses it. Every refusal
 * of readSog carries its message; where the reference would throw a
 * TypeError (a meta.json member missing), the message names the member.
 */
int ws_cloud_read(ws_ctx* ctx, const uint8_t* bytes, size_t nbytes, ws_decode_image decode, void* user,
                  ws_cloud** out);
/* The cloud's harmonics degree (0-3) and, when words is not NULL, its
 * count x ceil(3 c / 2) packed words (the layout of ws_cloud_set_harmonics). */
int ws_cloud_harmonics(const ws_cloud* cloud, int* degree, uint32_t* words);
/* As ws_cloud_from_splat for records already in device memory. */
int ws_cloud_from_device(ws_ctx* ctx, const void* device_bytes, size_t nbytes, ws_cloud** out);
/* Splats.count / .min / .max (src/render/splats.js:401-403). min/max may be NULL. */
int ws_cloud_info(const ws_cloud* cloud, uint32_t* count, double min[3], double max[3]);
/* Copies the decoded arrays to host memory: centers 4 f32 a splat (the 4th
 * holds the colour word's bits), covariances 6 f32 a splat (xx xy xz yy yz
 * zz): the `centers` / `covariances` of parseSplats. Either may be NULL. */
int ws_cloud_download(const ws_cloud* cloud, float* centers, float* covariances);
/* Replaces Splats.destroy (src/render/splats.js:411-415). */
int ws_cloud_free(ws_cloud* cloud);

/*
 * The per-cloud depth range of prepare (src/render/splats.js:561-582), in
 * FP64: *visible is 0 when the cloud is wholly behind the camera (the
 * reference skips it), else depth_min / depth_scale are the f32 values of
 * Cloud.depthMin / Cloud.depthScale.
 */
int ws_depth_range(const ws_cloud* cloud, const float model_view[16], int* visible, float* depth_min,
                   float* depth_scale);

/* ------------------------------------------------------------ sorting */

/* Output placement for ws_sort. */
#define WS_HOST_OUTPUT 0   /* order/keys/count are host memory; returns when they are filled */
#define WS_DEVICE_OUTPUT 1 /* device memory; returns once the work is queued on `stream` */

/*
 * One cloud, one view. Replaces SplatPass._encodeSort's three dispatches for
 * a cloud (makeKeys, scanCounts, place: src/render/splats.js:676-697, WGSL
 * :155-219) and its outputs: `order` (binding 6) and args.instanceCount
 * (binding 7), here `count`. order and keys (keys may be NULL) must hold the
 * cloud's count of u32; entries [0, *count) are written: order[j] is a splat
 * index, keys[j] its key (65535 - depth bucket, so the farthest first).
 * A cloud wholly behind the camera yields *count == 0. With WS_HOST_OUTPUT
 * into pinned host memory (cudaHostAlloc / cudaMallocHost, or registered),
 * the survivors are written into it by the device and the call synchronises
 * once; other host memory is filled by copies after the count is known.
 * Errors: WS_ERR_ARG for a cull that is negative or not finite, with the
 * reference's message "splatCull must be 0 or more, got <cull>"
 * (src/render/renderer.js:1529); WS_ERR_UNLOADED for a freed cloud
 * (src/render/splats.js:556).
 */
int ws_sort(ws_ctx* ctx, const ws_cloud* cloud, const ws_view* view, uint32_t* order, uint32_t* keys,
            uint32_t* count, int flags, void* stream);

/* One job of a batch: device-memory outputs, as ws_sort with WS_DEVICE_OUTPUT. */
typedef struct ws_job {
    const ws_cloud* cloud;
    ws_view view;
    uint32_t* order;
    uint32_t* keys;      /* may be NULL */
    uint32_t* count;
} ws_job;

/*
 * Many (cloud, view) jobs in one persistent launch. Replaces the per-cloud
 * loop of SplatPass._encodeSort (src/render/splats.js:678-696), which
 * dispatches three kernels per cloud. Each job's result is identical to what
 * ws_sort gives for it alone. Queued on `stream`; returns once queued.
 */
int ws_sort_batch(ws_ctx* ctx, int njobs, const ws_job* jobs, void* stream);

/*
 * ws_sort_batch with host outputs: the same one launch for all jobs, then
 * each job's survivors and count into host memory -- the loop of
 * SplatPass._encodeSort (src/render/splats.js:678-696) with the reference's
 * outputs (order, args.instanceCount) read back. jobs[j].order, .keys (may
 * be NULL) and .count are host memory; when every one is pinned
 * (cudaHostAlloc / registered), one kernel writes them all, starting on each
 * job as soon as its sort is done (so it overlaps the rest of the launch),
 * and the call synchronises once; else the counts come back first and then
 * the orders. At most 65535 jobs. Returns when the outputs are filled.
 */
int ws_sort_batch_host(ws_ctx* ctx, int njobs, const ws_job* jobs, void* stream);

/*
 * A batch frozen into a CUDA graph: the job set (clouds, output buffers) is
 * fixed at creation; views can change between launches with
 * ws_plan_set_views, which waits for the plan's previous launch to finish
 * reading them and uploads the new ones. The job table stays in device
 * memory; the graph holds the reset of the counters and the sort's launch.
 */
int ws_plan_create(ws_ctx* ctx, int njobs, const ws_job* jobs, ws_plan** out);
int ws_plan_set_views(ws_plan* plan, const ws_view* views);
int ws_plan_launch(ws_plan* plan, void* stream);
int ws_plan_destroy(ws_plan* plan);

/* ------------------------------------------------------------ device buffers */

/*
 * Device memory for per-cloud sort outputs, for callers without a CUDA
 * allocator of their own (a JavaScript host, for one). Replaces the
 * createBuffer calls of SplatPass._stateFor (src/render/splats.js:629-652):
 * the `order` buffer and the count word of `args`.
 */
int ws_device_alloc(ws_ctx* ctx, size_t bytes, void** out);
int ws_device_free(ws_ctx* ctx, void* ptr);
/* Copies `bytes` from device memory to host memory, after the context's
 * queued work (and `stream`'s, if given) has finished. */
int ws_device_download(ws_ctx* ctx, const void* device_src, void* host_dst, size_t bytes, void* stream);

/* ------------------------------------------------------------ harmonics */

/*
 * A cloud's higher spherical harmonics (a capture whose colour changes with
 * the view; src/render/splats.js:406-408): degree 1, 2 or 3, packed as the
 * reference packs them (src/scene/splats.js:43-47, :306-333): per splat,
 * ceil(3 c / 2) 32-bit words (c = 3, 8 or 15 coefficients past the
 * constant one) of half floats, coefficient by coefficient, red, green and
 * blue in each. Copied into device memory the cloud owns (host words, or
 * device words when on_device). Degree 0 drops them. WS_ERR_ARG when fewer
 * than n ceil(3 c / 2) words are given.
 */
int ws_cloud_set_harmonics(ws_cloud* cloud, int degree, const uint32_t* words, size_t nwords, int on_device);

/* The shade pass of one job: the eye in the cloud's own space (Cloud.eye,
 * src/render/splats.js:585-586) and the per-splat colour words it writes. */
typedef struct ws_shade {
    float eye[3];
    uint32_t reserved;
    uint32_t* shaded;    /* device, >= cloud count words; entries of survivors only are written */
} ws_shade;

/*
 * ws_sort_batch plus the shade pass after the sort (src/render/splats.js:
 * 691-695, shade :371-381), fused into the same launch: for every survivor
 * i of a job whose cloud has harmonics, shaded[i] = pack4x8unorm(clamp(
 * colour + harmonics(normalize(centre - eye)), 0, 1), alpha). Jobs whose
 * cloud has none are sorted only.
 */
int ws_sort_batch_shaded(ws_ctx* ctx, int njobs, const ws_job* jobs, const ws_shade* shades, void* stream);

/* ------------------------------------------------------------ particles */

/*
 * The particle sort of an alpha emitter: the live slots of its ring in the
 * particle pool, far to near. Replaces makeKeys / scanCounts / place of
 * src/render/particles.js:197-243 (one dispatch triple per emitter,
 * _encodeSort :824-850) with the same persistent sort as ws_sort_batch.
 * A slot is live unless age >= lifetime (:202); its key is
 * 4095 - bucket (:203-205), bucket = u32(clamp((log2(depth) + 10) * 4095 / 30,
 * 0, 4095)) of depth = max(dot(position - eye, forward), 1e-6), with log2
 * the f32 nearest the real log2. Slots of equal key keep slot order (the
 * reference's atomics leave them in any order).
 */
#define WS_PARTICLE_BUCKETS 4096u
typedef struct ws_emitter {
    const void* pool;    /* device, 16-byte aligned: 32-byte particles (render/particles.js:51-56):
                            position xyz f32, age f32, velocity xyz f32, lifetime f32 */
    uint32_t offset;     /* the ring's first slot in the pool (Emitter.offset) */
    uint32_t capacity;   /* slots in the ring (Emitter.capacity) */
    float eye[3];        /* camera position (View.eye, filled at :688-693) */
    float forward[3];    /* -view[2], -view[6], -view[10] (View.forward) */
    uint32_t* order;     /* device, >= capacity: the live slots (pool indices), far to near */
    uint32_t* keys;      /* device or NULL: their keys */
    uint32_t* count;     /* device: live slots (args.instanceCount) */
} ws_emitter;

/* Sorts n emitters in one launch on `stream` (NULL: the context's stream);
 * returns once queued. WS_ERR_ARG: a null pointer, an unaligned pool, a ring
 * past slot 2^32 - 1; WS_ERR_CAPACITY: a ring of more than WS_MAX_SPLATS. */
int ws_sort_particles(ws_ctx* ctx, int n, const ws_emitter* emitters, void* stream);

/* The WS_PARTICLE_BUCKETS depth thresholds the kernel compares with:
 * out[b] is the least f32 depth whose bucket is b or more (out[0] = 0).
 * Host only; needs no device. */
int ws_particle_thresholds(float* out);

/* ------------------------------------------------------------ drawing */

/*
 * The splat draw (vs / fs, src/render/splats.js:252-312) into a headless
 * image: the first *count splats of `order` (a sort's device output, far
 * first) blended, premultiplied, over `image` (device, width x height RGBA
 * f32, row 0 at the top, 16-byte aligned; its contents are the background).
 * shaded (device, or NULL): the shade pass's colour words, read in place of
 * the splats' own (the reference's SHADED pipeline). The view is the one
 * sorted for; its viewport must be width x height (1 to 4096 a side). No fog
 * and no depth test. Rasterisation and the shader's exp / log / pow are
 * pinned (the library's notes on the draw say how). Synchronises `stream`
 * once (the number of (tile, splat) pairs sizes the binning).
 */
int ws_draw(ws_ctx* ctx, const ws_cloud* cloud, const ws_view* view, const uint32_t* order, const uint32_t* count,
            const uint32_t* shaded, float* image, uint32_t width, uint32_t height, void* stream);

/* Which tiles ws_draw draws as crowded: those whose splat list holds
 * min_splats or more (a power of two; 0: none; 1: every tile with a splat;
 * default 256). A crowded tile is split into four bands of 4 rows, each with
 * its own list (the splats whose box meets it, in order) and drawn by its
 * own CTA, the fragments evaluated by most of the CTA's warps; the other
 * tiles are drawn one CTA a tile. The image is the same either way; only
 * the time differs. */
int ws_set_draw_crowded(ws_ctx* ctx, uint32_t min_splats);

/* The draw's two 256-entry tables: decodeSRGB(byte / 255) and
 * log(255 (byte / 255)), as the f32 the draw uses. Host only. */
int ws_draw_tables(float* srgb, float* reach);

/* ------------------------------------------------------------ serving */

/*
 * A request loop over resident clouds (no counterpart in the reference,
 * which sorts once per frame on its own thread). Requests
 * (cloud, view) are submitted from any thread; a dispatcher thread batches
 * whatever has arrived into one persistent launch (continuous batching),
 * admitting requests in arrival order while their device memory (outputs
 * and sort scratch) fits the budget, with up to `streams` launches in flight
 * so a batch that arrives while another runs overlaps with it on the device.
 * Each result is identical to ws_sort's for the same request.
 */
typedef struct ws_server_opts {
    size_t memory_budget;       /* device bytes for requests in flight; 0: 50% of free memory */
    int max_batch;              /* most requests per launch (0: 64) */
    uint64_t max_batch_splats;  /* most splats per launch (0: no limit) */
    int streams;                /* launches in flight at once (0: 2) */
    int queue_capacity;         /* queued requests before submit returns WS_ERR_BUSY (0: 65536) */
    int collect_us;             /* after the first request of a batch, wait this long for more (0: none) */
} ws_server_opts;

typedef struct ws_server_stats {
    uint64_t submitted, completed, failed, batches, splats;
    uint64_t admission_waits;   /* times the head request waited for memory */
    uint64_t in_flight;         /* requests admitted, not yet collected */
    uint64_t peak_bytes;        /* most device memory in use by requests */
    double p50_ms, p99_ms, mean_ms;   /* submit -> device completion */
    double mean_batch;
    uint64_t max_batch_seen;
    uint64_t overlapped_batches; /* batches launched while another was still running */
    uint64_t cancelled;         /* requests withdrawn by ws_server_cancel */
} ws_server_stats;

int ws_server_create(ws_ctx* ctx, const ws_server_opts* opts, ws_server** out);
/* Queues a request; *ticket identifies it. The cloud must stay loaded until
 * the request is collected. WS_ERR_BUSY when the queue is full; WS_ERR_NOMEM
 * when the request alone exceeds the memory budget. */
int ws_server_submit(ws_server* server, const ws_cloud* cloud, const ws_view* view, uint64_t* ticket);
/* *done = 1 once the request's result is ready. */
int ws_server_poll(ws_server* server, uint64_t ticket, int* done);
/* Waits up to timeout_ms (< 0: forever) for the request, copies its count,
 * order and keys (keys may be NULL) to host memory and releases it.
 * WS_ERR_PENDING if it is not done in time (it stays queued). */
int ws_server_wait(ws_server* server, uint64_t ticket, uint32_t* order, uint32_t* keys, uint32_t* count,
                   int timeout_ms);
/* As ws_server_wait, but the result stays in device memory, as the
 * reference's order buffer does for its draw (src/render/splats.js:716-721):
 * *order / *keys point to it until ws_server_release(ticket); *count is the
 * survivor count. */
int ws_server_result(ws_server* server, uint64_t ticket, const uint32_t** order, const uint32_t** keys,
                     uint32_t* count, int timeout_ms);
int ws_server_release(ws_server* server, uint64_t ticket);
/* Withdraws a request that is still queued (not yet in a batch): its ticket
 * is forgotten and nothing is computed for it. WS_ERR_BUSY once it has been
 * dispatched (collect it with ws_server_wait / result + release);
 * WS_ERR_ARG for an unknown ticket. No counterpart in the reference (a frame
 * there is never withdrawn). */
int ws_server_cancel(ws_server* server, uint64_t ticket);
int ws_server_get_stats(ws_server* server, ws_server_stats* out);
/* Finishes the requests in flight, drops the queued ones, stops the threads. */
int ws_server_destroy(ws_server* server);

/* ------------------------------------------------------------ without allocation */

/*
 * No counterpart in the reference (whose WebGPU path allocates its per-cloud
 * sort buffers on first use). For callers that cannot allocate device memory
 * when they sort -- a plugin whose device memory belongs to the host
 * application's pool, a frame loop that may not stall on cudaMalloc or
 * cudaFree -- this is ws_sort with WS_DEVICE_OUTPUT that allocates nothing:
 * its scratch is one fixed array in the library's device memory, held by
 * every GPU that loads the library until the process exits. It covers clouds
 * of at most WS_NOALLOC_MAX_SPLATS splats (larger ones: WS_ERR_CAPACITY).
 * The first call on a device takes the array's address (make it before any
 * stream capture). All calls share the array and keep the last call's
 * contents; calls whose GPU work overlaps (other streams or threads) race
 * and must be serialised by the caller. order, keys (may be NULL) and count
 * are device memory; the work is queued on `stream` (NULL: the cloud's
 * context's stream). A device-side wait that gave up sets *count to
 * 0xFFFFFFFF. Other errors: WS_ERR_ARG (null pointer, cull negative or not
 * finite), WS_ERR_UNLOADED, WS_ERR_CUDA.
 */
#define WS_NOALLOC_MAX_SPLATS ((uint32_t)1 << 20)
int ws_sort_noalloc(const ws_cloud* cloud, const ws_view* view, uint32_t* order, uint32_t* keys, uint32_t* count,
                    void* stream);

/* ------------------------------------------------------------ self-test */

/*
 * Failure injection for tests: the next `count` growths of the library's
 * device buffers (a context's sort scratch, job and item tables, outputs)
 * fail as if the device were out of memory, across the process. The call
 * that meets one returns WS_ERR_NOMEM and the context stays usable.
 */
int ws_inject_alloc_failures(int count);

/*
 * Failure detection, exercised: queues one job whose first phase is left out,
 * so its next phase's wait can never be satisfied, and launches it with
 * `spin_limit` polls (1 to 2^20). The wait gives up, the kernel records the
 * error and drains, and this returns WS_ERR_TIMEOUT with the message every
 * real timeout gets; the context stays usable. No counterpart in the
 * reference (its WebGPU queue has no bounded waits).
 */
int ws_selftest_wait(ws_ctx* ctx, uint32_t spin_limit);

/*
 * The same for ws_sort_noalloc: queues, on `stream` (NULL: the context's),
 * one job on the library's fixed array whose first phase is left out, with
 * `spin_limit` polls (1 to 2^20), then the check ws_sort_noalloc ends with,
 * so that the device count *count becomes 0xFFFFFFFF as after a real wait
 * that gave up. The context only names the device; its own scratch is not
 * touched. Serialise it with ws_sort_noalloc calls as those are serialised.
 */
int ws_selftest_noalloc_wait(ws_ctx* ctx, uint32_t spin_limit, uint32_t* count, void* stream);

/* ------------------------------------------------------------ tuning */

/*
 * Kernel parameters. The launch's jobs, laid end to end, are cut into about
 * segs_per_cta segments per resident CTA (0: 1), each of at least `tile`
 * splats (a multiple of 256); a segment is one work item of each phase.
 * ctas_per_sm: 1 (0 too) runs CTAs of 1024 threads, one an SM; 2 runs CTAs
 * of 512 threads, two an SM. spin_limit: polls a device-side wait makes
 * before it gives up with WS_ERR_TIMEOUT. algorithm: 0 sorts in three phases
 * (keys, low digit, high digit) over segments of every job; 1 and 2 give each
 * job one CTA that sorts it in shared memory in one kernel, by two 8-bit
 * passes (1) or by one counting pass over all 65536 keys (2) — for launches
 * whose jobs are all of splats with at most 16384 each (others, and traced
 * launches, take the three phases). The result is the same whichever runs.
 */
typedef struct ws_params {
    uint32_t tile;
    uint32_t ctas_per_sm;
    uint32_t spin_limit;
    uint32_t segs_per_cta;
    uint32_t algorithm;
} ws_params;

int ws_get_params(const ws_ctx* ctx, ws_params* out);
int ws_set_params(ws_ctx* ctx, const ws_params* params);

/*
 * A tuning table (what winding_b200/autotune.py measures): entry b applies
 * to launches whose total splat count has floor(log2) == b; entries with
 * tile == 0, and sizes past the table, use ws_set_params's parameters.
 * n <= 32 entries; n == 0 clears the table.
 */
int ws_set_tuning(ws_ctx* ctx, const ws_params* table, int n);

/* ------------------------------------------------------------ measurement */

/*
 * Kernel timing for benchmarks (the reference's GpuProfiler role,
 * src/render/timing.js:1-33): while enabled, every sort launch on ctx is
 * bracketed by CUDA events recorded on its own stream. ws_timing_read waits
 * for them and returns the summed kernel time in ms and the number of sort
 * kernels launched since the previous read (or since enabling).
 */
int ws_timing(ws_ctx* ctx, int enable);
int ws_timing_read(ws_ctx* ctx, double* kernel_ms, uint64_t* launches);

/*
 * Bytes the sort calls of ctx moved between host and device since creation
 * (or the last reset): job tables and launch parameters up; counts, error
 * words and the survivors of host-output calls down. reset != 0 zeroes both
 * after reading. Resident clouds, plans' graph uploads and device-output
 * results are not counted.
 */
int ws_copy_stats(ws_ctx* ctx, uint64_t* h2d_bytes, uint64_t* d2h_bytes, int reset);

/*
 * Work-item tracing: while enabled, each sort launch of ctx (not plans)
 * stamps every work item with the GPU's global timer when its ticket was
 * claimed, when its dependency wait ended and when it finished, and the SM
 * it ran on. ws_trace_read waits for the last launch and copies up to `cap`
 * records of it; *n receives how many it has. phase: 0 keys, 1 low-digit
 * pass, 2 high-digit pass; segment: the launch's segment the item covered.
 */
typedef struct ws_trace_rec {
    uint64_t claim_ns, start_ns, end_ns;
    uint32_t job, phase, segment, sm;
    uint64_t mark_ns[3];   /* keys: -, first sub-tile swept, last; digit passes: prefix known, first
                              sub-tile staged, last (0: none) */
} ws_trace_rec;

int ws_trace(ws_ctx* ctx, int enable);
int ws_trace_read(ws_ctx* ctx, ws_trace_rec* out, size_t cap, size_t* n);

#ifdef __cplusplus
}
#endif

#endif /* WSORT_H */
