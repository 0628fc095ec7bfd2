// The request loop of include/wsort.h (ws_server_*): continuous batching of
// sort requests over resident clouds.
//
// A dispatcher thread takes the requests that have arrived, in arrival order,
// while a launch slot is free and their device memory fits the budget; one
// persistent sort launch carries the whole batch (the same kernel and work
// list ws_sort_batch uses). With `streams` slots, a batch that forms while
// another runs is launched at once on its own stream and overlaps with it on
// the device. A completion thread waits for each launch, stamps its requests'
// latency (submit to device completion) and returns the scratch to the arena.
// Requests hold their outputs (order, keys, count) in the arena until
// ws_server_wait copies them to the caller and releases them.
#include "wsort.h"
#include "wsort_dev.cuh"
#include "wsort_host.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

namespace wsort {
size_t launch_scratch_bytes(const uint32_t* ns, int njobs, const ws_params& p, int sms);
void layout_jobs(JobDesc* out, const ws_job* jobs, int njobs, const LaunchShape& S, char* scratch);

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

size_t round256(size_t v) { return (v + 255) / 256 * 256; }

// First-fit allocator over one device allocation, in 256-byte granules.
class Arena {
   public:
    cudaError_t init(size_t bytes) {
        size_ = round256(bytes);
        const cudaError_t e = cudaMalloc(&base_, size_);
        if (e != cudaSuccess) {
            base_ = nullptr;
            return e;
        }
        free_[0] = size_;
        return cudaSuccess;
    }
    void release() {
        if (base_) cudaFree(base_);
        base_ = nullptr;
    }
    char* alloc(size_t bytes) {
        bytes = round256(bytes ? bytes : 1);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            const size_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > bytes) free_[off + bytes] = len - bytes;
            used_ += bytes;
            return base_ + off;
        }
        return nullptr;
    }
    void free(char* p, size_t bytes) {
        if (!p) return;
        bytes = round256(bytes ? bytes : 1);
        size_t off = (size_t)(p - base_);
        used_ -= bytes;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + bytes == next->first) {
            bytes += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += bytes;
                return;
            }
        }
        free_[off] = bytes;
    }
    size_t size() const { return size_; }
    size_t used() const { return used_; }

   private:
    char* base_ = nullptr;
    size_t size_ = 0, used_ = 0;
    std::map<size_t, size_t> free_;
};

struct Request {
    uint64_t ticket = 0;
    const ws_cloud* cloud = nullptr;
    ws_view view{};
    uint32_t n = 0;
    double t_submit = 0, t_done = 0;
    char* mem = nullptr;            // order, keys, count in the arena
    size_t mem_bytes = 0;
    int state = 0;                  // 0 queued, 1 in flight, 2 done, 3 failed
};

size_t output_bytes(uint32_t n) { return round256((size_t)std::max(n, 1u) * 4) * 2 + 256; }

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    uint32_t* err_d = nullptr;
    uint32_t* err_h = nullptr;      // pinned: the launch's error words, copied back before `done`
    char* h_table = nullptr;        // pinned: the job and segment table
    char* d_table = nullptr;
    size_t cap_table = 0;           // bytes, sized at creation for the largest batch
    LaunchShape shape;              // the batch in flight
    char* scratch = nullptr;        // in the arena, for the batch in flight
    size_t scratch_bytes = 0;
    std::vector<Request*> batch;
    ws_params params{};             // the batch's kernel parameters
    bool busy = false;              // holds a batch (from forming it to its completion)
    bool launched = false;          // its launch is queued and its event recorded
    uint64_t seq = 0;
};

}  // namespace
}  // namespace wsort

using namespace wsort;

struct ws_server {
    ws_ctx* ctx = nullptr;
    int device = 0, sms = 0;
    ws_params params{};
    ws_params tuning[32] = {};      // the context's tuning table when the server started
    int tuning_n = 0;
    ws_server_opts opts{};
    Arena arena;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, Request*> reqs;
    uint64_t next_ticket = 1, launch_seq = 0;
    bool stopping = false;
    std::thread dispatcher, completer;
    std::vector<double> latencies;
    ws_server_stats stats{};
    double batch_sum = 0;

    int busy_slots() const {
        int b = 0;
        for (const Slot& s : slots) b += s.busy;
        return b;
    }
};

namespace {

// Sizes a slot's table staging for `bytes` (at creation; again only if a
// batch ever needs more, which the creation-time bound rules out).
cudaError_t ensure_table(Slot& s, size_t bytes) {
    if (bytes <= s.cap_table) return cudaSuccess;
    if (s.h_table) cudaFreeHost(s.h_table);
    if (s.d_table) cudaFree(s.d_table);
    s.h_table = nullptr;
    s.d_table = nullptr;
    s.cap_table = 0;
    cudaError_t e;
    if ((e = cudaHostAlloc(reinterpret_cast<void**>(&s.h_table), bytes, cudaHostAllocDefault)) != cudaSuccess) return e;
    if ((e = cudaMalloc(reinterpret_cast<void**>(&s.d_table), bytes)) != cudaSuccess) return e;
    s.cap_table = bytes;
    return cudaSuccess;
}

// The parameters for a batch of `splats` splats: the tuning table's entry
// for floor(log2(splats)), else the context's parameters.
const ws_params& batch_params(const ws_server* S, uint64_t splats) {
    int b = 0;
    while (b < 63 && (splats >> (b + 1))) ++b;
    if (b < S->tuning_n && S->tuning[b].tile) return S->tuning[b];
    return S->params;
}

// Takes the next batch off the queue (lock held). Returns false when the
// head request must wait for memory.
bool form_batch(ws_server* S, Slot& slot) {
    const int max_batch = S->opts.max_batch;
    const uint64_t max_splats = S->opts.max_batch_splats;
    std::vector<Request*> batch;
    std::vector<uint32_t> ns;
    uint64_t splats = 0;
    for (Request* r : S->queue) {
        if ((int)batch.size() >= max_batch) break;
        if (!batch.empty() && max_splats && splats + r->n > max_splats) break;
        r->mem_bytes = output_bytes(r->n);
        r->mem = S->arena.alloc(r->mem_bytes);
        if (!r->mem) break;
        batch.push_back(r);
        ns.push_back(r->n);
        splats += r->n;
    }
    // The batch's scratch; drop requests from the end until it fits.
    while (!batch.empty()) {
        uint64_t total = 0;
        for (uint32_t v : ns) total += v;
        slot.params = batch_params(S, total);
        const size_t need = launch_scratch_bytes(ns.data(), (int)ns.size(), slot.params, S->sms);
        slot.scratch = S->arena.alloc(need);
        if (slot.scratch) {
            slot.scratch_bytes = need;
            break;
        }
        Request* r = batch.back();
        S->arena.free(r->mem, r->mem_bytes);
        r->mem = nullptr;
        batch.pop_back();
        ns.pop_back();
    }
    if (batch.empty()) return false;
    for (Request* r : batch) {
        S->queue.pop_front();
        r->state = 1;
    }
    slot.batch = std::move(batch);
    S->stats.peak_bytes = std::max<uint64_t>(S->stats.peak_bytes, S->arena.used());
    return true;
}

// Stages and launches a formed batch on its slot (no lock held).
bool launch_batch(ws_server* S, Slot& slot) {
    NvtxRange nvtx("launch_batch");
    const int nj = (int)slot.batch.size();
    std::vector<ws_job> jobs(nj);
    for (int j = 0; j < nj; ++j) {
        Request* r = slot.batch[j];
        jobs[j].cloud = r->cloud;
        jobs[j].view = r->view;
        const size_t ob = round256((size_t)std::max(r->n, 1u) * 4);
        jobs[j].order = reinterpret_cast<uint32_t*>(r->mem);
        jobs[j].keys = reinterpret_cast<uint32_t*>(r->mem + ob);
        jobs[j].count = reinterpret_cast<uint32_t*>(r->mem + 2 * ob);
    }
    // The staging of this slot's previous launch has been consumed: the slot
    // is only reused after its completion.
    const ws_params& P = slot.params;
    std::vector<uint32_t> ns(nj);
    for (int j = 0; j < nj; ++j) ns[j] = slot.batch[j]->n;
    LaunchShape& SH = slot.shape;
    shape_launch(ns.data(), nj, P, S->sms, SH);
    std::vector<JobDesc> descs(nj);
    layout_jobs(descs.data(), jobs.data(), nj, SH, slot.scratch);
    const size_t tb = table_bytes(nj, SH);
    if (ensure_table(slot, tb) != cudaSuccess) return false;
    write_table(slot.h_table, descs.data(), nj, SH);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(slot.d_table, slot.h_table, tb, cudaMemcpyHostToDevice, slot.stream)) ||
        (e = cudaMemsetAsync(slot.scratch, 0, SH.ctl_bytes, slot.stream)) ||
        (e = cudaMemsetAsync(slot.err_d, 0, 2 * sizeof(uint32_t), slot.stream)))
        return false;
    const LaunchDesc L = launch_desc(slot.d_table, nj, SH, slot.scratch, slot.err_d, P.spin_limit, nullptr);
    e = P.algorithm != kAlgoPhases && one_cta_takes(descs.data(), nj)
            ? launch_one(L, P.algorithm, slot.stream)
            : launch_sort(L, SH.threads, (int)std::min<size_t>(SH.grid, SH.segs.size()), S->sms, slot.stream);
    if (e != cudaSuccess) return false;
    // The error words come back with the batch: the completion thread reads
    // them from pinned memory once the event has passed.
    if ((e = cudaMemcpyAsync(slot.err_h, slot.err_d, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, slot.stream)))
        return false;
    return cudaEventRecord(slot.done, slot.stream) == cudaSuccess;
}

void dispatcher_loop(ws_server* S) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lock(S->mu);
    for (;;) {
        S->cv_work.wait(lock, [&] {
            return S->stopping || (!S->queue.empty() && S->busy_slots() < (int)S->slots.size());
        });
        if (S->stopping) return;
        if (S->opts.collect_us > 0 && (int)S->queue.size() < S->opts.max_batch) {
            S->cv_work.wait_for(lock, std::chrono::microseconds(S->opts.collect_us),
                                [&] { return S->stopping || (int)S->queue.size() >= S->opts.max_batch; });
            if (S->stopping) return;
        }
        Slot* slot = nullptr;
        for (Slot& s : S->slots)
            if (!s.busy) {
                slot = &s;
                break;
            }
        if (!slot) continue;
        if (!form_batch(S, *slot)) {
            // The head request waits for memory: held by launches in flight,
            // or by results not yet collected. Every release notifies cv_done.
            ++S->stats.admission_waits;
            const size_t used = S->arena.used();
            S->cv_done.wait(lock, [&] { return S->stopping || S->arena.used() < used; });
            if (S->stopping) return;
            continue;
        }
        slot->busy = true;
        slot->seq = ++S->launch_seq;
        if (S->busy_slots() > 1) ++S->stats.overlapped_batches;
        ++S->stats.batches;
        S->batch_sum += (double)slot->batch.size();
        S->stats.max_batch_seen = std::max<uint64_t>(S->stats.max_batch_seen, slot->batch.size());
        lock.unlock();
        const bool ok = launch_batch(S, *slot);
        lock.lock();
        if (!ok) {
            for (Request* r : slot->batch) {
                r->state = 3;
                ++S->stats.failed;
            }
            S->arena.free(slot->scratch, slot->scratch_bytes);
            slot->scratch = nullptr;
            slot->batch.clear();
            slot->busy = false;
            S->cv_done.notify_all();
            continue;
        }
        slot->launched = true;
        S->cv_work.notify_all();   // the completion thread
    }
}

void completer_loop(ws_server* S) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lock(S->mu);
    for (;;) {
        Slot* oldest = nullptr;
        S->cv_work.wait(lock, [&] {
            oldest = nullptr;
            for (Slot& s : S->slots)
                if (s.busy && s.launched && (!oldest || s.seq < oldest->seq)) oldest = &s;
            return oldest != nullptr || (S->stopping && S->busy_slots() == 0);   // busy, unlaunched: not yet
        });
        if (!oldest) return;
        lock.unlock();
        cudaError_t e = cudaEventSynchronize(oldest->done);
        uint32_t err[2] = {0, 0};
        if (e == cudaSuccess) {
            err[0] = oldest->err_h[0];
            err[1] = oldest->err_h[1];
        }
        const double t = now_ms();
        lock.lock();
        const bool ok = e == cudaSuccess && err[0] == 0;
        for (Request* r : oldest->batch) {
            r->t_done = t;
            r->state = ok ? 2 : 3;
            if (ok) {
                S->latencies.push_back(t - r->t_submit);
                ++S->stats.completed;
                S->stats.splats += r->n;
            } else {
                ++S->stats.failed;
            }
        }
        S->arena.free(oldest->scratch, oldest->scratch_bytes);
        oldest->scratch = nullptr;
        oldest->batch.clear();
        oldest->busy = false;
        oldest->launched = false;
        S->cv_done.notify_all();
        S->cv_work.notify_all();   // a slot is free for the dispatcher
    }
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t lo = (size_t)pos;
    const size_t hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

extern "C" int ws_server_create(ws_ctx* ctx, const ws_server_opts* opts, ws_server** out) {
    if (!ctx || !out) return WS_ERR_ARG;
    *out = nullptr;
    ws_server* S = new (std::nothrow) ws_server();
    if (!S) return WS_ERR_NOMEM;
    S->ctx = ctx;
    S->device = ctx->device;
    S->sms = ctx->sms;
    S->params = ctx->params;
    for (int b = 0; b < 32; ++b) S->tuning[b] = ctx->tuning[b];
    S->tuning_n = ctx->tuning_n;
    if (opts) S->opts = *opts;
    if (S->opts.max_batch <= 0) S->opts.max_batch = 64;
    if (S->opts.streams <= 0) S->opts.streams = 2;
    if (S->opts.queue_capacity <= 0) S->opts.queue_capacity = 65536;
    cudaSetDevice(S->device);
    if (S->opts.memory_budget == 0) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        S->opts.memory_budget = free_b / 2;
    }
    if (S->arena.init(S->opts.memory_budget) != cudaSuccess) {
        cudaGetLastError();
        delete S;
        return WS_ERR_NOMEM;
    }
    // Each slot's table staging is sized now for the largest batch, so a
    // launch never allocates (an allocation or free there would synchronise
    // the device and stall the other slot): max_batch jobs and their
    // segments, at most segs_per_cta a resident CTA plus one a job, for the
    // parameters of any launch size.
    uint32_t per_cta = std::max(1u, S->params.segs_per_cta);
    for (int b = 0; b < S->tuning_n; ++b) per_cta = std::max(per_cta, S->tuning[b].segs_per_cta);
    const size_t max_segs = (size_t)S->sms * 2 * per_cta + (size_t)S->opts.max_batch;
    const size_t table = (size_t)S->opts.max_batch * sizeof(JobDesc) + max_segs * sizeof(SegDesc);
    S->slots.resize(S->opts.streams);
    for (Slot& s : S->slots) {
        if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMalloc(&s.err_d, 16) != cudaSuccess || cudaMemset(s.err_d, 0, 16) != cudaSuccess ||
            cudaHostAlloc(reinterpret_cast<void**>(&s.err_h), 16, cudaHostAllocDefault) != cudaSuccess ||
            ensure_table(s, table) != cudaSuccess) {
            ws_server_destroy(S);
            return WS_ERR_CUDA;
        }
        s.err_h[0] = s.err_h[1] = 0;
    }
    S->dispatcher = std::thread(dispatcher_loop, S);
    S->completer = std::thread(completer_loop, S);
    *out = S;
    return WS_OK;
}

extern "C" int ws_server_submit(ws_server* S, const ws_cloud* cloud, const ws_view* view, uint64_t* ticket) {
    if (!S || !cloud || !view || !ticket) return WS_ERR_ARG;
    if (cloud->magic != kCloudMagic) return WS_ERR_ARG;
    if (!cloud->alive) return WS_ERR_UNLOADED;
    if (cloud->ctx != S->ctx) return WS_ERR_ARG;
    if (!(view->cull >= 0.0f && std::isfinite(view->cull))) return WS_ERR_ARG;
    const uint32_t n = cloud->n;
    if (output_bytes(n) + launch_scratch_bytes(&n, 1, S->params, S->sms) > S->arena.size()) return WS_ERR_NOMEM;
    Request* r = new (std::nothrow) Request();
    if (!r) return WS_ERR_NOMEM;
    r->cloud = cloud;
    r->view = *view;
    r->n = n;
    std::lock_guard<std::mutex> lock(S->mu);
    if (S->stopping || (int)S->queue.size() >= S->opts.queue_capacity) {
        delete r;
        return WS_ERR_BUSY;
    }
    r->ticket = S->next_ticket++;
    r->t_submit = now_ms();
    S->queue.push_back(r);
    S->reqs[r->ticket] = r;
    ++S->stats.submitted;
    *ticket = r->ticket;
    S->cv_work.notify_all();
    return WS_OK;
}

extern "C" int ws_server_poll(ws_server* S, uint64_t ticket, int* done) {
    if (!S || !done) return WS_ERR_ARG;
    std::lock_guard<std::mutex> lock(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return WS_ERR_ARG;
    *done = it->second->state >= 2;
    return WS_OK;
}

extern "C" int ws_server_wait(ws_server* S, uint64_t ticket, uint32_t* order, uint32_t* keys, uint32_t* count,
                              int timeout_ms) {
    if (!S || !order || !count) return WS_ERR_ARG;
    std::unique_lock<std::mutex> lock(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return WS_ERR_ARG;
    Request* r = it->second;
    auto ready = [&] { return r->state >= 2; };
    if (timeout_ms < 0)
        S->cv_done.wait(lock, ready);
    else if (!S->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready))
        return WS_ERR_PENDING;
    S->reqs.erase(it);
    lock.unlock();
    int rc = WS_OK;
    if (r->state == 3) {
        rc = WS_ERR_TIMEOUT;
    } else {
        cudaSetDevice(S->device);
        const size_t ob = round256((size_t)std::max(r->n, 1u) * 4);
        uint32_t c = 0;
        cudaError_t e = cudaMemcpy(&c, r->mem + 2 * ob, sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && c) e = cudaMemcpy(order, r->mem, (size_t)c * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && c && keys) e = cudaMemcpy(keys, r->mem + ob, (size_t)c * 4, cudaMemcpyDeviceToHost);
        *count = c;
        if (e != cudaSuccess) rc = WS_ERR_CUDA;
    }
    lock.lock();
    if (r->mem) S->arena.free(r->mem, r->mem_bytes);
    S->cv_work.notify_all();   // memory freed: the dispatcher may admit more
    S->cv_done.notify_all();
    lock.unlock();
    delete r;
    return rc;
}

extern "C" int ws_server_result(ws_server* S, uint64_t ticket, const uint32_t** order, const uint32_t** keys,
                                uint32_t* count, int timeout_ms) {
    if (!S || !order || !count) return WS_ERR_ARG;
    std::unique_lock<std::mutex> lock(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return WS_ERR_ARG;
    Request* r = it->second;
    auto ready = [&] { return r->state >= 2; };
    if (timeout_ms < 0)
        S->cv_done.wait(lock, ready);
    else if (!S->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready))
        return WS_ERR_PENDING;
    if (r->state == 3) return WS_ERR_TIMEOUT;
    const size_t ob = round256((size_t)std::max(r->n, 1u) * 4);
    char* mem = r->mem;
    lock.unlock();
    cudaSetDevice(S->device);
    uint32_t c = 0;
    if (cudaMemcpy(&c, mem + 2 * ob, sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess) return WS_ERR_CUDA;
    *order = reinterpret_cast<const uint32_t*>(mem);
    if (keys) *keys = reinterpret_cast<const uint32_t*>(mem + ob);
    *count = c;
    return WS_OK;
}

extern "C" int ws_server_cancel(ws_server* S, uint64_t ticket) {
    if (!S) return WS_ERR_ARG;
    std::lock_guard<std::mutex> lock(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return WS_ERR_ARG;
    Request* r = it->second;
    if (r->state != 0) return WS_ERR_BUSY;   // dispatched: collect it instead
    for (auto q = S->queue.begin(); q != S->queue.end(); ++q)
        if (*q == r) {
            S->queue.erase(q);
            break;
        }
    S->reqs.erase(it);
    delete r;
    ++S->stats.cancelled;
    return WS_OK;
}

extern "C" int ws_server_release(ws_server* S, uint64_t ticket) {
    if (!S) return WS_ERR_ARG;
    std::unique_lock<std::mutex> lock(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return WS_ERR_ARG;
    Request* r = it->second;
    if (r->state < 2) return WS_ERR_PENDING;
    S->reqs.erase(it);
    if (r->mem) S->arena.free(r->mem, r->mem_bytes);
    S->cv_work.notify_all();   // memory freed: the dispatcher may admit more
    S->cv_done.notify_all();
    lock.unlock();
    delete r;
    return WS_OK;
}

extern "C" int ws_server_get_stats(ws_server* S, ws_server_stats* out) {
    if (!S || !out) return WS_ERR_ARG;
    std::lock_guard<std::mutex> lock(S->mu);
    *out = S->stats;
    out->in_flight = 0;
    for (const Slot& s : S->slots) out->in_flight += s.batch.size();
    out->p50_ms = percentile(S->latencies, 0.50);
    out->p99_ms = percentile(S->latencies, 0.99);
    double sum = 0;
    for (double v : S->latencies) sum += v;
    out->mean_ms = S->latencies.empty() ? 0.0 : sum / (double)S->latencies.size();
    out->mean_batch = S->stats.batches ? S->batch_sum / (double)S->stats.batches : 0.0;
    return WS_OK;
}

extern "C" int ws_server_destroy(ws_server* S) {
    if (!S) return WS_ERR_ARG;
    {
        std::lock_guard<std::mutex> lock(S->mu);
        S->stopping = true;
        for (Request* r : S->queue) r->state = 3;
        S->queue.clear();
    }
    S->cv_work.notify_all();
    S->cv_done.notify_all();
    if (S->dispatcher.joinable()) S->dispatcher.join();
    if (S->completer.joinable()) S->completer.join();
    cudaSetDevice(S->device);
    for (Slot& s : S->slots) {
        if (s.stream) cudaStreamSynchronize(s.stream);
        if (s.done) cudaEventDestroy(s.done);
        if (s.stream) cudaStreamDestroy(s.stream);
        if (s.err_d) cudaFree(s.err_d);
        if (s.err_h) cudaFreeHost(s.err_h);
        if (s.h_table) cudaFreeHost(s.h_table);
        if (s.d_table) cudaFree(s.d_table);
    }
    for (auto& kv : S->reqs) delete kv.second;
    S->arena.release();
    delete S;
    return WS_OK;
}
