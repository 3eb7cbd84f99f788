// Serving engine (bv_server_*): resident scenes, admission under an HBM
// budget, and continuous batching of render frames into persistent
// traversal launches replayed from captured CUDA graphs.
//
// No counterpart in the reference: its viewer renders one camera per frame
// (blade-volume-view/src/render.rs:145-567) and its trainer one batch per
// step.  The per-ray arithmetic is the tracer's (bv_walk.cu), so a frame
// renders bit for bit as bv_radfoam_tracer_dispatch_batch renders it.
//
// One scheduler thread owns every CUDA call after bv_server_start.  Its loop:
//   0. cancel: withdrawn requests drop their frames that are not launched;
//   1. retire: batches whose frame copies have landed, forward+backward
//      requests whose last copy has landed; a request whose outputs are all
//      on the host is done and its device buffers go back to the arena;
//   2. admit: pending requests in arrival order, while the head's buffers
//      fit in the arena (the budget left after scenes and scratch);
//   3. launch: while a batch slot is free and frames are waiting, pack
//      frames earliest-due first (frame k of a request is due k + 1 frame
//      periods after its arrival; up to max_batch_rays rays and
//      max_batch_views frames) into the slot's pinned table and replay the
//      slot's graph: table upload, work-counter reset, start cells, walk.
//      The slot's copy stream then moves each frame to its host buffer.
// Slots run on their own high-priority streams, so one batch's tail overlaps
// the next batch and a frame's blocks are scheduled ahead of training work;
// forward+backward requests run on a low-priority stream beside them, in
// launch pairs of at most train_chunk_rays work items, each short enough
// that waiting frames get the SMs between them.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "bv_internal.h"

using namespace bv;

namespace {

using Clock = std::chrono::steady_clock;

constexpr size_t kGranule = 256;
constexpr uint32_t kDefaultBatchRays = 1u << 21;  // one 1920x1080 frame (2,073,600 rays)
constexpr uint32_t kDefaultBatchViews = 256;
constexpr uint64_t kDefaultTrainRays = 16ull * 1920 * 1080;
constexpr uint32_t kDefaultTrainChunk = 1u << 19;
constexpr uint32_t kDefaultFramePeriodUs = 16000;
// Training step record of the serving engine: this many steps per ray of a
// launch pair (the replay recomputes steps past it).
constexpr uint32_t kServeRecSteps = 256;

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

bv_status sfail(bv_status code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_last_error(buf);
    return code;
}

bv_status scuda(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        return sfail(BV_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    return sfail(BV_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define SV_CUDA(call, what)                              \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return scuda(e_, what);   \
    } while (0)

// First-fit allocator over the request arena, 256-byte granules; free ranges
// are coalesced on release.
class Arena {
  public:
    void reset(size_t size) {
        size_ = size;
        used_ = peak_ = 0;
        free_.clear();
        if (size) free_[0] = size;
    }
    bool alloc(size_t bytes, size_t *off) {
        bytes = round_up(std::max<size_t>(bytes, 1), kGranule);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes, start = it->first + bytes;
            free_.erase(it);
            if (rest) free_[start] = rest;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = round_up(std::max<size_t>(bytes, 1), kGranule);
        used_ -= bytes;
        size_t start = off, len = bytes;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && next->first == off + bytes) {
            len += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == start) {
                prev->second += len;
                return;
            }
        }
        free_[start] = len;
    }
    size_t size() const { return size_; }
    size_t peak() const { return peak_; }
    size_t used() const { return used_; }

  private:
    size_t size_ = 0, used_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;
};

struct Request {
    uint64_t id = 0;
    bv_request r{};
    std::vector<bv_camera> cams;
    uint64_t rays = 0;
    size_t bytes = 0, off = 0;
    bool has_mem = false;
    float4 *out_dev = nullptr;
    float *target_dev = nullptr, *rgb_dev = nullptr, *loss_dev = nullptr;
    uint32_t frames_left = 0;
    double t_submit = 0, t_admit = -1, t_start = -1, t_done = -1;
    int status = BV_OK;
    std::string message;
    bool done = false;
    bool cancel = false;       // withdrawn: finish as soon as nothing of it is on the device
    cudaEvent_t ev = nullptr;  // forward+backward: last copy landed
};

// A frame waiting for a batch, ordered by due time (then submission order).
using FrameKey = std::pair<double, uint64_t>;
using FrameQueue = std::multimap<FrameKey, std::pair<Request *, uint32_t>>;

struct Scene {
    bv_tracer *t = nullptr;
    DeviceModel m{};
    uint32_t flags = 0;
    void *grad_block = nullptr;
    bv_grads grads{};
    size_t bytes = 0;
};

// A frame on its way to the host: its copy's event (the frame has landed
// when it completes) and the batch slot it came from.
struct Landing {
    cudaEvent_t copied = nullptr;
    Request *q = nullptr;
    uint32_t view = 0;
    uint32_t slot = 0;
};

// A batch slot: busy until its traversal is done and every frame of its
// batch has landed.  (Freeing it when the traversal ends, with the copies
// still running, lets batches be formed earlier from fewer queued frames:
// measured worse for frame latency under load, 44 vs 27 ms p99 at 50 req/s.)
struct Slot {
    cudaStream_t compute = nullptr, copy = nullptr;
    cudaEvent_t done = nullptr;
    bool computing = false;
    uint32_t copies = 0;  // frames of the batch not yet landed
    void *host_table = nullptr;  // pinned: ServeHeader + ServeView[max_views]
    void *dev_table = nullptr;
    uint32_t *counter = nullptr;
    double *partial_dist = nullptr;
    uint32_t *partial_index = nullptr;
    uint32_t *counters = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool busy = false;
    std::vector<std::pair<Request *, uint32_t>> frames;
};

}  // namespace

struct bv_server {
    bv_server_settings s{};
    int device = 0;
    Clock::time_point t0;
    std::vector<Scene> scenes;
    bool started = false;
    // device state
    void *arena_base = nullptr;
    Arena arena;
    RayState *ray_state = nullptr;
    uint32_t *step_rec = nullptr;  // training step record lent to every scene's tracer
    size_t resident = 0;
    std::vector<Slot> slots;
    std::deque<Landing> landings;           // frame copies in flight
    std::vector<cudaEvent_t> spare_events;  // their events, for reuse
    cudaStream_t train_stream = nullptr;
    ServeParams params{};
    int walk_grid = 0;
    size_t table_bytes = 0;
    // shared with submitters and waiters
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> pending;
    std::map<uint64_t, std::unique_ptr<Request>> live;
    uint64_t next_id = 1;
    bool stopping = false;
    std::string fatal;
    bv_server_stats st{};   // published copy, read under mu
    bv_server_stats wst{};  // scheduler's own counters
    std::vector<uint64_t> cancels;  // ids withdrawn since the scheduler last looked
    std::thread worker;
    // scheduler thread only
    FrameQueue frames;
    uint64_t frame_seq = 0;
    std::deque<Request *> train_inflight;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

size_t request_bytes(const bv_request &r) {
    const size_t px = (size_t)r.n_views * r.width * r.height;
    if (r.kind == BV_REQUEST_RENDER) return round_up(px * sizeof(float4), kGranule);
    size_t b = round_up(px * 3 * sizeof(float), kGranule) + kGranule;  // target, loss
    if (r.out_host) b += round_up(px * 3 * sizeof(float), kGranule);
    return b;
}

// Lays out a request's buffers in its arena range.
void place_request(bv_server *sv, Request *q) {
    char *base = static_cast<char *>(sv->arena_base) + q->off;
    const size_t px = (size_t)q->r.n_views * q->r.width * q->r.height;
    if (q->r.kind == BV_REQUEST_RENDER) {
        q->out_dev = reinterpret_cast<float4 *>(base);
        return;
    }
    size_t o = 0;
    q->target_dev = reinterpret_cast<float *>(base + o);
    o += round_up(px * 3 * sizeof(float), kGranule);
    q->loss_dev = reinterpret_cast<float *>(base + o);
    o += kGranule;
    if (q->r.out_host) q->rgb_dev = reinterpret_cast<float *>(base + o);
}

// The batch's device work: table upload, counter reset, start cells, walk.
// Captured once per slot into a graph, or issued directly.
bv_status enqueue_batch(bv_server *sv, Slot &sl, cudaStream_t s) {
    ServeParams p = sv->params;
    p.header = static_cast<const ServeHeader *>(sl.dev_table);
    p.views = reinterpret_cast<ServeView *>(static_cast<char *>(sl.dev_table) + sizeof(ServeHeader));
    p.work_counter = sl.counter;
    p.partial_dist = sl.partial_dist;
    p.partial_index = sl.partial_index;
    p.counters = sl.counters;
    SV_CUDA(cudaMemcpyAsync(sl.dev_table, sl.host_table, sv->table_bytes, cudaMemcpyHostToDevice, s),
            "batch table upload");
    SV_CUDA(cudaMemsetAsync(sl.counter, 0, sizeof(uint32_t), s), "counter reset");
    SV_CUDA(launch_serve_start_cells(p, s), "serve start-cell launch");
    SV_CUDA(launch_serve_walk(p, sv->walk_grid, s), "serve walk launch");
    return BV_OK;
}

// Copies the scheduler's counters into the published stats (mu held).
void publish(bv_server *sv) {
    bv_server_stats &o = sv->st;
    const bv_server_stats &w = sv->wst;
    o.frames_done = w.frames_done;
    o.batches = w.batches;
    o.graph_launches = w.graph_launches;
    o.kernel_launches = w.kernel_launches;
    o.admission_waits = w.admission_waits;
    o.busy_s = w.busy_s;
    o.arena_peak_bytes = sv->arena.peak();
    o.arena_used_bytes = sv->arena.used();
}

void finish_request(bv_server *sv, Request *q, double t) {
    if (q->has_mem) sv->arena.release(q->off, q->bytes);
    q->has_mem = false;
    if (q->ev) cudaEventDestroy(q->ev);
    q->ev = nullptr;
    std::lock_guard<std::mutex> lk(sv->mu);
    q->t_done = t;
    q->done = true;
    if (q->cancel && q->status == BV_OK) {
        q->status = BV_ERR_CANCELLED;
        q->message = "cancelled";
    }
    if (q->status == BV_OK) {
        sv->st.requests_done += 1;
        sv->st.rays_done += q->rays;
    }
    if (q->status == BV_ERR_CANCELLED) sv->st.requests_cancelled += 1;
    publish(sv);
    sv->cv_done.notify_all();
}

// Forward + loss + backward of an admitted request on stream s: target
// upload, the tracer's two-kernel gradient, colour and loss copies.
bv_status enqueue_train(bv_server *sv, Request *q, cudaStream_t s) {
    const bv_request &r = q->r;
    Scene &sc = sv->scenes[r.scene];
    const size_t px = (size_t)r.n_views * r.width * r.height;
    SV_CUDA(cudaMemcpyAsync(q->target_dev, r.target_host, px * 3 * sizeof(float),
                            cudaMemcpyHostToDevice, s), "target upload");
    const bv_grads *g = r.grads.d_density_dev ? &r.grads : &sc.grads;
    bv_status st = bv_forward_backward(sc.t, q->cams.data(), r.n_views, r.width, r.height,
                                       q->target_dev, &r.train, g, q->loss_dev, q->rgb_dev, s);
    if (st != BV_OK) return st;
    bv_launch_stats ls;
    if (bv_radfoam_tracer_last_stats(sc.t, &ls) == BV_OK) sv->wst.kernel_launches += ls.launches;
    if (r.out_host)
        SV_CUDA(cudaMemcpyAsync(r.out_host, q->rgb_dev, px * 3 * sizeof(float),
                                cudaMemcpyDeviceToHost, s), "colour copy");
    SV_CUDA(cudaMemcpyAsync(r.loss_host, q->loss_dev, sizeof(float), cudaMemcpyDeviceToHost, s),
            "loss copy");
    return BV_OK;
}

bv_status launch_batch(bv_server *sv, Slot &sl) {
    ServeHeader *h = static_cast<ServeHeader *>(sl.host_table);
    ServeView *views = reinterpret_cast<ServeView *>(h + 1);
    uint32_t n = 0, work = 0;
    const double t = sv->now();
    sl.frames.clear();
    while (!sv->frames.empty() && n < sv->s.max_batch_views) {
        Request *q = sv->frames.begin()->second.first;
        const uint32_t v = sv->frames.begin()->second.second;
        const uint32_t w = q->r.width, hh = q->r.height;
        const uint32_t fr = tile_padded_rays(w, hh);
        if (n > 0 && (uint64_t)work + fr > sv->s.max_batch_rays) break;
        ServeView &row = views[n];
        std::memset(&row, 0, sizeof(row));
        row.v = view_desc(q->cams[v], w, hh, work, 0);
        row.scene = q->r.scene;
        row.out = reinterpret_cast<uint64_t>(q->out_dev + (size_t)v * w * hh);
        if (q->t_start < 0) q->t_start = t;
        sl.frames.emplace_back(q, v);
        sv->frames.erase(sv->frames.begin());
        work += fr;
        ++n;
    }
    h->n_views = n;
    h->total_work = work;
    if (sv->s.use_graphs) {
        SV_CUDA(cudaGraphLaunch(sl.exec, sl.compute), "graph launch");
        sv->wst.graph_launches += 1;
    } else {
        bv_status st = enqueue_batch(sv, sl, sl.compute);
        if (st != BV_OK) return st;
    }
    sv->wst.kernel_launches += 2;
    sv->wst.batches += 1;
    SV_CUDA(cudaEventRecord(sl.done, sl.compute), "event");
    SV_CUDA(cudaStreamWaitEvent(sl.copy, sl.done, 0), "stream wait");
    // each frame lands on its own: one copy and one event per frame
    for (auto &f : sl.frames) {
        Request *q = f.first;
        const size_t px = (size_t)q->r.width * q->r.height;
        SV_CUDA(cudaMemcpyAsync(q->r.out_host + 4 * px * f.second, q->out_dev + px * f.second,
                                px * sizeof(float4), cudaMemcpyDeviceToHost, sl.copy),
                "frame copy");
        Landing ld;
        if (!sv->spare_events.empty()) {
            ld.copied = sv->spare_events.back();
            sv->spare_events.pop_back();
        } else {
            SV_CUDA(cudaEventCreateWithFlags(&ld.copied, cudaEventDisableTiming), "event");
        }
        ld.q = q;
        ld.view = f.second;
        ld.slot = (uint32_t)(&sl - sv->slots.data());
        const cudaError_t e = cudaEventRecord(ld.copied, sl.copy);
        if (e != cudaSuccess) {
            sv->spare_events.push_back(ld.copied);
            return scuda(e, "event");
        }
        sv->landings.push_back(ld);
        sl.copies += 1;
    }
    sl.frames.clear();
    sl.busy = true;
    sl.computing = true;
    return BV_OK;
}

// Marks every live request failed after a CUDA error in the scheduler.
void fail_all(bv_server *sv, const std::string &why) {
    cudaDeviceSynchronize();
    std::vector<Request *> all;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->fatal = why;
        for (auto &kv : sv->live)
            if (!kv.second->done) all.push_back(kv.second.get());
        sv->pending.clear();
    }
    for (Request *q : all) {
        q->status = BV_ERR_CUDA;
        q->message = why;
        finish_request(sv, q, sv->now());
    }
    sv->frames.clear();
    sv->train_inflight.clear();
    for (auto &sl : sv->slots) {
        sl.busy = sl.computing = false;
        sl.copies = 0;
        sl.frames.clear();
    }
    for (auto &ld : sv->landings) sv->spare_events.push_back(ld.copied);
    sv->landings.clear();
}

// Plain modes: the oldest request alone through the tracer calls, then a
// synchronize.  BV_SERVE_PLAIN renders view by view with
// bv_radfoam_tracer_dispatch (RadFoamGpuTracer::dispatch takes one camera,
// radfoam_trace.rs:106); BV_SERVE_PLAIN_BATCH renders all of a request's
// views with one bv_radfoam_tracer_dispatch_batch.
bv_status run_plain(bv_server *sv, Request *q) {
    const bv_request &r = q->r;
    Scene &sc = sv->scenes[r.scene];
    cudaStream_t s = sv->train_stream;
    q->t_start = sv->now();
    if (r.kind == BV_REQUEST_RENDER) {
        const size_t px = (size_t)r.width * r.height;
        const uint32_t per_call = sv->s.mode == BV_SERVE_PLAIN ? 1u : r.n_views;
        for (uint32_t v = 0; v < r.n_views; v += per_call) {
            bv_status st = bv_radfoam_tracer_dispatch_batch(
                sc.t, reinterpret_cast<float *>(q->out_dev + px * v), q->cams.data() + v,
                std::min(per_call, r.n_views - v), r.width, r.height, s);
            if (st != BV_OK) return st;
            bv_launch_stats ls;
            if (bv_radfoam_tracer_last_stats(sc.t, &ls) == BV_OK) sv->wst.kernel_launches += ls.launches;
        }
        SV_CUDA(cudaMemcpyAsync(r.out_host, q->out_dev, px * r.n_views * sizeof(float4),
                                cudaMemcpyDeviceToHost, s), "image copy");
    } else {
        bv_status st = enqueue_train(sv, q, s);
        if (st != BV_OK) return st;
    }
    SV_CUDA(cudaStreamSynchronize(s), "request synchronize");
    const double t = sv->now();
    if (r.frame_done_host)
        for (uint32_t v = 0; v < r.n_views; ++v) r.frame_done_host[v] = t;
    return BV_OK;
}

void scheduler(bv_server *sv) {
    cudaSetDevice(sv->device);
    const bool plain = sv->s.mode != BV_SERVE_BATCHED;
    double busy_since = -1.0;
    for (;;) {
        bool progress = false;
        // 0. withdrawn requests: drop their frames that are not launched
        std::vector<uint64_t> cancels;
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            cancels.swap(sv->cancels);
        }
        for (uint64_t id : cancels) {
            Request *q = nullptr;
            {
                std::lock_guard<std::mutex> lk(sv->mu);
                auto it = sv->live.find(id);
                if (it != sv->live.end() && !it->second->done) q = it->second.get();
            }
            if (!q || q->r.kind != BV_REQUEST_RENDER || !q->has_mem) continue;
            for (auto it = sv->frames.begin(); it != sv->frames.end();) {
                if (it->second.first == q) {
                    it = sv->frames.erase(it);
                    q->frames_left -= 1;
                } else {
                    ++it;
                }
            }
            if (q->frames_left == 0) finish_request(sv, q, sv->now());
            progress = true;
        }
        // 1. retire: traversals that are done, frames that landed, slots
        // with both
        bool failed = false;
        for (auto &sl : sv->slots) {
            if (!sl.computing) continue;
            const cudaError_t e = cudaEventQuery(sl.done);
            if (e == cudaErrorNotReady) continue;
            if (e != cudaSuccess) {
                fail_all(sv, std::string("batch: ") + cudaGetErrorString(e));
                failed = true;
                break;
            }
            sl.computing = false;
            progress = true;
        }
        for (auto it = sv->landings.begin(); !failed && it != sv->landings.end();) {
            const cudaError_t e = cudaEventQuery(it->copied);
            if (e == cudaErrorNotReady) {
                ++it;
                continue;
            }
            if (e != cudaSuccess) {
                fail_all(sv, std::string("frame copy: ") + cudaGetErrorString(e));
                break;
            }
            const double t = sv->now();
            Request *q = it->q;
            if (q->r.frame_done_host) q->r.frame_done_host[it->view] = t;
            sv->wst.frames_done += 1;
            if (--q->frames_left == 0) finish_request(sv, q, t);
            sv->slots[it->slot].copies -= 1;
            sv->spare_events.push_back(it->copied);
            it = sv->landings.erase(it);
            progress = true;
        }
        for (auto &sl : sv->slots)
            if (sl.busy && !sl.computing && sl.copies == 0) sl.busy = false;
        while (!sv->train_inflight.empty()) {
            Request *q = sv->train_inflight.front();
            const cudaError_t e = cudaEventQuery(q->ev);
            if (e == cudaErrorNotReady) break;
            sv->train_inflight.pop_front();
            if (e != cudaSuccess) {
                fail_all(sv, std::string("forward+backward: ") + cudaGetErrorString(e));
                break;
            }
            const double t = sv->now();
            if (q->r.frame_done_host)
                for (uint32_t v = 0; v < q->r.n_views; ++v) q->r.frame_done_host[v] = t;
            sv->wst.frames_done += q->r.n_views;
            finish_request(sv, q, t);
            progress = true;
        }
        // 2. admit, oldest first
        std::vector<Request *> admitted;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            const bool idle = sv->frames.empty() && sv->train_inflight.empty() &&
                              sv->landings.empty() &&
                              std::none_of(sv->slots.begin(), sv->slots.end(),
                                           [](const Slot &s) { return s.busy; });
            if (idle && busy_since >= 0) {
                sv->wst.busy_s += sv->now() - busy_since;
                busy_since = -1.0;
            }
            if (idle && sv->pending.empty()) {
                if (sv->stopping) break;
                if (!progress) sv->cv_work.wait(lk);
                continue;
            }
            const size_t admit_cap = plain ? (idle ? 1 : 0) : sv->pending.size();
            while (!sv->pending.empty() && admitted.size() < admit_cap) {
                Request *q = sv->pending.front();
                size_t off = 0;
                if (!sv->arena.alloc(q->bytes, &off)) {
                    sv->wst.admission_waits += 1;
                    break;
                }
                q->off = off;
                q->has_mem = true;
                q->t_admit = sv->now();
                sv->pending.pop_front();
                admitted.push_back(q);
            }
            publish(sv);
        }
        for (Request *q : admitted) {
            place_request(sv, q);
            if (busy_since < 0) busy_since = sv->now();
            progress = true;
            if (plain) {
                bv_status st = run_plain(sv, q);
                if (st != BV_OK) {
                    q->status = st;
                    q->message = bv_last_error();
                    cudaStreamSynchronize(sv->train_stream);
                }
                if (q->status == BV_OK) sv->wst.frames_done += q->r.n_views;
                finish_request(sv, q, sv->now());
                continue;
            }
            if (q->r.kind == BV_REQUEST_RENDER) {
                q->frames_left = q->r.n_views;
                const double period = 1e-6 * sv->s.frame_period_us;
                for (uint32_t v = 0; v < q->r.n_views; ++v)
                    sv->frames.emplace(FrameKey(q->t_submit + period * (v + 1), sv->frame_seq++),
                                       std::make_pair(q, v));
                continue;
            }
            q->t_start = sv->now();
            cudaError_t e = cudaEventCreateWithFlags(&q->ev, cudaEventDisableTiming);
            bv_status st = e == cudaSuccess ? enqueue_train(sv, q, sv->train_stream)
                                            : scuda(e, "cudaEventCreate");
            if (st == BV_OK) {
                e = cudaEventRecord(q->ev, sv->train_stream);
                if (e != cudaSuccess) st = scuda(e, "event");
            }
            if (st != BV_OK) {
                q->status = st;
                q->message = bv_last_error();
                cudaStreamSynchronize(sv->train_stream);
                finish_request(sv, q, sv->now());
                continue;
            }
            sv->train_inflight.push_back(q);
        }
        // 3. launch batches into free slots
        for (auto &sl : sv->slots) {
            if (sv->frames.empty()) break;
            if (sl.busy) continue;
            const bv_status st = launch_batch(sv, sl);
            if (st != BV_OK) {
                fail_all(sv, bv_last_error());
                break;
            }
            progress = true;
        }
        if (!progress) {
            std::unique_lock<std::mutex> lk(sv->mu);
            sv->cv_work.wait_for(lk, std::chrono::microseconds(20));
        }
    }
}

void free_server(bv_server *sv) {
    for (auto &ld : sv->landings) cudaEventDestroy(ld.copied);
    for (cudaEvent_t e : sv->spare_events) cudaEventDestroy(e);
    for (auto &sl : sv->slots) {
        if (sl.exec) cudaGraphExecDestroy(sl.exec);
        if (sl.compute) cudaStreamDestroy(sl.compute);
        if (sl.copy) cudaStreamDestroy(sl.copy);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.host_table) cudaFreeHost(sl.host_table);
        cudaFree(sl.dev_table);
        cudaFree(sl.counter);
        cudaFree(sl.partial_dist);
        cudaFree(sl.partial_index);
        cudaFree(sl.counters);
    }
    for (auto &sc : sv->scenes) {
        bv_radfoam_tracer_destroy(sc.t);
        cudaFree(sc.grad_block);
    }
    if (sv->train_stream) cudaStreamDestroy(sv->train_stream);
    cudaFree(sv->ray_state);
    cudaFree(sv->step_rec);
    cudaFree(sv->arena_base);
    delete sv;
}

}  // namespace

extern "C" {

bv_status bv_server_new(const bv_server_settings *settings, bv_server **out) {
    if (!settings || !out) return sfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    bv_server_settings s = *settings;
    if (s.mode != BV_SERVE_BATCHED && s.mode != BV_SERVE_PLAIN && s.mode != BV_SERVE_PLAIN_BATCH)
        return sfail(BV_ERR_INVALID_ARGUMENT, "unknown serving mode %u", s.mode);
    if (s.max_batch_rays == 0) s.max_batch_rays = kDefaultBatchRays;
    if (s.max_batch_views == 0) s.max_batch_views = kDefaultBatchViews;
    if (s.slots == 0) s.slots = 2;
    if (s.max_steps == 0) s.max_steps = 1024;
    if (s.max_train_rays == 0) s.max_train_rays = kDefaultTrainRays;
    if (s.train_chunk_rays == 0) s.train_chunk_rays = kDefaultTrainChunk;
    if (s.frame_period_us == 0) s.frame_period_us = kDefaultFramePeriodUs;
    if (s.train_record_steps != BV_SERVE_NO_RECORD && s.train_record_steps > kServeRecSteps)
        return sfail(BV_ERR_INVALID_ARGUMENT, "train_record_steps above %u", kServeRecSteps);
    if (s.max_batch_views > (uint32_t)kMaxServeViews)
        return sfail(BV_ERR_INVALID_ARGUMENT, "max_batch_views above %d", kMaxServeViews);
    if (s.slots > 4) return sfail(BV_ERR_INVALID_ARGUMENT, "at most 4 batch slots");
    if (s.max_batch_rays >= (1u << 31)) return sfail(BV_ERR_INVALID_ARGUMENT, "max_batch_rays too large");
    if (!(s.weight_threshold >= 0.0f)) return sfail(BV_ERR_INVALID_ARGUMENT, "weight_threshold must be >= 0");
    if (s.hbm_budget_bytes == 0) return sfail(BV_ERR_INVALID_ARGUMENT, "hbm_budget_bytes is zero");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return sfail(BV_ERR_NO_DEVICE, "no CUDA device");
    bv_server *sv = new bv_server();
    sv->s = s;
    sv->t0 = Clock::now();
    cudaGetDevice(&sv->device);
    *out = sv;
    return BV_OK;
}

bv_status bv_server_add_scene(bv_server *sv, const bv_model_desc *model, uint32_t flags,
                              uint32_t *scene_id) {
    if (!sv || !model || !scene_id) return sfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (sv->started) return sfail(BV_ERR_INVALID_ARGUMENT, "scenes are added before bv_server_start");
    if (sv->scenes.size() >= (size_t)kMaxServeScenes)
        return sfail(BV_ERR_INVALID_ARGUMENT, "at most %d scenes", kMaxServeScenes);
    if (flags & ~BV_SCENE_GRADIENTS) return sfail(BV_ERR_INVALID_ARGUMENT, "unknown scene flags");
    bv_trace_settings ts{};
    ts.max_steps = sv->s.max_steps;
    ts.weight_threshold = sv->s.weight_threshold;
    Scene sc;
    sc.flags = flags;
    bv_status st = bv_radfoam_tracer_new(model, &ts, &sc.t);
    if (st != BV_OK) return st;
    sc.m = tracer_device_model(sc.t);
    if (!sv->scenes.empty()) {
        const DeviceModel &a = sv->scenes[0].m;
        if (a.sh_degree != sc.m.sh_degree || a.bounded != sc.m.bounded || a.sh_bf16 != sc.m.sh_bf16) {
            bv_radfoam_tracer_destroy(sc.t);
            return sfail(BV_ERR_NOT_SUPPORTED,
                         "scenes of a server share SH degree, radii presence and SH storage");
        }
    }
    sc.bytes = tracer_device_bytes(sc.t);
    if (flags & BV_SCENE_GRADIENTS) {
        const size_t n = sc.m.n;
        const size_t nsh = 3 * (size_t)(sc.m.sh_degree + 1) * (sc.m.sh_degree + 1);
        const size_t b_den = round_up(n * 4, kGranule), b_sh = round_up(n * nsh * 4, kGranule);
        const size_t b_pos = round_up(n * 12, kGranule), b_rad = sc.m.bounded ? round_up(n * 4, kGranule) : 0;
        const size_t total = b_den + b_sh + b_pos + b_rad;
        cudaError_t e = cudaMalloc(&sc.grad_block, total);
        if (e == cudaSuccess) e = cudaMemset(sc.grad_block, 0, total);
        if (e != cudaSuccess) {
            bv_radfoam_tracer_destroy(sc.t);
            cudaFree(sc.grad_block);
            return scuda(e, "scene gradient tables");
        }
        char *b = static_cast<char *>(sc.grad_block);
        sc.grads.d_density_dev = reinterpret_cast<float *>(b);
        sc.grads.d_sh_dev = reinterpret_cast<float *>(b + b_den);
        sc.grads.d_positions_dev = reinterpret_cast<float *>(b + b_den + b_sh);
        sc.grads.d_radii_dev = b_rad ? reinterpret_cast<float *>(b + b_den + b_sh + b_pos) : nullptr;
        sc.bytes += total;
    }
    *scene_id = (uint32_t)sv->scenes.size();
    sv->scenes.push_back(sc);
    return BV_OK;
}

bv_status bv_server_scene_grads(bv_server *sv, uint32_t scene, bv_grads *out) {
    if (!sv || !out) return sfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (scene >= sv->scenes.size()) return sfail(BV_ERR_INVALID_ARGUMENT, "unknown scene %u", scene);
    if (!(sv->scenes[scene].flags & BV_SCENE_GRADIENTS))
        return sfail(BV_ERR_INVALID_ARGUMENT, "scene %u keeps no gradient tables", scene);
    *out = sv->scenes[scene].grads;
    return BV_OK;
}

bv_status bv_server_start(bv_server *sv) {
    if (!sv) return sfail(BV_ERR_INVALID_ARGUMENT, "null server");
    if (sv->started) return sfail(BV_ERR_INVALID_ARGUMENT, "server already started");
    if (sv->scenes.empty()) return sfail(BV_ERR_INVALID_ARGUMENT, "no scenes");
    SV_CUDA(cudaSetDevice(sv->device), "cudaSetDevice");
    const bv_server_settings &s = sv->s;
    // fixed scratch: ray state for forward+backward chunks, batch slots
    size_t resident = 0;
    for (auto &sc : sv->scenes) resident += sc.bytes;
    SV_CUDA(cudaMalloc(&sv->ray_state, sizeof(RayState) * s.max_train_rays), "ray-state scratch");
    resident += sizeof(RayState) * s.max_train_rays;
    for (auto &sc : sv->scenes) tracer_lend_ray_state(sc.t, sv->ray_state, s.max_train_rays);
    sv->table_bytes = sizeof(ServeHeader) + sizeof(ServeView) * s.max_batch_views;
    // training step record, shared by the scenes' tracers (one training
    // request runs at a time, on the training stream): train_record_steps
    // steps of every ray of a launch pair (the replay recomputes the steps
    // past them).  Automatic: kServeRecSteps within an eighth of the HBM
    // budget, none below one step per ray.
    size_t rec_words = 0;
    if (s.train_record_steps == 0) {
        rec_words = (size_t)s.train_chunk_rays * kServeRecSteps * 4;
        rec_words = std::min<size_t>(rec_words, s.hbm_budget_bytes / 8 / sizeof(uint32_t));
        if (rec_words < (size_t)s.train_chunk_rays * 4) rec_words = 0;
    } else if (s.train_record_steps != BV_SERVE_NO_RECORD) {
        rec_words = (size_t)s.train_chunk_rays * s.train_record_steps * 4;
    }
    if (rec_words) {
        SV_CUDA(cudaMalloc(&sv->step_rec, rec_words * sizeof(uint32_t)), "training step record");
        resident += rec_words * sizeof(uint32_t);
    }
    for (auto &sc : sv->scenes) {
        tracer_lend_step_record(sc.t, sv->step_rec, rec_words);
        tracer_set_train_chunk(sc.t, s.train_chunk_rays);
    }
    // frames on the highest stream priority, training on the lowest
    int prio_low = 0, prio_high = 0;
    SV_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high), "stream priorities");
    sv->slots.resize(s.slots);
    for (auto &sl : sv->slots) {
        SV_CUDA(cudaStreamCreateWithPriority(&sl.compute, cudaStreamNonBlocking, prio_high), "stream");
        SV_CUDA(cudaStreamCreateWithPriority(&sl.copy, cudaStreamNonBlocking, prio_high), "stream");
        SV_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "event");
        SV_CUDA(cudaHostAlloc(&sl.host_table, sv->table_bytes, cudaHostAllocDefault), "pinned table");
        std::memset(sl.host_table, 0, sv->table_bytes);
        SV_CUDA(cudaMalloc(&sl.dev_table, sv->table_bytes), "batch table");
        SV_CUDA(cudaMalloc(&sl.counter, sizeof(uint32_t)), "work counter");
        SV_CUDA(cudaMalloc(&sl.partial_dist, sizeof(double) * kMaxServeViews * kServeStartBlocks), "partials");
        SV_CUDA(cudaMalloc(&sl.partial_index, sizeof(uint32_t) * kMaxServeViews * kServeStartBlocks), "partials");
        SV_CUDA(cudaMalloc(&sl.counters, sizeof(uint32_t) * kMaxServeViews), "counters");
        SV_CUDA(cudaMemset(sl.counters, 0, sizeof(uint32_t) * kMaxServeViews), "counters");
        resident += 2 * sv->table_bytes + sizeof(uint32_t) * (1 + 2 * kMaxServeViews) +
                    sizeof(double) * kMaxServeViews * kServeStartBlocks;
    }
    SV_CUDA(cudaStreamCreateWithPriority(&sv->train_stream, cudaStreamNonBlocking, prio_low), "stream");
    sv->resident = resident;
    if (resident >= s.hbm_budget_bytes)
        return sfail(BV_ERR_OUT_OF_MEMORY, "HBM budget %llu below the resident %zu bytes",
                     (unsigned long long)s.hbm_budget_bytes, resident);
    size_t arena = round_up(s.hbm_budget_bytes - resident, kGranule) - kGranule;
    size_t free_b = 0, total_b = 0;
    SV_CUDA(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const size_t margin = (size_t)512 << 20;
    if (free_b > margin && arena > free_b - margin) arena = round_up(free_b - margin, kGranule) - kGranule;
    SV_CUDA(cudaMalloc(&sv->arena_base, arena), "request arena");
    sv->arena.reset(arena);
    // batch params shared by every slot
    ServeParams &p = sv->params;
    std::memset(&p, 0, sizeof(p));
    for (size_t i = 0; i < sv->scenes.size(); ++i) p.scenes[i] = sv->scenes[i].m;
    p.n_scenes = (uint32_t)sv->scenes.size();
    p.max_steps = s.max_steps;
    p.weight_threshold = s.weight_threshold;
    sv->walk_grid = serve_grid_size(sv->device);
    if (s.use_graphs) {
        for (auto &sl : sv->slots) {
            SV_CUDA(cudaStreamBeginCapture(sl.compute, cudaStreamCaptureModeThreadLocal), "capture");
            const bv_status st = enqueue_batch(sv, sl, sl.compute);
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(sl.compute, &g);
            if (st != BV_OK) {
                if (g) cudaGraphDestroy(g);
                return st;
            }
            SV_CUDA(e, "end capture");
            const cudaError_t ei = cudaGraphInstantiate(&sl.exec, g, 0);
            cudaGraphDestroy(g);
            SV_CUDA(ei, "graph instantiate");
        }
    }
    SV_CUDA(cudaDeviceSynchronize(), "server start");
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->st.arena_bytes = arena;
        sv->st.resident_bytes = resident;
    }
    sv->started = true;
    sv->worker = std::thread(scheduler, sv);
    return BV_OK;
}

bv_status bv_server_submit(bv_server *sv, const bv_request *req, uint64_t *id) {
    if (!sv || !req || !id) return sfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (!sv->started) return sfail(BV_ERR_INVALID_ARGUMENT, "server not started");
    const bv_request &r = *req;
    if (r.scene >= sv->scenes.size()) return sfail(BV_ERR_INVALID_ARGUMENT, "unknown scene %u", r.scene);
    if (r.kind != BV_REQUEST_RENDER && r.kind != BV_REQUEST_FORWARD_BACKWARD)
        return sfail(BV_ERR_INVALID_ARGUMENT, "unknown request kind %u", r.kind);
    if (r.n_views == 0 || r.n_views > (uint32_t)kMaxServeViews)
        return sfail(BV_ERR_INVALID_ARGUMENT, "n_views must be 1..%d", kMaxServeViews);
    if (r.width == 0 || r.height == 0) return sfail(BV_ERR_INVALID_ARGUMENT, "render size must be non-zero");
    if (!r.cameras) return sfail(BV_ERR_INVALID_ARGUMENT, "no cameras");
    for (uint32_t i = 0; i < r.n_views; ++i) {
        const bv_status st = validate_camera(r.cameras[i]);
        if (st != BV_OK) return st;
    }
    const uint64_t frame = tile_padded_rays(r.width, r.height);
    if (r.kind == BV_REQUEST_RENDER) {
        if (!r.out_host) return sfail(BV_ERR_INVALID_ARGUMENT, "render request without out_host");
        if (frame > sv->s.max_batch_rays)
            return sfail(BV_ERR_INVALID_ARGUMENT, "a %ux%u frame exceeds max_batch_rays", r.width, r.height);
    } else {
        if (!r.target_host || !r.loss_host)
            return sfail(BV_ERR_INVALID_ARGUMENT, "forward+backward request needs target_host and loss_host");
        if (r.train.loss != BV_LOSS_L2 && r.train.loss != BV_LOSS_L1)
            return sfail(BV_ERR_INVALID_ARGUMENT, "unknown loss %u", r.train.loss);
        if (!(r.train.max_dt > 0.0f)) return sfail(BV_ERR_INVALID_ARGUMENT, "max_dt must be positive");
        const bool own = r.grads.d_density_dev || r.grads.d_sh_dev || r.grads.d_positions_dev ||
                         r.grads.d_radii_dev;
        if (own && (!r.grads.d_density_dev || !r.grads.d_sh_dev))
            return sfail(BV_ERR_INVALID_ARGUMENT, "density and SH gradient tables are required");
        if (!own && !(sv->scenes[r.scene].flags & BV_SCENE_GRADIENTS))
            return sfail(BV_ERR_INVALID_ARGUMENT, "scene %u keeps no gradient tables; pass grads", r.scene);
        const uint64_t chunk = (uint64_t)std::min<uint32_t>(r.n_views, kMaxViewsPerLaunch) * r.width * r.height;
        if (chunk > sv->s.max_train_rays)
            return sfail(BV_ERR_INVALID_ARGUMENT, "forward+backward chunk of %llu rays above max_train_rays",
                         (unsigned long long)chunk);
    }
    const size_t bytes = request_bytes(r);
    if (bytes > sv->arena.size())
        return sfail(BV_ERR_OUT_OF_MEMORY, "request needs %zu device bytes; the arena holds %zu",
                     bytes, sv->arena.size());
    auto q = std::make_unique<Request>();
    q->r = r;
    q->cams.assign(r.cameras, r.cameras + r.n_views);
    q->r.cameras = nullptr;
    q->rays = (uint64_t)r.n_views * r.width * r.height;
    q->bytes = bytes;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (!sv->fatal.empty()) return sfail(BV_ERR_CUDA, "server failed: %s", sv->fatal.c_str());
        if (sv->stopping) return sfail(BV_ERR_INVALID_ARGUMENT, "server is stopping");
        q->id = sv->next_id++;
        q->t_submit = sv->now();
        *id = q->id;
        sv->pending.push_back(q.get());
        sv->live[q->id] = std::move(q);
    }
    sv->cv_work.notify_one();
    return BV_OK;
}

bv_status bv_server_wait(bv_server *sv, uint64_t id, double timeout_s, bv_request_result *out) {
    if (!sv || !out) return sfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->live.find(id);
    if (it == sv->live.end()) return sfail(BV_ERR_INVALID_ARGUMENT, "unknown request %llu", (unsigned long long)id);
    Request *q = it->second.get();
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                             std::chrono::duration<double>(std::max(timeout_s, 0.0)));
    while (!q->done) {
        if (sv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !q->done)
            return sfail(BV_ERR_TIMEOUT, "request %llu not finished", (unsigned long long)id);
    }
    std::memset(out, 0, sizeof(*out));
    out->id = q->id;
    out->status = q->status;
    out->kind = q->r.kind;
    out->submit_s = q->t_submit;
    out->admit_s = q->t_admit;
    out->start_s = q->t_start;
    out->done_s = q->t_done;
    out->rays = q->rays;
    std::snprintf(out->message, sizeof(out->message), "%s", q->message.c_str());
    sv->live.erase(it);
    return BV_OK;
}

bv_status bv_server_cancel(bv_server *sv, uint64_t id) {
    if (!sv) return sfail(BV_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->live.find(id);
    if (it == sv->live.end()) return sfail(BV_ERR_INVALID_ARGUMENT, "unknown request %llu", (unsigned long long)id);
    Request *q = it->second.get();
    if (q->done || q->cancel) return BV_OK;
    q->cancel = true;
    auto p = std::find(sv->pending.begin(), sv->pending.end(), q);
    if (p != sv->pending.end()) {  // not admitted: nothing of it is on the device
        sv->pending.erase(p);
        q->status = BV_ERR_CANCELLED;
        q->message = "cancelled";
        q->t_done = sv->now();
        q->done = true;
        sv->st.requests_cancelled += 1;
        sv->cv_done.notify_all();
        return BV_OK;
    }
    sv->cancels.push_back(id);
    lk.unlock();
    sv->cv_work.notify_one();
    return BV_OK;
}

bv_status bv_server_stats_get(bv_server *sv, bv_server_stats *out) {
    if (!sv || !out) return sfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    *out = sv->st;
    return BV_OK;
}

double bv_server_clock(const bv_server *sv) { return sv ? sv->now() : 0.0; }

void bv_server_destroy(bv_server *sv) {
    if (!sv) return;
    if (sv->worker.joinable()) {
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->stopping = true;
        }
        sv->cv_work.notify_all();
        sv->worker.join();
    }
    cudaDeviceSynchronize();
    free_server(sv);
}

}  // extern "C"
