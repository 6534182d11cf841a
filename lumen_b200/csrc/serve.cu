/*
 * serve.cu - the render server declared in include/lumen_serve.h.
 *
 * Threads: one scheduler thread forms batches from the request queue and
 * launches them; one completion thread per slot waits for its slot's batch
 * (a blocking-sync event, so it sleeps), reads the batch's counters back
 * (copied to page-locked memory by the batch itself) and completes or
 * re-queues the requests. One mutex guards the queue, the slots' state,
 * the estimates, the tuner and the results; CUDA work is issued outside it.
 *
 * A slot owns a stream, a frame (batch-sized work buffers), a device rgb8
 * staging area, page-locked copies of the view table (in) and of the
 * control block and view table (out), and one captured graph per launch
 * variant. The graph holds: table upload, frame init, the persistent
 * pipeline (grids fixed; sizes read from the table), counter read-back.
 * The per-request byte copies follow the graph on the same stream.
 */
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "splat_common.cuh"
#include "../../include/lumen_serve.h"

namespace lumen {
void configure_once();
int device_sm_count();
LumenStatus map_cuda(cudaError_t e);
void launch_init(const ScratchLayout& L, unsigned char* base, const BatchHeader* hdr, const ViewDesc* v0,
                 cudaStream_t s);
void launch_pipeline(const ScratchLayout& L, unsigned char* base, const LumenRenderOptions& opt,
                     const LumenGpuFrame& f, long long n_slots, long long n_tiles, int n_views, bool persistent,
                     const LaunchConfig& lc, cudaEvent_t* ev, cudaStream_t s, bool with_composite,
                     long long n_units);

namespace {

constexpr int kVariants = 6;
const LaunchConfig kVariantTable[kVariants] = {{256, 16, 16}, {128, 16, 16}, {512, 16, 16},
                                                {256, 16, 8},  {128, 16, 8},  {512, 16, 8}};

int variant_of(int chunk, int items) {
    for (int i = 0; i < kVariants; ++i)
        if (kVariantTable[i].composite_chunk == chunk && kVariantTable[i].tile_sort_items == items) return i;
    return -1;
}

/* Tiles a batch holds unless one view alone has more: batch-wide tile ids
 * below 2^16 sort in two 8-bit digit passes, and one tile more adds a third
 * pass over every instance of the batch. That pass costs more per view than
 * the further views share (1080p views of a 1M-Gaussian scene: 0.325 ms per
 * view in a batch of 8, 65 280 tiles; 0.364 ms in a batch of 9). */
constexpr int64_t kBatchTileIds = 1ll << 16;

/* FIFO admission: the longest prefix of the queue whose sums fit. */
int admit_prefix(const int64_t* slots, const int64_t* tiles, const int64_t* inst, const int64_t* pix, int n,
                 int max_views, int64_t max_slots, int64_t max_tiles, int64_t max_inst, int64_t max_pix) {
    int64_t s = 0, t = 0, k = 0, p = 0;
    int count = 0;
    for (int i = 0; i < n && count < max_views; ++i) {
        if (s + slots[i] > max_slots || t + tiles[i] > max_tiles || k + inst[i] > max_inst || p + pix[i] > max_pix)
            break;
        s += slots[i]; t += tiles[i]; k += inst[i]; p += pix[i];
        ++count;
    }
    return count;
}

double now_ms(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

struct Request {
    uint64_t id = 0;
    int scene = 0;
    LumenViewCamera cam{};
    uint8_t* out = nullptr;
    int64_t slots = 0, tiles = 0, pixels = 0, inst_est = 0;
    LumenServeResult result{};
    bool done = false;
};
using ReqPtr = std::shared_ptr<Request>;

struct Slot {
    int index = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_end = nullptr;
    LumenGpuFrame frame{};
    ScratchLayout layout{};
    uint8_t* d_rgb8 = nullptr;
    unsigned char* h_table = nullptr;      /* page-locked view table (in) */
    unsigned char* h_back = nullptr;       /* page-locked control block + view table (out) */
    cudaGraphExec_t exec[kVariants] = {};
    /* the batch on the device */
    std::vector<ReqPtr> batch;
    int variant = 0;
    int klass = 0;
    bool busy = false;
    bool launched = false;
    cudaError_t launch_error = cudaSuccess;
    std::condition_variable cv;
    std::thread completer;
};

/* Per batch class (log2 of pixels, log2 of instances), the mean device time
 * per instance of each variant; explores each variant kExplore times, then
 * uses the best, re-trying all every kRefresh batches of the class. While
 * frozen it explores nothing: a class uses its best variant so far, or the
 * best of the nearest class that has timings, or the fallback. */
struct Tuner {
    static constexpr int kExplore = 2, kRefresh = 256;
    struct Klass { int tries[kVariants] = {}; double cost[kVariants] = {}; int batches = 0; };
    std::map<int, Klass> classes;
    bool frozen = false;
    static int best_of(const Klass& c) {
        int best = -1;
        for (int v = 0; v < kVariants; ++v)
            if (c.tries[v] && (best < 0 || c.cost[v] / c.tries[v] < c.cost[best] / c.tries[best])) best = v;
        return best;
    }
    /* the variant for a batch of the class; *exploring tells whether it is
     * an exploratory pick */
    int pick(int klass, int fallback, bool* exploring) {
        *exploring = false;
        if (frozen) {
            int best = -1, dist = 1 << 30;
            for (const auto& kv : classes) {
                const int b = best_of(kv.second);
                const int d = std::abs(kv.first - klass);
                if (b >= 0 && d < dist) { best = b; dist = d; }
            }
            return best >= 0 ? best : fallback;
        }
        Klass& c = classes[klass];
        const int round = c.batches % kRefresh;
        if (round < kExplore * kVariants) {
            *exploring = true;
            return round % kVariants;
        }
        const int best = best_of(c);
        return best >= 0 ? best : fallback;
    }
    void record(int klass, int variant, double cost) {
        if (frozen) return;
        Klass& c = classes[klass];
        c.batches++;
        if (c.batches % kRefresh == 1) {   /* a new exploration round forgets old timings */
            std::memset(c.tries, 0, sizeof(c.tries));
            std::memset(c.cost, 0, sizeof(c.cost));
        }
        c.tries[variant]++;
        c.cost[variant] += cost;
    }
};

int log2_bucket(int64_t x) {
    int b = 0;
    while (x > 1 && b < 62) { x >>= 1; ++b; }
    return b;
}

}  // namespace
}  // namespace lumen

using namespace lumen;

struct LumenServer {
    LumenServerConfig cfg{};
    int device = 0;
    int sms = 148;
    std::chrono::steady_clock::time_point t0;
    int64_t max_slots = 0, max_tiles = 0, max_inst = 0, max_pix = 0, slot_bytes = 0;
    std::vector<LumenGpuGaussians> scenes;
    std::vector<std::unique_ptr<Slot>> slots;
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<ReqPtr> queue;
    std::unordered_map<uint64_t, ReqPtr> requests;
    std::map<std::tuple<int, int, int>, int64_t> observed;   /* (scene, W, H) -> max instances seen */
    Tuner tuner;
    LumenServeStats stats{};
    uint64_t next_id = 1;
    bool stop = false;
    std::thread scheduler;

    /* Instances a request is expected to make: the most seen for its scene
     * and resolution plus a quarter, or a first guess from the scene size
     * (about 8 tiles per Gaussian at 1080 lines, growing with the square of
     * the height). */
    int64_t estimate(int scene, const LumenViewCamera& cam) const {
        auto it = observed.find(std::make_tuple(scene, cam.width, cam.height));
        if (it != observed.end()) return it->second + it->second / 4 + 4096;
        const double h = (double)cam.height / 1080.0;
        const double f = std::max(0.5, h * h);
        return (int64_t)(8.0 * f * (double)scenes[(size_t)scene].count) + 65536;
    }
    /* The least it can make as far as is known (the most seen, no margin). */
    int64_t estimate_floor(int scene, const LumenViewCamera& cam) const {
        auto it = observed.find(std::make_tuple(scene, cam.width, cam.height));
        return it != observed.end() ? it->second : 0;
    }
};

namespace {

void free_slot(Slot* s) {
    for (int v = 0; v < kVariants; ++v)
        if (s->exec[v]) cudaGraphExecDestroy(s->exec[v]);
    LumenGpuFrame& f = s->frame;
    cudaFree(f.records); cudaFree(f.visible_ids); cudaFree(f.rects);
    for (int b = 0; b < 2; ++b) {
        cudaFree(f.depth_keys[b]); cudaFree(f.depth_order[b]); cudaFree(f.keys[b]); cudaFree(f.vals[b]);
    }
    cudaFree(f.ranges); cudaFree(f.scratch); cudaFree(s->d_rgb8);
    cudaFreeHost(s->h_table); cudaFreeHost(s->h_back);
    if (s->ev_start) cudaEventDestroy(s->ev_start);
    if (s->ev_end) cudaEventDestroy(s->ev_end);
    if (s->stream) cudaStreamDestroy(s->stream);
}

cudaError_t alloc_slot(LumenServer* srv, Slot* s) {
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&s->ev_start, cudaEventDefault)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&s->ev_end, cudaEventBlockingSync)) != cudaSuccess) return e;
    const int64_t S = srv->max_slots, K = srv->max_inst;
    LumenGpuFrame& f = s->frame;
    if ((e = cudaMalloc(&f.records, S * sizeof(LumenSplatRecord))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&f.visible_ids, S * sizeof(uint32_t))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&f.rects, S * sizeof(uint64_t))) != cudaSuccess) return e;
    for (int b = 0; b < 2; ++b) {
        if ((e = cudaMalloc(&f.depth_keys[b], S * sizeof(uint32_t))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&f.depth_order[b], S * sizeof(uint32_t))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&f.keys[b], K * sizeof(uint32_t))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&f.vals[b], K * sizeof(uint32_t))) != cudaSuccess) return e;
    }
    f.radii = nullptr;
    f.instance_capacity = K;
    if ((e = cudaMalloc(&f.ranges, srv->max_tiles * 2 * sizeof(int32_t))) != cudaSuccess) return e;
    s->layout = ScratchLayout::make(S, K, srv->cfg.max_views_per_batch);
    f.scratch_bytes = s->layout.total;
    if ((e = cudaMalloc(&f.scratch, f.scratch_bytes)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s->d_rgb8, srv->max_pix * 3)) != cudaSuccess) return e;
    const size_t tb = view_table_bytes(srv->cfg.max_views_per_batch);
    if ((e = cudaHostAlloc(&s->h_table, tb, cudaHostAllocDefault)) != cudaSuccess) return e;
    if ((e = cudaHostAlloc(&s->h_back, sizeof(Control) + tb, cudaHostAllocDefault)) != cudaSuccess) return e;
    std::memset(s->h_table, 0, tb);
    std::memset(s->h_back, 0, sizeof(Control) + tb);
    return cudaSuccess;
}

/* The batch's work on the slot's stream, up to the counter read-back. */
void enqueue_batch_work(LumenServer* srv, Slot* s, const LaunchConfig& lc, bool persistent, long long n_slots,
                        long long n_tiles, int n_views, size_t table_bytes, long long n_units) {
    unsigned char* base = (unsigned char*)s->frame.scratch;
    cudaMemcpyAsync(base + s->layout.table_off, s->h_table, table_bytes, cudaMemcpyHostToDevice, s->stream);
    {
        /* batches in flight share the GPU: plain launches (see ChainedLaunches) */
        ChainedLaunches plain(false);
        launch_init(s->layout, base, nullptr, nullptr, s->stream);
        launch_pipeline(s->layout, base, srv->cfg.options, s->frame, n_slots, n_tiles, n_views, persistent, lc,
                        nullptr, s->stream, true, n_units);
    }
    cudaMemcpyAsync(s->h_back, base + s->layout.control_off, sizeof(Control), cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(s->h_back + sizeof(Control), base + s->layout.table_off, table_bytes, cudaMemcpyDeviceToHost,
                    s->stream);
}

cudaError_t capture(LumenServer* srv, Slot* s, int variant) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    enqueue_batch_work(srv, s, kVariantTable[variant], true, srv->max_slots, srv->max_tiles, 0,
                       view_table_bytes(srv->cfg.max_views_per_batch), 0);
    e = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(&s->exec[variant], g, 0);
    cudaGraphDestroy(g);
    return e;
}

/* Fill the slot's page-locked view table for its batch; returns the
 * batch's projection slots, tiles and projection units (views of one scene
 * share their units). */
void build_table(LumenServer* srv, Slot* s, long long* n_slots, long long* n_tiles, long long* n_units) {
    ViewTable* vt = (ViewTable*)s->h_table;
    long long blocks = 0, tiles = 0, pix = 0;
    const int nv = (int)s->batch.size();
    for (int v = 0; v < nv; ++v) {
        const Request& r = *s->batch[(size_t)v];
        ViewDesc& d = vt->view[v];
        std::memset(&d, 0, sizeof(d));
        d.g = srv->scenes[(size_t)r.scene];
        d.cam = r.cam;
        d.tiles_x = (r.cam.width + kTile - 1) / kTile;
        d.img.rgb8 = s->d_rgb8 + pix * 3;
        d.block_begin = blocks;
        d.tile_begin = tiles;
        d.inst_begin = -1;
        blocks += (d.g.count + kProjThreads - 1) / kProjThreads;
        tiles += r.tiles;
        pix += r.pixels;
    }
    std::memset(&vt->hdr, 0, sizeof(vt->hdr));
    vt->hdr.n_views = nv;
    vt->hdr.total_blocks = blocks;
    vt->hdr.total_tiles = tiles;
    vt->hdr.total_units = assign_scene_groups(vt->view, nv);
    *n_slots = blocks * kProjThreads;
    *n_tiles = tiles;
    *n_units = vt->hdr.total_units;
}

/* Scheduler-thread side of a launch (no lock held). */
cudaError_t launch_batch(LumenServer* srv, Slot* s) {
    cudaSetDevice(srv->device);
    long long n_slots = 0, n_tiles = 0, n_units = 0;
    build_table(srv, s, &n_slots, &n_tiles, &n_units);
    const LaunchConfig lc = kVariantTable[s->variant];
    cudaError_t e = cudaEventRecord(s->ev_start, s->stream);
    if (e != cudaSuccess) return e;
    if (srv->cfg.use_graphs) {
        if (!s->exec[s->variant] && (e = capture(srv, s, s->variant)) != cudaSuccess) return e;
        if ((e = cudaGraphLaunch(s->exec[s->variant], s->stream)) != cudaSuccess) return e;
    } else {
        enqueue_batch_work(srv, s, lc, false, n_slots, n_tiles, (int)s->batch.size(),
                           view_table_bytes((int)s->batch.size()), n_units);
    }
    long long pix = 0;
    for (const ReqPtr& r : s->batch) {
        if (r->out && (e = cudaMemcpyAsync(r->out, s->d_rgb8 + pix * 3, (size_t)r->pixels * 3,
                                           cudaMemcpyDeviceToHost, s->stream)) != cudaSuccess)
            return e;
        pix += r->pixels;
    }
    if ((e = cudaEventRecord(s->ev_end, s->stream)) != cudaSuccess) return e;
    return cudaGetLastError();
}

void complete(LumenServer* srv, const ReqPtr& r, int status) {
    r->result.status = status;
    r->result.done_ms = now_ms(srv->t0);
    r->done = true;
    srv->stats.completed++;
}

void scheduler_main(LumenServer* srv) {
    cudaSetDevice(srv->device);
    std::unique_lock<std::mutex> lk(srv->mu);
    for (;;) {
        Slot* free_slot = nullptr;
        srv->cv_sched.wait(lk, [&] {
            if (srv->stop) return true;
            if (srv->queue.empty()) return false;
            for (auto& s : srv->slots)
                if (!s->busy) { free_slot = s.get(); return true; }
            return false;
        });
        if (srv->stop) break;
        /* admission */
        const int n = (int)std::min<size_t>(srv->queue.size(), (size_t)srv->cfg.max_views_per_batch);
        std::vector<int64_t> sl(n), ti(n), in(n), px(n);
        for (int i = 0; i < n; ++i) {
            Request& r = *srv->queue[(size_t)i];
            r.inst_est = srv->estimate(r.scene, r.cam);
            sl[i] = r.slots; ti[i] = r.tiles; in[i] = r.inst_est; px[i] = r.pixels;
        }
        int k = admit_prefix(sl.data(), ti.data(), in.data(), px.data(), n, srv->cfg.max_views_per_batch,
                             srv->max_slots, std::min<int64_t>(srv->max_tiles, kBatchTileIds), srv->max_inst,
                             srv->max_pix);
        if (k == 0 && ti[0] > kBatchTileIds)   /* a view of more tiles than that goes alone */
            k = admit_prefix(sl.data(), ti.data(), in.data(), px.data(), 1, 1, srv->max_slots, srv->max_tiles,
                             srv->max_inst, srv->max_pix);
        if (k == 0) {
            /* the front request does not fit with its margin: run it alone if
             * what it is known to need fits (an overflow raises the figure) */
            Request& r = *srv->queue.front();
            const int64_t floor = srv->estimate_floor(r.scene, r.cam);
            if (r.slots <= srv->max_slots && r.tiles <= srv->max_tiles && r.pixels <= srv->max_pix &&
                floor <= srv->max_inst) {
                r.inst_est = std::max<int64_t>(floor, 1);
                k = 1;
            }
        }
        if (k == 0) {   /* the front request can never fit an empty slot */
            ReqPtr r = srv->queue.front();
            srv->queue.pop_front();
            srv->stats.rejected++;
            complete(srv, r, LUMEN_ERROR_OUT_OF_MEMORY);
            srv->cv_done.notify_all();
            continue;
        }
        Slot* s = free_slot;
        s->batch.assign(srv->queue.begin(), srv->queue.begin() + k);
        srv->queue.erase(srv->queue.begin(), srv->queue.begin() + k);
        int64_t inst = 0, pix = 0;
        for (const ReqPtr& r : s->batch) { inst += r->inst_est; pix += r->pixels; }
        s->klass = log2_bucket(pix) * 64 + log2_bucket(inst);
        const int fixed = std::max(0, variant_of(srv->cfg.composite_chunk, srv->cfg.sort_items));
        bool exploring = false;
        s->variant = srv->cfg.autotune ? srv->tuner.pick(s->klass, fixed, &exploring) : fixed;
        if (exploring) srv->stats.explored_batches++;
        const double t = now_ms(srv->t0);
        for (const ReqPtr& r : s->batch) {
            r->result.start_ms = t;
            r->result.batch_views = k;
            r->result.composite_chunk = kVariantTable[s->variant].composite_chunk;
            r->result.sort_items = kVariantTable[s->variant].tile_sort_items;
        }
        s->busy = true;
        srv->stats.batches++;
        if (srv->cfg.use_graphs) srv->stats.graph_launches++;
        lk.unlock();
        const cudaError_t e = launch_batch(srv, s);
        lk.lock();
        s->launch_error = e;
        s->launched = true;
        s->cv.notify_one();
    }
}

void completer_main(LumenServer* srv, Slot* s) {
    cudaSetDevice(srv->device);
    std::unique_lock<std::mutex> lk(srv->mu);
    for (;;) {
        s->cv.wait(lk, [&] { return s->launched || (srv->stop && !s->busy); });
        if (!s->launched) break;
        const cudaError_t launch_error = s->launch_error;
        lk.unlock();
        cudaError_t e = launch_error;
        if (e == cudaSuccess) e = cudaEventSynchronize(s->ev_end);
        float ms = 0.0f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, s->ev_start, s->ev_end);
        Control c;
        std::memcpy(&c, s->h_back, sizeof(Control));
        const ViewTable* vt = (const ViewTable*)(s->h_back + sizeof(Control));
        lk.lock();
        const int nv = (int)s->batch.size();
        srv->stats.device_ms += ms;
        if (e != cudaSuccess) {
            for (const ReqPtr& r : s->batch) complete(srv, r, map_cuda(e));
        } else if (c.error_flags & LUMEN_GPU_ERR_CAPACITY) {
            /* more instances than estimated: raise every view's estimate by
             * the batch's overshoot and queue the requests again, in order */
            int64_t est = 0;
            for (const ReqPtr& r : s->batch) est += r->inst_est;
            const double f = std::max(1.5, (double)c.n_instances / (double)std::max<int64_t>(est, 1));
            for (const ReqPtr& r : s->batch) {
                auto key = std::make_tuple(r->scene, r->cam.width, r->cam.height);
                int64_t& o = srv->observed[key];
                o = std::max(o, (int64_t)(f * (double)r->inst_est));
            }
            if (srv->stop) {   /* no scheduler left to run them again */
                for (const ReqPtr& r : s->batch) complete(srv, r, LUMEN_ERROR_UNINITIALIZED);
            } else {
                srv->queue.insert(srv->queue.begin(), s->batch.begin(), s->batch.end());
                srv->stats.requeued_batches++;
            }
        } else {
            const int status = c.error_flags ? LUMEN_ERROR_IO_FAILURE : LUMEN_SUCCESS;
            const int64_t K = (int64_t)c.n_instances;
            if (c.error_flags == 0 && ms > 0.0f) srv->tuner.record(s->klass, s->variant, ms / (double)(K + 1));
            for (int v = 0; v < nv; ++v) {
                /* view v's instances: from its first to the next view's first */
                int64_t kv = 0;
                if (vt->view[v].inst_begin >= 0) {
                    int64_t end = K;
                    for (int u = v + 1; u < nv; ++u)
                        if (vt->view[u].inst_begin >= 0) { end = vt->view[u].inst_begin; break; }
                    kv = end - vt->view[v].inst_begin;
                }
                const ReqPtr& r = s->batch[(size_t)v];
                r->result.n_instances = kv;
                auto key = std::make_tuple(r->scene, r->cam.width, r->cam.height);
                int64_t& o = srv->observed[key];
                o = std::max(o, kv);
                complete(srv, r, status);
            }
        }
        s->batch.clear();
        s->launched = false;
        s->busy = false;
        srv->cv_sched.notify_all();
        srv->cv_done.notify_all();
    }
}

}  // namespace

extern "C" {

LumenServerConfig lumen_server_default_config(void) {
    LumenServerConfig c;
    std::memset(&c, 0, sizeof(c));
    c.work_budget_bytes = 8ll << 30;
    c.max_views_per_batch = 64;
    c.max_batches_in_flight = 2;
    c.use_graphs = 1;
    c.autotune = 1;
    c.composite_chunk = 256;
    c.sort_items = 16;
    c.options.lowpass = 0.3f;
    c.options.sh_degree = 3;
    c.options.compute_depth = 1;
    c.options.term_mode = 1;
    c.options.tile_size = 16;
    c.options.term_threshold = 0.99f;
    return c;
}

int32_t lumen_serve_admit(const int64_t* slots, const int64_t* tiles, const int64_t* instances,
                          const int64_t* pixels, int32_t n_requests, int32_t max_views, int64_t max_slots,
                          int64_t max_tiles, int64_t max_instances, int64_t max_pixels) {
    if (n_requests <= 0 || !slots || !tiles || !instances || !pixels || max_views <= 0) return 0;
    return admit_prefix(slots, tiles, instances, pixels, n_requests, max_views, max_slots, max_tiles, max_instances,
                        max_pixels);
}

LumenServer* lumen_server_create(const LumenServerConfig* config) {
    if (!config) return nullptr;
    const LumenServerConfig& c = *config;
    if (c.work_budget_bytes <= 0 || c.max_views_per_batch < 1 || c.max_views_per_batch > kMaxViews ||
        c.max_batches_in_flight < 1 || c.max_batches_in_flight > 16)
        return nullptr;
    if (!c.autotune && variant_of(c.composite_chunk, c.sort_items) < 0) return nullptr;
    if (c.options.tile_size != kTile || c.options.sh_degree < 0 || c.options.sh_degree > 3) return nullptr;
    LumenServer* srv = new (std::nothrow) LumenServer();
    if (!srv) return nullptr;
    srv->cfg = c;
    srv->t0 = std::chrono::steady_clock::now();
    if (cudaGetDevice(&srv->device) != cudaSuccess) { delete srv; return nullptr; }
    configure_once();
    srv->sms = device_sm_count();
    /* one slot's share of the budget: ~78 B per projection slot, ~18 B per
     * instance, 8 B per tile, 3 B per output pixel, split 20/55/3/22 % */
    const double b = (double)c.work_budget_bytes / c.max_batches_in_flight;
    srv->max_slots = std::max<int64_t>((int64_t)(0.20 * b / 78.0) / kProjThreads * kProjThreads, kProjThreads);
    srv->max_inst = std::min<int64_t>(std::max<int64_t>((int64_t)(0.55 * b / 18.0), 1 << 16), (1ll << 30) - 1);
    srv->max_tiles = std::max<int64_t>((int64_t)(0.03 * b / 8.0), 1024);
    srv->max_pix = std::max<int64_t>((int64_t)(0.22 * b / 3.0), 1 << 16);
    for (int i = 0; i < c.max_batches_in_flight; ++i) {
        auto s = std::make_unique<Slot>();
        s->index = i;
        const cudaError_t e = alloc_slot(srv, s.get());
        srv->slots.push_back(std::move(s));
        if (e != cudaSuccess) {
            for (auto& sl : srv->slots) free_slot(sl.get());
            delete srv;
            return nullptr;
        }
    }
    srv->slot_bytes = (int64_t)(srv->max_slots * 76 + srv->max_inst * 16 + srv->max_tiles * 8 + srv->max_pix * 3 +
                                (int64_t)srv->slots[0]->layout.total);
    srv->stats.slot_bytes = srv->slot_bytes;
    srv->stats.max_slots = srv->max_slots;
    srv->stats.max_tiles = srv->max_tiles;
    srv->stats.max_instances = srv->max_inst;
    srv->stats.max_pixels = srv->max_pix;
    for (auto& s : srv->slots) s->completer = std::thread(completer_main, srv, s.get());
    srv->scheduler = std::thread(scheduler_main, srv);
    return srv;
}

void lumen_server_destroy(LumenServer* srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
        for (const ReqPtr& r : srv->queue) complete(srv, r, LUMEN_ERROR_UNINITIALIZED);
        srv->queue.clear();
    }
    srv->cv_sched.notify_all();
    if (srv->scheduler.joinable()) srv->scheduler.join();
    for (auto& s : srv->slots) {
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            s->cv.notify_all();
        }
        if (s->completer.joinable()) s->completer.join();
    }
    srv->cv_done.notify_all();
    cudaSetDevice(srv->device);
    for (auto& s : srv->slots) free_slot(s.get());
    delete srv;
}

int32_t lumen_server_add_scene(LumenServer* srv, const LumenGpuGaussians* g) {
    if (!srv || !g || g->count < 0 || g->count >= (1ll << 31)) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (g->count > 0 && (!g->means || !g->scales || !g->quats || !g->opacities || !g->sh ||
                         ((uintptr_t)g->quats & 15u) || ((uintptr_t)g->sh & 15u)))
        return LUMEN_ERROR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->scenes.push_back(*g);
    return (int32_t)(srv->scenes.size() - 1);
}

LumenStatus lumen_server_submit(LumenServer* srv, int32_t scene, const LumenViewCamera* cam, uint8_t* out_rgb8,
                                uint64_t* request_id) {
    if (!srv || !cam || !request_id || !out_rgb8) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (cam->width <= 0 || cam->height <= 0 || cam->width > kMaxTilesPerAxis * kTile ||
        cam->height > kMaxTilesPerAxis * kTile)
        return LUMEN_ERROR_INVALID_ARGUMENT;
    auto r = std::make_shared<Request>();
    r->cam = *cam;
    r->out = out_rgb8;
    r->pixels = (int64_t)cam->width * cam->height;
    r->tiles = (int64_t)((cam->width + kTile - 1) / kTile) * ((cam->height + kTile - 1) / kTile);
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        if (srv->stop) return LUMEN_ERROR_UNINITIALIZED;
        if (scene < 0 || scene >= (int32_t)srv->scenes.size()) return LUMEN_ERROR_INVALID_ARGUMENT;
        r->scene = scene;
        r->slots = (srv->scenes[(size_t)scene].count + kProjThreads - 1) / kProjThreads * kProjThreads;
        r->id = srv->next_id++;
        r->result.request_id = r->id;
        r->result.submit_ms = now_ms(srv->t0);
        srv->requests[r->id] = r;
        srv->queue.push_back(r);
        srv->stats.submitted++;
        *request_id = r->id;
    }
    srv->cv_sched.notify_one();
    return LUMEN_SUCCESS;
}

LumenStatus lumen_server_wait(LumenServer* srv, uint64_t id, double timeout_ms, LumenServeResult* result) {
    if (!srv || !result) return LUMEN_ERROR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->requests.find(id);
    if (it == srv->requests.end()) return LUMEN_ERROR_INVALID_ARGUMENT;
    ReqPtr r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_ms < 0) {
        srv->cv_done.wait(lk, ready);
    } else if (!srv->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready)) {
        return LUMEN_ERROR_IO_FAILURE;
    }
    *result = r->result;
    srv->requests.erase(id);
    return LUMEN_SUCCESS;
}

LumenStatus lumen_server_freeze_tuning(LumenServer* srv, int32_t frozen) {
    if (!srv) return LUMEN_ERROR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->tuner.frozen = frozen != 0;
    return LUMEN_SUCCESS;
}

LumenStatus lumen_server_stats(LumenServer* srv, LumenServeStats* out) {
    if (!srv || !out) return LUMEN_ERROR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(srv->mu);
    *out = srv->stats;
    return LUMEN_SUCCESS;
}

}  // extern "C"
