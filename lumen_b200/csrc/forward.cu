/*
 * forward.cu - host side of the device API declared in include/lumen_gpu.h:
 * argument checks, scratch layout, the launch sequence of one frame, stage
 * timing, and a renderer that owns and grows its frame buffers.
 *
 * Launch sequence of a frame (all on the caller's stream, no host sync):
 *   frame_init         control block and look-back descriptors zeroed, view table
 *   batch_count        K1a: each block's visible count (geometry only)
 *   batch_offsets      K1b: the counts scanned into each block's first visible index
 *   batch_project      K1c: projection, cull, SH, records and depth keys at those offsets
 *   histogram<u32>     depth-key digits of the visible splats
 *   onesweep_pass x4   stable sort of visible splats by depth key
 *   emit               K2: (tile id, visible index) per covered tile, in depth order;
 *                      also the tile sort's digit counts, look-back tiles and ranges = -1
 *   onesweep_pass xb   stable sort of instances by tile id (b: the bytes a tile id
 *                      can vary in; with no Gaussians a histogram launch comes first);
 *                      the pass over the highest varying byte writes the tile ranges
 *   tile_ranges        K4: touched tiles and each view's first instance from the
 *                      ranges (the ranges themselves when no tile-id byte varies)
 *   composite          K5
 * Passes whose digit is constant exit at once (decided on the device).
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>
#include <cstddef>

#include "splat_common.cuh"

namespace lumen {
void launch_batch_project(const ViewTable* vt, const LumenRenderOptions& opt, const LumenGpuFrame& f,
                          Control* ctrl, unsigned long long* lb, long long n_units, long long n_blocks,
                          bool persistent, int num_sms, cudaStream_t st);
void launch_project(const ViewTable* vt, int n_views, const LumenRenderOptions& opt, const LumenGpuFrame& f,
                    Control* ctrl, unsigned long long* lb, long long n_blocks, bool persistent, int num_sms,
                    cudaStream_t st);
void launch_emit(const ViewTable* vt, const LumenGpuFrame& f, Control* ctrl, unsigned long long* lb,
                 unsigned int* sort_lb, long long sort_lb_tiles, int sort_tile_keys, long long n_blocks,
                 bool persistent, int num_sms, cudaStream_t st);
void launch_tile_sort_counted(unsigned int* k0, unsigned int* v0, unsigned int* k1, unsigned int* v1,
                              long long capacity, Control* ctrl, ViewTable* vt, int* ranges, unsigned int* lb,
                              long long lb_tiles_cap, int items, int key_bytes, int num_sms, cudaStream_t st);
void launch_sort32(unsigned int* k0, unsigned int* v0, unsigned int* k1, unsigned int* v1, long long capacity,
                   SortControl* sc, unsigned int* lb, long long lb_tiles_cap, int* ranges,
                   const long long* n_range_tiles, unsigned int* err, int items, int key_bytes, int num_sms,
                   cudaStream_t st);
void launch_sort64(unsigned long long* k0, unsigned int* v0, unsigned long long* k1, unsigned int* v1,
                   long long capacity, SortControl* sc, unsigned int* lb, long long lb_tiles_cap, unsigned int* err,
                   int num_sms, cudaStream_t st);
void launch_ranges(const LumenGpuFrame& f, Control* ctrl, ViewTable* vt, int num_sms, cudaStream_t st);
void launch_key_stats64(const unsigned long long* keys, long long n, SortControl* sc, int num_sms, cudaStream_t st);
void launch_sorted_keys64(const LumenGpuFrame& f, const Control* ctrl, int key_mode, unsigned long long* out,
                          int num_sms, cudaStream_t st);
void launch_composite(const ViewTable* vt, int n_views, const LumenGpuFrame& f, Control* ctrl,
                      const LumenRenderOptions& opt, long long tile_offset, long long n_tiles, bool persistent,
                      int chunk, bool track, int num_sms, cudaStream_t st);
void configure_sort_kernels();

int device_sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 148;
    return n;
}

void prime_persistent_launches();
void configure_backward_kernels();

/* Kernel attributes (the large dynamic shared memory limits) apply to the
 * device that is current when they are set, so they are set once per
 * device, before the first launch on it (and so before any graph capture);
 * the occupancy figures are the same on every B200. */
constexpr int kMaxConfiguredDevices = 64;

void configure_once() {
    static std::once_flag once[kMaxConfiguredDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxConfiguredDevices) {
        configure_sort_kernels();
        prime_persistent_launches();
        configure_backward_kernels();
        return;
    }
    std::call_once(once[dev], [] {
        configure_sort_kernels();
        prime_persistent_launches();
        configure_backward_kernels();
    });
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

static LumenStatus check_camera(const LumenViewCamera* cam) {
    if (!cam) return LUMEN_ERROR_INVALID_ARGUMENT;
    /* tile coordinates must fit the 12-bit fields of a splat's rectangle */
    if (cam->width <= 0 || cam->height <= 0 || cam->width > kMaxTilesPerAxis * kTile ||
        cam->height > kMaxTilesPerAxis * kTile)
        return LUMEN_ERROR_INVALID_ARGUMENT;
    return LUMEN_SUCCESS;
}

static LumenStatus check_gaussians(const LumenGpuGaussians* g) {
    if (!g) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (g->count < 0 || g->count >= (1ll << 31)) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (g->count > 0) {
        if (!g->means || !g->scales || !g->quats || !g->opacities || !g->sh) return LUMEN_ERROR_INVALID_ARGUMENT;
        if (!aligned16(g->quats) || !aligned16(g->sh)) return LUMEN_ERROR_INVALID_ARGUMENT;
    }
    return LUMEN_SUCCESS;
}

static LumenStatus check_options(const LumenRenderOptions* opt) {
    if (!opt) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (opt->tile_size != kTile) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (opt->sh_degree < 0 || opt->sh_degree > 3) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (opt->key_mode < 0 || opt->key_mode > 1 || opt->term_mode < 0 || opt->term_mode > 1)
        return LUMEN_ERROR_INVALID_ARGUMENT;
    return LUMEN_SUCCESS;
}

LumenStatus check_inputs(const LumenGpuGaussians* g, const LumenViewCamera* cam, const LumenRenderOptions* opt) {
    LumenStatus st = check_gaussians(g);
    if (st == LUMEN_SUCCESS) st = check_camera(cam);
    if (st == LUMEN_SUCCESS) st = check_options(opt);
    return st;
}

/* Device-side failures: capacity still exceeded -> out of memory; a bounded
 * wait that gave up, a failed index check or a bad launch -> I/O failure
 * (the device did not complete the frame correctly). */
LumenStatus status_from_flags(unsigned int flags) {
    if (flags & LUMEN_GPU_ERR_CAPACITY) return LUMEN_ERROR_OUT_OF_MEMORY;
    if (flags) return LUMEN_ERROR_IO_FAILURE;
    return LUMEN_SUCCESS;
}

LumenStatus map_cuda(cudaError_t e) {
    if (e == cudaSuccess) return LUMEN_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return LUMEN_ERROR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorInitializationError)
        return LUMEN_ERROR_UNINITIALIZED;
    return LUMEN_ERROR_INVALID_ARGUMENT;
}

static bool frame_ok(const LumenGpuFrame* f, int64_t n, bool need_radii) {
    if (!f || !f->scratch || !f->ranges || f->instance_capacity <= 0 || f->instance_capacity >= (1ll << 30)) return false;
    if (!f->keys[0] || !f->keys[1] || !f->vals[0] || !f->vals[1]) return false;
    if (n > 0 && (!f->records || !f->visible_ids || (need_radii && !f->radii) || !f->rects || !f->depth_keys[0] ||
                  !f->depth_keys[1] || !f->depth_order[0] || !f->depth_order[1]))
        return false;
    return true;
}

/* Zeroes the control block and the two scans' descriptors; with
 * write_view, first writes a one-view table. Block 0 then derives every
 * view's device camera (setup_camera) into the table. */
__global__ void frame_init_kernel(unsigned long long* zero, long long n_words, ViewTable* vt, BatchHeader hdr,
                                  ViewDesc v0, int write_view) {
    chain_begin();
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_words; i += nthreads) zero[i] = 0ull;
    if (blockIdx.x == 0) {
        if (write_view && threadIdx.x == 0) {
            vt->hdr = hdr;
            vt->view[0] = v0;
        }
        __syncthreads();
        const int nv = vt->hdr.n_views;
        for (int v = threadIdx.x; v < nv; v += blockDim.x) setup_camera(vt->view[v].cam, vt->view[v].dcam);
    }
}

/* The frame's kernels after the view table is in place. n_slots and
 * n_tiles are the batch's (plain launches) or upper bounds (persistent
 * launches, whose kernels read the batch's sizes from the table); n_views
 * is the batch's view count, or 0 when only the table knows it; n_units
 * the projection units (plain launches). Projection is a visibility count,
 * an offset scan and the projection proper, Gaussian-major (each distinct
 * scene read once); with n_units 0 a single view instead runs the one-pass
 * kernel with its compacting scan fused in (project_kernel). */
void launch_pipeline(const ScratchLayout& L, unsigned char* base, const LumenRenderOptions& opt,
                     const LumenGpuFrame& f, long long n_slots, long long n_tiles, int n_views, bool persistent,
                     const LaunchConfig& lc, cudaEvent_t* ev, cudaStream_t s, bool with_composite,
                     long long n_units) {
    Control* ctrl = (Control*)(base + L.control_off);
    ViewTable* vt = (ViewTable*)(base + L.table_off);
    unsigned long long* proj_lb = (unsigned long long*)(base + L.proj_lb_off);
    unsigned long long* emit_lb = (unsigned long long*)(base + L.emit_lb_off);
    unsigned int* depth_lb = (unsigned int*)(base + L.depth_lb_off);
    unsigned int* tile_lb = (unsigned int*)(base + L.tile_lb_off);
    const int sms = device_sm_count();
    if (n_slots > 0) {
        if (n_views == 1 && n_units == 0)
            launch_project(vt, n_views, opt, f, ctrl, proj_lb, L.proj_blocks, persistent, sms, s);
        else
            launch_batch_project(vt, opt, f, ctrl, proj_lb, n_units, L.proj_blocks, persistent, sms, s);
        if (ev) cudaEventRecord(ev[1], s);
        launch_sort32(f.depth_keys[0], f.depth_order[0], f.depth_keys[1], f.depth_order[1], n_slots,
                      &ctrl->depth_sort, depth_lb, L.depth_tiles, nullptr, nullptr, &ctrl->error_flags,
                      lc.depth_sort_items, 4, sms, s);
        launch_emit(vt, f, ctrl, emit_lb, tile_lb, 2 * L.sort_tiles, kSortThreads * lc.tile_sort_items,
                    L.proj_blocks, persistent, sms, s);
    } else if (ev) {
        cudaEventRecord(ev[1], s);
    }
    /* the tile-sort region holds 4 passes of 2048-key tiles; tile ids below
     * n_tiles (the batch's, or the bound a persistent launch is sized for)
     * vary in their low ceil(log2(n_tiles) / 8) bytes only. After an
     * emission the digit counts, look-back tiles and ranges are ready;
     * without one (no Gaussians) the sort's histogram kernel does that. */
    int tile_bytes = 0;
    for (long long t = n_tiles - 1; t > 0; t >>= 8) ++tile_bytes;
    if (n_slots > 0)
        launch_tile_sort_counted(f.keys[0], f.vals[0], f.keys[1], f.vals[1], f.instance_capacity, ctrl, vt,
                                 f.ranges, tile_lb, 2 * L.sort_tiles, lc.tile_sort_items, tile_bytes, sms, s);
    else
        launch_sort32(f.keys[0], f.vals[0], f.keys[1], f.vals[1], f.instance_capacity, &ctrl->tile_sort, tile_lb,
                      2 * L.sort_tiles, f.ranges, &vt->hdr.total_tiles, &ctrl->error_flags, lc.tile_sort_items,
                      tile_bytes, sms, s);
    if (ev) cudaEventRecord(ev[2], s);
    launch_ranges(f, ctrl, vt, sms, s);
    if (ev) cudaEventRecord(ev[3], s);
    if (!with_composite) return;
    launch_composite(vt, n_views, f, ctrl, opt, 0, n_tiles, persistent, lc.composite_chunk, lc.track != 0, sms, s);
    if (ev) cudaEventRecord(ev[4], s);
}

void launch_init(const ScratchLayout& L, unsigned char* base, const BatchHeader* hdr, const ViewDesc* v0,
                        cudaStream_t s) {
    const long long words = (long long)(L.zeroed_prefix() / sizeof(unsigned long long));
    long long grid = (words + 255) / 256;
    if (grid > 256) grid = 256;
    if (grid < 1) grid = 1;
    BatchHeader h{};
    ViewDesc v{};
    if (hdr) h = *hdr;
    if (v0) v = *v0;
    launch_chained(frame_init_kernel, dim3((int)grid), dim3(256), 0, s, (unsigned long long*)base, words,
                   (ViewTable*)(base + L.table_off), h, v, (int)(v0 != nullptr));
}

static bool launch_ok(const LaunchConfig& lc) {
    return (lc.composite_chunk == 128 || lc.composite_chunk == 256 || lc.composite_chunk == 512) &&
           (lc.depth_sort_items == 8 || lc.depth_sort_items == 16) &&
           (lc.tile_sort_items == 8 || lc.tile_sort_items == 16 || lc.tile_sort_items == 24);
}

/* The one-view table of a plain frame: the view leads its own scene group
 * and owns every projection unit. */
static void single_view_table(const LumenGpuGaussians* g, const LumenViewCamera* cam, const LumenGpuImage* img,
                              const ScratchLayout& L, long long tiles, BatchHeader* hdr, ViewDesc* v) {
    std::memset(hdr, 0, sizeof(*hdr));
    hdr->n_views = 1;
    hdr->total_blocks = L.proj_blocks;
    hdr->total_tiles = tiles;
    hdr->total_units = L.proj_blocks;
    std::memset(v, 0, sizeof(*v));
    v->g = *g;
    v->cam = *cam;
    v->tiles_x = (cam->width + kTile - 1) / kTile;
    v->img = *img;
    v->inst_begin = -1;
    v->unit_begin = 0;
    v->group_next = -1;
    v->group_lead = 1;
}

static LumenStatus forward_impl(const LumenGpuGaussians* g, const LumenViewCamera* cam, const LumenRenderOptions* opt,
                                LumenGpuFrame* f, LumenGpuImage* img, cudaEvent_t* ev, void* stream,
                                LaunchConfig lc = kDefaultLaunch) {
    if (!launch_ok(lc)) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (img) lc.track = img->n_contrib || img->last_idx;
    LumenStatus st = check_inputs(g, cam, opt);
    if (st != LUMEN_SUCCESS) return st;
    if (!img || (!img->rgb && !img->rgb8) || !frame_ok(f, g->count, true)) return LUMEN_ERROR_INVALID_ARGUMENT;
    const ScratchLayout L = ScratchLayout::make(g->count, f->instance_capacity);
    if (f->scratch_bytes < L.total) return LUMEN_ERROR_INVALID_ARGUMENT;
    configure_once();
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* base = (unsigned char*)f->scratch;
    const int tiles_x = (cam->width + kTile - 1) / kTile;
    const long long tiles = (long long)tiles_x * ((cam->height + kTile - 1) / kTile);
    BatchHeader hdr{};
    ViewDesc v{};
    single_view_table(g, cam, img, L, tiles, &hdr, &v);
    if (ev) cudaEventRecord(ev[0], s);
    launch_init(L, base, &hdr, &v, s);
    launch_pipeline(L, base, *opt, *f, g->count, tiles, 1, false, lc, ev, s, true, hdr.total_units);
    return map_cuda(cudaGetLastError());
}

/* The forward of one view with the compositor launched in n_bands row
 * bands of tiles; after each band, after_band(ctx, pixel_row_begin,
 * pixel_row_end, stream) may enqueue work that reads those rows of the
 * image (copies overlapping the next band). */
LumenStatus forward_banded(const LumenGpuGaussians* g, const LumenViewCamera* cam, const LumenRenderOptions* opt,
                           LumenGpuFrame* f, LumenGpuImage* img, int n_bands, BandHook after_band, void* ctx,
                           cudaStream_t s) {
    LumenStatus st = check_inputs(g, cam, opt);
    if (st != LUMEN_SUCCESS) return st;
    if (!img || (!img->rgb && !img->rgb8) || !frame_ok(f, g->count, true) || n_bands < 1)
        return LUMEN_ERROR_INVALID_ARGUMENT;
    const ScratchLayout L = ScratchLayout::make(g->count, f->instance_capacity);
    if (f->scratch_bytes < L.total) return LUMEN_ERROR_INVALID_ARGUMENT;
    configure_once();
    unsigned char* base = (unsigned char*)f->scratch;
    const int tiles_x = (cam->width + kTile - 1) / kTile;
    const int tiles_y = (cam->height + kTile - 1) / kTile;
    const long long tiles = (long long)tiles_x * tiles_y;
    BatchHeader hdr{};
    ViewDesc v{};
    single_view_table(g, cam, img, L, tiles, &hdr, &v);
    launch_init(L, base, &hdr, &v, s);
    launch_pipeline(L, base, *opt, *f, g->count, tiles, 1, false, kDefaultLaunch, nullptr, s, false,
                    hdr.total_units);
    Control* ctrl = (Control*)(base + L.control_off);
    const ViewTable* vt = (const ViewTable*)(base + L.table_off);
    const int sms = device_sm_count();
    if (n_bands > tiles_y) n_bands = tiles_y;
    for (int b = 0; b < n_bands; ++b) {
        const int r0 = (int)((long long)tiles_y * b / n_bands), r1 = (int)((long long)tiles_y * (b + 1) / n_bands);
        launch_composite(vt, 1, *f, ctrl, *opt, (long long)r0 * tiles_x, (long long)(r1 - r0) * tiles_x, false,
                         kDefaultLaunch.composite_chunk, img->n_contrib || img->last_idx, sms, s);
        const int y0 = r0 * kTile, y1 = r1 * kTile < cam->height ? r1 * kTile : cam->height;
        if (after_band) after_band(ctx, y0, y1, s);
    }
    return map_cuda(cudaGetLastError());
}

/* Offsets of a batch's views: blocks (256 Gaussians each) and tiles. */
static LumenStatus plan_batch(const LumenGpuBatchView* views, int n_views, const LumenRenderOptions* opt,
                              std::vector<ViewDesc>* out, BatchHeader* hdr) {
    if (!views || n_views <= 0 || n_views > kMaxViews) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (opt && check_options(opt) != LUMEN_SUCCESS) return LUMEN_ERROR_INVALID_ARGUMENT;
    long long blocks = 0, tiles = 0;
    if (out) out->resize((size_t)n_views);
    for (int v = 0; v < n_views; ++v) {
        const LumenGpuBatchView& bv = views[v];
        if (check_gaussians(&bv.gaussians) != LUMEN_SUCCESS || check_camera(&bv.camera) != LUMEN_SUCCESS)
            return LUMEN_ERROR_INVALID_ARGUMENT;
        if (out && !bv.image.rgb && !bv.image.rgb8) return LUMEN_ERROR_INVALID_ARGUMENT;
        const int tiles_x = (bv.camera.width + kTile - 1) / kTile;
        const long long vt = (long long)tiles_x * ((bv.camera.height + kTile - 1) / kTile);
        if (out) {
            ViewDesc& d = (*out)[(size_t)v];
            std::memset(&d, 0, sizeof(d));
            d.g = bv.gaussians;
            d.cam = bv.camera;
            d.tiles_x = tiles_x;
            d.img = bv.image;
            d.block_begin = blocks;
            d.tile_begin = tiles;
            d.inst_begin = -1;
        }
        blocks += (bv.gaussians.count + kProjThreads - 1) / kProjThreads;
        tiles += vt;
    }
    /* visible indices and tile ids are 32-bit on the device */
    if (blocks * kProjThreads >= (1ll << 31) || tiles >= (1ll << 31)) return LUMEN_ERROR_INVALID_ARGUMENT;
    std::memset(hdr, 0, sizeof(*hdr));
    hdr->n_views = n_views;
    hdr->total_blocks = blocks;
    hdr->total_tiles = tiles;
    if (out) hdr->total_units = assign_scene_groups(out->data(), n_views);
    return LUMEN_SUCCESS;
}

static LumenStatus batch_impl(const LumenGpuBatchView* views, int n_views, const LumenRenderOptions* opt,
                              LumenGpuFrame* f, cudaEvent_t* ev, void* stream) {
    if (!opt) return LUMEN_ERROR_INVALID_ARGUMENT;
    std::vector<ViewDesc> table;
    BatchHeader hdr;
    LumenStatus st = plan_batch(views, n_views, opt, &table, &hdr);
    if (st != LUMEN_SUCCESS) return st;
    const long long slots = hdr.total_blocks * kProjThreads;
    if (!frame_ok(f, slots, false)) return LUMEN_ERROR_INVALID_ARGUMENT;
    const ScratchLayout L = ScratchLayout::make(slots, f->instance_capacity, n_views);
    if (f->scratch_bytes < L.total) return LUMEN_ERROR_INVALID_ARGUMENT;
    configure_once();
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* base = (unsigned char*)f->scratch;
    /* header and views in one host block; a copy from pageable memory
     * returns once the bytes are staged, so the block may go out of scope */
    std::vector<unsigned char> host(view_table_bytes(n_views));
    std::memcpy(host.data(), &hdr, sizeof(hdr));
    std::memcpy(host.data() + offsetof(ViewTable, view), table.data(), table.size() * sizeof(ViewDesc));
    if (ev) cudaEventRecord(ev[0], s);
    cudaError_t e = cudaMemcpyAsync(base + L.table_off, host.data(), host.size(), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return map_cuda(e);
    launch_init(L, base, nullptr, nullptr, s);
    LaunchConfig lc = kDefaultLaunch;
    lc.track = 0;
    for (int v = 0; v < n_views; ++v)
        if (views[v].image.n_contrib || views[v].image.last_idx) lc.track = 1;
    launch_pipeline(L, base, *opt, *f, slots, hdr.total_tiles, n_views, false, lc, ev, s, true, hdr.total_units);
    return map_cuda(cudaGetLastError());
}

}  // namespace lumen

using namespace lumen;

struct LumenGpuStageTimer {
    int max_frames = 0;
    int next = 0;
    cudaEvent_t* ev = nullptr;   /* max_frames x 5 */
};

extern "C" {

size_t lumen_gpu_scratch_bytes(int64_t n_gaussians, int64_t instance_capacity, int64_t n_tiles) {
    (void)n_tiles;
    return ScratchLayout::make(n_gaussians, instance_capacity).total;
}

LumenStatus lumen_gpu_render_forward(const LumenGpuGaussians* g, const LumenViewCamera* cam,
                                     const LumenRenderOptions* opt, LumenGpuFrame* f, LumenGpuImage* img,
                                     void* stream) {
    return forward_impl(g, cam, opt, f, img, nullptr, stream);
}

LumenStatus lumen_gpu_render_forward_ex(const LumenGpuGaussians* g, const LumenViewCamera* cam,
                                        const LumenRenderOptions* opt, const LumenGpuLaunch* launch,
                                        LumenGpuFrame* f, LumenGpuImage* img, LumenGpuStageTimer* t, void* stream) {
    if (!launch) return LUMEN_ERROR_INVALID_ARGUMENT;
    const LaunchConfig lc = {launch->composite_chunk, launch->depth_sort_items, launch->tile_sort_items, 1};
    if (!t) return forward_impl(g, cam, opt, f, img, nullptr, stream, lc);
    if (t->next >= t->max_frames) return LUMEN_ERROR_INVALID_ARGUMENT;
    LumenStatus st = forward_impl(g, cam, opt, f, img, t->ev + (size_t)t->next * 5, stream, lc);
    if (st == LUMEN_SUCCESS) t->next++;
    return st;
}

LumenStatus lumen_gpu_read_counts(const LumenGpuFrame* f, LumenGpuCounts* c, void* stream) {
    if (!f || !c || !f->scratch) return LUMEN_ERROR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    Control h;
    cudaError_t e = cudaMemcpyAsync(&h, f->scratch, sizeof(Control), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return map_cuda(e);
    c->n_visible = h.n_visible;
    c->n_instances = (int64_t)h.n_instances;
    c->error_flags = h.error_flags;
    c->sorted_buffer = h.tile_sort.sorted_buffer;
    c->varying_digits = (h.tile_sort.varying & 0xFFu) | ((h.depth_sort.varying & 0xFFu) << 8);
    c->touched_tiles = h.touched_tiles;
    c->depth_sorted_buffer = h.depth_sort.sorted_buffer;
    c->reserved = 0;
    return LUMEN_SUCCESS;
}

LumenStatus lumen_gpu_frame_sorted_keys64(const LumenGpuFrame* f, const LumenRenderOptions* opt, uint64_t* out,
                                          void* stream) {
    if (!f || !opt || !out || !f->scratch) return LUMEN_ERROR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    launch_sorted_keys64(*f, (const Control*)f->scratch, opt->key_mode, reinterpret_cast<unsigned long long*>(out),
                         device_sm_count(), s);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return map_cuda(e);
}

LumenGpuStageTimer* lumen_gpu_stage_timer_create(int max_frames) {
    if (max_frames <= 0) return nullptr;
    LumenGpuStageTimer* t = new (std::nothrow) LumenGpuStageTimer();
    if (!t) return nullptr;
    t->ev = new (std::nothrow) cudaEvent_t[(size_t)max_frames * 5]();
    if (!t->ev) { delete t; return nullptr; }
    t->max_frames = max_frames;
    for (int i = 0; i < max_frames * 5; ++i)
        if (cudaEventCreate(&t->ev[i]) != cudaSuccess) { lumen_gpu_stage_timer_destroy(t); return nullptr; }
    return t;
}

void lumen_gpu_stage_timer_destroy(LumenGpuStageTimer* t) {
    if (!t) return;
    if (t->ev)
        for (int i = 0; i < t->max_frames * 5; ++i)
            if (t->ev[i]) cudaEventDestroy(t->ev[i]);
    delete[] t->ev;
    delete t;
}

LumenStatus lumen_gpu_render_forward_timed(const LumenGpuGaussians* g, const LumenViewCamera* cam,
                                           const LumenRenderOptions* opt, LumenGpuFrame* f, LumenGpuImage* img,
                                           LumenGpuStageTimer* t, void* stream) {
    if (!t || t->next >= t->max_frames) return LUMEN_ERROR_INVALID_ARGUMENT;
    LumenStatus st = forward_impl(g, cam, opt, f, img, t->ev + (size_t)t->next * 5, stream);
    if (st == LUMEN_SUCCESS) t->next++;
    return st;
}

LumenStatus lumen_gpu_batch_sizes(const LumenGpuBatchView* views, int32_t n_views, int64_t* slots, int64_t* tiles) {
    if (!slots || !tiles) return LUMEN_ERROR_INVALID_ARGUMENT;
    BatchHeader hdr;
    LumenStatus st = plan_batch(views, n_views, nullptr, nullptr, &hdr);
    if (st != LUMEN_SUCCESS) return st;
    *slots = hdr.total_blocks * kProjThreads;
    *tiles = hdr.total_tiles;
    return LUMEN_SUCCESS;
}

size_t lumen_gpu_batch_scratch_bytes(int64_t slots, int64_t instance_capacity, int32_t n_views) {
    if (slots < 0 || instance_capacity < 0 || n_views <= 0 || n_views > kMaxViews) return 0;
    return ScratchLayout::make(slots, instance_capacity, n_views).total;
}

LumenStatus lumen_gpu_render_batch(const LumenGpuBatchView* views, int32_t n_views, const LumenRenderOptions* opt,
                                   LumenGpuFrame* f, void* stream) {
    return batch_impl(views, n_views, opt, f, nullptr, stream);
}

LumenStatus lumen_gpu_render_batch_timed(const LumenGpuBatchView* views, int32_t n_views,
                                         const LumenRenderOptions* opt, LumenGpuFrame* f, LumenGpuStageTimer* t,
                                         void* stream) {
    if (!t || t->next >= t->max_frames) return LUMEN_ERROR_INVALID_ARGUMENT;
    LumenStatus st = batch_impl(views, n_views, opt, f, t->ev + (size_t)t->next * 5, stream);
    if (st == LUMEN_SUCCESS) t->next++;
    return st;
}

}  // extern "C"

namespace lumen {
/* The next frame's five events of a stage timer, or nullptr when it is full
 * (used by the timed backward). The caller records all five. */
cudaEvent_t* stage_timer_take(LumenGpuStageTimer* t) {
    if (!t || t->next >= t->max_frames) return nullptr;
    return t->ev + (size_t)(t->next++) * 5;
}
}  // namespace lumen

extern "C" {

LumenStatus lumen_gpu_stage_timer_read(LumenGpuStageTimer* t, float stage_ms[4], float* total_ms, int* n_frames) {
    if (!t || !stage_ms) return LUMEN_ERROR_INVALID_ARGUMENT;
    for (int s = 0; s < 4; ++s) stage_ms[s] = 0.0f;
    if (total_ms) *total_ms = 0.0f;
    if (n_frames) *n_frames = t->next;
    if (t->next == 0) return LUMEN_SUCCESS;
    cudaError_t e = cudaEventSynchronize(t->ev[(size_t)(t->next - 1) * 5 + 4]);
    if (e != cudaSuccess) return map_cuda(e);
    for (int fr = 0; fr < t->next; ++fr) {
        cudaEvent_t* ev = t->ev + (size_t)fr * 5;
        for (int s = 0; s < 4; ++s) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev[s], ev[s + 1]);
            stage_ms[s] += ms;
        }
    }
    if (total_ms) cudaEventElapsedTime(total_ms, t->ev[0], t->ev[(size_t)(t->next - 1) * 5 + 4]);
    t->next = 0;
    return LUMEN_SUCCESS;
}

LumenStatus lumen_gpu_sort_pairs(uint64_t* keys0, uint32_t* vals0, uint64_t* keys1, uint32_t* vals1, int64_t n,
                                 void* scratch, size_t scratch_bytes, uint32_t* sorted_buffer, void* stream) {
    if (n < 0 || n >= (1ll << 30) || !sorted_buffer) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (n > 0 && (!keys0 || !vals0 || !keys1 || !vals1 || !scratch)) return LUMEN_ERROR_INVALID_ARGUMENT;
    *sorted_buffer = 0;
    if (n == 0) return LUMEN_SUCCESS;
    const ScratchLayout L = ScratchLayout::make(0, n);
    if (scratch_bytes < L.total) return LUMEN_ERROR_INVALID_ARGUMENT;
    configure_once();
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* base = (unsigned char*)scratch;
    Control* ctrl = (Control*)(base + L.control_off);
    cudaError_t e = cudaMemsetAsync(base, 0, L.zeroed_prefix(), s);
    if (e != cudaSuccess) return map_cuda(e);
    const int sms = device_sm_count();
    unsigned long long* k0 = reinterpret_cast<unsigned long long*>(keys0);
    unsigned long long* k1 = reinterpret_cast<unsigned long long*>(keys1);
    launch_key_stats64(k0, n, &ctrl->tile_sort, sms, s);
    /* the tile-sort look-back region holds 8 digits x tiles x 256 entries */
    launch_sort64(k0, vals0, k1, vals1, n, &ctrl->tile_sort, (unsigned int*)(base + L.tile_lb_off), L.sort_tiles,
                  &ctrl->error_flags, sms, s);
    if ((e = cudaGetLastError()) != cudaSuccess) return map_cuda(e);
    Control h;
    e = cudaMemcpyAsync(&h, ctrl, sizeof(Control), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return map_cuda(e);
    *sorted_buffer = h.tile_sort.sorted_buffer;
    return status_from_flags(h.error_flags);
}

}  // extern "C"

/* ---------------------------------------------------------------- renderer */

struct LumenGpuRenderer {
    LumenGpuFrame frame;
    int64_t n_cap = 0;       /* Gaussians the per-Gaussian buffers hold */
    int64_t tiles_cap = 0;
    int64_t k_cap = 0;
    int device = -1;
};

namespace {

void free_per_gaussian(LumenGpuFrame& f) {
    cudaFree(f.records); cudaFree(f.visible_ids); cudaFree(f.radii); cudaFree(f.rects);
    for (int b = 0; b < 2; ++b) { cudaFree(f.depth_keys[b]); cudaFree(f.depth_order[b]); }
    f.records = nullptr; f.visible_ids = nullptr; f.radii = nullptr; f.rects = nullptr;
    for (int b = 0; b < 2; ++b) { f.depth_keys[b] = nullptr; f.depth_order[b] = nullptr; }
}

void free_frame(LumenGpuRenderer* r) {
    LumenGpuFrame& f = r->frame;
    free_per_gaussian(f);
    for (int b = 0; b < 2; ++b) { cudaFree(f.keys[b]); cudaFree(f.vals[b]); }
    cudaFree(f.ranges); cudaFree(f.scratch);
    std::memset(&f, 0, sizeof(f));
    r->n_cap = r->tiles_cap = r->k_cap = 0;
}

/* Grow the buffers to hold n Gaussians, `tiles` tiles and k instances. */
LumenStatus ensure(LumenGpuRenderer* r, int64_t n, int64_t tiles, int64_t k) {
    LumenGpuFrame& f = r->frame;
    cudaError_t e = cudaSuccess;
    if (n > r->n_cap) {
        const int64_t nn = n + n / 8 + 1024;
        free_per_gaussian(f);
        r->n_cap = 0;
        if ((e = cudaMalloc(&f.records, nn * sizeof(LumenSplatRecord))) != cudaSuccess) return map_cuda(e);
        if ((e = cudaMalloc(&f.visible_ids, nn * sizeof(uint32_t))) != cudaSuccess) return map_cuda(e);
        if ((e = cudaMalloc(&f.radii, nn * sizeof(int32_t))) != cudaSuccess) return map_cuda(e);
        if ((e = cudaMalloc(&f.rects, nn * sizeof(uint64_t))) != cudaSuccess) return map_cuda(e);
        for (int b = 0; b < 2; ++b) {
            if ((e = cudaMalloc(&f.depth_keys[b], nn * sizeof(uint32_t))) != cudaSuccess) return map_cuda(e);
            if ((e = cudaMalloc(&f.depth_order[b], nn * sizeof(uint32_t))) != cudaSuccess) return map_cuda(e);
        }
        r->n_cap = nn;
    }
    if (tiles > r->tiles_cap) {
        cudaFree(f.ranges);
        f.ranges = nullptr;
        r->tiles_cap = 0;
        if ((e = cudaMalloc(&f.ranges, tiles * 2 * sizeof(int32_t))) != cudaSuccess) return map_cuda(e);
        r->tiles_cap = tiles;
    }
    if (k > r->k_cap) {
        int64_t kk = k + k / 4 + 4096;
        if (kk >= (1ll << 30)) kk = (1ll << 30) - 1;
        if (k > kk) return LUMEN_ERROR_OUT_OF_MEMORY;
        for (int b = 0; b < 2; ++b) {
            cudaFree(f.keys[b]); cudaFree(f.vals[b]);
            f.keys[b] = nullptr; f.vals[b] = nullptr;
        }
        r->k_cap = 0;
        f.instance_capacity = 0;
        for (int b = 0; b < 2; ++b) {
            if ((e = cudaMalloc(&f.keys[b], kk * sizeof(uint32_t))) != cudaSuccess) return map_cuda(e);
            if ((e = cudaMalloc(&f.vals[b], kk * sizeof(uint32_t))) != cudaSuccess) return map_cuda(e);
        }
        r->k_cap = kk;
        f.instance_capacity = kk;
    }
    const size_t need = ScratchLayout::make(r->n_cap, r->k_cap).total;
    if (need > f.scratch_bytes) {
        cudaFree(f.scratch);
        f.scratch = nullptr;
        f.scratch_bytes = 0;
        if ((e = cudaMalloc(&f.scratch, need)) != cudaSuccess) return map_cuda(e);
        f.scratch_bytes = need;
    }
    return LUMEN_SUCCESS;
}

}  // namespace

extern "C" {

LumenGpuRenderer* lumen_gpu_renderer_create(void) {
    LumenGpuRenderer* r = new (std::nothrow) LumenGpuRenderer();
    if (!r) return nullptr;
    std::memset(&r->frame, 0, sizeof(r->frame));
    if (cudaGetDevice(&r->device) != cudaSuccess) { delete r; return nullptr; }
    return r;
}

void lumen_gpu_renderer_destroy(LumenGpuRenderer* r) {
    if (!r) return;
    free_frame(r);
    delete r;
}

const LumenGpuFrame* lumen_gpu_renderer_frame(const LumenGpuRenderer* r) { return r ? &r->frame : nullptr; }

LumenStatus lumen_gpu_renderer_render(LumenGpuRenderer* r, const LumenGpuGaussians* g, const LumenViewCamera* cam,
                                      const LumenRenderOptions* opt, LumenGpuImage* img, LumenGpuCounts* counts,
                                      void* stream) {
    if (!r) return LUMEN_ERROR_INVALID_ARGUMENT;
    LumenStatus st = check_inputs(g, cam, opt);
    if (st != LUMEN_SUCCESS) return st;
    const int64_t tiles = (int64_t)((cam->width + kTile - 1) / kTile) * ((cam->height + kTile - 1) / kTile);
    const int64_t k_guess = r->k_cap > 0 ? r->k_cap : (g->count * 8 > (1 << 20) ? g->count * 8 : (1 << 20));
    st = ensure(r, g->count > 0 ? g->count : 1, tiles, k_guess);
    if (st != LUMEN_SUCCESS) return st;
    LumenGpuCounts c;
    std::memset(&c, 0, sizeof(c));
    for (int attempt = 0; attempt < 2; ++attempt) {
        st = lumen_gpu_render_forward(g, cam, opt, &r->frame, img, stream);
        if (st != LUMEN_SUCCESS) return st;
        st = lumen_gpu_read_counts(&r->frame, &c, stream);
        if (st != LUMEN_SUCCESS) return st;
        if (!(c.error_flags & LUMEN_GPU_ERR_CAPACITY)) break;
        st = ensure(r, g->count, tiles, c.n_instances);
        if (st != LUMEN_SUCCESS) return st;
    }
    if (counts) *counts = c;
    return status_from_flags(c.error_flags);
}

}  // extern "C"

namespace lumen {

/* lumen_gpu_renderer_render with the compositor in row bands
 * (forward_banded): the whole frame is enqueued, bands and hooks included,
 * before the one host wait for the counts; on a capacity overflow the
 * buffers grow and the frame, hooks included, is enqueued again. */
LumenStatus renderer_render_banded(LumenGpuRenderer* r, const LumenGpuGaussians* g, const LumenViewCamera* cam,
                                   const LumenRenderOptions* opt, LumenGpuImage* img, LumenGpuCounts* counts,
                                   int n_bands, BandHook hook, void* ctx, cudaStream_t stream) {
    if (!r) return LUMEN_ERROR_INVALID_ARGUMENT;
    LumenStatus st = check_inputs(g, cam, opt);
    if (st != LUMEN_SUCCESS) return st;
    const int64_t tiles = (int64_t)((cam->width + kTile - 1) / kTile) * ((cam->height + kTile - 1) / kTile);
    const int64_t k_guess = r->k_cap > 0 ? r->k_cap : (g->count * 8 > (1 << 20) ? g->count * 8 : (1 << 20));
    st = ensure(r, g->count > 0 ? g->count : 1, tiles, k_guess);
    if (st != LUMEN_SUCCESS) return st;
    LumenGpuCounts c;
    std::memset(&c, 0, sizeof(c));
    for (int attempt = 0; attempt < 2; ++attempt) {
        st = forward_banded(g, cam, opt, &r->frame, img, n_bands, hook, ctx, stream);
        if (st != LUMEN_SUCCESS) return st;
        st = lumen_gpu_read_counts(&r->frame, &c, stream);
        if (st != LUMEN_SUCCESS) return st;
        if (!(c.error_flags & LUMEN_GPU_ERR_CAPACITY)) break;
        st = ensure(r, g->count, tiles, c.n_instances);
        if (st != LUMEN_SUCCESS) return st;
    }
    if (counts) *counts = c;
    return status_from_flags(c.error_flags);
}

}  // namespace lumen
