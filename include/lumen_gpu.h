/*
 * lumen_gpu.h - device-resident entry points of liblumen (B200, sm_100a).
 *
 * These functions take device pointers and a CUDA stream (as void*) and never
 * see a host copy of the scene. They are what the Python SDK, the torch
 * autograd function and the render server call through ctypes; lumen.h's
 * lumen_rasterize is built on them.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   lumen_gpu_render_forward  - rasterize_scene, src/raster/pipeline.mojo:48-52
 *                               (RenderOutput fields, pipeline.mojo:21-45)
 *   lumen_gpu_renderer_render - lumen_rasterize, c_api/include/lumen.h:153-159,
 *                               with library-owned work buffers
 *   lumen_gpu_render_backward - no counterpart: the reference has no
 *                               analytic backward (src/optim/gradients.mojo:11-106
 *                               only stores gradients)
 *   lumen_gpu_l1_loss         - compute_l1_loss, src/optim/loss.mojo:11-35
 *   lumen_gpu_sort_pairs      - radix_sort_64bit, src/raster/radix_sort.mojo:39-87
 *
 * Threading: no global state; every call works only on the buffers it is
 * given and enqueues on the given stream. Functions that wait say so.
 * Limits: instance counts below 2^30, Gaussian counts below 2^31.
 */
#ifndef LUMEN_GPU_H
#define LUMEN_GPU_H

#include "lumen.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Gaussians in device memory, float32, contiguous SoA:
 * means [N,3], scales [N,3] (linear, or log-scales when params_are_logits),
 * quats [N,4] (w,x,y,z, any norm), opacities [N] ([0,1], or logits),
 * sh [N,16,3] (sh[i*48 + coef*3 + ch]). */
typedef struct {
    const float* means;
    const float* scales;
    const float* quats;
    const float* opacities;
    const float* sh;
    int64_t count;
} LumenGpuGaussians;

/* Pinhole camera in the reference PinholeCamera convention
 * (src/scene/camera.mojo:24-79): camera-space point = rotation^-1 (p - position),
 * identity looks down +z, image x right and y down. */
typedef struct {
    float position[3];
    float rotation[4];              /* w, x, y, z; normalised by the kernels */
    float fx, fy, cx, cy;
    float near_plane, far_plane;
    int32_t width, height;
} LumenViewCamera;

/* RenderConfig fields read on the path (src/core/config.mojo:65-102) plus:
 * key_mode 0 = millimetre depth key (radix_sort.mojo:8-18), 1 = float bits;
 * term_mode 0 = stop a pixel when T <= term_threshold (1e-4, compositor.mojo:53),
 *           1 = stop when 1 - T >= term_threshold (0.99);
 * params_are_logits 1 = scales are log-scales, opacities are logits. */
typedef struct {
    float lowpass;
    int32_t sh_degree;
    int32_t white_background;
    int32_t compute_depth;
    int32_t key_mode;
    int32_t term_mode;
    int32_t params_are_logits;
    int32_t tile_size;              /* must be 16 */
    float term_threshold;
} LumenRenderOptions;

/* One projected splat (pipeline.mojo:141-149), 48 bytes, indexed by the
 * compacted visible index. ic* is Covariance2D.inverse(). */
typedef struct {
    float cx, cy, depth, opacity;
    float ic00, ic01, ic11, pad0;
    float r, g, b, pad1;
} LumenSplatRecord;

/* Work buffers of one frame, device memory owned by the caller.
 *
 * The reference sorts 64-bit (tile << 32 | depth key) instance keys with a
 * stable LSD sort over emission order (pipeline.mojo:152-166). The same
 * permutation is produced here in two smaller sorts: the visible splats are
 * stably sorted by depth key (depth_keys/depth_order), instances are emitted
 * in that order with 32-bit tile-id keys, and those are stably sorted by
 * tile (keys/vals). Within a tile both orders are (depth key, visible index).
 *
 * Per Gaussian (n_gaussians entries each): records, visible_ids, radii,
 * rects (tile rectangle of each visible splat: min_tx | min_ty << 16 |
 * max_tx << 32 | max_ty << 48), depth_keys[2] and depth_order[2] (ping-pong).
 * Per instance (instance_capacity entries each): keys[2] (tile ids) and
 * vals[2] (visible indices), ping-pong. ranges: 2 * n_tiles int32 (start,
 * end; -1,-1 for an empty tile, as binning.mojo:10-28). scratch:
 * lumen_gpu_scratch_bytes() bytes. */
typedef struct {
    LumenSplatRecord* records;
    uint32_t* visible_ids;
    int32_t* radii;
    uint64_t* rects;
    uint32_t* depth_keys[2];
    uint32_t* depth_order[2];
    uint32_t* keys[2];
    uint32_t* vals[2];
    int64_t instance_capacity;
    int32_t* ranges;
    void* scratch;
    size_t scratch_bytes;
} LumenGpuFrame;

/* Per-pixel outputs in device memory. rgb [H,W,3] or rgb8 is required;
 * the others may be NULL. depth [H,W] alpha-weighted depth; alpha [H,W] =
 * 1 - T; n_contrib [H,W] splats blended (the terminating one included);
 * last_idx [H,W] sorted index of the last instance visited, -1 if none;
 * rgb8 [H,W,3] bytes (uint8)(clamp(c, 0, 1) * 255), the conversion of
 * c_api/src/lumen_c.c:541-543 for a frame that starts cleared. */
typedef struct {
    float* rgb;
    float* depth;
    float* alpha;
    uint32_t* n_contrib;
    int32_t* last_idx;
    uint8_t* rgb8;
} LumenGpuImage;

/* Frame counters read back by lumen_gpu_read_counts. error_flags bits:
 * 1 = instances exceeded instance_capacity (outputs invalid; re-run with a
 *     larger frame), 2 = a bounded spin-wait gave up (outputs invalid),
 * 4 = invalid launch parameters, 8 = a device-side index check failed.
 * sorted_buffer: which of keys/vals [0] or [1] holds the tile-sorted
 * instances; depth_sorted_buffer: the same for depth_keys/depth_order.
 * varying_digits: bit d set when byte d of the tile ids varies, bit 8+d when
 * byte d of the depth keys varies (only those digit passes run). */
typedef struct {
    int64_t n_visible;
    int64_t n_instances;
    uint32_t error_flags;
    uint32_t sorted_buffer;
    uint32_t varying_digits;
    uint32_t touched_tiles;
    uint32_t depth_sorted_buffer;
    uint32_t reserved;
} LumenGpuCounts;

#define LUMEN_GPU_ERR_CAPACITY 1u
#define LUMEN_GPU_ERR_SPIN_TIMEOUT 2u
#define LUMEN_GPU_ERR_LAUNCH 4u
#define LUMEN_GPU_ERR_BOUNDS 8u   /* a device-side index check failed; the access was skipped */

/* Bytes of scratch a frame needs (control block, look-back descriptors,
 * digit histograms). */
size_t lumen_gpu_scratch_bytes(int64_t n_gaussians, int64_t instance_capacity, int64_t n_tiles);

/* Enqueue the whole forward on `stream`: project + cull + SH + compacting
 * scan + key emit, histogram, stable LSD digit passes, tile ranges,
 * compositing. Does not wait. */
LumenStatus lumen_gpu_render_forward(const LumenGpuGaussians* gaussians, const LumenViewCamera* camera,
                                     const LumenRenderOptions* options, LumenGpuFrame* frame,
                                     LumenGpuImage* image, void* stream);

/* Wait for `stream`, then read the frame counters. */
LumenStatus lumen_gpu_read_counts(const LumenGpuFrame* frame, LumenGpuCounts* counts, void* stream);

/* A renderer owns its work buffers and grows them on demand. */
typedef struct LumenGpuRenderer LumenGpuRenderer;
LumenGpuRenderer* lumen_gpu_renderer_create(void);
void lumen_gpu_renderer_destroy(LumenGpuRenderer* renderer);
/* Render and wait; re-runs once with larger buffers if the instance count
 * exceeded the current capacity. */
LumenStatus lumen_gpu_renderer_render(LumenGpuRenderer* renderer, const LumenGpuGaussians* gaussians,
                                      const LumenViewCamera* camera, const LumenRenderOptions* options,
                                      LumenGpuImage* image, LumenGpuCounts* counts, void* stream);
/* The renderer's frame (valid after a render; for inspection and backward). */
const LumenGpuFrame* lumen_gpu_renderer_frame(const LumenGpuRenderer* renderer);

/* The reference's sorted 64-bit keys (tile << 32 | depth key), rebuilt from
 * a finished frame's tile-sorted instances: out[i] for i < n_instances.
 * For inspection and parity checks; the pipeline itself never forms them.
 * Waits. */
LumenStatus lumen_gpu_frame_sorted_keys64(const LumenGpuFrame* frame, const LumenRenderOptions* options,
                                          uint64_t* out, void* stream);

/* Stable sort of n (key, value) pairs by key, in place in keys[0]/vals[0]
 * with keys[1]/vals[1] as the alternate buffers; the sorted data ends in the
 * set named by *sorted_buffer (device-side digit skipping decides). The
 * scratch must hold lumen_gpu_scratch_bytes(0, n, 0) bytes. Waits. */
LumenStatus lumen_gpu_sort_pairs(uint64_t* keys0, uint32_t* vals0, uint64_t* keys1, uint32_t* vals1,
                                 int64_t n, void* scratch, size_t scratch_bytes, uint32_t* sorted_buffer,
                                 void* stream);

/* Stage timing with CUDA events on the render stream. A timer holds events
 * for up to max_frames frames; each lumen_gpu_render_forward_timed call
 * records 5 events (before K1, after K1, after the sort, after the ranges,
 * after compositing) into the next frame slot without waiting.
 * lumen_gpu_stage_timer_read waits for the last event and returns the summed
 * milliseconds of the 4 stages over the recorded frames, then resets.
 * No counterpart in the reference (its timers are perf_counter_ns and clock(),
 * src/main.mojo:105-108, c_api/src/lumen_c.c:389,561). */
typedef struct LumenGpuStageTimer LumenGpuStageTimer;
LumenGpuStageTimer* lumen_gpu_stage_timer_create(int max_frames);
void lumen_gpu_stage_timer_destroy(LumenGpuStageTimer* timer);
LumenStatus lumen_gpu_render_forward_timed(const LumenGpuGaussians* gaussians, const LumenViewCamera* camera,
                                           const LumenRenderOptions* options, LumenGpuFrame* frame,
                                           LumenGpuImage* image, LumenGpuStageTimer* timer, void* stream);
LumenStatus lumen_gpu_stage_timer_read(LumenGpuStageTimer* timer, float stage_ms[4], float* total_ms,
                                       int* n_frames);

/* Launch parameters of the forward; none of them changes any output.
 * composite_chunk: sorted instances the compositor stages per round (128,
 * 256 or 512); *_sort_items: keys per thread in a digit pass of the depth
 * and tile sorts (depth: 8 or 16; tile: 8, 16 or 24 — tiles of 2048, 4096
 * or 6144 keys). Defaults 512, 16, 16. */
typedef struct {
    int32_t composite_chunk;
    int32_t depth_sort_items;
    int32_t tile_sort_items;
} LumenGpuLaunch;

/* lumen_gpu_render_forward with chosen launch parameters; with a stage
 * timer (may be NULL) it records stage events like the timed entry point. */
LumenStatus lumen_gpu_render_forward_ex(const LumenGpuGaussians* gaussians, const LumenViewCamera* camera,
                                        const LumenRenderOptions* options, const LumenGpuLaunch* launch,
                                        LumenGpuFrame* frame, LumenGpuImage* image, LumenGpuStageTimer* timer,
                                        void* stream);

/* ---------------------------------------------------------------- batches
 * Several views rendered by one pipeline: one projection over all views'
 * Gaussians, one depth sort, one tile sort whose 32-bit keys are batch-wide
 * tile ids (the view's first tile id + ty * tiles_x + tx, so the view id is
 * the key's high part), one range pass and one persistent compositor. A
 * view's image is identical to rendering it alone: within a (view, tile) the
 * instances are ordered by (depth key, visible index) either way, and the
 * visible indices of a view keep its Gaussian order.
 * No counterpart in the reference, which renders one camera per call
 * (pipeline.mojo:48-231). */
typedef struct {
    LumenGpuGaussians gaussians;    /* views may share a scene or not */
    LumenViewCamera camera;         /* views may differ in resolution */
    int32_t reserved;
    LumenGpuImage image;            /* this view's outputs ([H,W,3] rgb required) */
} LumenGpuBatchView;

/* Buffer lengths a batch needs: slots = sum over views of count rounded up
 * to a multiple of 128 (length of records, visible_ids, radii, rects,
 * depth_keys, depth_order; radii may be NULL in a batch frame, else
 * radii[slot] with slot = the slots of the views before + i), tiles = sum
 * over views of their tiles (ranges holds 2 * tiles). */
LumenStatus lumen_gpu_batch_sizes(const LumenGpuBatchView* views, int32_t n_views, int64_t* slots, int64_t* tiles);
size_t lumen_gpu_batch_scratch_bytes(int64_t slots, int64_t instance_capacity, int32_t n_views);
/* Enqueue a batch on `stream` (no host sync; the view list is copied before
 * the call returns). Counts and error flags: lumen_gpu_read_counts. */
LumenStatus lumen_gpu_render_batch(const LumenGpuBatchView* views, int32_t n_views, const LumenRenderOptions* options,
                                   LumenGpuFrame* frame, void* stream);
LumenStatus lumen_gpu_render_batch_timed(const LumenGpuBatchView* views, int32_t n_views,
                                         const LumenRenderOptions* options, LumenGpuFrame* frame,
                                         LumenGpuStageTimer* timer, void* stream);

/* The device camera lumen_rasterize uses for a look-at LumenCamera and a
 * width x height frame: fx = fy = H / (2 tan(fov_y / 2)), principal point
 * (W/2, H/2) (c_api/src/lumen_c.c:393-395,422-423), rotation with camera z
 * toward the target, x right and y down ("up" is up in the image), near and
 * far planes as given (lumen_rasterize passes the rasterizer config's). No
 * counterpart in the reference, which builds an OpenGL view matrix inline
 * (lumen_c.c:353-369,397). */
LumenStatus lumen_gpu_camera_from_lookat(const LumenCamera* camera, uint32_t width, uint32_t height,
                                         float near_plane, float far_plane, LumenViewCamera* out);

/* ------------------------------------------------------------- backward -- */

/* Gradient outputs, device memory, same layouts as LumenGpuGaussians:
 * means [N,3], scales [N,3], quats [N,4], opacities [N], sh [N,48]. When the
 * forward ran with params_are_logits, scales and opacities receive the
 * gradients of the log-scales and the opacity logits. splat2d is a work
 * buffer of N x 12 floats, 16-byte aligned (per-Gaussian gradients of the
 * 2-D splat: centre, conic, opacity, colour, depth, 2 unused), zeroed by
 * the call. */
typedef struct {
    float* means;
    float* scales;
    float* quats;
    float* opacities;
    float* sh;
    float* splat2d;
} LumenGpuGradients;

/* Gradients of a scalar loss L through the forward that filled `frame`
 * and `forward_image` (same gaussians, camera and options; neither reused
 * since). forward_image needs rgb, alpha and last_idx (and depth when
 * grad_depth is given with compute_depth). grad_rgb [H,W,3] = dL/d rgb is
 * required; grad_depth and grad_alpha ([H,W] each) may be NULL. Per tile,
 * each pixel's splats are walked front to back up to its last-visited
 * instance: the transmittance before every splat is recomputed (nothing
 * per splat is stored by the forward), the forward's skip and clamp
 * decisions are taken again exactly, and the colour blended behind a splat
 * is the forward's output minus the running sum. No counterpart in the reference:
 * it has no analytic backward (src/optim/gradients.mojo:11-106 stores
 * gradients, src/optim/trainer.mojo:61-66 injects placeholders). Does not
 * wait. */
LumenStatus lumen_gpu_render_backward(const LumenGpuGaussians* gaussians, const LumenViewCamera* camera,
                                      const LumenRenderOptions* options, const LumenGpuFrame* frame,
                                      const LumenGpuImage* forward_image, const float* grad_rgb,
                                      const float* grad_depth, const float* grad_alpha, LumenGpuGradients* grads,
                                      void* stream);
/* lumen_gpu_render_backward with CUDA events on its stream for the timer's
 * next frame (see lumen_gpu_stage_timer_create): stage 0 = the compositing
 * adjoint (with the clearing of splat2d), stage 1 = the projection
 * adjoint, stages 2 and 3 empty. No counterpart in the reference. */
LumenStatus lumen_gpu_render_backward_timed(const LumenGpuGaussians* gaussians, const LumenViewCamera* camera,
                                            const LumenRenderOptions* options, const LumenGpuFrame* frame,
                                            const LumenGpuImage* forward_image, const float* grad_rgb,
                                            const float* grad_depth, const float* grad_alpha,
                                            LumenGpuGradients* grads, LumenGpuStageTimer* timer, void* stream);

/* Mean L1 loss and its subgradient, compute_l1_loss (src/optim/loss.mojo:11-35):
 * loss = mean |pred - target|, grad[i] = +1/n if pred[i] - target[i] >= 0
 * else -1/n. loss is one device float; scratch holds
 * lumen_gpu_l1_loss_scratch_bytes() bytes (per-block partial sums, summed in
 * a fixed order so the loss is deterministic). Does not wait. */
size_t lumen_gpu_l1_loss_scratch_bytes(void);
LumenStatus lumen_gpu_l1_loss(const float* pred, const float* target, int64_t n, float* grad, float* loss,
                              void* scratch, void* stream);

/* Stable in-place sort of n (uint64 key, uint32 value) pairs that allocates
 * nothing. No counterpart in the reference. For callers that cannot call
 * cudaMalloc: code inside a host application that owns all device memory
 * (an engine plugin, an FFI host with its own allocator), or a frame loop
 * that must not allocate because allocation can synchronise the device.
 * The caller passes keys and vals (device memory) and gets them back sorted;
 * the sort's own work memory is a static device array of the library sized
 * for LUMEN_GPU_NOALLOC_MAX_PAIRS pairs (about 3.6 MB per GPU that loads the
 * library, kept until exit). Larger n returns LUMEN_ERROR_INVALID_ARGUMENT.
 * The first call on a device looks up the array's device address (make it
 * before any stream capture). All calls share the array: calls that overlap
 * on the GPU race and must be serialised by the caller. Waits for `stream`. */
#define LUMEN_GPU_NOALLOC_MAX_PAIRS 262144
LumenStatus lumen_gpu_sort_pairs_noalloc(uint64_t* keys, uint32_t* vals, int64_t n, void* stream);

/* Append n splats to a cloud in one copy. No counterpart in the reference:
 * the bulk form of lumen_cloud_add_gaussian (c_api/include/lumen.h:129),
 * with the same growth rule and error codes. */
LumenStatus lumen_cloud_append(LumenCloud* cloud, const LumenGaussian* gaussians, size_t n);

#ifdef __cplusplus
}
#endif
#endif /* LUMEN_GPU_H */
