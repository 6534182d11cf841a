/*
 * lumen_serve.h - a render server over resident scenes (B200, sm_100a).
 *
 * No counterpart in the reference, which renders one camera per synchronous
 * call (lumen_rasterize, c_api/include/lumen.h:153-159; rasterize_scene,
 * src/raster/pipeline.mojo:48-52). The server keeps scenes in device memory
 * and renders requests (scene, camera, resolution) with continuous
 * batching:
 *
 *  - requests queue in arrival order; a scheduler thread admits them into a
 *    batch while the batch fits a slot's work buffers (projection slots,
 *    tiles, an instance estimate learned per scene and resolution, output
 *    pixels) and max_views_per_batch, and while its tiles number at most
 *    65 536 (unless one view alone has more): batch-wide tile ids then sort
 *    in two digit passes, where one tile more would add a third pass over
 *    every instance of the batch;
 *  - up to max_batches_in_flight batches are on the device at once, each on
 *    its own stream with its own buffers, so a batch admitted while others
 *    run overlaps with them; a slot is reused as soon as its batch is done;
 *  - a batch is rendered by the multi-view pipeline (lumen_gpu_render_batch
 *    semantics: every view equals rendering it alone) as one launch of a
 *    captured CUDA graph whose persistent kernels read the batch from a
 *    device view table, then each view's bytes are copied to its request's
 *    host buffer;
 *  - the compositor chunk and the digit-pass tile size of each batch are
 *    chosen by an autotuner that times the variants on live batches (they
 *    do not change any result) per batch size class;
 *  - a batch whose instances exceeded the estimate is re-queued at the
 *    front with raised estimates (its requests are then re-admitted, in
 *    smaller batches if needed); a request that cannot fit an empty slot
 *    completes with LUMEN_ERROR_OUT_OF_MEMORY.
 *
 * Output per request: rgb8 [H,W,3] bytes, (uint8)(clamp(c,0,1)*255) of the
 * composited colour (c_api/src/lumen_c.c:541-543 on a cleared frame). The
 * host buffer should be page-locked for the copy to be asynchronous.
 */
#ifndef LUMEN_SERVE_H
#define LUMEN_SERVE_H

#include "lumen_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct LumenServer LumenServer;

typedef struct {
    int64_t work_budget_bytes;      /* device memory for all slots' work buffers (scenes excluded) */
    int32_t max_views_per_batch;    /* >= 1 */
    int32_t max_batches_in_flight;  /* slots (streams with their own buffers), >= 1 */
    int32_t use_graphs;             /* 1: one CUDA graph launch per batch; 0: plain launches */
    int32_t autotune;               /* 1: pick launch parameters per batch class by timing */
    int32_t composite_chunk;        /* fixed choice when autotune is 0: 128, 256 or 512 */
    int32_t sort_items;             /* fixed choice when autotune is 0: keys per thread of the
                                       tile sort's digit passes, 8 or 16 (the depth sort uses 8) */
    LumenRenderOptions options;     /* shared by every request */
} LumenServerConfig;

typedef struct {
    uint64_t request_id;
    int32_t status;                 /* LumenStatus of this request */
    int32_t batch_views;            /* views in the batch that rendered it */
    double submit_ms;               /* server clock: ms since the server was created */
    double start_ms;                /* its batch was launched */
    double done_ms;                 /* its bytes were in the host buffer */
    int64_t n_instances;            /* tile instances of this view */
    int32_t composite_chunk;        /* launch parameters of its batch */
    int32_t sort_items;             /* of the tile sort */
} LumenServeResult;

typedef struct {
    uint64_t submitted;
    uint64_t completed;
    uint64_t batches;
    uint64_t requeued_batches;      /* re-run after exceeding the instance estimate */
    uint64_t rejected;              /* could not fit an empty slot */
    uint64_t graph_launches;
    double device_ms;               /* sum of batch device times */
    int64_t slot_bytes;             /* work buffers of one slot */
    int64_t max_slots, max_tiles, max_instances, max_pixels;   /* per-batch capacities */
    uint64_t explored_batches;      /* batches whose launch variant was an autotuner exploration */
} LumenServeStats;

/* Defaults: 8 GiB budget, 64 views, 2 batches in flight, graphs and
 * autotuning on, chunk 256, 16 tile-sort items, alpha >= 0.99 termination. */
LumenServerConfig lumen_server_default_config(void);
/* On the current device. NULL on failure (bad config, no device, memory). */
LumenServer* lumen_server_create(const LumenServerConfig* config);
/* Waits for the batches in flight; requests still queued complete with
 * LUMEN_ERROR_UNINITIALIZED. */
void lumen_server_destroy(LumenServer* server);
/* A resident scene: the device arrays stay owned by the caller and must
 * outlive the server. Returns the scene id (>= 0) or a negative LumenStatus. */
int32_t lumen_server_add_scene(LumenServer* server, const LumenGpuGaussians* gaussians);
/* Queue a render; out_rgb8 (camera->width * camera->height * 3 bytes of
 * host memory) is written before the request completes. */
LumenStatus lumen_server_submit(LumenServer* server, int32_t scene, const LumenViewCamera* camera,
                                uint8_t* out_rgb8, uint64_t* request_id);
/* Block until the request completes (timeout_ms < 0: no limit); each
 * request's result can be taken once. LUMEN_ERROR_IO_FAILURE on timeout. */
LumenStatus lumen_server_wait(LumenServer* server, uint64_t request_id, double timeout_ms,
                              LumenServeResult* result);
LumenStatus lumen_server_stats(LumenServer* server, LumenServeStats* stats);
/* Stop (frozen = 1) or resume (0) the autotuner's exploration: while
 * frozen, every batch uses the best launch variant timed so far for its
 * class (or for the nearest class with timings; the configured variant when
 * there are none) and no timing is recorded. For a measurement window
 * after a warm-up. */
LumenStatus lumen_server_freeze_tuning(LumenServer* server, int32_t frozen);

/* The admission rule alone (host only, for tests): requests given as
 * (slots, tiles, instance estimate, pixels) in queue order; writes how many
 * of them, from the front, the next batch admits (0 when the first one can
 * never fit). */
int32_t lumen_serve_admit(const int64_t* slots, const int64_t* tiles, const int64_t* instances,
                          const int64_t* pixels, int32_t n_requests, int32_t max_views, int64_t max_slots,
                          int64_t max_tiles, int64_t max_instances, int64_t max_pixels);

#ifdef __cplusplus
}
#endif

#endif /* LUMEN_SERVE_H */
