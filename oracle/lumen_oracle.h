/*
 * lumen_oracle.h - C interface of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle is a literal C++ restatement of the reference's Mojo forward
 * splatting path (src/raster/pipeline.mojo:48-231 and the math it calls).
 * It is the checker for the CUDA kernels in lumen_b200/ and the timed CPU
 * baseline; nothing in the product links, loads or calls it.
 *
 * Parity pinning: the reference's Mojo toolchain cannot run here, so the
 * oracle is pinned by the reference's own known-answer tests (the tests/ directory's
 * Mojo files, restated in tests/test_oracle_kat.py) rather than by executing the
 * reference. The exponential is lumen_expf (shared header), because Mojo's
 * exp cannot be observed; the restatement defines the bits.
 */
#ifndef LUMEN_ORACLE_H
#define LUMEN_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Camera in the reference PinholeCamera convention (src/scene/camera.mojo:24-40):
 * world_to_cam = rotation^-1 applied to (p - position); identity looks down +z,
 * image x right, y down. Same layout as LumenViewCamera in include/lumen_gpu.h. */
typedef struct {
    float position[3];
    float rotation[4];      /* w, x, y, z (normalised on construction, camera.mojo:229) */
    float fx, fy, cx, cy;
    float near_plane, far_plane;
    int32_t width, height;
} OracleCamera;

/* Same layout as LumenRenderOptions in include/lumen_gpu.h. */
typedef struct {
    float lowpass;             /* RenderConfig.lowpass_filter, 0.3 */
    int32_t sh_degree;         /* RenderConfig.max_sh_degree, 3 */
    int32_t white_background;  /* RenderConfig.white_background */
    int32_t compute_depth;     /* RenderConfig.compute_depth */
    int32_t key_mode;          /* 0: millimetre depth key (radix_sort.mojo:8-18); 1: float bits */
    int32_t term_mode;         /* 0: stop when T <= threshold (compositor.mojo:53); 1: when 1-T >= threshold */
    int32_t params_are_logits; /* 1: scales are log-scales and opacities are logits */
    int32_t tile_size;         /* 16 */
    float term_threshold;      /* mode 0: T <= this (1e-4); mode 1: 1-T >= this (0.99) */
} OracleOptions;

/* Per-visible-splat projected record, pipeline.mojo:141-149, in visible order. */
typedef struct {
    float cx, cy, depth;
    float ic00, ic01, ic11;    /* Covariance2D.inverse() */
    float r, g, b;
    float opacity;
} OracleRecord;

typedef struct {
    float* rgb;            /* [H*W*3] HWC */
    float* depth;          /* [H*W] */
    float* alpha;          /* [H*W] 1 - T */
    uint32_t* n_contrib;   /* [H*W] splats blended, terminating one included */
    int32_t* last_idx;     /* [H*W] range offset of the last instance visited, -1 if none */
    /* optional stage outputs (NULL to skip); capacities in elements */
    OracleRecord* records; int64_t records_cap;
    uint64_t* keys_unsorted; uint32_t* vals_unsorted;
    uint64_t* keys_sorted; uint32_t* vals_sorted; int64_t keys_cap;
    int32_t* ranges;       /* [T*2] start,end; (-1,-1) for empty (binning.mojo:10-28) */
    int32_t* radii;        /* [N] eigen radius, 0 for culled */
    /* results */
    int64_t n_visible;
    int64_t n_instances;
} OracleOutputs;

/* Full forward in float32. Gaussian arrays are SoA, contiguous:
 * means [N,3], scales [N,3], quats [N,4] (w,x,y,z), opacities [N], sh [N,48]
 * with sh[i*48 + coef*3 + ch]. nthreads <= 1 runs the literal single-thread
 * path; > 1 splits projection, the sort's histograms and the compositing
 * over host threads with identical results. Returns 0, or -1 when an
 * optional stage buffer is too small (the counts are still filled in). */
int oracle_render_f32(const float* means, const float* scales, const float* quats,
                      const float* opacities, const float* sh, int64_t n,
                      const OracleCamera* cam, const OracleOptions* opt,
                      OracleOutputs* out, int nthreads);

/* The same forward in float64 (for central finite differences). */
int oracle_render_f64(const double* means, const double* scales, const double* quats,
                      const double* opacities, const double* sh, int64_t n,
                      const OracleCamera* cam, const OracleOptions* opt,
                      double* rgb, double* depth, double* alpha,
                      uint64_t* decision_hash);

/* Stable 8-pass LSD radix sort of 64-bit keys with 32-bit values,
 * radix_sort.mojo:39-87. */
void oracle_radix_sort64(uint64_t* keys, uint32_t* vals, int64_t n, int nthreads);

/* Tile ranges from sorted keys, binning.mojo:51-73. ranges[T*2]. */
void oracle_tile_ranges(const uint64_t* keys, int64_t n, int64_t total_tiles, int32_t* ranges);

/* Key encoders, radix_sort.mojo:8-27. */
uint64_t oracle_encode_key(uint32_t tile_id, float depth, int key_mode);

/* L1 loss with subgradient, loss.mojo:11-35. Returns the loss. */
float oracle_l1_loss(const float* pred, const float* target, int64_t n, float* grad);

/* Unit restatements for the known-answer tests. */
void oracle_ewa_cov2d(const float cov3d[6], const float t[3], const float view_rot[9],
                      float fx, float fy, float lowpass, float out[3]);
void oracle_jacobian(const float t[3], float fx, float fy, float out[6]);
void oracle_cov3d(const float scale[3], const float quat[4], float out[6]);
void oracle_eigen2x2(const float cov[3], float out_lmax_lmin[2], int64_t* radius);
void oracle_cov2d_inverse(const float cov[3], float out[3]);
void oracle_sh_basis(const float dir[3], float out[16]);
void oracle_sh_color(const float* sh48, const float dir[3], int degree, float out[3]);
int  oracle_depth_visible(float z, float near_plane, float far_plane);
int  oracle_screen_box_visible(float cx, float cy, int64_t radius, int32_t w, int32_t h);
void oracle_world_to_screen(const OracleCamera* cam, const float p[3], float out_cam[3], float out_screen[2]);
/* PixelAccumulator.blend sequence; returns the terminated flag of the last blend. */
int  oracle_blend_sequence(const float* colors, const float* alphas, const float* depths, int n,
                           int term_mode, float out_color[3], float* out_T, float* out_depth,
                           float* out_alpha);
float oracle_pixel_alpha(float px, float py, float cx, float cy, const float icov[3], float opacity);

#ifdef __cplusplus
}
#endif
#endif
