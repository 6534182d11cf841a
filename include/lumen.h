/*
 * lumen.h - the liblumen C interface, served by the B200 pipeline.
 *
 * This header keeps the reference library's binary interface unchanged
 * (reference: c_api/include/lumen.h:1-165): the same 22 exported functions,
 * the same struct layouts and the same status codes, so a program or an FFI
 * binding written against the reference links against this library as is.
 * What changes is behind lumen_rasterize: it runs the GPU splatting pipeline
 * (EWA projection, degree-3 SH, 16x16 tile binning, stable radix sort, tile
 * ranges, front-to-back compositing) instead of the reference's isotropic
 * CPU approximation. Device-resident entry points live in lumen_gpu.h.
 *
 * Each declaration cites the reference line it replaces.
 */
#ifndef LUMEN_H
#define LUMEN_H

#ifdef __cplusplus
extern "C" {
#endif

#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

/* reference lumen.h:23-26 */
#define LUMEN_VERSION_MAJOR 0
#define LUMEN_VERSION_MINOR 1
#define LUMEN_VERSION_PATCH 0
#define LUMEN_VERSION_STRING "0.1.0"

/* Status codes, reference lumen.h:29-36. Every entry point returns one of
 * these; CUDA failures map to LUMEN_ERROR_OUT_OF_MEMORY (allocation) or
 * LUMEN_ERROR_UNINITIALIZED (no usable device). Nothing aborts. */
typedef enum {
    LUMEN_SUCCESS = 0,
    LUMEN_ERROR_INVALID_ARGUMENT = -1,
    LUMEN_ERROR_OUT_OF_MEMORY = -2,
    LUMEN_ERROR_UNINITIALIZED = -3,
    LUMEN_ERROR_IO_FAILURE = -4,
    LUMEN_ERROR_MATH_SINGULAR = -5
} LumenStatus;

/* Rasterizer settings, reference lumen.h:39-47 (28 bytes).
 * image_width/height are informational (the frame buffer decides the size);
 * near_plane/far_plane bound the visible depth; tile_size must be 16; a
 * pixel stops compositing once its accumulated alpha 1 - T reaches
 * early_termination_alpha (0.99 by default); gaussian_radius_sigma is kept for
 * layout (the footprint radius is always the 3-sigma eigenvalue radius). */
typedef struct {
    uint32_t image_width;
    uint32_t image_height;
    uint32_t tile_size;
    float near_plane;
    float far_plane;
    float early_termination_alpha;
    float gaussian_radius_sigma;
} LumenConfig;

/* reference lumen.h:50-54 */
typedef struct {
    float x;
    float y;
    float z;
} LumenVec3;

/* reference lumen.h:57-62 (w first) */
typedef struct {
    float w;
    float x;
    float y;
    float z;
} LumenQuat;

/* Look-at pinhole camera, reference lumen.h:65-73. The vertical field of
 * view sets fx = fy = H / (2 tan(fov_y/2)) with the principal point at the
 * image centre; "up" points up in the image. */
typedef struct {
    LumenVec3 position;
    LumenVec3 target;
    LumenVec3 up;
    float fov_x_degrees;
    float fov_y_degrees;
    float near_plane;
    float far_plane;
} LumenCamera;

/* One splat, reference lumen.h:76-82 (236 bytes): position, linear scale,
 * rotation (w,x,y,z), opacity in [0,1], SH coefficients sh[coef*3 + ch]. */
typedef struct {
    LumenVec3 position;
    LumenVec3 scale;
    LumenQuat rotation;
    float opacity;
    float sh_coeffs[48];
} LumenGaussian;

/* Host frame buffer, reference lumen.h:85-91. rgb is 8-bit HWC, depth is the
 * alpha-weighted depth (1000 where nothing was drawn), alpha is 1 - T. */
typedef struct {
    uint32_t width;
    uint32_t height;
    uint8_t* rgb_data;
    float* depth_data;
    float* alpha_data;
} LumenFrameBuffer;

/* reference lumen.h:94-102. rasterize_time_ms is GPU time (CUDA events) of
 * the render, upload and read-back included. */
typedef struct {
    size_t total_splats;
    size_t visible_splats;
    size_t culled_splats;
    size_t total_tiles;
    size_t touched_tiles;
    float rasterize_time_ms;
    float frames_per_second;
} LumenStats;

typedef struct LumenCloud LumenCloud;             /* reference lumen.h:105 */
typedef struct LumenRasterizer LumenRasterizer;   /* reference lumen.h:106 */

/* reference lumen.h:112-115 */
const char* lumen_get_version(void);
int lumen_get_version_major(void);
int lumen_get_version_minor(void);
int lumen_get_version_patch(void);

/* reference lumen.h:118; defaults of c_api/src/lumen_c.c:67-77 */
LumenConfig lumen_default_config(void);

/* Host-side cloud with a device mirror refreshed on the next render after
 * any change. reference lumen.h:124-131 */
LumenCloud* lumen_cloud_create(size_t initial_capacity);
void lumen_cloud_destroy(LumenCloud* cloud);
LumenStatus lumen_cloud_reserve(LumenCloud* cloud, size_t new_capacity);
size_t lumen_cloud_get_count(const LumenCloud* cloud);
size_t lumen_cloud_get_capacity(const LumenCloud* cloud);
LumenStatus lumen_cloud_add_gaussian(LumenCloud* cloud, const LumenGaussian* gaussian);
LumenStatus lumen_cloud_get_gaussian(const LumenCloud* cloud, size_t index, LumenGaussian* out_gaussian);
void lumen_cloud_clear(LumenCloud* cloud);

/* reference lumen.h:134-135 */
LumenCloud* lumen_create_synthetic_cube(size_t points_per_axis, float cube_size);
LumenCloud* lumen_create_synthetic_sphere(size_t point_count, float radius);

/* reference lumen.h:141-143 */
LumenFrameBuffer* lumen_framebuffer_create(uint32_t width, uint32_t height);
void lumen_framebuffer_destroy(LumenFrameBuffer* fb);
void lumen_framebuffer_clear(LumenFrameBuffer* fb, uint8_t r, uint8_t g, uint8_t b);

/* A rasterizer owns a CUDA stream and its device work buffers; calls on
 * different rasterizers are independent. reference lumen.h:149-151 */
LumenRasterizer* lumen_rasterizer_create(const LumenConfig* config);
void lumen_rasterizer_destroy(LumenRasterizer* rasterizer);
LumenStatus lumen_rasterizer_set_config(LumenRasterizer* rasterizer, const LumenConfig* config);

/* Render cloud through camera into out_framebuffer (its width and height set
 * the resolution). reference lumen.h:153-159 */
LumenStatus lumen_rasterize(
    LumenRasterizer* rasterizer,
    const LumenCloud* cloud,
    const LumenCamera* camera,
    LumenFrameBuffer* out_framebuffer,
    LumenStats* out_stats
);

#ifdef __cplusplus
}
#endif

#endif /* LUMEN_H */
