/*
 * lumen_depth.h - products of a rendered depth buffer, in one pass on the device.
 *
 * Reference (paths relative to the reference project):
 *   range    DepthMap.compute_min_max, src/raster/depth_map.mojo:31-46: the
 *            smallest and largest depth above 0.001 (starting from 1e9 and
 *            -1e9), or (0, 1) when no pixel qualifies
 *   normals  DepthMap.extract_normal, depth_map.mojo:48-68, at every pixel:
 *            central differences of the depth with edge-clamped neighbours,
 *            normal = normalise(-dz/dx, -dz/dy, 1) (Vec3f.normalized,
 *            src/math/vector.mojo:106-110)
 *   heatmap  export_depth_visualization, python/lumen/visualizer.py:16-48: the
 *            false-colour RGB bytes the SDK writes to its depth PPM (depths
 *            >= 999 or <= 0 are background; near is bright), computed in
 *            double precision as the SDK's Python floats are
 *
 * The depth buffer is the one lumen_gpu_render_forward writes
 * (compute_depth = 1): height x width float32, row-major.
 */
#ifndef LUMEN_DEPTH_H
#define LUMEN_DEPTH_H

#include "lumen_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    float* normals;        /* height x width x 3 float32 (x, y, z), or NULL */
    float* range;          /* 2 float32 (min, max), or NULL */
    uint8_t* heatmap;      /* height x width x 3 bytes (r, g, b), or NULL */
    double near_plane;     /* heatmap mapping; the SDK's defaults are 0.5 and 10.0 */
    double far_plane;
} LumenDepthProducts;

/* Reads the depth buffer once and writes the requested products (device
 * pointers). far_plane must differ from near_plane when heatmap is set (the
 * SDK divides by their difference). Does not wait. */
LumenStatus lumen_gpu_depth_products(const float* depth, int32_t width, int32_t height,
                                     const LumenDepthProducts* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LUMEN_DEPTH_H */
