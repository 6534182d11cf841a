/*
 * lumen_spatial.h - picking: Morton codes, the LBVH and closest-splat ray
 * casts, on the device.
 *
 * Reference (paths relative to the reference project):
 *   lumen_gpu_bvh_build    LBVH.build_from_cloud, src/spatial/bvh.mojo:45-120:
 *                          30-bit Morton codes of the positions normalised to
 *                          the cloud's bounding box (src/spatial/morton.mojo:7-46,
 *                          the box as GaussianCloud.add_gaussian tracks it,
 *                          src/scene/gaussian_cloud.mojo:21-42), a stable sort
 *                          by code (radix_sort_64bit, src/raster/radix_sort.mojo),
 *                          one leaf per Gaussian in code order with the box
 *                          position +- 3 x its largest scale, then parents that
 *                          pair adjacent nodes level by level up to one root
 *                          (AABB3f.expand_box, src/spatial/aabb.mojo:55-66)
 *   lumen_gpu_raycast      raycast_closest_splat, src/spatial/raycast.mojo:30-95,
 *                          one ray per thread (rays are normalised as Ray3f does,
 *                          src/scene/camera.mojo:12-21; slab test AABB3f.intersect_ray,
 *                          aabb.mojo:68-98)
 *   lumen_gpu_pick_pixels  PinholeCamera.generate_ray, camera.mojo:85-90, followed
 *                          by raycast_closest_splat, for a batch of pixel positions
 *
 * Node layout and numbering are the reference's: nodes[0 .. n) are the leaves
 * in Morton order, then each level's parents follow, the root last.
 */
#ifndef LUMEN_SPATIAL_H
#define LUMEN_SPATIAL_H

#include "lumen_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One node (32 bytes). Leaves have left_child = right_child = -1; a parent
 * without a right child (the last of an odd level) has right_child = -1. */
typedef struct {
    float min_pt[3];
    int32_t left_child;
    float max_pt[3];
    int32_t right_child;
} LumenBvhNode;

typedef struct {
    LumenBvhNode* nodes;      /* device, lumen_bvh_node_count(n) entries */
    int32_t* splat_index;     /* device, n entries: the Gaussian of leaf i */
    int64_t leaf_count;       /* set by the build */
    int64_t node_count;       /* set by the build */
    int64_t root_index;       /* set by the build: node_count - 1, or -1 when empty */
} LumenGpuBvh;

typedef struct {
    float origin[3];
    float direction[3];       /* any length; normalised before the cast (Ray3f) */
} LumenRay;

/* RayHit (raycast.mojo:11-27): hit 0 leaves splat_index -1, point (0, 0, 0)
 * and distance = max_dist (1e9 when the hierarchy is empty). */
typedef struct {
    int32_t hit;
    int32_t splat_index;
    float distance;
    float point[3];
} LumenRayHit;

/* Nodes of the hierarchy over n leaves (0 for n = 0). */
int64_t lumen_bvh_node_count(int64_t n);
size_t lumen_gpu_bvh_scratch_bytes(int64_t n);

/* Builds the hierarchy over gaussians (means and scales are read) into bvh
 * (nodes and splat_index allocated by the caller). scratch: device memory of
 * lumen_gpu_bvh_scratch_bytes(n) bytes. Waits for the build, to report
 * device-side errors. n below 2^30. */
LumenStatus lumen_gpu_bvh_build(const LumenGpuGaussians* gaussians, LumenGpuBvh* bvh, void* scratch,
                                size_t scratch_bytes, void* stream);

/* The closest Gaussian along each of n_rays rays (device arrays). The
 * hierarchy must have been built over these gaussians. Does not wait. */
LumenStatus lumen_gpu_raycast(const LumenGpuBvh* bvh, const LumenGpuGaussians* gaussians, const LumenRay* rays,
                              int64_t n_rays, float max_dist, LumenRayHit* hits, void* stream);

/* Picks at n pixel positions (device float pairs x, y): the camera ray
 * through each (generate_ray), then the closest Gaussian along it. rays may
 * be NULL; when given, the generated rays are written there. Does not wait. */
LumenStatus lumen_gpu_pick_pixels(const LumenGpuBvh* bvh, const LumenGpuGaussians* gaussians,
                                  const LumenViewCamera* camera, const float* pixels_xy, int64_t n, float max_dist,
                                  LumenRay* rays, LumenRayHit* hits, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LUMEN_SPATIAL_H */
