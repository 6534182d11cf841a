/*
 * depth_oracle.cpp - CPU restatement of the reference's depth-buffer products
 * (TEST INFRASTRUCTURE ONLY: the checker for lumen_b200/csrc/depth.cu).
 *
 *   oracle_depth_min_max  DepthMap.compute_min_max, src/raster/depth_map.mojo:31-46
 *   oracle_depth_normal   DepthMap.extract_normal, depth_map.mojo:48-68, with
 *                         DepthMap.get_depth (:22-25) and Vec3f.normalized
 *                         (src/math/vector.mojo:100-110)
 *   oracle_depth_heatmap  the per-pixel colour of export_depth_visualization,
 *                         python/lumen/visualizer.py:16-46, in double precision
 *                         (the SDK's Python floats) with Python's int(),
 *                         min() and max() semantics written out
 *
 * Float32 arithmetic in the reference's operation order, no contraction
 * (-ffp-contract=off).
 */
#include <cmath>
#include <cstdint>

namespace {

float get_depth(const float* d, int32_t w, int32_t h, int32_t x, int32_t y) {
    if (x >= 0 && x < w && y >= 0 && y < h) return d[(int64_t)y * w + x];
    return 0.0f;
}

int py_clamp255(int v) {          /* max(0, min(255, v)) */
    const int m = 255 < v ? 255 : v;
    return 0 > m ? 0 : m;
}

}  // namespace

extern "C" {

void oracle_depth_min_max(const float* d, int64_t n, float* out_min, float* out_max) {
    float min_val = (float)1e9;
    float max_val = (float)-1e9;
    for (int64_t i = 0; i < n; ++i) {
        const float v = d[i];
        if (v > (float)0.001) {
            if (v < min_val) min_val = v;
            if (v > max_val) max_val = v;
        }
    }
    if (min_val > max_val) {
        min_val = 0.0f;
        max_val = 1.0f;
    }
    *out_min = min_val;
    *out_max = max_val;
}

void oracle_depth_normal(const float* d, int32_t w, int32_t h, int32_t x, int32_t y, float out[3]) {
    int32_t x0 = x - 1;
    if (x0 < 0) x0 = 0;
    int32_t x1 = x + 1;
    if (x1 >= w) x1 = w - 1;
    int32_t y0 = y - 1;
    if (y0 < 0) y0 = 0;
    int32_t y1 = y + 1;
    if (y1 >= h) y1 = h - 1;
    const float dz_dx = (get_depth(d, w, h, x1, y) - get_depth(d, w, h, x0, y)) * 0.5f;
    const float dz_dy = (get_depth(d, w, h, x, y1) - get_depth(d, w, h, x, y0)) * 0.5f;
    const float nx = -dz_dx, ny = -dz_dy, nz = 1.0f;
    const float l = std::sqrt(nx * nx + ny * ny + nz * nz);
    if (l > (float)0.000001) {
        out[0] = nx / l;
        out[1] = ny / l;
        out[2] = nz / l;
    } else {
        out[0] = out[1] = out[2] = 0.0f;
    }
}

void oracle_depth_normals(const float* d, int32_t w, int32_t h, float* out) {
    for (int32_t y = 0; y < h; ++y)
        for (int32_t x = 0; x < w; ++x) oracle_depth_normal(d, w, h, x, y, out + ((int64_t)y * w + x) * 3);
}

void oracle_depth_heatmap(const float* d, int64_t n, double near_plane, double far_plane, uint8_t* rgb) {
    for (int64_t i = 0; i < n; ++i) {
        const double v = (double)d[i];
        double norm_d;
        if (v >= 999.0 || v <= 0.0) {
            norm_d = 1.0;
        } else {
            norm_d = (v - near_plane) / (far_plane - near_plane);
            const double m = norm_d < 1.0 ? norm_d : 1.0;      /* min(1.0, norm_d) */
            norm_d = m > 0.0 ? m : 0.0;                        /* max(0.0, ...) */
        }
        const int intensity = (int)((1.0 - norm_d) * 255.0);
        const int r = (int)(intensity * 1.0);
        const int g = (int)(intensity * 0.8);
        const int b = (int)(255 - intensity * 0.7);
        rgb[i * 3 + 0] = (uint8_t)py_clamp255(r);
        rgb[i * 3 + 1] = (uint8_t)py_clamp255(g);
        rgb[i * 3 + 2] = (uint8_t)py_clamp255(b);
    }
}

}  // extern "C"
