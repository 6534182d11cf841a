/*
 * depth.cu - products of a rendered depth buffer (include/lumen_depth.h).
 *
 * Reference: DepthMap.compute_min_max and DepthMap.extract_normal
 * (src/raster/depth_map.mojo:31-68), the SDK's export_depth_visualization
 * (python/lumen/visualizer.py:16-48).
 *
 * One kernel reads each depth once (the four neighbours of the normal come
 * from L1/L2: the 8 MB buffer of a 1080p frame stays resident in the 126 MB
 * L2) and writes the requested products: 12 B of normal and 3 B of heatmap
 * per pixel, so the pass is HBM-bound at 4 + 12 + 3 = 19 B per pixel. The
 * range is reduced without a scratch buffer: the output's two words hold
 * max(~bits(d)) and max(bits(d)) over qualifying depths while the kernel
 * runs (for positive floats the bit patterns order like the values), and a
 * one-thread kernel turns them into (min, max) with the reference's initial
 * values and its (0, 1) fallback. Float arithmetic is written in the
 * reference's operation order and built with --fmad=false; the heatmap is
 * computed in double precision, as the SDK's Python floats are.
 */
#include "splat_common.cuh"
#include "../../include/lumen_depth.h"

namespace lumen {
LumenStatus map_cuda(cudaError_t e);
int device_sm_count();

namespace {

constexpr int kDepthThreads = 256;

__global__ void __launch_bounds__(kDepthThreads)
depth_products_kernel(const float* __restrict__ depth, int w, int h, float* __restrict__ normals,
                      unsigned char* __restrict__ heat, unsigned int* __restrict__ range_enc, double near_p,
                      double span) {
    __shared__ unsigned int s_lo[kDepthThreads / 32], s_hi[kDepthThreads / 32];
    unsigned int lo = 0u, hi = 0u;   /* max of ~bits (the minimum), max of bits (the maximum) */
    const long long npix = (long long)w * h;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += stride) {
        const int y = (int)(i / w);
        const int x = (int)(i - (long long)y * w);
        const float d = depth[i];
        if (d > (float)0.001) {                                        /* depth_map.mojo:37-41 */
            const unsigned int b = __float_as_uint(d);
            lo = max(lo, ~b);
            hi = max(hi, b);
        }
        if (normals) {                                                 /* depth_map.mojo:52-68 */
            const int x0 = x > 0 ? x - 1 : 0, x1 = x + 1 < w ? x + 1 : w - 1;
            const int y0 = y > 0 ? y - 1 : 0, y1 = y + 1 < h ? y + 1 : h - 1;
            const float* row = depth + (long long)y * w;
            const float dz_dx = (__ldg(row + x1) - __ldg(row + x0)) * 0.5f;
            const float dz_dy = (__ldg(depth + (long long)y1 * w + x) - __ldg(depth + (long long)y0 * w + x)) * 0.5f;
            const float nx = -dz_dx, ny = -dz_dy, nz = 1.0f;
            const float l = sqrtf(nx * nx + ny * ny + nz * nz);       /* vector.mojo:100-110 */
            float ox = 0.0f, oy = 0.0f, oz = 0.0f;
            if (l > (float)0.000001) {
                ox = nx / l;
                oy = ny / l;
                oz = nz / l;
            }
            normals[i * 3 + 0] = ox;
            normals[i * 3 + 1] = oy;
            normals[i * 3 + 2] = oz;
        }
        if (heat) {                                                    /* visualizer.py:28-46 */
            const double dd = (double)d;
            double norm = 1.0;
            if (!(dd >= 999.0 || dd <= 0.0)) {
                norm = (dd - near_p) / span;
                norm = norm < 1.0 ? norm : 1.0;       /* min(1.0, norm): 1.0 unless norm < 1 (also for NaN) */
                norm = norm > 0.0 ? norm : 0.0;       /* max(0.0, norm) */
            }
            const int inten = (int)((1.0 - norm) * 255.0);
            const int r = inten;
            const int g = (int)((double)inten * 0.8);
            const int b = (int)(255.0 - (double)inten * 0.7);
            heat[i * 3 + 0] = (unsigned char)max(0, min(255, r));
            heat[i * 3 + 1] = (unsigned char)max(0, min(255, g));
            heat[i * 3 + 2] = (unsigned char)max(0, min(255, b));
        }
    }
    if (!range_enc) return;
    lo = __reduce_max_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_lo[warp] = lo;
        s_hi[warp] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kDepthThreads / 32; ++k) {
            lo = max(lo, s_lo[k]);
            hi = max(hi, s_hi[k]);
        }
        if (lo) atomicMax(range_enc, lo);
        if (hi) atomicMax(range_enc + 1, hi);
    }
}

/* depth_map.mojo:32-46: min from 1e9, max from -1e9, (0, 1) when empty */
__global__ void depth_range_finish_kernel(float* range) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const unsigned int* enc = reinterpret_cast<const unsigned int*>(range);
    const unsigned int lo = enc[0], hi = enc[1];
    float mn = (float)1e9, mx = (float)-1e9;
    if (lo) {
        const float v = __uint_as_float(~lo);
        if (v < mn) mn = v;
    }
    if (hi) {
        const float v = __uint_as_float(hi);
        if (v > mx) mx = v;
    }
    if (mn > mx) {
        mn = 0.0f;
        mx = 1.0f;
    }
    range[0] = mn;
    range[1] = mx;
}

}  // namespace
}  // namespace lumen

using namespace lumen;

extern "C" {

LumenStatus lumen_gpu_depth_products(const float* depth, int32_t width, int32_t height,
                                     const LumenDepthProducts* out, void* stream) {
    if (!depth || !out || width <= 0 || height <= 0) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (((uintptr_t)depth | (uintptr_t)out->normals | (uintptr_t)out->range) & 3u) return LUMEN_ERROR_INVALID_ARGUMENT;
    const double span = out->far_plane - out->near_plane;
    if (out->heatmap && span == 0.0) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (!out->normals && !out->range && !out->heatmap) return LUMEN_SUCCESS;
    cudaStream_t s = (cudaStream_t)stream;
    if (out->range) {
        const cudaError_t e = cudaMemsetAsync(out->range, 0, 2 * sizeof(float), s);
        if (e != cudaSuccess) return map_cuda(e);
    }
    const long long npix = (long long)width * height;
    long long grid = (npix + kDepthThreads - 1) / kDepthThreads;
    const long long cap = (long long)device_sm_count() * 8;
    if (grid > cap) grid = cap;
    depth_products_kernel<<<(unsigned int)grid, kDepthThreads, 0, s>>>(
        depth, width, height, out->normals, out->heatmap, reinterpret_cast<unsigned int*>(out->range),
        out->near_plane, span);
    if (out->range) depth_range_finish_kernel<<<1, 32, 0, s>>>(out->range);
    return map_cuda(cudaGetLastError());
}

}  // extern "C"
