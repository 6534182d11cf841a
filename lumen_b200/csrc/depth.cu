/*
 * depth.cu - products of a rendered depth buffer (include/lumen_depth.h).
 *
 * Reference: DepthMap.compute_min_max and DepthMap.extract_normal
 * (src/raster/depth_map.mojo:31-68), the SDK's export_depth_visualization
 * (python/lumen/visualizer.py:16-48).
 *
 * One kernel reads each depth once (the rows above and below come from
 * L1/L2: the 8 MB buffer of a 1080p frame stays resident in the 126 MB L2),
 * four pixels of a row per thread when the width allows 16-byte accesses,
 * and writes the requested products: 12 B of normal and 3 B of heatmap
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

/* One pixel's products from its depth and its four clamped neighbours. */
__device__ __forceinline__ void pixel_products(float d, float left, float right, float up, float down,
                                               float n_out[3], unsigned char h_out[3], double near_p, double span,
                                               unsigned int& lo, unsigned int& hi) {
    if (d > (float)0.001) {                                            /* depth_map.mojo:37-41 */
        const unsigned int b = __float_as_uint(d);
        lo = max(lo, ~b);
        hi = max(hi, b);
    }
    {                                                                  /* depth_map.mojo:52-68 */
        const float dz_dx = (right - left) * 0.5f;
        const float dz_dy = (down - up) * 0.5f;
        const float nx = -dz_dx, ny = -dz_dy, nz = 1.0f;
        const float l = sqrtf(nx * nx + ny * ny + nz * nz);           /* vector.mojo:100-110 */
        float ox = 0.0f, oy = 0.0f, oz = 0.0f;
        if (l > (float)0.000001) {
            ox = nx / l;
            oy = ny / l;
            oz = nz / l;
        }
        n_out[0] = ox;
        n_out[1] = oy;
        n_out[2] = oz;
    }
    {                                                                  /* visualizer.py:28-46 */
        const double dd = (double)d;
        double norm = 1.0;
        if (!(dd >= 999.0 || dd <= 0.0)) {
            norm = (dd - near_p) / span;
            /* max(0.0, min(1.0, norm)) in Python: 1.0 unless norm < 1, so a NaN
             * (a NaN depth) gives 1.0; the NaN test is explicit */
            if (isnan(norm) || norm >= 1.0) norm = 1.0;
            else if (norm <= 0.0) norm = 0.0;
        }
        const int inten = (int)((1.0 - norm) * 255.0);
        const int g = (int)((double)inten * 0.8);
        const int b = (int)(255.0 - (double)inten * 0.7);
        h_out[0] = (unsigned char)max(0, min(255, inten));
        h_out[1] = (unsigned char)max(0, min(255, g));
        h_out[2] = (unsigned char)max(0, min(255, b));
    }
}

/* Block reduction of the range keys into the output's two words. */
__device__ __forceinline__ void reduce_range(unsigned int lo, unsigned int hi, unsigned int* range_enc) {
    __shared__ unsigned int s_lo[kDepthThreads / 32], s_hi[kDepthThreads / 32];
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

/* Four pixels of a row per thread: one 16-byte load of the depths and of
 * the rows above and below, 16-byte stores of the normals and 4-byte stores
 * of the heatmap (width a multiple of 4, buffers aligned). */
__global__ void __launch_bounds__(kDepthThreads)
depth_products_vec4_kernel(const float* __restrict__ depth, int w, int h, float* __restrict__ normals,
                           unsigned char* __restrict__ heat, unsigned int* __restrict__ range_enc, double near_p,
                           double span) {
    unsigned int lo = 0u, hi = 0u;
    const long long nquads = (long long)w * h / 4;
    const int qpr = w / 4;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nquads; q += stride) {
        const int y = (int)(q / qpr);
        const int x0 = (int)(q - (long long)y * qpr) * 4;
        const long long i0 = (long long)y * w + x0;
        const int y0 = y > 0 ? y - 1 : 0, y1 = y + 1 < h ? y + 1 : h - 1;
        const float4 c = __ldg(reinterpret_cast<const float4*>(depth + i0));
        const float4 up = __ldg(reinterpret_cast<const float4*>(depth + (long long)y0 * w + x0));
        const float4 dn = __ldg(reinterpret_cast<const float4*>(depth + (long long)y1 * w + x0));
        const float L = x0 > 0 ? __ldg(depth + i0 - 1) : c.x;
        const float R = x0 + 4 < w ? __ldg(depth + i0 + 4) : c.w;
        const float dv[4] = {c.x, c.y, c.z, c.w}, uv[4] = {up.x, up.y, up.z, up.w}, nv[4] = {dn.x, dn.y, dn.z, dn.w};
        float nrm[12];
        unsigned char hb[12];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float left = k == 0 ? L : dv[k - 1];
            const float right = k == 3 ? R : dv[k + 1];
            pixel_products(dv[k], left, right, uv[k], nv[k], nrm + 3 * k, hb + 3 * k, near_p, span, lo, hi);
        }
        if (normals) {
            float4* o = reinterpret_cast<float4*>(normals + i0 * 3);
            o[0] = make_float4(nrm[0], nrm[1], nrm[2], nrm[3]);
            o[1] = make_float4(nrm[4], nrm[5], nrm[6], nrm[7]);
            o[2] = make_float4(nrm[8], nrm[9], nrm[10], nrm[11]);
        }
        if (heat) {
            unsigned int* o = reinterpret_cast<unsigned int*>(heat + i0 * 3);
#pragma unroll
            for (int k = 0; k < 3; ++k)
                o[k] = (unsigned int)hb[4 * k] | ((unsigned int)hb[4 * k + 1] << 8) |
                       ((unsigned int)hb[4 * k + 2] << 16) | ((unsigned int)hb[4 * k + 3] << 24);
        }
    }
    if (range_enc) reduce_range(lo, hi, range_enc);
}

__global__ void __launch_bounds__(kDepthThreads)
depth_products_kernel(const float* __restrict__ depth, int w, int h, float* __restrict__ normals,
                      unsigned char* __restrict__ heat, unsigned int* __restrict__ range_enc, double near_p,
                      double span) {
    unsigned int lo = 0u, hi = 0u;
    const long long npix = (long long)w * h;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += stride) {
        const int y = (int)(i / w);
        const int x = (int)(i - (long long)y * w);
        const int x0 = x > 0 ? x - 1 : 0, x1 = x + 1 < w ? x + 1 : w - 1;
        const int y0 = y > 0 ? y - 1 : 0, y1 = y + 1 < h ? y + 1 : h - 1;
        const float* row = depth + (long long)y * w;
        float nrm[3];
        unsigned char hb[3];
        pixel_products(row[x], __ldg(row + x0), __ldg(row + x1), __ldg(depth + (long long)y0 * w + x),
                       __ldg(depth + (long long)y1 * w + x), nrm, hb, near_p, span, lo, hi);
        if (normals) {
            normals[i * 3 + 0] = nrm[0];
            normals[i * 3 + 1] = nrm[1];
            normals[i * 3 + 2] = nrm[2];
        }
        if (heat) {
            heat[i * 3 + 0] = hb[0];
            heat[i * 3 + 1] = hb[1];
            heat[i * 3 + 2] = hb[2];
        }
    }
    if (range_enc) reduce_range(lo, hi, range_enc);
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
    const bool vec4 = width % 4 == 0 && !(((uintptr_t)depth | (uintptr_t)out->normals) & 15u) &&
                      !((uintptr_t)out->heatmap & 3u);
    const long long units = vec4 ? npix / 4 : npix;
    long long grid = (units + kDepthThreads - 1) / kDepthThreads;
    const long long cap = (long long)device_sm_count() * 8;
    if (grid > cap) grid = cap;
    unsigned int* enc = reinterpret_cast<unsigned int*>(out->range);
    if (vec4)
        depth_products_vec4_kernel<<<(unsigned int)grid, kDepthThreads, 0, s>>>(
            depth, width, height, out->normals, out->heatmap, enc, out->near_plane, span);
    else
        depth_products_kernel<<<(unsigned int)grid, kDepthThreads, 0, s>>>(
            depth, width, height, out->normals, out->heatmap, enc, out->near_plane, span);
    if (out->range) depth_range_finish_kernel<<<1, 32, 0, s>>>(out->range);
    return map_cuda(cudaGetLastError());
}

}  // extern "C"
