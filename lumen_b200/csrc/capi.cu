/*
 * capi.cu - the liblumen C interface of include/lumen.h on the B200 pipeline.
 *
 * Reference: c_api/src/lumen_c.c (the 22 exported functions). Handles,
 * ownership, defaults and error codes behave as there; lumen_rasterize runs
 * the device pipeline of forward.cu instead of the reference's CPU
 * approximation.
 *
 * Semantics of lumen_rasterize (reference lumen_c.c:380-575):
 *  - the frame buffer's width and height set the resolution (:391-392);
 *  - fx = fy = H / (2 tan(fov_y / 2)), principal point (W/2, H/2) (:393-395,
 *    :422-423); near and far planes come from the rasterizer config (:416);
 *  - position/target/up become a camera rotation with z forward, x right and
 *    y down ("up" is up in the image);
 *  - the frame buffer's current contents are the background the splats are
 *    composited over: rgb = clamp(C + T * existing/255) stored as
 *    (uint8)(v * 255) by truncation (:541-543); alpha = 1 - T; depth = the
 *    alpha-weighted depth where alpha > 0, the existing value elsewhere;
 *  - a pixel stops once its accumulated alpha reaches early_termination_alpha;
 *  - stats as the reference fills them, with rasterize_time_ms measured by
 *    CUDA events around upload, render and read-back.
 */
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>

#include "splat_common.cuh"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace {

std::atomic<unsigned long long> g_generation{1};

}  // namespace

struct LumenCloud {
    LumenGaussian* data;
    size_t count;
    size_t capacity;
    unsigned long long generation;   /* changes on every mutation */
};

/* Row bands per lumen_rasterize frame (the read-back of a band overlaps
 * the compositing of the next). */
constexpr int kRasterBands = 4;

struct LumenRasterizer {
    LumenConfig config;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;   /* frame-buffer copies, overlapping the render */
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_up = nullptr, ev_down = nullptr;
    cudaEvent_t ev_band[kRasterBands] = {};   /* one per compositor band */
    LumenGpuRenderer* renderer = nullptr;
    /* device mirror of the last cloud rendered */
    const LumenCloud* cached_cloud = nullptr;
    unsigned long long cached_generation = 0;
    size_t dev_cap = 0;
    LumenGaussian* d_aos = nullptr;
    float* d_soa = nullptr;          /* means | scales | quats | opacities | sh */
    /* device image buffers */
    size_t img_cap = 0;
    float* d_rgb = nullptr;
    float* d_depth = nullptr;             /* rendered | old (uploaded) | out, npix each */
    float* d_alpha = nullptr;
    unsigned char* d_rgb8 = nullptr;      /* old (uploaded) | out, npix * 3 each */
};

namespace lumen {

LumenStatus renderer_render_banded(LumenGpuRenderer* r, const LumenGpuGaussians* g, const LumenViewCamera* cam,
                                   const LumenRenderOptions* opt, LumenGpuImage* img, LumenGpuCounts* counts,
                                   int n_bands, BandHook hook, void* ctx, cudaStream_t stream);

/* AoS LumenGaussian (59 floats) to the five SoA arrays the kernels read. */
__global__ void aos_to_soa_kernel(const float* __restrict__ aos, long long n, float* __restrict__ means,
                                  float* __restrict__ scales, float* __restrict__ quats,
                                  float* __restrict__ opac, float* __restrict__ sh) {
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n * 59; j += nthreads) {
        const long long i = j / 59;
        const int f = (int)(j - i * 59);
        const float v = aos[j];
        if (f < 3) means[i * 3 + f] = v;
        else if (f < 6) scales[i * 3 + f - 3] = v;
        else if (f < 10) quats[i * 4 + f - 6] = v;
        else if (f == 10) opac[i] = v;
        else sh[i * 48 + f - 11] = v;
    }
}

/* Float image to the 8-bit frame buffer, compositing over its old contents. */
/* Pixels [p0, p1) of the frame buffer: the render over the old contents
 * (old colour weighted by the transmittance; the rendered depth where
 * anything was blended, the old depth elsewhere). */
__global__ void to_framebuffer_kernel(const float* __restrict__ rgb, const float* __restrict__ depth,
                                      const float* __restrict__ alpha, const unsigned char* __restrict__ old8,
                                      const float* __restrict__ old_depth, unsigned char* __restrict__ out8,
                                      float* __restrict__ out_depth, long long p0, long long p1) {
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    for (long long p = p0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < p1; p += nthreads) {
        const float a = alpha[p];
        const float T = 1.0f - a;
        for (int c = 0; c < 3; ++c) {
            float v = rgb[p * 3 + c] + T * ((float)old8[p * 3 + c] / 255.0f);
            if (v < 0.0f) v = 0.0f;
            if (v > 1.0f) v = 1.0f;
            out8[p * 3 + c] = (unsigned char)(v * 255.0f);
        }
        out_depth[p] = a > 0.0f ? depth[p] : old_depth[p];
    }
}

}  // namespace lumen

using namespace lumen;

namespace {

LumenStatus cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return LUMEN_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return LUMEN_ERROR_OUT_OF_MEMORY;
    return LUMEN_ERROR_UNINITIALIZED;
}

/* Camera-to-world rotation with columns (right, down, forward), as a unit
 * quaternion (w, x, y, z) by the four-branch method. */
void look_at_rotation(const LumenVec3& eye, const LumenVec3& target, const LumenVec3& up, float q_out[4]) {
    double f[3] = {(double)target.x - eye.x, (double)target.y - eye.y, (double)target.z - eye.z};
    double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    if (fl < 1e-12) { q_out[0] = 1; q_out[1] = q_out[2] = q_out[3] = 0; return; }
    for (double& v : f) v /= fl;
    double u[3] = {up.x, up.y, up.z};
    double r[3] = {f[1] * u[2] - f[2] * u[1], f[2] * u[0] - f[0] * u[2], f[0] * u[1] - f[1] * u[0]};
    double rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (rl < 1e-12) {   /* up parallel to the view direction: any perpendicular */
        double a[3] = {1, 0, 0};
        if (std::fabs(f[0]) > 0.9) { a[0] = 0; a[1] = 1; }
        r[0] = f[1] * a[2] - f[2] * a[1]; r[1] = f[2] * a[0] - f[0] * a[2]; r[2] = f[0] * a[1] - f[1] * a[0];
        rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    }
    for (double& v : r) v /= rl;
    double d[3] = {f[1] * r[2] - f[2] * r[1], f[2] * r[0] - f[0] * r[2], f[0] * r[1] - f[1] * r[0]};
    /* m[row][col], columns r, d, f */
    double m[3][3] = {{r[0], d[0], f[0]}, {r[1], d[1], f[1]}, {r[2], d[2], f[2]}};
    double w, x, y, z;
    double tr = m[0][0] + m[1][1] + m[2][2];
    if (tr > 0) {
        double s = std::sqrt(tr + 1.0) * 2.0;
        w = 0.25 * s; x = (m[2][1] - m[1][2]) / s; y = (m[0][2] - m[2][0]) / s; z = (m[1][0] - m[0][1]) / s;
    } else if (m[0][0] > m[1][1] && m[0][0] > m[2][2]) {
        double s = std::sqrt(1.0 + m[0][0] - m[1][1] - m[2][2]) * 2.0;
        w = (m[2][1] - m[1][2]) / s; x = 0.25 * s; y = (m[0][1] + m[1][0]) / s; z = (m[0][2] + m[2][0]) / s;
    } else if (m[1][1] > m[2][2]) {
        double s = std::sqrt(1.0 + m[1][1] - m[0][0] - m[2][2]) * 2.0;
        w = (m[0][2] - m[2][0]) / s; x = (m[0][1] + m[1][0]) / s; y = 0.25 * s; z = (m[1][2] + m[2][1]) / s;
    } else {
        double s = std::sqrt(1.0 + m[2][2] - m[0][0] - m[1][1]) * 2.0;
        w = (m[1][0] - m[0][1]) / s; x = (m[0][2] + m[2][0]) / s; y = (m[1][2] + m[2][1]) / s; z = 0.25 * s;
    }
    double n = std::sqrt(w * w + x * x + y * y + z * z);
    if (w < 0) n = -n;
    q_out[0] = (float)(w / n); q_out[1] = (float)(x / n); q_out[2] = (float)(y / n); q_out[3] = (float)(z / n);
}

LumenStatus ensure_cloud(LumenRasterizer* r, const LumenCloud* c) {
    if (r->cached_cloud == c && r->cached_generation == c->generation) return LUMEN_SUCCESS;
    const size_t n = c->count;
    cudaError_t e = cudaSuccess;
    if (n > r->dev_cap) {
        cudaFree(r->d_aos); cudaFree(r->d_soa);
        r->d_aos = nullptr; r->d_soa = nullptr; r->dev_cap = 0;
        const size_t cap = (n + n / 8 + 16 + 3) / 4 * 4;   /* multiple of 4 keeps quats/sh 16-B aligned */
        if ((e = cudaMalloc(&r->d_aos, cap * sizeof(LumenGaussian))) != cudaSuccess) return cuda_status(e);
        if ((e = cudaMalloc(&r->d_soa, cap * 59 * sizeof(float) + 256)) != cudaSuccess) return cuda_status(e);
        r->dev_cap = cap;
    }
    if (n > 0) {
        if ((e = cudaMemcpyAsync(r->d_aos, c->data, n * sizeof(LumenGaussian), cudaMemcpyHostToDevice,
                                 r->stream)) != cudaSuccess)
            return cuda_status(e);
        float* base = r->d_soa;
        const size_t cap = r->dev_cap;
        aos_to_soa_kernel<<<1024, 256, 0, r->stream>>>((const float*)r->d_aos, (long long)n, base, base + cap * 3,
                                                      base + cap * 6, base + cap * 10, base + cap * 11);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e);
    }
    r->cached_cloud = c;
    r->cached_generation = c->generation;
    return LUMEN_SUCCESS;
}

LumenStatus ensure_image(LumenRasterizer* r, size_t npix) {
    if (npix <= r->img_cap) return LUMEN_SUCCESS;
    cudaFree(r->d_rgb); cudaFree(r->d_depth); cudaFree(r->d_alpha); cudaFree(r->d_rgb8);
    r->d_rgb = r->d_depth = r->d_alpha = nullptr;
    r->d_rgb8 = nullptr;
    r->img_cap = 0;
    cudaError_t e;
    if ((e = cudaMalloc(&r->d_rgb, npix * 3 * sizeof(float))) != cudaSuccess) return cuda_status(e);
    if ((e = cudaMalloc(&r->d_depth, npix * 3 * sizeof(float))) != cudaSuccess) return cuda_status(e);
    if ((e = cudaMalloc(&r->d_alpha, npix * sizeof(float))) != cudaSuccess) return cuda_status(e);
    if ((e = cudaMalloc(&r->d_rgb8, npix * 6)) != cudaSuccess) return cuda_status(e);
    r->img_cap = npix;
    return LUMEN_SUCCESS;
}

bool create_band_events(LumenRasterizer* r) {
    for (cudaEvent_t& ev : r->ev_band)
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return false;
    return true;
}

/* Compositor row bands of lumen_rasterize: after each band the render
 * stream blends the band's rows over the old contents (a short kernel), and
 * the copy stream reads them back while the next band is composited (the
 * copy engines need no SM, so the read-back is not held up by the
 * compositor's blocks). */

struct BandCopy {
    LumenRasterizer* r;
    LumenFrameBuffer* fb;
    size_t npix;
    int next;
    cudaError_t err;
};

void band_copy_hook(void* vctx, int y0, int y1, cudaStream_t main) {
    BandCopy* c = static_cast<BandCopy*>(vctx);
    if (c->err != cudaSuccess || y1 <= y0) return;
    LumenRasterizer* r = c->r;
    const size_t npix = c->npix;
    const size_t p0 = (size_t)y0 * c->fb->width, p1 = (size_t)y1 * c->fb->width;
    cudaError_t e;
    if (c->next == 0 && (e = cudaStreamWaitEvent(main, r->ev_up, 0)) != cudaSuccess) {   /* the old contents */
        c->err = e;
        return;
    }
    unsigned char* out8 = r->d_rgb8 + npix * 3;
    float* out_depth = r->d_depth + 2 * npix;
    to_framebuffer_kernel<<<148, 256, 0, main>>>(r->d_rgb, r->d_depth, r->d_alpha, r->d_rgb8, r->d_depth + npix,
                                                 out8, out_depth, (long long)p0, (long long)p1);
    cudaEvent_t ev = r->ev_band[c->next++ % kRasterBands];
    if ((e = cudaEventRecord(ev, main)) != cudaSuccess || (e = cudaStreamWaitEvent(r->copy_stream, ev, 0)) != cudaSuccess) {
        c->err = e;
        return;
    }
    if ((e = cudaMemcpyAsync(c->fb->rgb_data + p0 * 3, out8 + p0 * 3, (p1 - p0) * 3, cudaMemcpyDeviceToHost,
                             r->copy_stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(c->fb->depth_data + p0, out_depth + p0, (p1 - p0) * sizeof(float),
                             cudaMemcpyDeviceToHost, r->copy_stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(c->fb->alpha_data + p0, r->d_alpha + p0, (p1 - p0) * sizeof(float),
                             cudaMemcpyDeviceToHost, r->copy_stream)) != cudaSuccess)
        c->err = e;
}

void release(LumenRasterizer* r) {
    if (r->renderer) lumen_gpu_renderer_destroy(r->renderer);
    cudaFree(r->d_aos); cudaFree(r->d_soa);
    cudaFree(r->d_rgb); cudaFree(r->d_depth); cudaFree(r->d_alpha); cudaFree(r->d_rgb8);
    if (r->ev0) cudaEventDestroy(r->ev0);
    if (r->ev1) cudaEventDestroy(r->ev1);
    if (r->ev_down) cudaEventDestroy(r->ev_down);
    if (r->ev_up) cudaEventDestroy(r->ev_up);
    for (cudaEvent_t ev : r->ev_band)
        if (ev) cudaEventDestroy(ev);
    if (r->copy_stream) cudaStreamDestroy(r->copy_stream);
    if (r->stream) cudaStreamDestroy(r->stream);
}

void fill_cube_gaussian(LumenGaussian& g, float px, float py, float pz, float scale, float opacity,
                        float nr, float ng, float nb) {
    std::memset(&g, 0, sizeof(g));
    g.position = {px, py, pz};
    g.scale = {scale, scale, scale};
    g.rotation = {1.0f, 0.0f, 0.0f, 0.0f};
    g.opacity = opacity;
    const float c0 = 0.2820947917f;   /* SH degree-0 basis value */
    g.sh_coeffs[0] = (nr - 0.5f) / c0;
    g.sh_coeffs[1] = (ng - 0.5f) / c0;
    g.sh_coeffs[2] = (nb - 0.5f) / c0;
}

}  // namespace

extern "C" {

const char* lumen_get_version(void) { return LUMEN_VERSION_STRING; }
int lumen_get_version_major(void) { return LUMEN_VERSION_MAJOR; }
int lumen_get_version_minor(void) { return LUMEN_VERSION_MINOR; }
int lumen_get_version_patch(void) { return LUMEN_VERSION_PATCH; }

LumenConfig lumen_default_config(void) {
    LumenConfig c;
    c.image_width = 800;
    c.image_height = 600;
    c.tile_size = 16;
    c.near_plane = 0.1f;
    c.far_plane = 100.0f;
    c.early_termination_alpha = 0.99f;
    c.gaussian_radius_sigma = 3.0f;
    return c;
}

LumenCloud* lumen_cloud_create(size_t initial_capacity) {
    LumenCloud* c = (LumenCloud*)std::malloc(sizeof(LumenCloud));
    if (!c) return nullptr;
    const size_t cap = initial_capacity > 0 ? initial_capacity : 16;
    c->data = (LumenGaussian*)std::malloc(cap * sizeof(LumenGaussian));
    if (!c->data) { std::free(c); return nullptr; }
    c->count = 0;
    c->capacity = cap;
    c->generation = g_generation.fetch_add(1);
    return c;
}

void lumen_cloud_destroy(LumenCloud* c) {
    if (!c) return;
    std::free(c->data);
    std::free(c);
}

LumenStatus lumen_cloud_reserve(LumenCloud* c, size_t new_capacity) {
    if (!c) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (new_capacity <= c->capacity) return LUMEN_SUCCESS;
    if (new_capacity > SIZE_MAX / sizeof(LumenGaussian)) return LUMEN_ERROR_OUT_OF_MEMORY;
    LumenGaussian* d = (LumenGaussian*)std::realloc(c->data, new_capacity * sizeof(LumenGaussian));
    if (!d) return LUMEN_ERROR_OUT_OF_MEMORY;
    c->data = d;
    c->capacity = new_capacity;
    c->generation = g_generation.fetch_add(1);
    return LUMEN_SUCCESS;
}

size_t lumen_cloud_get_count(const LumenCloud* c) { return c ? c->count : 0; }
size_t lumen_cloud_get_capacity(const LumenCloud* c) { return c ? c->capacity : 0; }

LumenStatus lumen_cloud_add_gaussian(LumenCloud* c, const LumenGaussian* g) {
    if (!c || !g) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (c->count >= c->capacity) {
        size_t next = c->capacity * 2;
        if (next < 16) next = 16;
        LumenStatus st = lumen_cloud_reserve(c, next);
        if (st != LUMEN_SUCCESS) return st;
    }
    c->data[c->count++] = *g;
    c->generation = g_generation.fetch_add(1);
    return LUMEN_SUCCESS;
}

LumenStatus lumen_cloud_get_gaussian(const LumenCloud* c, size_t index, LumenGaussian* out) {
    if (!c || !out) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (index >= c->count) return LUMEN_ERROR_INVALID_ARGUMENT;
    *out = c->data[index];
    return LUMEN_SUCCESS;
}

void lumen_cloud_clear(LumenCloud* c) {
    if (!c) return;
    c->count = 0;
    c->generation = g_generation.fetch_add(1);
}

LumenCloud* lumen_create_synthetic_cube(size_t per_axis, float cube_size) {
    if (per_axis < 1) per_axis = 1;
    const size_t total = per_axis * per_axis * per_axis;
    LumenCloud* c = lumen_cloud_create(total);
    if (!c) return nullptr;
    const float step = per_axis > 1 ? cube_size / (float)(per_axis - 1) : 0.0f;
    const float half = cube_size * 0.5f;
    float scale = step * 0.6f;
    if (scale < 0.01f) scale = 0.05f;
    for (size_t x = 0; x < per_axis; ++x)
        for (size_t y = 0; y < per_axis; ++y)
            for (size_t z = 0; z < per_axis; ++z) {
                const float px = -half + (float)x * step, py = -half + (float)y * step, pz = -half + (float)z * step;
                LumenGaussian g;
                fill_cube_gaussian(g, px, py, pz, scale, 0.85f, (px + half) / cube_size, (py + half) / cube_size,
                                   (pz + half) / cube_size);
                lumen_cloud_add_gaussian(c, &g);
            }
    return c;
}

LumenCloud* lumen_create_synthetic_sphere(size_t count, float radius) {
    if (count < 1) count = 1;
    LumenCloud* c = lumen_cloud_create(count);
    if (!c) return nullptr;
    const float golden = 1.6180339887f;
    for (size_t i = 0; i < count; ++i) {
        const float theta = 2.0f * (float)M_PI * (float)i / golden;
        const float phi = acosf(1.0f - 2.0f * ((float)i + 0.5f) / (float)count);
        const float px = radius * sinf(phi) * cosf(theta);
        const float py = radius * sinf(phi) * sinf(theta);
        const float pz = radius * cosf(phi);
        LumenGaussian g;
        fill_cube_gaussian(g, px, py, pz, radius * 0.12f, 0.90f, 0.5f + 0.5f * (px / radius),
                           0.5f + 0.5f * (py / radius), 0.5f + 0.5f * (pz / radius));
        lumen_cloud_add_gaussian(c, &g);
    }
    return c;
}

/* The library owns a frame buffer's arrays (lumen.h), so it places them in
 * page-locked memory when a CUDA device is present: lumen_rasterize's
 * upload of the old contents and read-back of the new run at the full
 * host-link rate and asynchronously. Without a device they are plain heap
 * memory. Which one was used is kept after the struct (the caller holds
 * only the pointer returned here). */
struct FrameBufferBlock {
    LumenFrameBuffer fb;
    int page_locked;
};

LumenFrameBuffer* lumen_framebuffer_create(uint32_t width, uint32_t height) {
    if (width == 0 || height == 0) return nullptr;
    FrameBufferBlock* blk = (FrameBufferBlock*)std::calloc(1, sizeof(FrameBufferBlock));
    if (!blk) return nullptr;
    LumenFrameBuffer* fb = &blk->fb;
    fb->width = width;
    fb->height = height;
    const size_t n = (size_t)width * (size_t)height;
    void *rgb = nullptr, *depth = nullptr, *alpha = nullptr;
    if (cudaHostAlloc(&rgb, n * 3, cudaHostAllocPortable) == cudaSuccess &&
        cudaHostAlloc(&depth, n * sizeof(float), cudaHostAllocPortable) == cudaSuccess &&
        cudaHostAlloc(&alpha, n * sizeof(float), cudaHostAllocPortable) == cudaSuccess) {
        blk->page_locked = 1;
    } else {
        cudaFreeHost(rgb);
        cudaFreeHost(depth);
        cudaGetLastError();
        rgb = std::malloc(n * 3);
        depth = std::malloc(n * sizeof(float));
        alpha = std::malloc(n * sizeof(float));
        blk->page_locked = 0;
    }
    fb->rgb_data = (uint8_t*)rgb;
    fb->depth_data = (float*)depth;
    fb->alpha_data = (float*)alpha;
    if (!fb->rgb_data || !fb->depth_data || !fb->alpha_data) {
        lumen_framebuffer_destroy(fb);
        return nullptr;
    }
    lumen_framebuffer_clear(fb, 0, 0, 0);
    return fb;
}

void lumen_framebuffer_destroy(LumenFrameBuffer* fb) {
    if (!fb) return;
    FrameBufferBlock* blk = reinterpret_cast<FrameBufferBlock*>(fb);
    if (blk->page_locked) {
        cudaFreeHost(fb->rgb_data);
        cudaFreeHost(fb->depth_data);
        cudaFreeHost(fb->alpha_data);
    } else {
        std::free(fb->rgb_data);
        std::free(fb->depth_data);
        std::free(fb->alpha_data);
    }
    std::free(blk);
}

void lumen_framebuffer_clear(LumenFrameBuffer* fb, uint8_t r, uint8_t g, uint8_t b) {
    if (!fb) return;
    const size_t n = (size_t)fb->width * (size_t)fb->height;
    for (size_t i = 0; i < n; ++i) {
        fb->rgb_data[i * 3 + 0] = r;
        fb->rgb_data[i * 3 + 1] = g;
        fb->rgb_data[i * 3 + 2] = b;
        fb->depth_data[i] = 1000.0f;
        fb->alpha_data[i] = 0.0f;
    }
}

LumenRasterizer* lumen_rasterizer_create(const LumenConfig* config) {
    LumenRasterizer* r = new (std::nothrow) LumenRasterizer();
    if (!r) return nullptr;
    r->config = config ? *config : lumen_default_config();
    if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&r->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&r->ev0) != cudaSuccess || cudaEventCreate(&r->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->ev_down, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->ev_up, cudaEventDisableTiming) != cudaSuccess ||
        !create_band_events(r) || !(r->renderer = lumen_gpu_renderer_create())) {
        release(r);
        delete r;
        return nullptr;
    }
    return r;
}

void lumen_rasterizer_destroy(LumenRasterizer* r) {
    if (!r) return;
    release(r);
    delete r;
}

LumenStatus lumen_rasterizer_set_config(LumenRasterizer* r, const LumenConfig* config) {
    if (!r || !config) return LUMEN_ERROR_INVALID_ARGUMENT;
    r->config = *config;
    return LUMEN_SUCCESS;
}

LumenStatus lumen_rasterize(LumenRasterizer* r, const LumenCloud* cloud, const LumenCamera* camera,
                            LumenFrameBuffer* fb, LumenStats* stats) {
    if (!r || !cloud || !camera || !fb) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (fb->width == 0 || fb->height == 0 || !fb->rgb_data || !fb->depth_data || !fb->alpha_data)
        return LUMEN_ERROR_INVALID_ARGUMENT;
    if (r->config.tile_size != (uint32_t)kTile) return LUMEN_ERROR_INVALID_ARGUMENT;
    const uint32_t W = fb->width, H = fb->height;
    const size_t npix = (size_t)W * H;
    cudaEventRecord(r->ev0, r->stream);
    LumenStatus st = ensure_cloud(r, cloud);
    if (st != LUMEN_SUCCESS) return st;
    if ((st = ensure_image(r, npix)) != LUMEN_SUCCESS) return st;

    LumenViewCamera cam;
    lumen_gpu_camera_from_lookat(camera, W, H, r->config.near_plane, r->config.far_plane, &cam);

    LumenRenderOptions opt;
    std::memset(&opt, 0, sizeof(opt));
    opt.lowpass = 0.3f;
    opt.sh_degree = 3;
    opt.compute_depth = 1;
    opt.key_mode = 0;
    opt.term_mode = 1;
    opt.term_threshold = r->config.early_termination_alpha;
    opt.tile_size = kTile;

    const size_t cap = r->dev_cap;
    LumenGpuGaussians g;
    g.count = (int64_t)cloud->count;
    g.means = r->d_soa; g.scales = r->d_soa + cap * 3; g.quats = r->d_soa + cap * 6;
    g.opacities = r->d_soa + cap * 10; g.sh = r->d_soa + cap * 11;
    LumenGpuImage img;
    std::memset(&img, 0, sizeof(img));
    img.rgb = r->d_rgb; img.depth = r->d_depth; img.alpha = r->d_alpha;

    /* copy stream: the old contents (the background) go up while the frame
     * renders; after each compositor band, that band's rows are blended over
     * them and read back while the next band is composited */
    cudaError_t e;
    if ((e = cudaStreamWaitEvent(r->copy_stream, r->ev0, 0)) != cudaSuccess ||
        (e = cudaMemcpyAsync(r->d_rgb8, fb->rgb_data, npix * 3, cudaMemcpyHostToDevice, r->copy_stream)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(r->d_depth + npix, fb->depth_data, npix * sizeof(float), cudaMemcpyHostToDevice,
                             r->copy_stream)) != cudaSuccess ||
        (e = cudaEventRecord(r->ev_up, r->copy_stream)) != cudaSuccess)
        return cuda_status(e);
    LumenGpuCounts counts;
    BandCopy bc{r, fb, npix, 0, cudaSuccess};
    st = lumen::renderer_render_banded(r->renderer, &g, &cam, &opt, &img, &counts, kRasterBands, band_copy_hook, &bc,
                                       r->stream);
    /* the read-back ends before the call returns, whatever happened */
    if ((e = cudaEventRecord(r->ev_down, r->copy_stream)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(r->stream, r->ev_down, 0)) != cudaSuccess) {
        cudaStreamSynchronize(r->copy_stream);
        return cuda_status(e);
    }
    if (st != LUMEN_SUCCESS) {
        cudaStreamSynchronize(r->stream);
        return st;
    }
    if (bc.err != cudaSuccess) {
        cudaStreamSynchronize(r->stream);
        return cuda_status(bc.err);
    }
    cudaEventRecord(r->ev1, r->stream);
    if ((e = cudaEventSynchronize(r->ev1)) != cudaSuccess) return cuda_status(e);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, r->ev0, r->ev1);
    if (stats) {
        stats->total_splats = cloud->count;
        stats->visible_splats = (size_t)counts.n_visible;
        stats->culled_splats = cloud->count - (size_t)counts.n_visible;
        stats->total_tiles = (size_t)((W + kTile - 1) / kTile) * (size_t)((H + kTile - 1) / kTile);
        stats->touched_tiles = counts.touched_tiles;
        stats->rasterize_time_ms = ms;
        stats->frames_per_second = ms > 0.001f ? 1000.0f / ms : 10000.0f;
    }
    return LUMEN_SUCCESS;
}

LumenStatus lumen_gpu_camera_from_lookat(const LumenCamera* camera, uint32_t W, uint32_t H, float near_plane,
                                         float far_plane, LumenViewCamera* cam) {
    if (!camera || !cam || W == 0 || H == 0) return LUMEN_ERROR_INVALID_ARGUMENT;
    std::memset(cam, 0, sizeof(*cam));
    cam->position[0] = camera->position.x;
    cam->position[1] = camera->position.y;
    cam->position[2] = camera->position.z;
    look_at_rotation(camera->position, camera->target, camera->up, cam->rotation);
    const float fov_y = camera->fov_y_degrees * (float)M_PI / 180.0f;
    const float fy = (float)H / (2.0f * tanf(fov_y * 0.5f));
    cam->fx = fy;
    cam->fy = fy;
    cam->cx = (float)W * 0.5f;
    cam->cy = (float)H * 0.5f;
    cam->near_plane = near_plane;
    cam->far_plane = far_plane;
    cam->width = (int32_t)W;
    cam->height = (int32_t)H;
    return LUMEN_SUCCESS;
}

/* Bulk append: one copy instead of n calls (declared in lumen_gpu.h). */
LumenStatus lumen_cloud_append(LumenCloud* c, const LumenGaussian* g, size_t n) {
    if (!c || (!g && n > 0)) return LUMEN_ERROR_INVALID_ARGUMENT;
    /* neither count + n nor the byte count of the copy may wrap */
    if (n > SIZE_MAX / sizeof(LumenGaussian) - c->count) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (c->count + n > c->capacity) {
        size_t next = c->capacity * 2;
        if (next < c->count + n) next = c->count + n;
        LumenStatus st = lumen_cloud_reserve(c, next);
        if (st != LUMEN_SUCCESS) return st;
    }
    std::memcpy(c->data + c->count, g, n * sizeof(LumenGaussian));
    c->count += n;
    c->generation = g_generation.fetch_add(1);
    return LUMEN_SUCCESS;
}

}  // extern "C"
