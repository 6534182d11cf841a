/*
 * composite.cu - K5: per-tile front-to-back alpha compositing.
 *
 * Reference: the per-tile pixel loop of rasterize_scene,
 * src/raster/pipeline.mojo:172-229, with compute_gaussian_pixel_alpha and
 * PixelAccumulator.blend/finalize, src/raster/compositor.mojo:10-89.
 *
 * One CTA per 16x16 tile, one thread per pixel, each warp an 8x4 block. The
 * tile's sorted instances are processed in chunks of 256: each thread
 * gathers one instance's 48-byte record (through the sorted visible index)
 * into shared memory and computes which warp blocks the splat can reach at
 * all (reach_mask); each warp then walks, in sorted order, only the splats
 * that can reach it, so each pixel blends exactly the reference's sequence.
 * A pixel stops after the blend that saturates it; a warp leaves the chunk
 * once all its pixels stopped, and the CTA stops loading chunks once all 256
 * pixels stopped.
 *
 * Built with --fmad=false: power, alpha, weights and transmittance round as
 * in the reference, so contributor counts match the CPU restatement bit for
 * bit. The exponential is lumen_expf (shared with the restatement).
 */
#include "composite_common.cuh"

namespace lumen {

struct CompositeSmem {
    float4 geo[kTilePixels];            /* cx, cy, depth, opacity */
    float4 con[kTilePixels];            /* ic00, ic01, ic11, - */
    float4 col[kTilePixels];            /* r, g, b, - */
    unsigned char mask[kTilePixels];    /* bit w: the splat can reach warp w's pixels */
    unsigned short list[kTilePixels / 32][kTilePixels];
};

__global__ void __launch_bounds__(kTilePixels, 6)
composite_kernel(const LumenSplatRecord* __restrict__ records, LumenGpuFrame f, long long capacity,
                 Control* __restrict__ ctrl, int width, int height, int tiles_x,
                 LumenRenderOptions opt, LumenGpuImage img) {
    __shared__ CompositeSmem s;
    const int tile = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tx = tile % tiles_x, ty = tile / tiles_x;
    const int px = tx * kTile + warp_block_x(warp) + (lane & 7);
    const int py = ty * kTile + warp_block_y(warp) + (lane >> 3);
    const bool inside = px < width && py < height;
    const long long pix = (long long)py * width + px;
    const long long K = (long long)ctrl->n_instances < capacity ? (long long)ctrl->n_instances : capacity;

    float T = 1.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f, dep = 0.0f, acc = 0.0f;
    unsigned int count = 0;
    int last = -1;
    bool background = opt.white_background != 0;

    if (K == 0) {
        /* pipeline.mojo:162-163: no instances, the output stays zero */
        background = false;
    } else {
        int rs = f.ranges[2 * tile], re = f.ranges[2 * tile + 1];
        const unsigned int n_visible = ctrl->n_visible;
        if (!(rs == -1 || rs >= re) && (rs < 0 || (long long)re > K)) {
            /* self-check: a range outside the sorted instances */
            if (tid == 0) atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_BOUNDS);
            rs = re = -1;
        }
        if (!(rs == -1 || rs >= re)) {
            const unsigned int* __restrict__ vals = ctrl->tile_sort.sorted_buffer ? f.vals[1] : f.vals[0];
            const float pxc = (float)px + 0.5f, pyc = (float)py + 0.5f;
            const float tile_x0 = (float)(tx * kTile), tile_y0 = (float)(ty * kTile);
            const float thr = opt.term_threshold;
            const bool mode_alpha = opt.term_mode == 1;
            bool done = !inside;
            for (int cs = rs; cs < re; cs += kTilePixels) {
                if (__syncthreads_count(!done) == 0) break;
                const int i = cs + tid;
                unsigned int m = 0;
                if (i < re) {
                    unsigned int v = vals[i];
                    if (v >= n_visible) {   /* self-check: an index beyond the visible records */
                        atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_BOUNDS);
                    } else {
                        const float4* r4 = reinterpret_cast<const float4*>(records + v);
                        const float4 geo = __ldg(r4), con = __ldg(r4 + 1);
                        s.geo[tid] = geo;
                        /* 0.5 folded into the conic: scaling by a power of two commutes
                         * with rounding, so the power below equals the reference's
                         * 0.5 * (a dx dx + 2 b dx dy + c dy dy) bit for bit */
                        s.con[tid] = make_float4(0.5f * con.x, con.y, 0.5f * con.z, 0.0f);
                        s.col[tid] = __ldg(r4 + 2);
                        m = reach_mask(geo, con, tile_x0, tile_y0);
                    }
                }
                s.mask[tid] = (unsigned char)m;
                __syncthreads();
                /* this warp's splats of the chunk, in sorted order */
                const int n = re - cs < kTilePixels ? re - cs : kTilePixels;
                int cnt = 0;
                for (int base = 0; base < n; base += 32) {
                    const int j = base + lane;
                    const bool bit = j < n && ((s.mask[j] >> warp) & 1u);
                    const unsigned int bal = __ballot_sync(0xffffffffu, bit);
                    if (bit) s.list[warp][cnt + __popc(bal & lanemask_lt())] = (unsigned short)j;
                    cnt += __popc(bal);
                }
                __syncwarp();
                for (int t = 0; t < cnt; ++t) {
                    const int j = s.list[warp][t];
                    if (!done) {
                        const float4 gg = s.geo[j];
                        const float4 cc = s.con[j];
                        /* compute_gaussian_pixel_alpha, compositor.mojo:62-89 */
                        const float dx = pxc - gg.x;
                        const float dy = pyc - gg.y;
                        float power = cc.x * dx * dx + cc.y * dx * dy + cc.z * dy * dy;
                        bool skip = false;
                        if (power < 0.0f) power = 0.0f;
                        else if (power > 4.5f) skip = true;
                        if (!skip) {
                            float alpha = gg.w * lumen_expf_core(-power);
                            if (alpha > (float)0.99) alpha = (float)0.99;
                            /* PixelAccumulator.blend, compositor.mojo:25-53 */
                            if (!(alpha < min_alpha())) {
                                const float4 col = s.col[j];
                                const float w = alpha * T;
                                cr += col.x * w;
                                cg += col.y * w;
                                cb += col.z * w;
                                dep += gg.z * w;
                                T *= (1.0f - alpha);
                                acc = 1.0f - T;
                                ++count;
                                if (mode_alpha ? (acc >= thr) : (T <= thr)) {
                                    done = true;
                                    last = cs + j;
                                }
                            }
                        }
                    }
                    if (__all_sync(0xffffffffu, done)) break;
                }
                __syncthreads();
            }
            /* a pixel that never saturated visited the whole range */
            if (!done) last = re - 1;
        }
    }
    if (!inside) return;
    /* finalize, compositor.mojo:55-59 */
    if (background) { cr += T; cg += T; cb += T; }
    img.rgb[pix * 3 + 0] = cr;
    img.rgb[pix * 3 + 1] = cg;
    img.rgb[pix * 3 + 2] = cb;
    if (img.depth) img.depth[pix] = opt.compute_depth ? dep : 0.0f;
    if (img.alpha) img.alpha[pix] = acc;
    if (img.n_contrib) img.n_contrib[pix] = count;
    if (img.last_idx) img.last_idx[pix] = last;
}

void launch_composite(const LumenGpuFrame& f, Control* ctrl, const LumenViewCamera& cam,
                      const LumenRenderOptions& opt, const LumenGpuImage& img, cudaStream_t st) {
    const int tiles_x = (cam.width + kTile - 1) / kTile;
    const int tiles_y = (cam.height + kTile - 1) / kTile;
    composite_kernel<<<tiles_x * tiles_y, kTilePixels, 0, st>>>(
        f.records, f, (long long)f.instance_capacity, ctrl, cam.width, cam.height, tiles_x, opt, img);
}

}  // namespace lumen
