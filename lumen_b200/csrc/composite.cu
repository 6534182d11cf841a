/*
 * composite.cu - K5: per-tile front-to-back alpha compositing.
 *
 * Reference: the per-tile pixel loop of rasterize_scene,
 * src/raster/pipeline.mojo:172-229, with compute_gaussian_pixel_alpha and
 * PixelAccumulator.blend/finalize, src/raster/compositor.mojo:10-89.
 *
 * One CTA per 16x16 tile (or persistent CTAs taking tiles in ticket order),
 * one thread per pixel, each warp an 8x4 block. The tile's sorted instances
 * are processed in chunks of 128, 256 or 512 (a launch parameter the
 * autotuner picks): the threads gather the chunk's 48-byte records (through
 * the sorted visible index) into shared memory and compute which warp
 * blocks each splat can reach at all (reach_mask); each warp then walks, in
 * sorted order, only the splats
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

/* (uint8)(clamp(c, 0, 1) * 255), truncating (c_api/src/lumen_c.c:541-543). */
__device__ __forceinline__ unsigned char to_byte(float c) {
    if (c < 0.0f) c = 0.0f;
    if (c > 1.0f) c = 1.0f;
    return (unsigned char)(c * 255.0f);
}

/* Threads per tile: each thread shades two vertically adjacent pixels, and
 * warp w an 8x8 block (x offset (w & 1) * 8, y offset (w >> 1) * 8). */
constexpr int kCompositeThreads = kTilePixels / 2;
constexpr int kCompositeWarps = kCompositeThreads / 32;

/* A chunk of kChunk sorted instances is staged at a time. */
template <int kChunk>
struct CompositeSmem {
    float4 geo[kChunk];                 /* cx, cy, depth, opacity */
    float4 con[kChunk];                 /* 0.5 ic00, ic01, 0.5 ic11, 1 when colour and depth are finite */
    float4 col[kChunk];                 /* r, g, b, - */
    unsigned char mask[kChunk];         /* bit w: the splat can reach warp w's pixels */
    unsigned short list[kCompositeWarps][kChunk];
    unsigned int ticket;
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

/* Packed two-lane float arithmetic of sm_100 (add/mul/fma .rn .f32x2),
 * written in PTX with the explicit round-to-nearest modifier: per lane it
 * is the IEEE operation, and an operation with an explicit rounding mode is
 * never contracted with another, so each product and sum rounds on its own
 * as in the reference. */
__device__ __forceinline__ unsigned long long pack2(float2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long r) {
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)));
    return unpack2(r);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)));
    return unpack2(r);
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)), "l"(pack2(c)));
    return unpack2(r);
}

/* lumen_expf_core on two arguments (per lane the same operations, so the
 * same bits). fmaf(-k, c, x) is written fmaf(k, -c, x): the same exact
 * product. */
__device__ __forceinline__ float2 expf_core2(float2 x) {
    const float LN2_HI = 0.693145751953125f;
    const float LN2_LO = 1.42860682030941723e-6f;
    const float LOG2E = 1.44269504088896341f;
    const float SHIFTER = 12582912.0f;
    const float2 t = fma2(x, f2(LOG2E), f2(SHIFTER));
    const float2 k = add2(t, f2(-SHIFTER));
    float2 r = fma2(k, f2(-LN2_HI), x);
    r = fma2(k, f2(-LN2_LO), r);
    float2 p = f2(1.98412698412698413e-4f);
    p = fma2(p, r, f2(1.38888888888888889e-3f));
    p = fma2(p, r, f2(8.33333333333333333e-3f));
    p = fma2(p, r, f2(4.16666666666666667e-2f));
    p = fma2(p, r, f2(1.66666666666666667e-1f));
    p = fma2(p, r, f2(0.5f));
    p = fma2(p, r, f2(1.0f));
    p = fma2(p, r, f2(1.0f));
    const float2 sc = f2(__uint_as_float(__float_as_uint(t.x) * 8388608u + 0x3F800000u),
                         __uint_as_float(__float_as_uint(t.y) * 8388608u + 0x3F800000u));
    return mul2(p, sc);
}

/* Per-pixel state of the front-to-back blend (PixelAccumulator). */
struct PixelPair {
    float2 T, cr, cg, cb, dep, acc;
    unsigned int count0, count1;
    int last0, last1;
    bool done0, done1;
};

/* compute_gaussian_pixel_alpha (compositor.mojo:62-89) for both pixels:
 * alpha, and whether each pixel blends (PixelAccumulator.blend's test,
 * compositor.mojo:33-35, and the pixel still open). */
__device__ __forceinline__ float2 pair_alpha(const PixelPair& q, float pxc, float2 pyc, float4 gg, float4 cc,
                                             bool& bl0, bool& bl1) {
    /* power = (cx dx) dx + (cy dx) dy + (cz dy) dy, in that order; the two
     * pixels share dx */
    const float dx = pxc - gg.x;
    const float a = cc.x * dx * dx;
    const float b = cc.y * dx;
    const float2 dy = add2(pyc, f2(-gg.y));
    const float2 s = add2(f2(a), mul2(f2(b), dy));
    const float2 power = add2(s, mul2(mul2(f2(cc.z), dy), dy));
    float p0 = power.x, p1 = power.y;
    bool skip0 = false, skip1 = false;
    if (p0 < 0.0f) p0 = 0.0f;
    else if (p0 > 4.5f) skip0 = true;
    if (p1 < 0.0f) p1 = 0.0f;
    else if (p1 > 4.5f) skip1 = true;
    float2 alpha = mul2(f2(gg.w), expf_core2(f2(-p0, -p1)));
    if (alpha.x > (float)0.99) alpha.x = (float)0.99;
    if (alpha.y > (float)0.99) alpha.y = (float)0.99;
    bl0 = !q.done0 && !skip0 && !(alpha.x < min_alpha());
    bl1 = !q.done1 && !skip1 && !(alpha.y < min_alpha());
    return alpha;
}

/* PixelAccumulator.blend (compositor.mojo:25-53) and the termination test,
 * for a splat whose colour and depth are finite: a pixel that does not
 * blend gets weight 0 and factor 1, which leaves its sums and transmittance
 * exactly as they were (its sums are never -0, and 0 times a finite value
 * is a signed zero). */
__device__ __forceinline__ void pair_blend_finite(PixelPair& q, float2 alpha, bool bl0, bool bl1, float4 col,
                                                  float depth, int idx, bool mode_alpha, float thr) {
    const float2 wt = mul2(alpha, q.T);
    const float2 om = add2(f2(1.0f), f2(-alpha.x, -alpha.y));
    const float2 w = f2(bl0 ? wt.x : 0.0f, bl1 ? wt.y : 0.0f);
    const float2 fac = f2(bl0 ? om.x : 1.0f, bl1 ? om.y : 1.0f);
    q.cr = add2(q.cr, mul2(f2(col.x), w));
    q.cg = add2(q.cg, mul2(f2(col.y), w));
    q.cb = add2(q.cb, mul2(f2(col.z), w));
    q.dep = add2(q.dep, mul2(f2(depth), w));
    q.T = mul2(q.T, fac);
    q.acc = add2(f2(1.0f), f2(-q.T.x, -q.T.y));
    q.count0 += bl0;
    q.count1 += bl1;
    if (bl0 && (mode_alpha ? (q.acc.x >= thr) : (q.T.x <= thr))) { q.done0 = true; q.last0 = idx; }
    if (bl1 && (mode_alpha ? (q.acc.y >= thr) : (q.T.y <= thr))) { q.done1 = true; q.last1 = idx; }
}

/* The same blend one pixel at a time, for a splat with a non-finite colour
 * or depth (where weight 0 would not leave the sums unchanged). */
__device__ __forceinline__ void blend_one(float& T, float& cr, float& cg, float& cb, float& dep, float& acc,
                                          unsigned int& count, bool& done, int& last, float alpha, float4 col,
                                          float depth, int idx, bool mode_alpha, float thr) {
    const float w = alpha * T;
    cr += col.x * w;
    cg += col.y * w;
    cb += col.z * w;
    dep += depth * w;
    T *= (1.0f - alpha);
    acc = 1.0f - T;
    ++count;
    if (mode_alpha ? (acc >= thr) : (T <= thr)) {
        done = true;
        last = idx;
    }
}

/* One tile of the batch (batch-wide id gtile, owned by the last view whose
 * tile_begin <= gtile). */
template <int kChunk>
__device__ __forceinline__ void composite_tile(CompositeSmem<kChunk>& s, const ViewTable* __restrict__ vt,
                                               const LumenSplatRecord* __restrict__ records, const LumenGpuFrame& f,
                                               long long capacity, Control* __restrict__ ctrl,
                                               const LumenRenderOptions& opt, int n_views, long long gtile) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int view = n_views == 1 ? 0 : find_view_by_tile(vt, n_views, gtile);
    int tx, ty, px, py;
    bool inside0, inside1, any_instance;
    {
        const ViewDesc& vd = vt->view[view];
        const int tiles_x = vd.tiles_x;
        const int tile = (int)(gtile - vd.tile_begin);
        tx = tile % tiles_x;
        ty = tile / tiles_x;
        px = tx * kTile + (warp & 1) * 8 + (lane & 7);
        py = ty * kTile + (warp >> 1) * 8 + (lane >> 3) * 2;
        inside0 = px < vd.cam.width && py < vd.cam.height;
        inside1 = px < vd.cam.width && py + 1 < vd.cam.height;
        any_instance = vd.inst_begin >= 0;
    }

    PixelPair q;
    q.T = f2(1.0f);
    q.cr = q.cg = q.cb = q.dep = q.acc = f2(0.0f);
    q.count0 = q.count1 = 0;
    q.last0 = q.last1 = -1;
    q.done0 = !inside0;
    q.done1 = !inside1;
    bool background = opt.white_background != 0;

    if (!any_instance) {
        /* pipeline.mojo:162-163: no instances in the view, the output stays zero */
        background = false;
    } else {
        const long long K = (long long)ctrl->n_instances < capacity ? (long long)ctrl->n_instances : capacity;
        int rs = f.ranges[2 * gtile], re = f.ranges[2 * gtile + 1];
        const unsigned int n_visible = ctrl->n_visible;
        if (!(rs == -1 || rs >= re) && (rs < 0 || (long long)re > K)) {
            /* self-check: a range outside the sorted instances */
            if (tid == 0) atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_BOUNDS);
            rs = re = -1;
        }
        if (!(rs == -1 || rs >= re)) {
            const unsigned int* __restrict__ vals = ctrl->tile_sort.sorted_buffer ? f.vals[1] : f.vals[0];
            const float pxc = (float)px + 0.5f;
            const float2 pyc = f2((float)py + 0.5f, (float)(py + 1) + 0.5f);
            const float tile_x0 = (float)(tx * kTile), tile_y0 = (float)(ty * kTile);
            const float thr = opt.term_threshold;
            const bool mode_alpha = opt.term_mode == 1;
            for (int cs = rs; cs < re; cs += kChunk) {
                if (__syncthreads_count(!(q.done0 && q.done1)) == 0) break;
#pragma unroll
                for (int r = 0; r < (kChunk + kCompositeThreads - 1) / kCompositeThreads; ++r) {
                    const int slot = r * kCompositeThreads + tid;
                    if (kChunk % kCompositeThreads != 0 && slot >= kChunk) break;
                    const int i = cs + slot;
                    unsigned int m = 0;
                    if (i < re) {
                        unsigned int v = vals[i];
                        if (v >= n_visible) {   /* self-check: an index beyond the visible records */
                            atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_BOUNDS);
                        } else {
                            const float4* r4 = reinterpret_cast<const float4*>(records + v);
                            const float4 geo = __ldg(r4), con = __ldg(r4 + 1), col = __ldg(r4 + 2);
                            s.geo[slot] = geo;
                            /* 0.5 folded into the conic: scaling by a power of two commutes
                             * with rounding, so the power equals the reference's
                             * 0.5 * (a dx dx + 2 b dx dy + c dy dy) bit for bit */
                            const bool finite = isfinite(col.x) && isfinite(col.y) && isfinite(col.z) &&
                                                isfinite(geo.z);
                            s.con[slot] = make_float4(0.5f * con.x, con.y, 0.5f * con.z, finite ? 1.0f : 0.0f);
                            s.col[slot] = col;
                            m = reach_mask_8x8(geo, con, tile_x0, tile_y0);
                        }
                    }
                    s.mask[slot] = (unsigned char)m;
                }
                __syncthreads();
                /* this warp's splats of the chunk, in sorted order */
                const int n = re - cs < kChunk ? re - cs : kChunk;
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
                    if (!(q.done0 && q.done1)) {
                        const float4 gg = s.geo[j];
                        const float4 cc = s.con[j];
                        bool bl0, bl1;
                        const float2 alpha = pair_alpha(q, pxc, pyc, gg, cc, bl0, bl1);
                        if (cc.w != 0.0f) {             /* uniform across the warp */
                            if (bl0 || bl1)
                                pair_blend_finite(q, alpha, bl0, bl1, s.col[j], gg.z, cs + j, mode_alpha, thr);
                        } else {
                            const float4 col = s.col[j];
                            if (bl0)
                                blend_one(q.T.x, q.cr.x, q.cg.x, q.cb.x, q.dep.x, q.acc.x, q.count0, q.done0,
                                          q.last0, alpha.x, col, gg.z, cs + j, mode_alpha, thr);
                            if (bl1)
                                blend_one(q.T.y, q.cr.y, q.cg.y, q.cb.y, q.dep.y, q.acc.y, q.count1, q.done1,
                                          q.last1, alpha.y, col, gg.z, cs + j, mode_alpha, thr);
                        }
                    }
                    if (__all_sync(0xffffffffu, q.done0 && q.done1)) break;
                }
                __syncthreads();
            }
            /* a pixel that never saturated visited the whole range */
            if (!q.done0) q.last0 = re - 1;
            if (!q.done1) q.last1 = re - 1;
            /* (a pixel outside the image was marked done and is not written) */
        }
    }
    /* finalize, compositor.mojo:55-59 */
    const ViewDesc& vd = vt->view[view];
    const LumenGpuImage& img = vd.img;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (!(k == 0 ? inside0 : inside1)) continue;
        float cr = k == 0 ? q.cr.x : q.cr.y, cg = k == 0 ? q.cg.x : q.cg.y, cb = k == 0 ? q.cb.x : q.cb.y;
        const float T = k == 0 ? q.T.x : q.T.y;
        int last = k == 0 ? q.last0 : q.last1;
        const long long pix = (long long)(py + k) * vd.cam.width + px;
        /* last visited instance as an offset within the view's instances
         * (positions are below 2^30) */
        if (last >= 0) last -= (int)vd.inst_begin;
        if (background) { cr += T; cg += T; cb += T; }
        if (img.rgb) {
            img.rgb[pix * 3 + 0] = cr;
            img.rgb[pix * 3 + 1] = cg;
            img.rgb[pix * 3 + 2] = cb;
        }
        if (img.rgb8) {
            img.rgb8[pix * 3 + 0] = to_byte(cr);
            img.rgb8[pix * 3 + 1] = to_byte(cg);
            img.rgb8[pix * 3 + 2] = to_byte(cb);
        }
        if (img.depth) img.depth[pix] = opt.compute_depth ? (k == 0 ? q.dep.x : q.dep.y) : 0.0f;
        if (img.alpha) img.alpha[pix] = k == 0 ? q.acc.x : q.acc.y;
        if (img.n_contrib) img.n_contrib[pix] = k == 0 ? q.count0 : q.count1;
        if (img.last_idx) img.last_idx[pix] = last;
    }
}

/* One CTA per tile of the batch. */
template <int kChunk>
__global__ void __launch_bounds__(kCompositeThreads, 8)
composite_kernel(const ViewTable* __restrict__ vt, int n_views, const LumenSplatRecord* __restrict__ records,
                 LumenGpuFrame f, long long capacity, Control* __restrict__ ctrl, LumenRenderOptions opt) {
    __shared__ CompositeSmem<kChunk> s;
    composite_tile(s, vt, records, f, capacity, ctrl, opt, n_views, blockIdx.x);
}

/* Persistent form for a grid fixed in advance (a captured graph replayed
 * for batches of any size): CTAs take tiles in ticket order. */
template <int kChunk>
__global__ void __launch_bounds__(kCompositeThreads, 8)
composite_persistent_kernel(const ViewTable* __restrict__ vt, const LumenSplatRecord* __restrict__ records,
                            LumenGpuFrame f, long long capacity, Control* __restrict__ ctrl, LumenRenderOptions opt) {
    __shared__ CompositeSmem<kChunk> s;
    const long long total = vt->hdr.total_tiles;
    const int n_views = vt->hdr.n_views;
    for (;;) {
        if (threadIdx.x == 0) s.ticket = atomicAdd(&ctrl->composite_ticket, 1u);
        __syncthreads();
        const long long t = s.ticket;
        if (t >= total) break;
        composite_tile(s, vt, records, f, capacity, ctrl, opt, n_views, t);
        __syncthreads();
    }
}

template <int kChunk>
static void launch_composite_chunk(const ViewTable* vt, int n_views, const LumenGpuFrame& f, Control* ctrl,
                                   const LumenRenderOptions& opt, long long n_tiles, bool persistent, int num_sms,
                                   cudaStream_t st) {
    if (persistent) {
        composite_persistent_kernel<kChunk><<<8 * num_sms, kCompositeThreads, 0, st>>>(
            vt, f.records, f, (long long)f.instance_capacity, ctrl, opt);
    } else {
        composite_kernel<kChunk><<<(unsigned int)n_tiles, kCompositeThreads, 0, st>>>(
            vt, n_views, f.records, f, (long long)f.instance_capacity, ctrl, opt);
    }
}

/* chunk: instances staged per round, one of kCompositeChunks. */
void launch_composite(const ViewTable* vt, int n_views, const LumenGpuFrame& f, Control* ctrl,
                      const LumenRenderOptions& opt, long long n_tiles, bool persistent, int chunk, int num_sms,
                      cudaStream_t st) {
    if (n_tiles <= 0) return;
    switch (chunk) {
        case 128: launch_composite_chunk<128>(vt, n_views, f, ctrl, opt, n_tiles, persistent, num_sms, st); break;
        case 512: launch_composite_chunk<512>(vt, n_views, f, ctrl, opt, n_tiles, persistent, num_sms, st); break;
        default: launch_composite_chunk<256>(vt, n_views, f, ctrl, opt, n_tiles, persistent, num_sms, st); break;
    }
}

}  // namespace lumen
