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

/* A chunk of kChunk sorted instances is staged at a time; a warp walks its
 * list of the chunk's splats kVoteGroup at a time. */
constexpr int kVoteGroup = 8;

/* Resident CTAs per SM the compositor is compiled for: 64 registers per
 * thread, enough for the unrolled group without spills. */
constexpr int kCompositeBlocksPerSm = 4;

template <int kChunk>
struct CompositeSmem {
    float4 geo[kChunk + 1];             /* cx, cy, depth, opacity; slot kChunk: the padding splat */
    float4 con[kChunk + 1];             /* 0.5 ic00, ic01, 0.5 ic11, - */
    float4 col[kChunk + 1];             /* r, g, b, - */
    unsigned char mask[kChunk];         /* bit w: the splat can reach warp w's pixels */
    unsigned short list[kTilePixels / 32][kChunk + kVoteGroup];
    unsigned int ticket;
};

/* The warp lists are padded to a multiple of kVoteGroup with slot kChunk, a
 * splat of opacity 0 whose power is above 4.5 away from (0, 0) (conic
 * 1e30): it is skipped like any out-of-reach splat and changes nothing. The
 * splat loop then runs in groups of kVoteGroup, unrolled, with one warp
 * vote per group. */
template <int kChunk>
__device__ __forceinline__ void init_padding_splat(CompositeSmem<kChunk>& s) {
    if (threadIdx.x == 0) {
        s.geo[kChunk] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        s.con[kChunk] = make_float4(1e30f, 0.0f, 1e30f, 0.0f);
        s.col[kChunk] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

/* A pixel's front-to-back state (PixelAccumulator, compositor.mojo:10-59). */
struct PixelState {
    float T, cr, cg, cb, dep, acc;
    unsigned int count;
    int last;
    bool done;
};

/* The warp's list of splats of the staged chunk, in sorted order, for the
 * warp's pixel. kClamp: some staged splat has opacity above 0.99, so the
 * 0.99 alpha clamp can apply (without one, alpha = opacity * exp(-power)
 * with exp(-power) <= 1 never exceeds it and the test is left out).
 * kModeAlpha: stop when 1 - T reaches the threshold, else when T falls to
 * it. kTrack: count the blended splats and note where the pixel stopped
 * (only when the view's image asks for contributor counts or last-visited
 * offsets). Either way the arithmetic is the reference's, operation by
 * operation. */
template <int kChunk, bool kClamp, bool kModeAlpha, bool kTrack>
__device__ __forceinline__ void blend_list(const CompositeSmem<kChunk>& s, int warp, int cnt, int cs, float pxc,
                                           float pyc, float thr, PixelState& p) {
    for (int t0 = 0; t0 < cnt; t0 += kVoteGroup) {
#pragma unroll
    for (int u = 0; u < kVoteGroup; ++u) {
        const int j = s.list[warp][t0 + u];
        if (!p.done) {
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
                if (kClamp && alpha > (float)0.99) alpha = (float)0.99;
                /* PixelAccumulator.blend, compositor.mojo:25-53 */
                if (!(alpha < min_alpha())) {
                    const float4 col = s.col[j];
                    const float w = alpha * p.T;
                    p.cr += col.x * w;
                    p.cg += col.y * w;
                    p.cb += col.z * w;
                    p.dep += gg.z * w;
                    p.T *= (1.0f - alpha);
                    if (kTrack) ++p.count;
                    if (kModeAlpha) {
                        p.acc = 1.0f - p.T;
                        if (p.acc >= thr) {
                            p.done = true;
                            if (kTrack) p.last = cs + j;
                        }
                    } else if (p.T <= thr) {
                        p.done = true;
                        if (kTrack) p.last = cs + j;
                    }
                }
            }
        }
    }
        if (__all_sync(0xffffffffu, p.done)) break;
    }
    if (!kModeAlpha) p.acc = 1.0f - p.T;     /* the value the reference's blend leaves (compositor.mojo:51) */
}

/* One tile of the batch (batch-wide id gtile, owned by the last view whose
 * tile_begin <= gtile). */
template <int kChunk, bool kTrack>
__device__ __forceinline__ void composite_tile(CompositeSmem<kChunk>& s, const ViewTable* __restrict__ vt,
                                               const LumenSplatRecord* __restrict__ records, const LumenGpuFrame& f,
                                               long long capacity, Control* __restrict__ ctrl,
                                               const LumenRenderOptions& opt, int n_views, long long gtile) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int view = n_views == 1 ? 0 : find_view_by_tile(vt, n_views, gtile);
    int tx, ty, px, py;
    bool inside, any_instance;
    {
        const ViewDesc& vd = vt->view[view];
        const int tiles_x = vd.tiles_x;
        const int tile = (int)(gtile - vd.tile_begin);
        tx = tile % tiles_x;
        ty = tile / tiles_x;
        px = tx * kTile + warp_block_x(warp) + (lane & 7);
        py = ty * kTile + warp_block_y(warp) + (lane >> 3);
        inside = px < vd.cam.width && py < vd.cam.height;
        any_instance = vd.inst_begin >= 0;
    }

    float T = 1.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f, dep = 0.0f, acc = 0.0f;
    unsigned int count = 0;
    int last = -1;
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
            const float pxc = (float)px + 0.5f, pyc = (float)py + 0.5f;
            const float tile_x0 = (float)(tx * kTile), tile_y0 = (float)(ty * kTile);
            const float thr = opt.term_threshold;
            const bool mode_alpha = opt.term_mode == 1;
            bool done = !inside;
            for (int cs = rs; cs < re; cs += kChunk) {
                if (__syncthreads_count(!done) == 0) break;
                int high = 0;
#pragma unroll
                for (int r = 0; r < (kChunk + kTilePixels - 1) / kTilePixels; ++r) {
                    const int slot = r * kTilePixels + tid;
                    if (kChunk % kTilePixels != 0 && slot >= kChunk) break;
                    const int i = cs + slot;
                    unsigned int m = 0;
                    if (i < re) {
                        unsigned int v = vals[i];
                        if (v >= n_visible) {   /* self-check: an index beyond the visible records */
                            atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_BOUNDS);
                        } else {
                            const float4* r4 = reinterpret_cast<const float4*>(records + v);
                            const float4 geo = __ldg(r4), con = __ldg(r4 + 1);
                            s.geo[slot] = geo;
                            /* 0.5 folded into the conic: scaling by a power of two commutes
                             * with rounding, so the power below equals the reference's
                             * 0.5 * (a dx dx + 2 b dx dy + c dy dy) bit for bit */
                            s.con[slot] = make_float4(0.5f * con.x, con.y, 0.5f * con.z, 0.0f);
                            s.col[slot] = __ldg(r4 + 2);
                            m = reach_mask(geo, con, tile_x0, tile_y0);
                            high |= geo.w > (float)0.99;
                        }
                    }
                    s.mask[slot] = (unsigned char)m;
                }
                /* whether any staged splat has opacity above 0.99: only those can
                 * reach the 0.99 alpha clamp (exp(-power) <= 1 for power >= 0) */
                const bool clamp = __syncthreads_or(high) != 0;
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
                if (lane < ((kVoteGroup - (cnt & (kVoteGroup - 1))) & (kVoteGroup - 1)))
                    s.list[warp][cnt + lane] = (unsigned short)kChunk;
                cnt = (cnt + kVoteGroup - 1) & ~(kVoteGroup - 1);
                __syncwarp();
                PixelState px_state{T, cr, cg, cb, dep, acc, count, last, done};
                if (clamp) {
                    if (mode_alpha) blend_list<kChunk, true, true, kTrack>(s, warp, cnt, cs, pxc, pyc, thr, px_state);
                    else blend_list<kChunk, true, false, kTrack>(s, warp, cnt, cs, pxc, pyc, thr, px_state);
                } else {
                    if (mode_alpha) blend_list<kChunk, false, true, kTrack>(s, warp, cnt, cs, pxc, pyc, thr, px_state);
                    else blend_list<kChunk, false, false, kTrack>(s, warp, cnt, cs, pxc, pyc, thr, px_state);
                }
                T = px_state.T; cr = px_state.cr; cg = px_state.cg; cb = px_state.cb; dep = px_state.dep;
                acc = px_state.acc; count = px_state.count; last = px_state.last; done = px_state.done;
                __syncthreads();
            }
            /* a pixel that never saturated visited the whole range */
            if (!done) last = re - 1;
        }
    }
    if (!inside) return;
    /* finalize, compositor.mojo:55-59 */
    const ViewDesc& vd = vt->view[view];
    const LumenGpuImage& img = vd.img;
    const long long pix = (long long)py * vd.cam.width + px;
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
    if (img.depth) img.depth[pix] = opt.compute_depth ? dep : 0.0f;
    if (img.alpha) img.alpha[pix] = acc;
    if (img.n_contrib) img.n_contrib[pix] = count;
    if (img.last_idx) img.last_idx[pix] = last;
}

/* One CTA per tile of the batch. kTrack: keep contributor counts and
 * last-visited offsets (some view's image asks for them). */
template <int kChunk, bool kTrack>
__global__ void __launch_bounds__(kTilePixels, kCompositeBlocksPerSm)
composite_kernel(const ViewTable* __restrict__ vt, int n_views, const LumenSplatRecord* __restrict__ records,
                 LumenGpuFrame f, long long capacity, Control* __restrict__ ctrl, LumenRenderOptions opt,
                 long long tile_offset) {
    chain_begin();
    __shared__ CompositeSmem<kChunk> s;
    init_padding_splat(s);
    composite_tile<kChunk, kTrack>(s, vt, records, f, capacity, ctrl, opt, n_views, tile_offset + blockIdx.x);
}

/* Persistent form for a grid fixed in advance (a captured graph replayed
 * for batches of any size): CTAs take tiles in ticket order. */
template <int kChunk, bool kTrack>
__global__ void __launch_bounds__(kTilePixels, kCompositeBlocksPerSm)
composite_persistent_kernel(const ViewTable* __restrict__ vt, const LumenSplatRecord* __restrict__ records,
                            LumenGpuFrame f, long long capacity, Control* __restrict__ ctrl, LumenRenderOptions opt) {
    chain_begin();
    __shared__ CompositeSmem<kChunk> s;
    init_padding_splat(s);
    const long long total = vt->hdr.total_tiles;
    const int n_views = vt->hdr.n_views;
    for (;;) {
        if (threadIdx.x == 0) s.ticket = atomicAdd(&ctrl->composite_ticket, 1u);
        __syncthreads();
        const long long t = s.ticket;
        if (t >= total) break;
        composite_tile<kChunk, kTrack>(s, vt, records, f, capacity, ctrl, opt, n_views, t);
        __syncthreads();
    }
}

template <int kChunk, bool kTrack>
static void launch_composite_chunk(const ViewTable* vt, int n_views, const LumenGpuFrame& f, Control* ctrl,
                                   const LumenRenderOptions& opt, long long tile_offset, long long n_tiles,
                                   bool persistent, int num_sms, cudaStream_t st) {
    if (persistent) {
        launch_chained(composite_persistent_kernel<kChunk, kTrack>, dim3(kCompositeBlocksPerSm * num_sms),
                       dim3(kTilePixels), 0, st, vt, (const LumenSplatRecord*)f.records, f,
                       (long long)f.instance_capacity, ctrl, opt);
    } else {
        launch_chained(composite_kernel<kChunk, kTrack>, dim3((unsigned int)n_tiles), dim3(kTilePixels), 0, st, vt,
                       n_views, (const LumenSplatRecord*)f.records, f, (long long)f.instance_capacity, ctrl, opt,
                       tile_offset);
    }
}

template <int kChunk>
static void launch_composite_track(const ViewTable* vt, int n_views, const LumenGpuFrame& f, Control* ctrl,
                                   const LumenRenderOptions& opt, long long tile_offset, long long n_tiles,
                                   bool persistent, bool track, int num_sms, cudaStream_t st) {
    if (track)
        launch_composite_chunk<kChunk, true>(vt, n_views, f, ctrl, opt, tile_offset, n_tiles, persistent, num_sms, st);
    else
        launch_composite_chunk<kChunk, false>(vt, n_views, f, ctrl, opt, tile_offset, n_tiles, persistent, num_sms, st);
}

/* chunk: instances staged per round, one of kCompositeChunks. Plain
 * launches shade tiles [tile_offset, tile_offset + n_tiles) of the batch;
 * persistent launches take every tile of the table by ticket. track: some
 * view's image asks for contributor counts or last-visited offsets. */
void launch_composite(const ViewTable* vt, int n_views, const LumenGpuFrame& f, Control* ctrl,
                      const LumenRenderOptions& opt, long long tile_offset, long long n_tiles, bool persistent,
                      int chunk, bool track, int num_sms, cudaStream_t st) {
    if (n_tiles <= 0) return;
    switch (chunk) {
        case 128:
            launch_composite_track<128>(vt, n_views, f, ctrl, opt, tile_offset, n_tiles, persistent, track, num_sms,
                                        st);
            break;
        case 512:
            launch_composite_track<512>(vt, n_views, f, ctrl, opt, tile_offset, n_tiles, persistent, track, num_sms,
                                        st);
            break;
        default:
            launch_composite_track<256>(vt, n_views, f, ctrl, opt, tile_offset, n_tiles, persistent, track, num_sms,
                                        st);
            break;
    }
}

}  // namespace lumen
