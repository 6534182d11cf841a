/*
 * project.cu - K1 (projection with the compacting scan) and K2 (instance
 * emission in depth order).
 *
 * Reference: the geometry-and-culling loop of rasterize_scene,
 * src/raster/pipeline.mojo:84-157. There, visible splats get consecutive
 * indices in Gaussian order (pipeline.mojo:141-149) and each appends one
 * key per covered tile (:152-157); the keys are then stably sorted (:166).
 *
 * K1: a block of 128 threads projects 128 consecutive Gaussians (their SH
 * coefficients staged in shared memory by asynchronous copies) and scans
 * their visibility flags; the global offset comes from a decoupled look-back
 * over blocks taken in ticket order, so visible indices are exactly the
 * reference's sequential ones. Each visible splat writes its 48-byte record,
 * its Gaussian index, its tile rectangle and its depth key.
 *
 * K2 (after the visible splats were stably sorted by depth key): a block
 * takes 256 consecutive splats of the depth order, scans their tile counts
 * (decoupled look-back again), and writes one (tile id, visible index) pair
 * per covered tile, cooperatively, so consecutive threads write consecutive
 * instances. A stable sort of these pairs by tile id yields the reference's
 * permutation: in both, a tile's instances are ordered by (depth key,
 * visible index).
 *
 * Memory: K1 reads 236 B per Gaussian once and writes 68 B per visible
 * splat + 4 B per Gaussian; K2 reads 12 B per visible splat and writes 8 B
 * per instance.
 */
#include "splat_common.cuh"

namespace lumen {

struct ProjSmem {
    ViewDesc vd;                 /* the block's view, copied from the table */
    unsigned int blk;
    int view;
    unsigned int warp_tot[kProjThreads / 32];
    unsigned long long vis_base;
    unsigned long long key_or, key_or_not;
};

constexpr int kViewWords = (int)(sizeof(ViewDesc) / 4);
static_assert(sizeof(ViewDesc) % 4 == 0 && kViewWords <= kProjThreads - 32, "view copy layout");

/* Each CTA takes a 128-Gaussian block by ticket (kPersistent: blocks until
 * the batch's blocks are exhausted, for a grid fixed in advance). Block b
 * belongs to the last view whose block_begin <= b, and covers that view's
 * Gaussians (b - block_begin) * 128 onward; visible indices run over the
 * whole batch in block order. n_views_hint: the batch's view count, or 0
 * to read it from the table; with one view, the view is copied to shared
 * memory while the ticket is being taken. */
template <bool kPersistent>
__global__ void __launch_bounds__(kProjThreads)
project_kernel(const ViewTable* __restrict__ vt, int n_views_hint, LumenRenderOptions opt, LumenGpuFrame f,
               Control* ctrl, unsigned long long* lb) {
    chain_begin();
    __shared__ ProjSmem s;
    extern __shared__ float4 sh_stage[];   /* kProjThreads x 12: the block's SH coefficients */
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n_views = n_views_hint > 0 ? n_views_hint : vt->hdr.n_views;
    const long long total_blocks = vt->hdr.total_blocks;
    if (n_views == 1) {
        if (tid >= 32 && tid < 32 + kViewWords)
            reinterpret_cast<unsigned int*>(&s.vd)[tid - 32] = reinterpret_cast<const unsigned int*>(&vt->view[0])[tid - 32];
        if (tid == 0) s.view = 0;
    }
    for (;;) {
        if (tid == 0) {
            s.blk = atomicAdd(&ctrl->proj_ticket, 1u);
            s.key_or = 0ull;
            s.key_or_not = 0ull;
        }
        __syncthreads();
        const int blk = (int)s.blk;
        if ((long long)blk >= total_blocks) break;
        if (n_views > 1) {
            if (warp == 0) {
                const int v = find_view_by_block(vt, n_views, blk);
                const unsigned int* src = reinterpret_cast<const unsigned int*>(&vt->view[v]);
                for (int w = lane; w < kViewWords; w += 32) reinterpret_cast<unsigned int*>(&s.vd)[w] = src[w];
                if (lane == 0) s.view = v;
            }
            __syncthreads();
        }
        const long long slot = (long long)blk * kProjThreads + tid;
        const long long i0 = (long long)(blk - s.vd.block_begin) * kProjThreads;
        const long long i = i0 + tid;
        const long long count = s.vd.g.count;
        /* the block's SH rows (192 B per Gaussian, contiguous) go to shared
         * memory with coalesced 16-byte asynchronous copies, overlapped with
         * the loads of the other parameters */
        {
            const int nblk = (int)(count - i0 < kProjThreads ? count - i0 : kProjThreads);
            const float4* src = reinterpret_cast<const float4*>(s.vd.g.sh + i0 * 48);
            for (int c = tid; c < nblk * 12; c += kProjThreads) {
                const int t = c / 12, q = c - 12 * t;
                cp_async16(sh_stage + 12 * t + (q ^ sh_swizzle(t)), src + c);
            }
            cp_async_commit();
        }
        float mx = 0.0f, my = 0.0f, mz = 0.0f, sx = 0.0f, sy = 0.0f, sz = 0.0f, op = 0.0f;
        float4 q = make_float4(1.0f, 0.0f, 0.0f, 0.0f);
        if (i < count) {
            const LumenGpuGaussians& g = s.vd.g;
            const float* m = g.means + i * 3;
            const float* sc = g.scales + i * 3;
            q = __ldg(reinterpret_cast<const float4*>(g.quats) + i);
            mx = __ldg(m); my = __ldg(m + 1); mz = __ldg(m + 2);
            sx = __ldg(sc); sy = __ldg(sc + 1); sz = __ldg(sc + 2);
            op = __ldg(g.opacities + i);
        }
        cp_async_wait_all();
        __syncthreads();

        Projected p;
        p.visible = false;
        p.radius = 0;
        if (i < count) {
            p = project_gaussian(s.vd.dcam, mx, my, mz, sx, sy, sz, Quat{q.x, q.y, q.z, q.w}, op,
                                 reinterpret_cast<const float*>(sh_stage + tid * 12), opt, sh_swizzle(tid));
            if (f.radii) f.radii[slot] = p.visible ? p.radius : 0;
        }
        unsigned int block_vis = 0;
        const unsigned int vis_local = block_exclusive_scan<kProjThreads>(p.visible ? 1u : 0u, s.warp_tot, &block_vis);
        if (tid == 0) st_volatile_u64(lb + blk, (blk == 0 ? kDescIncl64 : kDescAgg64) | block_vis);
        if (warp == 0) {
            const unsigned long long e = blk > 0 ? lookback64(lb, blk, &ctrl->error_flags) : 0ull;
            if (lane == 0) {
                s.vis_base = e;
                if (blk > 0) st_volatile_u64(lb + blk, kDescIncl64 | (e + block_vis));
            }
        }
        __syncthreads();
        const unsigned long long vis_base = s.vis_base;
        unsigned long long kor = 0ull, knot = 0ull;
        if (p.visible) {
            const unsigned long long vid = vis_base + vis_local;
            float4* dst = reinterpret_cast<float4*>(f.records + vid);
            dst[0] = make_float4(p.cx, p.cy, p.z, p.op);
            dst[1] = make_float4(p.ic00, p.ic01, p.ic11, 0.0f);
            dst[2] = make_float4(p.r, p.g, p.b, 0.0f);
            f.visible_ids[vid] = (unsigned int)i;
            f.rects[vid] = pack_rect(p.min_tx, p.min_ty, p.max_tx, p.max_ty, s.view);
            const unsigned int dk = depth_key(p.z, opt.key_mode);
            f.depth_keys[0][vid] = dk;
            f.depth_order[0][vid] = (unsigned int)vid;
            kor = dk;
            knot = ~(unsigned long long)dk & 0xFFFFFFFFull;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            kor |= __shfl_xor_sync(0xffffffffu, kor, o);
            knot |= __shfl_xor_sync(0xffffffffu, knot, o);
        }
        if (lane == 0 && block_vis) {
            atomicOr(&s.key_or, kor);
            atomicOr(&s.key_or_not, knot);
        }
        __syncthreads();
        if (tid == 0) {
            if (block_vis) {
                atomicOr(&ctrl->depth_sort.key_or, s.key_or);
                atomicOr(&ctrl->depth_sort.key_or_not, s.key_or_not);
            }
            if ((long long)blk == total_blocks - 1) {
                ctrl->n_visible = (unsigned int)(vis_base + block_vis);
                ctrl->depth_sort.n = vis_base + block_vis;
            }
        }
        if (!kPersistent) break;
        __syncthreads();
    }
}

/* Instances of an emission warp resolved to their splats per window. */
constexpr int kEmitWindow = 256;
constexpr int kEmitPerLane = kEmitWindow / 32;
static_assert(kEmitPerLane == 8, "two 16-byte slot groups per lane");

struct EmitSmem {
    /* per warp and window slot: 1 + the lane whose splat holds the instance */
    __align__(16) unsigned int owner[kEmitThreads / 32][kEmitWindow];
    unsigned int blk;
    unsigned int warp_tot[kEmitThreads / 32];
    unsigned long long inst_base;
    /* per splat: its first instance (block-relative), tiles per rectangle
     * row, the batch-wide id of its first tile, tiles per view row */
    uint4 run[kEmitThreads];
    /* per splat: 1 / (tiles per rectangle row), as bits, for the row of an
     * instance; its visible index */
    uint2 aux[kEmitThreads];
    unsigned int hist[4][256];            /* the block's tile ids: counts of each digit value */
    unsigned long long key_or, key_or_not;
};
static_assert(kEmitThreads == 256, "one emission thread per digit value clears and adds the block's counts");

/* Owners of the warp's window [a, a + kEmitWindow): slot k of s.owner[warp]
 * gets 1 + the lane whose splat holds instance a + k (block-relative). Returns
 * the window's instance count. */
__device__ __forceinline__ unsigned int emit_window_owners(EmitSmem& s, int warp, int lane, unsigned int a,
                                                           unsigned int excl, unsigned int cnt, unsigned int w_end) {
    unsigned int* own = s.owner[warp];
    uint4* o4 = reinterpret_cast<uint4*>(own) + lane * 2;
    o4[0] = make_uint4(0u, 0u, 0u, 0u);
    o4[1] = make_uint4(0u, 0u, 0u, 0u);
    __syncwarp();
    if (cnt && excl + cnt > a && excl < a + kEmitWindow) own[(excl > a ? excl : a) - a] = (unsigned int)lane + 1u;
    __syncwarp();
    /* inclusive prefix maximum: eight consecutive slots per lane, then
     * across the lanes */
    const uint4 g0 = o4[0], g1 = o4[1];
    unsigned int m[kEmitPerLane] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
#pragma unroll
    for (int k = 1; k < kEmitPerLane; ++k) m[k] = max(m[k], m[k - 1]);
    unsigned int x = m[kEmitPerLane - 1];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, y);
    }
    unsigned int pre = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) pre = 0u;
    o4[0] = make_uint4(max(pre, m[0]), max(pre, m[1]), max(pre, m[2]), max(pre, m[3]));
    o4[1] = make_uint4(max(pre, m[4]), max(pre, m[5]), max(pre, m[6]), max(pre, m[7]));
    __syncwarp();
    return w_end - a < (unsigned int)kEmitWindow ? w_end - a : kEmitWindow;
}

/* Batch-wide tile id of block-relative instance j of splat lo: rows outer,
 * columns inner (pipeline.mojo:152-153). */
__device__ __forceinline__ unsigned int emit_tile(const EmitSmem& s, int lo, unsigned int j) {
    const uint4 rn = s.run[lo];
    const unsigned int w = rn.y;
    const unsigned int q = j - rn.x;
    /* q / w through the reciprocal (exact after one correction step while
     * q < 2^20), integer division beyond */
    unsigned int row;
    if (q < (1u << 20)) {
        row = (unsigned int)((float)q * __uint_as_float(s.aux[lo].x));
        if (row * w > q) --row;
        else if ((row + 1u) * w <= q) ++row;
    } else {
        row = q / w;
    }
    return rn.z + row * rn.w + (q - row * w);
}

/* Writes the instance at pos when it is within the capacity; counts its low
 * tile-id digit. Returns whether it was written. */
__device__ __forceinline__ bool emit_store(const LumenGpuFrame& f, EmitSmem& s, unsigned long long pos,
                                           long long cap, unsigned int tile, int lo) {
    if (pos >= (unsigned long long)cap) return false;
    f.keys[0][pos] = tile;
    f.vals[0][pos] = s.aux[lo].y;
    atomicAdd(&s.hist[0][tile & 0xFFu], 1u);
    return true;
}

/* The higher tile-id digits of the warp's written instances (a prefix of
 * its lanes). They change rarely from one instance to the next (a splat's
 * row of tiles): each run of equal values over consecutive lanes is counted
 * once, by its first lane. */
__device__ __forceinline__ void emit_count(EmitSmem& s, int lane, int nd, unsigned int tile, bool kept) {
    const unsigned int n_kept = __popc(__ballot_sync(0xffffffffu, kept));
    for (int d = 1; d < nd; ++d) {
        const unsigned int dv = kept ? (tile >> (8 * d)) & 0xFFu : 0x100u;
        const unsigned int prev = __shfl_up_sync(0xffffffffu, dv, 1);
        const bool first = kept && (lane == 0 || prev != dv);
        const unsigned int firsts = __ballot_sync(0xffffffffu, first);
        if (first) {
            const unsigned int later = firsts & ~((2u << lane) - 1u);
            const unsigned int run_end = later ? (unsigned int)(__ffs(later) - 1) : n_kept;
            atomicAdd(&s.hist[d][dv], run_end - (unsigned int)lane);
        }
    }
}

/* Like project_kernel: 256 consecutive splats of the depth order per ticket.
 * Tile ids are batch-wide (view tile_begin + ty * tiles_x + tx).
 *
 * The emission also does the tile sort's preparation, so that the sort
 * needs no pass of its own over the instances: it counts the digit values
 * of the tile ids it writes (per block in shared memory, then added to the
 * sort's histogram), clears the sort's look-back descriptors of the
 * 256 * sort_items-key tiles that start among its instances, and fills the
 * tile ranges with (-1, -1). */
template <bool kPersistent>
__global__ void __launch_bounds__(kEmitThreads, 8)
emit_kernel(const ViewTable* __restrict__ vt, LumenGpuFrame f, Control* ctrl, unsigned long long* lb,
            unsigned int* sort_lb, long long sort_lb_tiles, int sort_tile_keys) {
    chain_begin();
    __shared__ EmitSmem s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long V = ctrl->n_visible;
    const unsigned int* order = ctrl->depth_sort.sorted_buffer ? f.depth_order[1] : f.depth_order[0];
    const long long cap = f.instance_capacity;
    /* the tile-id bytes that can vary: ids are below the batch's tile count */
    const long long n_tiles = vt->hdr.total_tiles;
    int nd = 0;
    for (long long t = n_tiles - 1; t > 0 && nd < 4; t >>= 8) ++nd;
    {
        const long long nthreads = (long long)gridDim.x * blockDim.x;
        for (long long j = (long long)blockIdx.x * blockDim.x + tid; j < 2 * n_tiles; j += nthreads) f.ranges[j] = -1;
    }
    for (;;) {
        if (tid == 0) {
            s.blk = atomicAdd(&ctrl->emit_ticket, 1u);
            s.key_or = 0ull;
            s.key_or_not = 0ull;
        }
        for (int d = 0; d < nd; ++d) s.hist[d][tid] = 0u;
        __syncthreads();
        const int blk = (int)s.blk;
        if ((long long)blk * kEmitThreads >= V) break;   /* past the visible splats: no look-back waits on it */
        const long long p = (long long)blk * kEmitThreads + tid;
        unsigned int cnt = 0, v = 0, w = 1, tile0 = 0, tiles_x = 0;
        if (p < V) {
            v = order[p];
            const unsigned long long r = f.rects[v];
            const int mnx = rect_min_tx(r), mny = rect_min_ty(r);
            w = (unsigned int)(rect_max_tx(r) - mnx + 1);
            const unsigned int h = (unsigned int)(rect_max_ty(r) - mny + 1);
            cnt = w * h;
            const ViewDesc& vd = vt->view[rect_view(r)];
            tiles_x = (unsigned int)vd.tiles_x;
            tile0 = (unsigned int)vd.tile_begin + (unsigned int)mny * tiles_x + (unsigned int)mnx;
        }
        unsigned int block_inst = 0;
        const unsigned int excl = block_exclusive_scan<kEmitThreads>(cnt, s.warp_tot, &block_inst);
        if (tid == 0) st_volatile_u64(lb + blk, (blk == 0 ? kDescIncl64 : kDescAgg64) | block_inst);
        s.run[tid] = make_uint4(excl, w, tile0, tiles_x);
        s.aux[tid] = make_uint2(__float_as_uint(1.0f / (float)w), v);
        if (warp == 0) {
            const unsigned long long e = blk > 0 ? lookback64(lb, blk, &ctrl->error_flags) : 0ull;
            if (lane == 0) {
                s.inst_base = e;
                if (blk > 0) st_volatile_u64(lb + blk, kDescIncl64 | (e + block_inst));
            }
        }
        __syncthreads();
        const unsigned long long inst_base = s.inst_base;
        unsigned int kor = 0u, knot = 0u;
        /* The warp's instances (those of its 32 splats, consecutive in the
         * block's instance order), kEmitWindow at a time. Each splat marks
         * the slot where its run of instances enters the window (the splat
         * already running at the window's start marks slot 0); a prefix
         * maximum over the marks then gives every slot its splat without a
         * search, and consecutive lanes write consecutive instances. Warps
         * work through their windows independently: only warp barriers. */
        const unsigned int my_end = excl + cnt;
        const unsigned int w_begin = __shfl_sync(0xffffffffu, excl, 0);
        const unsigned int w_end = __shfl_sync(0xffffffffu, my_end, 31);
        for (unsigned int a = w_begin; a < w_end; a += kEmitWindow) {
            const unsigned int nwin = emit_window_owners(s, warp, lane, a, excl, cnt, w_end);
            for (unsigned int b0 = 0; b0 < nwin; b0 += 32) {
                const unsigned int jj = b0 + lane;
                unsigned int tile = 0u;
                bool kept = false;
                if (jj < nwin) {
                    const int lo = warp * 32 + (int)s.owner[warp][jj] - 1;
                    tile = emit_tile(s, lo, a + jj);
                    kor |= tile;
                    knot |= ~tile;
                    kept = emit_store(f, s, inst_base + a + jj, cap, tile, lo);
                }
                emit_count(s, lane, nd, tile, kept);
            }
            __syncwarp();
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            kor |= __shfl_xor_sync(0xffffffffu, kor, o);
            knot |= __shfl_xor_sync(0xffffffffu, knot, o);
        }
        if (lane == 0 && block_inst) {
            atomicOr(&s.key_or, (unsigned long long)kor);
            atomicOr(&s.key_or_not, (unsigned long long)knot);
        }
        __syncthreads();
        for (int d = 0; d < nd; ++d) {
            const unsigned int c = s.hist[d][tid];
            if (c) atomicAdd(&ctrl->tile_sort.hist[d][tid], c);
        }
        /* look-back descriptors of the sort tiles whose first key is one of
         * this block's instances (every tile of the sort has one) */
        {
            /* only the first `capacity` instances are sorted (capacity < 2^30) */
            const unsigned long long ucap = (unsigned long long)cap;
            const unsigned long long e0 = inst_base, e1 = inst_base + block_inst;
            const unsigned int i0 = (unsigned int)(e0 < ucap ? e0 : ucap), i1 = (unsigned int)(e1 < ucap ? e1 : ucap);
            const unsigned int tk = (unsigned int)sort_tile_keys;
            const unsigned int t0 = (i0 + tk - 1u) / tk;
            unsigned int t1 = (i1 + tk - 1u) / tk;
            if ((long long)t1 > sort_lb_tiles) t1 = (unsigned int)sort_lb_tiles;
            for (int d = 0; d < nd; ++d) {
                unsigned int* region = sort_lb + (size_t)d * (size_t)sort_lb_tiles * 256;
                for (unsigned int j = t0 * 256u + (unsigned int)tid; j < t1 * 256u; j += kEmitThreads) region[j] = 0u;
            }
        }
        if (tid == 0) {
            if (block_inst) {
                atomicOr(&ctrl->tile_sort.key_or, s.key_or);
                atomicOr(&ctrl->tile_sort.key_or_not, s.key_or_not);
            }
            if ((long long)blk == (V - 1) / kEmitThreads) {
                const unsigned long long K = inst_base + block_inst;
                ctrl->n_instances = K;
                ctrl->tile_sort.n = K;
                if (K > (unsigned long long)cap) atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_CAPACITY);
            }
        }
        if (!kPersistent) break;
        __syncthreads();
    }
}

/* ---------------------------------------------------------------------
 * Gaussian-major batch projection. Views of one scene in a batch share
 * every input of the projection but the camera, so a unit of work is one
 * 128-Gaussian block of a distinct scene, projected into every view of
 * that scene: its 236 bytes per Gaussian are read once per batch instead of
 * once per view. The visible indices stay the per-view-major order of
 * project_kernel (view v's block b at the position the blocks before it in
 * (view, block) order leave), so every output is the one-view-at-a-time
 * pipeline's. Three launches:
 *   batch_count_kernel:   per unit and view, the block's visible count
 *                         (geometry only: 44 bytes per Gaussian);
 *   batch_offsets_kernel: exclusive scan of the counts in (view, block)
 *                         order (decoupled look-back over 2048-count tiles),
 *                         written over the counts;
 *   batch_project_kernel: per unit, the SH rows staged once, then for every
 *                         view the full projection, the record, index,
 *                         rectangle and depth key at the view's offset.
 * --------------------------------------------------------------------- */

constexpr int kCamWords = (int)(sizeof(DevCamera) / 4);
static_assert(sizeof(DevCamera) % 4 == 0 && kCamWords <= kProjThreads, "camera copy layout");
constexpr int kOffsetsThreads = 1024;
constexpr int kOffsetsItems = 8;    /* 8192 counts per tile: one tile for a 1M-Gaussian view */
constexpr int kOffsetsTile = kOffsetsThreads * kOffsetsItems;
/* resident projection CTAs per SM: 64 registers, 8 x 24.6 KB of staged SH rows */
constexpr int kBatchProjectCtas = 8;

struct BatchProjSmem {
    DevCamera cam;
    unsigned long long unit;
    unsigned int warp_tot[kProjThreads / 32];
    unsigned long long key_or, key_or_not;
};

/* The counts (u32 per (view, block)) and, after them, the scan's
 * descriptors, in the project look-back region of the scratch. */
__device__ __forceinline__ unsigned long long* offsets_desc(unsigned long long* lb, long long total_blocks) {
    return lb + (total_blocks + 1) / 2;
}

__device__ __forceinline__ void copy_camera(DevCamera& dst, const DevCamera& src) {
    const int tid = threadIdx.x;
    if (tid < kCamWords) reinterpret_cast<unsigned int*>(&dst)[tid] = reinterpret_cast<const unsigned int*>(&src)[tid];
}

/* The unit's Gaussian parameters (zeros past the scene's end). */
struct UnitParams {
    float mx, my, mz;
    Prepared pr;
};

__device__ __forceinline__ UnitParams load_unit_params(const LumenGpuGaussians& g, long long i,
                                                       const LumenRenderOptions& opt) {
    UnitParams u;
    u.mx = u.my = u.mz = 0.0f;
    u.pr.ok = false;
    u.pr.op = 0.0f;
    u.pr.s00 = u.pr.s01 = u.pr.s02 = u.pr.s11 = u.pr.s12 = u.pr.s22 = 0.0f;
    if (i < g.count) {
        const float* m = g.means + i * 3;
        const float* sc = g.scales + i * 3;
        const float4 q = __ldg(reinterpret_cast<const float4*>(g.quats) + i);
        u.mx = __ldg(m); u.my = __ldg(m + 1); u.mz = __ldg(m + 2);
        u.pr = prepare_gaussian(__ldg(sc), __ldg(sc + 1), __ldg(sc + 2), Quat{q.x, q.y, q.z, q.w},
                                __ldg(g.opacities + i), opt);
    }
    return u;
}

template <bool kPersistent>
__global__ void __launch_bounds__(kProjThreads)
batch_count_kernel(const ViewTable* __restrict__ vt, LumenRenderOptions opt, Control* ctrl,
                   unsigned long long* lb) {
    chain_begin();
    __shared__ BatchProjSmem s;
    const int tid = threadIdx.x;
    const int n_views = vt->hdr.n_views;
    const long long total_units = vt->hdr.total_units;
    unsigned int* counts = reinterpret_cast<unsigned int*>(lb);
    for (;;) {
        if (kPersistent) {
            if (tid == 0) s.unit = atomicAdd(&ctrl->count_ticket, 1u);
            __syncthreads();
        } else if (tid == 0) {
            s.unit = blockIdx.x;
        }
        __syncthreads();
        const long long u = (long long)s.unit;
        if (u >= total_units) break;
        const int lead = find_view_by_unit(vt, n_views, u);
        const long long b = u - vt->view[lead].unit_begin;
        const UnitParams up = load_unit_params(vt->view[lead].g, b * kProjThreads + tid, opt);
        for (int v = lead; v >= 0; v = vt->view[v].group_next) {
            copy_camera(s.cam, vt->view[v].dcam);
            __syncthreads();
            const bool vis = project_prepared<false>(s.cam, up.mx, up.my, up.mz, up.pr, nullptr, opt).visible;
            const int c = __syncthreads_count(vis);
            if (tid == 0) counts[vt->view[v].block_begin + b] = (unsigned int)c;
        }
        if (!kPersistent) break;
        __syncthreads();
    }
}

/* Exclusive scan of the (view, block) visible counts in place; the total
 * is the batch's visible count. */
__global__ void __launch_bounds__(kOffsetsThreads)
batch_offsets_kernel(const ViewTable* __restrict__ vt, Control* ctrl, unsigned long long* lb) {
    chain_begin();
    __shared__ unsigned int warp_tot[kOffsetsThreads / 32];
    __shared__ unsigned int tile_s;
    __shared__ unsigned long long base_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long nb = vt->hdr.total_blocks;
    const long long ntiles = (nb + kOffsetsTile - 1) / kOffsetsTile;
    unsigned int* counts = reinterpret_cast<unsigned int*>(lb);
    unsigned long long* desc = offsets_desc(lb, nb);
    for (;;) {
        if (tid == 0) tile_s = atomicAdd(&ctrl->offsets_ticket, 1u);
        __syncthreads();
        const long long t = tile_s;
        if (t >= ntiles) break;
        const long long i0 = t * kOffsetsTile + (long long)tid * kOffsetsItems;
        unsigned int c[kOffsetsItems];
        unsigned int sum = 0;
#pragma unroll
        for (int k = 0; k < kOffsetsItems; ++k) {
            c[k] = i0 + k < nb ? counts[i0 + k] : 0u;
            sum += c[k];
        }
        unsigned int tot = 0;
        const unsigned int ex = block_exclusive_scan<kOffsetsThreads>(sum, warp_tot, &tot);
        if (tid == 0) st_volatile_u64(desc + t, (t == 0 ? kDescIncl64 : kDescAgg64) | tot);
        if (warp == 0) {
            const unsigned long long e = t > 0 ? lookback64(desc, (int)t, &ctrl->error_flags) : 0ull;
            if (lane == 0) {
                base_s = e;
                if (t > 0) st_volatile_u64(desc + t, kDescIncl64 | (e + tot));
            }
        }
        __syncthreads();
        unsigned long long run = base_s + ex;
#pragma unroll
        for (int k = 0; k < kOffsetsItems; ++k) {
            if (i0 + k < nb) counts[i0 + k] = (unsigned int)run;
            run += c[k];
        }
        if (tid == 0 && t == ntiles - 1) {
            ctrl->n_visible = (unsigned int)(base_s + tot);
            ctrl->depth_sort.n = base_s + tot;
        }
        __syncthreads();
    }
}

template <bool kPersistent>
__global__ void __launch_bounds__(kProjThreads, kBatchProjectCtas)
batch_project_kernel(const ViewTable* __restrict__ vt, LumenRenderOptions opt, LumenGpuFrame f, Control* ctrl,
                     const unsigned long long* lb) {
    chain_begin();
    __shared__ BatchProjSmem s;
    extern __shared__ float4 sh_stage[];   /* kProjThreads x 12: the unit's SH coefficients */
    const int tid = threadIdx.x, lane = tid & 31;
    const int n_views = vt->hdr.n_views;
    const long long total_units = vt->hdr.total_units;
    const unsigned int* offsets = reinterpret_cast<const unsigned int*>(lb);
    for (;;) {
        if (tid == 0) {
            s.unit = kPersistent ? (unsigned long long)atomicAdd(&ctrl->proj_ticket, 1u) : blockIdx.x;
            s.key_or = 0ull;
            s.key_or_not = 0ull;
        }
        __syncthreads();
        const long long u = (long long)s.unit;
        if (u >= total_units) break;
        const int lead = find_view_by_unit(vt, n_views, u);
        const LumenGpuGaussians& g = vt->view[lead].g;
        const long long b = u - vt->view[lead].unit_begin;
        const long long i0 = b * kProjThreads, i = i0 + tid;
        {
            const long long count = g.count;
            const int nblk = (int)(count - i0 < kProjThreads ? count - i0 : kProjThreads);
            const float4* src = reinterpret_cast<const float4*>(g.sh + i0 * 48);
            for (int c = tid; c < nblk * 12; c += kProjThreads) {
                const int t = c / 12, q = c - 12 * t;
                cp_async16(sh_stage + 12 * t + (q ^ sh_swizzle(t)), src + c);
            }
            cp_async_commit();
        }
        const UnitParams up = load_unit_params(g, i, opt);
        const bool in_scene = i < g.count;
        cp_async_wait_all();
        unsigned long long kor = 0ull, knot = 0ull;
        for (int v = lead; v >= 0; v = vt->view[v].group_next) {
            copy_camera(s.cam, vt->view[v].dcam);
            __syncthreads();
            const Projected p = project_prepared<true>(s.cam, up.mx, up.my, up.mz, up.pr,
                                                       reinterpret_cast<const float*>(sh_stage + tid * 12), opt,
                                                       sh_swizzle(tid));
            const long long blk = vt->view[v].block_begin + b;
            if (f.radii && in_scene) f.radii[blk * kProjThreads + tid] = p.visible ? p.radius : 0;
            unsigned int n_vis = 0;
            const unsigned int vis_local = block_exclusive_scan<kProjThreads>(p.visible ? 1u : 0u, s.warp_tot, &n_vis);
            if (p.visible) {
                const unsigned long long vid = (unsigned long long)offsets[blk] + vis_local;
                float4* dst = reinterpret_cast<float4*>(f.records + vid);
                dst[0] = make_float4(p.cx, p.cy, p.z, p.op);
                dst[1] = make_float4(p.ic00, p.ic01, p.ic11, 0.0f);
                dst[2] = make_float4(p.r, p.g, p.b, 0.0f);
                f.visible_ids[vid] = (unsigned int)i;
                f.rects[vid] = pack_rect(p.min_tx, p.min_ty, p.max_tx, p.max_ty, v);
                const unsigned int dk = depth_key(p.z, opt.key_mode);
                f.depth_keys[0][vid] = dk;
                f.depth_order[0][vid] = (unsigned int)vid;
                kor |= dk;
                knot |= ~(unsigned long long)dk & 0xFFFFFFFFull;
            }
            __syncthreads();   /* s.cam and s.warp_tot are rewritten for the next view */
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            kor |= __shfl_xor_sync(0xffffffffu, kor, o);
            knot |= __shfl_xor_sync(0xffffffffu, knot, o);
        }
        if (lane == 0 && (kor | knot)) {
            atomicOr(&s.key_or, kor);
            atomicOr(&s.key_or_not, knot);
        }
        __syncthreads();
        if (tid == 0 && (s.key_or | s.key_or_not)) {
            atomicOr(&ctrl->depth_sort.key_or, s.key_or);
            atomicOr(&ctrl->depth_sort.key_or_not, s.key_or_not);
        }
        if (!kPersistent) break;
        __syncthreads();
    }
}

static int resident_ctas(const void* kernel, int threads, size_t smem) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm <= 0)
        per_sm = 1;
    return per_sm;
}

static int g_project_per_sm = 0, g_emit_per_sm = 0, g_batch_count_per_sm = 0, g_batch_project_per_sm = 0;
constexpr size_t kProjStageBytes = (size_t)kProjThreads * 48 * sizeof(float);

/* Kernel attributes and the occupancy of the persistent kernels, set and
 * queried once (before any capture). */
void prime_persistent_launches() {
    cudaFuncSetAttribute(project_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kProjStageBytes);
    cudaFuncSetAttribute(project_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kProjStageBytes);
    g_project_per_sm = resident_ctas((const void*)project_kernel<true>, kProjThreads, kProjStageBytes);
    g_emit_per_sm = resident_ctas((const void*)emit_kernel<true>, kEmitThreads, 0);
    cudaFuncSetAttribute(batch_project_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kProjStageBytes);
    cudaFuncSetAttribute(batch_project_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kProjStageBytes);
    g_batch_count_per_sm = resident_ctas((const void*)batch_count_kernel<true>, kProjThreads, 0);
    g_batch_project_per_sm = resident_ctas((const void*)batch_project_kernel<true>, kProjThreads, kProjStageBytes);
}

/* Gaussian-major projection of a batch: n_units is the batch's unit count
 * (plain launches: one CTA per unit) or 0 for persistent launches, which
 * read the count from the table. */
void launch_batch_project(const ViewTable* vt, const LumenRenderOptions& opt, const LumenGpuFrame& f,
                          Control* ctrl, unsigned long long* lb, long long n_units, long long n_blocks,
                          bool persistent, int num_sms, cudaStream_t st) {
    if (persistent) {
        const int pc = g_batch_count_per_sm > 0 ? g_batch_count_per_sm : 1;
        launch_chained(batch_count_kernel<true>, dim3(pc * num_sms), dim3(kProjThreads), 0, st, vt, opt, ctrl, lb);
        launch_chained(batch_offsets_kernel, dim3(2 * num_sms), dim3(kOffsetsThreads), 0, st, vt, ctrl, lb);
        const int pp = g_batch_project_per_sm > 0 ? g_batch_project_per_sm : 1;
        launch_chained(batch_project_kernel<true>, dim3(pp * num_sms), dim3(kProjThreads), kProjStageBytes, st, vt,
                       opt, f, ctrl, (const unsigned long long*)lb);
        return;
    }
    if (n_units <= 0) return;
    const long long tiles = (n_blocks + kOffsetsTile - 1) / kOffsetsTile;
    launch_chained(batch_count_kernel<false>, dim3((unsigned int)n_units), dim3(kProjThreads), 0, st, vt, opt, ctrl,
                   lb);
    launch_chained(batch_offsets_kernel, dim3((unsigned int)(tiles > 0 ? tiles : 1)), dim3(kOffsetsThreads), 0, st,
                   vt, ctrl, lb);
    launch_chained(batch_project_kernel<false>, dim3((unsigned int)n_units), dim3(kProjThreads), kProjStageBytes, st,
                   vt, opt, f, ctrl, (const unsigned long long*)lb);
}

/* Plain launches: one CTA per block (n_blocks known on the host).
 * Persistent launches: every resident CTA, taking tickets. */
void launch_project(const ViewTable* vt, int n_views, const LumenRenderOptions& opt, const LumenGpuFrame& f,
                    Control* ctrl, unsigned long long* lb, long long n_blocks, bool persistent, int num_sms,
                    cudaStream_t st) {
    if (n_blocks <= 0) return;
    if (persistent) {
        const int per_sm = g_project_per_sm > 0 ? g_project_per_sm : 1;
        launch_chained(project_kernel<true>, dim3(per_sm * num_sms), dim3(kProjThreads), kProjStageBytes, st, vt,
                       n_views, opt, f, ctrl, lb);
    } else {
        launch_chained(project_kernel<false>, dim3((unsigned int)n_blocks), dim3(kProjThreads), kProjStageBytes, st,
                       vt, n_views, opt, f, ctrl, lb);
    }
}

/* sort_lb: the tile sort's look-back region (sort_lb_tiles descriptor
 * tiles per digit) for digit passes of sort_tile_keys keys per tile. */
void launch_emit(const ViewTable* vt, const LumenGpuFrame& f, Control* ctrl, unsigned long long* lb,
                 unsigned int* sort_lb, long long sort_lb_tiles, int sort_tile_keys, long long n_blocks,
                 bool persistent, int num_sms, cudaStream_t st) {
    if (n_blocks <= 0) return;
    if (persistent) {
        const int per_sm = g_emit_per_sm > 0 ? g_emit_per_sm : 1;
        launch_chained(emit_kernel<true>, dim3(per_sm * num_sms), dim3(kEmitThreads), 0, st, vt, f, ctrl, lb, sort_lb,
                       sort_lb_tiles, sort_tile_keys);
    } else {
        launch_chained(emit_kernel<false>,
                       dim3((unsigned int)((n_blocks * kProjThreads + kEmitThreads - 1) / kEmitThreads)),
                       dim3(kEmitThreads), 0, st, vt, f, ctrl, lb, sort_lb, sort_lb_tiles, sort_tile_keys);
    }
}

}  // namespace lumen
