/*
 * project.cu - K1 (projection with the compacting scan) and K2 (instance
 * emission in depth order).
 *
 * Reference: the geometry-and-culling loop of rasterize_scene,
 * src/raster/pipeline.mojo:84-157. There, visible splats get consecutive
 * indices in Gaussian order (pipeline.mojo:141-149) and each appends one
 * key per covered tile (:152-157); the keys are then stably sorted (:166).
 *
 * K1: a block of 256 threads projects 256 consecutive Gaussians and scans
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

/* Warp-parallel decoupled look-back over 64-bit descriptors: the sum of all
 * blocks before `blk`. Called by one full warp. */
__device__ unsigned long long lookback64(const unsigned long long* desc, int blk, unsigned int* err) {
    const int lane = threadIdx.x & 31;
    unsigned long long excl = 0;
    int base = blk - 1;
    while (base >= 0) {
        int idx = base - lane;
        unsigned long long v = kDescIncl64;   /* before block 0: inclusive 0 */
        if (idx >= 0) {
            int spins = 0;
            for (;;) {
                v = ld_volatile_u64(desc + idx);
                if (v >> 62) break;
                if (++spins >= kSpinLimit) {
                    atomicOr(err, LUMEN_GPU_ERR_SPIN_TIMEOUT);
                    v = kDescIncl64;
                    break;
                }
                __nanosleep(64);
            }
        }
        unsigned int incl = __ballot_sync(0xffffffffu, (v >> 62) == 2);
        int first = incl ? __ffs(incl) - 1 : 31;
        unsigned long long c = lane <= first ? (v & kDescMask64) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        excl += c;
        if (incl) break;
        base -= 32;
    }
    return excl;
}

/* Block-wide exclusive scan of one value per thread (256 threads). */
__device__ __forceinline__ unsigned int block_exclusive_scan(unsigned int x, unsigned int* warp_tot,
                                                             unsigned int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    unsigned int before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < kProjThreads / 32; ++w) {
        const unsigned int t = warp_tot[w];
        if (w < warp) before += t;
        all += t;
    }
    *total = all;
    return before + incl - x;
}

struct ProjSmem {
    DevCamera cam;
    unsigned int blk;
    unsigned int warp_tot[kProjThreads / 32];
    unsigned long long vis_base;
    unsigned long long key_or, key_or_not;
};

__global__ void __launch_bounds__(kProjThreads)
project_kernel(LumenGpuGaussians g, LumenViewCamera camera, LumenRenderOptions opt, LumenGpuFrame f, Control* ctrl,
               unsigned long long* lb, int nblocks) {
    __shared__ ProjSmem s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s.blk = atomicAdd(&ctrl->proj_ticket, 1u);
        setup_camera(camera, s.cam);
        s.key_or = 0ull;
        s.key_or_not = 0ull;
    }
    __syncthreads();
    const int blk = (int)s.blk;
    const long long i = (long long)blk * kProjThreads + tid;

    Projected p;
    p.visible = false;
    p.radius = 0;
    if (i < g.count) {
        const float* m = g.means + i * 3;
        const float* sc = g.scales + i * 3;
        const float4 q = __ldg(reinterpret_cast<const float4*>(g.quats) + i);
        p = project_gaussian(s.cam, __ldg(m), __ldg(m + 1), __ldg(m + 2), __ldg(sc), __ldg(sc + 1),
                             __ldg(sc + 2), Quat{q.x, q.y, q.z, q.w}, __ldg(g.opacities + i),
                             g.sh + i * 48, opt);
        f.radii[i] = p.visible ? p.radius : 0;
    }
    unsigned int block_vis = 0;
    const unsigned int vis_local = block_exclusive_scan(p.visible ? 1u : 0u, s.warp_tot, &block_vis);
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
        f.rects[vid] = pack_rect(p.min_tx, p.min_ty, p.max_tx, p.max_ty);
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
        if (blk == nblocks - 1) {
            ctrl->n_visible = (unsigned int)(vis_base + block_vis);
            ctrl->depth_sort.n = vis_base + block_vis;
        }
    }
}

struct EmitSmem {
    unsigned int blk;
    unsigned int warp_tot[kProjThreads / 32];
    unsigned long long inst_base;
    unsigned int incl[kProjThreads];
    unsigned int vis[kProjThreads];
    unsigned long long rect[kProjThreads];
    unsigned long long key_or, key_or_not;
};

__global__ void __launch_bounds__(kProjThreads)
emit_kernel(LumenGpuFrame f, Control* ctrl, unsigned long long* lb, int tiles_x) {
    __shared__ EmitSmem s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s.blk = atomicAdd(&ctrl->emit_ticket, 1u);
        s.key_or = 0ull;
        s.key_or_not = 0ull;
    }
    __syncthreads();
    const long long V = ctrl->n_visible;
    const int blk = (int)s.blk;
    if ((long long)blk * kProjThreads >= V) return;   /* past the visible splats: no look-back waits on it */
    const long long p = (long long)blk * kProjThreads + tid;
    const unsigned int* order = ctrl->depth_sort.sorted_buffer ? f.depth_order[1] : f.depth_order[0];
    unsigned int cnt = 0, v = 0;
    unsigned long long r = 0ull;
    if (p < V) {
        v = order[p];
        r = f.rects[v];
        const unsigned int w = (unsigned int)((r >> 32) & 0xFFFF) - (unsigned int)(r & 0xFFFF) + 1u;
        const unsigned int h = (unsigned int)((r >> 48) & 0xFFFF) - (unsigned int)((r >> 16) & 0xFFFF) + 1u;
        cnt = w * h;
    }
    unsigned int block_inst = 0;
    const unsigned int excl = block_exclusive_scan(cnt, s.warp_tot, &block_inst);
    if (tid == 0) st_volatile_u64(lb + blk, (blk == 0 ? kDescIncl64 : kDescAgg64) | block_inst);
    s.incl[tid] = excl + cnt;
    s.vis[tid] = v;
    s.rect[tid] = r;
    if (warp == 0) {
        const unsigned long long e = blk > 0 ? lookback64(lb, blk, &ctrl->error_flags) : 0ull;
        if (lane == 0) {
            s.inst_base = e;
            if (blk > 0) st_volatile_u64(lb + blk, kDescIncl64 | (e + block_inst));
        }
    }
    __syncthreads();
    const unsigned long long inst_base = s.inst_base;
    const long long cap = f.instance_capacity;
    unsigned long long kor = 0ull, knot = 0ull;
    for (unsigned int j = tid; j < block_inst; j += kProjThreads) {
        int lo = 0, hi = kProjThreads - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (s.incl[mid] > j) hi = mid; else lo = mid + 1;
        }
        const unsigned int start = lo > 0 ? s.incl[lo - 1] : 0u;
        const unsigned long long rr = s.rect[lo];
        const unsigned int min_tx = (unsigned int)(rr & 0xFFFF), min_ty = (unsigned int)((rr >> 16) & 0xFFFF);
        const unsigned int w = (unsigned int)((rr >> 32) & 0xFFFF) - min_tx + 1u;
        const unsigned int q = j - start;
        /* rows outer, columns inner (pipeline.mojo:152-153) */
        const unsigned int tile = (min_ty + q / w) * (unsigned int)tiles_x + min_tx + q % w;
        const unsigned long long pos = inst_base + j;
        kor |= tile;
        knot |= ~(unsigned long long)tile & 0xFFFFFFFFull;
        if (pos < (unsigned long long)cap) {
            f.keys[0][pos] = tile;
            f.vals[0][pos] = s.vis[lo];
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kor |= __shfl_xor_sync(0xffffffffu, kor, o);
        knot |= __shfl_xor_sync(0xffffffffu, knot, o);
    }
    if (lane == 0 && block_inst) {
        atomicOr(&s.key_or, kor);
        atomicOr(&s.key_or_not, knot);
    }
    __syncthreads();
    if (tid == 0) {
        if (block_inst) {
            atomicOr(&ctrl->tile_sort.key_or, s.key_or);
            atomicOr(&ctrl->tile_sort.key_or_not, s.key_or_not);
        }
        if ((long long)blk == (V - 1) / kProjThreads) {
            const unsigned long long K = inst_base + block_inst;
            ctrl->n_instances = K;
            ctrl->tile_sort.n = K;
            if (K > (unsigned long long)cap) atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_CAPACITY);
        }
    }
}

void launch_project(const LumenGpuGaussians& g, const LumenViewCamera& cam, const LumenRenderOptions& opt,
                    const LumenGpuFrame& f, Control* ctrl, unsigned long long* lb, int nblocks, cudaStream_t st) {
    project_kernel<<<nblocks, kProjThreads, 0, st>>>(g, cam, opt, f, ctrl, lb, nblocks);
}

void launch_emit(const LumenGpuFrame& f, Control* ctrl, unsigned long long* lb, int nblocks, int tiles_x,
                 cudaStream_t st) {
    emit_kernel<<<nblocks, kProjThreads, 0, st>>>(f, ctrl, lb, tiles_x);
}

}  // namespace lumen
