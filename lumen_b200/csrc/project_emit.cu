/*
 * project_emit.cu - K1: per-Gaussian projection fused with the compacting
 * scan and the key emission, in one pass over the parameters.
 *
 * Reference: the geometry-and-culling loop of rasterize_scene,
 * src/raster/pipeline.mojo:84-157. There, visible splats get consecutive
 * indices in Gaussian order and each one appends one key per covered tile,
 * rows (ty) outer and columns (tx) inner. Here a block of 256 threads
 * projects 256 consecutive Gaussians, scans (visible, tile count) pairs in
 * the block, and obtains the global offsets of both counts through a
 * decoupled look-back over blocks taken in ticket order, so the record
 * indices and the key positions are exactly the reference's sequential ones.
 * The block then writes its keys cooperatively: consecutive threads write
 * consecutive instances, so the key/value stores are fully coalesced no
 * matter how unequal the per-Gaussian tile counts are.
 *
 * Memory per Gaussian: 236 B of parameters read once; 48 B record + 4 B
 * visible id + 4 B radius written; 12 B per emitted instance.
 */
#include "splat_common.cuh"

namespace lumen {

/* Warp-parallel decoupled look-back over 64-bit descriptors: returns the sum
 * of all blocks before `blk`. Called by one full warp. */
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

struct ProjSmem {
    DevCamera cam;
    unsigned int blk;
    unsigned int warp_vis[kProjThreads / 32];
    unsigned int warp_inst[kProjThreads / 32];
    unsigned long long vis_base, inst_base;
    unsigned int block_vis, block_inst;
    unsigned int incl[kProjThreads];      /* inclusive instance prefix in the block */
    unsigned int dkey[kProjThreads];
    unsigned int vis_id[kProjThreads];
    unsigned short min_tx[kProjThreads], min_ty[kProjThreads], width[kProjThreads];
    unsigned long long key_or, key_or_not;
};

__global__ void __launch_bounds__(kProjThreads)
project_emit_kernel(LumenGpuGaussians g, LumenViewCamera camera, LumenRenderOptions opt,
                    LumenSplatRecord* __restrict__ records, unsigned int* __restrict__ visible_ids,
                    int* __restrict__ radii, unsigned long long* __restrict__ keys,
                    unsigned int* __restrict__ vals, long long capacity, Control* ctrl,
                    unsigned long long* lb_vis, unsigned long long* lb_inst, int nblocks) {
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
        float4 q = __ldg(reinterpret_cast<const float4*>(g.quats) + i);
        p = project_gaussian(s.cam, __ldg(m), __ldg(m + 1), __ldg(m + 2), __ldg(sc), __ldg(sc + 1),
                             __ldg(sc + 2), Quat{q.x, q.y, q.z, q.w}, __ldg(g.opacities + i),
                             g.sh + i * 48, opt);
        radii[i] = p.visible ? p.radius : 0;
    }
    const unsigned int vis = p.visible ? 1u : 0u;
    const unsigned int cnt = p.visible ? (unsigned int)((p.max_tx - p.min_tx + 1) * (p.max_ty - p.min_ty + 1)) : 0u;

    /* block scan of (vis, cnt) */
    unsigned int sv = vis, sc_ = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned int a = __shfl_up_sync(0xffffffffu, sv, o);
        unsigned int b = __shfl_up_sync(0xffffffffu, sc_, o);
        if (lane >= o) { sv += a; sc_ += b; }
    }
    if (lane == 31) { s.warp_vis[warp] = sv; s.warp_inst[warp] = sc_; }
    __syncthreads();
    if (tid == 0) {
        unsigned int rv = 0, ri = 0;
        for (int w = 0; w < kProjThreads / 32; ++w) {
            unsigned int a = s.warp_vis[w], b = s.warp_inst[w];
            s.warp_vis[w] = rv; s.warp_inst[w] = ri;
            rv += a; ri += b;
        }
        s.block_vis = rv;
        s.block_inst = ri;
        /* publish this block's aggregates (inclusive right away for block 0) */
        const unsigned long long flag = blk == 0 ? kDescIncl64 : kDescAgg64;
        st_volatile_u64(lb_vis + blk, flag | rv);
        st_volatile_u64(lb_inst + blk, flag | ri);
    }
    __syncthreads();
    const unsigned int vis_local = sv - vis + s.warp_vis[warp];       /* exclusive */
    const unsigned int inst_incl = sc_ + s.warp_inst[warp];           /* inclusive */

    /* decoupled look-back: warp 0 for instances, warp 1 for visible counts */
    if (warp == 0) {
        unsigned long long e = blk > 0 ? lookback64(lb_inst, blk, &ctrl->error_flags) : 0ull;
        if (lane == 0) {
            s.inst_base = e;
            if (blk > 0) st_volatile_u64(lb_inst + blk, kDescIncl64 | (e + s.block_inst));
        }
    } else if (warp == 1) {
        unsigned long long e = blk > 0 ? lookback64(lb_vis, blk, &ctrl->error_flags) : 0ull;
        if (lane == 0) {
            s.vis_base = e;
            if (blk > 0) st_volatile_u64(lb_vis + blk, kDescIncl64 | (e + s.block_vis));
        }
    }
    const unsigned int dk = p.visible ? depth_key(p.z, opt.key_mode) : 0u;
    s.incl[tid] = inst_incl;
    s.dkey[tid] = dk;
    s.min_tx[tid] = (unsigned short)p.min_tx;
    s.min_ty[tid] = (unsigned short)p.min_ty;
    s.width[tid] = (unsigned short)(p.visible ? (p.max_tx - p.min_tx + 1) : 1);
    __syncthreads();

    const unsigned long long vis_base = s.vis_base, inst_base = s.inst_base;
    if (p.visible) {
        const unsigned long long vid = vis_base + vis_local;
        s.vis_id[tid] = (unsigned int)vid;
        LumenSplatRecord rec;
        rec.cx = p.cx; rec.cy = p.cy; rec.depth = p.z; rec.opacity = p.op;
        rec.ic00 = p.ic00; rec.ic01 = p.ic01; rec.ic11 = p.ic11; rec.pad0 = 0.0f;
        rec.r = p.r; rec.g = p.g; rec.b = p.b; rec.pad1 = 0.0f;
        float4* dst = reinterpret_cast<float4*>(records + vid);
        dst[0] = make_float4(rec.cx, rec.cy, rec.depth, rec.opacity);
        dst[1] = make_float4(rec.ic00, rec.ic01, rec.ic11, 0.0f);
        dst[2] = make_float4(rec.r, rec.g, rec.b, 0.0f);
        visible_ids[vid] = (unsigned int)i;
    }
    if (blk == nblocks - 1 && tid == 0) {
        ctrl->n_visible = (unsigned int)(vis_base + s.block_vis);
        ctrl->n_instances = inst_base + s.block_inst;
        if (inst_base + s.block_inst > (unsigned long long)capacity)
            atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_CAPACITY);
    }
    __syncthreads();

    /* cooperative emission: instance j of the block belongs to the Gaussian
     * whose inclusive prefix is the first one above j */
    const unsigned int total = s.block_inst;
    const int tiles_x = s.cam.tiles_x;
    unsigned long long kor = 0ull, knot = 0ull;
    for (unsigned int j = tid; j < total; j += kProjThreads) {
        int lo = 0, hi = kProjThreads - 1;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (s.incl[mid] > j) hi = mid; else lo = mid + 1;
        }
        const unsigned int start = lo > 0 ? s.incl[lo - 1] : 0u;
        const unsigned int r = j - start;
        const unsigned int w = s.width[lo];
        const unsigned int ty = s.min_ty[lo] + r / w;
        const unsigned int tx = s.min_tx[lo] + r % w;
        const unsigned long long key = ((unsigned long long)(ty * tiles_x + tx) << 32) | s.dkey[lo];
        const unsigned long long pos = inst_base + j;
        kor |= key;
        knot |= ~key;
        if (pos < (unsigned long long)capacity) {
            keys[pos] = key;
            vals[pos] = s.vis_id[lo];
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kor |= __shfl_xor_sync(0xffffffffu, kor, o);
        knot |= __shfl_xor_sync(0xffffffffu, knot, o);
    }
    if (lane == 0 && total > 0) {
        atomicOr(&s.key_or, kor);
        atomicOr(&s.key_or_not, knot);
    }
    __syncthreads();
    if (tid == 0 && total > 0) {
        atomicOr(&ctrl->key_or, s.key_or);
        atomicOr(&ctrl->key_or_not, s.key_or_not);
    }
}

void launch_project_emit(const LumenGpuGaussians& g, const LumenViewCamera& cam, const LumenRenderOptions& opt,
                         LumenGpuFrame& f, Control* ctrl, unsigned long long* lb, int nblocks, cudaStream_t st) {
    project_emit_kernel<<<nblocks, kProjThreads, 0, st>>>(
        g, cam, opt, f.records, f.visible_ids, f.radii, reinterpret_cast<unsigned long long*>(f.keys[0]),
        f.vals[0], (long long)f.instance_capacity,
        ctrl, lb, lb + nblocks, nblocks);
}

}  // namespace lumen
