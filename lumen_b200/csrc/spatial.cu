/*
 * spatial.cu - picking on the device (include/lumen_spatial.h): the LBVH
 * build and closest-splat ray casts.
 *
 * Reference: LBVH.build_from_cloud (src/spatial/bvh.mojo:45-120),
 * compute_morton_3d / expand_bits_10_to_30 (src/spatial/morton.mojo:7-46),
 * AABB3f.expand_point / expand_box / intersect_ray (src/spatial/aabb.mojo:47-98),
 * raycast_closest_splat (src/spatial/raycast.mojo:30-95), Ray3f and
 * PinholeCamera.generate_ray (src/scene/camera.mojo:12-21, 85-90).
 *
 * Build, all on one stream:
 *   K1 bbox_kernel      the cloud's box: per-axis min and max of the positions
 *                       (NaN skipped, as add_gaussian's comparisons skip it),
 *                       reduced with atomicMax on order-preserving bit keys
 *   K2 morton_kernel    one 30-bit code per Gaussian, index as the value
 *   K3 the library's stable onesweep radix sort (32-bit keys, 4 digit passes)
 *   K4 bvh_levels_kernel, once per ten levels: a block writes 1024 leaves
 *                       (or loads 1024 nodes of the level reached so far)
 *                       and builds their ancestors ten levels up in shared
 *                       memory, one barrier per level. Parents pair adjacent
 *                       nodes, so 1024 aligned nodes never need another
 *                       block's: each parent is built once, in the
 *                       reference's order (left box expanded by the right),
 *                       and the nodes equal the reference's level-by-level
 *                       pairing bit for bit (1M leaves: two launches).
 *                       Node numbering is the reference's: leaves, then each
 *                       level's parents.
 * Casts: one thread per ray, the reference's depth-first traversal with its
 * stack order (left pushed before right) and its pruning against the
 * closest hit so far, so hits agree bit for bit, ties included.
 *
 * Memory: the build reads 24 B per Gaussian twice and writes 32 B per node
 * (n + ceil(n / 2) + ceil(n / 4) + ... nodes, about 64 MB for 1M Gaussians) plus the sort's traffic.
 */
#include "splat_common.cuh"
#include "../../include/lumen_spatial.h"

namespace lumen {
LumenStatus map_cuda(cudaError_t e);
LumenStatus status_from_flags(unsigned int flags);
int device_sm_count();
void configure_once();
void launch_key_stats32(const unsigned int* keys, long long n, SortControl* sc, int num_sms, cudaStream_t st);
void launch_sort32(unsigned int* k0, unsigned int* v0, unsigned int* k1, unsigned int* v1, long long capacity,
                   SortControl* sc, unsigned int* lb, long long lb_tiles_cap, int* ranges,
                   const long long* n_range_tiles, unsigned int* err, int items, int key_bytes, int num_sms,
                   cudaStream_t st);

namespace {

constexpr int kMaxLevels = 40;        /* 2^30 leaves need 31 levels */
constexpr int kRayStack = 64;         /* a traversal holds at most levels + 1 entries */
constexpr int kBvhSortItems = 16;     /* 4096-key sort tiles */

struct BvhControl {
    SortControl sort;
    unsigned int error_flags;
    unsigned int lo[3];               /* max of ~key(p): the minimum, 0 when none */
    unsigned int hi[3];               /* max of key(p): the maximum, 0 when none */
};

struct BvhLevels {
    int n_levels;
    long long start[kMaxLevels];
    long long count[kMaxLevels];
};

struct BvhLayout {
    size_t control_off, keys0_off, vals0_off, keys1_off, vals1_off, lb_off, total;
    long long sort_tiles;
    size_t zeroed() const { return keys0_off; }
};

BvhLevels make_levels(long long n) {
    BvhLevels L;
    L.n_levels = 0;
    if (n <= 0) return L;
    long long start = 0, count = n;
    L.start[0] = 0;
    L.count[0] = n;
    L.n_levels = 1;
    while (count > 1) {                                    /* bvh.mojo:96-117 */
        start += count;
        count = (count + 1) / 2;
        L.start[L.n_levels] = start;
        L.count[L.n_levels] = count;
        ++L.n_levels;
    }
    return L;
}

long long node_count_of(long long n) {
    if (n <= 0) return 0;
    const BvhLevels L = make_levels(n);
    return L.start[L.n_levels - 1] + 1;
}

BvhLayout make_layout(long long n) {
    BvhLayout B;
    B.sort_tiles = (n + 256 * kBvhSortItems - 1) / (256 * kBvhSortItems);
    B.control_off = 0;
    B.keys0_off = align_up(sizeof(BvhControl), 256);
    B.vals0_off = align_up(B.keys0_off + (size_t)n * 4, 256);
    B.keys1_off = align_up(B.vals0_off + (size_t)n * 4, 256);
    B.vals1_off = align_up(B.keys1_off + (size_t)n * 4, 256);
    B.lb_off = align_up(B.vals1_off + (size_t)n * 4, 256);
    B.total = align_up(B.lb_off + (size_t)8 * (size_t)(B.sort_tiles > 0 ? B.sort_tiles : 1) * 256 * 4, 256);
    return B;
}

/* order-preserving key of a float (NaN excluded by the callers) */
__device__ __forceinline__ unsigned int ord_key(float f) {
    const unsigned int b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_value(unsigned int k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

__global__ void __launch_bounds__(256)
bbox_kernel(const float* __restrict__ means, long long n, BvhControl* ctrl) {
    __shared__ unsigned int s_lo[3][8], s_hi[3][8];
    unsigned int lo[3] = {0u, 0u, 0u}, hi[3] = {0u, 0u, 0u};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float p = means[i * 3 + c];
            if (p == p) {                                  /* gaussian_cloud.mojo:36-42 skip NaN */
                const unsigned int k = ord_key(p);
                lo[c] = max(lo[c], ~k);
                hi[c] = max(hi[c], k);
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        lo[c] = __reduce_max_sync(0xffffffffu, lo[c]);
        hi[c] = __reduce_max_sync(0xffffffffu, hi[c]);
        if (lane == 0) {
            s_lo[c][warp] = lo[c];
            s_hi[c][warp] = hi[c];
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int c = threadIdx.x;
        unsigned int a = 0u, b = 0u;
        for (int w = 0; w < 8; ++w) {
            a = max(a, s_lo[c][w]);
            b = max(b, s_hi[c][w]);
        }
        if (a) atomicMax(&ctrl->lo[c], a);
        if (b) atomicMax(&ctrl->hi[c], b);
    }
}

/* expand_bits_10_to_30, morton.mojo:7-18 */
__device__ __forceinline__ unsigned int expand_bits(unsigned int val) {
    unsigned int v = val & 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

/* compute_morton_3d, morton.mojo:21-46 (a NaN coordinate counts as 0) */
__device__ __forceinline__ unsigned int morton3(float nx, float ny, float nz) {
    float c[3] = {nx, ny, nz};
    unsigned int q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float v = c[k];
        if (v < 0.0f) v = 0.0f;
        else if (v > 1.0f) v = 1.0f;
        q[k] = v == v ? (unsigned int)(v * 1023.0f) : 0u;
    }
    return expand_bits(q[0]) | (expand_bits(q[1]) << 1) | (expand_bits(q[2]) << 2);
}

__global__ void __launch_bounds__(256)
morton_kernel(const float* __restrict__ means, long long n, const BvhControl* __restrict__ ctrl,
              unsigned int* __restrict__ keys, unsigned int* __restrict__ vals) {
    /* the box as add_gaussian leaves it: min from 1e9, max from -1e9 */
    float mn[3], inv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float lo = (float)1e9, hi = (float)-1e9;
        const unsigned int a = ctrl->lo[c], b = ctrl->hi[c];
        if (a) {
            const float v = ord_value(~a);
            if (v < lo) lo = v;
        }
        if (b) {
            const float v = ord_value(b);
            if (v > hi) hi = v;
        }
        const float extent = hi - lo;                                    /* bvh.mojo:52-58 */
        mn[c] = lo;
        inv[c] = 1.0f / (extent > (float)0.001 ? extent : 1.0f);
    }
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float nx = (means[i * 3 + 0] - mn[0]) * inv[0];                /* bvh.mojo:64-72 */
        const float ny = (means[i * 3 + 1] - mn[1]) * inv[1];
        const float nz = (means[i * 3 + 2] - mn[2]) * inv[2];
        keys[i] = morton3(nx, ny, nz);
        vals[i] = (unsigned int)i;
    }
}

struct Box {
    float mn[3], mx[3];
};

__device__ __forceinline__ Box load_box_cg(const LumenBvhNode* node, int* left, int* right) {
    const float4 a = __ldcg(reinterpret_cast<const float4*>(node));
    const float4 b = __ldcg(reinterpret_cast<const float4*>(node) + 1);
    if (left) *left = __float_as_int(a.w);
    if (right) *right = __float_as_int(b.w);
    return Box{{a.x, a.y, a.z}, {b.x, b.y, b.z}};
}

__device__ __forceinline__ void store_node(LumenBvhNode* node, const Box& b, int left, int right) {
    float4* p = reinterpret_cast<float4*>(node);
    __stcg(p, make_float4(b.mn[0], b.mn[1], b.mn[2], __int_as_float(left)));
    __stcg(p + 1, make_float4(b.mx[0], b.mx[1], b.mx[2], __int_as_float(right)));
}

/* AABB3f.expand_point, aabb.mojo:47-54 */
__device__ __forceinline__ void expand_point(Box& b, const float p[3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
        if (p[c] < b.mn[c]) b.mn[c] = p[c];
#pragma unroll
    for (int c = 0; c < 3; ++c)
        if (p[c] > b.mx[c]) b.mx[c] = p[c];
}

/* Levels of the hierarchy built per launch: a block takes 1024 consecutive
 * nodes of level L0 (for L0 = 0 it first writes them as leaves) and builds
 * their ancestors up to level L0 + 10 in shared memory, one level per
 * barrier; parents pair adjacent nodes exactly as bvh.mojo:96-117 does, so
 * a block's subtree never needs another block's nodes. */
constexpr int kRefitSpan = 10;
constexpr int kRefitNodes = 1 << kRefitSpan;
constexpr int kRefitThreads = 256;

__global__ void __launch_bounds__(kRefitThreads)
bvh_levels_kernel(const float* __restrict__ means, const float* __restrict__ scales, long long n,
                  const BvhControl* __restrict__ ctrl, const unsigned int* __restrict__ v0,
                  const unsigned int* __restrict__ v1, LumenBvhNode* __restrict__ nodes,
                  int* __restrict__ splat_index, BvhLevels lv, int L0) {
    __shared__ Box cur[kRefitNodes];
    __shared__ Box nxt[kRefitNodes / 2];
    const int tid = threadIdx.x;
    const long long b = blockIdx.x;
    const long long first = b * kRefitNodes;
    const long long cnt0 = lv.count[L0];
    const int m0 = (int)(cnt0 - first < kRefitNodes ? cnt0 - first : kRefitNodes);
    if (L0 == 0) {
        const unsigned int* perm = ctrl->sort.sorted_buffer ? v1 : v0;
        for (int k = tid; k < m0; k += kRefitThreads) {
            const long long i = first + k;
            const long long g = perm[i];
            /* leaf: position +- 3 x the largest scale (bvh.mojo:78-93) */
            float r = scales[g * 3 + 0];
            if (scales[g * 3 + 1] > r) r = scales[g * 3 + 1];
            if (scales[g * 3 + 2] > r) r = scales[g * 3 + 2];
            const float r3 = r * 3.0f;
            Box leaf;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float pc = means[g * 3 + c];
                leaf.mn[c] = pc - r3;
                leaf.mx[c] = pc + r3;
            }
            store_node(nodes + i, leaf, -1, -1);
            splat_index[i] = (int)g;
            cur[k] = leaf;
        }
    } else {
        for (int k = tid; k < m0; k += kRefitThreads)
            cur[k] = load_box_cg(nodes + lv.start[L0] + first + k, nullptr, nullptr);
    }
    __syncthreads();
    Box* src = cur;
    Box* dst = nxt;
    for (int sft = 1; sft <= kRefitSpan && L0 + sft < lv.n_levels; ++sft) {
        const int L = L0 + sft;
        const long long pfirst = first >> sft;                 /* this block's first parent at level L */
        const long long pend = ((first + kRefitNodes) >> sft) < lv.count[L] ? ((first + kRefitNodes) >> sft)
                                                                             : lv.count[L];
        const int np = (int)(pend - pfirst);
        for (int k = tid; k < np; k += kRefitThreads) {
            const long long pg = pfirst + k;
            const long long left = lv.start[L - 1] + 2 * pg;
            const bool has_right = 2 * pg + 1 < lv.count[L - 1];
            Box bx = src[2 * k];
            if (has_right) {
                expand_point(bx, src[2 * k + 1].mn);           /* AABB3f.expand_box, aabb.mojo:56-58 */
                expand_point(bx, src[2 * k + 1].mx);
            }
            store_node(nodes + lv.start[L] + pg, bx, (int)left, has_right ? (int)(left + 1) : -1);
            dst[k] = bx;
        }
        __syncthreads();
        /* ping-pong: the next level reads what this one wrote (an odd level
         * writes at most 512 parents, into the smaller buffer) */
        Box* t = src;
        src = dst;
        dst = t;
    }
}

struct RayState {
    float o[3], d[3], inv[3];
};

/* Vec3f.normalized, vector.mojo:106-110 */
__device__ __forceinline__ void normalize3(const float v[3], float out[3]) {
    const float l = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (l > (float)0.000001) {
        out[0] = v[0] / l;
        out[1] = v[1] / l;
        out[2] = v[2] / l;
    } else {
        out[0] = out[1] = out[2] = 0.0f;
    }
}

/* AABB3f.intersect_ray, aabb.mojo:60-98 (the reciprocals are the same on
 * every call, so they are taken once per ray) */
__device__ __forceinline__ bool intersect(const float4& a, const float4& b, const RayState& r, float t_min,
                                          float t_max) {
    const float t1x = (a.x - r.o[0]) * r.inv[0], t2x = (b.x - r.o[0]) * r.inv[0];
    const float t1y = (a.y - r.o[1]) * r.inv[1], t2y = (b.y - r.o[1]) * r.inv[1];
    const float t1z = (a.z - r.o[2]) * r.inv[2], t2z = (b.z - r.o[2]) * r.inv[2];
    const float tx_min = fminf(t1x, t2x), tx_max = fmaxf(t1x, t2x);
    const float ty_min = fminf(t1y, t2y), ty_max = fmaxf(t1y, t2y);
    const float tz_min = fminf(t1z, t2z), tz_max = fmaxf(t1z, t2z);
    const float t_enter = fmaxf(fmaxf(tx_min, ty_min), tz_min);
    const float t_exit = fminf(fminf(tx_max, ty_max), tz_max);
    return !(t_enter > t_exit || t_exit < t_min || t_enter > t_max);
}

struct CastArgs {
    const LumenBvhNode* nodes;
    const int* splat_index;   /* n_leaves entries */
    long long node_count, root, n_gauss, n_leaves;
    const float* means;
    const float* scales;
    float max_dist;
};

/* raycast_closest_splat, raycast.mojo:30-95 */
__device__ LumenRayHit cast_ray(const CastArgs& A, const float origin[3], const float dir[3]) {
    LumenRayHit best;
    best.hit = 0;
    best.splat_index = -1;
    best.point[0] = best.point[1] = best.point[2] = 0.0f;
    if (A.node_count == 0 || A.root < 0) {
        best.distance = (float)1e9;
        return best;
    }
    best.distance = A.max_dist;
    RayState r;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        r.o[c] = origin[c];
        r.d[c] = dir[c];
        r.inv[c] = 1.0f / (dir[c] != 0.0f ? dir[c] : (float)1e-6);
    }
    int stack[kRayStack];
    int sp = 0;
    stack[sp++] = (int)A.root;
    /* a built hierarchy visits each node at most once; the bound and the
     * index check keep a damaged one from looping or reading out of range */
    for (long long visits = 0; sp > 0 && visits <= A.node_count; ++visits) {
        const int idx = stack[--sp];
        if (idx < 0 || (long long)idx >= A.node_count) continue;
        const float4 a = __ldg(reinterpret_cast<const float4*>(A.nodes + idx));
        const float4 b = __ldg(reinterpret_cast<const float4*>(A.nodes + idx) + 1);
        if (!intersect(a, b, r, 0.0f, best.distance)) continue;
        const int left = __float_as_int(a.w), right = __float_as_int(b.w);
        if (left == -1 && right == -1) {
            /* leaves are nodes [0, n_leaves) of a built hierarchy; a damaged
             * one cannot make the read leave the array */
            const int s = (long long)idx < A.n_leaves ? A.splat_index[idx] : -1;
            if (s >= 0 && (long long)s < A.n_gauss) {
                const float cx = A.means[(long long)s * 3], cy = A.means[(long long)s * 3 + 1],
                            cz = A.means[(long long)s * 3 + 2];
                const float ocx = cx - r.o[0], ocy = cy - r.o[1], ocz = cz - r.o[2];
                const float t_proj = ocx * r.d[0] + ocy * r.d[1] + ocz * r.d[2];
                if (t_proj > 0.0f && t_proj < best.distance) {
                    const float px = r.o[0] + r.d[0] * t_proj, py = r.o[1] + r.d[1] * t_proj,
                                pz = r.o[2] + r.d[2] * t_proj;
                    const float dx = px - cx, dy = py - cy, dz = pz - cz;
                    const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
                    float rad = A.scales[(long long)s * 3];
                    if (A.scales[(long long)s * 3 + 1] > rad) rad = A.scales[(long long)s * 3 + 1];
                    if (A.scales[(long long)s * 3 + 2] > rad) rad = A.scales[(long long)s * 3 + 2];
                    if (dist <= rad * 3.0f) {
                        best.hit = 1;
                        best.splat_index = s;
                        best.distance = t_proj;
                        best.point[0] = px;
                        best.point[1] = py;
                        best.point[2] = pz;
                    }
                }
            }
        } else {
            /* at most levels + 1 entries: 32 below 2^30 leaves */
            if (left >= 0 && sp < kRayStack) stack[sp++] = left;
            if (right >= 0 && sp < kRayStack) stack[sp++] = right;
        }
    }
    return best;
}

__global__ void __launch_bounds__(128)
raycast_kernel(CastArgs A, const LumenRay* __restrict__ rays, long long n_rays, LumenRayHit* __restrict__ hits) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_rays; i += stride) {
        const LumenRay ray = rays[i];
        float d[3];
        normalize3(ray.direction, d);                          /* Ray3f.__init__, camera.mojo:16-18 */
        hits[i] = cast_ray(A, ray.origin, d);
    }
}

__global__ void __launch_bounds__(128)
pick_kernel(CastArgs A, LumenViewCamera cam, const float* __restrict__ pixels, long long n,
            LumenRay* __restrict__ rays, LumenRayHit* __restrict__ hits) {
    /* PinholeCamera keeps its rotation normalised (camera.mojo:37-40) */
    const Quat q = q_normalized({cam.rotation[0], cam.rotation[1], cam.rotation[2], cam.rotation[3]});
    const Quat qi = q_inverse(q);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        /* generate_ray, camera.mojo:85-90 */
        const float x_norm = (pixels[2 * i] - cam.cx) / cam.fx;
        const float y_norm = (pixels[2 * i + 1] - cam.cy) / cam.fy;
        const float v[3] = {x_norm, y_norm, 1.0f};
        float dc[3];
        normalize3(v, dc);
        const Quat rq = q_mul(q_mul(q, Quat{0.0f, dc[0], dc[1], dc[2]}), qi);    /* rotate_vec, quaternion.mojo:80-87 */
        const float dw[3] = {rq.x, rq.y, rq.z};
        float d[3];
        normalize3(dw, d);                                                         /* Ray3f */
        if (rays) {
            LumenRay out;
            out.origin[0] = cam.position[0];
            out.origin[1] = cam.position[1];
            out.origin[2] = cam.position[2];
            out.direction[0] = d[0];
            out.direction[1] = d[1];
            out.direction[2] = d[2];
            rays[i] = out;
        }
        hits[i] = cast_ray(A, cam.position, d);
    }
}

int ray_grid(long long n) {
    long long g = (n + 127) / 128;
    const long long cap = (long long)device_sm_count() * 16;
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

bool bvh_ok(const LumenGpuBvh* b, const LumenGpuGaussians* g) {
    if (!b || !g || b->leaf_count < 0 || b->leaf_count >= (1ll << 30) || b->leaf_count != g->count) return false;
    if (b->node_count != node_count_of(b->leaf_count)) return false;
    if (b->node_count > 0 && (!b->nodes || !b->splat_index || !g->means || !g->scales)) return false;
    if (((uintptr_t)b->nodes) & 15u) return false;
    return true;
}

}  // namespace
}  // namespace lumen

using namespace lumen;

extern "C" {

int64_t lumen_bvh_node_count(int64_t n) { return node_count_of(n); }

size_t lumen_gpu_bvh_scratch_bytes(int64_t n) { return n < 0 ? 0 : make_layout(n).total; }

LumenStatus lumen_gpu_bvh_build(const LumenGpuGaussians* g, LumenGpuBvh* bvh, void* scratch, size_t scratch_bytes,
                                void* stream) {
    if (!g || !bvh || g->count < 0 || g->count >= (1ll << 30)) return LUMEN_ERROR_INVALID_ARGUMENT;
    const long long n = g->count;
    if (n == 0) {
        bvh->leaf_count = 0;
        bvh->node_count = 0;
        bvh->root_index = -1;
        return LUMEN_SUCCESS;
    }
    if (!g->means || !g->scales || !bvh->nodes || !bvh->splat_index || !scratch) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (((uintptr_t)bvh->nodes | (uintptr_t)scratch) & 15u) return LUMEN_ERROR_INVALID_ARGUMENT;
    const BvhLayout B = make_layout(n);
    if (scratch_bytes < B.total) return LUMEN_ERROR_INVALID_ARGUMENT;
    const BvhLevels lv = make_levels(n);
    configure_once();
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* base = (unsigned char*)scratch;
    BvhControl* ctrl = (BvhControl*)(base + B.control_off);
    unsigned int* k0 = (unsigned int*)(base + B.keys0_off);
    unsigned int* v0 = (unsigned int*)(base + B.vals0_off);
    unsigned int* k1 = (unsigned int*)(base + B.keys1_off);
    unsigned int* v1 = (unsigned int*)(base + B.vals1_off);
    unsigned int* lb = (unsigned int*)(base + B.lb_off);
    cudaError_t e = cudaMemsetAsync(base, 0, B.zeroed(), s);
    if (e != cudaSuccess) return map_cuda(e);
    const int sms = device_sm_count();
    long long grid = (n + 255) / 256;
    if (grid > (long long)sms * 8) grid = (long long)sms * 8;
    bbox_kernel<<<(unsigned int)grid, 256, 0, s>>>(g->means, n, ctrl);
    morton_kernel<<<(unsigned int)grid, 256, 0, s>>>(g->means, n, ctrl, k0, v0);
    launch_key_stats32(k0, n, &ctrl->sort, sms, s);
    launch_sort32(k0, v0, k1, v1, n, &ctrl->sort, lb, B.sort_tiles, nullptr, nullptr, &ctrl->error_flags,
                  kBvhSortItems, 4, sms, s);
    for (int L0 = 0; L0 + 1 < lv.n_levels; L0 += kRefitSpan) {
        const long long blocks = (lv.count[L0] + kRefitNodes - 1) / kRefitNodes;
        bvh_levels_kernel<<<(unsigned int)blocks, kRefitThreads, 0, s>>>(g->means, g->scales, n, ctrl, v0, v1,
                                                                         bvh->nodes, bvh->splat_index, lv, L0);
    }
    if (lv.n_levels == 1)   /* a single leaf: the kernel writes it without climbing */
        bvh_levels_kernel<<<1, kRefitThreads, 0, s>>>(g->means, g->scales, n, ctrl, v0, v1, bvh->nodes,
                                                      bvh->splat_index, lv, 0);
    if ((e = cudaGetLastError()) != cudaSuccess) return map_cuda(e);
    unsigned int h_flags = 0;
    e = cudaMemcpyAsync(&h_flags, &ctrl->error_flags, sizeof(h_flags), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return map_cuda(e);
    bvh->leaf_count = n;
    bvh->node_count = node_count_of(n);
    bvh->root_index = bvh->node_count - 1;
    return status_from_flags(h_flags);
}

LumenStatus lumen_gpu_raycast(const LumenGpuBvh* bvh, const LumenGpuGaussians* g, const LumenRay* rays,
                              int64_t n_rays, float max_dist, LumenRayHit* hits, void* stream) {
    if (!bvh_ok(bvh, g) || n_rays < 0) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (n_rays == 0) return LUMEN_SUCCESS;
    if (!rays || !hits) return LUMEN_ERROR_INVALID_ARGUMENT;
    const CastArgs A{bvh->nodes, bvh->splat_index, bvh->node_count, bvh->root_index, g->count, bvh->leaf_count,
                     g->means, g->scales, max_dist};
    raycast_kernel<<<ray_grid(n_rays), 128, 0, (cudaStream_t)stream>>>(A, rays, n_rays, hits);
    return map_cuda(cudaGetLastError());
}

LumenStatus lumen_gpu_pick_pixels(const LumenGpuBvh* bvh, const LumenGpuGaussians* g, const LumenViewCamera* cam,
                                  const float* pixels_xy, int64_t n, float max_dist, LumenRay* rays,
                                  LumenRayHit* hits, void* stream) {
    if (!bvh_ok(bvh, g) || !cam || n < 0) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (n == 0) return LUMEN_SUCCESS;
    if (!pixels_xy || !hits) return LUMEN_ERROR_INVALID_ARGUMENT;
    const CastArgs A{bvh->nodes, bvh->splat_index, bvh->node_count, bvh->root_index, g->count, bvh->leaf_count,
                     g->means, g->scales, max_dist};
    pick_kernel<<<ray_grid(n), 128, 0, (cudaStream_t)stream>>>(A, *cam, pixels_xy, n, rays, hits);
    return map_cuda(cudaGetLastError());
}

}  // extern "C"
