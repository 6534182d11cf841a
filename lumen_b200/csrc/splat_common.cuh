/*
 * splat_common.cuh - device structures and per-splat math shared by the
 * forward kernels.
 *
 * Everything here is compiled with --fmad=false and without fast-math, so
 * each float operation rounds exactly as written; the operation order follows
 * the reference Mojo code line by line (cited per function), which is what
 * makes the projected records, radii and keys bit-identical to the CPU
 * restatement the tests compare against.
 *
 * Literal constants are written (float)(double literal) because the
 * reference materialises its FloatLiterals as Float32 from 64-bit values.
 */
#pragma once

#include <stdint.h>
#include <map>
#include <tuple>
#include <cuda_runtime.h>

#include "../../include/lumen_gpu.h"
#include "lumen_expf.h"

namespace lumen {

constexpr int kTile = 16;
constexpr int kTilePixels = 256;

/* State of one stable radix sort of (key, value) pairs. The producer of the
 * keys fills n and the OR / OR-of-complement of all keys; a digit (byte)
 * varies iff some key has a 1 and some key a 0 in it, and only varying
 * digits get a pass. */
struct SortControl {
    unsigned long long n;                /* pairs to sort */
    unsigned long long key_or;
    unsigned long long key_or_not;
    unsigned int varying;                /* bit d: byte d varies */
    unsigned int sorted_buffer;          /* 0 or 1: where the sorted pairs end */
    unsigned int pass_ticket[8];         /* tile order of each digit pass */
    unsigned int hist[8][256];           /* histograms of the varying digits */
};

/* Control block at the start of a frame's scratch. Zeroed by the host
 * before every frame (one cudaMemsetAsync), then owned by the kernels. */
struct Control {
    unsigned long long n_instances;      /* K, even if above capacity */
    unsigned int n_visible;              /* V */
    unsigned int proj_ticket;            /* block order of the project look-back */
    unsigned int emit_ticket;            /* block order of the emit look-back */
    unsigned int error_flags;            /* LUMEN_GPU_ERR_* */
    unsigned int touched_tiles;
    unsigned int composite_ticket;       /* tile order of the compositor */
    unsigned int count_ticket;           /* unit order of the batch visibility count */
    unsigned int offsets_ticket;         /* tile order of the batch offset scan */
    unsigned int ranges_by_sort;         /* 1: the tile sort's last digit pass wrote the tile ranges */
    unsigned int pad[5];
    SortControl depth_sort;              /* visible splats by depth key */
    SortControl tile_sort;               /* instances by tile id */
};

constexpr int kProjThreads = 128;   /* Gaussians per projection block (a view's slots are a multiple) */
constexpr int kEmitThreads = 256;   /* splats per emission block */
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;   /* 4096 keys per tile */
constexpr int kSortTileMin = kSortThreads * 8;         /* the smallest tile a digit pass may use */
constexpr int kSort64Items = 16;                       /* keys per thread of the 64-bit pair sort */
constexpr int kSort64Tile = kSortThreads * kSort64Items;

/* Launch parameters an autotuner may choose; none of them changes a result. */
struct LaunchConfig {
    int composite_chunk;   /* instances staged per compositing round: 128, 256 or 512 */
    int depth_sort_items;  /* keys per thread in a depth-sort digit pass: 8 or 16 */
    int tile_sort_items;   /* keys per thread in a tile-sort digit pass: 8, 16 or 24 */
    int track;             /* 1: some view's image asks for contributor counts or last-visited
                              offsets (the compositor then keeps them); set by the host */
};
/* measured on B200 at 1080p with 1 M Gaussians: 512-instance compositor
 * chunks (0.233 against 0.238 ms for 256, 0.259 for 128); 4096-key tiles
 * for both sorts (sort stage 0.1955 ms, against 0.1978 with 2048-key depth
 * tiles, 0.2002 with 6144-key and 0.2232 with 2048-key tile-sort tiles) */
constexpr LaunchConfig kDefaultLaunch = {512, 16, 16, 1};

__host__ __device__ constexpr inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Quat { float w, x, y, z; };

/* Per-view constants, computed on the device in the same order as
 * PinholeCamera (src/scene/camera.mojo:24-79). */
struct DevCamera {
    float px, py, pz;
    Quat qi;      /* rotation.inverse()            (world_to_cam)       */
    Quat qii;     /* rotation.inverse().inverse()  (inside rotate_vec)  */
    float W[9];   /* rotation.inverse().to_rotation_matrix()            */
    float fx, fy, cx, cy, near_plane, far_plane;
    int width, height, tiles_x, tiles_y;
};

/* One view of a batch as the kernels read it. A batch is a list of views,
 * each with its own scene, camera and output image; a single-view frame is a
 * batch of one. Projection treats the batch as consecutive 128-Gaussian
 * blocks (block_begin: the view's first block; its Gaussian i has slot
 * block_begin * 128 + i), and tiles get batch-wide ids (tile_begin: the
 * global id of the view's tile 0), so one sort orders every view at once:
 * the tile-id key carries the view in its high part. */
struct ViewDesc {
    LumenGpuGaussians g;
    LumenViewCamera cam;
    int tiles_x;
    LumenGpuImage img;
    long long block_begin;
    long long tile_begin;
    long long inst_begin;     /* first tile-sorted instance of the view, or -1
                                 (written on the device by the range pass) */
    long long unit_begin;     /* batch projection: the first unit of the view's scene group
                                 when the view leads the group (units of the views before it
                                 otherwise, so the view owns none) */
    int group_next;           /* the next view of the same scene, or -1 */
    int group_lead;           /* 1: the first view of its scene in the batch */
    DevCamera dcam;           /* derived from cam on the device before projection */
};

struct BatchHeader {
    int n_views;
    int reserved0;
    long long total_blocks;   /* projection blocks of all views */
    long long total_tiles;    /* tiles of all views */
    long long total_units;    /* batch projection: blocks of the batch's distinct scenes */
};

/* Header and views, in scratch; written before the frame's kernels run. */
struct ViewTable {
    BatchHeader hdr;
    ViewDesc view[1];
};

__host__ __device__ constexpr inline size_t view_table_bytes(int max_views) {
    return sizeof(BatchHeader) + (size_t)(max_views > 0 ? max_views : 1) * sizeof(ViewDesc);
}

/* Scratch layout: [Control][project look-back: u64 per block][emit
 * look-back: u64 per block][view table][depth-sort look-back: 4 passes x
 * 2048-key tiles x 256 x u32][tile-sort look-back: 8 passes x 4096-key tiles
 * x 256 x u32, which is also 4 passes x 2048-key tiles (8 passes for the
 * standalone 64-bit pair sort)]. n counts projection slots (the Gaussians
 * of all views, each view rounded up to a multiple of kProjThreads). The
 * emit look-back uses at most as many entries as the project look-back. */
struct ScratchLayout {
    size_t control_off, proj_lb_off, emit_lb_off, table_off, depth_lb_off, tile_lb_off, total;
    int64_t proj_blocks, depth_tiles, sort_tiles;
    __host__ __device__ static ScratchLayout make(int64_t n, int64_t capacity, int max_views = 1) {
        ScratchLayout L;
        L.proj_blocks = (n + kProjThreads - 1) / kProjThreads;
        L.depth_tiles = (n + kSortTileMin - 1) / kSortTileMin;
        L.sort_tiles = (capacity + kSortTile - 1) / kSortTile;
        L.control_off = 0;
        L.proj_lb_off = align_up(sizeof(Control), 256);
        L.emit_lb_off = align_up(L.proj_lb_off + (size_t)L.proj_blocks * sizeof(unsigned long long), 256);
        L.table_off = align_up(L.emit_lb_off + (size_t)L.proj_blocks * sizeof(unsigned long long), 256);
        L.depth_lb_off = align_up(L.table_off + view_table_bytes(max_views), 256);
        L.tile_lb_off = align_up(L.depth_lb_off + (size_t)4 * (size_t)L.depth_tiles * 256 * sizeof(unsigned int), 256);
        L.total = align_up(L.tile_lb_off + (size_t)8 * (size_t)L.sort_tiles * 256 * sizeof(unsigned int), 256);
        return L;
    }
    /* bytes zeroed before a frame: control and both scans */
    size_t zeroed_prefix() const { return table_off; }
};

/* Groups a batch's views by scene (identical LumenGpuGaussians) for the
 * Gaussian-major batch projection: each view's group_next and group_lead,
 * and the unit numbering (one unit per 128-Gaussian block of each distinct
 * scene, in order of the scenes' first views). Returns the unit count. */
inline long long assign_scene_groups(ViewDesc* v, int n) {
    using Key = std::tuple<const void*, const void*, const void*, const void*, const void*, long long>;
    std::map<Key, int> last;   /* the latest view of each scene so far */
    long long units = 0;
    for (int i = 0; i < n; ++i) {
        const LumenGpuGaussians& g = v[i].g;
        const Key key{g.means, g.scales, g.quats, g.opacities, g.sh, (long long)g.count};
        v[i].group_next = -1;
        auto it = last.find(key);
        v[i].group_lead = it == last.end() ? 1 : 0;
        if (it != last.end()) {
            v[it->second].group_next = i;
            it->second = i;
        } else {
            last.emplace(key, i);
        }
        v[i].unit_begin = units;
        if (v[i].group_lead) units += (g.count + kProjThreads - 1) / kProjThreads;
    }
    return units;
}

/* Tile rectangle of a visible splat and its view: 12 bits per bound (tile
 * coordinates below 4096, images up to 65520 pixels a side), view in the
 * top 16 bits. */
constexpr int kMaxTilesPerAxis = 4095;
constexpr int kMaxViews = 65535;

__host__ __device__ inline unsigned long long pack_rect(int min_tx, int min_ty, int max_tx, int max_ty, int view) {
    return (unsigned long long)(min_tx & 0xFFF) | ((unsigned long long)(min_ty & 0xFFF) << 12) |
           ((unsigned long long)(max_tx & 0xFFF) << 24) | ((unsigned long long)(max_ty & 0xFFF) << 36) |
           ((unsigned long long)(view & 0xFFFF) << 48);
}
__host__ __device__ inline int rect_min_tx(unsigned long long r) { return (int)(r & 0xFFF); }
__host__ __device__ inline int rect_min_ty(unsigned long long r) { return (int)((r >> 12) & 0xFFF); }
__host__ __device__ inline int rect_max_tx(unsigned long long r) { return (int)((r >> 24) & 0xFFF); }
__host__ __device__ inline int rect_max_ty(unsigned long long r) { return (int)((r >> 36) & 0xFFF); }
__host__ __device__ inline int rect_view(unsigned long long r) { return (int)(r >> 48); }

/* The view whose [begin, next begin) holds x: the last view with begin <= x
 * (views with no blocks or tiles are skipped over). */
__device__ __forceinline__ int find_view_by_block(const ViewTable* vt, int n_views, long long blk) {
    int lo = 0, hi = n_views - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (vt->view[mid].block_begin <= blk) lo = mid; else hi = mid - 1;
    }
    return lo;
}
/* The scene group that owns batch projection unit u: the last view with
 * unit_begin <= u (non-leading views own no units). */
__device__ __forceinline__ int find_view_by_unit(const ViewTable* vt, int n_views, long long u) {
    int lo = 0, hi = n_views - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (vt->view[mid].unit_begin <= u) lo = mid; else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int find_view_by_tile(const ViewTable* vt, int n_views, long long tile) {
    int lo = 0, hi = n_views - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (vt->view[mid].tile_begin <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

/* Bounded spin: after this many polls a wait gives up, sets
 * LUMEN_GPU_ERR_SPIN_TIMEOUT and continues with a zero contribution. */
constexpr int kSpinLimit = 1 << 22;

/* Look-back descriptor flags (top bits). */
constexpr unsigned long long kDescAgg64 = 1ull << 62;
constexpr unsigned long long kDescIncl64 = 2ull << 62;
constexpr unsigned long long kDescMask64 = (1ull << 62) - 1;
constexpr unsigned int kDescAgg32 = 1u << 30;
constexpr unsigned int kDescIncl32 = 2u << 30;
constexpr unsigned int kDescMask32 = (1u << 30) - 1;

/* ---------------------------------------------------------------- math -- */


/* Quatf.normalized, src/math/quaternion.mojo:46-57 */
__device__ __forceinline__ Quat q_normalized(Quat q) {
    float ns = q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z;
    float n = sqrtf(ns);
    if (n > (float)0.000001) {
        float inv_n = 1.0f / n;
        return {q.w * inv_n, q.x * inv_n, q.y * inv_n, q.z * inv_n};
    }
    return {1.0f, 0.0f, 0.0f, 0.0f};
}

/* Quatf.inverse, quaternion.mojo:62-67 */
__device__ __forceinline__ Quat q_inverse(Quat q) {
    float ns = q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z;
    if (ns > (float)0.000001) {
        float inv_ns = 1.0f / ns;
        return {q.w * inv_ns, -q.x * inv_ns, -q.y * inv_ns, -q.z * inv_ns};
    }
    return {1.0f, 0.0f, 0.0f, 0.0f};
}

/* Quatf.mul (Hamilton product), quaternion.mojo:69-78 */
__device__ __forceinline__ Quat q_mul(Quat a, Quat b) {
    return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
            a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}

/* Quatf.to_rotation_matrix (normalises first), quaternion.mojo:89-117 */
__device__ __forceinline__ void q_to_matrix(Quat q0, float m[9]) {
    Quat q = q_normalized(q0);
    float x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
    float xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
    float yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
    float wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
    m[0] = 1.0f - (yy + zz); m[1] = xy - wz;          m[2] = xz + wy;
    m[3] = xy + wz;          m[4] = 1.0f - (xx + zz); m[5] = yz - wx;
    m[6] = xz - wy;          m[7] = yz + wx;          m[8] = 1.0f - (xx + yy);
}

__device__ __forceinline__ void setup_camera(const LumenViewCamera& c, DevCamera& d) {
    Quat r = q_normalized({c.rotation[0], c.rotation[1], c.rotation[2], c.rotation[3]});  /* camera.mojo:229 */
    d.px = c.position[0]; d.py = c.position[1]; d.pz = c.position[2];
    d.qi = q_inverse(r);
    d.qii = q_inverse(d.qi);
    q_to_matrix(d.qi, d.W);
    d.fx = c.fx; d.fy = c.fy; d.cx = c.cx; d.cy = c.cy;
    d.near_plane = c.near_plane; d.far_plane = c.far_plane;
    d.width = c.width; d.height = c.height;
    d.tiles_x = (c.width + kTile - 1) / kTile;
    d.tiles_y = (c.height + kTile - 1) / kTile;
}

/* Mojo Int(x) on a Float32: truncation toward zero; NaN and |x| >= 2^63 give
 * INT64_MIN (the reference's x86-64 conversion result). */
__device__ __forceinline__ long long mojo_int(float x) {
    if (!(x > -9.2233720368547758e18f && x < 9.2233720368547758e18f)) return (long long)(-9223372036854775807ll - 1);
    return (long long)x;
}

/* MIN_ALPHA_THRESHOLD, src/core/types.mojo:34 */
__device__ __forceinline__ float min_alpha() { return (float)0.00392156862; }

/* Result of one Gaussian through pipeline.mojo:84-149. */
struct Projected {
    float cx, cy, z, op;
    float ic00, ic01, ic11;
    float r, g, b;
    int radius;              /* 0 when culled */
    int min_tx, min_ty, max_tx, max_ty;
    bool visible;
};

/* A Gaussian's SH row staged in shared memory as 12 16-byte chunks: chunk
 * q of row t sits at 12 t + (q ^ sh_swizzle(t)). Rows are 48 words apart,
 * so without the swizzle the 8 lanes of each phase of a 16-byte load hit
 * only 2 of the 8 chunk slots of the 32 banks (a 4-way conflict); the XOR
 * spreads them over all 8, and it keeps every chunk in its row. */
__device__ __forceinline__ int sh_swizzle(int t) { return (t >> 1) & 3; }

/* SHBasis.evaluate + evaluate_sh_color, spherical_harmonics.mojo:68-111,133-172;
 * sh points at the Gaussian's 48 coefficients (16-byte aligned; the
 * projection kernels stage them in shared memory, chunk q at q ^ swz). */
__device__ __forceinline__ void sh_color(const float* __restrict__ sh, float dx0, float dy0, float dz0,
                                         int degree, float& r, float& g, float& b, int swz = 0) {
    const float C0 = (float)0.28209479177387814, C1 = (float)0.4886025119029199;
    const float C2_0 = (float)1.0925484305920792, C2_1 = (float)0.31539156525252005;
    const float C2_2 = (float)0.5462742152960396, C3_0 = (float)0.5900435899266435;
    const float C3_1 = (float)2.890611442640554, C3_2 = (float)0.4570457994644658;
    const float C3_3 = (float)0.3731763325901154, C3_4 = (float)1.445305721320277;
    /* second normalisation inside SHBasis.evaluate (vector.mojo:106-110) */
    float l = sqrtf(dx0 * dx0 + dy0 * dy0 + dz0 * dz0);
    float x = 0.0f, y = 0.0f, z = 0.0f;
    if (l > (float)0.000001) { x = dx0 / l; y = dy0 / l; z = dz0 / l; }
    float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    float Y[16];
    Y[0] = C0;
    Y[1] = -C1 * y;
    Y[2] = C1 * z;
    Y[3] = -C1 * x;
    Y[4] = C2_0 * xy;
    Y[5] = -C2_0 * yz;
    Y[6] = C2_1 * (2.0f * zz - xx - yy);
    Y[7] = -C2_0 * xz;
    Y[8] = C2_2 * (xx - yy);
    Y[9] = -C3_0 * y * (3.0f * xx - yy);
    Y[10] = C3_1 * xy * z;
    Y[11] = -C3_2 * y * (4.0f * zz - xx - yy);
    Y[12] = C3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    Y[13] = -C3_2 * x * (4.0f * zz - xx - yy);
    Y[14] = C3_4 * z * (xx - yy);
    Y[15] = -C3_0 * x * (xx - 3.0f * yy);
    int n = 16;
    if (degree == 0) n = 1;
    else if (degree == 1) n = 4;
    else if (degree == 2) n = 9;
    const float4* s4 = reinterpret_cast<const float4*>(sh);
    float c[48];
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        float4 v = s4[k ^ swz];
        c[4 * k + 0] = v.x; c[4 * k + 1] = v.y; c[4 * k + 2] = v.z; c[4 * k + 3] = v.w;
    }
    float rr = 0.5f, gg = 0.5f, bb = 0.5f;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        if (i < n) {
            rr += c[i * 3 + 0] * Y[i];
            gg += c[i * 3 + 1] * Y[i];
            bb += c[i * 3 + 2] * Y[i];
        }
    }
    if (rr < 0.0f) rr = 0.0f; else if (rr > 1.0f) rr = 1.0f;
    if (gg < 0.0f) gg = 0.0f; else if (gg > 1.0f) gg = 1.0f;
    if (bb < 0.0f) bb = 0.0f; else if (bb > 1.0f) bb = 1.0f;
    r = rr; g = gg; b = bb;
}

/* The view-independent part of a Gaussian's projection: activations, the
 * normalised rotation, the opacity cull and Sigma = M M^T with M = R(q) S
 * (gaussian.mojo:36-44, culling.mojo:47-51, covariance.mojo:41-83). */
struct Prepared {
    float op;
    float s00, s01, s02, s11, s12, s22;
    bool ok;                 /* passed the opacity cull */
};

__device__ __forceinline__ Prepared prepare_gaussian(float sx, float sy, float sz, Quat qraw, float op,
                                                     const LumenRenderOptions& o) {
    Prepared pr;
    if (o.params_are_logits) {
        sx = lumen_expf(sx); sy = lumen_expf(sy); sz = lumen_expf(sz);
        op = 1.0f / (1.0f + lumen_expf(-op));                 /* gaussian.mojo:43-44 */
    }
    Quat rot = q_normalized(qraw);                            /* gaussian.mojo:36 */
    pr.op = op;
    pr.ok = op >= min_alpha();                                /* culling.mojo:47-51 */
    /* Covariance3D.from_scale_and_rotation, covariance.mojo:41-83 */
    if (sx < (float)0.00001) sx = (float)0.00001;
    if (sy < (float)0.00001) sy = (float)0.00001;
    if (sz < (float)0.00001) sz = (float)0.00001;
    float R[9];
    q_to_matrix(rot, R);
    float m00 = R[0] * sx, m01 = R[1] * sy, m02 = R[2] * sz;
    float m10 = R[3] * sx, m11 = R[4] * sy, m12 = R[5] * sz;
    float m20 = R[6] * sx, m21 = R[7] * sy, m22 = R[8] * sz;
    pr.s00 = m00 * m00 + m01 * m01 + m02 * m02;
    pr.s01 = m00 * m10 + m01 * m11 + m02 * m12;
    pr.s02 = m00 * m20 + m01 * m21 + m02 * m22;
    pr.s11 = m10 * m10 + m11 * m11 + m12 * m12;
    pr.s12 = m10 * m20 + m11 * m21 + m12 * m22;
    pr.s22 = m20 * m20 + m21 * m21 + m22 * m22;
    return pr;
}

/* The per-view part: camera transform and cull, screen position, EWA,
 * radius, tile rectangle, colour (kFull; without it only the visibility,
 * radius and rectangle are formed, with the same arithmetic). Follows
 * pipeline.mojo:85-149 and the functions it calls. */
template <bool kFull = true>
__device__ __forceinline__ Projected project_prepared(const DevCamera& cam, float mx, float my, float mz,
                                                      const Prepared& pr, const float* __restrict__ sh,
                                                      const LumenRenderOptions& o, int sh_swz = 0) {
    Projected p;
    p.visible = false;
    p.radius = 0;
    if (!pr.ok) return p;
    /* world_to_cam, camera.mojo:69-71, quaternion.mojo:80-87 */
    float rx = mx - cam.px, ry = my - cam.py, rz = mz - cam.pz;
    Quat t = q_mul(cam.qi, Quat{0.0f, rx, ry, rz});
    Quat pc = q_mul(t, cam.qii);
    float tx = pc.x, ty = pc.y, tz = pc.z;
    if (!(tz >= cam.near_plane && tz <= cam.far_plane)) return p;   /* culling.mojo:41-45 */
    /* cam_to_screen, camera.mojo:73-79 */
    float tzs = tz;
    if (tzs < (float)0.0001 && tzs > (float)-0.0001) tzs = (float)0.0001;
    float u = cam.fx * (tx / tzs) + cam.cx;
    float v = cam.fy * (ty / tzs) + cam.cy;
    /* ProjectiveJacobian.compute, projection.mojo:80-96 */
    float jz = tz;
    if (jz < (float)0.0001) jz = (float)0.0001;
    float inv_tz = 1.0f / jz;
    float inv_tz2 = inv_tz * inv_tz;
    float j00 = cam.fx * inv_tz, j02 = -cam.fx * tx * inv_tz2;
    float j11 = cam.fy * inv_tz, j12 = -cam.fy * ty * inv_tz2;
    /* compute_ewa_covariance, projection.mojo:99-148 */
    const float* W = cam.W;
    float t00 = j00 * W[0] + j02 * W[6];
    float t01 = j00 * W[1] + j02 * W[7];
    float t02 = j00 * W[2] + j02 * W[8];
    float t10 = j11 * W[3] + j12 * W[6];
    float t11 = j11 * W[4] + j12 * W[7];
    float t12 = j11 * W[5] + j12 * W[8];
    float q00 = t00 * pr.s00 + t01 * pr.s01 + t02 * pr.s02;
    float q01 = t00 * pr.s01 + t01 * pr.s11 + t02 * pr.s12;
    float q02 = t00 * pr.s02 + t01 * pr.s12 + t02 * pr.s22;
    float q10 = t10 * pr.s00 + t11 * pr.s01 + t12 * pr.s02;
    float q11 = t10 * pr.s01 + t11 * pr.s11 + t12 * pr.s12;
    float q12 = t10 * pr.s02 + t11 * pr.s12 + t12 * pr.s22;
    float c00 = q00 * t00 + q01 * t01 + q02 * t02 + o.lowpass;
    float c01 = q00 * t10 + q01 * t11 + q02 * t12;
    float c11 = q10 * t10 + q11 * t11 + q12 * t12 + o.lowpass;
    /* solve_eigenvalues_2x2, cholesky.mojo:28-51 */
    float mid = (c00 + c11) * 0.5f;
    float diff = (c00 - c11) * 0.5f;
    float disc = diff * diff + c01 * c01;
    float root = sqrtf(disc);
    float l_max = mid + root;
    float r_float = 3.0f * sqrtf(l_max);
    long long radius = mojo_int(ceilf(r_float));
    if (radius < 1) return p;                                 /* pipeline.mojo:108 */
    /* is_screen_box_visible, culling.mojo:53-71 */
    float r_f = (float)radius;
    if (u + r_f < 0.0f || u - r_f >= (float)cam.width || v + r_f < 0.0f || v - r_f >= (float)cam.height)
        return p;
    /* get_gaussian_tile_overlap, tile.mojo:62-97 */
    long long min_px = mojo_int(u - r_f), max_px = mojo_int(u + r_f);
    long long min_py = mojo_int(v - r_f), max_py = mojo_int(v + r_f);
    if (max_px < 0 || min_px >= cam.width || max_py < 0 || min_py >= cam.height) return p;
    if (min_px < 0) min_px = 0;
    if (max_px >= cam.width) max_px = cam.width - 1;
    if (min_py < 0) min_py = 0;
    if (max_py >= cam.height) max_py = cam.height - 1;
    p.min_tx = (int)(min_px / kTile); p.max_tx = (int)(max_px / kTile);
    p.min_ty = (int)(min_py / kTile); p.max_ty = (int)(max_py / kTile);
    p.radius = radius > 0x7FFFFFFFll ? 0x7FFFFFFF : (int)radius;
    p.visible = true;
    if (!kFull) return p;
    /* view direction (vector.mojo:106-110) and colour, pipeline.mojo:133-139 */
    float vx = mx - cam.px, vy = my - cam.py, vz = mz - cam.pz;
    float vl = sqrtf(vx * vx + vy * vy + vz * vz);
    float dx = 0.0f, dy = 0.0f, dz = 0.0f;
    if (vl > (float)0.000001) { dx = vx / vl; dy = vy / vl; dz = vz / vl; }
    sh_color(sh, dx, dy, dz, o.sh_degree, p.r, p.g, p.b, sh_swz);
    /* Covariance2D.inverse, projection.mojo:30-42 */
    float det = c00 * c11 - c01 * c01;
    if (det > (float)-0.0000001 && det < (float)0.0000001) {
        p.ic00 = 0.0f; p.ic01 = 0.0f; p.ic11 = 0.0f;
    } else {
        float inv_det = 1.0f / det;
        p.ic00 = c11 * inv_det;
        p.ic01 = -c01 * inv_det;
        p.ic11 = c00 * inv_det;
    }
    p.cx = u; p.cy = v; p.z = tz; p.op = pr.op;
    return p;
}

/* One Gaussian: cull, camera transform, EWA, radius, tile rectangle, colour.
 * Follows pipeline.mojo:85-149 and the functions it calls. */
__device__ __forceinline__ Projected project_gaussian(const DevCamera& cam, float mx, float my, float mz,
                                                      float sx, float sy, float sz, Quat qraw, float op,
                                                      const float* __restrict__ sh, const LumenRenderOptions& o,
                                                      int sh_swz = 0) {
    return project_prepared<true>(cam, mx, my, mz, prepare_gaussian(sx, sy, sz, qraw, op, o), sh, o, sh_swz);
}

/* float_to_ordered_uint32 (radix_sort.mojo:8-18) or the raw float bits. */
__device__ __forceinline__ unsigned int depth_key(float z, int key_mode) {
    if (key_mode == 1) return __float_as_uint(z);
    long long s = mojo_int(z * 1000.0f);
    if (s < 0) s = 0;
    else if (s > 0x7FFFFFFFll) s = 0x7FFFFFFFll;
    return (unsigned int)s;
}

/* ------------------------------------------------------------- helpers -- */

/* 16-byte asynchronous copy global -> shared (bypassing L1), and its waits. */
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned int dst = (unsigned int)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ unsigned int lanemask_lt() {
    unsigned int m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ unsigned int ld_volatile_u32(const unsigned int* p) {
    return *reinterpret_cast<const volatile unsigned int*>(p);
}
__device__ __forceinline__ void st_volatile_u64(unsigned long long* p, unsigned long long v) {
    *reinterpret_cast<volatile unsigned long long*>(p) = v;
}
__device__ __forceinline__ void st_volatile_u32(unsigned int* p, unsigned int v) {
    *reinterpret_cast<volatile unsigned int*>(p) = v;
}

/* Warp-parallel decoupled look-back over 64-bit descriptors: the sum of all
 * blocks before `blk`. Called by one full warp. */
__device__ __forceinline__ unsigned long long lookback64(const unsigned long long* desc, int blk, unsigned int* err) {
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

/* Block-wide exclusive scan of one value per thread (kThreads threads). */
template <int kThreads>
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
    for (int w = 0; w < kThreads / 32; ++w) {
        const unsigned int t = warp_tot[w];
        if (w < warp) before += t;
        all += t;
    }
    *total = all;
    return before + incl - x;
}

/* Programmatic dependent launch (sm_90 and later): the frame's kernels are
 * launched with launch_chained, so the hardware may schedule a kernel's
 * blocks while its predecessor's last blocks still run. chain_begin(), the
 * first statement of every kernel launched that way, waits until the
 * predecessor has completed and its writes are visible, then allows the
 * next kernel to be scheduled in turn: nothing is read or written before
 * the wait, so the stream order of the results is unchanged; only the
 * launch latency and the predecessor's tail are hidden. */
__device__ __forceinline__ void chain_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

/* Whether launch_chained sets the dependent-launch attribute on this host
 * thread (ChainedLaunches turns it off for a scope). The render server,
 * which keeps several batches in flight on separate streams, launches
 * without it: a chained kernel's blocks wait resident on their SMs, which
 * would hold back the other stream's batch. */
inline thread_local bool g_chained_launches = true;

struct ChainedLaunches {
    bool saved;
    explicit ChainedLaunches(bool on) : saved(g_chained_launches) { g_chained_launches = on; }
    ~ChainedLaunches() { g_chained_launches = saved; }
};

template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                  Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = g_chained_launches ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

/* Host hook called after each row band of a banded frame has been
 * enqueued (pixel rows [row_begin, row_end)). */
using BandHook = void (*)(void* ctx, int row_begin, int row_end, cudaStream_t s);

}  // namespace lumen
