/*
 * spatial_oracle.cpp - CPU restatement of the reference's picking path
 * (TEST INFRASTRUCTURE ONLY: the checker for lumen_b200/csrc/spatial.cu).
 *
 *   oracle_expand_bits     expand_bits_10_to_30, src/spatial/morton.mojo:7-18
 *   oracle_morton3d        compute_morton_3d, morton.mojo:21-46
 *   oracle_bvh_build       LBVH.build_from_cloud, src/spatial/bvh.mojo:45-120, over
 *                          a cloud whose box add_gaussian tracked
 *                          (src/scene/gaussian_cloud.mojo:21-42); the sort is the
 *                          oracle's radix_sort_64bit restatement; boxes grow with
 *                          AABB3f.expand_point / expand_box (src/spatial/aabb.mojo:47-58)
 *   oracle_raycast         raycast_closest_splat, src/spatial/raycast.mojo:30-95, with
 *                          AABB3f.intersect_ray (aabb.mojo:60-98) and Ray3f
 *                          (src/scene/camera.mojo:12-21)
 *   oracle_generate_ray    PinholeCamera.generate_ray, camera.mojo:85-90
 *
 * Float32 arithmetic in the reference's operation order, no contraction
 * (-ffp-contract=off). Nodes use the 32-byte layout of LumenBvhNode:
 * min xyz, left child, max xyz, right child. Two choices where the reference
 * leaves the result to its platform: a NaN normalised coordinate gets Morton
 * digit 0, and the slab test's min/max ignore a NaN operand (fminf/fmaxf).
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "lumen_oracle.h"

namespace {

struct Node {
    float mn[3];
    int32_t left;
    float mx[3];
    int32_t right;
};
static_assert(sizeof(Node) == 32, "node layout");

void normalize3(const float v[3], float out[3]) {          /* vector.mojo:100-110 */
    const float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (l > (float)0.000001) {
        out[0] = v[0] / l;
        out[1] = v[1] / l;
        out[2] = v[2] / l;
    } else {
        out[0] = out[1] = out[2] = 0.0f;
    }
}

void expand_point(Node& b, const float p[3]) {             /* aabb.mojo:47-54 */
    for (int c = 0; c < 3; ++c)
        if (p[c] < b.mn[c]) b.mn[c] = p[c];
    for (int c = 0; c < 3; ++c)
        if (p[c] > b.mx[c]) b.mx[c] = p[c];
}

bool intersect_ray(const Node& b, const float o[3], const float d[3], float t_min, float t_max) {
    float inv[3];
    for (int c = 0; c < 3; ++c) inv[c] = 1.0f / (d[c] != 0.0f ? d[c] : (float)1e-6);
    float tmin[3], tmax[3];
    for (int c = 0; c < 3; ++c) {
        const float t1 = (b.mn[c] - o[c]) * inv[c];
        const float t2 = (b.mx[c] - o[c]) * inv[c];
        tmin[c] = std::fmin(t1, t2);
        tmax[c] = std::fmax(t1, t2);
    }
    const float t_enter = std::fmax(std::fmax(tmin[0], tmin[1]), tmin[2]);
    const float t_exit = std::fmin(std::fmin(tmax[0], tmax[1]), tmax[2]);
    return !(t_enter > t_exit || t_exit < t_min || t_enter > t_max);
}

float max_scale(const float* s) {
    float r = s[0];
    if (s[1] > r) r = s[1];
    if (s[2] > r) r = s[2];
    return r;
}

}  // namespace

extern "C" {

uint32_t oracle_expand_bits(uint32_t val) {
    uint32_t v = val & 0x3FF;
    v = (v | (v << 16)) & 0x030000FF;
    v = (v | (v << 8)) & 0x0300F00F;
    v = (v | (v << 4)) & 0x030C30C3;
    v = (v | (v << 2)) & 0x09249249;
    return v;
}

uint32_t oracle_morton3d(float nx, float ny, float nz) {
    float c[3] = {nx, ny, nz};
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
        float v = c[k];
        if (v < 0.0f) v = 0.0f;
        else if (v > 1.0f) v = 1.0f;
        q[k] = v == v ? (uint32_t)(v * 1023.0f) : 0u;
    }
    return oracle_expand_bits(q[0]) | (oracle_expand_bits(q[1]) << 1) | (oracle_expand_bits(q[2]) << 2);
}

/* Writes the nodes (capacity: n plus ceil(n / 2^k) for each level k, at
 * most 2n + log2(n)) and the leaves' Gaussians; returns the node count (the
 * root is the last node). codes_out (n, optional): the Morton
 * code of each Gaussian, in input order. */
int64_t oracle_bvh_build(const float* means, const float* scales, int64_t n, void* nodes_out,
                         int32_t* splat_index, uint32_t* codes_out) {
    if (n <= 0) return 0;
    Node* nodes = (Node*)nodes_out;
    /* the cloud's box as add_gaussian maintains it */
    float bmin[3] = {(float)1e9, (float)1e9, (float)1e9}, bmax[3] = {(float)-1e9, (float)-1e9, (float)-1e9};
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            const float p = means[i * 3 + c];
            if (p < bmin[c]) bmin[c] = p;
        }
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            const float p = means[i * 3 + c];
            if (p > bmax[c]) bmax[c] = p;
        }
    float inv[3];
    for (int c = 0; c < 3; ++c) {
        const float ext = bmax[c] - bmin[c];
        inv[c] = 1.0f / (ext > (float)0.001 ? ext : 1.0f);
    }
    std::vector<uint64_t> keys((size_t)n);
    std::vector<uint32_t> idx((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t m = oracle_morton3d((means[i * 3] - bmin[0]) * inv[0], (means[i * 3 + 1] - bmin[1]) * inv[1],
                                           (means[i * 3 + 2] - bmin[2]) * inv[2]);
        keys[(size_t)i] = m;
        idx[(size_t)i] = (uint32_t)i;
        if (codes_out) codes_out[i] = m;
    }
    oracle_radix_sort64(keys.data(), idx.data(), n, 1);
    for (int64_t i = 0; i < n; ++i) {                        /* leaves, bvh.mojo:78-93 */
        const int64_t g = idx[(size_t)i];
        const float r3 = max_scale(scales + g * 3) * 3.0f;
        Node& L = nodes[i];
        for (int c = 0; c < 3; ++c) {
            L.mn[c] = means[g * 3 + c] - r3;
            L.mx[c] = means[g * 3 + c] + r3;
        }
        L.left = L.right = -1;
        splat_index[i] = (int32_t)g;
    }
    int64_t start = 0, count = n, total = n;                 /* bvh.mojo:96-117 */
    while (count > 1) {
        const int64_t next = (count + 1) / 2;
        for (int64_t i = 0; i < next; ++i) {
            const int64_t l = start + i * 2, r = l + 1;
            Node p = nodes[l];
            p.left = (int32_t)l;
            p.right = -1;
            if (r < start + count) {
                p.right = (int32_t)r;
                expand_point(p, nodes[r].mn);
                expand_point(p, nodes[r].mx);
            }
            nodes[total++] = p;
        }
        start += count;
        count = next;
    }
    return total;
}

/* Ray3f(origin, direction): the stored direction, normalised (camera.mojo:16-18). */
void oracle_ray_direction(const float direction[3], float out[3]) { normalize3(direction, out); }

/* hit_out: LumenRayHit layout (hit, splat index, distance, point xyz).
 * direction: the ray's stored direction (a Ray3f's, already normalised). */
void oracle_raycast(const void* nodes_in, const int32_t* splat_index, int64_t node_count, int64_t root,
                    const float* means, const float* scales, int64_t n, const float origin[3],
                    const float direction[3], float max_dist, void* hit_out) {
    struct Hit {
        int32_t hit, splat;
        float distance, point[3];
    } h{0, -1, (float)1e9, {0.0f, 0.0f, 0.0f}};
    const Node* nodes = (const Node*)nodes_in;
    if (node_count == 0 || root == -1) {
        std::memcpy(hit_out, &h, sizeof(h));
        return;
    }
    const float d[3] = {direction[0], direction[1], direction[2]};
    h.distance = max_dist;
    std::vector<int64_t> stack;
    stack.push_back(root);
    while (!stack.empty()) {
        const int64_t ci = stack.back();
        stack.pop_back();
        const Node& nd = nodes[ci];
        if (!intersect_ray(nd, origin, d, 0.0f, h.distance)) continue;
        if (nd.left == -1 && nd.right == -1) {
            const int32_t s = splat_index[ci];
            if (s >= 0 && s < n) {
                const float* c = means + (int64_t)s * 3;
                const float oc[3] = {c[0] - origin[0], c[1] - origin[1], c[2] - origin[2]};
                const float t_proj = oc[0] * d[0] + oc[1] * d[1] + oc[2] * d[2];
                if (t_proj > 0.0f && t_proj < h.distance) {
                    const float pt[3] = {origin[0] + d[0] * t_proj, origin[1] + d[1] * t_proj,
                                         origin[2] + d[2] * t_proj};
                    const float df[3] = {pt[0] - c[0], pt[1] - c[1], pt[2] - c[2]};
                    const float dist = std::sqrt(df[0] * df[0] + df[1] * df[1] + df[2] * df[2]);
                    if (dist <= max_scale(scales + (int64_t)s * 3) * 3.0f) {
                        h.hit = 1;
                        h.splat = s;
                        h.distance = t_proj;
                        std::memcpy(h.point, pt, sizeof(pt));
                    }
                }
            }
        } else {
            if (nd.left >= 0) stack.push_back(nd.left);
            if (nd.right >= 0) stack.push_back(nd.right);
        }
    }
    std::memcpy(hit_out, &h, sizeof(h));
}

/* ray_out: origin xyz, direction xyz (normalised, as Ray3f stores it) */
void oracle_generate_ray(const OracleCamera* cam, float px, float py, float ray_out[6]) {
    const float x_norm = (px - cam->cx) / cam->fx;
    const float y_norm = (py - cam->cy) / cam->fy;
    const float v[3] = {x_norm, y_norm, 1.0f};
    float dc[3];
    normalize3(v, dc);
    /* rotation normalised by PinholeCamera (camera.mojo:37-40), rotate_vec
     * q * (0, v) * q^-1 (quaternion.mojo:80-87) */
    float q[4] = {cam->rotation[0], cam->rotation[1], cam->rotation[2], cam->rotation[3]};
    {
        const float ns = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        const float nn = std::sqrt(ns);
        if (nn > (float)0.000001) {
            const float inv_n = 1.0f / nn;
            for (int k = 0; k < 4; ++k) q[k] = q[k] * inv_n;
        } else {
            q[0] = 1.0f;
            q[1] = q[2] = q[3] = 0.0f;
        }
    }
    float qi[4] = {1.0f, 0.0f, 0.0f, 0.0f};
    {
        const float ns = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        if (ns > (float)0.000001) {
            const float inv_ns = 1.0f / ns;
            qi[0] = q[0] * inv_ns;
            qi[1] = -q[1] * inv_ns;
            qi[2] = -q[2] * inv_ns;
            qi[3] = -q[3] * inv_ns;
        }
    }
    auto mul = [](const float a[4], const float b[4], float o[4]) {
        o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
        o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
        o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
        o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
    };
    const float p[4] = {0.0f, dc[0], dc[1], dc[2]};
    float t[4], r[4];
    mul(q, p, t);
    mul(t, qi, r);
    const float dw[3] = {r[1], r[2], r[3]};
    float d[3];
    normalize3(dw, d);
    ray_out[0] = cam->position[0];
    ray_out[1] = cam->position[1];
    ray_out[2] = cam->position[2];
    ray_out[3] = d[0];
    ray_out[4] = d[1];
    ray_out[5] = d[2];
}

}  // extern "C"
