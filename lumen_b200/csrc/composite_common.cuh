/*
 * composite_common.cuh - pixel blocking and the splat reach test shared by
 * the forward and backward compositors.
 */
#pragma once

#include <cfloat>

#include "splat_common.cuh"

namespace lumen {

/* Warp w of a tile shades an 8x4 block of pixels. */
__device__ __forceinline__ int warp_block_x(int w) { return (w & 1) * 8; }
__device__ __forceinline__ int warp_block_y(int w) { return (w >> 1) * 4; }

/* Minimum of q(x, y) = a x^2 + 2 b x y + c y^2 over [x0,x1] x [y0,y1]
 * (a > 0, c > 0, ac > b^2): 0 if the origin (q's minimum) is inside,
 * otherwise the least of the minima over the edges that face the origin:
 * the segment from the origin to any point p of the rectangle enters it
 * through such an edge, at a point t p (0 < t <= 1) where q = t^2 q(p) <=
 * q(p). At most one vertical and one horizontal edge face the origin (the
 * edge x = x0 when x0 > 0, x = x1 when x1 < 0, and likewise in y); q is
 * convex along each edge, so its minimum there is at the clamped
 * stationary point. Branch-free: both edges are evaluated and the ones that
 * do not face the origin are dropped. */
__device__ __forceinline__ float quad_min_rect(float a, float b, float c, float b_over_a, float b_over_c,
                                               float x0, float x1, float y0, float y1) {
    const float x = x0 > 0.0f ? x0 : x1;   /* the vertical edge nearer the origin */
    const float y = y0 > 0.0f ? y0 : y1;
    const float ye = fminf(fmaxf(-b_over_c * x, y0), y1);
    const float xe = fminf(fmaxf(-b_over_a * y, x0), x1);
    /* fused multiply-adds (this is a conservative filter, not the blend's
     * arithmetic; its rounding is covered by the caller's margin) */
    const float b2 = 2.0f * b;
    const float mv = __fmaf_rn(c * ye, ye, __fmaf_rn(b2 * x, ye, a * x * x));
    const float mh = __fmaf_rn(a * xe, xe, __fmaf_rn(b2 * xe, y, c * y * y));
    const bool fv = x0 > 0.0f || x1 < 0.0f, fh = y0 > 0.0f || y1 < 0.0f;
    if (!fv && !fh) return 0.0f;   /* the origin is inside */
    return fminf(fv ? mv : INFINITY, fh ? mh : INFINITY);
}

/* The power above which a splat cannot be blended at any pixel: the
 * reference skips power > 4.5 (compositor.mojo:80-82), and alpha =
 * opacity * exp(-power) falls below the 1/255 skip (compositor.mojo:33-35)
 * once power exceeds ln(opacity / (1/255)); the 1e-3 margin is far above
 * the rounding of the exponential and the logarithm, so a pixel beyond the
 * cutoff is one the exact test skips too (and one at or below it takes the
 * exact test). */
__device__ __forceinline__ float splat_power_cutoff(float opacity) {
    return fminf(4.5f, logf(opacity / min_alpha()) + 1e-3f);
}

/* Bit w set when the splat may reach the blend threshold at some pixel
 * centre of warp w's block. A pixel is blended only if
 * power <= 4.5 and opacity * exp(-power) >= 1/255 (compositor.mojo:62-89,
 * :33-35), i.e. 2 * power <= 2 * min(4.5, ln(255 * opacity)); the test uses
 * that bound with a 0.1% + 0.01 margin, plus a margin for the rounding of
 * the two float evaluations (the block's minimum here, a pixel's power in
 * the blend): each is within a few units in the last place of the sum of
 * the absolute terms, |a| x^2 + 2 |b x y| + |c| y^2 <= S (x^2 + y^2) with
 * S = |a| + |c| + 2 |b|, so 1e-6 S R^2 (R^2 bounding x^2 + y^2 over the
 * tile's pixel centres, about 16 float ulps) covers both. That term matters only for
 * needle-like splats (conic condition numbers above about 1e4, whose terms
 * cancel); for the others the fixed margin dominates. Culling therefore
 * never removes a splat that the per-pixel loop would blend and the
 * results are unchanged. */
__device__ __forceinline__ unsigned int reach_mask(float4 geo, float4 con, float tile_x0, float tile_y0) {
    const float a = con.x, b = con.y, c = con.z, op = geo.w;
    /* degenerate, non-finite or subnormal conics (whose approximate
     * reciprocals below flush to infinity): every block, as the blend decides */
    if (!(a >= FLT_MIN && c >= FLT_MIN && a * c - b * b > 0.0f) || !isfinite(a * c)) return 0xFFu;
    const float pcut = fminf(4.5f, __logf(op / min_alpha()) + 0.01f);
    if (pcut < 0.0f) return 0u;
    const float qcut = 2.0f * pcut * 1.001f + 1e-3f;
    /* the stationary points only need to be close: an error d in one moves
     * the edge's value by c d^2 (second order) */
    float ra, rc;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(ra) : "f"(a));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rc) : "f"(c));
    const float b_over_a = b * ra, b_over_c = b * rc;
    /* R^2 over the whole tile's pixel centres bounds it for every block */
    const float tx0 = tile_x0 + 0.5f - geo.x, tx1 = tx0 + (float)(kTile - 1);
    const float ty0 = tile_y0 + 0.5f - geo.y, ty1 = ty0 + (float)(kTile - 1);
    const float r2 = fmaxf(tx0 * tx0, tx1 * tx1) + fmaxf(ty0 * ty0, ty1 * ty1);
    const float thr = qcut + 1e-6f * (fabsf(a) + fabsf(c) + 2.0f * fabsf(b)) * r2;
    unsigned int m = 0;
#pragma unroll
    for (int w = 0; w < kTilePixels / 32; ++w) {
        const float x0 = tile_x0 + (float)warp_block_x(w) + 0.5f - geo.x;
        const float y0 = tile_y0 + (float)warp_block_y(w) + 0.5f - geo.y;
        if (quad_min_rect(a, b, c, b_over_a, b_over_c, x0, x0 + 7.0f, y0, y0 + 3.0f) <= thr) m |= 1u << w;
    }
    return m;
}

}  // namespace lumen
