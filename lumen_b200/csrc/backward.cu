/*
 * backward.cu - the adjoint of the forward pipeline (no reference
 * counterpart: the reference has no analytic backward; its gradient code
 * only stores buffers, src/optim/gradients.mojo:11-106).
 *
 * K6 composite_backward_kernel: per 16x16 tile, per pixel, one front-to-
 * back sweep over the splats the forward blended, up to the pixel's
 * last-visited instance (the forward's last_idx output, so the sweep stops
 * on the splat where the forward stopped). Per splat j, with the
 * transmittance T_j before it and w_j = alpha_j T_j:
 *   dL/dc = G_rgb w, dL/dz = G_depth w,
 *   dL/dalpha = T_j (G . col_j) - (G . C - G . P_j - g_tail) / (1 - alpha),
 * where G . C is the upstream gradient dotted with the forward's blended
 * colour and depth, G . P_j the same dot product of the running sum up to
 * and including j (so G . (C - P_j) is what is blended behind j) and g_tail
 * = (G_alpha - [white] sum_ch G_ch) T_final; then through
 * alpha = min(op exp(-power), 0.99) (no gradient when clamped) and power =
 * 0.5 (a dx^2 + 2 b dx dy + c dy^2) to the centre, the conic and the
 * opacity. Gradient arithmetic uses fused multiply-adds and the hardware
 * exponential and reciprocal; the decisions the forward took (power above
 * 4.5, alpha below 1/255, the 0.99 clamp) are taken exactly as the forward
 * took them: the power is formed with separately rounded operations in the
 * forward's order, and an alpha within a few parts per million of a
 * threshold is recomputed with the shared exponential. The 10 values per
 * splat are summed over the warp through a shared-memory transpose (each
 * lane writes its row; lanes 0..29 each add 11 entries of one column,
 * three partial sums per value combine by two shuffles), over the CTA with
 * shared atomics, and added to the splat's Gaussian with three vector
 * atomics per tile.
 *
 * K7 project_backward_kernel: per Gaussian, the chain rule through the
 * conic inverse, the EWA product T Sigma T^T with T = J W, the projective
 * Jacobian, the screen projection, Sigma = M M^T with M = R(q) S, the
 * quaternion normalisation, the SH colour (clamped channels get none) and
 * the view direction, and the exp / sigmoid activations.
 *
 * K8 l1_loss_kernel: compute_l1_loss (src/optim/loss.mojo:11-35).
 *
 * This file is compiled with fused multiply-add contraction; the few
 * operations that must round as the forward's do are written with
 * explicitly rounded intrinsics.
 */
#include "composite_common.cuh"

namespace lumen {

constexpr int kGrad2D = 10;   /* cx, cy, ic00, ic01, ic11, opacity, r, g, b, depth */
constexpr int kGrad2DStride = 12;   /* floats per Gaussian in splat2d: 16-byte rows for vector atomics */
constexpr int kBwdChunk = kTilePixels;   /* instances staged per round */
/* per warp: 32 rows of kGrad2D values, then zero padding up to the last
 * word a lane of the transposed read touches (31 + 30 * 10) */
constexpr int kRedRows = 32 * kGrad2D;
constexpr int kRedWords = 360;
constexpr int kRedReads = 11;

struct BackwardSmem {
    float4 geo[kBwdChunk];        /* cx, cy, depth, opacity */
    float4 con[kBwdChunk];        /* 0.5 ic00, ic01, 0.5 ic11 (the forward's prescaled conic), power cutoff */
    float4 col[kBwdChunk];        /* r, g, b, - */
    unsigned char mask[kBwdChunk];
    unsigned short list[kTilePixels / 32][kBwdChunk];
    float acc[kBwdChunk][kGrad2D];
    unsigned int gid[kBwdChunk];
    float red[kTilePixels / 32][kRedWords];
    int tile_last;
};

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

/* Stage chunk [cs, min(cs + kBwdChunk, end)) of the tile's sorted
 * instances: records, reach masks, Gaussian ids. Returns the warp's splat
 * list length. */
__device__ __forceinline__ int stage_chunk(BackwardSmem& s, const LumenSplatRecord* __restrict__ records,
                                           const unsigned int* __restrict__ vals,
                                           const unsigned int* __restrict__ visible_ids, unsigned int n_visible,
                                           Control* ctrl, int cs, int end, float tile_x0, float tile_y0) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i = cs + tid;
    unsigned int m = 0;
    if (i < end) {
        const unsigned int v = vals[i];
        if (v >= n_visible) {
            atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_BOUNDS);
        } else {
            const float4* r4 = reinterpret_cast<const float4*>(records + v);
            const float4 geo = __ldg(r4), con = __ldg(r4 + 1);
            s.geo[tid] = geo;
            s.con[tid] = make_float4(0.5f * con.x, con.y, 0.5f * con.z, splat_power_cutoff(geo.w));
            s.col[tid] = __ldg(r4 + 2);
            s.gid[tid] = visible_ids[v];
            m = reach_mask(geo, con, tile_x0, tile_y0);
        }
    }
    s.mask[tid] = (unsigned char)m;
#pragma unroll
    for (int k = 0; k < kGrad2D; ++k) s.acc[tid][k] = 0.0f;
    __syncthreads();
    const int n = end - cs < kBwdChunk ? end - cs : kBwdChunk;
    int cnt = 0;
    for (int base = 0; base < n; base += 32) {
        const int j = base + lane;
        const bool bit = j < n && ((s.mask[j] >> warp) & 1u);
        const unsigned int bal = __ballot_sync(0xffffffffu, bit);
        if (bit) s.list[warp][cnt + __popc(bal & lanemask_lt())] = (unsigned short)j;
        cnt += __popc(bal);
    }
    __syncwarp();
    return cnt;
}

/* The hardware exponential of -p (p in [0, 4.5]): within a few parts per
 * million of lumen_expf_core(-p). */
__device__ __forceinline__ float fast_exp_neg(float p) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(p * -1.44269504088896341f));
    return r;
}

__device__ __forceinline__ float fast_rcp(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__global__ void __launch_bounds__(kTilePixels, 5)
composite_backward_kernel(const LumenSplatRecord* __restrict__ records, LumenGpuFrame f, Control* ctrl,
                          int width, int height, int tiles_x, LumenRenderOptions opt,
                          const float* __restrict__ out_rgb, const float* __restrict__ out_depth,
                          const float* __restrict__ out_alpha, const int* __restrict__ out_last,
                          const float* __restrict__ grad_rgb, const float* __restrict__ grad_depth,
                          const float* __restrict__ grad_alpha, float* __restrict__ grad2d) {
    chain_begin();
    __shared__ BackwardSmem s;
    const int tile = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tx = tile % tiles_x, ty = tile / tiles_x;
    const int px = tx * kTile + warp_block_x(warp) + (lane & 7);
    const int py = ty * kTile + warp_block_y(warp) + (lane >> 3);
    const bool inside = px < width && py < height;
    const long long pix = (long long)py * width + px;
    const long long cap = f.instance_capacity;
    const long long K = (long long)ctrl->n_instances < cap ? (long long)ctrl->n_instances : cap;
    if (K == 0) return;
    const int rs = f.ranges[2 * tile], re = f.ranges[2 * tile + 1];
    if (rs == -1 || rs >= re) return;
    if (rs < 0 || (long long)re > K) {
        if (tid == 0) atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_BOUNDS);
        return;
    }
    const unsigned int n_visible = ctrl->n_visible;
    const unsigned int* __restrict__ vals = ctrl->tile_sort.sorted_buffer ? f.vals[1] : f.vals[0];
    const float pxc = (float)px + 0.5f, pyc = (float)py + 0.5f;
    const float tile_x0 = (float)(tx * kTile), tile_y0 = (float)(ty * kTile);

    /* the pixel's upstream gradient and the forward's outputs */
    float g_r = 0.0f, g_g = 0.0f, g_b = 0.0f, g_d = 0.0f, Gc = 0.0f;
    int last = -1;
    if (tid == 0) s.tile_last = -1;
    for (int w = kRedRows + lane; w < kRedWords; w += 32) s.red[warp][w] = 0.0f;
    if (inside) {
        last = out_last[pix];
        if (last >= re) {   /* self-check: a last-visited instance beyond the tile's range */
            atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_BOUNDS);
            last = re - 1;
        }
        g_r = grad_rgb[pix * 3 + 0];
        g_g = grad_rgb[pix * 3 + 1];
        g_b = grad_rgb[pix * 3 + 2];
        float C_z = 0.0f;
        if (grad_depth && opt.compute_depth) {
            g_d = grad_depth[pix];
            C_z = out_depth[pix];
        }
        const float g_a = grad_alpha ? grad_alpha[pix] : 0.0f;
        const float T_final = 1.0f - out_alpha[pix];
        const float bg = opt.white_background ? T_final : 0.0f;
        /* terms of dL/dalpha_j that scale with 1 / (1 - alpha_j) and do not
         * change along the sweep: G . C - g_tail */
        const float g_tail = (g_a - (opt.white_background ? (g_r + g_g + g_b) : 0.0f)) * T_final;
        Gc = g_r * (out_rgb[pix * 3 + 0] - bg) + g_g * (out_rgb[pix * 3 + 1] - bg) +
             g_b * (out_rgb[pix * 3 + 2] - bg) + g_d * C_z - g_tail;
    }
    /* the tile's sweep ends at the last instance any of its pixels visited */
    const int wlast = __reduce_max_sync(0xffffffffu, last);
    __syncthreads();
    if (lane == 0 && wlast >= rs) atomicMax(&s.tile_last, wlast);
    __syncthreads();
    const int end = s.tile_last + 1;   /* <= re */
    if (end <= rs) return;

    float T = 1.0f, GP = 0.0f;
    float* red = s.red[warp];
    for (int cs = rs; cs < end; cs += kBwdChunk) {
        const int cnt = stage_chunk(s, records, vals, f.visible_ids, n_visible, ctrl, cs, end, tile_x0, tile_y0);
        for (int t = 0; t < cnt; ++t) {
            const int j = s.list[warp][t];
            if (cs + j > wlast) break;   /* every pixel of the warp is past its last splat */
            float gcx = 0.0f, gcy = 0.0f, ga = 0.0f, gb = 0.0f, gc = 0.0f, gop = 0.0f;
            float gr = 0.0f, gg_ = 0.0f, gbl = 0.0f, gz = 0.0f;
            bool contrib = false;
            if (cs + j <= last) {
                const float4 geo = s.geo[j], cc = s.con[j];
                const float dx = pxc - geo.x, dy = pyc - geo.y;
                /* the forward's power, operation by operation */
                float power = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(cc.x, dx), dx), __fmul_rn(__fmul_rn(cc.y, dx), dy)),
                                        __fmul_rn(__fmul_rn(cc.z, dy), dy));
                bool pclamp = false;
                if (power < 0.0f) { power = 0.0f; pclamp = true; }
                if (!(power > cc.w)) {   /* beyond 4.5, or certain to fall below 1/255 */
                    float gexp = fast_exp_neg(power);
                    float raw = geo.w * gexp;
                    /* near the 1/255 skip or the 0.99 clamp the decision is taken
                     * with the forward's exponential */
                    if (fabsf(raw - min_alpha()) <= 4e-6f * min_alpha() || fabsf(raw - (float)0.99) <= 4e-6f) {
                        gexp = lumen_expf_core(-power);
                        raw = __fmul_rn(geo.w, gexp);
                    }
                    const bool aclamp = raw > (float)0.99;
                    const float alpha = aclamp ? (float)0.99 : raw;
                    if (!(alpha < min_alpha())) {
                        contrib = true;
                        const float4 col = s.col[j];
                        const float w = alpha * T;
                        gr = g_r * w;
                        gg_ = g_g * w;
                        gbl = g_b * w;
                        gz = g_d * w;
                        const float gcol = g_r * col.x + g_g * col.y + g_b * col.z + g_d * geo.z;
                        GP += w * gcol;
                        const float one_minus = 1.0f - alpha;
                        const float dalpha = T * gcol - (Gc - GP) * fast_rcp(one_minus);
                        T *= one_minus;
                        if (!aclamp) {
                            gop = dalpha * gexp;
                            if (!pclamp) {
                                const float dpower = -gop * geo.w;
                                const float dxp = dx * dpower;
                                ga = 0.5f * dx * dxp;
                                gb = dy * dxp;
                                gc = 0.5f * dy * dy * dpower;
                                /* d dx / d cx = -1; the staged conic holds 0.5 a and 0.5 c */
                                gcx = -(2.0f * cc.x * dx + cc.y * dy) * dpower;
                                gcy = -(cc.y * dx + 2.0f * cc.z * dy) * dpower;
                            }
                        }
                    }
                }
            }
            if (__any_sync(0xffffffffu, contrib)) {
                /* warp sum by a shared-memory transpose: row `lane` holds this
                 * lane's 10 values; lane l < 30 adds words l, l + 30, ...
                 * (value l % 10 of rows l / 10, l / 10 + 3, ...) */
                float2* row = reinterpret_cast<float2*>(red + lane * kGrad2D);
                row[0] = make_float2(gcx, gcy);
                row[1] = make_float2(ga, gb);
                row[2] = make_float2(gc, gop);
                row[3] = make_float2(gr, gg_);
                row[4] = make_float2(gbl, gz);
                __syncwarp();
                float sum = 0.0f;
#pragma unroll
                for (int r = 0; r < kRedReads; ++r) sum += red[lane + 30 * r];
                sum += __shfl_down_sync(0xffffffffu, sum, 10) + __shfl_down_sync(0xffffffffu, sum, 20);
                if (lane < kGrad2D && sum != 0.0f) atomicAdd(&s.acc[j][lane], sum);
                __syncwarp();
            }
        }
        __syncthreads();
        /* per (splat, tile): three vector atomics (4 + 4 + 2 values) */
        const int i = cs + tid;
        if (i < end) {
            float* dst = grad2d + (size_t)s.gid[tid] * kGrad2DStride;
            const float* a = s.acc[tid];
            if (a[0] != 0.0f || a[1] != 0.0f || a[2] != 0.0f || a[3] != 0.0f)
                atomicAdd(reinterpret_cast<float4*>(dst), make_float4(a[0], a[1], a[2], a[3]));
            if (a[4] != 0.0f || a[5] != 0.0f || a[6] != 0.0f || a[7] != 0.0f)
                atomicAdd(reinterpret_cast<float4*>(dst + 4), make_float4(a[4], a[5], a[6], a[7]));
            if (a[8] != 0.0f || a[9] != 0.0f)
                atomicAdd(reinterpret_cast<float2*>(dst + 8), make_float2(a[8], a[9]));
        }
    }
}

/* ---------------------------------------------------------------- K7 -- */

__device__ __forceinline__ void rot_from_quat(float w, float x, float y, float z, float R[9]) {
    R[0] = 1.0f - 2.0f * (y * y + z * z); R[1] = 2.0f * (x * y - w * z); R[2] = 2.0f * (x * z + w * y);
    R[3] = 2.0f * (x * y + w * z); R[4] = 1.0f - 2.0f * (x * x + z * z); R[5] = 2.0f * (y * z - w * x);
    R[6] = 2.0f * (x * z - w * y); R[7] = 2.0f * (y * z + w * x); R[8] = 1.0f - 2.0f * (x * x + y * y);
}

/* SH basis function k and its gradient with respect to the (unit)
 * direction components, for the constants of spherical_harmonics.mojo:17-26
 * (k is a compile-time constant after unrolling). */
__device__ __forceinline__ void sh_term(int k, float x, float y, float z, float& Y, float& dX, float& dY,
                                        float& dZ) {
    const float C0 = (float)0.28209479177387814, C1 = (float)0.4886025119029199;
    const float C2_0 = (float)1.0925484305920792, C2_1 = (float)0.31539156525252005;
    const float C2_2 = (float)0.5462742152960396, C3_0 = (float)0.5900435899266435;
    const float C3_1 = (float)2.890611442640554, C3_2 = (float)0.4570457994644658;
    const float C3_3 = (float)0.3731763325901154, C3_4 = (float)1.445305721320277;
    const float xx = x * x, yy = y * y, zz = z * z;
    switch (k) {
        case 0: Y = C0; dX = 0.0f; dY = 0.0f; dZ = 0.0f; break;
        case 1: Y = -C1 * y; dX = 0.0f; dY = -C1; dZ = 0.0f; break;
        case 2: Y = C1 * z; dX = 0.0f; dY = 0.0f; dZ = C1; break;
        case 3: Y = -C1 * x; dX = -C1; dY = 0.0f; dZ = 0.0f; break;
        case 4: Y = C2_0 * x * y; dX = C2_0 * y; dY = C2_0 * x; dZ = 0.0f; break;
        case 5: Y = -C2_0 * y * z; dX = 0.0f; dY = -C2_0 * z; dZ = -C2_0 * y; break;
        case 6: Y = C2_1 * (2.0f * zz - xx - yy); dX = -2.0f * C2_1 * x; dY = -2.0f * C2_1 * y; dZ = 4.0f * C2_1 * z;
            break;
        case 7: Y = -C2_0 * x * z; dX = -C2_0 * z; dY = 0.0f; dZ = -C2_0 * x; break;
        case 8: Y = C2_2 * (xx - yy); dX = 2.0f * C2_2 * x; dY = -2.0f * C2_2 * y; dZ = 0.0f; break;
        case 9: Y = -C3_0 * y * (3.0f * xx - yy); dX = -6.0f * C3_0 * x * y; dY = -3.0f * C3_0 * (xx - yy);
            dZ = 0.0f; break;
        case 10: Y = C3_1 * x * y * z; dX = C3_1 * y * z; dY = C3_1 * x * z; dZ = C3_1 * x * y; break;
        case 11: Y = -C3_2 * y * (4.0f * zz - xx - yy); dX = 2.0f * C3_2 * x * y;
            dY = -C3_2 * (4.0f * zz - xx - 3.0f * yy); dZ = -8.0f * C3_2 * y * z; break;
        case 12: Y = C3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy); dX = -6.0f * C3_3 * x * z;
            dY = -6.0f * C3_3 * y * z; dZ = C3_3 * (6.0f * zz - 3.0f * xx - 3.0f * yy); break;
        case 13: Y = -C3_2 * x * (4.0f * zz - xx - yy); dX = -C3_2 * (4.0f * zz - 3.0f * xx - yy);
            dY = 2.0f * C3_2 * x * y; dZ = -8.0f * C3_2 * x * z; break;
        case 14: Y = C3_4 * z * (xx - yy); dX = 2.0f * C3_4 * x * z; dY = -2.0f * C3_4 * y * z;
            dZ = C3_4 * (xx - yy); break;
        default: Y = -C3_0 * x * (xx - 3.0f * yy); dX = -3.0f * C3_0 * (xx - yy); dY = 6.0f * C3_0 * x * y;
            dZ = 0.0f; break;
    }
}

constexpr int kProjBwdThreads = 128;
constexpr size_t kProjBwdStageBytes = (size_t)kProjBwdThreads * 48 * sizeof(float);

/* One visible Gaussian's gradients. row: its 48 SH coefficients staged in
 * shared memory (chunk q at q ^ swz), overwritten with dL/dsh. */
__device__ __forceinline__ void project_backward_gaussian(const LumenGpuGaussians& g, const DevCamera& cam,
                                                          const LumenRenderOptions& opt, long long i,
                                                          const float* __restrict__ grad2d,
                                                          const LumenGpuGradients& out, float4* row, int swz) {
    float* gm = out.means + i * 3;
    float* gs = out.scales + i * 3;
    float* gq = out.quats + i * 4;
    const float4 G0 = reinterpret_cast<const float4*>(grad2d + i * kGrad2DStride)[0];
    const float4 G1 = reinterpret_cast<const float4*>(grad2d + i * kGrad2DStride)[1];
    const float2 G2 = reinterpret_cast<const float2*>(grad2d + i * kGrad2DStride)[4];
    const float g_cx = G0.x, g_cy = G0.y, g_a = G0.z, g_b = G0.w, g_c = G1.x, g_op = G1.y;
    const float g_col[3] = {G1.z, G1.w, G2.x};
    const float g_z = G2.y;

    /* parameters and activations */
    const float mx = g.means[i * 3], my = g.means[i * 3 + 1], mz = g.means[i * 3 + 2];
    float s3[3] = {g.scales[i * 3], g.scales[i * 3 + 1], g.scales[i * 3 + 2]};
    float op = g.opacities[i];
    if (opt.params_are_logits) {
        for (int k = 0; k < 3; ++k) s3[k] = lumen_expf(s3[k]);
        op = 1.0f / (1.0f + lumen_expf(-op));
    }
    const float4 q4 = reinterpret_cast<const float4*>(g.quats)[i];
    const float qn2 = q4.x * q4.x + q4.y * q4.y + q4.z * q4.z + q4.w * q4.w;
    const float qlen = sqrtf(qn2);
    const bool qok = qlen > (float)0.000001;
    const float qw = qok ? q4.x / qlen : 1.0f, qx = qok ? q4.y / qlen : 0.0f;
    const float qy = qok ? q4.z / qlen : 0.0f, qz = qok ? q4.w / qlen : 0.0f;
    float R[9];
    rot_from_quat(qw, qx, qy, qz, R);
    float sc[3];
    bool sclamp[3];
    for (int k = 0; k < 3; ++k) {
        sclamp[k] = s3[k] < (float)0.00001;
        sc[k] = sclamp[k] ? (float)0.00001 : s3[k];
    }
    float M[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) M[r * 3 + c] = R[r * 3 + c] * sc[c];
    float S[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) S[r * 3 + c] = M[r * 3] * M[c * 3] + M[r * 3 + 1] * M[c * 3 + 1] + M[r * 3 + 2] * M[c * 3 + 2];
    /* camera space (the Hamilton-product transform equals W (mu - position)) */
    const float* W = cam.W;
    const float vx = mx - cam.px, vy = my - cam.py, vz = mz - cam.pz;
    const float x = W[0] * vx + W[1] * vy + W[2] * vz;
    const float y = W[3] * vx + W[4] * vy + W[5] * vz;
    float z = W[6] * vx + W[7] * vy + W[8] * vz;
    const bool zclamp = z < (float)0.0001;
    const float zj = zclamp ? (float)0.0001 : z;
    const float iz = 1.0f / zj, iz2 = iz * iz, iz3 = iz2 * iz;
    const float fx = cam.fx, fy = cam.fy;
    const float j00 = fx * iz, j02 = -fx * x * iz2, j11 = fy * iz, j12 = -fy * y * iz2;
    float t0[3], t1[3];
    for (int k = 0; k < 3; ++k) {
        t0[k] = j00 * W[k] + j02 * W[6 + k];
        t1[k] = j11 * W[3 + k] + j12 * W[6 + k];
    }
    float St0[3], St1[3];
    for (int r = 0; r < 3; ++r) {
        St0[r] = S[r * 3] * t0[0] + S[r * 3 + 1] * t0[1] + S[r * 3 + 2] * t0[2];
        St1[r] = S[r * 3] * t1[0] + S[r * 3 + 1] * t1[1] + S[r * 3 + 2] * t1[2];
    }
    const float A = t0[0] * St0[0] + t0[1] * St0[1] + t0[2] * St0[2] + opt.lowpass;
    const float B = t0[0] * St1[0] + t0[1] * St1[1] + t0[2] * St1[2];
    const float Cc = t1[0] * St1[0] + t1[1] * St1[1] + t1[2] * St1[2] + opt.lowpass;
    const float det = A * Cc - B * B;

    /* conic -> Sigma2D (A, B, C) */
    float gA = 0.0f, gB = 0.0f, gC = 0.0f;
    if (!(det > (float)-0.0000001 && det < (float)0.0000001)) {
        const float id2 = 1.0f / (det * det);
        gA = (-Cc * Cc * g_a + B * Cc * g_b - B * B * g_c) * id2;
        gB = (2.0f * B * Cc * g_a - (det + 2.0f * B * B) * g_b + 2.0f * A * B * g_c) * id2;
        gC = (-B * B * g_a + A * B * g_b - A * A * g_c) * id2;
    }
    /* Sigma2D = T Sigma T^T (+ low pass) -> rows of T and Sigma */
    float dt0[3], dt1[3];
    for (int k = 0; k < 3; ++k) {
        dt0[k] = 2.0f * gA * St0[k] + gB * St1[k];
        dt1[k] = gB * St0[k] + 2.0f * gC * St1[k];
    }
    float Gs[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) Gs[r * 3 + c] = gA * t0[r] * t0[c] + gB * t0[r] * t1[c] + gC * t1[r] * t1[c];
    /* T = J W -> Jacobian entries */
    const float gj00 = dt0[0] * W[0] + dt0[1] * W[1] + dt0[2] * W[2];
    const float gj02 = dt0[0] * W[6] + dt0[1] * W[7] + dt0[2] * W[8];
    const float gj11 = dt1[0] * W[3] + dt1[1] * W[4] + dt1[2] * W[5];
    const float gj12 = dt1[0] * W[6] + dt1[1] * W[7] + dt1[2] * W[8];
    /* camera-space point: screen centre (camera.mojo:73-79), Jacobian, depth */
    const float iz_s = 1.0f / z, iz2_s = iz_s * iz_s;
    float gx = g_cx * fx * iz_s;
    float gy = g_cy * fy * iz_s;
    float gzc = -(g_cx * fx * x + g_cy * fy * y) * iz2_s + g_z;
    gx += gj02 * (-fx * iz2);
    gy += gj12 * (-fy * iz2);
    if (!zclamp) gzc += gj00 * (-fx * iz2) + gj02 * (2.0f * fx * x * iz3) + gj11 * (-fy * iz2) + gj12 * (2.0f * fy * y * iz3);
    float gmu[3];
    for (int k = 0; k < 3; ++k) gmu[k] = W[k] * gx + W[3 + k] * gy + W[6 + k] * gzc;

    /* colour: clamp(0.5 + sum sh_k Y_k(d)), d = normalize(mu - position) */
    {
        const float len = sqrtf(vx * vx + vy * vy + vz * vz);
        const bool dok = len > (float)0.000001;
        const float dx_ = dok ? vx / len : 0.0f, dy_ = dok ? vy / len : 0.0f, dz_ = dok ? vz / len : 0.0f;
        const int n = opt.sh_degree == 0 ? 1 : opt.sh_degree == 1 ? 4 : opt.sh_degree == 2 ? 9 : 16;
        /* two streaming passes over the coefficients, 4 at a time (12 floats
         * = 3 float4): the colour before the clamp (which channels pass a
         * gradient), then the direction gradient and dL/dsh */
        float v0 = 0.5f, v1 = 0.5f, v2 = 0.5f;
#pragma unroll
        for (int grp = 0; grp < 4; ++grp) {
            if (4 * grp >= n) break;
            const float4 a = row[(3 * grp) ^ swz], b = row[(3 * grp + 1) ^ swz], c = row[(3 * grp + 2) ^ swz];
            const float e[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const int k = 4 * grp + kk;
                if (k < n) {
                    float Y, dX, dY, dZ;
                    sh_term(k, dx_, dy_, dz_, Y, dX, dY, dZ);
                    v0 += e[3 * kk] * Y;
                    v1 += e[3 * kk + 1] * Y;
                    v2 += e[3 * kk + 2] * Y;
                }
            }
        }
        const float gc0 = (v0 < 0.0f || v0 > 1.0f) ? 0.0f : g_col[0];
        const float gc1 = (v1 < 0.0f || v1 > 1.0f) ? 0.0f : g_col[1];
        const float gc2 = (v2 < 0.0f || v2 > 1.0f) ? 0.0f : g_col[2];
        float gd0 = 0.0f, gd1 = 0.0f, gd2 = 0.0f;
#pragma unroll
        for (int grp = 0; grp < 4; ++grp) {
            float o[12];
            if (4 * grp < n) {
                const float4 a = row[(3 * grp) ^ swz], b = row[(3 * grp + 1) ^ swz], c = row[(3 * grp + 2) ^ swz];
                const float e[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const int k = 4 * grp + kk;
                    float Y = 0.0f, dX = 0.0f, dY = 0.0f, dZ = 0.0f;
                    if (k < n) sh_term(k, dx_, dy_, dz_, Y, dX, dY, dZ);
                    const float s3 = gc0 * e[3 * kk] + gc1 * e[3 * kk + 1] + gc2 * e[3 * kk + 2];
                    gd0 += s3 * dX;
                    gd1 += s3 * dY;
                    gd2 += s3 * dZ;
                    /* dL/dsh[k][ch] = gcol[ch] Y_k */
                    o[3 * kk] = gc0 * Y;
                    o[3 * kk + 1] = gc1 * Y;
                    o[3 * kk + 2] = gc2 * Y;
                }
            } else {
#pragma unroll
                for (int q = 0; q < 12; ++q) o[q] = 0.0f;
            }
            row[(3 * grp) ^ swz] = make_float4(o[0], o[1], o[2], o[3]);
            row[(3 * grp + 1) ^ swz] = make_float4(o[4], o[5], o[6], o[7]);
            row[(3 * grp + 2) ^ swz] = make_float4(o[8], o[9], o[10], o[11]);
        }
        if (dok) {
            const float dot = gd0 * dx_ + gd1 * dy_ + gd2 * dz_;
            gmu[0] += (gd0 - dx_ * dot) / len;
            gmu[1] += (gd1 - dy_ * dot) / len;
            gmu[2] += (gd2 - dz_ * dot) / len;
        }
    }
    gm[0] = gmu[0]; gm[1] = gmu[1]; gm[2] = gmu[2];

    /* Sigma = M M^T, M = R diag(s) */
    float gM[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            float a = 0.0f;
            for (int k = 0; k < 3; ++k) a += (Gs[r * 3 + k] + Gs[k * 3 + r]) * M[k * 3 + c];
            gM[r * 3 + c] = a;
        }
    float gsc[3];
    for (int c = 0; c < 3; ++c) {
        float a = 0.0f;
        for (int r = 0; r < 3; ++r) a += gM[r * 3 + c] * R[r * 3 + c];
        gsc[c] = sclamp[c] ? 0.0f : a;
    }
    float gR[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) gR[r * 3 + c] = gM[r * 3 + c] * sc[c];
    /* R(q) for the unit quaternion (w, x, y, z) */
    float gqw = 2.0f * (-qz * gR[1] + qy * gR[2] + qz * gR[3] - qx * gR[5] - qy * gR[6] + qx * gR[7]);
    float gqx = 2.0f * (qy * gR[1] + qz * gR[2] + qy * gR[3] - 2.0f * qx * gR[4] - qw * gR[5] + qz * gR[6] +
                        qw * gR[7] - 2.0f * qx * gR[8]);
    float gqy = 2.0f * (-2.0f * qy * gR[0] + qx * gR[1] + qw * gR[2] + qx * gR[3] + qz * gR[5] - qw * gR[6] +
                        qz * gR[7] - 2.0f * qy * gR[8]);
    float gqz = 2.0f * (-2.0f * qz * gR[0] - qw * gR[1] + qx * gR[2] + qw * gR[3] - 2.0f * qz * gR[4] + qy * gR[5] +
                        qx * gR[6] + qy * gR[7]);
    if (qok) {   /* through q / |q| */
        const float dot = gqw * qw + gqx * qx + gqy * qy + gqz * qz;
        gq[0] = (gqw - qw * dot) / qlen;
        gq[1] = (gqx - qx * dot) / qlen;
        gq[2] = (gqy - qy * dot) / qlen;
        gq[3] = (gqz - qz * dot) / qlen;
    } else {
        gq[0] = gq[1] = gq[2] = gq[3] = 0.0f;
    }
    if (opt.params_are_logits) {
        for (int k = 0; k < 3; ++k) gs[k] = gsc[k] * s3[k];
        out.opacities[i] = g_op * op * (1.0f - op);
    } else {
        for (int k = 0; k < 3; ++k) gs[k] = gsc[k];
        out.opacities[i] = g_op;
    }
}

/* Per block of 128 Gaussians: the SH rows come in with coalesced
 * asynchronous 16-byte copies (swizzled rows, see sh_swizzle), each thread
 * forms its Gaussian's gradients (its dL/dsh in place of its row), and the
 * rows go out with coalesced 16-byte stores. Culled Gaussians get zeros. */
__global__ void __launch_bounds__(kProjBwdThreads, 8)
project_backward_kernel(LumenGpuGaussians g, LumenViewCamera camera, LumenRenderOptions opt,
                        const int* __restrict__ radii, const float* __restrict__ grad2d, LumenGpuGradients out) {
    chain_begin();
    __shared__ DevCamera cam_s;
    extern __shared__ float4 sh_rows[];   /* kProjBwdThreads x 12 chunks */
    const int tid = threadIdx.x;
    const long long i0 = (long long)blockIdx.x * kProjBwdThreads;
    const int nblk = (int)(g.count - i0 < kProjBwdThreads ? g.count - i0 : kProjBwdThreads);
    {
        const float4* src = reinterpret_cast<const float4*>(g.sh + i0 * 48);
        for (int c = tid; c < nblk * 12; c += kProjBwdThreads) {
            const int t = c / 12, q = c - 12 * t;
            cp_async16(sh_rows + 12 * t + (q ^ sh_swizzle(t)), src + c);
        }
        cp_async_commit();
    }
    if (tid == 0) setup_camera(camera, cam_s);
    const long long i = i0 + tid;
    const bool visible = tid < nblk && radii[i] > 0;
    cp_async_wait_all();
    __syncthreads();
    float4* row = sh_rows + tid * 12;
    const int swz = sh_swizzle(tid);
    if (visible) {
        project_backward_gaussian(g, cam_s, opt, i, grad2d, out, row, swz);
    } else if (tid < nblk) {
        float* gm = out.means + i * 3;
        float* gs = out.scales + i * 3;
        float* gq = out.quats + i * 4;
        gm[0] = gm[1] = gm[2] = 0.0f;
        gs[0] = gs[1] = gs[2] = 0.0f;
        gq[0] = gq[1] = gq[2] = gq[3] = 0.0f;
        out.opacities[i] = 0.0f;
#pragma unroll
        for (int k = 0; k < 12; ++k) row[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    __syncthreads();
    float4* dst = reinterpret_cast<float4*>(out.sh + i0 * 48);
    for (int c = tid; c < nblk * 12; c += kProjBwdThreads) {
        const int t = c / 12, q = c - 12 * t;
        dst[c] = sh_rows[12 * t + (q ^ sh_swizzle(t))];
    }
}

/* ---------------------------------------------------------------- K8 -- */

constexpr int kL1Blocks = 1024;

__global__ void __launch_bounds__(256)
l1_loss_kernel(const float* __restrict__ pred, const float* __restrict__ target, long long n,
               float* __restrict__ grad, float* __restrict__ partial) {
    chain_begin();
    __shared__ float ws[8];
    const float inv_n = 1.0f / (float)n;
    float sum = 0.0f;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float diff = pred[i] - target[i];
        /* loss.mojo:27-33: the diff >= 0 branch takes +1/n */
        if (diff >= 0.0f) { sum += diff; grad[i] = inv_n; }
        else { sum -= diff; grad[i] = -inv_n; }
    }
    sum = warp_sum(sum);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < 8; ++w) t += ws[w];
        partial[blockIdx.x] = t;
    }
}

__global__ void l1_finish_kernel(const float* __restrict__ partial, long long n, float* loss) {
    chain_begin();
    __shared__ float ws[32];
    float t = 0.0f;
    for (int b = threadIdx.x; b < kL1Blocks; b += blockDim.x) t += partial[b];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        float a = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += ws[w];
        *loss = n > 0 ? a * (1.0f / (float)n) : 0.0f;
    }
}

}  // namespace lumen

using namespace lumen;

namespace lumen {

/* Five 39.4 KB CTAs of the compositing adjoint per SM need the largest
 * shared-memory carveout; set per device by configure_once. */
void configure_backward_kernels() {
    cudaFuncSetAttribute(composite_backward_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
}

void configure_once();
LumenStatus check_inputs(const LumenGpuGaussians* g, const LumenViewCamera* cam, const LumenRenderOptions* opt);
LumenStatus map_cuda(cudaError_t e);
cudaEvent_t* stage_timer_take(LumenGpuStageTimer* t);

/* timer: a stage timer whose next frame receives five events (start,
 * after the compositing adjoint, then three after the projection adjoint),
 * taken once the arguments are valid; or nullptr. */
static LumenStatus backward_impl(const LumenGpuGaussians* g, const LumenViewCamera* cam,
                                 const LumenRenderOptions* opt, const LumenGpuFrame* f,
                                 const LumenGpuImage* fwd, const float* grad_rgb, const float* grad_depth,
                                 const float* grad_alpha, LumenGpuGradients* out, LumenGpuStageTimer* timer,
                                 void* stream) {
    LumenStatus st = check_inputs(g, cam, opt);
    if (st != LUMEN_SUCCESS) return st;
    if (!f || !f->scratch || !grad_rgb || !out || !fwd || !fwd->rgb || !fwd->alpha || !fwd->last_idx)
        return LUMEN_ERROR_INVALID_ARGUMENT;
    if (grad_depth && opt->compute_depth && !fwd->depth) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (g->count > 0 &&
        (!out->means || !out->scales || !out->quats || !out->opacities || !out->sh || !out->splat2d ||
         !f->records || !f->visible_ids || !f->radii || !f->ranges || !f->vals[0] || !f->vals[1] ||
         ((uintptr_t)out->splat2d & 15u) != 0))
        return LUMEN_ERROR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    configure_once();
    cudaEvent_t* ev = nullptr;
    if (timer && !(ev = stage_timer_take(timer))) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (g->count == 0) {
        if (ev)
            for (int k = 0; k < 5; ++k) cudaEventRecord(ev[k], s);
        return LUMEN_SUCCESS;
    }
    Control* ctrl = (Control*)f->scratch;
    if (ev) cudaEventRecord(ev[0], s);
    cudaError_t e = cudaMemsetAsync(out->splat2d, 0, (size_t)g->count * kGrad2DStride * sizeof(float), s);
    if (e != cudaSuccess) return map_cuda(e);
    const int tiles_x = (cam->width + kTile - 1) / kTile;
    const int tiles = tiles_x * ((cam->height + kTile - 1) / kTile);
    launch_chained(composite_backward_kernel, dim3(tiles), dim3(kTilePixels), 0, s,
                   (const LumenSplatRecord*)f->records, *f, ctrl, cam->width, cam->height, tiles_x, *opt,
                   (const float*)fwd->rgb, (const float*)fwd->depth, (const float*)fwd->alpha,
                   (const int*)fwd->last_idx, grad_rgb, grad_depth, grad_alpha, out->splat2d);
    if (ev) cudaEventRecord(ev[1], s);
    const long long nb = (g->count + kProjBwdThreads - 1) / kProjBwdThreads;
    launch_chained(project_backward_kernel, dim3((unsigned int)nb), dim3(kProjBwdThreads), kProjBwdStageBytes, s,
                   *g, *cam, *opt, (const int*)f->radii, (const float*)out->splat2d, *out);
    if (ev)
        for (int k = 2; k < 5; ++k) cudaEventRecord(ev[k], s);
    return map_cuda(cudaGetLastError());
}
}  // namespace lumen

extern "C" {

LumenStatus lumen_gpu_render_backward(const LumenGpuGaussians* g, const LumenViewCamera* cam,
                                      const LumenRenderOptions* opt, const LumenGpuFrame* f,
                                      const LumenGpuImage* fwd, const float* grad_rgb, const float* grad_depth,
                                      const float* grad_alpha, LumenGpuGradients* out, void* stream) {
    return backward_impl(g, cam, opt, f, fwd, grad_rgb, grad_depth, grad_alpha, out, nullptr, stream);
}

LumenStatus lumen_gpu_render_backward_timed(const LumenGpuGaussians* g, const LumenViewCamera* cam,
                                            const LumenRenderOptions* opt, const LumenGpuFrame* f,
                                            const LumenGpuImage* fwd, const float* grad_rgb, const float* grad_depth,
                                            const float* grad_alpha, LumenGpuGradients* out,
                                            LumenGpuStageTimer* timer, void* stream) {
    if (!timer) return LUMEN_ERROR_INVALID_ARGUMENT;
    return backward_impl(g, cam, opt, f, fwd, grad_rgb, grad_depth, grad_alpha, out, timer, stream);
}

size_t lumen_gpu_l1_loss_scratch_bytes(void) { return (size_t)kL1Blocks * sizeof(float); }

LumenStatus lumen_gpu_l1_loss(const float* pred, const float* target, int64_t n, float* grad, float* loss,
                              void* scratch, void* stream) {
    if (n < 0 || !loss || !scratch || (n > 0 && (!pred || !target || !grad))) return LUMEN_ERROR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    float* partial = (float*)scratch;
    if (n > 0) {
        launch_chained(l1_loss_kernel, dim3(kL1Blocks), dim3(256), 0, s, pred, target, (long long)n, grad, partial);
    } else {
        cudaMemsetAsync(partial, 0, lumen_gpu_l1_loss_scratch_bytes(), s);
    }
    launch_chained(l1_finish_kernel, dim3(1), dim3(256), 0, s, (const float*)partial, (long long)n, loss);
    return map_cuda(cudaGetLastError());
}

}  // extern "C"
