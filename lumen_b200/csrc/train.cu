/*
 * train.cu - the training step's device kernels (include/lumen_train.h).
 *
 * Reference: AdamOptimizer.step (src/optim/optimizer.mojo:106-170),
 * densify_and_prune / reset_opacities (src/optim/density_control.mojo:25-109),
 * GaussianGradients viewspace accumulation (src/optim/gradients.mojo:96-106),
 * compute_mse_loss / compute_psnr (src/optim/loss.mojo:38-60), TrainingConfig
 * (src/core/config.mojo:114-174).
 *
 * The per-Gaussian arithmetic follows the reference's operation order in
 * float32 (built with --fmad=false); the step's scalars (position rate, bias
 * corrections) are computed once on the host with powf, as the CPU
 * restatement does, so updates agree bit for bit. Density control runs as one
 * ticket-ordered kernel: each block decides every Gaussian's outputs (0 when
 * pruned, 1 kept, 2 cloned or split), scans the counts, resolves its offset
 * by decoupled look-back and writes the outputs in the reference's order.
 *
 * Memory: Adam reads and writes 16 B of parameters, 16 B of gradients and
 * 32 B of moments per Gaussian; density control reads 236 B (+ 32 B of
 * moments) and writes up to twice that per Gaussian.
 */
#include <cmath>
#include <cstring>

#include "splat_common.cuh"
#include "../../include/lumen_train.h"

namespace lumen {
LumenStatus map_cuda(cudaError_t e);
int device_sm_count();

namespace {

constexpr int kTrainThreads = 256;
constexpr int kPsnrBlocks = 1024;   /* partial sums; fits the L1 loss scratch */

__global__ void __launch_bounds__(256)
adam_kernel(float* __restrict__ means, float* __restrict__ opac, const float* __restrict__ gm,
            const float* __restrict__ gop, float* __restrict__ m_pos, float* __restrict__ v_pos,
            float* __restrict__ m_op, float* __restrict__ v_op, long long n, float pos_lr, float opacity_lr,
            float b1, float b2, float eps, float ib1, float ib2) {
    chain_begin();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {                         /* optimizer.mojo:135-157 */
            const long long j = i * 3 + k;
            const float g = gm[j];
            const float m = b1 * m_pos[j] + (1.0f - b1) * g;
            const float v = b2 * v_pos[j] + (1.0f - b2) * g * g;
            m_pos[j] = m;
            v_pos[j] = v;
            const float m_hat = m * ib1;
            const float v_hat = v * ib2;
            means[j] = means[j] - pos_lr * m_hat / (sqrtf(v_hat) + eps);
        }
        const float g = gop[i];                               /* optimizer.mojo:159-170 */
        const float m = b1 * m_op[i] + (1.0f - b1) * g;
        const float v = b2 * v_op[i] + (1.0f - b2) * g * g;
        m_op[i] = m;
        v_op[i] = v;
        const float m_hat = m * ib1;
        const float v_hat = v * ib2;
        float new_op = opac[i] - opacity_lr * m_hat / (sqrtf(v_hat) + eps);
        if (new_op < (float)0.01) new_op = (float)0.01;
        else if (new_op > (float)0.99) new_op = (float)0.99;
        opac[i] = new_op;
    }
}

__global__ void __launch_bounds__(256)
viewspace_kernel(const float* __restrict__ g2d, int stride_f, const int* __restrict__ radii, long long n,
                 float sx, float sy, float* __restrict__ sum, int* __restrict__ count) {
    chain_begin();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (radii[i] <= 0) continue;
        const float gx = g2d[i * stride_f] * sx, gy = g2d[i * stride_f + 1] * sy;
        sum[i] += sqrtf(gx * gx + gy * gy);
        count[i] += 1;
    }
}

__global__ void reset_kernel(float* __restrict__ op, long long n, float max_value) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (op[i] > max_value) op[i] = max_value;
}

__global__ void __launch_bounds__(256)
sq_diff_kernel(const float* __restrict__ pred, const float* __restrict__ target, long long n,
               float* __restrict__ partial) {
    chain_begin();
    __shared__ float ws[8];
    float sum = 0.0f;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float d = pred[i] - target[i];
        sum += d * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < 8; ++w) t += ws[w];
        partial[blockIdx.x] = t;
    }
}

/* One warp: each lane sums a strided share of the partials, then a fixed
 * butterfly (the same order on every call, so the result is deterministic). */
__global__ void psnr_finish_kernel(const float* __restrict__ partial, int nparts, long long n, float* psnr) {
    chain_begin();
    float s = 0.0f;
    for (int b = threadIdx.x; b < nparts; b += 32) s += partial[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x != 0) return;
    const float mse = s / (float)n;                           /* loss.mojo:38-48 */
    *psnr = mse < (float)1e-10 ? (float)99.99 : (float)-4.3429448 * logf(mse);   /* loss.mojo:51-60 */
}

/* ---------------------------------------------------------------- density control */

struct DensifyControl {
    unsigned long long n_out;
    unsigned long long cloned, split, pruned;
    unsigned int ticket;
    unsigned int error_flags;
};

struct DensifyParams {
    const float* means; const float* scales; const float* quats; const float* opac; const float* sh;
    const float* vs_sum; const int* vs_count;
    float* d_means; float* d_scales; float* d_quats; float* d_opac; float* d_sh;
    const float* m_pos; const float* v_pos; const float* m_op; const float* v_op;
    float* dm_pos; float* dv_pos; float* dm_op; float* dv_op;
    long long n;
    float grad_thr, prune_thr, extent;
};

struct DensifySmem {
    unsigned int blk;
    unsigned int warp_tot[kTrainThreads / 32];
    unsigned long long base;
    unsigned int counts[3];
};

__device__ __forceinline__ void densify_emit(const DensifyParams& P, long long i, long long out, const float pos[3],
                                             const float scl[3], const float q[4], float op) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        P.d_means[out * 3 + k] = pos[k];
        P.d_scales[out * 3 + k] = scl[k];
    }
    reinterpret_cast<float4*>(P.d_quats)[out] = make_float4(q[0], q[1], q[2], q[3]);
    P.d_opac[out] = op;
    const float4* src = reinterpret_cast<const float4*>(P.sh + i * 48);
    float4* dst = reinterpret_cast<float4*>(P.d_sh + out * 48);
#pragma unroll
    for (int k = 0; k < 12; ++k) dst[k] = src[k];
    if (P.m_pos && P.dm_pos)
        for (int k = 0; k < 3; ++k) P.dm_pos[out * 3 + k] = P.m_pos[i * 3 + k];
    if (P.v_pos && P.dv_pos)
        for (int k = 0; k < 3; ++k) P.dv_pos[out * 3 + k] = P.v_pos[i * 3 + k];
    if (P.m_op && P.dm_op) P.dm_op[out] = P.m_op[i];
    if (P.v_op && P.dv_op) P.dv_op[out] = P.v_op[i];
}

__global__ void __launch_bounds__(kTrainThreads)
densify_kernel(DensifyParams P, DensifyControl* ctrl, unsigned long long* lb) {
    __shared__ DensifySmem s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s.blk = atomicAdd(&ctrl->ticket, 1u);
        s.counts[0] = s.counts[1] = s.counts[2] = 0u;
    }
    __syncthreads();
    const int blk = (int)s.blk;
    const long long i = (long long)blk * kTrainThreads + tid;
    /* 0 pruned, 1 kept, 2 cloned, 3 split (density_control.mojo:45-96) */
    int action = 0;
    float pos[3] = {0, 0, 0}, scl[3] = {0, 0, 0}, q[4] = {1, 0, 0, 0}, op = 0.0f;
    if (i < P.n) {
        op = P.opac[i];
        for (int k = 0; k < 3; ++k) { pos[k] = P.means[i * 3 + k]; scl[k] = P.scales[i * 3 + k]; }
        const float4 q4 = reinterpret_cast<const float4*>(P.quats)[i];
        const Quat r = q_normalized(Quat{q4.x, q4.y, q4.z, q4.w});   /* Gaussian3D, gaussian.mojo:35 */
        q[0] = r.w; q[1] = r.x; q[2] = r.y; q[3] = r.z;
        float max_scale = scl[0];
        if (scl[1] > max_scale) max_scale = scl[1];
        if (scl[2] > max_scale) max_scale = scl[2];
        if (op < P.prune_thr || max_scale > P.extent * 0.5f) {
            action = 0;
        } else {
            float avg = 0.0f;                                            /* gradients.mojo:101-106 */
            const int c = P.vs_count[i];
            if (c > 0) avg = P.vs_sum[i] / (float)c;
            if (avg > P.grad_thr) action = max_scale <= P.extent * (float)0.01 ? 2 : 3;
            else action = 1;
        }
    }
    const unsigned int cnt = action == 0 ? 0u : action == 1 ? 1u : 2u;
    if (i < P.n) {
        if (action == 0) atomicAdd(&s.counts[2], 1u);
        else if (action == 2) atomicAdd(&s.counts[0], 1u);
        else if (action == 3) atomicAdd(&s.counts[1], 1u);
    }
    unsigned int block_out = 0;
    const unsigned int excl = block_exclusive_scan<kTrainThreads>(cnt, s.warp_tot, &block_out);
    if (tid == 0) st_volatile_u64(lb + blk, (blk == 0 ? kDescIncl64 : kDescAgg64) | block_out);
    if (warp == 0) {
        const unsigned long long e = blk > 0 ? lookback64(lb, blk, &ctrl->error_flags) : 0ull;
        if (lane == 0) {
            s.base = e;
            if (blk > 0) st_volatile_u64(lb + blk, kDescIncl64 | (e + block_out));
        }
    }
    __syncthreads();
    const long long out = (long long)(s.base + excl);
    if (action == 1) {
        densify_emit(P, i, out, pos, scl, q, op);
    } else if (action == 2) {                                            /* clone, :72-80 */
        densify_emit(P, i, out, pos, scl, q, op);
        const float off[3] = {pos[0] + (float)0.01 * scl[0], pos[1] + (float)0.01 * scl[1],
                              pos[2] + (float)0.01 * scl[2]};
        densify_emit(P, i, out + 1, off, scl, q, op);
    } else if (action == 3) {                                            /* split, :81-90 */
        const float ns[3] = {scl[0] / (float)1.6, scl[1] / (float)1.6, scl[2] / (float)1.6};
        const float p1[3] = {pos[0] + ns[0] * 0.5f, pos[1] + ns[1] * 0.5f, pos[2] + ns[2] * 0.5f};
        const float p2[3] = {pos[0] - ns[0] * 0.5f, pos[1] - ns[1] * 0.5f, pos[2] - ns[2] * 0.5f};
        densify_emit(P, i, out, p1, ns, q, op);
        densify_emit(P, i, out + 1, p2, ns, q, op);
    }
    __syncthreads();
    if (tid == 0) {
        if (s.counts[0]) atomicAdd(&ctrl->cloned, (unsigned long long)s.counts[0]);
        if (s.counts[1]) atomicAdd(&ctrl->split, (unsigned long long)s.counts[1]);
        if (s.counts[2]) atomicAdd(&ctrl->pruned, (unsigned long long)s.counts[2]);
        if ((long long)blk == (P.n - 1) / kTrainThreads) ctrl->n_out = s.base + block_out;
    }
}

size_t densify_scratch(int64_t n) {
    const int64_t blocks = (n + kTrainThreads - 1) / kTrainThreads;
    return align_up(sizeof(DensifyControl), 256) + (size_t)(blocks > 0 ? blocks : 1) * sizeof(unsigned long long);
}

int grid_for(long long n) {
    long long g = (n + 255) / 256;
    const long long cap = (long long)device_sm_count() * 8;
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace
}  // namespace lumen

using namespace lumen;

extern "C" {

LumenTrainingConfig lumen_training_default_config(void) {
    LumenTrainingConfig c;
    c.iterations = 30000;
    c.position_lr_init = (float)0.00016;
    c.position_lr_final = (float)0.0000016;
    c.feature_lr = (float)0.0025;
    c.opacity_lr = (float)0.05;
    c.scaling_lr = (float)0.005;
    c.rotation_lr = (float)0.001;
    c.lambda_dssim = (float)0.2;
    c.densify_from_iter = 500;
    c.densify_until_iter = 15000;
    c.densification_interval = 100;
    c.opacity_reset_interval = 3000;
    c.densify_grad_threshold = (float)0.0002;
    c.prune_opacity_threshold = (float)0.005;
    c.max_screen_size_ratio = (float)20.0;
    return c;
}

int32_t lumen_training_should_densify(const LumenTrainingConfig* c, int64_t it) {
    if (!c || c->densification_interval <= 0) return 0;
    if (it >= c->densify_from_iter && it <= c->densify_until_iter) return (it % c->densification_interval) == 0;
    return 0;
}

int32_t lumen_training_should_reset_opacity(const LumenTrainingConfig* c, int64_t it) {
    if (!c || c->opacity_reset_interval <= 0) return 0;
    if (it > 0 && it <= c->densify_until_iter) return (it % c->opacity_reset_interval) == 0;
    return 0;
}

LumenStatus lumen_gpu_adam_step(LumenGpuGaussians* g, const float* grad_means, const float* grad_op,
                                LumenAdamState* st, const LumenTrainingConfig* c, void* stream) {
    if (!g || !st || !c || c->iterations <= 0 || g->count < 0) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (g->count > 0 && (!g->means || !g->opacities || !grad_means || !grad_op || !st->m_pos || !st->v_pos ||
                         !st->m_opacity || !st->v_opacity))
        return LUMEN_ERROR_INVALID_ARGUMENT;
    st->step += 1;
    /* get_position_lr and the bias corrections (optimizer.mojo:106-131) */
    float progress = (float)st->step / (float)c->iterations;
    if (progress > 1.0f) progress = 1.0f;
    const float pos_lr = c->position_lr_init * powf(c->position_lr_final / c->position_lr_init, progress);
    const float b1 = 0.9f, b2 = 0.999f, eps = (float)1e-8;
    const float t = (float)st->step;
    const float ib1 = 1.0f / (1.0f - powf(b1, t));
    const float ib2 = 1.0f / (1.0f - powf(b2, t));
    if (g->count == 0) return LUMEN_SUCCESS;
    launch_chained(adam_kernel, dim3(grid_for(g->count)), dim3(256), 0, (cudaStream_t)stream,
                   const_cast<float*>(g->means), const_cast<float*>(g->opacities), grad_means, grad_op, st->m_pos,
                   st->v_pos, st->m_opacity, st->v_opacity, (long long)g->count, pos_lr, c->opacity_lr, b1, b2, eps,
                   ib1, ib2);
    return map_cuda(cudaGetLastError());
}

LumenStatus lumen_gpu_accumulate_viewspace(const float* splat2d, int32_t stride, const int32_t* radii, int64_t n,
                                           float scale_x, float scale_y, float* sum, int32_t* count, void* stream) {
    if (n < 0 || stride < 2) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (n == 0) return LUMEN_SUCCESS;
    if (!splat2d || !radii || !sum || !count) return LUMEN_ERROR_INVALID_ARGUMENT;
    launch_chained(viewspace_kernel, dim3(grid_for(n)), dim3(256), 0, (cudaStream_t)stream, splat2d, (int)stride,
                   (const int*)radii, (long long)n, scale_x, scale_y, sum, (int*)count);
    return map_cuda(cudaGetLastError());
}

size_t lumen_gpu_densify_scratch_bytes(int64_t n) { return n < 0 ? 0 : densify_scratch(n); }

LumenStatus lumen_gpu_densify_and_prune(const LumenGpuGaussians* src, const float* vs_sum, const int32_t* vs_count,
                                        const LumenTrainingConfig* c, float extent, LumenGpuGaussians* dst,
                                        const LumenAdamState* sm, LumenAdamState* dm, void* scratch,
                                        size_t scratch_bytes, LumenDensifyStats* stats, void* stream) {
    if (!src || !dst || !c || !stats || src->count < 0 || src->count >= (1ll << 30)) return LUMEN_ERROR_INVALID_ARGUMENT;
    std::memset(stats, 0, sizeof(*stats));
    const long long n = src->count;
    if (n == 0) { dst->count = 0; return LUMEN_SUCCESS; }
    if (dst->count < 2 * n || !vs_sum || !vs_count || !scratch || scratch_bytes < densify_scratch(n))
        return LUMEN_ERROR_INVALID_ARGUMENT;
    const LumenGpuGaussians& a = *src;
    if (!a.means || !a.scales || !a.quats || !a.opacities || !a.sh || !dst->means || !dst->scales || !dst->quats ||
        !dst->opacities || !dst->sh)
        return LUMEN_ERROR_INVALID_ARGUMENT;
    if (((uintptr_t)a.quats | (uintptr_t)a.sh | (uintptr_t)dst->quats | (uintptr_t)dst->sh) & 15u)
        return LUMEN_ERROR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    DensifyParams P;
    std::memset(&P, 0, sizeof(P));
    P.means = a.means; P.scales = a.scales; P.quats = a.quats; P.opac = a.opacities; P.sh = a.sh;
    P.vs_sum = vs_sum; P.vs_count = vs_count;
    P.d_means = const_cast<float*>(dst->means); P.d_scales = const_cast<float*>(dst->scales);
    P.d_quats = const_cast<float*>(dst->quats); P.d_opac = const_cast<float*>(dst->opacities);
    P.d_sh = const_cast<float*>(dst->sh);
    if (sm && dm) {
        P.m_pos = sm->m_pos; P.v_pos = sm->v_pos; P.m_op = sm->m_opacity; P.v_op = sm->v_opacity;
        P.dm_pos = dm->m_pos; P.dv_pos = dm->v_pos; P.dm_op = dm->m_opacity; P.dv_op = dm->v_opacity;
    }
    P.n = n;
    P.grad_thr = c->densify_grad_threshold;
    P.prune_thr = c->prune_opacity_threshold;
    P.extent = extent;
    DensifyControl* ctrl = (DensifyControl*)scratch;
    unsigned long long* lb = (unsigned long long*)((unsigned char*)scratch + align_up(sizeof(DensifyControl), 256));
    cudaError_t e = cudaMemsetAsync(scratch, 0, densify_scratch(n), s);
    if (e != cudaSuccess) return map_cuda(e);
    const long long blocks = (n + kTrainThreads - 1) / kTrainThreads;
    densify_kernel<<<(unsigned int)blocks, kTrainThreads, 0, s>>>(P, ctrl, lb);
    if ((e = cudaGetLastError()) != cudaSuccess) return map_cuda(e);
    DensifyControl h;
    if ((e = cudaMemcpyAsync(&h, ctrl, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return map_cuda(e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return map_cuda(e);
    if (h.error_flags) return LUMEN_ERROR_IO_FAILURE;
    stats->cloned = (int64_t)h.cloned;
    stats->split = (int64_t)h.split;
    stats->pruned = (int64_t)h.pruned;
    stats->count = (int64_t)h.n_out;
    dst->count = (int64_t)h.n_out;
    if (sm && dm) dm->step = sm->step;
    return LUMEN_SUCCESS;
}

LumenStatus lumen_gpu_reset_opacities(float* op, int64_t n, float max_value, void* stream) {
    if (n < 0 || (n > 0 && !op)) return LUMEN_ERROR_INVALID_ARGUMENT;
    if (n == 0) return LUMEN_SUCCESS;
    reset_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(op, n, max_value);
    return map_cuda(cudaGetLastError());
}

LumenStatus lumen_gpu_psnr(const float* pred, const float* target, int64_t n, float* psnr, void* scratch,
                           void* stream) {
    if (n <= 0 || !pred || !target || !psnr || !scratch) return LUMEN_ERROR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    float* partial = (float*)scratch;
    launch_chained(sq_diff_kernel, dim3(kPsnrBlocks), dim3(256), 0, s, pred, target, (long long)n, partial);
    launch_chained(psnr_finish_kernel, dim3(1), dim3(32), 0, s, (const float*)partial, (int)kPsnrBlocks, (long long)n,
                   psnr);
    return map_cuda(cudaGetLastError());
}

}  // extern "C"
