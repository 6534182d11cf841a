/*
 * train_oracle.cpp - CPU restatement of the reference's training-step pieces
 * (TEST INFRASTRUCTURE ONLY: the checker for lumen_b200/csrc/train.cu).
 *
 *   oracle_position_lr       AdamOptimizer.get_position_lr, src/optim/optimizer.mojo:106-113
 *   oracle_adam_scalars      the bias corrections of AdamOptimizer.step, optimizer.mojo:123-131
 *   oracle_adam_step         AdamOptimizer.step per Gaussian, optimizer.mojo:133-170
 *                            (beta1 0.9, beta2 0.999, epsilon 1e-8: optimizer.mojo:74-76)
 *   oracle_densify_and_prune densify_and_prune, src/optim/density_control.mojo:25-99,
 *                            with get_average_viewspace_grad, src/optim/gradients.mojo:101-106
 *                            (outputs built through Gaussian3D, which normalises the
 *                            rotation, src/scene/gaussian.mojo:27-37, quaternion.mojo:52-57)
 *   oracle_reset_opacities   reset_opacities, density_control.mojo:102-109
 *   oracle_psnr              compute_mse_loss + compute_psnr, src/optim/loss.mojo:38-60
 *   oracle_accumulate_viewspace
 *                            GaussianGradients.accumulate_viewspace_grad, gradients.mojo:96-99,
 *                            given the norm of the scaled screen-centre gradient
 *
 * Literal float32 arithmetic in the reference's operation order,
 * (float)(double literal) constants, no contraction (-ffp-contract=off).
 * Where the reference leaves behaviour undefined (its optimizer keeps the
 * moment arrays of the original cloud after densification), the
 * restatement follows the product's documented rule: moments follow their
 * Gaussian (copied to both children, dropped with a pruned one).
 */
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

struct Quat { float w, x, y, z; };

Quat normalized(Quat q) {                                  /* quaternion.mojo:52-57 */
    const float ns = q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z;
    const float n = std::sqrt(ns);
    if (n > (float)0.000001) {
        const float inv_n = 1.0f / n;
        return {q.w * inv_n, q.x * inv_n, q.y * inv_n, q.z * inv_n};
    }
    return {1.0f, 0.0f, 0.0f, 0.0f};
}

struct Out {
    float *means, *scales, *quats, *op, *sh;
    const float *m_pos, *v_pos, *m_op, *v_op;
    float *dm_pos, *dv_pos, *dm_op, *dv_op;
};

/* GaussianCloud.add_gaussian(Gaussian3D(pos, scale, rot, op), sh), with the
 * source's moments carried along. */
void add(const Out& o, int64_t k, int64_t src, const float pos[3], const float scl[3], Quat r, float op,
         const float* sh48) {
    for (int c = 0; c < 3; ++c) {
        o.means[k * 3 + c] = pos[c];
        o.scales[k * 3 + c] = scl[c];
    }
    o.quats[k * 4 + 0] = r.w;
    o.quats[k * 4 + 1] = r.x;
    o.quats[k * 4 + 2] = r.y;
    o.quats[k * 4 + 3] = r.z;
    o.op[k] = op;
    std::memcpy(o.sh + k * 48, sh48, 48 * sizeof(float));
    if (o.m_pos && o.dm_pos) for (int c = 0; c < 3; ++c) o.dm_pos[k * 3 + c] = o.m_pos[src * 3 + c];
    if (o.v_pos && o.dv_pos) for (int c = 0; c < 3; ++c) o.dv_pos[k * 3 + c] = o.v_pos[src * 3 + c];
    if (o.m_op && o.dm_op) o.dm_op[k] = o.m_op[src];
    if (o.v_op && o.dv_op) o.dv_op[k] = o.v_op[src];
}

}  // namespace

extern "C" {

float oracle_position_lr(float init, float final_lr, int32_t iterations, int64_t iteration) {
    float progress = (float)iteration / (float)iterations;
    if (progress > 1.0f) progress = 1.0f;
    const float ratio = final_lr / init;
    return init * std::pow(ratio, progress);
}

void oracle_adam_scalars(float beta1, float beta2, int64_t step, float* inv_b1, float* inv_b2) {
    const float t = (float)step;
    const float beta1_t = std::pow(beta1, t);
    const float beta2_t = std::pow(beta2, t);
    *inv_b1 = 1.0f / (1.0f - beta1_t);
    *inv_b2 = 1.0f / (1.0f - beta2_t);
}

void oracle_adam_step(float* means, float* op, const float* gm, const float* gop, float* m_pos, float* v_pos,
                      float* m_op, float* v_op, int64_t n, float pos_lr, float opacity_lr, float beta1,
                      float beta2, float eps, float inv_b1, float inv_b2) {
    for (int64_t i = 0; i < n; ++i) {
        for (int c = 0; c < 3; ++c) {
            const int64_t j = i * 3 + c;
            const float g = gm[j];
            m_pos[j] = beta1 * m_pos[j] + (1.0f - beta1) * g;
            v_pos[j] = beta2 * v_pos[j] + (1.0f - beta2) * g * g;
            const float m_hat = m_pos[j] * inv_b1;
            const float v_hat = v_pos[j] * inv_b2;
            means[j] -= pos_lr * m_hat / (std::sqrt(v_hat) + eps);
        }
        const float g = gop[i];
        m_op[i] = beta1 * m_op[i] + (1.0f - beta1) * g;
        v_op[i] = beta2 * v_op[i] + (1.0f - beta2) * g * g;
        const float m_hat = m_op[i] * inv_b1;
        const float v_hat = v_op[i] * inv_b2;
        float new_op = op[i] - opacity_lr * m_hat / (std::sqrt(v_hat) + eps);
        if (new_op < (float)0.01) new_op = (float)0.01;
        else if (new_op > (float)0.99) new_op = (float)0.99;
        op[i] = new_op;
    }
}

/* Returns the number of Gaussians written (capacity 2n). */
int64_t oracle_densify_and_prune(const float* means, const float* scales, const float* quats, const float* op,
                                 const float* sh, const float* vs_sum, const int32_t* vs_count, int64_t n,
                                 float grad_thr, float prune_thr, float scene_extent,
                                 float* o_means, float* o_scales, float* o_quats, float* o_op, float* o_sh,
                                 const float* m_pos, const float* v_pos, const float* m_op, const float* v_op,
                                 float* dm_pos, float* dv_pos, float* dm_op, float* dv_op,
                                 int64_t* cloned, int64_t* split, int64_t* pruned) {
    *cloned = *split = *pruned = 0;
    const Out o{o_means, o_scales, o_quats, o_op, o_sh, m_pos, v_pos, m_op, v_op, dm_pos, dv_pos, dm_op, dv_op};
    const float scale_threshold = scene_extent * (float)0.01;
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
        const float opacity = op[i];
        if (opacity < prune_thr) { ++*pruned; continue; }
        const float pos[3] = {means[i * 3], means[i * 3 + 1], means[i * 3 + 2]};
        const float scl[3] = {scales[i * 3], scales[i * 3 + 1], scales[i * 3 + 2]};
        const Quat rot = normalized({quats[i * 4], quats[i * 4 + 1], quats[i * 4 + 2], quats[i * 4 + 3]});
        float max_scale = scl[0];
        if (scl[1] > max_scale) max_scale = scl[1];
        if (scl[2] > max_scale) max_scale = scl[2];
        if (max_scale > scene_extent * 0.5f) { ++*pruned; continue; }
        float avg = 0.0f;
        if (vs_count[i] > 0) avg = vs_sum[i] / (float)vs_count[i];
        const float* s48 = sh + i * 48;
        if (avg > grad_thr) {
            if (max_scale <= scale_threshold) {
                ++*cloned;
                add(o, k++, i, pos, scl, rot, opacity, s48);
                const float off[3] = {pos[0] + (float)0.01 * scl[0], pos[1] + (float)0.01 * scl[1],
                                      pos[2] + (float)0.01 * scl[2]};
                add(o, k++, i, off, scl, rot, opacity, s48);
            } else {
                ++*split;
                const float ns[3] = {scl[0] / (float)1.6, scl[1] / (float)1.6, scl[2] / (float)1.6};
                const float p1[3] = {pos[0] + ns[0] * 0.5f, pos[1] + ns[1] * 0.5f, pos[2] + ns[2] * 0.5f};
                const float p2[3] = {pos[0] - ns[0] * 0.5f, pos[1] - ns[1] * 0.5f, pos[2] - ns[2] * 0.5f};
                add(o, k++, i, p1, ns, rot, opacity, s48);
                add(o, k++, i, p2, ns, rot, opacity, s48);
            }
        } else {
            add(o, k++, i, pos, scl, rot, opacity, s48);
        }
    }
    return k;
}

void oracle_reset_opacities(float* op, int64_t n, float max_value) {
    for (int64_t i = 0; i < n; ++i)
        if (op[i] > max_value) op[i] = max_value;
}

float oracle_psnr(const float* pred, const float* target, int64_t n) {
    if (n == 0) return (float)99.99;        /* compute_mse_loss returns 0 for n == 0 */
    float sum_sq = 0.0f;
    for (int64_t i = 0; i < n; ++i) {
        const float d = pred[i] - target[i];
        sum_sq += d * d;
    }
    const float mse = sum_sq / (float)n;
    if (mse < (float)1e-10) return (float)99.99;
    return (float)-4.3429448 * std::log(mse);
}

void oracle_accumulate_viewspace(const float* grad2d, int32_t stride, const int32_t* radii, int64_t n,
                                 float scale_x, float scale_y, float* sum, int32_t* count) {
    for (int64_t i = 0; i < n; ++i) {
        if (radii[i] <= 0) continue;
        const float gx = grad2d[i * stride] * scale_x, gy = grad2d[i * stride + 1] * scale_y;
        sum[i] += std::sqrt(gx * gx + gy * gy);
        count[i] += 1;
    }
}

}  // extern "C"
