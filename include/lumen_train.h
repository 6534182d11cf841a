/*
 * lumen_train.h - the training step around the adjoint, as device kernels.
 *
 * Reference (paths relative to the reference project):
 *   lumen_training_default_config  TrainingConfig, src/core/config.mojo:114-164
 *   lumen_training_should_densify  TrainingConfig.should_densify, config.mojo:166-169
 *   lumen_training_should_reset_opacity
 *                                  TrainingConfig.should_reset_opacity, config.mojo:171-174
 *   lumen_gpu_adam_step            AdamOptimizer.get_position_lr + step,
 *                                  src/optim/optimizer.mojo:106-170: positions with an
 *                                  exponentially decaying rate, opacity clamped to
 *                                  [0.01, 0.99]; the reference updates no other
 *                                  parameter group
 *   lumen_gpu_accumulate_viewspace GaussianGradients.accumulate_viewspace_grad,
 *                                  src/optim/gradients.mojo:96-99, fed with the norm of
 *                                  the screen-centre gradient from the backward
 *   lumen_gpu_densify_and_prune    densify_and_prune, src/optim/density_control.mojo:25-99
 *                                  (with get_average_viewspace_grad, gradients.mojo:101-106)
 *   lumen_gpu_reset_opacities      reset_opacities, density_control.mojo:102-109
 *   lumen_gpu_psnr                 compute_mse_loss + compute_psnr, src/optim/loss.mojo:38-60
 * The reference's training step (src/optim/trainer.mojo:38-76) injects
 * placeholder gradients; here the gradients come from lumen_gpu_render_backward.
 *
 * Parameters are the reference's stored values: linear scales and opacities
 * (render and differentiate with params_are_logits = 0).
 */
#ifndef LUMEN_TRAIN_H
#define LUMEN_TRAIN_H

#include "lumen_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t iterations;
    float position_lr_init, position_lr_final;
    float feature_lr, opacity_lr, scaling_lr, rotation_lr, lambda_dssim;
    int32_t densify_from_iter, densify_until_iter, densification_interval, opacity_reset_interval;
    float densify_grad_threshold, prune_opacity_threshold, max_screen_size_ratio;
} LumenTrainingConfig;

/* The reference's defaults (30000 iterations, position rate 1.6e-4 -> 1.6e-6,
 * opacity rate 0.05, densify every 100 iterations in [500, 15000], opacity
 * reset every 3000, gradient threshold 2e-4, prune below opacity 0.005). */
LumenTrainingConfig lumen_training_default_config(void);
int32_t lumen_training_should_densify(const LumenTrainingConfig* config, int64_t iteration);
int32_t lumen_training_should_reset_opacity(const LumenTrainingConfig* config, int64_t iteration);

/* First and second Adam moments of the updated parameter groups (device
 * float32: m_pos/v_pos N x 3, m_opacity/v_opacity N), zero-initialised by
 * the caller, and the step counter. */
typedef struct {
    float* m_pos;
    float* v_pos;
    float* m_opacity;
    float* v_opacity;
    int64_t step;
} LumenAdamState;

/* One Adam step on gaussians->means and gaussians->opacities in place (the
 * other groups are left as they are, as in the reference). state->step is
 * incremented first (optimizer.mojo:123); the position rate and the bias
 * corrections are computed on the host in float32 with powf. */
LumenStatus lumen_gpu_adam_step(LumenGpuGaussians* gaussians, const float* grad_means, const float* grad_opacities,
                                LumenAdamState* state, const LumenTrainingConfig* config, void* stream);

/* For every Gaussian with radii[i] > 0: sum[i] += |(scale_x * g_x, scale_y * g_y)|
 * and count[i] += 1, where (g_x, g_y) are the first two floats of its splat2d
 * row (stride floats per row): the gradient with respect to the screen centre
 * in pixels. scale_x = width / 2 and scale_y = height / 2 express it in
 * normalised device units, the units densify_grad_threshold is given in. */
LumenStatus lumen_gpu_accumulate_viewspace(const float* splat2d, int32_t stride, const int32_t* radii, int64_t n,
                                           float scale_x, float scale_y, float* sum, int32_t* count, void* stream);

typedef struct {
    int64_t cloned, split, pruned;
    int64_t count;      /* Gaussians written to dst */
} LumenDensifyStats;

/* Density control: src's N Gaussians are written to dst (capacity
 * dst->count >= 2N) in the reference's order: pruned ones dropped (opacity
 * below the threshold, or largest scale above extent / 2), clones followed
 * by their offset copy, splits as their two halves, the rest unchanged;
 * every output rotation normalised (Gaussian3D, src/scene/gaussian.mojo:27-37).
 * When src_moments and dst_moments are given, each output Gaussian carries
 * its source's Adam moments. Synchronises the stream to read the counts;
 * dst->count is set to the number written. scratch: device memory of
 * lumen_gpu_densify_scratch_bytes(N) bytes. quats and sh 16-byte aligned. */
size_t lumen_gpu_densify_scratch_bytes(int64_t n);
LumenStatus lumen_gpu_densify_and_prune(const LumenGpuGaussians* src, const float* vs_sum, const int32_t* vs_count,
                                        const LumenTrainingConfig* config, float scene_extent, LumenGpuGaussians* dst,
                                        const LumenAdamState* src_moments, LumenAdamState* dst_moments,
                                        void* scratch, size_t scratch_bytes, LumenDensifyStats* stats, void* stream);

/* opacities[i] = min(opacities[i], max_value) */
LumenStatus lumen_gpu_reset_opacities(float* opacities, int64_t n, float max_value, void* stream);

/* PSNR in dB of pred against target (n floats each) into *psnr (device);
 * 99.99 when the mean squared error is below 1e-10. scratch: device memory
 * of lumen_gpu_l1_loss_scratch_bytes() bytes. */
LumenStatus lumen_gpu_psnr(const float* pred, const float* target, int64_t n, float* psnr, void* scratch,
                           void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LUMEN_TRAIN_H */
