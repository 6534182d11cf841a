"""Training step around the adjoint (include/lumen_train.h).

``Trainer.train_step(camera, ground_truth, iteration)`` is the reference's
TrainingCoordinator.train_step (src/optim/trainer.mojo:38-76) on the device
with real gradients where the reference injects placeholders:

1. forward render (rasterize_scene, pipeline.mojo:48-231),
2. L1 loss and PSNR (loss.mojo:11-60),
3. the hand-written backward (lumen_gpu_render_backward),
4. Adam on positions and opacity (optimizer.mojo:106-170),
5. view-space gradient accumulation (gradients.mojo:96-99), in normalised
   device units (the screen-centre gradient times width/2 and height/2),
6. densify_and_prune when config.should_densify(iteration)
   (density_control.mojo:25-99; moments follow their Gaussian, the
   accumulators restart), reset_opacities when should_reset_opacity.

Parameters are the reference's stored values (linear scales and opacity).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _lib as L
from . import render as R
from .types import RenderOptions, ViewCamera


@dataclass
class TrainingMetrics:
    iteration: int
    loss: float
    psnr: float
    splat_count: int
    cloned: int = 0
    split: int = 0
    pruned: int = 0


def default_config() -> L.LumenTrainingConfig:
    return L.load().lumen_training_default_config()


class Trainer:
    """Owns the cloud's parameters, the Adam moments and the view-space
    accumulators on one device."""

    def __init__(self, means, scales, quats, opacities, sh, config: Optional[L.LumenTrainingConfig] = None,
                 options: Optional[RenderOptions] = None, scene_extent: float = 1.0, device="cuda"):
        self.lib = L.load()
        self.dev = torch.device(device)
        self.config = config or default_config()
        self.options = (options or RenderOptions()).with_(params_are_logits=False)
        self.scene_extent = float(scene_extent)
        t = lambda a, shape: torch.as_tensor(np.asarray(a, np.float32)).reshape(shape).to(self.dev).contiguous()
        n = int(np.asarray(means).shape[0])
        self.params = [t(means, (n, 3)), t(scales, (n, 3)), t(quats, (n, 4)), t(opacities, (n,)), t(sh, (n, 48))]
        self.step_count = 0
        self._reset_state(n)
        self.frame = None
        self.capacity = 0
        self.image = None
        self.l1_scratch = torch.empty(int(self.lib.lumen_gpu_l1_loss_scratch_bytes()), dtype=torch.uint8,
                                      device=self.dev)
        self.psnr_scratch = torch.empty_like(self.l1_scratch)
        self.metrics_dev = torch.zeros(2, device=self.dev)              # loss, PSNR
        self.metrics_host = torch.zeros(2).pin_memory() if torch.cuda.is_available() else torch.zeros(2)
        self.last_densify_ms = 0.0

    def _reset_state(self, n: int, moments=None):
        z = lambda *s: torch.zeros(s, dtype=torch.float32, device=self.dev)
        self.moments = moments if moments is not None else [z(n, 3), z(n, 3), z(n), z(n)]
        self.vs_sum = z(n)
        self.vs_count = torch.zeros(n, dtype=torch.int32, device=self.dev)
        self.grads = [torch.empty_like(p) for p in self.params]
        self.splat2d = torch.empty((max(n, 1), 12), dtype=torch.float32, device=self.dev)

    @property
    def count(self) -> int:
        return int(self.params[0].shape[0])

    def _gaussians(self) -> L.LumenGpuGaussians:
        return R.gaussians_struct(*self.params)

    @staticmethod
    def _adam_state(moments, step) -> L.LumenAdamState:
        s = L.LumenAdamState()
        s.m_pos, s.v_pos, s.m_opacity, s.v_opacity = (m.data_ptr() for m in moments)
        s.step = step
        return s

    def _images(self, h: int, w: int):
        if self.image is None or self.image[0].shape[:2] != (h, w):
            e = lambda *s: torch.empty(s, dtype=torch.float32, device=self.dev)
            self.image = (e(h, w, 3), e(h, w), e(h, w), e(h, w, 3),        # rgb, depth, alpha, dL/drgb,
                          torch.empty((h, w), dtype=torch.int32, device=self.dev))   # last-visited splat
        return self.image

    def train_step(self, camera: ViewCamera, ground_truth: torch.Tensor, iteration: int) -> TrainingMetrics:
        """One step with a single host wait: the forward, loss, PSNR and
        backward are enqueued, then the instance count, loss and PSNR are read
        together; if the frame outgrew its instance buffers nothing has been
        updated yet, so the buffers grow and the step is enqueued again.
        Adam, the accumulation and the scheduled density control follow
        without another wait (density control reads its counts back)."""
        lib, dev = self.lib, self.dev
        stream = torch.cuda.current_stream(dev).cuda_stream
        n = self.count
        gt = ground_truth.to(dev).float().contiguous()
        H, W = int(camera.height), int(camera.width)
        if gt.numel() != H * W * 3:
            raise L.LumenError(-1, "train_step: ground truth does not match the camera's image size")
        rgb, depth, alpha, gimg, last = self._images(H, W)
        g = self._gaussians()
        cam, opt = L.view_camera(camera), L.render_options(self.options)
        img = L.LumenGpuImage()
        img.rgb, img.depth, img.alpha = rgb.data_ptr(), depth.data_ptr(), alpha.data_ptr()
        img.last_idx = last.data_ptr()
        out = L.LumenGpuGradients()
        out.means, out.scales, out.quats, out.opacities, out.sh = (t.data_ptr() for t in self.grads)
        out.splat2d = self.splat2d.data_ptr()
        tiles = camera.n_tiles
        counts = L.LumenGpuCounts()
        for _ in range(2):
            cap = self.capacity or max(1 << 16, 8 * n)
            if self.frame is None or not self.frame.fits(n, tiles) or self.frame.capacity < cap:
                self.frame = R.Frame.allocate(n, tiles, cap, dev)
            fs = self.frame.c_struct()
            # 1. forward, 2. L1 loss and PSNR, 3. backward
            L.check(lib.lumen_gpu_render_forward(C.byref(g), C.byref(cam), C.byref(opt), C.byref(fs), C.byref(img),
                                                 stream), "render_forward")
            L.check(lib.lumen_gpu_l1_loss(rgb.data_ptr(), gt.data_ptr(), rgb.numel(), gimg.data_ptr(),
                                          self.metrics_dev.data_ptr(), self.l1_scratch.data_ptr(), stream), "l1_loss")
            L.check(lib.lumen_gpu_psnr(rgb.data_ptr(), gt.data_ptr(), rgb.numel(), self.metrics_dev.data_ptr() + 4,
                                       self.psnr_scratch.data_ptr(), stream), "psnr")
            L.check(lib.lumen_gpu_render_backward(C.byref(g), C.byref(cam), C.byref(opt), C.byref(fs), C.byref(img),
                                                  gimg.data_ptr(), None, None, C.byref(out), stream), "backward")
            self.metrics_host.copy_(self.metrics_dev, non_blocking=True)
            L.check(lib.lumen_gpu_read_counts(C.byref(fs), C.byref(counts), stream), "read_counts")   # the wait
            if not counts.error_flags & L.ERR_CAPACITY:
                break
            need = int(counts.n_instances)
            self.capacity = need + need // 4 + 4096
        if counts.error_flags:
            raise L.LumenError(-4 if not counts.error_flags & L.ERR_CAPACITY else -2,
                               f"train_step device flags {counts.error_flags:#x}")
        self.capacity = max(self.capacity, self.frame.capacity)
        # 4. Adam on positions and opacity
        st = self._adam_state(self.moments, self.step_count)
        cfg = self.config
        L.check(lib.lumen_gpu_adam_step(C.byref(g), self.grads[0].data_ptr(), self.grads[3].data_ptr(),
                                        C.byref(st), C.byref(cfg), stream), "adam_step")
        self.step_count = int(st.step)
        # 5. view-space gradients of the visible Gaussians
        L.check(lib.lumen_gpu_accumulate_viewspace(self.splat2d.data_ptr(), 12, self.frame.radii.data_ptr(), n,
                                                   0.5 * camera.width, 0.5 * camera.height,
                                                   self.vs_sum.data_ptr(), self.vs_count.data_ptr(), stream),
                "accumulate_viewspace")
        metrics = TrainingMetrics(iteration, float(self.metrics_host[0]), float(self.metrics_host[1]), n)
        # 6. density control and opacity reset
        if lib.lumen_training_should_densify(C.byref(cfg), iteration):
            metrics.cloned, metrics.split, metrics.pruned = self.densify_and_prune()
        if lib.lumen_training_should_reset_opacity(C.byref(cfg), iteration):
            L.check(lib.lumen_gpu_reset_opacities(self.params[3].data_ptr(), self.count, 0.01, stream), "reset")
        metrics.splat_count = self.count
        return metrics

    def densify_and_prune(self):
        """Density control over the accumulated view-space gradients; returns
        (cloned, split, pruned). last_densify_ms: the device time of the
        density-control call itself."""
        lib, dev = self.lib, self.dev
        stream = torch.cuda.current_stream(dev)
        n = self.count
        cap = 2 * max(n, 1)
        z = lambda *s: torch.empty(s, dtype=torch.float32, device=dev)
        new = [z(cap, 3), z(cap, 3), z(cap, 4), z(cap), z(cap, 48)]
        new_m = [z(cap, 3), z(cap, 3), z(cap), z(cap)]
        dst = R.gaussians_struct(*new)
        src = self._gaussians()
        sm, dm = self._adam_state(self.moments, self.step_count), self._adam_state(new_m, self.step_count)
        scratch = torch.empty(int(lib.lumen_gpu_densify_scratch_bytes(n)), dtype=torch.uint8, device=dev)
        stats = L.LumenDensifyStats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        L.check(lib.lumen_gpu_densify_and_prune(C.byref(src), self.vs_sum.data_ptr(), self.vs_count.data_ptr(),
                                                C.byref(self.config), self.scene_extent, C.byref(dst), C.byref(sm),
                                                C.byref(dm), scratch.data_ptr(), scratch.numel(), C.byref(stats),
                                                stream.cuda_stream), "densify_and_prune")
        e1.record(stream)
        e1.synchronize()
        self.last_densify_ms = float(e0.elapsed_time(e1))
        k = int(stats.count)
        self.params = [p[:k].contiguous() for p in new]
        self._reset_state(k, [m[:k].contiguous() for m in new_m])
        self.frame = None
        return int(stats.cloned), int(stats.split), int(stats.pruned)
