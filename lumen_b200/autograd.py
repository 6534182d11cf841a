"""Differentiable render: a torch.autograd.Function over the C ABI.

``render(means, log_scales, quats, opacity_logits, sh, camera, options)``
returns (rgb [H,W,3], depth [H,W], alpha [H,W]); its backward is the
hand-written CUDA adjoint (lumen_gpu_render_backward): per-tile
transmittance recomputed in the backward (front to back, up to each pixel's
last-visited splat, from the forward's outputs), then the chain rule through the
compositing, the conic, EWA, the projective Jacobian, Sigma = R S S^T R^T,
the quaternion normalisation, degree-3 SH and the exp / sigmoid activations.
It returns dL/d(means, log-scales, quats, opacity logits, SH).

``l1_loss(pred, target)`` is compute_l1_loss (src/optim/loss.mojo:11-35)
as an autograd function: mean |pred - target| with subgradient +-1/n
(+1/n where pred == target).

The reference has no analytic backward (src/optim/gradients.mojo stores
gradient buffers; src/optim/trainer.mojo:61-66 injects placeholders).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import torch

from . import _lib as L
from . import render as R
from .types import RenderOptions, ViewCamera


class _RenderFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, log_scales, quats, opacity_logits, sh, camera: ViewCamera, options: RenderOptions):
        opt = options.with_(params_are_logits=True)
        n = means.shape[0]
        tensors = [t.detach().contiguous().float() for t in (means, log_scales, quats, opacity_logits)]
        sh_flat = sh.detach().contiguous().float().reshape(n, 48)
        res = R.render(tensors[0], tensors[1], tensors[2], tensors[3].reshape(n), sh_flat, camera, opt)
        ctx.camera, ctx.options, ctx.frame = camera, opt, res.frame
        ctx.sh_shape = sh.shape
        ctx.save_for_backward(tensors[0], tensors[1], tensors[2], tensors[3].reshape(n), sh_flat, res.rgb, res.depth,
                              res.alpha, res.last_idx)
        ctx.mark_non_differentiable(res.last_idx)
        return res.rgb, res.depth, res.alpha

    @staticmethod
    def backward(ctx, g_rgb, g_depth, g_alpha):
        means, log_scales, quats, logits, sh, rgb, depth, alpha, last_idx = ctx.saved_tensors
        n = means.shape[0]
        dev = means.device
        lib = L.load()
        grads = [torch.empty_like(means), torch.empty_like(log_scales), torch.empty_like(quats),
                 torch.empty_like(logits), torch.empty_like(sh)]
        if n == 0:
            return grads[0], grads[1], grads[2], grads[3], grads[4].reshape(ctx.sh_shape), None, None
        splat2d = torch.empty((n, 12), dtype=torch.float32, device=dev)
        out = L.LumenGpuGradients()
        out.means, out.scales, out.quats, out.opacities, out.sh = (g.data_ptr() for g in grads)
        out.splat2d = splat2d.data_ptr()
        g = R.gaussians_struct(means, log_scales, quats, logits, sh)
        cam, opt = L.view_camera(ctx.camera), L.render_options(ctx.options)
        fs = ctx.frame.c_struct()
        g_rgb = g_rgb.contiguous().float() if g_rgb is not None else torch.zeros(
            (ctx.camera.height, ctx.camera.width, 3), device=dev)
        g_depth = g_depth.contiguous().float() if g_depth is not None else None
        g_alpha = g_alpha.contiguous().float() if g_alpha is not None else None
        fwd = L.LumenGpuImage()
        fwd.rgb, fwd.depth, fwd.alpha = rgb.data_ptr(), depth.data_ptr(), alpha.data_ptr()
        fwd.last_idx = last_idx.data_ptr()
        L.check(lib.lumen_gpu_render_backward(C.byref(g), C.byref(cam), C.byref(opt), C.byref(fs), C.byref(fwd),
                                              g_rgb.data_ptr(),
                                              None if g_depth is None else g_depth.data_ptr(),
                                              None if g_alpha is None else g_alpha.data_ptr(), C.byref(out),
                                              torch.cuda.current_stream(dev).cuda_stream), "render_backward")
        return grads[0], grads[1], grads[2], grads[3].reshape(logits.shape), grads[4].reshape(ctx.sh_shape), None, None


def render(means: torch.Tensor, log_scales: torch.Tensor, quats: torch.Tensor, opacity_logits: torch.Tensor,
           sh: torch.Tensor, camera: ViewCamera, options: Optional[RenderOptions] = None
           ) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """Differentiable forward render: (rgb, depth, alpha)."""
    return _RenderFunction.apply(means, log_scales, quats, opacity_logits, sh, camera, options or RenderOptions())


class _L1Function(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pred, target):
        lib = L.load()
        p = pred.detach().contiguous().float()
        t = target.detach().contiguous().float()
        grad = torch.empty_like(p)
        loss = torch.empty((), dtype=torch.float32, device=p.device)
        scratch = torch.empty(int(lib.lumen_gpu_l1_loss_scratch_bytes()), dtype=torch.uint8, device=p.device)
        L.check(lib.lumen_gpu_l1_loss(p.data_ptr(), t.data_ptr(), p.numel(), grad.data_ptr(), loss.data_ptr(),
                                      scratch.data_ptr(), torch.cuda.current_stream(p.device).cuda_stream), "l1_loss")
        ctx.save_for_backward(grad)
        return loss

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return grad * g, None


def l1_loss(pred: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
    """Mean L1 loss with the reference's subgradient (loss.mojo:11-35)."""
    return _L1Function.apply(pred, target)


def smoke_backward() -> None:
    """One small forward + backward on cuda:0: gradients finite and non-zero."""
    from . import scenes
    sc = scenes.grid_scene(0)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(a).to(dev).requires_grad_(True)
    params = [t(sc.means), t(sc.log_scales), t(sc.quats), t(sc.opacity_logits), t(sc.sh)]
    rgb, depth, alpha = render(*params, scenes.camera_config0(), RenderOptions())
    target = torch.full_like(rgb, 0.5)
    loss = l1_loss(rgb, target)
    loss.backward()
    for p in params:
        assert torch.isfinite(p.grad).all()
    assert float(params[0].grad.abs().sum()) > 0 and float(params[4].grad.abs().sum()) > 0
