"""The hand-written backward against central finite differences of the
float64 oracle forward, and the L1 loss kernel against the reference's KAT.

Loss used for the gradient checks: L = sum(Wc * rgb) + sum(Wd * depth) +
sum(Wa * alpha) with seeded random weights, so dL/d(image) = W. For a random
subset of parameters of every group, fd = (L(p + eps) - L(p - eps)) / (2 eps)
in float64. A parameter is skipped when the perturbation changes any discrete
decision of the forward (visibility, radius, tile rectangle, SH clamps, sort
order, which pixel/splat pairs pass the 4.5 cutoff, the 1/255 skip, the 0.99
clamp or the termination) - the oracle hashes all of them - because the
loss is not differentiable across those. Tolerance: relative error
||g - fd|| / ||fd|| <= 1e-3 per parameter group.
"""
import numpy as np
import pytest

import oracle as O
from lumen_b200 import scenes
from lumen_b200.types import RenderOptions, ViewCamera

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_TOL = 1e-3


def _loss64(params, cam, opt, W):
    rgb, depth, alpha, h = O.render_f64(params["means"], params["log_scales"], params["quats"],
                                        params["logits"], params["sh"], cam, opt)
    return float((W["rgb"] * rgb).sum() + (W["depth"] * depth).sum() + (W["alpha"] * alpha).sum()), h


def _gpu_grads(params, cam, opt, W):
    from lumen_b200 import autograd as A
    t = {k: torch.from_numpy(np.ascontiguousarray(v, np.float32)).cuda().requires_grad_(True)
         for k, v in params.items()}
    rgb, depth, alpha = A.render(t["means"], t["log_scales"], t["quats"], t["logits"], t["sh"], cam, opt)
    loss = (rgb * torch.from_numpy(W["rgb"]).cuda().float()).sum() + \
        (depth * torch.from_numpy(W["depth"]).cuda().float()).sum() + \
        (alpha * torch.from_numpy(W["alpha"]).cuda().float()).sum()
    loss.backward()
    return {k: v.grad.cpu().numpy().astype(np.float64) for k, v in t.items()}


def _check(params, cam, opt, per_group=48, eps=1e-5, seed=0, min_checked=12):
    rng = np.random.default_rng(seed)
    H, W_ = cam.height, cam.width
    W = {"rgb": rng.normal(size=(H, W_, 3)), "depth": rng.normal(size=(H, W_)) * 0.05,
         "alpha": rng.normal(size=(H, W_))}
    p64 = {k: np.asarray(v, np.float64) for k, v in params.items()}
    g = _gpu_grads(params, cam, opt, W)
    _, h0 = _loss64(p64, cam, opt, W)
    report = {}
    for name in ("means", "log_scales", "quats", "logits", "sh"):
        arr = p64[name]
        flat_idx = rng.choice(arr.size, size=min(per_group, arr.size), replace=False)
        fd, gg = [], []
        for fi in flat_idx:
            idx = np.unravel_index(fi, arr.shape)
            plus, minus = {k: v.copy() for k, v in p64.items()}, {k: v.copy() for k, v in p64.items()}
            plus[name][idx] += eps
            minus[name][idx] -= eps
            lp, hp = _loss64(plus, cam, opt, W)
            lm, hm = _loss64(minus, cam, opt, W)
            if hp != h0 or hm != h0:
                continue   # the perturbation crosses a discontinuity of the forward
            fd.append((lp - lm) / (2 * eps))
            gg.append(g[name][idx])
        fd, gg = np.array(fd), np.array(gg)
        assert len(fd) >= min_checked, f"{name}: only {len(fd)} smooth parameters"
        nz = np.linalg.norm(fd)
        rel = np.linalg.norm(gg - fd) / nz if nz > 0 else np.linalg.norm(gg)
        report[name] = (rel, len(fd), nz)
    return report


def _assert_report(report):
    for name, (rel, n, nz) in report.items():
        assert nz > 0, f"{name}: all finite differences are zero"
        assert rel <= REL_TOL, f"{name}: relative error {rel:.2e} over {n} parameters"


def _config3_subset(n=2000, seed=3):
    sc = scenes.box_scene(500_000, seed=seed)
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(sc.n, size=n, replace=False))
    sub = sc.subset(idx)
    return {"means": sub.means, "log_scales": sub.log_scales, "quats": sub.quats, "logits": sub.opacity_logits,
            "sh": sub.sh.reshape(n, 48)}


def test_fd_config3_subset_128():
    """2k Gaussians drawn as configuration 3, 128x128, transmittance rule."""
    params = _config3_subset()
    cam = scenes.camera_config1(128, 128, fov=50.0)
    _assert_report(_check(params, cam, RenderOptions(params_are_logits=True)))


@pytest.mark.parametrize("term_mode,white", [(1, False), (0, True)])
def test_fd_dense_scene(term_mode, white):
    """2k larger Gaussians covering a 96x64 view densely, so most pixels
    blend many splats and terminate."""
    sc = scenes.box_scene(2000, seed=11, centre=(0.0, 0.0, 6.0))
    ls = sc.log_scales + np.float32(1.6)
    params = {"means": sc.means, "log_scales": ls, "quats": sc.quats, "logits": sc.opacity_logits + np.float32(1.0),
              "sh": sc.sh.reshape(-1, 48)}
    cam = ViewCamera.from_fov(96, 64, 60.0)
    opt = RenderOptions(params_are_logits=True, term_mode=term_mode, white_background=white)
    _assert_report(_check(params, cam, opt, seed=term_mode + 7))


def test_fd_sh_degrees():
    sc = scenes.box_scene(600, seed=5, centre=(0.0, 0.0, 5.0))
    params = {"means": sc.means, "log_scales": sc.log_scales + np.float32(1.2), "quats": sc.quats,
              "logits": sc.opacity_logits, "sh": sc.sh.reshape(-1, 48) * np.float32(3.0)}
    cam = ViewCamera.from_fov(64, 48, 60.0)
    for deg in (0, 1, 2):
        rep = _check(params, cam, RenderOptions(params_are_logits=True, sh_degree=deg), per_group=24, seed=deg,
                     min_checked=8)
        _assert_report(rep)


# ---- tests/test_loss.mojo:9-41 on the GPU ----
def test_l1_loss_kernel_known_answer():
    from lumen_b200.autograd import l1_loss
    pred = torch.tensor([0.8, 0.2, 0.5, 0.1], device="cuda", requires_grad=True)
    target = torch.tensor([0.5, 0.5, 0.5, 0.5], device="cuda")
    loss = l1_loss(pred, target)
    loss.backward()
    assert abs(loss.item() - 0.25) < 1e-6
    assert pred.grad.cpu().tolist() == [0.25, -0.25, 0.25, -0.25]
    z = torch.zeros(4, device="cuda", requires_grad=True)
    assert abs(l1_loss(z, torch.zeros(4, device="cuda")).item()) < 1e-7


def test_l1_loss_kernel_matches_oracle():
    from lumen_b200.autograd import l1_loss
    rng = np.random.default_rng(2)
    p = rng.random((270, 480, 3), dtype=np.float32)
    t = rng.random((270, 480, 3), dtype=np.float32)
    t.reshape(-1)[::97] = p.reshape(-1)[::97]   # exact ties take the + branch
    ref_loss, ref_grad = O.l1_loss(p, t)
    pt = torch.from_numpy(p).cuda().requires_grad_(True)
    loss = l1_loss(pt, torch.from_numpy(t).cuda())
    loss.backward()
    assert np.array_equal(pt.grad.cpu().numpy().reshape(-1), ref_grad)
    assert abs(loss.item() - ref_loss) <= 1e-6 * abs(ref_loss)
