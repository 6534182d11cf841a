"""The training step's device kernels (include/lumen_train.h) against the CPU
restatement of the reference's optimizer, density control and loss code:
bit-exact for Adam, density control, opacity reset and view-space
accumulation; PSNR within 1e-3 dB (its sum is reduced in a different order
from the reference's sequential float sum). Then the Trainer: a few steps of
real training lower the loss, and a scheduled densification changes the
count by clones + splits - prunes and restarts the accumulators."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from lumen_b200 import _lib as L
from lumen_b200 import render as R
from lumen_b200 import scenes
from lumen_b200.types import RenderOptions

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _stream():
    return torch.cuda.current_stream().cuda_stream


def test_adam_matches_restatement():
    lib = L.load()
    rng = np.random.default_rng(0)
    n = 100_003
    means = rng.normal(size=(n, 3)).astype(np.float32)
    op = rng.uniform(0.0, 1.0, n).astype(np.float32)
    cfg = lib.lumen_training_default_config()
    cfg.iterations = 50
    dm, dop = _t(means), _t(op)
    mom = [torch.zeros((n, 3), device="cuda"), torch.zeros((n, 3), device="cuda"), torch.zeros(n, device="cuda"),
           torch.zeros(n, device="cuda")]
    st = L.LumenAdamState()
    st.m_pos, st.v_pos, st.m_opacity, st.v_opacity = (m.data_ptr() for m in mom)
    hm = [np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32)]
    for step in range(1, 4):
        gm = rng.normal(size=(n, 3)).astype(np.float32) * np.float32(10 ** -step)
        gop = rng.normal(size=n).astype(np.float32)
        g = L.LumenGpuGaussians()
        g.means, g.opacities, g.count = dm.data_ptr(), dop.data_ptr(), n
        tgm, tgop = _t(gm), _t(gop)       # held until the kernel has run
        L.check(lib.lumen_gpu_adam_step(C.byref(g), tgm.data_ptr(), tgop.data_ptr(), C.byref(st),
                                        C.byref(cfg), _stream()), "adam")
        lr = O.position_lr(cfg.position_lr_init, cfg.position_lr_final, cfg.iterations, step)
        O.adam_step(means, op, gm, gop, *hm, pos_lr=lr, opacity_lr=cfg.opacity_lr, step=step)
        assert st.step == step
        assert np.array_equal(dm.cpu().numpy(), means) and np.array_equal(dop.cpu().numpy(), op)
        for a, b in zip(mom, hm):
            assert np.array_equal(a.cpu().numpy(), b)


def test_densify_matches_restatement():
    lib = L.load()
    rng = np.random.default_rng(1)
    n = 50_001
    means = rng.normal(size=(n, 3)).astype(np.float32)
    scales = np.exp(rng.uniform(np.log(0.01), np.log(8.0), (n, 3))).astype(np.float32)
    quats = rng.normal(size=(n, 4)).astype(np.float32)
    quats[::97] = 0.0
    op = rng.uniform(0.0, 1.0, n).astype(np.float32)
    op[::13] = 0.001
    sh = rng.normal(size=(n, 48)).astype(np.float32)
    vs_sum = rng.uniform(0, 0.01, n).astype(np.float32)
    vs_cnt = rng.integers(0, 20, n).astype(np.int32)
    mom = {k: rng.normal(size=s).astype(np.float32) for k, s in
           (("m_pos", (n, 3)), ("v_pos", (n, 3)), ("m_op", (n,)), ("v_op", (n,)))}
    cfg = lib.lumen_training_default_config()
    extent = 12.0
    want, want_m, want_stats = O.densify_and_prune(means, scales, quats, op, sh, vs_sum, vs_cnt,
                                                   cfg.densify_grad_threshold, cfg.prune_opacity_threshold,
                                                   extent, moments=mom)
    src_t = [_t(a) for a in (means, scales, quats, op, sh)]
    dst_t = [torch.empty((2 * n,) + a.shape[1:], device="cuda") for a in (means, scales, quats, op, sh)]
    src, dst = R.gaussians_struct(*src_t), R.gaussians_struct(*dst_t)
    dst.count = 2 * n
    sm_t = [_t(mom[k]) for k in ("m_pos", "v_pos", "m_op", "v_op")]
    dm_t = [torch.empty((2 * n,) + m.shape[1:], device="cuda") for m in sm_t]
    sm, dm = L.LumenAdamState(), L.LumenAdamState()
    sm.m_pos, sm.v_pos, sm.m_opacity, sm.v_opacity = (m.data_ptr() for m in sm_t)
    dm.m_pos, dm.v_pos, dm.m_opacity, dm.v_opacity = (m.data_ptr() for m in dm_t)
    scratch = torch.empty(int(lib.lumen_gpu_densify_scratch_bytes(n)), dtype=torch.uint8, device="cuda")
    stats = L.LumenDensifyStats()
    tvs, tvc = _t(vs_sum), _t(vs_cnt)     # held until the kernel has run
    L.check(lib.lumen_gpu_densify_and_prune(C.byref(src), tvs.data_ptr(), tvc.data_ptr(),
                                            C.byref(cfg), extent, C.byref(dst), C.byref(sm), C.byref(dm),
                                            scratch.data_ptr(), scratch.numel(), C.byref(stats), _stream()),
            "densify")
    k = int(stats.count)
    assert (stats.cloned, stats.split, stats.pruned) == want_stats
    assert k == want["means"].shape[0] and 0 < want_stats[0] and 0 < want_stats[1] and 0 < want_stats[2]
    for t, name in zip(dst_t, ("means", "scales", "quats", "opacities", "sh")):
        assert np.array_equal(t[:k].cpu().numpy(), want[name].reshape(t[:k].shape)), name
    for t, name in zip(dm_t, ("m_pos", "v_pos", "m_op", "v_op")):
        assert np.array_equal(t[:k].cpu().numpy(), want_m[name]), name


def test_reset_accumulate_and_psnr():
    lib = L.load()
    rng = np.random.default_rng(2)
    n = 70_000
    op = rng.uniform(0, 0.05, n).astype(np.float32)
    dop = _t(op)
    L.check(lib.lumen_gpu_reset_opacities(dop.data_ptr(), n, 0.01, _stream()), "reset")
    O.reset_opacities(op, 0.01)
    assert np.array_equal(dop.cpu().numpy(), op)
    g2d = rng.normal(size=(n, 12)).astype(np.float32)
    radii = rng.integers(-1, 3, n).astype(np.int32)
    s0, c0 = rng.uniform(0, 1, n).astype(np.float32), rng.integers(0, 5, n).astype(np.int32)
    ds, dc = _t(s0.copy()), _t(c0.copy())
    tg2d, trad = _t(g2d), _t(radii)
    L.check(lib.lumen_gpu_accumulate_viewspace(tg2d.data_ptr(), 12, trad.data_ptr(), n, 960.0, 540.0,
                                               ds.data_ptr(), dc.data_ptr(), _stream()), "accumulate")
    O.accumulate_viewspace(g2d, 12, radii, s0, c0, 960.0, 540.0)
    assert np.array_equal(ds.cpu().numpy(), s0) and np.array_equal(dc.cpu().numpy(), c0)
    a = rng.uniform(0, 1, (96, 128, 3)).astype(np.float32)
    b = (a + rng.normal(0, 0.05, a.shape)).astype(np.float32)
    out = torch.zeros((), device="cuda")
    scratch = torch.empty(int(lib.lumen_gpu_l1_loss_scratch_bytes()), dtype=torch.uint8, device="cuda")
    ta, tb = _t(a), _t(b)
    L.check(lib.lumen_gpu_psnr(ta.data_ptr(), tb.data_ptr(), a.size, out.data_ptr(), scratch.data_ptr(),
                               _stream()), "psnr")
    assert float(out.item()) == pytest.approx(O.psnr(a, b), abs=1e-3)


def test_trainer_lowers_the_loss_and_densifies():
    from lumen_b200 import train as T
    sc = scenes.box_scene(20_000, seed=31)
    s, op = sc.activated()
    tg = scenes.perturbed(sc, seed=32)
    ts, top = tg.activated()
    cam = scenes.camera_config1(320, 180)
    opt = RenderOptions(term_mode=1)
    target = R.render(_t(tg.means), _t(ts), _t(tg.quats), _t(top), _t(tg.sh.reshape(-1, 48)), cam, opt).rgb
    cfg = T.default_config()
    cfg.iterations, cfg.densify_from_iter, cfg.densification_interval = 100, 6, 6
    cfg.opacity_lr = 0.01
    cfg.densify_grad_threshold = 1e-5     # low enough that a handful of steps densify
    tr = T.Trainer(sc.means, s, sc.quats, op, sc.sh.reshape(-1, 48), config=cfg, options=opt, scene_extent=6.0)
    losses = []
    for it in range(1, 6):
        m = tr.train_step(cam, target, it)
        losses.append(m.loss)
        assert m.splat_count == 20_000 and 0.0 < m.psnr < 99.0
    assert losses[-1] < losses[0]
    assert tr.vs_count.max().item() == 5
    # step 6 is scheduled for density control (its parity with the
    # restatement is checked on its own above)
    m = tr.train_step(cam, target, 6)
    assert m.cloned + m.split > 0
    assert m.splat_count == 20_000 + m.cloned + m.split - m.pruned
    assert tr.vs_sum.abs().max().item() == 0.0 and tr.params[0].shape[0] == m.splat_count
    assert tr.moments[0].shape[0] == m.splat_count
    m = tr.train_step(cam, target, 7)
    assert m.splat_count == tr.count and np.isfinite(m.loss)
