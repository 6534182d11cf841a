"""The CPU restatement of the reference's training-step pieces (the checker
for the device kernels), on hand-computed cases, plus the host-side
schedule of the C ABI."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from lumen_b200 import _lib as L


def test_position_learning_rate_schedule():
    # AdamOptimizer.get_position_lr, optimizer.mojo:106-113
    init, final = np.float32(0.00016), np.float32(0.0000016)
    assert O.position_lr(init, final, 30000, 0) == pytest.approx(float(init), rel=1e-6)
    assert O.position_lr(init, final, 30000, 30000) == pytest.approx(float(final), rel=1e-5)
    assert O.position_lr(init, final, 30000, 60000) == pytest.approx(float(final), rel=1e-5)
    assert O.position_lr(init, final, 30000, 15000) == pytest.approx(float(np.sqrt(init * final)), rel=1e-5)


def test_first_adam_step_moves_by_the_rate():
    """After one step m_hat = g and v_hat = g^2: each coordinate moves by
    lr * g / (|g| + eps); opacity is clamped to [0.01, 0.99]."""
    n = 4
    means = np.zeros((n, 3), np.float32)
    op = np.array([0.5, 0.02, 0.985, 0.3], np.float32)
    gm = np.array([[1, -2, 0.5]] * n, np.float32)
    gop = np.array([1.0, 1.0, -1.0, 0.0], np.float32)
    m_pos, v_pos = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32)
    m_op, v_op = np.zeros(n, np.float32), np.zeros(n, np.float32)
    O.adam_step(means, op, gm, gop, m_pos, v_pos, m_op, v_op, pos_lr=0.01, opacity_lr=0.05, step=1)
    np.testing.assert_allclose(means, -0.01 * np.sign(gm), rtol=1e-5)
    np.testing.assert_allclose(m_pos, 0.1 * gm, rtol=1e-6)
    # (1 - beta2) rounds to 0.0010000467 in float32
    np.testing.assert_allclose(v_pos, (np.float32(1) - np.float32(0.999)) * gm * gm, rtol=1e-6)
    assert op[0] == pytest.approx(0.45, rel=1e-5)
    assert op[1] == np.float32(0.01)          # clamped low
    assert op[2] == np.float32(0.99)          # clamped high
    assert op[3] == np.float32(0.3)           # zero gradient leaves it


def _cloud(rows):
    """rows: (pos, scale, opacity, vs_sum, vs_count); identity rotations."""
    n = len(rows)
    means = np.array([r[0] for r in rows], np.float32)
    scales = np.array([r[1] for r in rows], np.float32)
    quats = np.tile(np.array([2.0, 0, 0, 0], np.float32), (n, 1))   # unnormalised on purpose
    op = np.array([r[2] for r in rows], np.float32)
    sh = np.arange(n * 48, dtype=np.float32).reshape(n, 48)
    return means, scales, quats, op, sh, np.array([r[3] for r in rows], np.float32), \
        np.array([r[4] for r in rows], np.int32)


def test_densify_and_prune_cases():
    extent = 10.0   # scale threshold 0.1, size limit 5.0
    rows = [((0, 0, 0), (0.05, 0.05, 0.05), 0.5, 0.01, 10),     # high grad, small: clone
            ((1, 1, 1), (0.5, 0.2, 0.3), 0.5, 0.01, 10),        # high grad, large: split
            ((2, 2, 2), (0.05, 0.05, 0.05), 0.001, 0.01, 10),   # transparent: prune
            ((3, 3, 3), (6.0, 0.1, 0.1), 0.5, 0.0, 0),          # larger than half the scene: prune
            ((4, 4, 4), (0.05, 0.05, 0.05), 0.5, 0.0001, 10),   # low grad: keep
            ((5, 5, 5), (0.05, 0.05, 0.05), 0.5, 0.0, 0)]       # never seen: keep
    means, scales, quats, op, sh, vs, vc = _cloud(rows)
    d, _, (cloned, split, pruned) = O.densify_and_prune(means, scales, quats, op, sh, vs, vc, 0.0002, 0.005, extent)
    assert (cloned, split, pruned) == (1, 1, 2)
    assert d["means"].shape[0] == 2 + 2 + 1 + 1
    f32 = np.float32
    np.testing.assert_array_equal(d["means"][0], means[0])
    np.testing.assert_array_equal(d["means"][1], means[0] + f32(0.01) * scales[0])
    ns = scales[1] / f32(1.6)
    np.testing.assert_array_equal(d["scales"][2], ns)
    np.testing.assert_array_equal(d["means"][2], means[1] + ns * f32(0.5))
    np.testing.assert_array_equal(d["means"][3], means[1] - ns * f32(0.5))
    np.testing.assert_array_equal(d["means"][4:6], means[4:6])
    np.testing.assert_array_equal(d["quats"], np.tile([1, 0, 0, 0], (6, 1)))   # normalised (gaussian.mojo:35)
    for out, src in ((0, 0), (1, 0), (2, 1), (3, 1), (4, 4), (5, 5)):
        np.testing.assert_array_equal(d["sh"][out], sh[src])


def test_moments_follow_their_gaussian():
    means, scales, quats, op, sh, vs, vc = _cloud([((0, 0, 0), (0.05,) * 3, 0.5, 0.01, 10),
                                                  ((1, 1, 1), (0.05,) * 3, 0.001, 0.0, 0),
                                                  ((2, 2, 2), (0.05,) * 3, 0.5, 0.0, 0)])
    mom = {"m_pos": np.arange(9, dtype=np.float32).reshape(3, 3), "v_pos": -np.arange(9, dtype=np.float32).reshape(3, 3),
           "m_op": np.array([1, 2, 3], np.float32), "v_op": np.array([4, 5, 6], np.float32)}
    d, dm, stats = O.densify_and_prune(means, scales, quats, op, sh, vs, vc, 0.0002, 0.005, 10.0, moments=mom)
    assert stats == (1, 0, 1)
    np.testing.assert_array_equal(dm["m_pos"], mom["m_pos"][[0, 0, 2]])
    np.testing.assert_array_equal(dm["v_op"], mom["v_op"][[0, 0, 2]])


def test_viewspace_accumulation_in_device_units():
    g2d = np.zeros((3, 12), np.float32)
    g2d[:, 0], g2d[:, 1] = [3e-4, 1.0, 2.0], [4e-4, 1.0, 2.0]
    radii = np.array([2, 0, 1], np.int32)
    s, c = np.zeros(3, np.float32), np.zeros(3, np.int32)
    O.accumulate_viewspace(g2d, 12, radii, s, c, 2.0, 2.0)
    np.testing.assert_allclose(s, [1e-3, 0.0, np.sqrt(32.0)], rtol=1e-6)
    np.testing.assert_array_equal(c, [1, 0, 1])


def test_reset_opacities_and_psnr():
    op = np.array([0.5, 0.005, 0.01, 0.02], np.float32)
    O.reset_opacities(op, 0.01)
    np.testing.assert_array_equal(op, np.array([0.01, 0.005, 0.01, 0.01], np.float32))
    a = np.full(300, 0.5, np.float32)
    assert O.psnr(a, a) == pytest.approx(99.99)
    b = a + np.float32(0.1)
    assert O.psnr(a, b) == pytest.approx(20.0, abs=1e-3)      # -10 log10(0.01)


def test_schedule_helpers():
    lib = L.load()
    c = lib.lumen_training_default_config()
    assert (c.iterations, c.densify_from_iter, c.densify_until_iter, c.densification_interval,
            c.opacity_reset_interval) == (30000, 500, 15000, 100, 3000)
    assert abs(c.densify_grad_threshold - 0.0002) < 1e-9 and abs(c.prune_opacity_threshold - 0.005) < 1e-9
    sd = lambda i: lib.lumen_training_should_densify(C.byref(c), i)
    sr = lambda i: lib.lumen_training_should_reset_opacity(C.byref(c), i)
    assert [sd(i) for i in (400, 500, 550, 600, 15000, 15100)] == [0, 1, 0, 1, 1, 0]
    assert [sr(i) for i in (0, 3000, 4500, 15000, 18000)] == [0, 1, 0, 1, 0]


def test_empty_inputs_and_argument_errors():
    """The C ABI's host-side paths for empty clouds and bad arguments (no
    device work is enqueued for these)."""
    lib = L.load()
    cfg = lib.lumen_training_default_config()
    g = L.LumenGpuGaussians()
    st = L.LumenAdamState()
    assert lib.lumen_gpu_adam_step(C.byref(g), None, None, C.byref(st), C.byref(cfg), None) == 0
    assert st.step == 1                                    # the counter advances even for an empty cloud
    assert lib.lumen_gpu_adam_step(None, None, None, C.byref(st), C.byref(cfg), None) == -1
    bad = lib.lumen_training_default_config()
    bad.iterations = 0
    assert lib.lumen_gpu_adam_step(C.byref(g), None, None, C.byref(st), C.byref(bad), None) == -1
    g.count = 5                                            # parameters missing
    assert lib.lumen_gpu_adam_step(C.byref(g), None, None, C.byref(st), C.byref(cfg), None) == -1
    assert lib.lumen_gpu_accumulate_viewspace(None, 12, None, 0, 1.0, 1.0, None, None, None) == 0
    assert lib.lumen_gpu_accumulate_viewspace(None, 1, None, 0, 1.0, 1.0, None, None, None) == -1
    assert lib.lumen_gpu_reset_opacities(None, 0, 0.01, None) == 0
    assert lib.lumen_gpu_reset_opacities(None, 3, 0.01, None) == -1
    assert lib.lumen_gpu_psnr(None, None, 0, None, None, None) == -1
    src, dst = L.LumenGpuGaussians(), L.LumenGpuGaussians()
    stats = L.LumenDensifyStats()
    assert lib.lumen_gpu_densify_and_prune(C.byref(src), None, None, C.byref(cfg), 1.0, C.byref(dst), None, None,
                                           None, 0, C.byref(stats), None) == 0
    assert dst.count == 0 and (stats.cloned, stats.split, stats.pruned, stats.count) == (0, 0, 0, 0)
    src.count = 4                                          # output capacity below 2N
    dst.count = 7
    assert lib.lumen_gpu_densify_and_prune(C.byref(src), None, None, C.byref(cfg), 1.0, C.byref(dst), None, None,
                                           None, 0, C.byref(stats), None) == -1
    assert lib.lumen_gpu_densify_scratch_bytes(-1) == 0 and lib.lumen_gpu_densify_scratch_bytes(1000) > 0
