"""GPU forward parity: the CUDA pipeline (through the C ABI) against the CPU
oracle on identical seeded inputs.

Bit-exact: visible counts, radii, projected records, sorted keys, sorted
values (permutation indices), tile ranges, per-pixel contributor counts and
last-visited indices. Images: max abs error <= 1e-4 per channel (the
north-star tolerance; in practice they agree bit for bit as well).
"""
import os

import numpy as np
import pytest

import oracle as O
from lumen_b200 import scenes
from lumen_b200.types import RenderOptions, ViewCamera

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

IMAGE_TOL = 1e-4
NT = max(1, min(16, os.cpu_count() or 1))


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def gpu_render(means, scales, quats, opac, sh, cam, opt, **kw):
    from lumen_b200 import render as R
    return R.render(_dev(means), _dev(scales), _dev(quats), _dev(opac).reshape(-1), _dev(sh).reshape(-1, 48),
                    cam, opt, **kw)


def assert_parity(g, o, check_image_bits=False):
    assert g.n_visible == o.n_visible
    assert g.n_instances == o.n_instances
    n = o.radii.shape[0]
    assert np.array_equal(g.frame.radii[:n].cpu().numpy(), o.radii)
    V, K = o.n_visible, o.n_instances
    if V:
        rec = g.records.cpu().numpy()
        ours = rec[:, [0, 1, 2, 4, 5, 6, 8, 9, 10, 3]].copy()
        ref = o.records.view(np.float32).reshape(V, 10)
        assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32)), "projected records differ"
        vis = g.frame.visible_ids[:V].cpu().numpy()
        assert np.array_equal(vis, np.nonzero(o.radii > 0)[0].astype(np.int32))
    if K:
        assert np.array_equal(g.sorted_keys.cpu().numpy().view(np.uint64), o.keys_sorted), "sorted keys differ"
        assert np.array_equal(g.sorted_vals.cpu().numpy().view(np.uint32), o.vals_sorted), "permutation differs"
    assert np.array_equal(g.ranges.cpu().numpy(), o.ranges), "tile ranges differ"
    assert np.array_equal(g.n_contrib.cpu().numpy().view(np.uint32), o.n_contrib), "contributor counts differ"
    assert np.array_equal(g.last_idx.cpu().numpy(), o.last_idx)
    for name in ("rgb", "depth", "alpha"):
        a, b = getattr(g, name).cpu().numpy(), getattr(o, name)
        err = float(np.abs(a - b).max()) if a.size else 0.0
        assert err <= IMAGE_TOL, f"{name} max abs err {err}"
        if check_image_bits:
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"{name} not bit-identical"


def run_both(means, scales, quats, opac, sh, cam, opt, **kw):
    o = O.render(means, scales, quats, opac, sh, cam, opt, nthreads=NT)
    g = gpu_render(means, scales, quats, opac, sh, cam, opt, **kw)
    return g, o


# ---- tests/test_rasterizer.mojo:15-71 on the GPU ----
def test_single_splat_known_answer():
    cam = ViewCamera((0, 0, 0), (1, 0, 0, 0), 50, 50, 32, 32, 0.1, 100, 64, 64)
    sh = np.zeros((1, 48), np.float32)
    sh[0, :3] = [1.77245, -1.77245, -1.77245]
    args = (np.array([[0, 0, 5]], np.float32), np.full((1, 3), 0.5, np.float32), np.array([[1, 0, 0, 0]], np.float32),
            np.ones(1, np.float32), sh, cam, RenderOptions())
    g, o = run_both(*args)
    assert g.n_visible == 1 and g.n_instances > 0
    c = g.rgb[32, 32].cpu().numpy()
    assert c[0] > 0.8 and c[1] < 0.2 and c[2] < 0.2
    assert np.allclose(g.rgb[0, 0].cpu().numpy(), 0, atol=1e-4)
    assert 4.5 < float(g.depth[32, 32]) < 5.5
    assert_parity(g, o, check_image_bits=True)


@pytest.mark.parametrize("term_mode", [0, 1])
@pytest.mark.parametrize("key_mode", [0, 1])
def test_grid_scene_parity(term_mode, key_mode):
    sc = scenes.grid_scene(0)
    s, op = sc.activated()
    opt = RenderOptions(term_mode=term_mode, key_mode=key_mode)
    g, o = run_both(sc.means, s, sc.quats, op, sc.sh, scenes.camera_config0(), opt)
    assert_parity(g, o, check_image_bits=True)


def test_grid_scene_logit_parameters():
    sc = scenes.grid_scene(0)
    opt = RenderOptions(params_are_logits=True)
    g, o = run_both(sc.means, sc.log_scales, sc.quats, sc.opacity_logits, sc.sh, scenes.camera_config0(), opt)
    assert_parity(g, o, check_image_bits=True)


@pytest.mark.parametrize("degree", [0, 1, 2, 3])
def test_options_background_depth_degree(degree):
    sc = scenes.box_scene(3000, seed=5, centre=(0, 0, 6))
    s, op = sc.activated()
    cam = ViewCamera.from_fov(200, 150, 55.0)
    opt = RenderOptions(sh_degree=degree, white_background=degree % 2 == 1, compute_depth=degree != 2)
    g, o = run_both(sc.means, s, sc.quats, op, sc.sh, cam, opt)
    assert_parity(g, o, check_image_bits=True)


@pytest.mark.parametrize("wh", [(1, 1), (17, 17), (100, 75), (333, 129)])
def test_ragged_resolutions_and_orbit_cameras(wh):
    sc = scenes.box_scene(5000, seed=11)
    s, op = sc.activated()
    for cam in scenes.orbit_cameras(3, wh[0], wh[1], fov=60.0, radius=9.0):
        g, o = run_both(sc.means, s, sc.quats, op, sc.sh, cam, RenderOptions())
        assert_parity(g, o, check_image_bits=True)


def test_empty_and_fully_culled():
    cam = ViewCamera((0, 0, 0), (1, 0, 0, 0), 20, 20, 16, 16, 0.1, 50, 32, 32)
    z = np.zeros((0, 3), np.float32)
    g, o = run_both(z, z, np.zeros((0, 4), np.float32), np.zeros(0, np.float32), np.zeros((0, 48), np.float32),
                    cam, RenderOptions(white_background=True))
    assert g.n_visible == 0 and float(g.rgb.abs().max()) == 0.0
    assert_parity(g, o)
    # tests/test_regressions.mojo:139-146: an extreme off-screen splat is culled
    g, o = run_both(np.array([[1e5, 1e5, 5]], np.float32), np.full((1, 3), 0.1, np.float32),
                    np.array([[1, 0, 0, 0]], np.float32), np.ones(1, np.float32), np.zeros((1, 48), np.float32),
                    cam, RenderOptions())
    assert g.n_visible == 0
    assert_parity(g, o)
    # every splat behind the camera (tests/test_regressions.mojo:59-85)
    sc = scenes.box_scene(1000, seed=3, centre=(0, 0, -8))
    s, op = sc.activated()
    g, o = run_both(sc.means, s, sc.quats, op, sc.sh, cam, RenderOptions())
    assert g.n_visible == 0 and g.n_instances == 0
    assert_parity(g, o)


def test_every_instance_in_one_tile_of_many():
    """Small splats stacked over one tile of a 4x4-tile frame: every tile id
    is equal, so no digit pass reorders anything and the ranges come from
    the sorted ids (the tile sort's last pass writes them only when a
    tile-id byte varies); then a frame of a single instance."""
    cam = ViewCamera((0, 0, 0), (1, 0, 0, 0), 50, 50, 32, 32, 0.1, 100, 64, 64)
    n = 5
    z = 4.0 + 0.5 * np.arange(n, dtype=np.float32)
    means = np.stack([(24.0 - 32.0) / 50 * z, (40.0 - 32.0) / 50 * z, z], 1).astype(np.float32)
    scales = np.full((n, 3), 0.001, np.float32)
    quats = np.tile(np.array([1, 0, 0, 0], np.float32), (n, 1))
    op = np.full(n, 0.6, np.float32)
    sh = np.zeros((n, 48), np.float32)
    sh[:, 0] = 1.0
    for m in (n, 1):
        g, o = run_both(means[:m], scales[:m], quats[:m], op[:m], sh[:m], cam, RenderOptions())
        assert o.n_instances == m and np.unique(o.keys_sorted >> np.uint64(32)).size == 1
        assert_parity(g, o, check_image_bits=True)


def test_degenerate_parameters():
    # zero scales (tests/test_regressions.mojo:26-57), unnormalised and zero quaternions,
    # transparent splats, splats on the near plane
    rng = np.random.default_rng(4)
    n = 4000
    means = rng.uniform([-2, -2, 0.0], [2, 2, 6], size=(n, 3)).astype(np.float32)
    scales = rng.uniform(0, 0.2, size=(n, 3)).astype(np.float32)
    scales[::7] = 0
    quats = rng.normal(size=(n, 4)).astype(np.float32) * 3
    quats[::11] = 0
    op = rng.uniform(0, 1, size=n).astype(np.float32)
    op[::5] = 0.001
    sh = rng.normal(0, 0.5, size=(n, 48)).astype(np.float32)
    cam = ViewCamera.from_fov(160, 120, 70.0, near_plane=0.5)
    g, o = run_both(means, scales, quats, op, sh, cam, RenderOptions())
    assert_parity(g, o, check_image_bits=True)


def test_needle_splats_parity():
    """Needle-like splats (one scale up to 4, the others down to 1e-4) at
    random rotations: projected conics with condition numbers up to about
    1e6, whose quadratic terms cancel. The compositors' reach test must
    keep every warp block where the blend's own float power admits a pixel
    (its rounding margin grows with the terms), so counts, last-visited
    offsets and images stay bit-exact against the oracle, which culls
    nothing."""
    rng = np.random.default_rng(41)
    n = 6000
    means = rng.uniform([-3, -2, 4.0], [3, 2, 10], size=(n, 3)).astype(np.float32)
    scales = np.exp(rng.uniform(np.log(1e-4), np.log(2e-3), size=(n, 3))).astype(np.float32)
    scales[np.arange(n), rng.integers(0, 3, n)] = rng.uniform(0.5, 4.0, n).astype(np.float32)
    quats = rng.normal(size=(n, 4)).astype(np.float32)
    op = rng.uniform(0.3, 1.0, size=n).astype(np.float32)
    sh = rng.normal(0, 0.3, size=(n, 48)).astype(np.float32)
    cam = ViewCamera.from_fov(640, 360, 60.0)
    for opt in (RenderOptions(), RenderOptions(term_mode=1)):
        g, o = run_both(means, scales, quats, op, sh, cam, opt)
        assert g.n_instances > 10 * n
        assert_parity(g, o, check_image_bits=True)


def test_medium_box_scene():
    sc = scenes.box_scene(50_000, seed=1)
    s, op = sc.activated()
    cam = scenes.camera_config1(480, 270)
    g, o = run_both(sc.means, s, sc.quats, op, sc.sh, cam, RenderOptions())
    # tile ids < 2^16 and millimetre depth keys 5000..11000: two digit passes per sort
    assert g.varying_digits & 0xFF == 0x3 and (g.varying_digits >> 8) & 0xFF == 0x3
    assert_parity(g, o, check_image_bits=True)


def test_capacity_growth_rerun():
    sc = scenes.box_scene(20_000, seed=2)
    s, op = sc.activated()
    cam = scenes.camera_config1(320, 180)
    g, o = run_both(sc.means, s, sc.quats, op, sc.sh, cam, RenderOptions(), capacity=1000)
    assert g.frame.capacity >= g.n_instances > 1000
    assert_parity(g, o, check_image_bits=True)


def test_config1_full_scale_parity():
    """1M Gaussians at 1920x1080: bit-exact keys, permutation, ranges and
    contributor counts; images within 1e-4."""
    sc = scenes.box_scene(1_000_000, seed=1)
    s, op = sc.activated()
    g, o = run_both(sc.means, s, sc.quats, op, sc.sh, scenes.camera_config1(), RenderOptions())
    assert g.n_instances > 5_000_000
    assert_parity(g, o)


# ---- the sort alone: tests/test_radix_sort.mojo:14-68 and stability ----
def test_sort_known_answer_and_lcg():
    from lumen_b200.render import sort_pairs
    keys = np.array([O.encode_key(1, 5.0), O.encode_key(0, 10.0), O.encode_key(0, 2.0), O.encode_key(1, 1.0)],
                    np.uint64)
    k, v = sort_pairs(torch.from_numpy(keys.view(np.int64)).cuda(), torch.arange(4, dtype=torch.int32).cuda())
    assert v.cpu().tolist() == [2, 1, 3, 0]
    seed, lcg = 123456789, []
    for _ in range(1000):
        seed = (seed * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        lcg.append(seed)
    lcg = np.array(lcg, np.uint64)
    k, v = sort_pairs(torch.from_numpy(lcg.view(np.int64)).cuda(), torch.arange(1000, dtype=torch.int32).cuda())
    assert np.array_equal(k.cpu().numpy().view(np.uint64), np.sort(lcg))


@pytest.mark.parametrize("n", [1, 4095, 4096, 4097, 300_001])
def test_sort_stability_random(n):
    from lumen_b200.render import sort_pairs
    rng = np.random.default_rng(n)
    keys = (rng.integers(0, 300, size=n).astype(np.uint64) << np.uint64(32)) | rng.integers(0, 50, size=n).astype(np.uint64)
    keys[::3] |= np.uint64(1) << np.uint64(63)
    k, v = sort_pairs(torch.from_numpy(keys.view(np.int64)).cuda(), torch.arange(n, dtype=torch.int32).cuda())
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(v.cpu().numpy(), order.astype(np.int32))
    assert np.array_equal(k.cpu().numpy().view(np.uint64), keys[order])
