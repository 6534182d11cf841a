"""Batched multi-view forward (lumen_gpu_render_batch): one pipeline over
several views, with batch-wide tile ids as the sort key's high part.

Each view of a batch must equal rendering it alone, bit for bit: images,
contributor counts, last-visited offsets, and its segment of the sorted
instances (keys shifted by the view's tile offset; values mapped to Gaussian
indices). One view per batch is also checked against the CPU oracle.
"""
import os

import numpy as np
import pytest

import oracle as O
from lumen_b200 import scenes
from lumen_b200.types import RenderOptions, ViewCamera

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

NT = max(1, min(16, os.cpu_count() or 1))


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def device_scene(sc, logits=False):
    from lumen_b200 import render as R
    if logits:
        s, op = sc.log_scales, sc.opacity_logits
    else:
        s, op = sc.activated()
    return R.Scene(_dev(sc.means), _dev(s), _dev(sc.quats), _dev(op).reshape(-1), _dev(sc.sh).reshape(-1, 48))


def single(scene, cam, opt):
    from lumen_b200 import render as R
    return R.render(*scene.tensors, cam, opt)


def check_views_against_single(views, opt):
    from lumen_b200 import render as R
    b = R.render_batch(views, opt)
    keys = b.sorted_keys.cpu().numpy().view(np.uint64)
    vals = b.sorted_vals.cpu().numpy().view(np.uint32)
    vis_ids = b.frame.frame.visible_ids.cpu().numpy()
    pos = 0
    total_k = 0
    for v, (scene, cam) in enumerate(views):
        s = single(scene, cam, opt)
        im = b.images[v]
        for name in ("rgb", "depth", "alpha"):
            a, c = getattr(im, name).cpu().numpy(), getattr(s, name).cpu().numpy()
            assert np.array_equal(a.view(np.uint32), c.view(np.uint32)), f"view {v}: {name} differs"
        assert np.array_equal(im.n_contrib.cpu().numpy(), s.n_contrib.cpu().numpy()), f"view {v}: n_contrib"
        assert np.array_equal(im.last_idx.cpu().numpy(), s.last_idx.cpu().numpy()), f"view {v}: last_idx"
        k = s.n_instances
        total_k += k
        seg = keys[pos:pos + k]
        ref = s.sorted_keys.cpu().numpy().view(np.uint64) + (np.uint64(b.tile_begin[v]) << np.uint64(32))
        assert np.array_equal(seg, ref), f"view {v}: sorted keys differ"
        gids = vis_ids[vals[pos:pos + k]]
        ref_g = s.frame.visible_ids.cpu().numpy()[s.sorted_vals.cpu().numpy().view(np.uint32)]
        assert np.array_equal(gids, ref_g), f"view {v}: permutation differs"
        pos += k
    assert b.n_instances == total_k
    return b


def test_orbit_views_of_one_scene():
    sc = scenes.box_scene(20_000, seed=21)
    ds = device_scene(sc)
    cams = scenes.orbit_cameras(6, 320, 180, fov=50.0, radius=10.0)
    check_views_against_single([(ds, c) for c in cams], RenderOptions())


@pytest.mark.parametrize("key_mode,term_mode", [(0, 0), (1, 1)])
def test_mixed_scenes_and_resolutions(key_mode, term_mode):
    a = device_scene(scenes.box_scene(15_000, seed=22))
    b = device_scene(scenes.box_scene(4_000, seed=23))
    c = device_scene(scenes.grid_scene(0))
    views = [(a, scenes.orbit_cameras(3, 320, 240, radius=9.0)[0]),
             (b, scenes.orbit_cameras(3, 97, 61, radius=7.0)[1]),
             (c, scenes.camera_config0()),
             (a, scenes.orbit_cameras(3, 640, 360, radius=11.0)[2]),
             (b, scenes.orbit_cameras(5, 17, 17, radius=8.0)[3])]
    opt = RenderOptions(key_mode=key_mode, term_mode=term_mode)
    check_views_against_single(views, opt)


def test_empty_views_and_white_background():
    """A view with no Gaussians, or with every splat culled, stays zero (as
    when rendered alone, pipeline.mojo:162-163) even though other views of
    the batch have instances; other views get the white background."""
    from lumen_b200 import render as R
    empty = R.Scene(*(torch.zeros((0, k), device="cuda") for k in (3, 3, 4)), torch.zeros(0, device="cuda"),
                    torch.zeros((0, 48), device="cuda"))
    behind = device_scene(scenes.box_scene(500, seed=3, centre=(0, 0, -8)))
    full = device_scene(scenes.box_scene(3000, seed=24, centre=(0, 0, 6)))
    cam = ViewCamera.from_fov(96, 64, 60.0)
    views = [(empty, cam), (full, cam), (behind, cam), (full, ViewCamera.from_fov(33, 47, 40.0)), (empty, cam)]
    opt = RenderOptions(white_background=True)
    b = check_views_against_single(views, opt)
    for v in (0, 2, 4):
        assert float(b.images[v].rgb.abs().max()) == 0.0
    assert float(b.images[1].rgb.max()) > 0.0


def test_logit_parameters_and_oracle():
    sc = scenes.box_scene(8_000, seed=25)
    ds = device_scene(sc, logits=True)
    cams = scenes.orbit_cameras(4, 200, 120, radius=9.0)
    opt = RenderOptions(params_are_logits=True)
    b = check_views_against_single([(ds, c) for c in cams], opt)
    o = O.render(sc.means, sc.log_scales, sc.quats, sc.opacity_logits, sc.sh, cams[2], opt, nthreads=NT)
    im = b.images[2]
    assert np.array_equal(im.n_contrib.cpu().numpy().view(np.uint32), o.n_contrib)
    assert np.array_equal(im.last_idx.cpu().numpy(), o.last_idx)
    assert float(np.abs(im.rgb.cpu().numpy() - o.rgb).max()) <= 1e-4


def test_config2_shape_batch():
    """300k Gaussians from 64 orbit cameras at 1280x720 in one batch: every
    view against its standalone render is checked for a sample of views,
    the instance total for all."""
    from lumen_b200 import render as R
    sc = scenes.box_scene(300_000, seed=2, centre=(0, 0, 8))
    ds = device_scene(sc)
    cams = scenes.orbit_cameras(64, 1280, 720, radius=10.0, centre=(0, 0, 8))
    views = [(ds, c) for c in cams]
    opt = RenderOptions()
    b = R.render_batch(views, opt)
    total = 0
    for v in range(64):
        s = single(ds, cams[v], opt)
        total += s.n_instances
        if v % 9 == 0:
            for name in ("rgb", "n_contrib", "last_idx"):
                a, c = getattr(b.images[v], name), getattr(s, name)
                assert torch.equal(a, c), f"view {v}: {name} differs"
    assert b.n_instances == total


@pytest.mark.parametrize("term_mode", [0, 1])
def test_interleaved_scene_groups(term_mode):
    """Views of one scene scattered among views of others (A B A C B A C),
    the order a server queue gives: the Gaussian-major projection groups the
    views of each scene wherever they sit in the batch, and every view still
    equals its standalone render."""
    a = device_scene(scenes.box_scene(6_000, seed=31))
    b = device_scene(scenes.box_scene(2_500, seed=32))
    c = device_scene(scenes.box_scene(9_000, seed=33, centre=(0, 0, 4)))
    ca = scenes.orbit_cameras(3, 160, 96, radius=9.0)
    cb = scenes.orbit_cameras(2, 123, 77, radius=7.0)
    cc = scenes.orbit_cameras(2, 256, 144, radius=11.0, centre=(0, 0, 4))
    views = [(a, ca[0]), (b, cb[0]), (a, ca[1]), (c, cc[0]), (b, cb[1]), (a, ca[2]), (c, cc[1])]
    check_views_against_single(views, RenderOptions(term_mode=term_mode))


@pytest.mark.parametrize("term_mode", [0, 1])
def test_distinct_scenes_with_empty_culled_and_ragged_views(term_mode):
    """No two views share a scene, so every projection unit is one view's
    block and the offset scan runs over the blocks of all views in turn:
    views with no Gaussians, with every splat culled and with ragged block
    counts between them, each equal to its standalone render."""
    from lumen_b200 import render as R
    empty = R.Scene(*(torch.zeros((0, k), device="cuda") for k in (3, 3, 4)), torch.zeros(0, device="cuda"),
                    torch.zeros((0, 48), device="cuda"))
    big = device_scene(scenes.box_scene(41_003, seed=41))
    behind = device_scene(scenes.box_scene(700, seed=42, centre=(0, 0, -8)))
    small = device_scene(scenes.box_scene(129, seed=43))
    mid = device_scene(scenes.box_scene(9_871, seed=44, centre=(0, 0, 4)))
    cams = scenes.orbit_cameras(5, 200, 136, radius=9.0)
    views = [(big, cams[0]), (empty, cams[1]), (behind, ViewCamera.from_fov(120, 80, 60.0)), (small, cams[3]),
             (mid, cams[4])]
    b = check_views_against_single(views, RenderOptions(term_mode=term_mode))
    assert float(b.images[2].rgb.abs().max()) == 0.0


def test_same_scene_storage_with_different_counts_is_not_grouped():
    """Two scenes sharing parameter storage but with different Gaussian
    counts (a prefix of the arrays) are different groups: each view equals
    its standalone render."""
    from lumen_b200 import render as R
    full = device_scene(scenes.box_scene(5_000, seed=34))
    t = full.tensors
    prefix = R.Scene(t[0][:3_000], t[1][:3_000], t[2][:3_000], t[3][:3_000], t[4][:3_000])
    cams = scenes.orbit_cameras(4, 144, 96, radius=9.0)
    views = [(full, cams[0]), (prefix, cams[1]), (full, cams[2]), (prefix, cams[3])]
    check_views_against_single(views, RenderOptions(term_mode=1))
