"""GPU parity against the CPU oracle on exactly the settings the measured
workloads run: accumulated-alpha termination at 0.99 (the early-termination
rule of c_api/src/lumen_c.c:514 and python/lumen/client.py:166), full-size
scenes, a 3840x2160 frame with 32 400 tiles, views of a 64-view batch, and
the logit-parameter forward of the differentiable workload.

Bit-exact: visible counts, radii, projected records, sorted 64-bit keys,
the permutation, tile ranges, per-pixel contributor counts and last-visited
indices. Images: max abs error <= 1e-4 per channel.
"""
import numpy as np
import pytest

import oracle as O
from lumen_b200 import scenes
from lumen_b200.types import RenderOptions

from test_gpu_forward import IMAGE_TOL, NT, _dev, assert_parity, run_both

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_config1_full_scale_alpha_termination():
    """1M Gaussians at 1920x1080, compositing stops at accumulated alpha >=
    0.99: the settings of the per-call forward measurement."""
    sc = scenes.box_scene(1_000_000, seed=1)
    s, op = sc.activated()
    opt = RenderOptions(term_mode=1, term_threshold=0.99)
    g, o = run_both(sc.means, s, sc.quats, op, sc.sh, scenes.camera_config1(), opt)
    assert g.n_instances > 5_000_000
    # some pixels stop on the alpha rule before the end of their tile's list
    last = g.last_idx.cpu().numpy()
    assert (last >= 0).any()
    assert_parity(g, o)


def test_serving_2m_scene_at_3840x2160():
    """The largest served frame: the 2M-Gaussian scene of the serving mix
    from an orbit camera at 3840x2160 (240x135 = 32 400 tiles)."""
    sc = scenes.box_scene(2_000_000, seed=107)
    s, op = sc.activated()
    cam = scenes.orbit_cameras(64, 3840, 2160, radius=10.0)[5]
    assert cam.n_tiles == 32_400
    opt = RenderOptions(term_mode=1)
    g, o = run_both(sc.means, s, sc.quats, op, sc.sh, cam, opt)
    assert g.n_instances > 10_000_000
    # tile ids beyond 2^14 (a third digit byte of the tile id varies) and
    # tile lists longer than several compositor chunks
    r = g.ranges.cpu().numpy()
    filled = np.nonzero(r[:, 0] >= 0)[0]
    assert filled.max() > 30_000
    assert int((r[filled, 1] - r[filled, 0]).max()) > 4096
    assert_parity(g, o)


def test_config3_logit_forward_full_scale():
    """500k Gaussians at 1920x1080 with log-scales and opacity logits
    activated on the device: the forward of the differentiable workload."""
    sc = scenes.box_scene(500_000, seed=3)
    opt = RenderOptions(term_mode=1, params_are_logits=True)
    g, o = run_both(sc.means, sc.log_scales, sc.quats, sc.opacity_logits, sc.sh, scenes.camera_config1(), opt)
    assert g.n_instances > 2_000_000
    assert_parity(g, o)


def test_config2_batch_views_against_oracle():
    """300k Gaussians from 64 orbit cameras at 1280x720 in one batch; four
    views are compared with the oracle: their segments of the batch's
    sorted keys (view tile offset removed) and of the permutation (view's
    first visible index removed), their tile ranges, contributor counts,
    last-visited offsets and images."""
    from lumen_b200 import render as R
    sc = scenes.box_scene(300_000, seed=2)
    s, op = sc.activated()
    ds = R.Scene(_dev(sc.means), _dev(s), _dev(sc.quats), _dev(op).reshape(-1), _dev(sc.sh).reshape(-1, 48))
    cams = scenes.orbit_cameras(64, 1280, 720, radius=10.0)
    opt = RenderOptions(term_mode=1)
    b = R.render_batch([(ds, c) for c in cams], opt)
    # per-view visible and instance counts give each view's offsets in the batch
    counts = [R.render(*ds.tensors, c, opt) for c in cams]
    vbeg = np.cumsum([0] + [r.n_visible for r in counts])
    kbeg = np.cumsum([0] + [r.n_instances for r in counts])
    assert b.n_visible == vbeg[-1] and b.n_instances == kbeg[-1]
    keys = b.sorted_keys.cpu().numpy().view(np.uint64)
    vals = b.sorted_vals.cpu().numpy().view(np.uint32)
    ranges = b.frame.frame.ranges.cpu().numpy()
    for v in (0, 21, 42, 63):
        o = O.render(sc.means, s, sc.quats, op, sc.sh, cams[v], opt, nthreads=NT)
        assert (o.n_visible, o.n_instances) == (counts[v].n_visible, counts[v].n_instances)
        k0, k1 = int(kbeg[v]), int(kbeg[v + 1])
        seg = keys[k0:k1]
        tb = np.uint64(b.tile_begin[v])
        local = ((seg >> np.uint64(32)) - tb) << np.uint64(32) | (seg & np.uint64(0xFFFFFFFF))
        assert np.array_equal(local, o.keys_sorted), f"view {v}: sorted keys differ"
        assert np.array_equal(vals[k0:k1] - np.uint32(vbeg[v]), o.vals_sorted), f"view {v}: permutation differs"
        T = cams[v].n_tiles
        vr = ranges[b.tile_begin[v]:b.tile_begin[v] + T].astype(np.int64)
        vr = np.where(vr >= 0, vr - k0, vr)
        assert np.array_equal(vr, o.ranges.astype(np.int64)), f"view {v}: tile ranges differ"
        im = b.images[v]
        assert np.array_equal(im.n_contrib.cpu().numpy().view(np.uint32), o.n_contrib), f"view {v}: counts"
        assert np.array_equal(im.last_idx.cpu().numpy(), o.last_idx), f"view {v}: last index"
        for name in ("rgb", "depth", "alpha"):
            err = float(np.abs(getattr(im, name).cpu().numpy() - getattr(o, name)).max())
            assert err <= IMAGE_TOL, f"view {v}: {name} max abs err {err}"
