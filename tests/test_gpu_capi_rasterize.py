"""lumen_rasterize (the drop-in C entry, include/lumen.h) on the GPU: the
frame is composited in row bands whose rows are blended over the frame
buffer's old contents and read back while the next band renders. Checked
bit for bit against the device forward at the same camera, over a
patterned old buffer (colour weighted by the transmittance, old depth where
nothing blended, c_api/src/lumen_c.c:541-543 truncation), at 1080p and at
ragged sizes, including a first call whose instance count exceeds the
renderer's initial capacity (the frame is re-enqueued with its read-backs)."""
import ctypes as C

import numpy as np
import pytest

from lumen_b200 import _lib as L
from lumen_b200 import render as R
from lumen_b200 import scenes
from lumen_b200.types import RenderOptions

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _rasterize(lib, rast, cloud, cam, w, h, seed):
    fb = lib.lumen_framebuffer_create(w, h)
    assert fb
    try:
        f = fb.contents
        n = w * h
        rng = np.random.default_rng(seed)
        old8 = rng.integers(0, 256, n * 3).astype(np.uint8)
        oldd = rng.uniform(1.0, 2000.0, n).astype(np.float32)
        np.ctypeslib.as_array(f.rgb_data, shape=(n * 3,))[:] = old8
        np.ctypeslib.as_array(f.depth_data, shape=(n,))[:] = oldd
        st = L.LumenStats()
        L.check(lib.lumen_rasterize(rast, cloud, C.byref(cam), fb, C.byref(st)), "rasterize")
        out8 = np.ctypeslib.as_array(f.rgb_data, shape=(n * 3,)).copy()
        outd = np.ctypeslib.as_array(f.depth_data, shape=(n,)).copy()
        outa = np.ctypeslib.as_array(f.alpha_data, shape=(n,)).copy()
    finally:
        lib.lumen_framebuffer_destroy(fb)
    return old8, oldd, out8, outd, outa, st


def _expected(g, old8, oldd):
    rgb = g.rgb.cpu().numpy().reshape(-1, 3)
    a = g.alpha.cpu().numpy().reshape(-1)
    T = (np.float32(1.0) - a)[:, None]
    v = rgb + T * (old8.reshape(-1, 3).astype(np.float32) / np.float32(255.0))
    v = np.clip(v, np.float32(0.0), np.float32(1.0))
    want8 = (v * np.float32(255.0)).astype(np.uint8).reshape(-1)
    wantd = np.where(a > 0.0, g.depth.cpu().numpy().reshape(-1), oldd)
    return want8, wantd, a


@pytest.mark.parametrize("w,h,n,big", [(1920, 1080, 200_000, False), (333, 127, 30_000, False),
                                       (1280, 720, 60_000, True)])
def test_rasterize_matches_device_forward_over_old_contents(w, h, n, big):
    lib = L.load()
    sc = scenes.box_scene(n, seed=21, centre=(0, 0, 8))
    s, o = sc.activated()
    if big:
        s = s * np.float32(12.0)        # large splats: many tiles each, over the first capacity guess
    aos = np.zeros((n, 59), np.float32)
    aos[:, 0:3], aos[:, 3:6], aos[:, 6:10], aos[:, 10] = sc.means, s, sc.quats, o
    aos[:, 11:] = sc.sh.reshape(n, 48)
    cloud = lib.lumen_cloud_create(n)
    L.check(lib.lumen_cloud_append(cloud, aos.ctypes.data_as(C.POINTER(L.LumenGaussian)), n), "append")
    cfg = lib.lumen_default_config()
    cfg.near_plane, cfg.far_plane = 0.1, 100.0
    rast = lib.lumen_rasterizer_create(C.byref(cfg))
    assert rast
    try:
        cam = L.LumenCamera(L.LumenVec3(0.3, 0.2, -1.0), L.LumenVec3(0.0, 0.0, 8.0), L.LumenVec3(0.0, 1.0, 0.0),
                            60.0, 50.0, 0.1, 100.0)
        vc = L.LumenViewCamera()
        L.check(lib.lumen_gpu_camera_from_lookat(C.byref(cam), w, h, cfg.near_plane, cfg.far_plane, C.byref(vc)),
                "camera")
        from lumen_b200.types import ViewCamera
        view = ViewCamera(tuple(vc.position), tuple(vc.rotation), vc.fx, vc.fy, vc.cx, vc.cy, vc.near_plane,
                          vc.far_plane, vc.width, vc.height)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
        g = R.render(t(sc.means), t(s), t(sc.quats), t(o), t(sc.sh).reshape(n, 48), view,
                     RenderOptions(term_mode=1, term_threshold=cfg.early_termination_alpha))
        if big:
            assert g.n_instances > max(8 * n, 1 << 20)      # the first rasterize call must grow its buffers
        for call in range(2):
            old8, oldd, out8, outd, outa, st = _rasterize(lib, rast, cloud, cam, w, h, seed=call)
            want8, wantd, a = _expected(g, old8, oldd)
            assert np.array_equal(outa, a)
            assert np.array_equal(out8, want8)
            assert np.array_equal(outd, wantd)
            assert st.visible_splats == g.n_visible and st.touched_tiles == g.touched_tiles
    finally:
        lib.lumen_rasterizer_destroy(rast)
        lib.lumen_cloud_destroy(cloud)
