"""The SDK mirror (lumen_b200 as a drop-in for the reference's python/lumen):
the reference's python/tests/test_client.py restated. Camera, trajectory,
cloud and PLY tests run on the CPU; the two render tests need the GPU."""
import math
import os
import tempfile

import numpy as np
import pytest

import lumen_b200 as lumen
from lumen_b200 import (Camera, CameraTrajectory, GaussianCloud, LumenEngine, RasterizerConfig, ascii_render,
                        export_depth_visualization, export_ppm)


# ---- test_client.py:16-48 ----
def test_camera_forward():
    f = Camera(position=(0.0, 0.0, 5.0), target=(0.0, 0.0, 0.0)).forward_vector()
    assert abs(f[0]) < 1e-5 and abs(f[1]) < 1e-5 and abs(f[2] + 1.0) < 1e-5


def test_view_matrix_identity():
    mat = Camera(position=(0.0, 0.0, 0.0), target=(0.0, 0.0, -1.0)).view_matrix_4x4()
    assert len(mat) == 4 and len(mat[0]) == 4 and abs(mat[3][3] - 1.0) < 1e-5


def test_orbit_trajectory():
    cams = CameraTrajectory.orbit(target=(0.0, 0.0, 0.0), radius=4.0, num_frames=12)
    assert len(cams) == 12
    for c in cams:
        assert math.hypot(c.position[0], c.position[2]) > 0.5


def test_camera_interpolation():
    mid = CameraTrajectory.interpolate(Camera(position=(0.0, 0.0, 2.0)), Camera(position=(0.0, 0.0, 4.0)), 0.5)
    assert abs(mid.position[2] - 3.0) < 1e-5


# ---- test_client.py:51-80 ----
def test_cube_generation():
    cube = GaussianCloud.synthetic_cube(points_per_axis=3, cube_size=2.0)
    assert len(cube) == 27
    lo, hi = cube.bounding_box()
    assert abs(lo[0] + 1.0) < 1e-5 and abs(hi[0] - 1.0) < 1e-5
    assert all(abs(c) < 1e-5 for c in cube.centroid())


def test_sphere_generation():
    assert len(GaussianCloud.synthetic_sphere(point_count=50, radius=2.0)) == 50


def test_ply_roundtrip():
    cloud = GaussianCloud.synthetic_cube(points_per_axis=2, cube_size=1.0)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "c.ply")
        cloud.save_ply(p)
        loaded = GaussianCloud.load_ply(p)
    assert len(loaded) == len(cloud)
    assert abs(loaded.splats[0].position[0] - cloud.splats[0].position[0]) < 1e-4


def test_array_backed_cloud_packs_like_splats():
    cube = GaussianCloud.synthetic_cube(3, 1.0)
    a = cube.to_aos()
    arr = GaussianCloud.from_arrays(a[:, 0:3], a[:, 3:6], a[:, 6:10], a[:, 10], a[:, 11:59])
    assert np.array_equal(arr.to_aos(), a) and len(arr) == 27


def test_sdk_names_mirror_reference():
    for name in ("Camera", "CameraTrajectory", "GaussianCloud", "Gaussian3D", "LumenEngine", "RasterizerConfig",
                 "RenderResult", "export_ppm", "export_depth_visualization", "ascii_render"):
        assert hasattr(lumen, name)


def test_view_camera_matches_c_abi_focal():
    cam = Camera(position=(0, 0, 3), target=(0, 0, 0), fov_y_deg=45.0).view_camera(80, 60)
    # float32 arithmetic of c_api/src/lumen_c.c:393-395
    assert abs(cam.fy - 60 / (2 * math.tan(math.radians(22.5)))) < 1e-5 and cam.fx == cam.fy
    assert (cam.cx, cam.cy) == (40.0, 30.0)


# ---- test_client.py:83-117 (GPU) ----
@pytest.mark.gpu
def test_rasterize_scene():
    cfg = RasterizerConfig(image_width=80, image_height=60, tile_size=16, near_plane=0.1, far_plane=50.0)
    engine = LumenEngine(cfg)
    cube = GaussianCloud.synthetic_cube(points_per_axis=3, cube_size=1.0)
    res = engine.render(cube, Camera(position=(0.0, 0.0, 2.5), target=(0.0, 0.0, 0.0)))
    assert (res.width, res.height) == (80, 60)
    assert len(res.rgb_bytes) == 80 * 60 * 3 and len(res.depth_values) == 4800 and len(res.alpha_values) == 4800
    assert res.stats["total_splats"] == 27
    assert res.stats["visible_splats"] > 0 and res.stats["touched_tiles"] > 0
    assert res.alpha_values[30 * 80 + 40] > 0.0
    art = ascii_render(res.width, res.height, res.alpha_values, 30, 15)
    assert isinstance(art, str) and len(art) > 0


# ---- test_client.py:119-136 (GPU) ----
@pytest.mark.gpu
def test_image_export():
    engine = LumenEngine(RasterizerConfig(image_width=40, image_height=30))
    res = engine.render(GaussianCloud.synthetic_cube(points_per_axis=2, cube_size=0.8), Camera(position=(0.0, 0.0, 2.0)))
    with tempfile.TemporaryDirectory() as d:
        p, q = os.path.join(d, "r.ppm"), os.path.join(d, "d.ppm")
        export_ppm(p, res.width, res.height, res.rgb_bytes)
        export_depth_visualization(q, res.width, res.height, res.depth_values)
        assert os.path.getsize(p) > 0 and os.path.getsize(q) > 0


@pytest.mark.gpu
def test_engine_matches_device_render():
    """LumenEngine.render (C ABI, uint8 frame buffer) against the device
    forward at the same camera: alpha equal, rgb equal after the same
    quantisation, depth where alpha > 0."""
    import torch
    from lumen_b200 import render as R
    from lumen_b200.types import RenderOptions
    from lumen_b200 import scenes
    sc = scenes.box_scene(20_000, seed=9, centre=(0, 0, 0))
    s, o = sc.activated()
    cloud = GaussianCloud.from_arrays(sc.means, s, sc.quats, o, sc.sh.reshape(-1, 48))
    cam = Camera(position=(0.0, 0.5, 9.0), target=(0.0, 0.0, 0.0), fov_y_deg=50.0)
    cfg = RasterizerConfig(image_width=160, image_height=96, near_plane=0.1, far_plane=50.0)
    res = LumenEngine(cfg).render(cloud, cam)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    g = R.render(dev(sc.means), dev(s), dev(sc.quats), dev(o), dev(sc.sh).reshape(-1, 48),
                 cam.view_camera(160, 96, 0.1, 50.0), RenderOptions(term_mode=1, term_threshold=0.99))
    alpha = g.alpha.cpu().numpy().reshape(-1)
    assert np.array_equal(np.asarray(res.alpha_values, np.float32), alpha)
    rgb = np.clip(g.rgb.cpu().numpy().reshape(-1, 3), 0, 1)
    q = (rgb * np.float32(255.0)).astype(np.uint8)
    assert np.array_equal(np.frombuffer(res.rgb_bytes, np.uint8).reshape(-1, 3), q)
    d = np.asarray(res.depth_values, np.float32)
    m = alpha > 0
    assert np.array_equal(d[m], g.depth.cpu().numpy().reshape(-1)[m]) and np.all(d[~m] == 1000.0)
