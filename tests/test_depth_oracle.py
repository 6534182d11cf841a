"""The CPU restatement of the depth-buffer products (the checker for the
device pass): the reference's own known answers (tests/test_depth_map.mojo),
the range rule of compute_min_max, and the SDK's depth heatmap against the
bytes the reference SDK wrote (tests/golden/sdk_depth_heatmap.npz, made by
tests/golden/make_golden.py). Also the host-side SDK mirror against the
same bytes."""
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sdk_depth_heatmap.npz")


def test_flat_surface_normal():
    # test_depth_map.mojo:9-20: constant depth 10 on 5 x 5, normal (0, 0, 1) at (2, 2)
    d = np.full((5, 5), 10.0, np.float32)
    np.testing.assert_allclose(O.depth_normal(d, 2, 2), [0.0, 0.0, 1.0], atol=1e-5)


def test_slanted_surface_normal():
    # test_depth_map.mojo:22-34: z = x, normal (-1, 0, 1) / sqrt(2) at (2, 2)
    d = np.tile(np.arange(5, dtype=np.float32), (5, 1))
    np.testing.assert_allclose(O.depth_normal(d, 2, 2), [-0.707106, 0.0, 0.707106], atol=1e-4)


def test_edges_use_clamped_neighbours():
    d = np.tile(np.arange(5, dtype=np.float32) * 2.0, (3, 1))
    # at x = 0 the difference is d[1] - d[0] = 2, halved: dz/dx = 1
    np.testing.assert_allclose(O.depth_normal(d, 0, 1), np.array([-1, 0, 1]) / np.sqrt(2), rtol=1e-6)
    one = np.full((1, 1), 3.0, np.float32)
    np.testing.assert_array_equal(O.depth_normal(one, 0, 0), [0.0, 0.0, 1.0])
    n = O.depth_normals(d)
    assert n.shape == (3, 5, 3)
    np.testing.assert_array_equal(n[1, 0], O.depth_normal(d, 0, 1))


def test_min_max_rule():
    assert O.depth_min_max(np.zeros(7, np.float32)) == (0.0, 1.0)          # nothing above 0.001
    assert O.depth_min_max(np.array([0.001, -5.0], np.float32)) == (0.0, 1.0)
    lo, hi = O.depth_min_max(np.array([0.0, 3.5, 0.002, 7.25, np.nan], np.float32))
    assert (lo, hi) == (np.float32(0.002), 7.25)
    assert O.depth_min_max(np.array([2e9], np.float32)) == (1e9, 2e9)      # min starts at 1e9
    assert O.depth_min_max(np.array([np.inf, 4.0], np.float32)) == (4.0, np.inf)


@pytest.mark.parametrize("tag,near,far", [("default", 0.5, 10.0), ("near1.25_far7.5", 1.25, 7.5)])
def test_heatmap_matches_the_reference_sdk_bytes(tag, near, far):
    z = np.load(GOLDEN)
    np.testing.assert_array_equal(O.depth_heatmap(z["depth"], near, far), z[tag])


def test_sdk_mirror_heatmap_matches_the_reference_sdk_bytes(tmp_path):
    from lumen_b200.visualizer import export_depth_visualization
    z = np.load(GOLDEN)
    d = z["depth"]
    h, w = d.shape
    p = tmp_path / "d.ppm"
    export_depth_visualization(str(p), w, h, [float(v) for v in d.reshape(-1)])
    raw = p.read_bytes()
    header = f"P6\n{w} {h}\n255\n".encode("ascii")
    assert raw.startswith(header)
    np.testing.assert_array_equal(np.frombuffer(raw[len(header):], np.uint8).reshape(h, w, 3), z["default"])


def test_c_abi_argument_checks():
    """lumen_gpu_depth_products rejects what the SDK would (host-side; nothing
    is launched for these)."""
    import ctypes as C
    from lumen_b200 import _lib as L
    lib = L.load()
    out = L.LumenDepthProducts()
    assert lib.lumen_gpu_depth_products(None, 4, 4, C.byref(out), None) == -1
    assert lib.lumen_gpu_depth_products(C.c_void_p(16), 0, 4, C.byref(out), None) == -1
    assert lib.lumen_gpu_depth_products(C.c_void_p(16), 4, 4, None, None) == -1
    out.heatmap, out.near_plane, out.far_plane = C.c_void_p(16), 2.0, 2.0            # far == near
    assert lib.lumen_gpu_depth_products(C.c_void_p(16), 4, 4, C.byref(out), None) == -1
    out.heatmap = None                                                                # nothing requested
    assert lib.lumen_gpu_depth_products(C.c_void_p(16), 4, 4, C.byref(out), None) == 0
