"""The C-ABI library without a GPU: it loads, exports every function the
headers in include/ declare, and its host-only entry points behave like the
reference library's (c_api/src/lumen_c.c; restated from
c_api/test/test_c_api.c:26-125)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from lumen_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in ("lumen.h", "lumen_gpu.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(lumen_\w+)\s*\(", src)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    return L.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 22 + 8
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (lumen_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert n in L.SIGNATURES, f"{n} has no ctypes signature"


def test_reference_22_symbols_present(lib):
    ref = ["lumen_get_version", "lumen_get_version_major", "lumen_get_version_minor", "lumen_get_version_patch",
           "lumen_default_config", "lumen_cloud_create", "lumen_cloud_destroy", "lumen_cloud_reserve",
           "lumen_cloud_get_count", "lumen_cloud_get_capacity", "lumen_cloud_add_gaussian",
           "lumen_cloud_get_gaussian", "lumen_cloud_clear", "lumen_create_synthetic_cube",
           "lumen_create_synthetic_sphere", "lumen_framebuffer_create", "lumen_framebuffer_destroy",
           "lumen_framebuffer_clear", "lumen_rasterizer_create", "lumen_rasterizer_destroy",
           "lumen_rasterizer_set_config", "lumen_rasterize"]
    assert len(ref) == 22
    for n in ref:
        assert hasattr(lib, n)


def test_struct_sizes():
    assert C.sizeof(L.LumenConfig) == 28
    assert C.sizeof(L.LumenGaussian) == 236
    assert C.sizeof(L.LumenCamera) == 52
    assert C.sizeof(L.LumenViewCamera) == 60
    assert C.sizeof(L.LumenRenderOptions) == 36


# ---- c_api/test/test_c_api.c:26-44 ----
def test_version_and_config(lib):
    assert lib.lumen_get_version() == b"0.1.0"
    assert (lib.lumen_get_version_major(), lib.lumen_get_version_minor(), lib.lumen_get_version_patch()) == (0, 1, 0)
    c = lib.lumen_default_config()
    assert (c.image_width, c.image_height, c.tile_size) == (800, 600, 16)
    assert c.near_plane > 0 and c.far_plane > c.near_plane and c.early_termination_alpha > 0.9


# ---- c_api/test/test_c_api.c:46-83 ----
def test_cloud_lifecycle(lib):
    cloud = lib.lumen_cloud_create(8)
    assert cloud
    assert lib.lumen_cloud_get_count(cloud) == 0 and lib.lumen_cloud_get_capacity(cloud) >= 8
    g = L.LumenGaussian()
    g.position = L.LumenVec3(1, 2, 3)
    g.scale = L.LumenVec3(0.1, 0.1, 0.1)
    g.rotation = L.LumenQuat(1, 0, 0, 0)
    g.opacity = 0.9
    assert lib.lumen_cloud_add_gaussian(cloud, C.byref(g)) == 0
    out = L.LumenGaussian()
    assert lib.lumen_cloud_get_gaussian(cloud, 0, C.byref(out)) == 0
    assert (out.position.x, out.position.y, out.position.z) == (1.0, 2.0, 3.0)
    for i in range(30):
        g.position.x = float(i)
        lib.lumen_cloud_add_gaussian(cloud, C.byref(g))
    assert lib.lumen_cloud_get_count(cloud) == 31 and lib.lumen_cloud_get_capacity(cloud) >= 31
    assert lib.lumen_cloud_get_gaussian(cloud, 31, C.byref(out)) == -1
    assert lib.lumen_cloud_add_gaussian(None, C.byref(g)) == -1
    arr = (L.LumenGaussian * 5)()
    assert lib.lumen_cloud_append(cloud, arr, 5) == 0 and lib.lumen_cloud_get_count(cloud) == 36
    lib.lumen_cloud_clear(cloud)
    assert lib.lumen_cloud_get_count(cloud) == 0
    lib.lumen_cloud_destroy(cloud)
    lib.lumen_cloud_destroy(None)


def _cloud_array(lib, cloud):
    n = lib.lumen_cloud_get_count(cloud)
    out = np.zeros((n, 59), np.float32)
    g = L.LumenGaussian()
    for i in range(n):
        lib.lumen_cloud_get_gaussian(cloud, i, C.byref(g))
        out[i] = np.frombuffer(bytes(g), dtype=np.float32)
    return out


# ---- c_api/test/test_c_api.c:85-104, pinned to the reference library's output ----
def test_synthetic_scenes_match_reference_golden(lib):
    gold = np.load(os.path.join(ROOT, "tests", "golden", "capi_synthetic.npz"))
    cube = lib.lumen_create_synthetic_cube(4, 2.0)
    assert lib.lumen_cloud_get_count(cube) == 64
    assert np.array_equal(_cloud_array(lib, cube), gold["cube_4_2"])
    lib.lumen_cloud_destroy(cube)
    sphere = lib.lumen_create_synthetic_sphere(128, 1.5)
    assert lib.lumen_cloud_get_count(sphere) == 128
    np.testing.assert_allclose(_cloud_array(lib, sphere), gold["sphere_128_1.5"], rtol=0, atol=2e-6)
    lib.lumen_cloud_destroy(sphere)


# ---- c_api/test/test_c_api.c:106-125 ----
def test_framebuffer(lib):
    fb = lib.lumen_framebuffer_create(128, 96)
    assert fb and fb.contents.width == 128 and fb.contents.height == 96
    lib.lumen_framebuffer_clear(fb, 42, 84, 126)
    f = fb.contents
    assert (f.rgb_data[0], f.rgb_data[1], f.rgb_data[2]) == (42, 84, 126)
    assert f.alpha_data[0] == 0.0 and f.depth_data[0] == 1000.0
    lib.lumen_framebuffer_destroy(fb)
    assert not lib.lumen_framebuffer_create(0, 10)


def test_rasterize_argument_errors(lib):
    # c_api/src/lumen_c.c:387: NULL arguments are INVALID_ARGUMENT, before any device work
    assert lib.lumen_rasterize(None, None, None, None, None) == -1
    assert lib.lumen_rasterizer_set_config(None, None) == -1
