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
    for h in ("lumen.h", "lumen_gpu.h", "lumen_serve.h", "lumen_ply.h", "lumen_train.h", "lumen_depth.h", "lumen_spatial.h"):
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


GPU_STRUCTS = ["LumenGpuGaussians", "LumenViewCamera", "LumenRenderOptions", "LumenSplatRecord", "LumenGpuFrame",
               "LumenGpuImage", "LumenGpuCounts", "LumenGpuGradients", "LumenGpuBatchView", "LumenGpuLaunch",
               "LumenServerConfig",
               "LumenServeResult", "LumenServeStats", "LumenPlyInfo", "LumenTrainingConfig", "LumenAdamState",
               "LumenDensifyStats", "LumenDepthProducts", "LumenBvhNode", "LumenGpuBvh", "LumenRay",
               "LumenRayHit"]


def test_ctypes_layouts_match_the_header(tmp_path):
    """sizeof and every field offset of the ctypes mirrors equal what a C
    compiler gives for include/lumen_gpu.h and include/lumen_serve.h."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "lumen_serve.h"', '#include "lumen_ply.h"', '#include "lumen_train.h"', '#include "lumen_depth.h"', '#include "lumen_spatial.h"',
             "int main(void) {"]
    for name in GPU_STRUCTS:
        if not hasattr(L, name):
            continue
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for field, _ in getattr(L, name)._fields_:
            lines.append(f'printf("{name}.{field} %zu\\n", offsetof({name}, {field}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.split() for line in out if line.strip())
    for name in GPU_STRUCTS:
        if not hasattr(L, name):
            continue
        cls = getattr(L, name)
        assert int(got[name]) == C.sizeof(cls), name
        for field, _ in cls._fields_:
            assert int(got[f"{name}.{field}"]) == getattr(cls, field).offset, f"{name}.{field}"


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
    # counts whose sum with the current count, or whose byte size, wraps are refused before any copy
    size_max = (1 << 64) - 1
    for n in (size_max, size_max - 10, size_max // C.sizeof(L.LumenGaussian) - 35, 1 << 62):
        assert lib.lumen_cloud_append(cloud, arr, n) == -1
    assert lib.lumen_cloud_get_count(cloud) == 36
    assert lib.lumen_cloud_reserve(cloud, size_max // 8) == -2
    assert lib.lumen_cloud_get_capacity(cloud) < 1 << 20
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


def test_server_default_config_and_create_without_device(lib):
    c = lib.lumen_server_default_config()
    assert c.max_views_per_batch == 64 and c.max_batches_in_flight == 2 and c.use_graphs == 1
    assert c.options.tile_size == 16 and c.options.term_mode == 1 and abs(c.options.term_threshold - 0.99) < 1e-7
    bad = lib.lumen_server_default_config()
    bad.max_views_per_batch = 0
    assert not lib.lumen_server_create(C.byref(bad))
    bad = lib.lumen_server_default_config()
    bad.autotune, bad.composite_chunk = 0, 100
    assert not lib.lumen_server_create(C.byref(bad))
    assert lib.lumen_server_submit(None, 0, None, None, None) == -1
    assert lib.lumen_server_stats(None, None) == -1


def _admit(lib, reqs, max_views=64, caps=(1000, 1000, 1000, 1000)):
    a = [(C.c_int64 * max(len(reqs), 1))(*[r[i] for r in reqs]) for i in range(4)]
    return lib.lumen_serve_admit(a[0], a[1], a[2], a[3], len(reqs), max_views, *caps)


def test_admission_is_fifo_prefix_within_every_capacity(lib):
    """The server admits the longest queue prefix whose projection slots,
    tiles, instance estimates and pixels all fit one slot's buffers."""
    r = (256, 10, 100, 200)
    assert _admit(lib, [r] * 3) == 3
    assert _admit(lib, [r] * 10) == 3          # slots: 4 x 256 > 1000
    assert _admit(lib, [r] * 10, max_views=2) == 2
    assert _admit(lib, [(1, 1, 400, 1)] * 5) == 2   # instances
    assert _admit(lib, [(1, 600, 1, 1)] * 5) == 1   # tiles
    assert _admit(lib, [(1, 1, 1, 999), (1, 1, 1, 2)]) == 1   # pixels; no skipping ahead
    assert _admit(lib, [(1001, 1, 1, 1), r]) == 0   # the front request can never fit
    assert _admit(lib, []) == 0
