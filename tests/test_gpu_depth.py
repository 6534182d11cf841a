"""The device depth pass (lumen_gpu_depth_products, include/lumen_depth.h)
against the CPU restatement of DepthMap.compute_min_max / extract_normal
and the SDK's depth heatmap: bit-exact normals, range and bytes, on a
rendered depth buffer, on seeded buffers full of edge values, on ragged and
one-pixel sizes, and on the reference SDK's own heatmap fixture."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
from lumen_b200 import _lib as L
from lumen_b200 import depth as D
from lumen_b200 import render as R
from lumen_b200 import scenes
from lumen_b200.types import RenderOptions

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sdk_depth_heatmap.npz")


def _edge_buffer(h, w, seed):
    rng = np.random.default_rng(seed)
    d = rng.uniform(0.2, 12.0, (h, w)).astype(np.float32)
    flat = d.reshape(-1)
    k = min(flat.size, 64)
    idx = rng.choice(flat.size, k, replace=False)
    pool = np.array([0.0, -1.0, -0.0, 1e-4, 0.001, 0.0011, 0.5, 10.0, 998.99, 999.0, 1e4, 2e9, np.inf, -np.inf,
                     np.nan, 1e-30], np.float32)
    flat[idx] = pool[rng.integers(0, pool.size, k)]
    return d


def _same_floats(a, b):
    """Bit-equal, except that any NaN matches any NaN (the device's NaN
    results carry the canonical payload, the host's the x86 default)."""
    a, b = np.ascontiguousarray(a, np.float32), np.ascontiguousarray(b, np.float32)
    return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())


def _check(d, near=0.5, far=10.0):
    t = torch.from_numpy(d).cuda()
    p = D.products(t, normals=True, range=True, heatmap=True, near_plane=near, far_plane=far)
    torch.cuda.synchronize()
    want_n = O.depth_normals(d)
    got_n = p.normals.cpu().numpy()
    # bit patterns, so signed zeros compare too
    assert _same_floats(got_n, want_n)
    lo, hi = O.depth_min_max(d)
    r = p.range.cpu().numpy()
    assert r[0] == np.float32(lo) and r[1] == np.float32(hi)
    got_h, want_h = p.heatmap.cpu().numpy(), O.depth_heatmap(d, near, far)
    bad = np.argwhere((got_h != want_h).any(axis=-1))
    detail = [(tuple(int(v) for v in b), float(d[tuple(b)]), hex(int(d[tuple(b)].view(np.uint32))),
               got_h[tuple(b)].tolist(), want_h[tuple(b)].tolist()) for b in bad[:6]]
    assert bad.shape[0] == 0, f"{bad.shape[0]} heatmap pixels differ: {detail}"


@pytest.mark.parametrize("h,w,seed", [(1080, 1920, 0), (13, 17, 1), (1, 1, 2), (1, 300, 3), (257, 1, 4),
                                      (720, 1280, 5)])
def test_products_match_restatement(h, w, seed):
    _check(_edge_buffer(h, w, seed))


def test_rendered_depth_buffer():
    sc = scenes.box_scene(200_000, seed=5)
    s, op = sc.activated()
    cam = scenes.camera_config1(960, 540)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    res = R.render(t(sc.means), t(s), t(sc.quats), t(op).reshape(-1), t(sc.sh).reshape(-1, 48), cam,
                   RenderOptions(compute_depth=True))
    d = res.depth.cpu().numpy()
    assert (d > 0.001).any() and (d == 0).any()
    _check(d, 2.0, 14.0)
    dm = D.DepthMap.from_render(res)
    assert dm.compute_min_max() == O.depth_min_max(d)
    x, y = 480, 270
    assert np.array_equal(np.array(dm.extract_normal(x, y), np.float32), O.depth_normal(d, x, y))


def test_reference_sdk_heatmap_fixture():
    z = np.load(GOLDEN)
    t = torch.from_numpy(z["depth"]).cuda()
    assert np.array_equal(D.heatmap(t).cpu().numpy(), z["default"])
    assert np.array_equal(D.heatmap(t, 1.25, 7.5).cpu().numpy(), z["near1.25_far7.5"])


def test_empty_range_and_invalid_arguments():
    lib = L.load()
    z = torch.zeros((4, 5), device="cuda")
    assert D.min_max(z) == (0.0, 1.0)
    s = L.LumenDepthProducts()
    hm = torch.empty((4, 5, 3), dtype=torch.uint8, device="cuda")
    s.heatmap, s.near_plane, s.far_plane = hm.data_ptr(), 3.0, 3.0
    st = torch.cuda.current_stream().cuda_stream
    assert lib.lumen_gpu_depth_products(z.data_ptr(), 5, 4, C.byref(s), st) == -1
    s.far_plane = 4.0
    assert lib.lumen_gpu_depth_products(None, 5, 4, C.byref(s), st) == -1
    assert lib.lumen_gpu_depth_products(z.data_ptr(), 0, 4, C.byref(s), st) == -1
    assert lib.lumen_gpu_depth_products(z.data_ptr(), 5, 4, C.byref(s), st) == 0
    torch.cuda.synchronize()
    with pytest.raises(ZeroDivisionError):
        D.heatmap(z, 1.0, 1.0)
