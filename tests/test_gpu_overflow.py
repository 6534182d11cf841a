"""A frame whose instances exceed its capacity.

The emission writes, and counts for the tile sort, only the first
`capacity` instances of its depth-ordered stream; the frame reports
LUMEN_GPU_ERR_CAPACITY with the full instance count (the host then renders
again with larger buffers), and its tile sort orders exactly the written
prefix: a stable sort by tile id. The expected prefix is rebuilt from the
oracle's emission (pipeline.mojo:141-157, one splat's tiles rows outer,
columns inner) in this pipeline's order: visible splats by (depth key,
visible index).
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
from lumen_b200 import scenes
from lumen_b200.types import RenderOptions

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

NT = max(1, min(16, os.cpu_count() or 1))


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _expected_prefix(o, cap):
    """(tile id, visible index) of the first `cap` instances of the
    depth-ordered emission, stably sorted by tile id."""
    ku = o.keys_unsorted.astype(np.uint64)
    vu = o.vals_unsorted.astype(np.int64)
    assert np.all(np.diff(vu) >= 0), "the oracle emits visible splat by visible splat"
    V = o.n_visible
    first = np.searchsorted(vu, np.arange(V + 1))
    count = np.diff(first)
    assert count.min() >= 1
    depth_key = (ku[first[:V]] & np.uint64(0xFFFFFFFF)).astype(np.int64)
    order = np.lexsort((np.arange(V), depth_key))
    seg = np.concatenate([np.arange(first[v], first[v + 1]) for v in order])
    pre = seg[:cap]
    tiles = (ku[pre] >> np.uint64(32)).astype(np.int64)
    perm = np.argsort(tiles, kind="stable")
    return tiles[perm], vu[pre][perm]


@pytest.mark.parametrize("cap_fraction", [0.37, 0.81])
def test_overflowing_frame_sorts_the_written_prefix(cap_fraction):
    from lumen_b200 import _lib as L
    from lumen_b200 import render as R
    sc = scenes.box_scene(20_000, seed=2)
    s, op = sc.activated()
    cam = scenes.camera_config1(320, 180)
    opt = RenderOptions()
    o = O.render(sc.means, s, sc.quats, op, sc.sh, cam, opt, nthreads=NT)
    K = o.n_instances
    cap = int(K * cap_fraction) | 1          # odd: the last sort tile is partial
    assert 0 < cap < K

    lib = L.load()
    n = sc.means.shape[0]
    ts = (_dev(sc.means), _dev(s), _dev(sc.quats), _dev(op).reshape(-1), _dev(sc.sh).reshape(-1, 48))
    g = R.gaussians_struct(*ts)
    H, W = cam.height, cam.width
    outs = [torch.empty(shape, dtype=dt, device="cuda")
            for shape, dt in (((H, W, 3), torch.float32), ((H, W), torch.float32), ((H, W), torch.float32),
                              ((H, W), torch.int32), ((H, W), torch.int32))]
    img = L.LumenGpuImage()
    img.rgb, img.depth, img.alpha, img.n_contrib, img.last_idx = (t.data_ptr() for t in outs)
    frame = R.Frame.allocate(n, cam.n_tiles, cap, torch.device("cuda"))
    fs = frame.c_struct()
    stream = torch.cuda.current_stream().cuda_stream
    L.check(lib.lumen_gpu_render_forward(C.byref(g), C.byref(L.view_camera(cam)), C.byref(L.render_options(opt)),
                                         C.byref(fs), C.byref(img), stream), "render_forward")
    counts = L.LumenGpuCounts()
    L.check(lib.lumen_gpu_read_counts(C.byref(fs), C.byref(counts), stream), "read_counts")
    torch.cuda.synchronize()
    assert counts.error_flags == L.ERR_CAPACITY, hex(counts.error_flags)
    assert int(counts.n_instances) == K and int(counts.n_visible) == o.n_visible

    b = int(counts.sorted_buffer)
    keys = frame.keys[b][:cap].cpu().numpy().view(np.uint32).astype(np.int64)
    vals = frame.vals[b][:cap].cpu().numpy().view(np.uint32).astype(np.int64)
    exp_tiles, exp_vis = _expected_prefix(o, cap)
    assert np.array_equal(keys, exp_tiles), "sorted tile ids of the written prefix differ"
    assert np.array_equal(vals, exp_vis), "permutation of the written prefix differs"
