"""Picking on the device (include/lumen_spatial.h) against the CPU
restatement of LBVH.build_from_cloud and raycast_closest_splat: the nodes
and leaf order bit for bit (repeated positions, NaN positions, flat axes and
sizes from 1 to 1M), every hit bit for bit for batches of rays and of pixel
positions, the reference's own raycast known answers, and the empty
hierarchy."""
import numpy as np
import pytest

import oracle as O
from lumen_b200 import _lib as L
from lumen_b200 import scenes
from lumen_b200 import spatial as S

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def _cloud(n, seed, flat=False, nan=False):
    rng = np.random.default_rng(seed)
    means = rng.normal(0, 3, (n, 3)).astype(np.float32)
    means[::11] = means[0]
    if flat:
        means[:, 2] = 4.0
    if nan and n > 5:
        means[3, 1] = np.nan
    scales = rng.uniform(0.01, 0.3, (n, 3)).astype(np.float32)
    return means, scales


def _nodes_equal(bvh, nodes, idx):
    """Bit-equal nodes; a NaN box coordinate (from a NaN position) matches
    any NaN, since device and host NaN payloads differ."""
    k = bvh.node_count()
    got = bvh.nodes[:k].cpu().numpy().view(np.uint32)
    want = np.ascontiguousarray(nodes).view(np.uint32).reshape(-1, 8)
    assert got.shape == want.shape
    gf, wf = got.view(np.float32), want.view(np.float32)
    nan_ok = np.isnan(gf) & np.isnan(wf)
    nan_ok[:, [3, 7]] = False                          # child indices are integers
    assert ((got == want) | nan_ok).all()
    assert np.array_equal(bvh.splat_index[:len(idx)].cpu().numpy(), idx)


@pytest.mark.parametrize("n,seed,flat,nan", [(1, 0, False, False), (2, 1, False, False), (5, 2, False, False),
                                             (4097, 3, False, False), (100_003, 4, False, True),
                                             (30_000, 5, True, False), (1_000_000, 6, False, False)])
def test_build_matches_restatement(n, seed, flat, nan):
    means, scales = _cloud(n, seed, flat, nan)
    nodes, idx, root, _ = O.bvh_build(means, scales)
    bvh = S.LBVH(_t(means), _t(scales))
    assert bvh.root_index == root and bvh.node_count() == nodes.shape[0]
    _nodes_equal(bvh, nodes, idx)


def _compare_hits(raw, want):
    got = raw.cpu().numpy().view(np.uint32)
    exp = np.ascontiguousarray(want).view(np.uint32).reshape(-1, 6)
    bad = np.nonzero((got != exp).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} rays differ, first {bad[:5]}"


def test_raycast_matches_restatement():
    n = 200_000
    means, scales = _cloud(n, 7)
    nodes, idx, root, _ = O.bvh_build(means, scales)
    bvh = S.LBVH(_t(means), _t(scales))
    rng = np.random.default_rng(8)
    m = 4000
    origins = rng.uniform(-12, 12, (m, 3)).astype(np.float32)
    targets = means[rng.integers(0, n, m)]
    dirs = (targets - origins).astype(np.float32)
    dirs[::50] = rng.normal(size=(dirs[::50].shape[0], 3))          # some rays aim nowhere in particular
    dirs[7] = 0.0                                                    # zero direction
    dirs[9] = [0.0, 0.0, 1.0]                                        # axis-aligned (slab reciprocal 1e6)
    rays = np.concatenate([origins, dirs], axis=1)
    raw = bvh.raycast(_t(rays), max_dist=40.0)
    want = np.array([O.raycast(nodes, idx, root, means, scales, rays[i, :3], rays[i, 3:], 40.0) for i in range(m)],
                    O.RAY_HIT_DTYPE)
    assert want["hit"].sum() > m // 2
    _compare_hits(raw, want)


def test_pick_pixels_matches_restatement():
    sc = scenes.box_scene(300_000, seed=9)
    s, _ = sc.activated()
    cam = scenes.camera_config1(640, 360)
    nodes, idx, root, _ = O.bvh_build(sc.means, s)
    bvh = S.LBVH(_t(sc.means), _t(s))
    ys, xs = np.mgrid[0:360:7, 0:640:9]
    px = np.stack([xs.reshape(-1) + 0.5, ys.reshape(-1) + 0.25], axis=1).astype(np.float32)
    rays = torch.empty((px.shape[0], 6), dtype=torch.float32, device="cuda")
    raw = bvh.pick(cam, _t(px), rays_out=rays)
    want_rays = np.array([np.concatenate(O.generate_ray(cam, x, y)) for x, y in px], np.float32)
    assert np.array_equal(rays.cpu().numpy().view(np.uint32), want_rays.view(np.uint32))
    want = np.array([O.raycast(nodes, idx, root, sc.means, s, r[:3], r[3:], 1000.0, unit=True) for r in want_rays],
                    O.RAY_HIT_DTYPE)
    assert want["hit"].sum() > 0
    _compare_hits(raw, want)


def test_reference_raycast_known_answers_and_empty():
    # test_raycast.mojo:14-44
    means = np.array([[0, 0, 5], [0, 0, 10], [5, 5, 5]], np.float32)
    scales = np.full((3, 3), 0.5, np.float32)
    bvh = S.LBVH(_t(means), _t(scales))
    h = S.raycast_closest_splat(bvh, (0, 0, 0), (0, 0, 1))
    assert h.hit and h.splat_index == 0 and abs(h.distance - 5.0) < 1e-3
    h = S.raycast_closest_splat(bvh, (0, 0, 0), (0, 0, -1))
    assert not h.hit and h.splat_index == -1 and h.distance == 1000.0
    empty = S.LBVH(torch.zeros((0, 3), device="cuda"), torch.zeros((0, 3), device="cuda"))
    assert empty.node_count() == 0 and empty.root_index == -1
    h = S.raycast_closest_splat(empty, (0, 0, 0), (0, 0, 1))
    assert not h.hit and h.distance == np.float32(1e9)


def test_rejects_a_mismatched_hierarchy():
    lib = L.load()
    means, scales = _cloud(100, 10)
    bvh = S.LBVH(_t(means), _t(scales))
    g = L.LumenGpuGaussians()
    g.means, g.scales, g.count = bvh.means.data_ptr(), bvh.scales.data_ptr(), 99
    rays = _t(np.zeros((1, 6), np.float32))
    out = torch.empty((1, 6), dtype=torch.int32, device="cuda")
    import ctypes as C
    st = lib.lumen_gpu_raycast(C.byref(bvh.struct), C.byref(g), rays.data_ptr(), 1, 10.0, out.data_ptr(),
                               torch.cuda.current_stream().cuda_stream)
    assert st == -1
