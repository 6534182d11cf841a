"""The CPU restatement of the picking path (the checker for the device
build and casts): the reference's own known answers (tests/test_morton.mojo,
tests/test_bvh.mojo, tests/test_raycast.mojo) restated, the hierarchy's
structure, and ray casts against a brute-force search."""
import numpy as np
import pytest

import oracle as O


def test_morton_known_answers():
    # test_morton.mojo:9-24
    assert O.morton3d(0.0, 0.0, 0.0) == 0
    assert O.morton3d(1.0, 1.0, 1.0) == 0x3FFFFFFF
    assert O.expand_bits(1) == 1 and O.expand_bits(2) == 8
    # test_morton.mojo:26-43: nearby points get nearby codes
    a, b, c = O.morton3d(0.5, 0.5, 0.5), O.morton3d(0.501, 0.501, 0.501), O.morton3d(0.9, 0.9, 0.9)
    assert abs(b - a) < abs(c - a)
    # clamping and the x | y << 1 | z << 2 interleave
    assert O.morton3d(-3.0, 7.0, 0.0) == O.morton3d(0.0, 1.0, 0.0) == O.expand_bits(1023) << 1
    assert O.morton3d(1.0 / 1023.0, 0.0, 0.0) == 1
    assert O.morton3d(float("nan"), 0.0, 0.0) == 0


def cube_scene(per_axis=4, spacing=0.5):
    """create_synthetic_cube_scene (src/scene/datasets.mojo:46-80): positions
    and scales."""
    f = np.float32
    half = f(per_axis - 1) * f(spacing) * f(0.5)
    pts = []
    for i in range(per_axis):
        x = f(i) * f(spacing) - half
        for j in range(per_axis):
            y = f(j) * f(spacing) - half
            for k in range(per_axis):
                pts.append((x, y, f(k) * f(spacing) - half))
    means = np.array(pts, np.float32)
    scales = np.full_like(means, f(spacing) * f(0.3))
    return means, scales


def test_lbvh_cube_known_answers():
    # test_bvh.mojo:9-34
    means, scales = cube_scene(4, 0.5)
    nodes, idx, root, _ = O.bvh_build(means, scales)
    assert nodes.shape[0] > 64 and root >= 0
    r = nodes[root]
    assert not (r["left_child"] == -1 and r["right_child"] == -1)
    assert (r["min_pt"] <= 0).all() and (r["max_pt"] >= 0).all()
    assert r["min_pt"][0] <= means[:, 0].min() and r["max_pt"][0] >= means[:, 0].max()
    for i in range(64):
        assert nodes[i]["left_child"] == -1 and nodes[i]["right_child"] == -1
        assert 0 <= idx[i] < 64


@pytest.mark.parametrize("n", [1, 2, 3, 5, 64, 1000, 4097])
def test_hierarchy_structure(n):
    rng = np.random.default_rng(n)
    means = rng.normal(size=(n, 3)).astype(np.float32)
    means[::7] = means[0]                       # repeated positions: equal codes keep input order
    scales = rng.uniform(0.01, 0.2, (n, 3)).astype(np.float32)
    nodes, idx, root, codes = O.bvh_build(means, scales)
    count, total = n, n
    while count > 1:
        count = (count + 1) // 2
        total += count
    assert nodes.shape[0] == total and root == total - 1
    order = np.argsort(codes, kind="stable")
    np.testing.assert_array_equal(idx, order)
    for i in range(n, total):
        l, r = nodes[i]["left_child"], nodes[i]["right_child"]
        assert 0 <= l < i and (r == -1 or r == l + 1)
        kids = [nodes[l]] + ([nodes[r]] if r >= 0 else [])
        np.testing.assert_array_equal(nodes[i]["min_pt"], np.min([k["min_pt"] for k in kids], axis=0))
        np.testing.assert_array_equal(nodes[i]["max_pt"], np.max([k["max_pt"] for k in kids], axis=0))


def test_raycast_known_answers():
    # test_raycast.mojo:14-44
    means = np.array([[0, 0, 5], [0, 0, 10], [5, 5, 5]], np.float32)
    scales = np.full((3, 3), 0.5, np.float32)
    nodes, idx, root, _ = O.bvh_build(means, scales)
    h = O.raycast(nodes, idx, root, means, scales, (0, 0, 0), (0, 0, 1))
    assert h["hit"] == 1 and h["splat_index"] == 0 and abs(h["distance"] - 5.0) < 1e-3
    h = O.raycast(nodes, idx, root, means, scales, (0, 0, 0), (0, 0, -1))
    assert h["hit"] == 0 and h["splat_index"] == -1 and h["distance"] == 1000.0
    empty = O.raycast(np.zeros(0, O.BVH_NODE_DTYPE), np.zeros(0, np.int32), -1, means[:0], scales[:0],
                      (0, 0, 0), (0, 0, 1))
    assert empty["hit"] == 0 and empty["distance"] == np.float32(1e9)


def test_raycast_finds_the_nearest_valid_splat():
    rng = np.random.default_rng(3)
    n = 2000
    means = rng.uniform(-5, 5, (n, 3)).astype(np.float32)
    scales = rng.uniform(0.02, 0.15, (n, 3)).astype(np.float32)
    nodes, idx, root, _ = O.bvh_build(means, scales)
    for k in range(200):
        o = rng.uniform(-8, 8, 3).astype(np.float32)
        d = (means[rng.integers(n)] - o).astype(np.float32)
        h = O.raycast(nodes, idx, root, means, scales, o, d)
        dn = d / np.float32(np.sqrt(np.float32((d * d).sum())))
        t = ((means - o) * dn).sum(axis=1)
        dist = np.linalg.norm(o + dn * t[:, None] - means, axis=1)
        ok = (t > 0) & (dist <= scales.max(axis=1) * 3.0) & (t < 1000.0)
        assert bool(h["hit"]) == bool(ok.any())
        if ok.any():
            assert h["distance"] == pytest.approx(t[ok].min(), rel=1e-5, abs=1e-5)


def test_c_abi_host_paths():
    """Node counts, scratch sizes and argument checks of include/lumen_spatial.h
    (host-side; nothing is launched)."""
    import ctypes as C
    from lumen_b200 import _lib as L
    lib = L.load()
    for n in (0, 1, 2, 3, 5, 1000, 4097, 1 << 20):
        total, count = n, n
        while count > 1:
            count = (count + 1) // 2
            total += count
        assert lib.lumen_bvh_node_count(n) == total
    assert lib.lumen_gpu_bvh_scratch_bytes(-1) == 0 and lib.lumen_gpu_bvh_scratch_bytes(1000) > 0
    g, bvh = L.LumenGpuGaussians(), L.LumenGpuBvh()
    assert lib.lumen_gpu_bvh_build(C.byref(g), C.byref(bvh), None, 0, None) == 0      # empty cloud
    assert (bvh.leaf_count, bvh.node_count, bvh.root_index) == (0, 0, -1)
    g.count = 10                                                                      # no arrays
    assert lib.lumen_gpu_bvh_build(C.byref(g), C.byref(bvh), None, 0, None) == -1
    g.count = 0
    assert lib.lumen_gpu_raycast(C.byref(bvh), C.byref(g), None, 0, 1.0, None, None) == 0
    g.count = 3                                                                       # hierarchy of another cloud
    assert lib.lumen_gpu_raycast(C.byref(bvh), C.byref(g), None, 1, 1.0, None, None) == -1
