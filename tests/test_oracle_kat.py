"""The reference's known-answer tests, restated against the CPU oracle.

Each test cites the reference test it restates (tests/*.mojo in the reference
project). Passing all of them is what pins the oracle to the reference, whose
Mojo code cannot run here.
"""
import math

import numpy as np
import pytest

import oracle as O
from lumen_b200.types import RenderOptions, ViewCamera

f32 = np.float32


def arr(*v):
    return np.array(v, dtype=np.float32)


# ---- tests/test_radix_sort.mojo:14-50 ----
def test_radix_sort_composite_keys():
    keys = np.array([O.encode_key(1, 5.0), O.encode_key(0, 10.0), O.encode_key(0, 2.0), O.encode_key(1, 1.0)],
                    np.uint64)
    k, v = O.radix_sort64(keys, np.arange(4, dtype=np.uint32))
    assert v.tolist() == [2, 1, 3, 0]
    assert [(int(x) >> 32) for x in k] == [0, 0, 1, 1]


# ---- tests/test_radix_sort.mojo:52-68 ----
@pytest.mark.parametrize("nthreads", [1, 4])
def test_radix_sort_large_monotonicity(nthreads):
    seed = 123456789
    keys = []
    for _ in range(1000):
        seed = (seed * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        keys.append(seed)
    k, v = O.radix_sort64(np.array(keys, np.uint64), np.arange(1000, dtype=np.uint32), nthreads)
    assert np.all(k[:-1] <= k[1:])
    assert sorted(v.tolist()) == list(range(1000))


def test_radix_sort_stable_on_ties():
    rng = np.random.default_rng(7)
    keys = rng.integers(0, 8, size=5000).astype(np.uint64) << np.uint64(32)
    k, v = O.radix_sort64(keys, np.arange(5000, dtype=np.uint32), 3)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(v, order.astype(np.uint32))


# ---- tests/test_binning.mojo:10-51 ----
def test_tile_range_construction():
    keys = np.array([O.encode_key(0, 1.0), O.encode_key(0, 2.0), O.encode_key(2, 3.0), O.encode_key(2, 4.0),
                     O.encode_key(2, 5.0), O.encode_key(3, 6.0), O.encode_key(3, 7.0)], np.uint64)
    r = O.tile_ranges(keys, 4)
    assert r.tolist() == [[0, 2], [-1, -1], [2, 5], [5, 7]]


def test_depth_key_encoding():
    # radix_sort.mojo:8-27: millimetre truncation, clamped to [0, 2^31-1]
    assert O.encode_key(3, 2.0) == (3 << 32) | 2000
    assert O.encode_key(0, -1.0) == 0
    assert O.encode_key(0, 1e10) == 0x7FFFFFFF
    assert O.encode_key(0, 0.0015) == 1
    bits = int(np.array([2.5], np.float32).view(np.uint32)[0])
    assert O.encode_key(5, 2.5, key_mode=1) == (5 << 32) | bits


# ---- tests/test_compositor.mojo:10-50 ----
def _blend(colors, alphas, depths, term_mode=0):
    c = np.zeros(3, np.float32)
    T = np.zeros(1, np.float32)
    d = np.zeros(1, np.float32)
    a = np.zeros(1, np.float32)
    cols = np.ascontiguousarray(colors, np.float32)
    al = np.ascontiguousarray(alphas, np.float32)
    de = np.ascontiguousarray(depths, np.float32)
    term = O.lib().oracle_blend_sequence(cols.ctypes.data, al.ctypes.data, de.ctypes.data, len(al), term_mode,
                                         c.ctypes.data, T.ctypes.data, d.ctypes.data, a.ctypes.data)
    return c, float(T[0]), float(d[0]), float(a[0]), term


def test_single_splat_compositing():
    c, T, d, a, term = _blend([[1, 0, 0]], [0.6], [5.0])
    assert not term
    assert abs(c[0] - 0.6) < 1e-5 and abs(c[1]) < 1e-5 and abs(c[2]) < 1e-5
    assert abs(T - 0.4) < 1e-5 and abs(a - 0.6) < 1e-5 and abs(d - 3.0) < 1e-5


def test_two_splat_order():
    c, T, d, a, _ = _blend([[0, 1, 0], [0, 0, 1]], [0.5, 0.8], [2.0, 4.0])
    assert abs(c[1] - 0.5) < 1e-5 and abs(c[2] - 0.4) < 1e-5 and abs(T - 0.1) < 1e-5


def test_early_ray_termination():
    c, T, d, a, term = _blend([[1, 1, 1]] * 10, [0.9] * 10, [1.0] * 10)
    assert T <= 1e-4 and term
    # accumulated-alpha rule: 1 - T >= 0.99 after the second 0.9 blend
    _, _, _, a2, term2 = _blend([[1, 1, 1]] * 2, [0.9] * 2, [1.0] * 2, term_mode=1)
    assert term2 and a2 >= 0.99


def test_pixel_alpha_cutoffs():
    # compositor.mojo:62-89: beyond power 4.5 the alpha is 0, and alpha clamps at 0.99
    ic = arr(1.0, 0.0, 1.0)
    L = O.lib()
    assert abs(L.oracle_pixel_alpha(3.5, 0.5, 0.5, 0.5, ic.ctypes.data, 1.0) - math.exp(-4.5)) < 1e-8  # 4.5 is kept
    assert L.oracle_pixel_alpha(3.6, 0.5, 0.5, 0.5, ic.ctypes.data, 1.0) == 0.0   # power 4.805 > 4.5
    assert abs(L.oracle_pixel_alpha(0.5, 0.5, 0.5, 0.5, ic.ctypes.data, 1.0) - f32(0.99)) == 0
    assert abs(L.oracle_pixel_alpha(1.5, 0.5, 0.5, 0.5, ic.ctypes.data, 0.5) - 0.5 * math.exp(-0.5)) < 1e-7


# ---- tests/test_projection.mojo:12-59 ----
def test_jacobian_analytical():
    out = np.zeros(6, np.float32)
    O.lib().oracle_jacobian(arr(0, 0, 10).ctypes.data, 1000.0, 1000.0, out.ctypes.data)
    assert abs(out[0] - 100) < 1e-4 and abs(out[4] - 100) < 1e-4 and abs(out[2]) < 1e-4 and abs(out[5]) < 1e-4
    O.lib().oracle_jacobian(arr(2, 3, 10).ctypes.data, 1000.0, 1000.0, out.ctypes.data)
    assert abs(out[2] + 20) < 1e-4 and abs(out[5] + 30) < 1e-4


def test_ewa_screen_covariance():
    out = np.zeros(3, np.float32)
    eye = np.eye(3, dtype=np.float32).reshape(-1)
    O.lib().oracle_ewa_cov2d(arr(1, 0, 0, 1, 0, 1).ctypes.data, arr(0, 0, 10).ctypes.data, eye.ctypes.data,
                             100.0, 100.0, 0.3, out.ctypes.data)
    assert abs(out[0] - 100.3) < 1e-3 and abs(out[2] - 100.3) < 1e-3 and abs(out[1]) < 1e-4
    inv = np.zeros(3, np.float32)
    O.lib().oracle_cov2d_inverse(out.ctypes.data, inv.ctypes.data)
    m = np.array([[out[0], out[1]], [out[1], out[2]]])
    mi = np.array([[inv[0], inv[1]], [inv[1], inv[2]]])
    p = m @ mi
    assert abs(p[0, 0] - 1) < 1e-4 and abs(p[1, 1] - 1) < 1e-4


# ---- tests/test_cholesky.mojo:10-27 ----
@pytest.mark.parametrize("cov,lmax,lmin,radius", [((16, 0, 9), 16, 9, 12), ((2, 1, 2), 3, 1, 6)])
def test_eigenvalues(cov, lmax, lmin, radius):
    lm = np.zeros(2, np.float32)
    r = np.zeros(1, np.int64)
    O.lib().oracle_eigen2x2(arr(*cov).ctypes.data, lm.ctypes.data, r.ctypes.data)
    assert abs(lm[0] - lmax) < 1e-5 and abs(lm[1] - lmin) < 1e-5 and int(r[0]) == radius


# ---- tests/test_covariance.mojo:11-37 ----
def _det(c):
    m = np.array([[c[0], c[1], c[2]], [c[1], c[3], c[4]], [c[2], c[4], c[5]]], np.float64)
    return np.linalg.det(m)


def test_covariance_axis_aligned():
    out = np.zeros(6, np.float32)
    O.lib().oracle_cov3d(arr(2, 3, 4).ctypes.data, arr(1, 0, 0, 0).ctypes.data, out.ctypes.data)
    assert np.allclose(out, [4, 0, 0, 9, 0, 16], atol=1e-5)
    assert abs(_det(out) - 576) < 1e-3


def test_covariance_rotation_invariance():
    h = f32(math.pi / 2) * f32(0.5)
    q = arr(math.cos(h), 0, math.sin(h), 0)
    out = np.zeros(6, np.float32)
    O.lib().oracle_cov3d(arr(1.5, 2.5, 3.5).ctypes.data, q.ctypes.data, out.ctypes.data)
    assert abs(_det(out) - (1.5 * 1.5 * 2.5 * 2.5 * 3.5 * 3.5)) < 1e-2


# ---- tests/test_spherical_harmonics.mojo:10-47 ----
def test_sh_basis_degrees():
    y = np.zeros(16, np.float32)
    O.lib().oracle_sh_basis(arr(0, 0, 1).ctypes.data, y.ctypes.data)
    assert abs(y[0] - 0.2820948) < 1e-5 and abs(y[1]) < 1e-5 and abs(y[3]) < 1e-5 and abs(y[2] - 0.4886025) < 1e-5
    O.lib().oracle_sh_basis(arr(0, 0, -1).ctypes.data, y.ctypes.data)
    assert abs(y[2] + 0.4886025) < 1e-5


def test_sh_color_evaluation():
    sh = np.zeros(48, np.float32)
    inv_y0 = f32(1.0) / f32(0.28209479)
    sh[0:3] = [(f32(0.8) - f32(0.5)) * inv_y0, (f32(0.4) - f32(0.5)) * inv_y0, (f32(0.2) - f32(0.5)) * inv_y0]
    out = np.zeros(3, np.float32)
    O.lib().oracle_sh_color(sh.ctypes.data, arr(0, 1, 0).ctypes.data, 0, out.ctypes.data)
    assert np.allclose(out, [0.8, 0.4, 0.2], atol=1e-4)


# ---- tests/test_culling.mojo:10-42 ----
def test_frustum_depth_culling():
    v = lambda z: O.lib().oracle_depth_visible(z, 0.1, 100.0)
    assert v(5.0) and v(0.1) and v(100.0)
    assert not v(-1.0) and not v(0.0) and not v(0.05) and not v(150.0)


def test_frustum_screen_culling():
    s = lambda x, y, r: O.lib().oracle_screen_box_visible(x, y, r, 800, 600)
    assert s(400.0, 300.0, 20) and s(-10.0, 300.0, 20) and s(810.0, 300.0, 20)
    assert not s(-50.0, 300.0, 20) and not s(900.0, 300.0, 20) and not s(400.0, -50.0, 20)
    assert not s(400.0, 700.0, 20)


# ---- tests/test_camera.mojo:11-34 ----
def test_camera_projection_center():
    cam = O.make_camera(ViewCamera((0, 0, 0), (1, 0, 0, 0), 800, 800, 640, 360, 0.01, 1000, 1280, 720))
    pc, ps = np.zeros(3, np.float32), np.zeros(2, np.float32)
    O.lib().oracle_world_to_screen(cam, arr(0, 0, 10).ctypes.data, pc.ctypes.data, ps.ctypes.data)
    assert np.allclose(ps, [640, 360], atol=1e-4)
    O.lib().oracle_world_to_screen(cam, arr(2, 0, 10).ctypes.data, pc.ctypes.data, ps.ctypes.data)
    assert np.allclose(ps, [800, 360], atol=1e-4)


# ---- tests/test_rasterizer.mojo:15-71 ----
def single_splat_case():
    cam = ViewCamera((0, 0, 0), (1, 0, 0, 0), 50, 50, 32, 32, 0.1, 100, 64, 64)
    sh = np.zeros((1, 48), np.float32)
    sh[0, :3] = [1.77245, -1.77245, -1.77245]
    return (arr(0, 0, 5).reshape(1, 3), arr(0.5, 0.5, 0.5).reshape(1, 3), arr(1, 0, 0, 0).reshape(1, 4),
            arr(1.0), sh, cam)


def test_single_splat_render():
    m, s, q, o, sh, cam = single_splat_case()
    r = O.render(m, s, q, o, sh, cam, RenderOptions())
    assert r.n_visible == 1 and r.n_instances > 0
    c = r.rgb[32, 32]
    assert c[0] > 0.8 and c[1] < 0.2 and c[2] < 0.2
    assert np.allclose(r.rgb[0, 0], 0, atol=1e-4)
    assert 4.5 < r.depth[32, 32] < 5.5


# ---- tests/test_regressions.mojo:26-57 ----
def test_regression_singular_covariance():
    c3 = np.zeros(6, np.float32)
    O.lib().oracle_cov3d(arr(1, 0, 0).ctypes.data, arr(1, 0, 0, 0).ctypes.data, c3.ctypes.data)
    c2 = np.zeros(3, np.float32)
    eye = np.eye(3, dtype=np.float32).reshape(-1)
    O.lib().oracle_ewa_cov2d(c3.ctypes.data, arr(0, 0, 2).ctypes.data, eye.ctypes.data, 100.0, 100.0, 0.3,
                             c2.ctypes.data)
    assert c2[0] * c2[2] - c2[1] * c2[1] > 0
    inv = np.zeros(3, np.float32)
    O.lib().oracle_cov2d_inverse(c2.ctypes.data, inv.ctypes.data)
    assert inv[0] > 0 and inv[2] > 0


# ---- tests/test_regressions.mojo:59-85 ----
def test_regression_behind_camera_culling():
    v = lambda z: O.lib().oracle_depth_visible(z, 0.5, 100.0)
    assert not v(-5.0) and not v(0.2) and v(5.0)


# ---- tests/test_regressions.mojo:115-146 ----
def test_regression_empty_and_extreme_rasterize():
    cam = ViewCamera((0, 0, 0), (1, 0, 0, 0), 20, 20, 16, 16, 0.1, 50, 32, 32)
    z = np.zeros((0, 3), np.float32)
    r = O.render(z, z, np.zeros((0, 4), np.float32), np.zeros(0, np.float32), np.zeros((0, 48), np.float32),
                 cam, RenderOptions())
    assert r.n_visible == 0
    r = O.render(arr(100000, 100000, 5).reshape(1, 3), arr(0.1, 0.1, 0.1).reshape(1, 3),
                 arr(1, 0, 0, 0).reshape(1, 4), arr(1.0), np.zeros((1, 48), np.float32), cam, RenderOptions())
    assert r.n_visible == 0


# ---- tests/test_loss.mojo:9-41 ----
def test_l1_loss_and_gradients():
    loss, g = O.l1_loss(np.zeros(4), np.zeros(4))
    assert abs(loss) < 1e-5
    loss, g = O.l1_loss([0.8, 0.2, 0.5, 0.1], [0.5] * 4)
    assert abs(loss - 0.25) < 1e-5
    assert abs(g[0] - 0.25) < 1e-5 and abs(g[1] + 0.25) < 1e-5 and abs(g[3] + 0.25) < 1e-5
    assert g[2] == 0.25   # diff == 0 takes the + branch (loss.mojo:28-33)


def test_multithreaded_oracle_matches_single_thread():
    from lumen_b200 import scenes
    sc = scenes.grid_scene(0)
    s, o = sc.activated()
    cam = scenes.camera_config0()
    a = O.render(sc.means, s, sc.quats, o, sc.sh, cam, RenderOptions(), nthreads=1)
    b = O.render(sc.means, s, sc.quats, o, sc.sh, cam, RenderOptions(), nthreads=4)
    assert np.array_equal(a.rgb, b.rgb) and np.array_equal(a.n_contrib, b.n_contrib)
    assert np.array_equal(a.keys_sorted, b.keys_sorted) and np.array_equal(a.vals_sorted, b.vals_sorted)
