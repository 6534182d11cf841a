"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s cpu_baseline leg and
reference arm import this module, as the checker and the timed CPU baseline.
The oracle restates the reference's Mojo forward path
(src/raster/pipeline.mojo:48-231), its training-step pieces (optimizer,
density control, PSNR, view-space accumulation), the depth-buffer
products and picking (Morton codes, LBVH, ray casts); see lumen_oracle.cpp and
train_oracle.cpp, depth_oracle.cpp and spatial_oracle.cpp for the
per-function citations. Parity pinning: the reference's own known-answer tests, restated in
tests/test_oracle_kat.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblumen_oracle.so")
_lib = None


class OracleCamera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("rotation", C.c_float * 4),
                ("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("near_plane", C.c_float), ("far_plane", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32)]


class OracleOptions(C.Structure):
    _fields_ = [("lowpass", C.c_float), ("sh_degree", C.c_int32), ("white_background", C.c_int32),
                ("compute_depth", C.c_int32), ("key_mode", C.c_int32), ("term_mode", C.c_int32),
                ("params_are_logits", C.c_int32), ("tile_size", C.c_int32), ("term_threshold", C.c_float)]


RECORD_DTYPE = np.dtype([("cx", "<f4"), ("cy", "<f4"), ("depth", "<f4"), ("ic00", "<f4"),
                         ("ic01", "<f4"), ("ic11", "<f4"), ("r", "<f4"), ("g", "<f4"),
                         ("b", "<f4"), ("opacity", "<f4")])

_P = C.c_void_p


class OracleOutputs(C.Structure):
    _fields_ = [("rgb", _P), ("depth", _P), ("alpha", _P), ("n_contrib", _P), ("last_idx", _P),
                ("records", _P), ("records_cap", C.c_int64),
                ("keys_unsorted", _P), ("vals_unsorted", _P),
                ("keys_sorted", _P), ("vals_sorted", _P), ("keys_cap", C.c_int64),
                ("ranges", _P), ("radii", _P),
                ("n_visible", C.c_int64), ("n_instances", C.c_int64)]


def build() -> str:
    """Compile the oracle with its Makefile if the library is missing."""
    if not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-C", _HERE, "liblumen_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB_PATH)
        _lib.oracle_render_f32.restype = C.c_int
        _lib.oracle_render_f32.argtypes = [_P] * 5 + [C.c_int64, C.POINTER(OracleCamera),
                                                      C.POINTER(OracleOptions), C.POINTER(OracleOutputs), C.c_int]
        _lib.oracle_render_f64.restype = C.c_int
        _lib.oracle_render_f64.argtypes = [_P] * 5 + [C.c_int64, C.POINTER(OracleCamera),
                                                      C.POINTER(OracleOptions), _P, _P, _P, _P]
        _lib.oracle_radix_sort64.argtypes = [_P, _P, C.c_int64, C.c_int]
        _lib.oracle_tile_ranges.argtypes = [_P, C.c_int64, C.c_int64, _P]
        _lib.oracle_encode_key.restype = C.c_uint64
        _lib.oracle_encode_key.argtypes = [C.c_uint32, C.c_float, C.c_int]
        _lib.oracle_l1_loss.restype = C.c_float
        _lib.oracle_l1_loss.argtypes = [_P, _P, C.c_int64, _P]
        _lib.oracle_position_lr.restype = C.c_float
        _lib.oracle_position_lr.argtypes = [C.c_float, C.c_float, C.c_int32, C.c_int64]
        _lib.oracle_adam_scalars.argtypes = [C.c_float, C.c_float, C.c_int64, _P, _P]
        _lib.oracle_adam_step.argtypes = [_P] * 8 + [C.c_int64] + [C.c_float] * 7
        _lib.oracle_densify_and_prune.restype = C.c_int64
        _lib.oracle_densify_and_prune.argtypes = ([_P] * 7 + [C.c_int64, C.c_float, C.c_float, C.c_float] +
                                                  [_P] * 13 + [_P, _P, _P])
        _lib.oracle_reset_opacities.argtypes = [_P, C.c_int64, C.c_float]
        _lib.oracle_psnr.restype = C.c_float
        _lib.oracle_psnr.argtypes = [_P, _P, C.c_int64]
        _lib.oracle_accumulate_viewspace.argtypes = [_P, C.c_int32, _P, C.c_int64, C.c_float, C.c_float, _P, _P]
        _lib.oracle_depth_min_max.argtypes = [_P, C.c_int64, _P, _P]
        _lib.oracle_depth_normal.argtypes = [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P]
        _lib.oracle_depth_normals.argtypes = [_P, C.c_int32, C.c_int32, _P]
        _lib.oracle_depth_heatmap.argtypes = [_P, C.c_int64, C.c_double, C.c_double, _P]
        _lib.oracle_expand_bits.restype = C.c_uint32
        _lib.oracle_expand_bits.argtypes = [C.c_uint32]
        _lib.oracle_morton3d.restype = C.c_uint32
        _lib.oracle_morton3d.argtypes = [C.c_float] * 3
        _lib.oracle_bvh_build.restype = C.c_int64
        _lib.oracle_bvh_build.argtypes = [_P, _P, C.c_int64, _P, _P, _P]
        _lib.oracle_raycast.argtypes = [_P, _P, C.c_int64, C.c_int64, _P, _P, C.c_int64, _P, _P, C.c_float, _P]
        _lib.oracle_generate_ray.argtypes = [C.POINTER(OracleCamera), C.c_float, C.c_float, _P]
        _lib.oracle_ray_direction.argtypes = [_P, _P]
        for name, args in [("oracle_ewa_cov2d", [_P, _P, _P, C.c_float, C.c_float, C.c_float, _P]),
                           ("oracle_jacobian", [_P, C.c_float, C.c_float, _P]),
                           ("oracle_cov3d", [_P, _P, _P]),
                           ("oracle_eigen2x2", [_P, _P, _P]),
                           ("oracle_cov2d_inverse", [_P, _P]),
                           ("oracle_sh_basis", [_P, _P]),
                           ("oracle_sh_color", [_P, _P, C.c_int, _P]),
                           ("oracle_world_to_screen", [C.POINTER(OracleCamera), _P, _P, _P])]:
            getattr(_lib, name).argtypes = args
            getattr(_lib, name).restype = None
        _lib.oracle_depth_visible.argtypes = [C.c_float, C.c_float, C.c_float]
        _lib.oracle_screen_box_visible.argtypes = [C.c_float, C.c_float, C.c_int64, C.c_int32, C.c_int32]
        _lib.oracle_blend_sequence.restype = C.c_int
        _lib.oracle_blend_sequence.argtypes = [_P, _P, _P, C.c_int, C.c_int, _P, _P, _P, _P]
        _lib.oracle_pixel_alpha.restype = C.c_float
        _lib.oracle_pixel_alpha.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, _P, C.c_float]
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def make_camera(cam) -> OracleCamera:
    c = OracleCamera()
    c.position[:] = [float(v) for v in cam.position]
    c.rotation[:] = [float(v) for v in cam.rotation]
    c.fx, c.fy, c.cx, c.cy = float(cam.fx), float(cam.fy), float(cam.cx), float(cam.cy)
    c.near_plane, c.far_plane = float(cam.near_plane), float(cam.far_plane)
    c.width, c.height = int(cam.width), int(cam.height)
    return c


def make_options(opt) -> OracleOptions:
    o = OracleOptions()
    o.lowpass = float(opt.lowpass)
    o.sh_degree = int(opt.sh_degree)
    o.white_background = int(bool(opt.white_background))
    o.compute_depth = int(bool(opt.compute_depth))
    o.key_mode = int(opt.key_mode)
    o.term_mode = int(opt.term_mode)
    o.params_are_logits = int(bool(opt.params_are_logits))
    o.tile_size = int(opt.tile_size)
    o.term_threshold = float(opt.term_threshold)
    return o


@dataclass
class OracleResult:
    rgb: np.ndarray
    depth: np.ndarray
    alpha: np.ndarray
    n_contrib: np.ndarray
    last_idx: np.ndarray
    n_visible: int
    n_instances: int
    records: Optional[np.ndarray] = None
    keys_unsorted: Optional[np.ndarray] = None
    vals_unsorted: Optional[np.ndarray] = None
    keys_sorted: Optional[np.ndarray] = None
    vals_sorted: Optional[np.ndarray] = None
    ranges: Optional[np.ndarray] = None
    radii: Optional[np.ndarray] = None


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def render(means, scales, quats, opacities, sh, cam, opt, stages: bool = True,
           nthreads: int = 1) -> OracleResult:
    """Float32 forward. ``scales``/``opacities`` are activated unless
    ``opt.params_are_logits`` (then log-scales and logits)."""
    L = lib()
    means, scales, quats, opacities, sh = (_f32(means), _f32(scales), _f32(quats),
                                           _f32(opacities).reshape(-1), _f32(sh).reshape(-1, 48))
    n = means.shape[0]
    H, W = int(cam.height), int(cam.width)
    tiles = ((W + 15) // 16) * ((H + 15) // 16)
    rgb = np.zeros((H, W, 3), np.float32)
    depth = np.zeros((H, W), np.float32)
    alpha = np.zeros((H, W), np.float32)
    nc = np.zeros((H, W), np.uint32)
    last = np.zeros((H, W), np.int32)
    out = OracleOutputs()
    out.rgb, out.depth, out.alpha, out.n_contrib, out.last_idx = (_ptr(rgb), _ptr(depth), _ptr(alpha),
                                                                  _ptr(nc), _ptr(last))
    ocam, oopt = make_camera(cam), make_options(opt)
    rec = ks = vs = ku = vu = ranges = radii = None
    if stages:
        rec = np.zeros(max(n, 1), RECORD_DTYPE)
        ranges = np.zeros((tiles, 2), np.int32)
        radii = np.zeros(max(n, 1), np.int32)
        out.records, out.records_cap = _ptr(rec), n
        out.ranges, out.radii = _ptr(ranges), _ptr(radii)
        # first call sizes the key buffers
        out.keys_cap = 0
        st = L.oracle_render_f32(_ptr(means), _ptr(scales), _ptr(quats), _ptr(opacities), _ptr(sh), n,
                                 C.byref(ocam), C.byref(oopt), C.byref(out), nthreads)
        k = int(out.n_instances)
        ku, vu = np.zeros(max(k, 1), np.uint64), np.zeros(max(k, 1), np.uint32)
        ks, vs = np.zeros(max(k, 1), np.uint64), np.zeros(max(k, 1), np.uint32)
        out.keys_unsorted, out.vals_unsorted = _ptr(ku), _ptr(vu)
        out.keys_sorted, out.vals_sorted = _ptr(ks), _ptr(vs)
        out.keys_cap = k
    st = L.oracle_render_f32(_ptr(means), _ptr(scales), _ptr(quats), _ptr(opacities), _ptr(sh), n,
                             C.byref(ocam), C.byref(oopt), C.byref(out), nthreads)
    assert st == 0, "oracle stage buffers too small"
    V, K = int(out.n_visible), int(out.n_instances)
    r = OracleResult(rgb, depth, alpha, nc, last, V, K)
    if stages:
        r.records = rec[:V]
        r.keys_unsorted, r.vals_unsorted = ku[:K], vu[:K]
        r.keys_sorted, r.vals_sorted = ks[:K], vs[:K]
        r.ranges, r.radii = ranges, radii[:n]
    return r


def render_f64(means, scales, quats, opacities, sh, cam, opt):
    """Float64 forward: (rgb, depth, alpha, decision_hash)."""
    L = lib()
    d = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    means, scales, quats, opacities, sh = d(means), d(scales), d(quats), d(opacities).reshape(-1), d(sh).reshape(-1, 48)
    H, W = int(cam.height), int(cam.width)
    rgb = np.zeros((H, W, 3), np.float64)
    depth = np.zeros((H, W), np.float64)
    alpha = np.zeros((H, W), np.float64)
    h = np.zeros(1, np.uint64)
    ocam, oopt = make_camera(cam), make_options(opt)
    L.oracle_render_f64(_ptr(means), _ptr(scales), _ptr(quats), _ptr(opacities), _ptr(sh), means.shape[0],
                        C.byref(ocam), C.byref(oopt), _ptr(rgb), _ptr(depth), _ptr(alpha), _ptr(h))
    return rgb, depth, alpha, int(h[0])


def radix_sort64(keys: np.ndarray, vals: np.ndarray, nthreads: int = 1):
    k = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    v = np.ascontiguousarray(vals, dtype=np.uint32).copy()
    lib().oracle_radix_sort64(_ptr(k), _ptr(v), k.shape[0], nthreads)
    return k, v


def tile_ranges(sorted_keys: np.ndarray, total_tiles: int) -> np.ndarray:
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint64)
    r = np.zeros((total_tiles, 2), np.int32)
    lib().oracle_tile_ranges(_ptr(k), k.shape[0], total_tiles, _ptr(r))
    return r


def encode_key(tile_id: int, depth: float, key_mode: int = 0) -> int:
    return int(lib().oracle_encode_key(tile_id, depth, key_mode))


def l1_loss(pred, target):
    p, t = _f32(pred).reshape(-1), _f32(target).reshape(-1)
    g = np.zeros_like(p)
    loss = lib().oracle_l1_loss(_ptr(p), _ptr(t), p.shape[0], _ptr(g))
    return float(loss), g


# ---------------------------------------------------------------- training step

ADAM_BETA1, ADAM_BETA2, ADAM_EPS = np.float32(0.9), np.float32(0.999), np.float32(1e-8)


def position_lr(init, final, iterations, iteration) -> float:
    return float(lib().oracle_position_lr(float(init), float(final), int(iterations), int(iteration)))


def adam_scalars(beta1, beta2, step):
    a, b = np.zeros(1, np.float32), np.zeros(1, np.float32)
    lib().oracle_adam_scalars(float(beta1), float(beta2), int(step), _ptr(a), _ptr(b))
    return float(a[0]), float(b[0])


def adam_step(means, opacities, grad_means, grad_op, m_pos, v_pos, m_op, v_op, pos_lr, opacity_lr, step):
    """One AdamOptimizer.step in place on float32 arrays (means and moments
    N x 3, opacities and their moments N); step is the counter after the
    increment."""
    for a in (means, opacities, m_pos, v_pos, m_op, v_op):
        assert a.dtype == np.float32 and a.flags.c_contiguous
    gm, go = _f32(grad_means), _f32(grad_op)
    ib1, ib2 = adam_scalars(ADAM_BETA1, ADAM_BETA2, step)
    lib().oracle_adam_step(_ptr(means), _ptr(opacities), _ptr(gm), _ptr(go), _ptr(m_pos), _ptr(v_pos), _ptr(m_op),
                           _ptr(v_op), means.shape[0], float(pos_lr), float(opacity_lr), float(ADAM_BETA1),
                           float(ADAM_BETA2), float(ADAM_EPS), ib1, ib2)


def densify_and_prune(means, scales, quats, opacities, sh, vs_sum, vs_count, grad_thr, prune_thr, extent,
                      moments=None):
    """densify_and_prune on copies: returns (cloud dict, moments dict or None,
    (cloned, split, pruned)). moments: dict m_pos, v_pos, m_op, v_op."""
    f = lambda a, s: np.ascontiguousarray(a, np.float32).reshape(s)
    n = int(np.asarray(means).shape[0])
    src = [f(means, (n, 3)), f(scales, (n, 3)), f(quats, (n, 4)), f(opacities, (n,)), f(sh, (n, 48))]
    vs, vc = f(vs_sum, (n,)), np.ascontiguousarray(vs_count, np.int32).reshape(n)
    cap = 2 * max(n, 1)
    out = [np.zeros((cap,) + a.shape[1:], np.float32) for a in src]
    names = ("m_pos", "v_pos", "m_op", "v_op")
    sm = [f(moments[k], (n, 3) if k.endswith("pos") else (n,)) for k in names] if moments else [None] * 4
    dm = [np.zeros((cap,) + m.shape[1:], np.float32) for m in sm] if moments else [None] * 4
    c, s, p = (np.zeros(1, np.int64) for _ in range(3))
    k = lib().oracle_densify_and_prune(*[_ptr(a) for a in src], _ptr(vs), _ptr(vc), n, float(grad_thr),
                                       float(prune_thr), float(extent), *[_ptr(a) for a in out],
                                       *[_ptr(a) for a in sm], *[_ptr(a) for a in dm], _ptr(c), _ptr(s), _ptr(p))
    cloud = {name: a[:k] for name, a in zip(("means", "scales", "quats", "opacities", "sh"), out)}
    mom = {name: a[:k] for name, a in zip(names, dm)} if moments else None
    return cloud, mom, (int(c[0]), int(s[0]), int(p[0]))


def reset_opacities(op, max_value=0.01):
    assert op.dtype == np.float32 and op.flags.c_contiguous
    lib().oracle_reset_opacities(_ptr(op), op.shape[0], float(max_value))


def psnr(pred, target) -> float:
    p, t = _f32(pred).reshape(-1), _f32(target).reshape(-1)
    return float(lib().oracle_psnr(_ptr(p), _ptr(t), p.shape[0]))


def accumulate_viewspace(grad2d, stride, radii, vs_sum, vs_count, scale_x=1.0, scale_y=1.0):
    """In place on vs_sum (float32) and vs_count (int32)."""
    g = _f32(grad2d)
    r = np.ascontiguousarray(radii, np.int32)
    lib().oracle_accumulate_viewspace(_ptr(g), int(stride), _ptr(r), r.shape[0], float(scale_x), float(scale_y),
                                      _ptr(vs_sum), _ptr(vs_count))


# ---------------------------------------------------------------- depth products

def depth_min_max(depth):
    d = _f32(depth).reshape(-1)
    lo, hi = np.zeros(1, np.float32), np.zeros(1, np.float32)
    lib().oracle_depth_min_max(_ptr(d), d.shape[0], _ptr(lo), _ptr(hi))
    return float(lo[0]), float(hi[0])


def depth_normal(depth, x, y):
    d = _f32(depth)
    h, w = d.shape
    out = np.zeros(3, np.float32)
    lib().oracle_depth_normal(_ptr(d), w, h, x, y, _ptr(out))
    return out


def depth_normals(depth):
    d = _f32(depth)
    h, w = d.shape
    out = np.zeros((h, w, 3), np.float32)
    lib().oracle_depth_normals(_ptr(d), w, h, _ptr(out))
    return out


def depth_heatmap(depth, near_plane=0.5, far_plane=10.0):
    d = _f32(depth)
    out = np.zeros(d.shape + (3,), np.uint8)
    lib().oracle_depth_heatmap(_ptr(d), d.size, float(near_plane), float(far_plane), _ptr(out))
    return out


# ---------------------------------------------------------------- picking

BVH_NODE_DTYPE = np.dtype([("min_pt", "<f4", 3), ("left_child", "<i4"), ("max_pt", "<f4", 3),
                           ("right_child", "<i4")])
RAY_HIT_DTYPE = np.dtype([("hit", "<i4"), ("splat_index", "<i4"), ("distance", "<f4"), ("point", "<f4", 3)])


def expand_bits(v: int) -> int:
    return int(lib().oracle_expand_bits(int(v)))


def morton3d(nx, ny, nz) -> int:
    return int(lib().oracle_morton3d(float(nx), float(ny), float(nz)))


def bvh_build(means, scales):
    """LBVH.build_from_cloud: (nodes [BVH_NODE_DTYPE], splat_index [n] int32,
    root index, Morton codes [n] uint32 in input order)."""
    m, s = _f32(means).reshape(-1, 3), _f32(scales).reshape(-1, 3)
    n = m.shape[0]
    total, count = n, n
    while count > 1:
        count = (count + 1) // 2
        total += count
    nodes = np.zeros(max(total, 1), BVH_NODE_DTYPE)
    idx = np.zeros(max(n, 1), np.int32)
    codes = np.zeros(max(n, 1), np.uint32)
    k = lib().oracle_bvh_build(_ptr(m), _ptr(s), n, nodes.ctypes.data, _ptr(idx), _ptr(codes))
    return nodes[:k], idx[:n], k - 1 if k > 0 else -1, codes[:n]


def raycast(nodes, splat_index, root, means, scales, origin, direction, max_dist=1000.0, unit=False):
    """raycast_closest_splat for one ray: a RAY_HIT_DTYPE record. The ray is
    Ray3f(origin, direction), which normalises the direction; unit=True
    passes a Ray3f's stored direction (from generate_ray) as it is."""
    m, s = _f32(means).reshape(-1, 3), _f32(scales).reshape(-1, 3)
    nd = np.ascontiguousarray(nodes, BVH_NODE_DTYPE)
    si = np.ascontiguousarray(splat_index, np.int32)
    o, d = _f32(origin).reshape(3), _f32(direction).reshape(3).copy()
    if not unit:
        dn = np.zeros(3, np.float32)
        lib().oracle_ray_direction(_ptr(d), _ptr(dn))
        d = dn
    out = np.zeros(1, RAY_HIT_DTYPE)
    lib().oracle_raycast(nd.ctypes.data, _ptr(si), nd.shape[0], int(root), _ptr(m), _ptr(s), m.shape[0], _ptr(o),
                         _ptr(d), float(max_dist), out.ctypes.data)
    return out[0]


def generate_ray(cam, px, py):
    """PinholeCamera.generate_ray: (origin [3], unit direction [3])."""
    oc = make_camera(cam)
    out = np.zeros(6, np.float32)
    lib().oracle_generate_ray(C.byref(oc), float(px), float(py), _ptr(out))
    return out[:3], out[3:]
