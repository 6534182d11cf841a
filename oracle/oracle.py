"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s cpu_baseline leg and
reference arm import this module, as the checker and the timed CPU baseline.
The oracle restates the reference's Mojo forward path
(src/raster/pipeline.mojo:48-231); see lumen_oracle.cpp for the per-function
citations. Parity pinning: the reference's own known-answer tests, restated in
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
