"""SDK engine: the reference Python SDK's ``LumenEngine.render(cloud, camera)
-> RenderResult`` (python/lumen/client.py:40-219), same signature, same
``RasterizerConfig`` and ``RenderResult`` fields, executed by liblumen's
``lumen_rasterize`` (include/lumen.h) on the GPU.

The reference loads liblumen through ctypes and never calls it
(client.py:45,47-65); here the library is the engine. There is no CPU
fallback: without liblumen.so or a CUDA device, render raises LumenError.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any, Dict, List, Optional

import numpy as np

from . import _lib as L
from .camera import Camera
from .cloud import GaussianCloud


@dataclass
class RasterizerConfig:
    """Reference client.py:17-26."""
    image_width: int = 400
    image_height: int = 300
    tile_size: int = 16
    near_plane: float = 0.1
    far_plane: float = 50.0
    early_termination_alpha: float = 0.99
    gaussian_radius_sigma: float = 3.0


@dataclass
class RenderResult:
    """Reference client.py:29-37: rgb_bytes is HWC uint8, depth_values is the
    alpha-weighted depth (1000 where nothing was drawn), alpha_values is 1 - T."""
    width: int
    height: int
    rgb_bytes: bytes
    depth_values: List[float]
    alpha_values: List[float]
    stats: Dict[str, Any]


class LumenEngine:
    """Gaussian-splatting engine on liblumen (reference client.py:40-67)."""

    def __init__(self, config: Optional[RasterizerConfig] = None):
        self.config = config if config is not None else RasterizerConfig()
        self._c_lib = L.load()
        self._rasterizer = None
        self._cloud = None
        self._cloud_key = None

    def __del__(self):
        lib = getattr(self, "_c_lib", None)
        if lib is None:
            return
        if self._rasterizer:
            lib.lumen_rasterizer_destroy(self._rasterizer)
        if self._cloud:
            lib.lumen_cloud_destroy(self._cloud)

    def _c_config(self) -> L.LumenConfig:
        c = L.LumenConfig()
        cfg = self.config
        c.image_width, c.image_height, c.tile_size = cfg.image_width, cfg.image_height, cfg.tile_size
        c.near_plane, c.far_plane = cfg.near_plane, cfg.far_plane
        c.early_termination_alpha, c.gaussian_radius_sigma = cfg.early_termination_alpha, cfg.gaussian_radius_sigma
        return c

    def _upload(self, cloud: GaussianCloud):
        """A liblumen cloud for this GaussianCloud. Array-backed clouds are
        uploaded once and reused while their array is unchanged; list-backed
        clouds are packed on every call (their splats may have been edited)."""
        aos = np.ascontiguousarray(cloud.to_aos(), dtype=np.float32)
        key = ("array", id(aos)) if cloud._aos is aos else None
        if self._cloud is not None and key is not None and key == self._cloud_key:
            return self._cloud
        lib = self._c_lib
        if self._cloud is not None:
            lib.lumen_cloud_destroy(self._cloud)
        handle = lib.lumen_cloud_create(max(1, aos.shape[0]))
        if not handle:
            raise L.LumenError(-2, "cloud_create")
        L.check(lib.lumen_cloud_append(handle, aos.ctypes.data_as(C.POINTER(L.LumenGaussian)), aos.shape[0]),
                "cloud_append")
        self._cloud, self._cloud_key = handle, key
        return handle

    def render(self, cloud: GaussianCloud, camera: Camera) -> RenderResult:
        """Render cloud from camera at the configured resolution."""
        lib = self._c_lib
        w, h = int(self.config.image_width), int(self.config.image_height)
        cfg = self._c_config()
        if self._rasterizer is None:
            self._rasterizer = lib.lumen_rasterizer_create(C.byref(cfg))
            if not self._rasterizer:
                raise L.LumenError(-3, "rasterizer_create (no usable CUDA device)")
        else:
            L.check(lib.lumen_rasterizer_set_config(self._rasterizer, C.byref(cfg)), "set_config")
        handle = self._upload(cloud)
        cam = L.LumenCamera(L.LumenVec3(*camera.position), L.LumenVec3(*camera.target), L.LumenVec3(*camera.up),
                            camera.fov_x_deg, camera.fov_y_deg, camera.near_plane, camera.far_plane)
        fb = lib.lumen_framebuffer_create(w, h)
        if not fb:
            raise L.LumenError(-2, "framebuffer_create")
        try:
            st = L.LumenStats()
            L.check(lib.lumen_rasterize(self._rasterizer, handle, C.byref(cam), fb, C.byref(st)), "rasterize")
            f = fb.contents
            n = w * h
            rgb = bytes(C.string_at(f.rgb_data, n * 3))
            depth = np.ctypeslib.as_array(f.depth_data, shape=(n,)).astype(np.float64).tolist()
            alpha = np.ctypeslib.as_array(f.alpha_data, shape=(n,)).astype(np.float64).tolist()
        finally:
            lib.lumen_framebuffer_destroy(fb)
        ms = float(st.rasterize_time_ms)
        stats = {"total_splats": int(st.total_splats), "visible_splats": int(st.visible_splats),
                 "culled_splats": int(st.culled_splats), "total_tiles": int(st.total_tiles),
                 "touched_tiles": int(st.touched_tiles), "elapsed_ms": ms,
                 "fps": (1000.0 / ms) if ms > 0 else 1000.0}
        return RenderResult(w, h, rgb, depth, alpha, stats)
