"""Products of a rendered depth buffer on the device (include/lumen_depth.h).

``DepthMap`` mirrors the reference's DepthMap (src/raster/depth_map.mojo:9-68:
get_depth, set_depth, compute_min_max, extract_normal) over a device buffer;
``products`` computes the range, the per-pixel normals and the SDK's depth
heatmap (python/lumen/visualizer.py:16-48) in one pass with
lumen_gpu_depth_products.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Tuple

import torch

from . import _lib as L


@dataclass
class DepthProducts:
    range: Optional[torch.Tensor]      # [2] float32 (min, max) on the device
    normals: Optional[torch.Tensor]    # [H, W, 3] float32
    heatmap: Optional[torch.Tensor]    # [H, W, 3] uint8


def _check_depth(depth: torch.Tensor) -> torch.Tensor:
    if not isinstance(depth, torch.Tensor) or not depth.is_cuda or depth.dtype != torch.float32 or depth.dim() != 2:
        raise ValueError("depth must be a [height, width] float32 CUDA tensor")
    return depth.contiguous()


def products(depth: torch.Tensor, normals: bool = True, range: bool = True, heatmap: bool = False,
             near_plane: float = 0.5, far_plane: float = 10.0) -> DepthProducts:
    """One pass over the depth buffer on its device's current stream (no wait)."""
    depth = _check_depth(depth)
    h, w = depth.shape
    dev = depth.device
    out = DepthProducts(torch.empty(2, dtype=torch.float32, device=dev) if range else None,
                        torch.empty((h, w, 3), dtype=torch.float32, device=dev) if normals else None,
                        torch.empty((h, w, 3), dtype=torch.uint8, device=dev) if heatmap else None)
    s = L.LumenDepthProducts()
    s.range = out.range.data_ptr() if range else None
    s.normals = out.normals.data_ptr() if normals else None
    s.heatmap = out.heatmap.data_ptr() if heatmap else None
    s.near_plane, s.far_plane = float(near_plane), float(far_plane)
    stream = torch.cuda.current_stream(dev).cuda_stream
    L.check(L.load().lumen_gpu_depth_products(depth.data_ptr(), w, h, C.byref(s), stream), "depth_products")
    return out


def min_max(depth: torch.Tensor) -> Tuple[float, float]:
    r = products(depth, normals=False, range=True).range.cpu()
    return float(r[0]), float(r[1])


def normals(depth: torch.Tensor) -> torch.Tensor:
    return products(depth, normals=True, range=False).normals


def heatmap(depth: torch.Tensor, near_plane: float = 0.5, far_plane: float = 10.0) -> torch.Tensor:
    if far_plane == near_plane:
        raise ZeroDivisionError("far_plane equals near_plane")
    return products(depth, normals=False, range=False, heatmap=True, near_plane=near_plane,
                    far_plane=far_plane).heatmap


class DepthMap:
    """A width x height float32 depth buffer on the device, zero-initialised
    like the reference's (depth_map.mojo:17-20)."""

    def __init__(self, width: int, height: int, device="cuda", buffer: Optional[torch.Tensor] = None):
        self.width, self.height = int(width), int(height)
        if buffer is None:
            buffer = torch.zeros((self.height, self.width), dtype=torch.float32, device=device)
        self.buffer = _check_depth(buffer)
        self._normals = None

    @classmethod
    def from_render(cls, result) -> "DepthMap":
        """The depth output of a render (lumen_b200.render.render)."""
        d = result.depth
        return cls(d.shape[1], d.shape[0], buffer=d)

    def get_depth(self, x: int, y: int) -> float:
        if 0 <= x < self.width and 0 <= y < self.height:
            return float(self.buffer[y, x].item())
        return 0.0

    def set_depth(self, x: int, y: int, val: float) -> None:
        if 0 <= x < self.width and 0 <= y < self.height:
            self.buffer[y, x] = val
            self._normals = None

    def compute_min_max(self) -> Tuple[float, float]:
        return min_max(self.buffer)

    def normals(self) -> torch.Tensor:
        if self._normals is None:
            self._normals = normals(self.buffer)
        return self._normals

    def extract_normal(self, x: int, y: int) -> Tuple[float, float, float]:
        n = self.normals()[y, x].cpu()
        return float(n[0]), float(n[1]), float(n[2])
