"""Picking on the device (include/lumen_spatial.h): the reference's LBVH
(src/spatial/bvh.mojo:29-120) built from Morton codes with the library's
radix sort, and raycast_closest_splat (src/spatial/raycast.mojo:30-95) for
batches of rays or of pixel positions under a camera."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib as L
from . import render as R
from .types import ViewCamera

NODE_BYTES = 32
HIT_BYTES = 24


@dataclass
class RayHit:
    """raycast.mojo:11-27."""
    hit: bool
    splat_index: int
    distance: float
    point: tuple


def _hits_from(buf: torch.Tensor):
    raw = buf.cpu().numpy()
    head = raw.view(np.int32).reshape(-1, 6)
    flt = raw.view(np.float32).reshape(-1, 6)
    return [RayHit(bool(head[i, 0]), int(head[i, 1]), float(flt[i, 2]), tuple(float(v) for v in flt[i, 3:6]))
            for i in range(head.shape[0])]


class LBVH:
    """The hierarchy over a scene's Gaussians, resident on its device.
    nodes: [node_count, 8] 32-bit words (min xyz, left, max xyz, right),
    leaves first in Morton order, the root last (the reference's numbering)."""

    def __init__(self, means: torch.Tensor, scales: torch.Tensor):
        self.lib = L.load()
        n = int(means.shape[0])
        self.means = means.reshape(n, 3).float().contiguous()
        self.scales = scales.reshape(n, 3).float().contiguous()
        dev = self.means.device
        nc = int(self.lib.lumen_bvh_node_count(n))
        self.nodes = torch.empty((max(nc, 1), 8), dtype=torch.int32, device=dev)
        self.splat_index = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
        self.struct = L.LumenGpuBvh()
        self.struct.nodes, self.struct.splat_index = self.nodes.data_ptr(), self.splat_index.data_ptr()
        scratch = torch.empty(max(int(self.lib.lumen_gpu_bvh_scratch_bytes(n)), 1), dtype=torch.uint8, device=dev)
        g = self._gaussians()
        stream = torch.cuda.current_stream(dev).cuda_stream
        L.check(self.lib.lumen_gpu_bvh_build(C.byref(g), C.byref(self.struct), scratch.data_ptr(), scratch.numel(),
                                             stream), "bvh_build")

    @classmethod
    def build_from_cloud(cls, scene) -> "LBVH":
        """From a lumen_b200.render.Scene (means and scales are read)."""
        means, scales = scene.tensors[0], scene.tensors[1]
        return cls(means, scales)

    def _gaussians(self) -> L.LumenGpuGaussians:
        g = L.LumenGpuGaussians()
        g.means, g.scales, g.count = self.means.data_ptr(), self.scales.data_ptr(), int(self.means.shape[0])
        return g

    @property
    def root_index(self) -> int:
        return int(self.struct.root_index)

    def node_count(self) -> int:
        return int(self.struct.node_count)

    def raycast(self, rays: torch.Tensor, max_dist: float = 1000.0) -> torch.Tensor:
        """rays: [n, 6] float32 (origin, direction) on the device. Returns the
        hits as raw [n, 6] 32-bit words (hit, splat, distance, point xyz);
        ``hits()`` turns them into RayHit records."""
        rays = rays.reshape(-1, 6).float().contiguous()
        n = int(rays.shape[0])
        out = torch.empty((max(n, 1), 6), dtype=torch.int32, device=rays.device)
        g = self._gaussians()
        stream = torch.cuda.current_stream(rays.device).cuda_stream
        L.check(self.lib.lumen_gpu_raycast(C.byref(self.struct), C.byref(g), rays.data_ptr(), n, float(max_dist),
                                           out.data_ptr(), stream), "raycast")
        return out[:n]

    def pick(self, camera: ViewCamera, pixels: torch.Tensor, max_dist: float = 1000.0,
             rays_out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Closest Gaussian under each pixel position ([n, 2] float32 x, y):
        generate_ray (camera.mojo:85-90) then the cast. Raw hits as raycast."""
        px = pixels.reshape(-1, 2).float().contiguous()
        n = int(px.shape[0])
        out = torch.empty((max(n, 1), 6), dtype=torch.int32, device=px.device)
        g = self._gaussians()
        cam = L.view_camera(camera)
        stream = torch.cuda.current_stream(px.device).cuda_stream
        L.check(self.lib.lumen_gpu_pick_pixels(C.byref(self.struct), C.byref(g), C.byref(cam), px.data_ptr(), n,
                                               float(max_dist), None if rays_out is None else rays_out.data_ptr(),
                                               out.data_ptr(), stream), "pick_pixels")
        return out[:n]

    @staticmethod
    def hits(raw: torch.Tensor):
        return _hits_from(raw.contiguous())


def raycast_closest_splat(bvh: LBVH, origin: Sequence[float], direction: Sequence[float],
                          max_dist: float = 1000.0) -> RayHit:
    """One ray (the reference's signature, with the cloud held by the LBVH)."""
    r = torch.tensor([list(origin) + list(direction)], dtype=torch.float32, device=bvh.means.device)
    return LBVH.hits(bvh.raycast(r, max_dist))[0]
