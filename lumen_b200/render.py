"""Device-resident forward render through the C ABI (lumen_gpu_render_forward).

PyTorch supplies device memory and the current CUDA stream; all computation
is in liblumen.so. This is the Python form of the reference's
``rasterize_scene(cloud, camera, config) -> RenderOutput``
(src/raster/pipeline.mojo:48-52): it returns the image, depth, alpha, the
per-pixel contributor counts and every intermediate stage (records, sorted
keys and values, tile ranges) for inspection.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib as L
from .types import RenderOptions, ViewCamera

RECORD_FLOATS = 12


def _p(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


@dataclass
class Frame:
    """Work buffers of one frame (torch-owned device memory); the layout of
    LumenGpuFrame in include/lumen_gpu.h."""
    records: torch.Tensor       # [N, 12] float32 (48-byte records by visible index)
    visible_ids: torch.Tensor   # [N] int32 (Gaussian index of each record)
    radii: torch.Tensor         # [N] int32
    rects: torch.Tensor         # [N] int64 packed tile rectangles
    depth_keys: list            # 2 x [N] int32 (uint32 depth keys)
    depth_order: list           # 2 x [N] int32 (visible indices in depth order)
    keys: list                  # 2 x [cap] int32 (uint32 tile ids)
    vals: list                  # 2 x [cap] int32 (uint32 visible indices)
    ranges: torch.Tensor        # [tiles, 2] int32
    scratch: torch.Tensor       # uint8
    capacity: int

    @staticmethod
    def allocate(n: int, tiles: int, capacity: int, device) -> "Frame":
        lib = L.load()
        n1 = max(n, 1)
        scratch_bytes = int(lib.lumen_gpu_scratch_bytes(n1, capacity, tiles))
        kw = dict(device=device)
        i32 = lambda m: torch.empty(m, dtype=torch.int32, **kw)
        return Frame(torch.empty((n1, RECORD_FLOATS), dtype=torch.float32, **kw), i32(n1), i32(n1),
                     torch.empty(n1, dtype=torch.int64, **kw), [i32(n1), i32(n1)], [i32(n1), i32(n1)],
                     [i32(capacity), i32(capacity)], [i32(capacity), i32(capacity)],
                     torch.empty((tiles, 2), dtype=torch.int32, **kw),
                     torch.empty(scratch_bytes, dtype=torch.uint8, **kw), capacity)

    def fits(self, n: int, tiles: int) -> bool:
        return self.records.shape[0] >= max(n, 1) and self.ranges.shape[0] >= tiles

    def c_struct(self) -> L.LumenGpuFrame:
        f = L.LumenGpuFrame()
        f.records, f.visible_ids, f.radii = _p(self.records), _p(self.visible_ids), _p(self.radii)
        f.rects = _p(self.rects)
        f.depth_keys[0], f.depth_keys[1] = _p(self.depth_keys[0]), _p(self.depth_keys[1])
        f.depth_order[0], f.depth_order[1] = _p(self.depth_order[0]), _p(self.depth_order[1])
        f.keys[0], f.keys[1] = _p(self.keys[0]), _p(self.keys[1])
        f.vals[0], f.vals[1] = _p(self.vals[0]), _p(self.vals[1])
        f.instance_capacity = self.capacity
        f.ranges = _p(self.ranges)
        f.scratch = _p(self.scratch)
        f.scratch_bytes = self.scratch.numel()
        return f


@dataclass
class RenderResult:
    rgb: torch.Tensor            # [H, W, 3]
    depth: torch.Tensor          # [H, W]
    alpha: torch.Tensor          # [H, W] 1 - T
    n_contrib: torch.Tensor      # [H, W] int32
    last_idx: torch.Tensor       # [H, W] int32
    n_visible: int
    n_instances: int
    touched_tiles: int
    varying_digits: int
    sorted_buffer: int
    frame: Frame
    options: RenderOptions = None

    @property
    def sorted_keys(self) -> torch.Tensor:
        """The reference's 64-bit keys (tile << 32 | depth key) in sorted
        order, rebuilt on the device (int64 tensor holding uint64 bits)."""
        lib = L.load()
        out = torch.empty(max(self.n_instances, 1), dtype=torch.int64, device=self.rgb.device)
        fs = self.frame.c_struct()
        opt = L.render_options(self.options or RenderOptions())
        L.check(lib.lumen_gpu_frame_sorted_keys64(C.byref(fs), C.byref(opt), _p(out),
                                                  _stream_handle(self.rgb.device)), "sorted_keys64")
        return out[: self.n_instances]

    @property
    def sorted_tiles(self) -> torch.Tensor:
        return self.frame.keys[self.sorted_buffer][: self.n_instances]

    @property
    def sorted_vals(self) -> torch.Tensor:
        return self.frame.vals[self.sorted_buffer][: self.n_instances]

    @property
    def records(self) -> torch.Tensor:
        return self.frame.records[: self.n_visible]

    @property
    def ranges(self) -> torch.Tensor:
        return self.frame.ranges


def gaussians_struct(means, scales, quats, opacities, sh) -> L.LumenGpuGaussians:
    n = int(means.shape[0])
    for name, t, shape in (("means", means, (n, 3)), ("scales", scales, (n, 3)), ("quats", quats, (n, 4)),
                           ("opacities", opacities, (n,)), ("sh", sh, (n, 48))):
        if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")
        if tuple(t.reshape(shape).shape) != shape:
            raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {shape}")
    g = L.LumenGpuGaussians()
    g.means, g.scales, g.quats, g.opacities, g.sh = _p(means), _p(scales), _p(quats), _p(opacities), _p(sh)
    g.count = n
    return g


_capacity_hint = {}


def render(means: torch.Tensor, scales: torch.Tensor, quats: torch.Tensor, opacities: torch.Tensor,
           sh: torch.Tensor, camera: ViewCamera, options: Optional[RenderOptions] = None,
           frame: Optional[Frame] = None, capacity: Optional[int] = None) -> RenderResult:
    """Forward render on the tensors' device. ``scales``/``opacities`` are linear
    and in [0, 1] unless ``options.params_are_logits``. Waits for the frame to
    finish (it reads the instance count back to check the buffer capacity)."""
    options = options or RenderOptions()
    lib = L.load()
    dev = means.device
    n = int(means.shape[0])
    H, W = int(camera.height), int(camera.width)
    tiles = camera.n_tiles
    g = gaussians_struct(means, scales, quats, opacities, sh.reshape(n, 48) if n else sh.reshape(0, 48))
    cam, opt = L.view_camera(camera), L.render_options(options)
    rgb = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
    depth = torch.empty((H, W), dtype=torch.float32, device=dev)
    alpha = torch.empty((H, W), dtype=torch.float32, device=dev)
    ncon = torch.empty((H, W), dtype=torch.int32, device=dev)
    last = torch.empty((H, W), dtype=torch.int32, device=dev)
    img = L.LumenGpuImage()
    img.rgb, img.depth, img.alpha, img.n_contrib, img.last_idx = _p(rgb), _p(depth), _p(alpha), _p(ncon), _p(last)
    key = (n, W, H)
    if capacity is None:
        capacity = _capacity_hint.get(key, max(1 << 16, 8 * n))
    if frame is None or not frame.fits(n, tiles) or frame.capacity < capacity:
        frame = Frame.allocate(n, tiles, capacity, dev)
    stream = _stream_handle(dev)
    counts = L.LumenGpuCounts()
    for _ in range(2):
        fs = frame.c_struct()
        L.check(lib.lumen_gpu_render_forward(C.byref(g), C.byref(cam), C.byref(opt), C.byref(fs), C.byref(img),
                                             stream), "render_forward")
        L.check(lib.lumen_gpu_read_counts(C.byref(fs), C.byref(counts), stream), "read_counts")
        if not counts.error_flags & L.ERR_CAPACITY:
            break
        need = int(counts.n_instances)
        capacity = need + need // 4 + 4096
        frame = Frame.allocate(n, tiles, capacity, dev)
    if counts.error_flags:
        raise L.LumenError(-4 if not counts.error_flags & L.ERR_CAPACITY else -2,
                           f"render_forward device flags {counts.error_flags:#x}")
    _capacity_hint[key] = frame.capacity
    return RenderResult(rgb, depth, alpha, ncon, last, int(counts.n_visible), int(counts.n_instances),
                        int(counts.touched_tiles), int(counts.varying_digits), int(counts.sorted_buffer), frame,
                        options)


class Scene:
    """A scene resident on the device: SoA parameter tensors (float32,
    contiguous) in the layout of LumenGpuGaussians."""

    def __init__(self, means, scales, quats, opacities, sh):
        n = int(means.shape[0])
        self.tensors = (means, scales, quats, opacities, sh.reshape(n, 48) if n else sh.reshape(0, 48))
        self.struct = gaussians_struct(*self.tensors)
        self.count = n

    @property
    def device(self):
        return self.tensors[0].device


@dataclass
class BatchFrame:
    """Work buffers of a batch (LumenGpuFrame sized by lumen_gpu_batch_sizes)."""
    frame: Frame
    slots: int
    tiles: int
    n_views: int

    @staticmethod
    def allocate(slots: int, tiles: int, capacity: int, n_views: int, device) -> "BatchFrame":
        lib = L.load()
        s1 = max(slots, 1)
        kw = dict(device=device)
        i32 = lambda m: torch.empty(m, dtype=torch.int32, **kw)
        scratch = int(lib.lumen_gpu_batch_scratch_bytes(s1, capacity, n_views))
        f = Frame(torch.empty((s1, RECORD_FLOATS), dtype=torch.float32, **kw), i32(s1), i32(s1),
                  torch.empty(s1, dtype=torch.int64, **kw), [i32(s1), i32(s1)], [i32(s1), i32(s1)],
                  [i32(capacity), i32(capacity)], [i32(capacity), i32(capacity)],
                  torch.empty((max(tiles, 1), 2), dtype=torch.int32, **kw),
                  torch.empty(scratch, dtype=torch.uint8, **kw), capacity)
        return BatchFrame(f, s1, tiles, n_views)

    def fits(self, slots: int, tiles: int, capacity: int, n_views: int) -> bool:
        lib = L.load()
        need = int(lib.lumen_gpu_batch_scratch_bytes(max(slots, 1), self.frame.capacity, n_views))
        return (self.slots >= slots and self.tiles >= tiles and self.frame.capacity >= capacity
                and self.frame.scratch.numel() >= need)


@dataclass
class ViewImage:
    rgb: torch.Tensor            # [H, W, 3]
    depth: torch.Tensor          # [H, W]
    alpha: torch.Tensor          # [H, W]
    n_contrib: torch.Tensor      # [H, W] int32
    last_idx: torch.Tensor       # [H, W] int32 (offset within the view's sorted instances)


@dataclass
class BatchResult:
    images: list                 # ViewImage per view
    n_visible: int
    n_instances: int
    sorted_buffer: int
    tile_begin: list             # batch-wide id of each view's tile 0
    frame: BatchFrame
    options: RenderOptions = None

    @property
    def sorted_keys(self) -> torch.Tensor:
        """The batch's 64-bit keys ((view tile offset + tile) << 32 | depth
        key), in sorted order."""
        lib = L.load()
        dev = self.images[0].rgb.device
        out = torch.empty(max(self.n_instances, 1), dtype=torch.int64, device=dev)
        fs = self.frame.frame.c_struct()
        opt = L.render_options(self.options or RenderOptions())
        L.check(lib.lumen_gpu_frame_sorted_keys64(C.byref(fs), C.byref(opt), _p(out), _stream_handle(dev)),
                "sorted_keys64")
        return out[: self.n_instances]

    @property
    def sorted_vals(self) -> torch.Tensor:
        return self.frame.frame.vals[self.sorted_buffer][: self.n_instances]


_batch_capacity_hint = {}


def batch_views(views, images) -> "C.Array":
    """The LumenGpuBatchView array for (Scene, ViewCamera) pairs and their
    ViewImage outputs."""
    arr = (L.LumenGpuBatchView * len(views))()
    for i, ((scene, cam), im) in enumerate(zip(views, images)):
        arr[i].gaussians = scene.struct
        arr[i].camera = L.view_camera(cam)
        img = L.LumenGpuImage()
        img.rgb, img.depth, img.alpha = _p(im.rgb), _p(im.depth), _p(im.alpha)
        img.n_contrib, img.last_idx = _p(im.n_contrib), _p(im.last_idx)
        arr[i].image = img
    return arr


def allocate_images(cameras, device) -> list:
    out = []
    for cam in cameras:
        H, W = int(cam.height), int(cam.width)
        out.append(ViewImage(torch.empty((H, W, 3), dtype=torch.float32, device=device),
                             torch.empty((H, W), dtype=torch.float32, device=device),
                             torch.empty((H, W), dtype=torch.float32, device=device),
                             torch.empty((H, W), dtype=torch.int32, device=device),
                             torch.empty((H, W), dtype=torch.int32, device=device)))
    return out


def render_batch(views, options: Optional[RenderOptions] = None, frame: Optional[BatchFrame] = None,
                 capacity: Optional[int] = None, images: Optional[list] = None) -> BatchResult:
    """Render several (Scene, ViewCamera) views in one pipeline
    (lumen_gpu_render_batch). Each view's outputs equal rendering it alone.
    Waits for the batch (reads the instance count back to check capacity)."""
    options = options or RenderOptions()
    lib = L.load()
    if not views:
        raise ValueError("render_batch needs at least one view")
    dev = views[0][0].device
    images = images or allocate_images([c for _, c in views], dev)
    arr = batch_views(views, images)
    nv = len(views)
    slots, tiles = C.c_int64(0), C.c_int64(0)
    L.check(lib.lumen_gpu_batch_sizes(arr, nv, C.byref(slots), C.byref(tiles)), "batch_sizes")
    slots, tiles = int(slots.value), int(tiles.value)
    key = (slots, tiles, nv)
    if capacity is None:
        capacity = _batch_capacity_hint.get(key, max(1 << 16, 8 * slots))
    if frame is None or not frame.fits(slots, tiles, capacity, nv):
        frame = BatchFrame.allocate(slots, tiles, capacity, nv, dev)
    opt = L.render_options(options)
    stream = _stream_handle(dev)
    counts = L.LumenGpuCounts()
    for _ in range(2):
        fs = frame.frame.c_struct()
        L.check(lib.lumen_gpu_render_batch(arr, nv, C.byref(opt), C.byref(fs), stream), "render_batch")
        L.check(lib.lumen_gpu_read_counts(C.byref(fs), C.byref(counts), stream), "read_counts")
        if not counts.error_flags & L.ERR_CAPACITY:
            break
        need = int(counts.n_instances)
        frame = BatchFrame.allocate(slots, tiles, need + need // 4 + 4096, nv, dev)
    if counts.error_flags:
        raise L.LumenError(-4 if not counts.error_flags & L.ERR_CAPACITY else -2,
                           f"render_batch device flags {counts.error_flags:#x}")
    _batch_capacity_hint[key] = frame.frame.capacity
    tile_begin, t = [], 0
    for _, cam in views:
        tile_begin.append(t)
        t += cam.n_tiles
    return BatchResult(images, int(counts.n_visible), int(counts.n_instances), int(counts.sorted_buffer),
                       tile_begin, frame, options)


def sort_pairs(keys: torch.Tensor, vals: torch.Tensor):
    """Stable sort of (uint64 key, uint32 value) pairs on the device
    (lumen_gpu_sort_pairs). Takes int64/int32 tensors holding the bits;
    returns sorted copies."""
    lib = L.load()
    n = int(keys.numel())
    k0, v0 = keys.contiguous().clone(), vals.contiguous().clone()
    k1, v1 = torch.empty_like(k0), torch.empty_like(v0)
    scratch = torch.empty(int(lib.lumen_gpu_scratch_bytes(0, max(n, 1), 0)), dtype=torch.uint8, device=keys.device)
    sb = C.c_uint32(0)
    L.check(lib.lumen_gpu_sort_pairs(_p(k0), _p(v0), _p(k1), _p(v1), n, _p(scratch), scratch.numel(), C.byref(sb),
                                     _stream_handle(keys.device)), "sort_pairs")
    return (k1, v1) if sb.value else (k0, v0)
