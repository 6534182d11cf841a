"""Render serving over resident scenes (include/lumen_serve.h).

``Server`` keeps scenes on the device and renders requests with continuous
batching: requests queue in arrival order, a native scheduler thread admits
them into multi-view batches within a device-memory budget, up to
``max_batches_in_flight`` batches run at once on their own streams, and
each batch is one CUDA graph launch of the persistent multi-view pipeline.
Each request's image is identical to rendering its view alone; the output
is the 8-bit RGB of the reference C ABI's frame buffer
(c_api/src/lumen_c.c:541-543) in a host tensor.

No counterpart in the reference, which renders one camera per synchronous
call (c_api/include/lumen.h:153-159).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib as L
from .render import Scene
from .types import RenderOptions, ViewCamera


@dataclass
class ServeResult:
    image: torch.Tensor          # [H, W, 3] uint8 on the host
    status: int
    batch_views: int
    submit_ms: float             # server clock (ms since creation)
    start_ms: float
    done_ms: float
    n_instances: int
    composite_chunk: int
    sort_items: int

    @property
    def latency_ms(self) -> float:
        return self.done_ms - self.submit_ms


@dataclass
class Request:
    id: int
    out: torch.Tensor
    server: "Server"

    def result(self, timeout_ms: float = -1.0) -> ServeResult:
        return self.server.result(self, timeout_ms)


class Server:
    def __init__(self, work_budget_bytes: int = 8 << 30, max_views_per_batch: int = 64,
                 max_batches_in_flight: int = 2, use_graphs: bool = True, autotune: bool = True,
                 composite_chunk: int = 256, sort_items: int = 16, options: Optional[RenderOptions] = None):
        lib = L.load()
        cfg = lib.lumen_server_default_config()
        cfg.work_budget_bytes = int(work_budget_bytes)
        cfg.max_views_per_batch = int(max_views_per_batch)
        cfg.max_batches_in_flight = int(max_batches_in_flight)
        cfg.use_graphs = int(bool(use_graphs))
        cfg.autotune = int(bool(autotune))
        cfg.composite_chunk = int(composite_chunk)
        cfg.sort_items = int(sort_items)
        cfg.options = L.render_options(options or RenderOptions(term_mode=1))
        self._lib = lib
        self._h = lib.lumen_server_create(C.byref(cfg))
        if not self._h:
            raise L.LumenError(-1, "lumen_server_create failed (configuration, device or memory)")
        self._scenes = []

    def add_scene(self, scene: Scene) -> int:
        sid = int(self._lib.lumen_server_add_scene(self._h, C.byref(scene.struct)))
        if sid < 0:
            raise L.LumenError(sid, "add_scene")
        self._scenes.append(scene)   # the device arrays must outlive the server
        return sid

    def submit(self, scene_id: int, camera: ViewCamera, out: Optional[torch.Tensor] = None) -> Request:
        H, W = int(camera.height), int(camera.width)
        if out is None:
            out = torch.empty((H, W, 3), dtype=torch.uint8, pin_memory=True)
        if out.dtype != torch.uint8 or out.is_cuda or not out.is_contiguous() or out.numel() != H * W * 3:
            raise ValueError("out must be a contiguous host uint8 tensor of H*W*3 elements")
        rid = C.c_uint64(0)
        cam = L.view_camera(camera)
        L.check(self._lib.lumen_server_submit(self._h, int(scene_id), C.byref(cam), out.data_ptr(), C.byref(rid)),
                "server_submit")
        return Request(int(rid.value), out, self)

    def result(self, request: Request, timeout_ms: float = -1.0) -> ServeResult:
        r = L.LumenServeResult()
        L.check(self._lib.lumen_server_wait(self._h, request.id, float(timeout_ms), C.byref(r)), "server_wait")
        return ServeResult(request.out, int(r.status), int(r.batch_views), float(r.submit_ms), float(r.start_ms),
                           float(r.done_ms), int(r.n_instances), int(r.composite_chunk), int(r.sort_items))

    def freeze_tuning(self, frozen: bool = True) -> None:
        """Stop (or resume) the autotuner's exploration: while frozen every
        batch runs the best launch variant timed so far for its class."""
        L.check(self._lib.lumen_server_freeze_tuning(self._h, int(bool(frozen))), "server_freeze_tuning")

    def stats(self) -> dict:
        s = L.LumenServeStats()
        L.check(self._lib.lumen_server_stats(self._h, C.byref(s)), "server_stats")
        return {name: getattr(s, name) for name, _ in L.LumenServeStats._fields_}

    def close(self) -> None:
        if self._h:
            self._lib.lumen_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
