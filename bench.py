#!/usr/bin/env python
"""Benchmark: 1080p frames/s of the forward splatting pipeline on B200.

Workload (configuration 1): 1M Gaussians uniform in a 6x4x6 box 8 units
ahead, 1920x1080, vertical FOV 50 degrees, degree-3 SH, 16x16 tiles,
millimetre depth keys, compositing stops at accumulated alpha >= 0.99.
Synthetic seeded data (numpy PCG64, seed 1); parameters stay resident in HBM.

A step is one full frame: project + cull + SH + scan + key emit, histogram,
stable digit passes, tile ranges, compositing. ``value`` times K back-to-back
frames on the device with CUDA events (inputs resident; the 236 MB of
parameters per frame exceed the 126 MB L2). ``e2e`` times the same frame
through the reference-facing C ABI call lumen_rasterize with a host frame
buffer (upload of the buffer's old contents, render, read-back of rgb8,
depth and alpha inside the timed region; the cloud is uploaded once, in the
warm-up, as the reference keeps it resident).

``--impl reference`` times the reference's CPU algorithm (the oracle
restatement of the Mojo path; the Mojo toolchain does not exist here) on all
host cores for the same workload. Under torchrun N > 1 every rank renders an
independent replica (the path has no exchange step); value = total frames/s.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1080p frames/s and p99 latency, served vs per-call render; fwd+bwd steps/s"
UNIT = "frames/s"
N_GAUSSIANS = 1_000_000
WIDTH, HEIGHT = 1920, 1080
# DRAM bytes (read + write) of one composite_kernel<512> launch at the 1 M-Gaussian
# 1080p workload, from an ncu capture (profiles/forward_config1_kernels.md)
COMPOSITE_DRAM_BYTES = 43.5e6
def kernels_per_frame(n_tiles: int) -> int:
    """Kernels one forward frame launches: init; the projection's count,
    offset scan and projection; the depth sort's histogram and 4 digit
    passes; the emission (which also counts the tile sort's digits); one
    tile-sort digit pass per byte a tile id can vary in; tile ranges;
    composite."""
    tile_bytes = 0
    t = n_tiles - 1
    while t > 0:
        tile_bytes += 1
        t >>= 8
    return 1 + 3 + (1 + 4) + 1 + tile_bytes + 1 + 1


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=300)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", choices=["lumen", "reference"], default="lumen")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fwd-bwd", action="store_true")
    p.add_argument("--no-multiview", action="store_true")
    p.add_argument("--no-serving", action="store_true")
    p.add_argument("--no-train", action="store_true")
    p.add_argument("--no-depth", action="store_true")
    p.add_argument("--no-picking", action="store_true")
    p.add_argument("--serve-requests", type=int, default=1000)
    return p.parse_args()


def workload_config(extra=None):
    c = {"workload": "config 1: 1M Gaussians, 1920x1080, per-call forward render",
         "n_gaussians": N_GAUSSIANS, "width": WIDTH, "height": HEIGHT, "sh_degree": 3, "tile": 16,
         "key": "tile<<32 | clamp(int(z*1000))", "termination": "accumulated alpha >= 0.99",
         "l2": "inputs larger than L2 (236 MB parameters per frame)", "data": "synthetic, numpy PCG64 seed 1"}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML every 10 ms while
    the timed region runs (nvidia-smi's -lms loop as a fallback)."""
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, cuda_index: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        idx = cuda_index
        if vis:
            try:
                idx = int(vis.split(",")[cuda_index])
            except (ValueError, IndexError):
                pass
        self.index = idx
        self.sm, self.reasons, self.max = [], 0, None
        self.stop = threading.Event()
        self.nvml = None

    def _loop(self):
        h = self.nvml.nvmlDeviceGetHandleByIndex(self.index)
        self.max = self.nvml.nvmlDeviceGetMaxClockInfo(h, self.nvml.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                self.sm.append(self.nvml.nvmlDeviceGetClockInfo(h, self.nvml.NVML_CLOCK_SM))
                self.reasons |= int(self.nvml.nvmlDeviceGetCurrentClocksEventReasons(h))
            except Exception:
                pass
            time.sleep(0.01)

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
            deadline = time.time() + 2.0
            while not self.sm and time.time() < deadline:
                time.sleep(0.005)
        except Exception:
            self.nvml = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml:
            self.t.join(timeout=2)

    def summary(self):
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.max,
                "reasons": sorted(v for k, v in self.REASONS.items() if self.reasons & k),
                "samples": len(self.sm), "source": "nvml, 10 ms"}


def replica_throughput(ms_per_step, world, pg, dev):
    """Independent replicas, one per rank: the step time is the slowest
    rank's (max over ranks) and the whole-job rate is world steps per that
    time. Returns (max ms per step, steps/s of the job)."""
    import torch
    t = torch.tensor([float(ms_per_step)], device=dev)
    if pg is not None and world > 1:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    ms_max = float(t.item())
    return ms_max, world * 1000.0 / ms_max


def replica_rate(rate, world, pg, dev):
    """A per-rank rate to the job's: the slowest rank's rate times world."""
    import torch
    t = torch.tensor([float(rate)], device=dev)
    if pg is not None and world > 1:
        pg.all_reduce(t, op=pg.ReduceOp.MIN)
    return float(t.item()) * world


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reference_arm(args, world, rank):
    """The reference's CPU algorithm (oracle port of the Mojo path), all host threads."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from lumen_b200 import scenes
    from lumen_b200.types import RenderOptions
    sc = scenes.box_scene(N_GAUSSIANS, seed=1)
    s, op = sc.activated()
    cam = scenes.camera_config1(WIDTH, HEIGHT)
    opt = RenderOptions(term_mode=1)
    nt = os.cpu_count() or 1
    for _ in range(args.warmup):
        O.render(sc.means, s, sc.quats, op, sc.sh, cam, opt, stages=False, nthreads=nt)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.render(sc.means, s, sc.quats, op, sc.sh, cam, opt, stages=False, nthreads=nt)
    dt = (time.perf_counter() - t0) / args.steps
    v = 1.0 / dt
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": workload_config({"parallelism": "host threads"}),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nt, "kind": "port",
                             "sample": "one full 1080p frame of config 1 per step (1M Gaussians)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _reference_c_rasterize(sc, scales, opac, n_sample):
    """The reference's own C renderer (c_api/src/lumen_c.c, built by
    oracle/Makefile into oracle/_ref/) on the first n_sample Gaussians of the
    workload at 1080p: seconds per frame, or None when it was not built. A
    different algorithm from the Mojo path (isotropic, DC-only, qsort)."""
    import numpy as np
    from lumen_b200 import _lib as L
    path = os.path.join(ROOT, "oracle", "_ref", "liblumen_ref.so")
    if not os.path.exists(path):
        return None
    ref = C.CDLL(path)
    for name in ("lumen_cloud_create", "lumen_cloud_destroy", "lumen_cloud_add_gaussian", "lumen_framebuffer_create",
                 "lumen_framebuffer_destroy", "lumen_rasterizer_create", "lumen_rasterizer_destroy",
                 "lumen_rasterize", "lumen_default_config"):
        res, args = L.SIGNATURES[name]
        fn = getattr(ref, name)
        fn.restype, fn.argtypes = res, args
    n = n_sample
    aos = np.zeros((n, 59), np.float32)
    aos[:, 0:3] = sc.means[:n]
    aos[:, 3:6] = scales[:n]
    aos[:, 6:10] = sc.quats[:n]
    aos[:, 10] = opac[:n]
    aos[:, 11:59] = sc.sh[:n].reshape(n, 48)
    cloud = ref.lumen_cloud_create(n)
    gs = (L.LumenGaussian * n).from_buffer_copy(aos.tobytes())
    for i in range(n):
        ref.lumen_cloud_add_gaussian(cloud, C.byref(gs[i]))
    cfg = ref.lumen_default_config()
    cfg.image_width, cfg.image_height = WIDTH, HEIGHT
    r = ref.lumen_rasterizer_create(C.byref(cfg))
    fb = ref.lumen_framebuffer_create(WIDTH, HEIGHT)
    cam = L.LumenCamera()
    cam.position, cam.target, cam.up = L.LumenVec3(0, 0, 0), L.LumenVec3(0, 0, 8), L.LumenVec3(0, 1, 0)
    cam.fov_x_degrees, cam.fov_y_degrees = 50.0 * WIDTH / HEIGHT, 50.0
    cam.near_plane, cam.far_plane = 0.01, 1000.0
    st = L.LumenStats()
    t0 = time.perf_counter()
    rc = ref.lumen_rasterize(r, cloud, C.byref(cam), fb, C.byref(st))
    dt = time.perf_counter() - t0
    ref.lumen_framebuffer_destroy(fb)
    ref.lumen_rasterizer_destroy(r)
    ref.lumen_cloud_destroy(cloud)
    return dt if rc == 0 else None


def cpu_baseline():
    """The oracle restatement of the reference path on the host: all threads
    (the reported value) and one thread (the reference's scalar execution),
    one full config-1 frame each; and the reference's own C renderer on a
    bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from lumen_b200 import scenes
    from lumen_b200.types import RenderOptions
    sc = scenes.box_scene(N_GAUSSIANS, seed=1)
    s, op = sc.activated()
    cam = scenes.camera_config1(WIDTH, HEIGHT)
    nt = os.cpu_count() or 1
    t0 = time.perf_counter()
    O.render(sc.means, s, sc.quats, op, sc.sh, cam, RenderOptions(term_mode=1), stages=False, nthreads=nt)
    dt = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.render(sc.means, s, sc.quats, op, sc.sh, cam, RenderOptions(term_mode=1), stages=False, nthreads=1)
    dt1 = time.perf_counter() - t0
    out = {"value": 1.0 / dt, "unit": UNIT, "cores": nt, "kind": "port",
           "sample": "one full 1080p frame of config 1 (1M Gaussians), oracle on all host threads",
           "single_thread": {"value": 1.0 / dt1, "unit": UNIT, "cores": 1,
                             "sample": "one full 1080p frame of config 1, oracle on one thread"}}
    n_sample = 200_000
    dtr = _reference_c_rasterize(sc, s, op, n_sample)
    if dtr is not None:
        scale = N_GAUSSIANS / n_sample
        out["reference_c_abi"] = {
            "value": 1.0 / (dtr * scale), "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"lumen_rasterize of the reference C library on the first {n_sample} Gaussians at 1080p "
                      f"({dtr:.2f} s), scaled by {scale:.0f} to a 1M frame; a different algorithm "
                      "(isotropic, DC-only, qsort) from the Mojo path"}
    return out


def e2e_rasterize(sc, scales, opac, steps, warmup):
    """lumen_rasterize (include/lumen.h) with a host frame buffer."""
    import numpy as np
    from lumen_b200 import _lib as L
    lib = L.load()
    n = sc.n
    aos = np.zeros((n, 59), np.float32)
    aos[:, 0:3] = sc.means
    aos[:, 3:6] = scales
    aos[:, 6:10] = sc.quats
    aos[:, 10] = opac
    aos[:, 11:59] = sc.sh.reshape(n, 48)
    cloud = lib.lumen_cloud_create(n)
    L.check(lib.lumen_cloud_append(cloud, aos.ctypes.data_as(C.POINTER(L.LumenGaussian)), n), "cloud_append")
    cfg = lib.lumen_default_config()
    cfg.image_width, cfg.image_height = WIDTH, HEIGHT
    cfg.near_plane, cfg.far_plane, cfg.early_termination_alpha = 0.01, 1000.0, 0.99
    r = lib.lumen_rasterizer_create(C.byref(cfg))
    fb = lib.lumen_framebuffer_create(WIDTH, HEIGHT)
    cam = L.LumenCamera(L.LumenVec3(0, 0, 0), L.LumenVec3(0, 0, 1), L.LumenVec3(0, -1, 0), 60.0, 50.0, 0.01, 1000.0)
    st = L.LumenStats()
    for _ in range(warmup):
        lib.lumen_framebuffer_clear(fb, 0, 0, 0)
        L.check(lib.lumen_rasterize(r, cloud, C.byref(cam), fb, C.byref(st)), "rasterize")
    gpu_ms, wall = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        L.check(lib.lumen_rasterize(r, cloud, C.byref(cam), fb, C.byref(st)), "rasterize")
        wall.append(time.perf_counter() - t0)
        gpu_ms.append(st.rasterize_time_ms)
    npix = WIDTH * HEIGHT
    wall_ms = [w * 1e3 for w in wall]
    # the host wall clock around each call (it returns once the frame buffer
    # is back in host memory); the library's own event time beside it
    out = {"value": 1.0 / (sum(wall) / len(wall)), "unit": UNIT,
           "h2d_bytes_per_step": npix * 3 + npix * 4, "d2h_bytes_per_step": npix * 3 + npix * 4 + npix * 4,
           "api": "lumen_rasterize (include/lumen.h), host LumenFrameBuffer",
           "timing": "host wall clock per call",
           "library_event_frames_per_s": 1000.0 / (sum(gpu_ms) / len(gpu_ms)),
           "p50_ms": statistics.median(wall_ms),
           "p99_ms": sorted(wall_ms)[min(len(wall_ms) - 1, int(0.99 * len(wall_ms)))],
           "visible": int(st.visible_splats), "touched_tiles": int(st.touched_tiles)}
    lib.lumen_framebuffer_destroy(fb)
    lib.lumen_rasterizer_destroy(r)
    lib.lumen_cloud_destroy(cloud)
    return out


def fwd_bwd_leg(dev, steps, warmup, hbm_peak):
    """Configuration 3: 500k Gaussians at 1920x1080; one step = forward +
    L1 loss against the render of the perturbed scene + the hand-written
    backward to (means, log-scales, quats, opacity logits, SH), all through
    the C ABI on one stream. Also the same step through the torch autograd
    API (public call path, one host sync per forward)."""
    import numpy as np
    import torch
    from lumen_b200 import _lib as L
    from lumen_b200 import autograd as A
    from lumen_b200 import render as R
    from lumen_b200 import scenes
    from lumen_b200.types import RenderOptions
    n = 500_000
    sc = scenes.box_scene(n, seed=3)
    tg = scenes.perturbed(sc, seed=33)
    cam = scenes.camera_config1(WIDTH, HEIGHT)
    opt = RenderOptions(term_mode=1, params_are_logits=True)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    params = [t(sc.means), t(sc.log_scales), t(sc.quats), t(sc.opacity_logits), t(sc.sh).reshape(n, 48)]
    target = R.render(t(tg.means), t(tg.log_scales), t(tg.quats), t(tg.opacity_logits), t(tg.sh).reshape(n, 48),
                      cam, opt).rgb.contiguous()
    first = R.render(*params, cam, opt)
    V, K, T, P = first.n_visible, first.n_instances, cam.n_tiles, WIDTH * HEIGHT
    passes = bin(first.varying_digits & 0xFFFF).count("1")
    lib = L.load()
    g = R.gaussians_struct(*params)
    ccam, copt = L.view_camera(cam), L.render_options(opt)
    fs = first.frame.c_struct()
    img = L.LumenGpuImage()
    rgb, depth, alpha = (torch.empty((HEIGHT, WIDTH, 3), device=dev), torch.empty((HEIGHT, WIDTH), device=dev),
                         torch.empty((HEIGHT, WIDTH), device=dev))
    last = torch.empty((HEIGHT, WIDTH), dtype=torch.int32, device=dev)
    img.rgb, img.depth, img.alpha, img.last_idx = rgb.data_ptr(), depth.data_ptr(), alpha.data_ptr(), last.data_ptr()
    grads = [torch.empty_like(p) for p in params]
    splat2d = torch.empty((n, 12), device=dev)
    out = L.LumenGpuGradients()
    out.means, out.scales, out.quats, out.opacities, out.sh = (x.data_ptr() for x in grads)
    out.splat2d = splat2d.data_ptr()
    gimg = torch.empty_like(rgb)
    loss = torch.empty((), device=dev)
    l1s = torch.empty(int(lib.lumen_gpu_l1_loss_scratch_bytes()), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def step():
        L.check(lib.lumen_gpu_render_forward(C.byref(g), C.byref(ccam), C.byref(copt), C.byref(fs), C.byref(img),
                                             stream), "forward")
        L.check(lib.lumen_gpu_l1_loss(rgb.data_ptr(), target.data_ptr(), rgb.numel(), gimg.data_ptr(),
                                      loss.data_ptr(), l1s.data_ptr(), stream), "l1")
        L.check(lib.lumen_gpu_render_backward(C.byref(g), C.byref(ccam), C.byref(copt), C.byref(fs), C.byref(img),
                                              gimg.data_ptr(), None, None, C.byref(out), stream), "backward")

    for _ in range(warmup):
        step()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    counts = L.LumenGpuCounts()
    L.check(lib.lumen_gpu_read_counts(C.byref(fs), C.byref(counts), stream), "counts")
    assert counts.error_flags == 0 and counts.n_instances == K
    # backward alone, for its share
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record()
    for _ in range(max(steps // 4, 1)):
        L.check(lib.lumen_gpu_render_backward(C.byref(g), C.byref(ccam), C.byref(copt), C.byref(fs), C.byref(img),
                                              gimg.data_ptr(), None, None, C.byref(out), stream), "backward")
    b1.record()
    torch.cuda.synchronize(dev)
    bwd_ms = b0.elapsed_time(b1) / max(steps // 4, 1)
    # stage split of the backward and of this workload's forward (a second,
    # event-instrumented run)
    reps = max(min(steps, 20), 1)
    timer = lib.lumen_gpu_stage_timer_create(reps)
    for _ in range(reps):
        L.check(lib.lumen_gpu_render_backward_timed(C.byref(g), C.byref(ccam), C.byref(copt), C.byref(fs), C.byref(img),
                                                    gimg.data_ptr(), None, None, C.byref(out), timer, stream),
                "backward_timed")
    bst = (C.c_float * 4)()
    btot, nfr = C.c_float(0), C.c_int(0)
    L.check(lib.lumen_gpu_stage_timer_read(timer, bst, C.byref(btot), C.byref(nfr)), "timer")
    for _ in range(reps):
        L.check(lib.lumen_gpu_render_forward_timed(C.byref(g), C.byref(ccam), C.byref(copt), C.byref(fs),
                                                   C.byref(img), timer, stream), "forward_timed")
    fst = (C.c_float * 4)()
    L.check(lib.lumen_gpu_stage_timer_read(timer, fst, C.byref(btot), C.byref(nfr)), "timer")
    lib.lumen_gpu_stage_timer_destroy(timer)
    # the public API: torch.autograd with the same step
    leaves = [p.clone().requires_grad_(True) for p in params]
    ta_steps = max(steps // 4, 3)
    for i in range(ta_steps + 2):
        if i == 2:
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
        r, _, _ = A.render(*leaves, cam, opt)
        A.l1_loss(r, target).backward()
    torch.cuda.synchronize(dev)
    api_ms = (time.perf_counter() - t0) * 1e3 / ta_steps
    b_fwd = 244 * n + 64 * V + (60 + 24 * passes) * K + 16 * T + 16 * P
    b_bwd = 80 * K + 12 * P + 88 * V + 472 * n
    total = b_fwd + 24 * P + b_bwd
    stages = {"project": fst[0] / reps, "sort": fst[1] / reps, "tile_ranges": fst[2] / reps,
              "composite": fst[3] / reps, "composite_backward": bst[0] / reps, "project_backward": bst[1] / reps}
    return {"workload": "config 3: 500k Gaussians, 1920x1080, L1 to the perturbed-scene render",
            "steps_per_s": 1000.0 / ms, "ms_per_step": ms, "backward_ms": bwd_ms,
            "stages_ms": {k: round(v, 4) for k, v in stages.items()},
            "stages_timing": "a second, event-instrumented run of the forward and of the backward",
            "sizes": {"n": n, "visible": V, "instances": K, "pixels": P, "tiles": T, "digit_passes": passes},
            "autograd_api_steps_per_s": 1000.0 / api_ms, "visible": V, "instances": K,
            "roofline": {"bytes": total, "achieved": total / (ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                         "frac": total / (ms * 1e-3) / 1e9 / hbm_peak}}


def train_leg(dev, steps):
    """The training step around the adjoint (lumen_b200.train.Trainer, the
    reference's TrainingCoordinator.train_step with real gradients) on the
    500k-Gaussian 1080p scene: forward, L1 + PSNR, backward, Adam on
    positions and opacity, view-space accumulation, metrics read back each
    step (as the reference returns them). Then one density-control pass over
    the accumulated gradients, timed on the device."""
    import numpy as np
    import torch
    from lumen_b200 import render as R
    from lumen_b200 import scenes
    from lumen_b200 import train as T
    from lumen_b200.types import RenderOptions
    n = 500_000
    sc = scenes.box_scene(n, seed=3)
    s, op = sc.activated()
    tg = scenes.perturbed(sc, seed=33)
    ts, top = tg.activated()
    cam = scenes.camera_config1(WIDTH, HEIGHT)
    opt = RenderOptions(term_mode=1)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    target = R.render(t(tg.means), t(ts), t(tg.quats), t(top).reshape(-1), t(tg.sh).reshape(n, 48), cam, opt).rgb
    cfg = T.default_config()
    cfg.densify_from_iter = 10 ** 9          # density control timed separately below
    tr = T.Trainer(sc.means, s, sc.quats, op, sc.sh.reshape(n, 48), config=cfg, options=opt, scene_extent=6.0,
                   device=dev)
    for it in range(1, 4):
        tr.train_step(cam, target, it)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    losses = []
    for it in range(4, 4 + steps):
        losses.append(tr.train_step(cam, target, it).loss)
    torch.cuda.synchronize(dev)
    ms = (time.perf_counter() - t0) * 1e3 / steps
    d0 = time.perf_counter()
    cl, sp, pr = tr.densify_and_prune()
    torch.cuda.synchronize(dev)
    densify_wall_ms = (time.perf_counter() - d0) * 1e3
    return {"workload": "500k Gaussians, 1920x1080, linear parameters, L1 to a perturbed copy of the scene",
            "steps_per_s": 1000.0 / ms, "ms_per_step": ms, "loss_first": losses[0], "loss_last": losses[-1],
            "timing": "host wall clock per step (each step reads its loss and PSNR back)",
            "densify": {"device_ms": tr.last_densify_ms, "wall_ms_with_allocation": densify_wall_ms,
                        "cloned": cl, "split": sp, "pruned": pr, "count": tr.count,
                        "observations": 3 + steps}}


def depth_leg(dev, steps, warmup, hbm_peak):
    """Depth products (lumen_gpu_depth_products: range, normals and the SDK
    heatmap in one pass) on 1920x1080 depth buffers rendered from the 1M
    scene. 16 buffers are cycled so inputs and outputs (0.6 GB) exceed L2.
    Algorithmic bytes: 4 read + 12 (normal) + 3 (heatmap) written per pixel.
    Also the oracle's time for the same products of one buffer on one host
    thread."""
    import numpy as np
    import torch
    from lumen_b200 import depth as D
    from lumen_b200 import render as R
    from lumen_b200 import scenes
    from lumen_b200.types import RenderOptions
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    sc = scenes.box_scene(1_000_000, seed=1)
    s, op = sc.activated()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    cam = scenes.camera_config1(WIDTH, HEIGHT)
    d0 = R.render(t(sc.means), t(s), t(sc.quats), t(op).reshape(-1), t(sc.sh).reshape(-1, 48), cam,
                  RenderOptions(compute_depth=True)).depth.contiguous()
    nbuf = 16
    depths = [d0 * (1.0 + 0.01 * i) for i in range(nbuf)]
    outs = [D.products(d, normals=True, range=True, heatmap=True, near_plane=2.0, far_plane=14.0)
            for d in depths]
    from lumen_b200 import _lib as lib
    structs = []
    for o in outs:
        st = lib.LumenDepthProducts()
        st.normals, st.range, st.heatmap = o.normals.data_ptr(), o.range.data_ptr(), o.heatmap.data_ptr()
        st.near_plane, st.far_plane = 2.0, 14.0
        structs.append(st)
    cdll = lib.load()
    stream = torch.cuda.current_stream(dev).cuda_stream

    def launch(i):
        lib.check(cdll.lumen_gpu_depth_products(depths[i % nbuf].data_ptr(), WIDTH, HEIGHT, C.byref(structs[i % nbuf]),
                                             stream), "depth_products")

    for i in range(max(warmup, 3)):
        launch(i)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(steps):
        launch(i)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    P = WIDTH * HEIGHT
    alg = 19 * P
    h = d0.cpu().numpy()
    c0 = time.perf_counter()
    O.depth_normals(h)
    O.depth_min_max(h)
    O.depth_heatmap(h, 2.0, 14.0)
    cpu_ms = (time.perf_counter() - c0) * 1e3
    return {"workload": "depth products of a 1920x1080 depth buffer (1M-Gaussian render): range, normals, heatmap",
            "ms": ms, "buffers_per_s": 1000.0 / ms, "gpu_launches_per_buffer": 2,
            "roofline": {"bound": "hbm", "bytes": alg, "achieved": alg / (ms * 1e-3) / 1e9, "peak": hbm_peak,
                         "unit": "GB/s", "frac": alg / (ms * 1e-3) / 1e9 / hbm_peak},
            "l2": "16 buffers cycled, 0.6 GB of inputs and outputs",
            "cpu_oracle_ms_one_thread": cpu_ms}


def picking_leg(dev, steps, warmup):
    """Picking on the 1M-Gaussian config-1 scene: the LBVH build (Morton
    codes, radix sort, leaves and parents; synchronous) and closest-splat
    casts for a 256x256 block of pixel positions under the config-1 camera.
    Also the oracle's build and casts on one host thread for comparison."""
    import numpy as np
    import torch
    from lumen_b200 import scenes
    from lumen_b200 import spatial as S
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    sc = scenes.box_scene(1_000_000, seed=1)
    s, _ = sc.activated()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    means, scales = t(sc.means), t(s)
    cam = scenes.camera_config1(WIDTH, HEIGHT)
    for _ in range(2):
        bvh = S.LBVH(means, scales)
    torch.cuda.synchronize(dev)
    b0 = time.perf_counter()
    nb = max(3, min(steps, 10))
    for _ in range(nb):
        bvh = S.LBVH(means, scales)
    torch.cuda.synchronize(dev)
    build_ms = (time.perf_counter() - b0) * 1e3 / nb
    ys, xs = np.mgrid[412:668, 832:1088]
    px = t(np.stack([xs.reshape(-1) + 0.5, ys.reshape(-1) + 0.5], axis=1))
    for _ in range(max(warmup, 3)):
        raw = bvh.pick(cam, px)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        raw = bvh.pick(cam, px)
    e1.record()
    torch.cuda.synchronize(dev)
    pick_ms = e0.elapsed_time(e1) / steps
    hits = int((raw[:, 0] != 0).sum().item())
    c0 = time.perf_counter()
    nodes, idx, root, _ = O.bvh_build(sc.means, s)
    cpu_build_ms = (time.perf_counter() - c0) * 1e3
    sample = np.asarray(px.cpu().numpy())[::256]
    c1 = time.perf_counter()
    for x, y in sample:
        o, d = O.generate_ray(cam, x, y)
        O.raycast(nodes, idx, root, sc.means, s, o, d, unit=True)
    cpu_ray_us = (time.perf_counter() - c1) * 1e6 / sample.shape[0]
    n_rays = int(px.shape[0])
    return {"workload": "LBVH over 1M Gaussians; picks at a 256x256 pixel block, 1920x1080 camera",
            "build_ms": build_ms, "pick_ms": pick_ms, "rays_per_s": n_rays / (pick_ms * 1e-3), "rays": n_rays,
            "hits": hits, "build_timing": "host wall clock per synchronous build",
            "cpu_oracle_one_thread": {"build_ms": cpu_build_ms, "us_per_ray": cpu_ray_us,
                                      "sample": f"{sample.shape[0]} of the rays"}}


def multiview_leg(dev, steps, warmup, hbm_peak):
    """Configuration 2: 300k Gaussians seen from 64 cameras on a Catmull-Rom
    orbit of radius 10 at 1280x720, all 64 views in one batch
    (lumen_gpu_render_batch: one pipeline, view-prefixed tile ids in the sort
    key). Also the same 64 views rendered one call each, for the batching
    gain. Both device-timed with CUDA events, inputs resident."""
    import numpy as np
    import torch
    from lumen_b200 import _lib as L
    from lumen_b200 import render as R
    from lumen_b200 import scenes
    from lumen_b200.types import RenderOptions
    n, n_views, W, H = 300_000, 64, 1280, 720
    sc = scenes.box_scene(n, seed=2)
    s, op = sc.activated()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    scene = R.Scene(t(sc.means), t(s), t(sc.quats), t(op).reshape(-1), t(sc.sh).reshape(n, 48))
    cams = scenes.orbit_cameras(n_views, W, H, radius=10.0)
    opt = RenderOptions(term_mode=1)
    views = [(scene, c) for c in cams]
    first = R.render_batch(views, opt)
    frame, images = first.frame, first.images
    lib = L.load()
    arr = R.batch_views(views, images)
    copt = L.render_options(opt)
    fs = frame.frame.c_struct()
    stream = torch.cuda.current_stream(dev).cuda_stream
    timer = lib.lumen_gpu_stage_timer_create(max(steps, 1))
    for _ in range(warmup):
        L.check(lib.lumen_gpu_render_batch(arr, n_views, C.byref(copt), C.byref(fs), stream), "batch")
    torch.cuda.synchronize(dev)
    for _ in range(steps):
        L.check(lib.lumen_gpu_render_batch_timed(arr, n_views, C.byref(copt), C.byref(fs), timer, stream), "batch")
    stage = (C.c_float * 4)()
    total = C.c_float(0)
    nfr = C.c_int(0)
    L.check(lib.lumen_gpu_stage_timer_read(timer, stage, C.byref(total), C.byref(nfr)), "timer")
    lib.lumen_gpu_stage_timer_destroy(timer)
    counts = L.LumenGpuCounts()
    L.check(lib.lumen_gpu_read_counts(C.byref(fs), C.byref(counts), stream), "counts")
    assert counts.error_flags == 0 and counts.n_instances == first.n_instances
    ms = total.value / steps
    # the same views, one render call each (device-resident, no host sync between calls)
    singles = [R.render(*scene.tensors, c, opt) for c in cams]
    per = []
    for c, r in zip(cams, singles):
        g1, c1 = scene.struct, L.view_camera(c)
        im = L.LumenGpuImage()
        im.rgb, im.depth, im.alpha = r.rgb.data_ptr(), r.depth.data_ptr(), r.alpha.data_ptr()
        per.append((g1, c1, r.frame.c_struct(), im))

    def one_by_one():
        for g1, c1, f1, im in per:
            L.check(lib.lumen_gpu_render_forward(C.byref(g1), C.byref(c1), C.byref(copt), C.byref(f1),
                                                 C.byref(im), stream), "forward")
    one_by_one()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(steps // 4, 2)
    e0.record()
    for _ in range(reps):
        one_by_one()
    e1.record()
    torch.cuda.synchronize(dev)
    ms_single = e0.elapsed_time(e1) / reps
    V, K = first.n_visible, first.n_instances
    T = sum(c.n_tiles for c in cams)
    P = n_views * W * H
    tile_bits = max(T - 1, 1).bit_length()
    depth_keys = [r.varying_digits >> 8 for r in singles]
    depth_bytes = bin(int(np.bitwise_or.reduce(np.array(depth_keys))) & 0xFF).count("1")
    p = (tile_bits + 7) // 8 + depth_bytes
    b = 236 * n + 8 * n * n_views + 64 * V + (60 + 24 * p) * K + 16 * T + 16 * P
    return {"workload": "config 2: 300k Gaussians, 64 orbit views at 1280x720, one batch per step",
            "views_per_s": n_views * 1000.0 / ms, "ms_per_batch": ms,
            "per_call_views_per_s": n_views * 1000.0 / ms_single, "per_call_ms_for_64": ms_single,
            "stages_ms": {k: round(v / steps, 4) for k, v in zip(["project", "sort", "tile_ranges", "composite"],
                                                                 stage)},
            "visible": V, "instances": K, "tiles": T, "digit_passes": p, "gpu_launches_per_batch": kernels_per_frame(T),
            "roofline": {"bytes": b, "achieved": b / (ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                         "frac": b / (ms * 1e-3) / 1e9 / hbm_peak}}


def _percentile(xs, q):
    s = sorted(xs)
    if not s:
        return None
    i = min(len(s) - 1, max(0, int(round(q / 100.0 * (len(s) - 1)))))
    return s[i]


def _poisson_stream(server, ids, scene_of, cams, rate, n, pools, seed):
    """Submit n requests at Poisson arrival times (rate per second) and
    collect their results; returns (results, wall seconds)."""
    import random
    rng = random.Random(seed)
    handles = []
    used = {k: [None] * len(v) for k, v in pools.items()}
    t0 = time.perf_counter()
    t_next = t0
    for i in range(n):
        t_next += rng.expovariate(rate)
        now = time.perf_counter()
        if t_next > now:
            time.sleep(t_next - now)
        cam = cams[i]
        key = (cam.width, cam.height)
        j = i % len(pools[key])
        prev = used[key][j]
        if prev is not None and prev[1] is None:   # buffer still owned by an earlier request
            prev[1] = prev[0].result(timeout_ms=120_000)
        h = server.submit(ids[scene_of[i]], cam, out=pools[key][j])
        entry = [h, None]
        used[key][j] = entry
        handles.append(entry)
    res = []
    for e in handles:
        if e[1] is None:
            e[1] = e[0].result(timeout_ms=120_000)
        res.append(e[1])
    return res, time.perf_counter() - t0


def _closed_loop(server, ids, scene_of, cams, depth, n, pools):
    """Keep `depth` requests outstanding: submit the first `depth`, then a new
    one each time the oldest completes; returns the n results."""
    from collections import deque
    pending = deque()
    res = []
    slot_of = {k: 0 for k in pools}
    for i in range(n):
        if len(pending) >= depth:
            res.append(pending.popleft().result(timeout_ms=120_000))
        cam = cams[i]
        key = (cam.width, cam.height)
        out = pools[key][slot_of[key] % len(pools[key])]
        slot_of[key] += 1
        pending.append(server.submit(ids[scene_of[i]], cam, out=out))
    while pending:
        res.append(pending.popleft().result(timeout_ms=120_000))
    return res


def _served_summary(res, n):
    lat = [r.latency_ms for r in res]
    span_s = (max(r.done_ms for r in res) - min(r.submit_ms for r in res)) * 1e-3
    return {"served_frames_per_s": n / span_s, "p50_ms": _percentile(lat, 50), "p99_ms": _percentile(lat, 99),
            "mean_batch_views": sum(r.batch_views for r in res) / max(len(res), 1)}


def _batch_ceiling(dev, dscene, lib, opt, n_views):
    """Per-view stage costs of a batch of n_views 1080p views of one scene
    (lumen_gpu_render_batch with stage events): projection is the only
    stage whose input is shared by the views; the sorts, ranges and
    compositing are per view. Returns the per-view milliseconds."""
    from lumen_b200 import _lib as L
    from lumen_b200 import render as R
    from lumen_b200 import scenes
    import torch
    cams = scenes.orbit_cameras(n_views, WIDTH, HEIGHT, radius=10.0)
    views = [(dscene, c) for c in cams]
    first = R.render_batch(views, opt)
    arr = R.batch_views(views, first.images)
    copt = L.render_options(opt)
    fs = first.frame.frame.c_struct()
    stream = torch.cuda.current_stream(dev).cuda_stream
    reps = 5
    timer = lib.lumen_gpu_stage_timer_create(reps)
    L.check(lib.lumen_gpu_render_batch(arr, n_views, C.byref(copt), C.byref(fs), stream), "batch")
    for _ in range(reps):
        L.check(lib.lumen_gpu_render_batch_timed(arr, n_views, C.byref(copt), C.byref(fs), timer, stream), "batch")
    stage = (C.c_float * 4)()
    total = C.c_float(0)
    nfr = C.c_int(0)
    L.check(lib.lumen_gpu_stage_timer_read(timer, stage, C.byref(total), C.byref(nfr)), "timer")
    lib.lumen_gpu_stage_timer_destroy(timer)
    per_view = {k: v / reps / n_views for k, v in zip(["project", "sort", "tile_ranges", "composite"], stage)}
    per_view["total"] = total.value / reps / n_views
    return per_view


def serving_leg(dev, n_requests, hbm_budget):
    """Render serving (configuration 4 and a 1080p stream of the 1M scene)
    through lumen_serve (continuous batching, graph launches, autotuned
    chunk and digit-pass tile), 8-bit RGB delivered to page-locked host
    buffers. One server: a warm-up that lets the autotuner time every launch
    variant on both workloads, then tuning frozen for every timed run. Timed
    runs: Poisson arrivals at offered rates up to and beyond capacity, and
    closed loops holding a fixed number of requests outstanding. Latency =
    delivery - arrival. The same request list is rendered per call
    (lumen_gpu_render_forward + copy of the 8-bit image to the host + wait,
    one request at a time) for comparison. The headline served rate is the
    highest served frames/s of any run whose p99 is at most 20 ms."""
    import random
    import numpy as np
    import torch
    from lumen_b200 import _lib as L
    from lumen_b200 import render as R
    from lumen_b200 import scenes
    from lumen_b200 import serve
    from lumen_b200.types import RenderOptions
    opt = RenderOptions(term_mode=1)
    lib = L.load()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    sizes = scenes.SERVING_SCENE_SIZES
    dscenes = []
    for i, n in enumerate(sizes):
        sc = scenes.box_scene(n, seed=100 + i)
        s, op = sc.activated()
        dscenes.append(R.Scene(t(sc.means), t(s), t(sc.quats), t(op).reshape(-1), t(sc.sh).reshape(n, 48)))
    res_list = scenes.SERVING_RESOLUTIONS
    orbit = {wh: scenes.orbit_cameras(64, wh[0], wh[1], radius=10.0) for wh in res_list}
    pools = {wh: [torch.empty((wh[1], wh[0], 3), dtype=torch.uint8, pin_memory=True)
                  for _ in range(96 if wh[1] < 2000 else 48)] for wh in res_list}

    def workload(kind, n, seed):
        rng = random.Random(seed)
        sc_of, cams = [], []
        for _ in range(n):
            if kind == "mixed":
                s = rng.randrange(len(sizes))
                wh = res_list[rng.randrange(len(res_list))]
            else:
                s, wh = sizes.index(1_000_000), (1920, 1080)
            sc_of.append(s)
            cams.append(orbit[wh][rng.randrange(64)])
        return sc_of, cams

    per_call_frames = {}

    def per_call(sc_of, cams):
        """One request at a time: render, copy the 8-bit image to the host, wait."""
        stream = torch.cuda.current_stream(dev)
        lat = []
        t0 = time.perf_counter()
        for s, cam in zip(sc_of, cams):
            key = (s, cam.width, cam.height)
            if key not in per_call_frames:
                first = R.render(*dscenes[s].tensors, cam, opt)
                rgb8 = torch.empty((cam.height, cam.width, 3), dtype=torch.uint8, device=dev)
                per_call_frames[key] = (first.frame, rgb8, pools[(cam.width, cam.height)][0])
            frame, rgb8, host = per_call_frames[key]
            c0 = time.perf_counter()
            img = L.LumenGpuImage()
            img.rgb8 = rgb8.data_ptr()
            fs = frame.c_struct()
            L.check(lib.lumen_gpu_render_forward(C.byref(dscenes[s].struct), C.byref(L.view_camera(cam)),
                                                 C.byref(L.render_options(opt)), C.byref(fs), C.byref(img),
                                                 stream.cuda_stream), "forward")
            host.copy_(rgb8, non_blocking=True)
            stream.synchronize()
            lat.append((time.perf_counter() - c0) * 1e3)
        return lat, time.perf_counter() - t0

    plans = {"1080p_1M": {"rates": (1400.0, 1800.0, 2200.0, 2600.0, 3200.0), "depths": (4, 8, 16, 32, 64)},
             "mixed": {"rates": (1400.0, 1800.0, 2200.0, 2600.0), "depths": (4, 8, 16, 32, 64)}}
    out = {}
    with serve.Server(work_budget_bytes=hbm_budget, max_views_per_batch=64, max_batches_in_flight=2,
                      use_graphs=True, autotune=True, options=opt) as srv:
        ids = [srv.add_scene(s) for s in dscenes]
        # warm-up: every launch variant of every batch class these runs meet is timed
        for kind in plans:
            for rate, depth, seed in ((2000.0, None, 91), (None, 16, 92), (None, 64, 93), (1400.0, None, 94)):
                w_of, w_cams = workload(kind, 600, seed=seed)
                if rate:
                    _poisson_stream(srv, ids, w_of, w_cams, rate, len(w_cams), pools, seed=seed)
                else:
                    _closed_loop(srv, ids, w_of, w_cams, depth, len(w_cams), pools)
        srv.freeze_tuning(True)
        for kind, plan in plans.items():
            sc_of, cams = workload(kind, n_requests, seed=7 if kind == "mixed" else 8)
            s0 = srv.stats()
            runs = []
            for rate in plan["rates"]:
                res, _ = _poisson_stream(srv, ids, sc_of, cams, rate, n_requests, pools, seed=6)
                assert all(r.status == 0 for r in res), "served request failed"
                runs.append(dict(mode="poisson", offered_req_per_s=rate, **_served_summary(res, n_requests)))
            for depth in plan["depths"]:
                res = _closed_loop(srv, ids, sc_of, cams, depth, n_requests, pools)
                assert all(r.status == 0 for r in res), "served request failed"
                runs.append(dict(mode="closed_loop", outstanding=depth, **_served_summary(res, n_requests)))
            s1 = srv.stats()
            # per-call: frames prepared by one untimed pass over the distinct (scene, resolution) pairs
            per_call(sc_of[:min(len(sc_of), 64)], cams[:min(len(cams), 64)])
            pc_lat, pc_wall = per_call(sc_of, cams)
            pc_fps = n_requests / pc_wall
            ok = [r for r in runs if r["p99_ms"] is not None and r["p99_ms"] <= 20.0]
            best = max(ok, key=lambda r: r["served_frames_per_s"]) if ok else None
            out[kind] = {
                "requests_per_run": n_requests, "runs": runs,
                "per_call_frames_per_s": pc_fps, "per_call_p50_ms": _percentile(pc_lat, 50),
                "per_call_p99_ms": _percentile(pc_lat, 99),
                "best_served_at_p99_le_20ms": best,
                "served_over_per_call": (best["served_frames_per_s"] / pc_fps) if best else None,
                "batches": s1["batches"] - s0["batches"],
                "requeued_batches": s1["requeued_batches"] - s0["requeued_batches"],
                "explored_batches_in_timed_runs": s1["explored_batches"] - s0["explored_batches"]}
    # the bound: what a batch of 1080p views of the 1M scene costs per view, by stage, at the
    # server's largest batch of such views (8: 65 280 tiles; a ninth view adds a tile-sort pass)
    ceil = _batch_ceiling(dev, dscenes[sizes.index(1_000_000)], lib, opt, 8)
    per_view_unshared = ceil["sort"] + ceil["tile_ranges"] + ceil["composite"]
    out["ceiling_1080p_1M"] = {
        "per_view_stage_ms_in_8_view_batch": {k: round(v, 4) for k, v in ceil.items()},
        "frames_per_s_if_projection_were_free": 1000.0 / per_view_unshared,
        "frames_per_s_at_measured_batch_cost": 1000.0 / ceil["total"],
        "note": "sorts, tile ranges and compositing read and write per-view data; only projection reads the "
                "shared scene, so no batching can serve more than frames_per_s_if_projection_were_free"}
    out["workload"] = ("config 4: 8 resident scenes {50k..2M} (6.4M Gaussians), random scene, orbit camera and "
                       "resolution in {640x480, 1280x720, 1920x1080, 3840x2160}; and a 1080p stream of the 1M "
                       "scene; 8-bit RGB to page-locked host memory; Poisson offered-rate sweep and closed loops")
    return out


def ncu_counters():
    """Per-kernel counters of the latest ncu captures (profiles/kernel_counters.csv:
    one row per kernel and workload, with the command that captured it)."""
    import csv
    path = os.path.join(ROOT, "profiles", "kernel_counters.csv")
    if not os.path.exists(path):
        return []
    with open(path) as f:
        rows = [r for r in csv.DictReader(l for l in f if not l.startswith("#"))]
    for r in rows:
        for k in list(r):
            try:
                r[k] = float(r[k]) if k not in ("stage", "kernel", "workload", "binding", "capture") else r[k]
            except (TypeError, ValueError):
                pass
    return rows


SMS, SCHEDULERS_PER_SM = 148, 4


def kernels_table(line, hbm_peak, sm_mhz=1965.0):
    """Each stage of the forward (configuration 1) and of the backward
    (configuration 3): live CUDA-event milliseconds, algorithmic bytes and
    their fraction of the HBM peak, and the instruction-issue and pipe
    figures of its kernels from the latest ncu capture. A stage whose
    kernels are issue-bound reports that as its bound.

    issue_roofline is the compute-side bound of a stage: its kernels' warp
    instructions (ncu's count, summed over the stage's launches) over the
    GPU's issue rate, one warp instruction per scheduler per cycle (148 SMs
    x 4 schedulers x sm_mhz), against the live stage time."""
    counters = ncu_counters()
    rows = []
    issue_rate = SMS * SCHEDULERS_PER_SM * sm_mhz * 1e6

    def add(stage, workload, ms, bytes_):
        gbs = bytes_ / (ms * 1e-3) / 1e9 if ms > 0 else None
        ncu = [{k: v for k, v in c.items() if k not in ("stage", "workload")} for c in counters
               if c.get("stage") == stage and c.get("workload") == workload]
        binding = None
        issue = None
        if ncu:
            top = max(ncu, key=lambda c: c.get("duration_us") or 0)
            binding = top.get("binding")
            instr = sum(c.get("warp_instructions") or 0 for c in ncu)
            if instr > 0 and ms > 0:
                min_ms = instr / issue_rate * 1e3
                issue = {"warp_instructions": int(instr), "min_ms": round(min_ms, 4),
                         "frac": round(min_ms / ms, 3), "sm_mhz": sm_mhz}
        rows.append({"stage": stage, "workload": workload, "ms": round(ms, 4), "algorithmic_bytes": int(bytes_),
                     "hbm_gbs": gbs, "hbm_frac": gbs / hbm_peak if gbs else None, "binding": binding,
                     "issue_roofline": issue, "ncu": ncu})

    c = line.get("counts", {})
    st = line.get("stages_ms", {})
    N, V, K, T, p = N_GAUSSIANS, c.get("visible", 0), c.get("instances", 0), c.get("tiles", 0), c.get("digit_passes", 0)
    P = WIDTH * HEIGHT
    if st:
        add("project", "config 1", st["project"], 236 * N + 48 * V + 4 * N)
        add("sort", "config 1", st["sort"], 8 * N + 16 * V + 12 * K + 8 * K + 24 * K * p + 8 * T)
        add("tile_ranges", "config 1", st["tile_ranges"], 8 * T)
        add("composite", "config 1", st["composite"], 40 * K + 16 * P)
    fb = line.get("fwd_bwd")
    if fb and "stages_ms" in fb:
        z, s3 = fb["sizes"], fb["stages_ms"]
        n3, V3, K3, P3, T3, p3 = z["n"], z["visible"], z["instances"], z["pixels"], z["tiles"], z["digit_passes"]
        add("project", "config 3", s3["project"], 236 * n3 + 48 * V3 + 4 * n3)
        add("sort", "config 3", s3["sort"], 8 * n3 + 16 * V3 + 12 * K3 + 8 * K3 + 24 * K3 * p3 + 8 * T3)
        add("tile_ranges", "config 3", s3["tile_ranges"], 8 * T3)
        add("composite", "config 3", s3["composite"], 40 * K3 + 16 * P3)
        add("composite_backward", "config 3", s3["composite_backward"], 80 * K3 + 12 * P3)
        add("project_backward", "config 3", s3["project_backward"], 88 * V3 + 472 * n3)
    return rows


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        reference_arm(args, world, rank)
        return
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist

    from lumen_b200 import _lib as L
    from lumen_b200 import render as R
    from lumen_b200 import scenes
    from lumen_b200.types import RenderOptions

    with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else open(os.devnull) as f:
        try:
            peaks = json.load(f)
        except ValueError:
            peaks = {}
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    sc = scenes.box_scene(N_GAUSSIANS, seed=1)
    scales, opac = sc.activated()
    cam = scenes.camera_config1(WIDTH, HEIGHT)
    opt = RenderOptions(term_mode=1)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    means, sc_t, quats, op_t, sh = t(sc.means), t(scales), t(sc.quats), t(opac), t(sc.sh).reshape(-1, 48)

    # first render sizes the frame buffers and gives V, K for the byte counts
    first = R.render(means, sc_t, quats, op_t, sh, cam, opt)
    frame = first.frame
    V, K, T = first.n_visible, first.n_instances, cam.n_tiles
    # bytes of the reference's 64-bit key that vary: tile-id bytes (low 8 bits of the mask,
    # key bytes 4..7) and depth-key bytes (next 8 bits, key bytes 0..3)
    passes = bin(first.varying_digits & 0xFFFF).count("1")
    lib = L.load()
    g = R.gaussians_struct(means, sc_t, quats, op_t, sh)
    ccam, copt = L.view_camera(cam), L.render_options(opt)
    fs = frame.c_struct()
    img = L.LumenGpuImage()
    rgb = torch.empty((HEIGHT, WIDTH, 3), dtype=torch.float32, device=dev)
    depth = torch.empty((HEIGHT, WIDTH), dtype=torch.float32, device=dev)
    alpha = torch.empty((HEIGHT, WIDTH), dtype=torch.float32, device=dev)
    img.rgb, img.depth, img.alpha = rgb.data_ptr(), depth.data_ptr(), alpha.data_ptr()
    stream = torch.cuda.current_stream(dev).cuda_stream
    timer = lib.lumen_gpu_stage_timer_create(max(args.steps, 1))

    for _ in range(args.warmup):
        L.check(lib.lumen_gpu_render_forward(C.byref(g), C.byref(ccam), C.byref(copt), C.byref(fs), C.byref(img),
                                             stream), "forward")
    torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        # the timed region: K back-to-back frames bracketed by two events on the render stream
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.current_stream(dev))
        for _ in range(args.steps):
            L.check(lib.lumen_gpu_render_forward(C.byref(g), C.byref(ccam), C.byref(copt), C.byref(fs),
                                                 C.byref(img), stream), "forward")
        e1.record(torch.cuda.current_stream(dev))
        torch.cuda.synchronize(dev)
        frames_ms = e0.elapsed_time(e1)
        # then the same K frames with events between the stages, for the stage split
        for _ in range(args.steps):
            L.check(lib.lumen_gpu_render_forward_timed(C.byref(g), C.byref(ccam), C.byref(copt), C.byref(fs),
                                                       C.byref(img), timer, stream), "forward")
        stage = (C.c_float * 4)()
        total = C.c_float(0)
        nfr = C.c_int(0)
        L.check(lib.lumen_gpu_stage_timer_read(timer, stage, C.byref(total), C.byref(nfr)), "timer")
        torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    counts = L.LumenGpuCounts()
    L.check(lib.lumen_gpu_read_counts(C.byref(fs), C.byref(counts), stream), "counts")
    assert counts.error_flags == 0, f"device flags {counts.error_flags:#x}"
    assert counts.n_instances == K
    lib.lumen_gpu_stage_timer_destroy(timer)
    steps = args.steps
    # event span over the K back-to-back frames (gaps included); the stage
    # split comes from the second, event-instrumented run of K frames
    ms = frames_ms / steps
    ms_max, value = replica_throughput(ms, world, pg, dev)

    stage_ms = [x / steps for x in stage]
    names = ["project", "sort", "tile_ranges", "composite"]
    # algorithmic bytes per launch; p = digit passes of the
    # reference's 64-bit key sort that vary (its 8-pass sort with constant digits skipped)
    P = WIDTH * HEIGHT
    p = passes
    alg = {"project": 236 * N_GAUSSIANS + 48 * V + 4 * N_GAUSSIANS,
           "sort": 8 * N_GAUSSIANS + 16 * V + 12 * K + 8 * K + 24 * K * p + 8 * T,
           "tile_ranges": 8 * T,
           "composite": 40 * K + 16 * P}
    # the dominant kernel: composite_kernel, the largest share of the frame's
    # launch list (profiles/forward_config1_launches.md); the sort stage is
    # nine kernels, none above an eighth of the frame
    dom = names.index("composite")
    dname = names[dom]
    achieved = alg[dname] / (stage_ms[dom] * 1e-3) / 1e9
    b_fwd = 244 * N_GAUSSIANS + 64 * V + (60 + 24 * passes) * K + 16 * T + 16 * P
    frame_gbs = b_fwd / (ms_max * 1e-3) / 1e9

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": args.warmup,
            "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": workload_config({"parallelism": f"replicas x{world}" if world > 1 else "single GPU"}),
            "gpu_launches": kernels_per_frame(T) * steps,
            "clocks": clk.summary(),
            "stages_ms": {n: round(v, 4) for n, v in zip(names, stage_ms)},
            "stages_timing": "a second run of the K frames with CUDA events between the stages",
            "counts": {"visible": V, "instances": K, "tiles": T, "digit_passes": passes},
            "roofline": {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": COMPOSITE_DRAM_BYTES, "peak_source": peak_src,
                         "algorithmic_bytes": alg[dname],
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one composite_kernel "
                                           "launch at this workload (profiles/forward_config1_kernels.md)"},
            "frame_roofline": {"bytes": b_fwd, "achieved": frame_gbs, "peak": hbm_peak, "unit": "GB/s",
                               "frac": frame_gbs / hbm_peak}}
    if not args.no_multiview:
        line["multiview"] = multiview_leg(dev, min(steps, 20), min(args.warmup, 3), hbm_peak)
    if not args.no_serving:
        line["serving"] = serving_leg(dev, args.serve_requests, 24 << 30)
    if not args.no_fwd_bwd:
        line["fwd_bwd"] = fwd_bwd_leg(dev, min(steps, 100), args.warmup, hbm_peak)
    if not args.no_train:
        line["train_step"] = train_leg(dev, min(steps, 50))
    if not args.no_depth:
        line["depth_products"] = depth_leg(dev, min(steps, 200), args.warmup, hbm_peak)
    if not args.no_picking:
        line["picking"] = picking_leg(dev, min(steps, 50), args.warmup)
    if not args.no_e2e:
        e2e = e2e_rasterize(sc, scales, opac, steps, args.warmup)
        if pg:   # replicas: the slowest rank's rate times the number of ranks
            e2e["value"] = replica_rate(e2e["value"], world, pg, dev)
        line["e2e"] = e2e
        srv = line.get("serving", {}).get("1080p_1M")
        if srv and srv["best_served_at_p99_le_20ms"]:   # served frames against the drop-in C ABI per call
            srv["served_over_capi_per_call"] = srv["best_served_at_p99_le_20ms"]["served_frames_per_s"] / e2e["value"]
    # the issue bound at the SM clock sampled during the timed frames
    sm_mhz = (line.get("clocks") or {}).get("sm_mhz") or float(peaks.get("sm_max_mhz", 1965.0))
    line["kernels"] = kernels_table(line, hbm_peak, float(sm_mhz))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
