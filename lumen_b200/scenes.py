"""Seeded synthetic scenes for the five workload configurations.

Every scene is drawn with numpy ``PCG64(seed)`` in float64 and cast to
float32, in this order: means, scales, rotations, opacities, SH. Rotations are
normalised 4-D standard normals (uniform on SO(3)); SH is ``[N, 16, 3]`` with
the DC term ~ N(0.5, 0.15) and higher orders ~ N(0, 0.05), laid out as
``sh[i*48 + coef*3 + ch]`` like the reference's ``GaussianSoA.sh_data``
(src/scene/gaussian.mojo:65,103-107).

Parameters are returned raw: ``log_scales`` and ``opacity_logits``.
``activate`` applies exp and sigmoid in float32 for the reference-style
(activated) entry points.

Configurations (sizes, shapes and distributions of the five workloads):

0. 512 Gaussians on an 8x8x8 grid over [-1,1]^3 with N(0, 0.02) jitter, centred
   4 units ahead of the camera, log-scales U(ln .02, ln .08), logits N(0, 1);
   800x600, vertical FOV 60 degrees.
1. 1M Gaussians uniform in a 6x4x6 box centred 8 units ahead, log-scales
   U(ln .003, ln .05), logits N(0, 1.5); 1920x1080, FOV 50 degrees.
2. 300k Gaussians as config 1; 64 cameras on a Catmull-Rom orbit of radius 10
   around the box centre, 1280x720.
3. 500k Gaussians as config 1 at 1920x1080; the target scene perturbs means by
   N(0, .01), log-scales by N(0, .05) and SH by N(0, .02).
4. 8 resident scenes of {50k, 100k, 250k, 500k, 1M, 1M, 1.5M, 2M} Gaussians
   drawn as config 1; requests pick a scene, an orbit camera and one of
   640x480, 1280x720, 1920x1080, 3840x2160.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Tuple

import numpy as np

from .types import ViewCamera, look_at_quaternion


@dataclass
class Scene:
    means: np.ndarray            # [N, 3] float32
    log_scales: np.ndarray       # [N, 3] float32
    quats: np.ndarray            # [N, 4] float32 (w, x, y, z)
    opacity_logits: np.ndarray   # [N]    float32
    sh: np.ndarray               # [N, 16, 3] float32

    @property
    def n(self) -> int:
        return int(self.means.shape[0])

    def activated(self) -> Tuple[np.ndarray, np.ndarray]:
        """(scales, opacities) in float32: exp(log_scales), sigmoid(logits)."""
        return activate(self.log_scales, self.opacity_logits)

    def subset(self, idx) -> "Scene":
        return Scene(self.means[idx].copy(), self.log_scales[idx].copy(), self.quats[idx].copy(),
                     self.opacity_logits[idx].copy(), self.sh[idx].copy())


def activate(log_scales: np.ndarray, logits: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    s = np.exp(log_scales.astype(np.float32)).astype(np.float32)
    o = (np.float32(1.0) / (np.float32(1.0) + np.exp(-logits.astype(np.float32)))).astype(np.float32)
    return s, o


def _draw_rest(rng: np.random.Generator, n: int, ls_lo: float, ls_hi: float, logit_sigma: float):
    log_scales = rng.uniform(math.log(ls_lo), math.log(ls_hi), size=(n, 3))
    q = rng.standard_normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    logits = rng.normal(0.0, logit_sigma, size=n)
    sh = rng.normal(0.0, 0.05, size=(n, 16, 3))
    sh[:, 0, :] = rng.normal(0.5, 0.15, size=(n, 3))
    return log_scales, q, logits, sh


def _pack(means, log_scales, q, logits, sh) -> Scene:
    f = np.float32
    return Scene(np.ascontiguousarray(means, dtype=f), np.ascontiguousarray(log_scales, dtype=f),
                 np.ascontiguousarray(q, dtype=f), np.ascontiguousarray(logits, dtype=f),
                 np.ascontiguousarray(sh, dtype=f))


def grid_scene(seed: int = 0) -> Scene:
    """Config 0: 8x8x8 jittered grid over [-1,1]^3 centred at (0, 0, 4)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ax = np.linspace(-1.0, 1.0, 8)
    g = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), axis=-1).reshape(-1, 3)
    means = g + rng.normal(0.0, 0.02, size=g.shape) + np.array([0.0, 0.0, 4.0])
    return _pack(means, *_draw_rest(rng, means.shape[0], 0.02, 0.08, 1.0))


def box_scene(n: int, seed: int = 1, centre=(0.0, 0.0, 8.0)) -> Scene:
    """Configs 1-4: n Gaussians uniform in a 6x4x6 box around ``centre``."""
    rng = np.random.Generator(np.random.PCG64(seed))
    half = np.array([3.0, 2.0, 3.0])
    means = rng.uniform(-half, half, size=(n, 3)) + np.asarray(centre)
    return _pack(means, *_draw_rest(rng, n, 0.003, 0.05, 1.5))


def perturbed(scene: Scene, seed: int) -> Scene:
    """Config 3 target: means + N(0,.01), log-scales + N(0,.05), SH + N(0,.02)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    m = scene.means + rng.normal(0.0, 0.01, size=scene.means.shape)
    ls = scene.log_scales + rng.normal(0.0, 0.05, size=scene.log_scales.shape)
    sh = scene.sh + rng.normal(0.0, 0.02, size=scene.sh.shape)
    return _pack(m, ls, scene.quats, scene.opacity_logits, sh)


def camera_config0() -> ViewCamera:
    return ViewCamera.from_fov(800, 600, 60.0)


def camera_config1(width: int = 1920, height: int = 1080, fov: float = 50.0) -> ViewCamera:
    return ViewCamera.from_fov(width, height, fov)


def catmull_rom(p0, p1, p2, p3, t: float) -> np.ndarray:
    """Catmull-Rom cubic through p1..p2 (src/scene/trajectory.mojo:24-42)."""
    t2 = t * t
    t3 = t2 * t
    f1 = -0.5 * t3 + t2 - 0.5 * t
    f2 = 1.5 * t3 - 2.5 * t2 + 1.0
    f3 = -1.5 * t3 + 2.0 * t2 + 0.5 * t
    f4 = 0.5 * t3 - 0.5 * t2
    return (np.asarray(p0) * f1 + np.asarray(p1) * f2 + np.asarray(p2) * f3 + np.asarray(p3) * f4)


def orbit_cameras(n_views: int, width: int, height: int, fov: float = 50.0, radius: float = 10.0,
                  centre=(0.0, 0.0, 8.0), height_offset: float = 2.0, n_keys: int = 8,
                  phase: float = 0.0) -> List[ViewCamera]:
    """Cameras sampled on a closed Catmull-Rom spline through ``n_keys`` key
    positions on a circle of ``radius`` around ``centre``, each looking at the
    centre (our own look-at, camera z forward)."""
    c = np.asarray(centre, dtype=np.float64)
    keys = [c + np.array([radius * math.cos(phase + 2 * math.pi * k / n_keys), height_offset,
                          radius * math.sin(phase + 2 * math.pi * k / n_keys)]) for k in range(n_keys)]
    cams = []
    for v in range(n_views):
        s = v * n_keys / n_views
        i = int(math.floor(s))
        t = s - i
        p = catmull_rom(keys[(i - 1) % n_keys], keys[i % n_keys], keys[(i + 1) % n_keys],
                        keys[(i + 2) % n_keys], t)
        q = look_at_quaternion(p, c, (0.0, 1.0, 0.0))
        cams.append(ViewCamera.from_fov(width, height, fov, position=tuple(p), rotation=q))
    return cams


SERVING_SCENE_SIZES = (50_000, 100_000, 250_000, 500_000, 1_000_000, 1_000_000, 1_500_000, 2_000_000)
SERVING_RESOLUTIONS = ((640, 480), (1280, 720), (1920, 1080), (3840, 2160))
