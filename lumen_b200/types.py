"""Host-side descriptors shared by the device API, the SDK mirror and the tests.

``ViewCamera`` is the reference's ``PinholeCamera`` (src/scene/camera.mojo:24-40):
a world position, a rotation quaternion (w, x, y, z) whose inverse maps world
offsets into camera space (camera.mojo:69-71), and the ``CameraConfig``
intrinsics (src/core/config.mojo:17-51). The identity rotation looks down +z
with image x to the right and y down.

``RenderOptions`` carries the ``RenderConfig`` fields the render path reads
(src/core/config.mojo:65-102) plus the switches this build adds:

* ``key_mode``: 0 keys depth in millimetres, ``clamp(Int64(z*1000), 0, 2^31-1)``
  (src/raster/radix_sort.mojo:8-18); 1 keys the raw float bits of z.
* ``term_mode``: 0 stops a pixel once T <= ``term_threshold`` after a blend
  (src/raster/compositor.mojo:53 with TRANSMITTANCE_EPSILON = 1e-4,
  types.mojo:35); 1 stops once the accumulated alpha 1 - T >=
  ``term_threshold`` (0.99, the early-termination alpha of the C and Python
  interfaces).
* ``params_are_logits``: 1 when scales are log-scales and opacities are
  logits; the kernels then apply exp and sigmoid themselves.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Sequence, Tuple

import numpy as np

TILE = 16


@dataclass
class ViewCamera:
    position: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rotation: Tuple[float, float, float, float] = (1.0, 0.0, 0.0, 0.0)
    fx: float = 800.0
    fy: float = 800.0
    cx: float = 640.0
    cy: float = 360.0
    near_plane: float = 0.01
    far_plane: float = 1000.0
    width: int = 1280
    height: int = 720

    @property
    def tiles_x(self) -> int:
        return (self.width + TILE - 1) // TILE

    @property
    def tiles_y(self) -> int:
        return (self.height + TILE - 1) // TILE

    @property
    def n_tiles(self) -> int:
        return self.tiles_x * self.tiles_y

    @staticmethod
    def from_fov(width: int, height: int, fov_y_deg: float, position=(0.0, 0.0, 0.0),
                 rotation=(1.0, 0.0, 0.0, 0.0), near_plane=0.01, far_plane=1000.0) -> "ViewCamera":
        """Pinhole intrinsics from a vertical field of view: fy = (H/2)/tan(fov/2), fx = fy,
        principal point at the image centre."""
        fy = (height * 0.5) / math.tan(math.radians(fov_y_deg) * 0.5)
        return ViewCamera(tuple(float(v) for v in position), tuple(float(v) for v in rotation),
                          float(fy), float(fy), width * 0.5, height * 0.5, near_plane, far_plane,
                          int(width), int(height))


@dataclass
class RenderOptions:
    lowpass: float = 0.3
    sh_degree: int = 3
    white_background: bool = False
    compute_depth: bool = True
    key_mode: int = 0
    term_mode: int = 0
    params_are_logits: bool = False
    tile_size: int = TILE
    term_threshold: float = -1.0   # < 0: the mode's default (1e-4 for mode 0, 0.99 for mode 1)

    def __post_init__(self):
        if self.term_threshold < 0:
            self.term_threshold = 1e-4 if self.term_mode == 0 else 0.99

    def with_(self, **kw) -> "RenderOptions":
        return replace(self, **kw)


def look_at_quaternion(eye: Sequence[float], target: Sequence[float],
                       up: Sequence[float] = (0.0, 1.0, 0.0)) -> Tuple[float, float, float, float]:
    """Rotation (w, x, y, z) of a camera at ``eye`` looking at ``target`` in the
    reference camera convention: camera z forward, x right, y down (image rows
    grow downward). The columns of the camera-to-world matrix are
    (right, down, forward); the quaternion is extracted with the four-branch
    method (largest diagonal term first), which is stable for every rotation.

    The reference's own ``PinholeCamera.look_at`` (camera.mojo:43-64) builds a
    -z-forward frame that culls every target; this function replaces it."""
    e = np.asarray(eye, dtype=np.float64)
    t = np.asarray(target, dtype=np.float64)
    u = np.asarray(up, dtype=np.float64)
    f = t - e
    f /= np.linalg.norm(f)
    r = np.cross(f, u)
    nr = np.linalg.norm(r)
    if nr < 1e-12:
        r = np.cross(f, np.array([1.0, 0.0, 0.0]))
        nr = np.linalg.norm(r)
    r /= nr
    d = np.cross(f, r)          # image down
    m = np.stack([r, d, f], axis=1)   # camera-to-world
    return rotation_matrix_to_quaternion(m)


def rotation_matrix_to_quaternion(m: np.ndarray) -> Tuple[float, float, float, float]:
    m = np.asarray(m, dtype=np.float64)
    tr = m[0, 0] + m[1, 1] + m[2, 2]
    if tr > 0.0:
        s = math.sqrt(tr + 1.0) * 2.0
        w = 0.25 * s
        x = (m[2, 1] - m[1, 2]) / s
        y = (m[0, 2] - m[2, 0]) / s
        z = (m[1, 0] - m[0, 1]) / s
    elif m[0, 0] > m[1, 1] and m[0, 0] > m[2, 2]:
        s = math.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2]) * 2.0
        w = (m[2, 1] - m[1, 2]) / s
        x = 0.25 * s
        y = (m[0, 1] + m[1, 0]) / s
        z = (m[0, 2] + m[2, 0]) / s
    elif m[1, 1] > m[2, 2]:
        s = math.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2]) * 2.0
        w = (m[0, 2] - m[2, 0]) / s
        x = (m[0, 1] + m[1, 0]) / s
        y = 0.25 * s
        z = (m[1, 2] + m[2, 1]) / s
    else:
        s = math.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1]) * 2.0
        w = (m[1, 0] - m[0, 1]) / s
        x = (m[0, 2] + m[2, 0]) / s
        y = (m[1, 2] + m[2, 1]) / s
        z = 0.25 * s
    q = np.array([w, x, y, z])
    q /= np.linalg.norm(q)
    if q[0] < 0:
        q = -q
    return tuple(float(v) for v in q)
