"""SDK camera types: the reference Python SDK's ``Camera`` and
``CameraTrajectory`` (python/lumen/camera.py:9-129), same constructor
arguments, attributes and return values.

A ``Camera`` is a look-at pinhole: position, target, up, horizontal and
vertical field of view, near and far planes. ``view_camera`` turns it into
the device-side ``ViewCamera`` (rotation with camera z forward, x right, y
down; "up" points up in the image) for a given resolution.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

from .types import ViewCamera


class Camera:
    """Pinhole camera descriptor (reference python/lumen/camera.py:9-28)."""

    def __init__(self, position: Sequence[float] = (0.0, 0.0, 3.0), target: Sequence[float] = (0.0, 0.0, 0.0),
                 up: Sequence[float] = (0.0, 1.0, 0.0), fov_x_deg: float = 60.0, fov_y_deg: float = 45.0,
                 near_plane: float = 0.1, far_plane: float = 100.0):
        self.position = [float(v) for v in position]
        self.target = [float(v) for v in target]
        self.up = [float(v) for v in up]
        self.fov_x_deg = float(fov_x_deg)
        self.fov_y_deg = float(fov_y_deg)
        self.near_plane = float(near_plane)
        self.far_plane = float(far_plane)

    def forward_vector(self) -> Tuple[float, float, float]:
        """Unit vector from position to target; (0, 0, -1) when they coincide
        (reference camera.py:30-38)."""
        d = [t - p for t, p in zip(self.target, self.position)]
        n = math.sqrt(sum(c * c for c in d))
        if n < 1e-6:
            return (0.0, 0.0, -1.0)
        return (d[0] / n, d[1] / n, d[2] / n)

    def view_matrix_4x4(self) -> List[List[float]]:
        """OpenGL-style look-at view matrix, rows (right, true up, -forward)
        with translations (reference camera.py:40-69)."""
        f = self.forward_vector()
        u = self.up
        r = (f[1] * u[2] - f[2] * u[1], f[2] * u[0] - f[0] * u[2], f[0] * u[1] - f[1] * u[0])
        rn = math.sqrt(sum(c * c for c in r))
        r = (1.0, 0.0, 0.0) if rn < 1e-6 else (r[0] / rn, r[1] / rn, r[2] / rn)
        tu = (r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0])
        p = self.position
        dot = lambda a, b: a[0] * b[0] + a[1] * b[1] + a[2] * b[2]
        return [[r[0], r[1], r[2], -dot(r, p)],
                [tu[0], tu[1], tu[2], -dot(tu, p)],
                [-f[0], -f[1], -f[2], dot(f, p)],
                [0.0, 0.0, 0.0, 1.0]]

    def view_camera(self, width: int, height: int, near_plane: float = None,
                    far_plane: float = None) -> ViewCamera:
        """Device camera for a width x height image, computed by liblumen's
        lumen_gpu_camera_from_lookat (the conversion lumen_rasterize uses):
        fx = fy = H / (2 tan(fov_y/2)), principal point at the centre
        (c_api/src/lumen_c.c:393-395,422-423), camera z toward the target."""
        import ctypes as C
        from . import _lib as L
        lib = L.load()
        src = L.LumenCamera(L.LumenVec3(*self.position), L.LumenVec3(*self.target), L.LumenVec3(*self.up),
                            self.fov_x_deg, self.fov_y_deg, self.near_plane, self.far_plane)
        out = L.LumenViewCamera()
        L.check(lib.lumen_gpu_camera_from_lookat(C.byref(src), int(width), int(height),
                                                 self.near_plane if near_plane is None else near_plane,
                                                 self.far_plane if far_plane is None else far_plane,
                                                 C.byref(out)), "camera_from_lookat")
        return ViewCamera(tuple(out.position), tuple(out.rotation), out.fx, out.fy, out.cx, out.cy,
                          out.near_plane, out.far_plane, out.width, out.height)


class CameraTrajectory:
    """Camera paths (reference python/lumen/camera.py:72-129)."""

    @staticmethod
    def orbit(target: Sequence[float] = (0.0, 0.0, 0.0), radius: float = 3.0, elevation_deg: float = 15.0,
              num_frames: int = 60, fov_y_deg: float = 45.0) -> List[Camera]:
        """num_frames cameras evenly spaced in azimuth on a circle of the given
        radius and elevation around target, all looking at it."""
        elev = math.radians(elevation_deg)
        y = target[1] + radius * math.sin(elev)
        horiz = radius * math.cos(elev)
        cams = []
        for i in range(num_frames):
            az = 2.0 * math.pi * i / num_frames
            cams.append(Camera(position=(target[0] + horiz * math.sin(az), y, target[2] + horiz * math.cos(az)),
                               target=tuple(target), up=(0.0, 1.0, 0.0), fov_y_deg=fov_y_deg))
        return cams

    @staticmethod
    def interpolate(cam_a: Camera, cam_b: Camera, t: float) -> Camera:
        """Linear blend of position, target and vertical FOV with t clamped to
        [0, 1]; up, near and far from cam_a."""
        t = max(0.0, min(1.0, t))
        mix = lambda a, b: tuple(x * (1.0 - t) + y * t for x, y in zip(a, b))
        return Camera(position=mix(cam_a.position, cam_b.position), target=mix(cam_a.target, cam_b.target),
                      up=cam_a.up, fov_y_deg=cam_a.fov_y_deg * (1.0 - t) + cam_b.fov_y_deg * t,
                      near_plane=cam_a.near_plane, far_plane=cam_a.far_plane)
