"""SDK scene types: the reference Python SDK's ``Gaussian3D`` and
``GaussianCloud`` (python/lumen/cloud.py:11-199) with the same fields,
generators and ASCII PLY round trip, plus array views for the device path.

``GaussianCloud.to_aos`` packs the splats into the 236-byte ``LumenGaussian``
layout of include/lumen.h (position, scale, rotation w-x-y-z, opacity, 48 SH
coefficients); a cloud built with ``from_arrays`` keeps its arrays and packs
without a Python loop.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

SH_C0 = 0.2820947917   # degree-0 real SH basis value, 0.5 * sqrt(1/pi)


@dataclass
class Gaussian3D:
    """One splat (reference cloud.py:11-18)."""
    position: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    scale: Tuple[float, float, float] = (0.05, 0.05, 0.05)
    rotation: Tuple[float, float, float, float] = (1.0, 0.0, 0.0, 0.0)
    opacity: float = 0.8
    sh_coeffs: List[float] = field(default_factory=lambda: [0.0] * 48)


class GaussianCloud:
    """A list of splats (reference cloud.py:21-65); optionally backed by arrays."""

    def __init__(self, splats: Optional[List[Gaussian3D]] = None):
        self.splats: List[Gaussian3D] = splats if splats is not None else []
        self._aos: Optional[np.ndarray] = None

    def __len__(self) -> int:
        return len(self.splats) if self._aos is None else int(self._aos.shape[0])

    def add(self, splat: Gaussian3D) -> None:
        self._materialize()
        self.splats.append(splat)

    def bounding_box(self):
        if len(self) == 0:
            return ((0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
        p = self.to_aos()[:, 0:3].astype(np.float64)
        return tuple(float(v) for v in p.min(0)), tuple(float(v) for v in p.max(0))

    def centroid(self):
        if len(self) == 0:
            return (0.0, 0.0, 0.0)
        return tuple(float(v) for v in self.to_aos()[:, 0:3].astype(np.float64).mean(0))

    # ---- array views -------------------------------------------------------------
    @classmethod
    def from_arrays(cls, means, scales, quats, opacities, sh) -> "GaussianCloud":
        """Array-backed cloud: scales linear, opacities in [0, 1], sh [N, 48] or [N, 16, 3]."""
        n = int(np.asarray(means).shape[0])
        aos = np.empty((n, 59), np.float32)
        aos[:, 0:3] = means
        aos[:, 3:6] = scales
        aos[:, 6:10] = quats
        aos[:, 10] = np.asarray(opacities).reshape(n)
        aos[:, 11:59] = np.asarray(sh).reshape(n, 48)
        c = cls()
        c._aos = aos
        return c

    def _materialize(self) -> None:
        if self._aos is not None:
            a = self._aos
            self.splats = [Gaussian3D(tuple(map(float, r[0:3])), tuple(map(float, r[3:6])),
                                      tuple(map(float, r[6:10])), float(r[10]), [float(v) for v in r[11:59]])
                           for r in a]
            self._aos = None

    def to_aos(self) -> np.ndarray:
        """[N, 59] float32 in LumenGaussian field order."""
        if self._aos is not None:
            return self._aos
        out = np.zeros((len(self.splats), 59), np.float32)
        for i, g in enumerate(self.splats):
            out[i, 0:3] = g.position
            out[i, 3:6] = g.scale
            out[i, 6:10] = g.rotation
            out[i, 10] = g.opacity
            sh = list(g.sh_coeffs)[:48]
            out[i, 11:11 + len(sh)] = sh
        return out

    # ---- generators (reference cloud.py:67-140) --------------------------------------
    @classmethod
    def synthetic_cube(cls, points_per_axis: int = 4, cube_size: float = 1.0) -> "GaussianCloud":
        """Lattice of points_per_axis^3 splats over a cube centred at the origin,
        coloured by position through the DC SH term."""
        n = points_per_axis
        step = cube_size / float(n - 1) if n > 1 else 0.0
        half = cube_size * 0.5
        s = step * 0.6 if step > 0 else 0.1
        cloud = cls()
        for xi in range(n):
            for yi in range(n):
                for zi in range(n):
                    p = (-half + xi * step, -half + yi * step, -half + zi * step)
                    norm = [(c + half) / cube_size if cube_size > 0 else 0.5 for c in p]
                    sh = [0.0] * 48
                    sh[0:3] = [(v - 0.5) / SH_C0 for v in norm]
                    cloud.add(Gaussian3D(p, (s, s, s), (1.0, 0.0, 0.0, 0.0), 0.85, sh))
        return cloud

    @classmethod
    def synthetic_sphere(cls, point_count: int = 128, radius: float = 1.0) -> "GaussianCloud":
        """Fibonacci-sphere distribution of point_count splats."""
        golden = 1.6180339887
        s = radius * 0.12
        cloud = cls()
        for i in range(point_count):
            theta = 2.0 * math.pi * i / golden
            phi = math.acos(1.0 - 2.0 * (i + 0.5) / point_count)
            p = (radius * math.sin(phi) * math.cos(theta), radius * math.sin(phi) * math.sin(theta),
                 radius * math.cos(phi))
            sh = [0.0] * 48
            sh[0:3] = [((0.5 + 0.5 * c / radius) - 0.5) / SH_C0 for c in p]
            cloud.add(Gaussian3D(p, (s, s, s), (1.0, 0.0, 0.0, 0.0), 0.90, sh))
        return cloud

    # ---- ASCII PLY, the reference SDK's column order (cloud.py:131-199) ---------------
    _COLUMNS = ("x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3", "opacity",
                "f_dc_0", "f_dc_1", "f_dc_2")

    def save_ply(self, filepath: str) -> None:
        a = self.to_aos()
        cols = np.concatenate([a[:, 0:11], a[:, 11:14]], axis=1)
        with open(filepath, "w", encoding="utf-8") as f:
            f.write("ply\nformat ascii 1.0\n")
            f.write(f"element vertex {a.shape[0]}\n")
            for c in self._COLUMNS:
                f.write(f"property float {c}\n")
            f.write("end_header\n")
            for r in cols:
                f.write(" ".join(f"{float(v):.6f}" for v in r) + "\n")

    @classmethod
    def load_ply(cls, filepath: str) -> "GaussianCloud":
        cloud = cls()
        with open(filepath, "r", encoding="utf-8") as f:
            for line in f:
                if line.strip() == "end_header":
                    break
            for line in f:
                parts = line.split()
                if len(parts) < 14:
                    continue
                v = [float(x) for x in parts[:14]]
                sh = [0.0] * 48
                sh[0:3] = v[11:14]
                cloud.add(Gaussian3D(tuple(v[0:3]), tuple(v[3:6]), tuple(v[6:10]), v[10], sh))
        return cloud
