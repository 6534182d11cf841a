"""Image export helpers of the SDK (reference python/lumen/visualizer.py):
binary PPM, a false-colour depth PPM and an ASCII alpha preview."""
from __future__ import annotations

from typing import Sequence

import numpy as np


def export_ppm(filepath: str, width: int, height: int, rgb_bytes: bytes) -> None:
    """Binary PPM (P6) of an HWC uint8 buffer."""
    with open(filepath, "wb") as f:
        f.write(f"P6\n{width} {height}\n255\n".encode("ascii"))
        f.write(bytes(rgb_bytes))


def export_depth_visualization(filepath: str, width: int, height: int, depth_values: Sequence[float],
                               near_plane: float = 0.5, far_plane: float = 10.0) -> None:
    """Depth as a PPM: near is bright, far dark; depths >= 999 or <= 0 count as
    background (reference visualizer.py:16-48). A depth buffer already on the
    GPU (a CUDA tensor) is coloured there by lumen_gpu_depth_products and only
    the bytes come back."""
    if getattr(depth_values, "is_cuda", False):
        from . import depth as D
        rgb = D.heatmap(depth_values.reshape(height, width), near_plane, far_plane)
        export_ppm(filepath, width, height, rgb.cpu().numpy().tobytes())
        return
    if far_plane == near_plane:
        raise ZeroDivisionError("far_plane equals near_plane")
    d = np.asarray(depth_values, dtype=np.float64)[: width * height]
    with np.errstate(invalid="ignore"):
        norm = np.clip((d - near_plane) / (far_plane - near_plane), 0.0, 1.0)
    norm = np.where(np.isnan(norm), 1.0, norm)           # min(1.0, nan) is 1.0 in Python
    norm = np.where((d >= 999.0) | (d <= 0.0), 1.0, norm)
    inten = ((1.0 - norm) * 255.0).astype(np.int64)
    rgb = np.stack([inten, (inten * 0.8).astype(np.int64), (255 - inten * 0.7).astype(np.int64)], axis=1)
    export_ppm(filepath, width, height, np.clip(rgb, 0, 255).astype(np.uint8).tobytes())


def ascii_render(width: int, height: int, alpha_values: Sequence[float], target_width: int = 60,
                 target_height: int = 25) -> str:
    """Coarse ASCII preview of the alpha buffer."""
    chars = " .:-=+*#%@"
    levels = len(chars) - 1
    a = np.asarray(alpha_values, dtype=np.float64)
    lines = []
    for y in range(target_height):
        oy = min(int(y * height / target_height), height - 1)
        row = []
        for x in range(target_width):
            ox = min(int(x * width / target_width), width - 1)
            v = max(0.0, min(1.0, float(a[oy * width + ox])))
            row.append(chars[int(v * levels)])
        lines.append("".join(row))
    return "\n".join(lines)
