"""Gaussian scenes from Stanford PLY files (include/lumen_ply.h).

``info(path)`` reads the header; ``load_host(path)`` returns numpy SoA
arrays; ``load(path, device)`` returns a device-resident ``render.Scene``
(binary vertex data de-interleaved by a kernel on the device). Columns are
found by property name, so the reference's two ASCII layouts
(src/scene/ply.mojo:32-70 and python/lumen/cloud.py:131-161) and the common
binary training layout (f_rest_* SH, log-scales, opacity logits) all load.
Render a loaded scene with ``RenderOptions(params_are_logits=info.log_values)``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Tuple

import numpy as np

from . import _lib as L

VALUES = {"auto": L.PLY_VALUES_AUTO, "linear": L.PLY_VALUES_LINEAR, "log": L.PLY_VALUES_LOG}


@dataclass
class PlyInfo:
    count: int
    binary: bool
    sh_degree: int
    log_values: bool
    vertex_stride: int
    data_offset: int


def _info(c: L.LumenPlyInfo) -> PlyInfo:
    return PlyInfo(int(c.count), bool(c.binary), int(c.sh_degree), bool(c.log_values), int(c.vertex_stride),
                   int(c.data_offset))


def info(path: str, values: str = "auto") -> PlyInfo:
    c = L.LumenPlyInfo()
    L.check(L.load().lumen_ply_info(str(path).encode(), VALUES[values], C.byref(c)), f"ply_info({path})")
    return _info(c)


def load_host(path: str, values: str = "auto") -> Tuple[dict, PlyInfo]:
    """SoA float32 arrays: means [N,3], scales [N,3], quats [N,4] (w,x,y,z),
    opacities [N], sh [N,48] (sh[k*3 + ch])."""
    n = info(path, values).count
    arrs = {"means": np.empty((n, 3), np.float32), "scales": np.empty((n, 3), np.float32),
            "quats": np.empty((n, 4), np.float32), "opacities": np.empty(n, np.float32),
            "sh": np.empty((n, 48), np.float32)}
    c = L.LumenPlyInfo()
    p = lambda a: a.ctypes.data if a.size else None
    L.check(L.load().lumen_ply_load_host(str(path).encode(), VALUES[values], p(arrs["means"]), p(arrs["scales"]),
                                         p(arrs["quats"]), p(arrs["opacities"]), p(arrs["sh"]), n, C.byref(c)),
            f"ply_load_host({path})")
    return arrs, _info(c)


def load(path: str, device="cuda", values: str = "auto"):
    """A device-resident render.Scene and the file's PlyInfo."""
    import torch
    from .render import Scene
    n = info(path, values).count
    dev = torch.device(device)
    t = lambda *shape: torch.empty(shape, dtype=torch.float32, device=dev)
    means, scales, quats, opac, sh = t(n, 3), t(n, 3), t(n, 4), t(n), t(n, 48)
    g = L.LumenGpuGaussians()
    g.means, g.scales, g.quats, g.opacities, g.sh = (x.data_ptr() for x in (means, scales, quats, opac, sh))
    g.count = n
    c = L.LumenPlyInfo()
    stream = torch.cuda.current_stream(dev).cuda_stream
    L.check(L.load().lumen_ply_load_device(str(path).encode(), VALUES[values], C.byref(g), C.byref(c), stream),
            f"ply_load_device({path})")
    return Scene(means, scales, quats, opac, sh), _info(c)


def write_binary(path: str, means, scales, quats, opacities, sh, sh_degree: int = 3, normals: bool = True) -> None:
    """Write the binary little-endian training layout: x y z [nx ny nz]
    f_dc_0..2 f_rest_* (channel-major) opacity scale_0..2 rot_0..3, the
    values as given (log-scales and logits by that layout's convention)."""
    n = int(np.asarray(means).shape[0])
    sh = np.asarray(sh, np.float32).reshape(n, 16, 3)
    m = (sh_degree + 1) ** 2 - 1
    cols = [np.asarray(means, np.float32)]
    names = ["x", "y", "z"]
    if normals:
        cols.append(np.zeros((n, 3), np.float32))
        names += ["nx", "ny", "nz"]
    cols.append(sh[:, 0, :])
    names += [f"f_dc_{i}" for i in range(3)]
    if m:
        cols.append(sh[:, 1:1 + m, :].transpose(0, 2, 1).reshape(n, 3 * m))
        names += [f"f_rest_{i}" for i in range(3 * m)]
    cols += [np.asarray(opacities, np.float32).reshape(n, 1), np.asarray(scales, np.float32),
             np.asarray(quats, np.float32)]
    names += ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    data = np.ascontiguousarray(np.concatenate(cols, axis=1), dtype="<f4")
    head = "ply\nformat binary_little_endian 1.0\nelement vertex %d\n" % n
    head += "".join(f"property float {nm}\n" for nm in names) + "end_header\n"
    with open(path, "wb") as f:
        f.write(head.encode("ascii"))
        f.write(data.tobytes())
