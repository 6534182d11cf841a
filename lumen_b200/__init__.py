"""lumen_b200: Lumen's forward Gaussian-splatting path and its adjoint on B200.

The names exported here mirror the reference Python SDK (python/lumen/
__init__.py), so ``import lumen_b200 as lumen`` is a drop-in: Camera,
CameraTrajectory, GaussianCloud, Gaussian3D, LumenEngine, RasterizerConfig,
RenderResult, export_ppm, export_depth_visualization, ascii_render.
Rendering runs in liblumen.so (hand-written sm_100a CUDA behind a C ABI).

Device-resident entry points: ``lumen_b200.render`` (forward with every
stage exposed), ``lumen_b200.autograd`` (torch.autograd.Function with the
hand-written backward), ``lumen_b200.serve`` (render server).
"""
from .camera import Camera, CameraTrajectory
from .client import LumenEngine, RasterizerConfig, RenderResult
from .cloud import Gaussian3D, GaussianCloud
from .types import RenderOptions, ViewCamera
from .visualizer import ascii_render, export_depth_visualization, export_ppm

__version__ = "0.1.0"
__all__ = [
    "Camera", "CameraTrajectory", "GaussianCloud", "Gaussian3D", "LumenEngine", "RasterizerConfig",
    "RenderResult", "export_ppm", "export_depth_visualization", "ascii_render", "RenderOptions", "ViewCamera",
]
