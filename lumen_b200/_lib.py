"""ctypes binding of liblumen.so (include/lumen.h and include/lumen_gpu.h).

The library is built in-tree by ``lumen_b200.build`` and loaded from
lumen_b200/liblumen.so. There is no fallback: if the library is missing or
no CUDA device is usable, the calls raise ``LumenError``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblumen.so")

LUMEN_SUCCESS = 0
STATUS_NAMES = {0: "SUCCESS", -1: "INVALID_ARGUMENT", -2: "OUT_OF_MEMORY", -3: "UNINITIALIZED",
                -4: "IO_FAILURE", -5: "MATH_SINGULAR"}

ERR_CAPACITY = 1
ERR_SPIN_TIMEOUT = 2
ERR_LAUNCH = 4
ERR_BOUNDS = 8


class LumenError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"liblumen {what}: {STATUS_NAMES.get(status, status)}")


_P = C.c_void_p


# ---- lumen.h -----------------------------------------------------------------
class LumenConfig(C.Structure):
    _fields_ = [("image_width", C.c_uint32), ("image_height", C.c_uint32), ("tile_size", C.c_uint32),
                ("near_plane", C.c_float), ("far_plane", C.c_float), ("early_termination_alpha", C.c_float),
                ("gaussian_radius_sigma", C.c_float)]


class LumenVec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class LumenQuat(C.Structure):
    _fields_ = [("w", C.c_float), ("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class LumenCamera(C.Structure):
    _fields_ = [("position", LumenVec3), ("target", LumenVec3), ("up", LumenVec3),
                ("fov_x_degrees", C.c_float), ("fov_y_degrees", C.c_float),
                ("near_plane", C.c_float), ("far_plane", C.c_float)]


class LumenGaussian(C.Structure):
    _fields_ = [("position", LumenVec3), ("scale", LumenVec3), ("rotation", LumenQuat),
                ("opacity", C.c_float), ("sh_coeffs", C.c_float * 48)]


class LumenFrameBuffer(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("rgb_data", C.POINTER(C.c_uint8)),
                ("depth_data", C.POINTER(C.c_float)), ("alpha_data", C.POINTER(C.c_float))]


class LumenStats(C.Structure):
    _fields_ = [("total_splats", C.c_size_t), ("visible_splats", C.c_size_t), ("culled_splats", C.c_size_t),
                ("total_tiles", C.c_size_t), ("touched_tiles", C.c_size_t),
                ("rasterize_time_ms", C.c_float), ("frames_per_second", C.c_float)]


# ---- lumen_gpu.h -------------------------------------------------------------
class LumenGpuGaussians(C.Structure):
    _fields_ = [("means", _P), ("scales", _P), ("quats", _P), ("opacities", _P), ("sh", _P),
                ("count", C.c_int64)]


class LumenViewCamera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("rotation", C.c_float * 4),
                ("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("near_plane", C.c_float), ("far_plane", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32)]


class LumenRenderOptions(C.Structure):
    _fields_ = [("lowpass", C.c_float), ("sh_degree", C.c_int32), ("white_background", C.c_int32),
                ("compute_depth", C.c_int32), ("key_mode", C.c_int32), ("term_mode", C.c_int32),
                ("params_are_logits", C.c_int32), ("tile_size", C.c_int32), ("term_threshold", C.c_float)]


class LumenGpuFrame(C.Structure):
    _fields_ = [("records", _P), ("visible_ids", _P), ("radii", _P), ("rects", _P), ("depth_keys", _P * 2),
                ("depth_order", _P * 2), ("keys", _P * 2), ("vals", _P * 2), ("instance_capacity", C.c_int64),
                ("ranges", _P), ("scratch", _P), ("scratch_bytes", C.c_size_t)]


class LumenGpuImage(C.Structure):
    _fields_ = [("rgb", _P), ("depth", _P), ("alpha", _P), ("n_contrib", _P), ("last_idx", _P), ("rgb8", _P)]


class LumenGpuLaunch(C.Structure):
    _fields_ = [("composite_chunk", C.c_int32), ("depth_sort_items", C.c_int32), ("tile_sort_items", C.c_int32)]


class LumenGpuBatchView(C.Structure):
    _fields_ = [("gaussians", LumenGpuGaussians), ("camera", LumenViewCamera), ("reserved", C.c_int32),
                ("image", LumenGpuImage)]


class LumenGpuCounts(C.Structure):
    _fields_ = [("n_visible", C.c_int64), ("n_instances", C.c_int64), ("error_flags", C.c_uint32),
                ("sorted_buffer", C.c_uint32), ("varying_digits", C.c_uint32), ("touched_tiles", C.c_uint32),
                ("depth_sorted_buffer", C.c_uint32), ("reserved", C.c_uint32)]


class LumenGpuGradients(C.Structure):
    _fields_ = [("means", _P), ("scales", _P), ("quats", _P), ("opacities", _P), ("sh", _P), ("splat2d", _P)]


# ---- lumen_serve.h ------------------------------------------------------------
class LumenServerConfig(C.Structure):
    _fields_ = [("work_budget_bytes", C.c_int64), ("max_views_per_batch", C.c_int32),
                ("max_batches_in_flight", C.c_int32), ("use_graphs", C.c_int32), ("autotune", C.c_int32),
                ("composite_chunk", C.c_int32), ("sort_items", C.c_int32), ("options", LumenRenderOptions)]


class LumenServeResult(C.Structure):
    _fields_ = [("request_id", C.c_uint64), ("status", C.c_int32), ("batch_views", C.c_int32),
                ("submit_ms", C.c_double), ("start_ms", C.c_double), ("done_ms", C.c_double),
                ("n_instances", C.c_int64), ("composite_chunk", C.c_int32), ("sort_items", C.c_int32)]


class LumenServeStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
                ("requeued_batches", C.c_uint64), ("rejected", C.c_uint64), ("graph_launches", C.c_uint64),
                ("device_ms", C.c_double), ("slot_bytes", C.c_int64), ("max_slots", C.c_int64),
                ("max_tiles", C.c_int64), ("max_instances", C.c_int64), ("max_pixels", C.c_int64),
                ("explored_batches", C.c_uint64)]


# ---- lumen_ply.h --------------------------------------------------------------
class LumenPlyInfo(C.Structure):
    _fields_ = [("count", C.c_int64), ("binary", C.c_int32), ("sh_degree", C.c_int32), ("log_values", C.c_int32),
                ("vertex_stride", C.c_int32), ("data_offset", C.c_int64)]


PLY_VALUES_AUTO, PLY_VALUES_LINEAR, PLY_VALUES_LOG = 0, 1, 2


class LumenTrainingConfig(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("position_lr_init", C.c_float), ("position_lr_final", C.c_float),
                ("feature_lr", C.c_float), ("opacity_lr", C.c_float), ("scaling_lr", C.c_float),
                ("rotation_lr", C.c_float), ("lambda_dssim", C.c_float), ("densify_from_iter", C.c_int32),
                ("densify_until_iter", C.c_int32), ("densification_interval", C.c_int32),
                ("opacity_reset_interval", C.c_int32), ("densify_grad_threshold", C.c_float),
                ("prune_opacity_threshold", C.c_float), ("max_screen_size_ratio", C.c_float)]


class LumenAdamState(C.Structure):
    _fields_ = [("m_pos", _P), ("v_pos", _P), ("m_opacity", _P), ("v_opacity", _P), ("step", C.c_int64)]


class LumenDepthProducts(C.Structure):
    _fields_ = [("normals", _P), ("range", _P), ("heatmap", _P), ("near_plane", C.c_double),
                ("far_plane", C.c_double)]


class LumenBvhNode(C.Structure):
    _fields_ = [("min_pt", C.c_float * 3), ("left_child", C.c_int32), ("max_pt", C.c_float * 3),
                ("right_child", C.c_int32)]


class LumenGpuBvh(C.Structure):
    _fields_ = [("nodes", _P), ("splat_index", _P), ("leaf_count", C.c_int64), ("node_count", C.c_int64),
                ("root_index", C.c_int64)]


class LumenRay(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("direction", C.c_float * 3)]


class LumenRayHit(C.Structure):
    _fields_ = [("hit", C.c_int32), ("splat_index", C.c_int32), ("distance", C.c_float), ("point", C.c_float * 3)]


class LumenDensifyStats(C.Structure):
    _fields_ = [("cloned", C.c_int64), ("split", C.c_int64), ("pruned", C.c_int64), ("count", C.c_int64)]

SPLAT_RECORD_BYTES = 48

# name -> (restype, argtypes); every symbol the two headers declare
SIGNATURES = {
    # lumen.h
    "lumen_get_version": (C.c_char_p, []),
    "lumen_get_version_major": (C.c_int, []),
    "lumen_get_version_minor": (C.c_int, []),
    "lumen_get_version_patch": (C.c_int, []),
    "lumen_default_config": (LumenConfig, []),
    "lumen_cloud_create": (_P, [C.c_size_t]),
    "lumen_cloud_destroy": (None, [_P]),
    "lumen_cloud_reserve": (C.c_int, [_P, C.c_size_t]),
    "lumen_cloud_get_count": (C.c_size_t, [_P]),
    "lumen_cloud_get_capacity": (C.c_size_t, [_P]),
    "lumen_cloud_add_gaussian": (C.c_int, [_P, C.POINTER(LumenGaussian)]),
    "lumen_cloud_get_gaussian": (C.c_int, [_P, C.c_size_t, C.POINTER(LumenGaussian)]),
    "lumen_cloud_clear": (None, [_P]),
    "lumen_create_synthetic_cube": (_P, [C.c_size_t, C.c_float]),
    "lumen_create_synthetic_sphere": (_P, [C.c_size_t, C.c_float]),
    "lumen_framebuffer_create": (C.POINTER(LumenFrameBuffer), [C.c_uint32, C.c_uint32]),
    "lumen_framebuffer_destroy": (None, [C.POINTER(LumenFrameBuffer)]),
    "lumen_framebuffer_clear": (None, [C.POINTER(LumenFrameBuffer), C.c_uint8, C.c_uint8, C.c_uint8]),
    "lumen_rasterizer_create": (_P, [C.POINTER(LumenConfig)]),
    "lumen_rasterizer_destroy": (None, [_P]),
    "lumen_rasterizer_set_config": (C.c_int, [_P, C.POINTER(LumenConfig)]),
    "lumen_rasterize": (C.c_int, [_P, _P, C.POINTER(LumenCamera), C.POINTER(LumenFrameBuffer),
                                  C.POINTER(LumenStats)]),
    # lumen_gpu.h
    "lumen_gpu_scratch_bytes": (C.c_size_t, [C.c_int64, C.c_int64, C.c_int64]),
    "lumen_gpu_render_forward": (C.c_int, [C.POINTER(LumenGpuGaussians), C.POINTER(LumenViewCamera),
                                           C.POINTER(LumenRenderOptions), C.POINTER(LumenGpuFrame),
                                           C.POINTER(LumenGpuImage), _P]),
    "lumen_gpu_read_counts": (C.c_int, [C.POINTER(LumenGpuFrame), C.POINTER(LumenGpuCounts), _P]),
    "lumen_gpu_renderer_create": (_P, []),
    "lumen_gpu_renderer_destroy": (None, [_P]),
    "lumen_gpu_renderer_render": (C.c_int, [_P, C.POINTER(LumenGpuGaussians), C.POINTER(LumenViewCamera),
                                            C.POINTER(LumenRenderOptions), C.POINTER(LumenGpuImage),
                                            C.POINTER(LumenGpuCounts), _P]),
    "lumen_gpu_renderer_frame": (C.POINTER(LumenGpuFrame), [_P]),
    "lumen_gpu_frame_sorted_keys64": (C.c_int, [C.POINTER(LumenGpuFrame), C.POINTER(LumenRenderOptions), _P, _P]),
    "lumen_gpu_sort_pairs": (C.c_int, [_P, _P, _P, _P, C.c_int64, _P, C.c_size_t, C.POINTER(C.c_uint32), _P]),
    "lumen_cloud_append": (C.c_int, [_P, C.POINTER(LumenGaussian), C.c_size_t]),
    "lumen_gpu_sort_pairs_noalloc": (C.c_int, [_P, _P, C.c_int64, _P]),
    "lumen_gpu_render_backward": (C.c_int, [C.POINTER(LumenGpuGaussians), C.POINTER(LumenViewCamera),
                                            C.POINTER(LumenRenderOptions), C.POINTER(LumenGpuFrame),
                                            C.POINTER(LumenGpuImage), _P, _P, _P, C.POINTER(LumenGpuGradients),
                                            _P]),
    "lumen_gpu_render_backward_timed": (C.c_int, [C.POINTER(LumenGpuGaussians), C.POINTER(LumenViewCamera),
                                                  C.POINTER(LumenRenderOptions), C.POINTER(LumenGpuFrame),
                                                  C.POINTER(LumenGpuImage), _P, _P, _P,
                                                  C.POINTER(LumenGpuGradients), _P, _P]),
    "lumen_gpu_l1_loss_scratch_bytes": (C.c_size_t, []),
    "lumen_gpu_l1_loss": (C.c_int, [_P, _P, C.c_int64, _P, _P, _P, _P]),
    "lumen_gpu_camera_from_lookat": (C.c_int, [C.POINTER(LumenCamera), C.c_uint32, C.c_uint32, C.c_float,
                                               C.c_float, C.POINTER(LumenViewCamera)]),
    "lumen_gpu_stage_timer_create": (_P, [C.c_int]),
    "lumen_gpu_stage_timer_destroy": (None, [_P]),
    "lumen_gpu_render_forward_timed": (C.c_int, [C.POINTER(LumenGpuGaussians), C.POINTER(LumenViewCamera),
                                                 C.POINTER(LumenRenderOptions), C.POINTER(LumenGpuFrame),
                                                 C.POINTER(LumenGpuImage), _P, _P]),
    "lumen_gpu_render_forward_ex": (C.c_int, [C.POINTER(LumenGpuGaussians), C.POINTER(LumenViewCamera),
                                              C.POINTER(LumenRenderOptions), C.POINTER(LumenGpuLaunch),
                                              C.POINTER(LumenGpuFrame), C.POINTER(LumenGpuImage), _P, _P]),
    "lumen_gpu_batch_sizes": (C.c_int, [C.POINTER(LumenGpuBatchView), C.c_int32, C.POINTER(C.c_int64),
                                        C.POINTER(C.c_int64)]),
    "lumen_gpu_batch_scratch_bytes": (C.c_size_t, [C.c_int64, C.c_int64, C.c_int32]),
    "lumen_gpu_render_batch": (C.c_int, [C.POINTER(LumenGpuBatchView), C.c_int32, C.POINTER(LumenRenderOptions),
                                         C.POINTER(LumenGpuFrame), _P]),
    "lumen_gpu_render_batch_timed": (C.c_int, [C.POINTER(LumenGpuBatchView), C.c_int32,
                                               C.POINTER(LumenRenderOptions), C.POINTER(LumenGpuFrame), _P, _P]),
    # lumen_ply.h
    "lumen_ply_info": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(LumenPlyInfo)]),
    "lumen_ply_load_host": (C.c_int, [C.c_char_p, C.c_int32, _P, _P, _P, _P, _P, C.c_int64,
                                      C.POINTER(LumenPlyInfo)]),
    "lumen_ply_load_device": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(LumenGpuGaussians),
                                        C.POINTER(LumenPlyInfo), _P]),
    # lumen_serve.h
    "lumen_server_default_config": (LumenServerConfig, []),
    "lumen_server_create": (_P, [C.POINTER(LumenServerConfig)]),
    "lumen_server_destroy": (None, [_P]),
    "lumen_server_add_scene": (C.c_int32, [_P, C.POINTER(LumenGpuGaussians)]),
    "lumen_server_submit": (C.c_int, [_P, C.c_int32, C.POINTER(LumenViewCamera), _P, C.POINTER(C.c_uint64)]),
    "lumen_server_wait": (C.c_int, [_P, C.c_uint64, C.c_double, C.POINTER(LumenServeResult)]),
    "lumen_server_stats": (C.c_int, [_P, C.POINTER(LumenServeStats)]),
    "lumen_server_freeze_tuning": (C.c_int, [_P, C.c_int32]),
    "lumen_serve_admit": (C.c_int32, [C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64), C.c_int32, C.c_int32, C.c_int64, C.c_int64,
                                      C.c_int64, C.c_int64]),
    # lumen_train.h
    "lumen_training_default_config": (LumenTrainingConfig, []),
    "lumen_training_should_densify": (C.c_int32, [C.POINTER(LumenTrainingConfig), C.c_int64]),
    "lumen_training_should_reset_opacity": (C.c_int32, [C.POINTER(LumenTrainingConfig), C.c_int64]),
    "lumen_gpu_adam_step": (C.c_int, [C.POINTER(LumenGpuGaussians), _P, _P, C.POINTER(LumenAdamState),
                                      C.POINTER(LumenTrainingConfig), _P]),
    "lumen_gpu_accumulate_viewspace": (C.c_int, [_P, C.c_int32, _P, C.c_int64, C.c_float, C.c_float, _P, _P, _P]),
    "lumen_gpu_densify_scratch_bytes": (C.c_size_t, [C.c_int64]),
    "lumen_gpu_densify_and_prune": (C.c_int, [C.POINTER(LumenGpuGaussians), _P, _P, C.POINTER(LumenTrainingConfig),
                                              C.c_float, C.POINTER(LumenGpuGaussians), C.POINTER(LumenAdamState),
                                              C.POINTER(LumenAdamState), _P, C.c_size_t,
                                              C.POINTER(LumenDensifyStats), _P]),
    "lumen_gpu_reset_opacities": (C.c_int, [_P, C.c_int64, C.c_float, _P]),
    "lumen_gpu_psnr": (C.c_int, [_P, _P, C.c_int64, _P, _P, _P]),
    # lumen_depth.h
    "lumen_gpu_depth_products": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(LumenDepthProducts), _P]),
    # lumen_spatial.h
    "lumen_bvh_node_count": (C.c_int64, [C.c_int64]),
    "lumen_gpu_bvh_scratch_bytes": (C.c_size_t, [C.c_int64]),
    "lumen_gpu_bvh_build": (C.c_int, [C.POINTER(LumenGpuGaussians), C.POINTER(LumenGpuBvh), _P, C.c_size_t, _P]),
    "lumen_gpu_raycast": (C.c_int, [C.POINTER(LumenGpuBvh), C.POINTER(LumenGpuGaussians), _P, C.c_int64, C.c_float,
                                    _P, _P]),
    "lumen_gpu_pick_pixels": (C.c_int, [C.POINTER(LumenGpuBvh), C.POINTER(LumenGpuGaussians),
                                        C.POINTER(LumenViewCamera), _P, C.c_int64, C.c_float, _P, _P, _P]),
    "lumen_gpu_stage_timer_read": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int)]),
}

_lib = None
_lock = threading.Lock()


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load liblumen.so (building it first when it is absent)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            if not build_if_missing:
                raise LumenError(-3, f"library not built ({LIB_PATH})")
            from . import build
            build.build()
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status: int, what: str) -> None:
    if status != LUMEN_SUCCESS:
        raise LumenError(status, what)


def view_camera(cam) -> LumenViewCamera:
    c = LumenViewCamera()
    c.position[:] = [float(v) for v in cam.position]
    c.rotation[:] = [float(v) for v in cam.rotation]
    c.fx, c.fy, c.cx, c.cy = float(cam.fx), float(cam.fy), float(cam.cx), float(cam.cy)
    c.near_plane, c.far_plane = float(cam.near_plane), float(cam.far_plane)
    c.width, c.height = int(cam.width), int(cam.height)
    return c


def render_options(opt) -> LumenRenderOptions:
    o = LumenRenderOptions()
    o.lowpass = float(opt.lowpass)
    o.sh_degree = int(opt.sh_degree)
    o.white_background = int(bool(opt.white_background))
    o.compute_depth = int(bool(opt.compute_depth))
    o.key_mode = int(opt.key_mode)
    o.term_mode = int(opt.term_mode)
    o.params_are_logits = int(bool(opt.params_are_logits))
    o.tile_size = int(opt.tile_size)
    o.term_threshold = float(opt.term_threshold)
    return o
