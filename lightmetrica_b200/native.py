"""ctypes binding of the C ABI declared in include/lmgpu.h.

The product path always goes through the native library
(lightmetrica_b200/_lib/liblmgpu.so unless LMGPU_LIBRARY names another
build); there is no CPU fallback. Loading fails loudly if it is missing.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# The in-tree build; LMGPU_LIBRARY names another build of the same sources
# (the bounds-checked CHECK_LIB_PATH, or one compiled with different tuning
# constants).
LIB_PATH = os.environ.get("LMGPU_LIBRARY") or os.path.join(HERE, "_lib", "liblmgpu.so")
CHECK_LIB_PATH = os.path.join(HERE, "_lib", "liblmgpu_check.so")

c_int32 = ctypes.c_int32
c_int64 = ctypes.c_int64
c_float = ctypes.c_float
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
c_uint64 = ctypes.c_uint64
P = ctypes.POINTER

# ---- status codes
OK = 0
ERR_INVALID = -1
ERR_OOM = -2
ERR_CUDA = -3
ERR_STACK_OVERFLOW = -4
ERR_QUEUE_OVERFLOW = -5
ERR_TIMEOUT = -6
ERR_UNSUPPORTED = -7
ERR_BOUNDS = -8
STATUS_NAMES = {OK: "OK", ERR_INVALID: "INVALID", ERR_OOM: "OOM", ERR_CUDA: "CUDA",
                ERR_STACK_OVERFLOW: "STACK_OVERFLOW", ERR_QUEUE_OVERFLOW: "QUEUE_OVERFLOW",
                ERR_TIMEOUT: "TIMEOUT", ERR_UNSUPPORTED: "UNSUPPORTED", ERR_BOUNDS: "BOUNDS"}

LAYOUT_BVH2, LAYOUT_BVH4, LAYOUT_NAIVE, LAYOUT_BVH2Q, LAYOUT_BVH2_QSHADOW = 0, 1, 2, 3, 4
RENDER_TREE_SAH, RENDER_TREE_REFERENCE = 0, 1
BSDF_DIFFUSE, BSDF_MIRROR, BSDF_DIFFUSE_MIRROR, BSDF_BLACK = 0, 1, 2, 3
RENDER_PT, RENDER_PT_DIRECT, RENDER_PT_MIS = 0, 1, 2
SAMPLING_STRATIFIED, SAMPLING_UNIFORM = 0, 1


class PrimitiveDesc(ctypes.Structure):
    _fields_ = [("positions", P(c_float)), ("normals", P(c_float)), ("texcoords", P(c_float)),
                ("faces", P(ctypes.c_uint32)), ("num_vertices", c_int32), ("num_faces", c_int32),
                ("transform", P(c_float)), ("material", c_int32), ("area_light", c_int32)]


class MaterialDesc(ctypes.Structure):
    _fields_ = [("type", c_int32), ("reflectance", c_float * 3)]


class AreaLightDesc(ctypes.Structure):
    _fields_ = [("luminance", c_float * 3)]


class SceneDesc(ctypes.Structure):
    _fields_ = [("primitives", P(PrimitiveDesc)), ("num_primitives", c_int32),
                ("materials", P(MaterialDesc)), ("num_materials", c_int32),
                ("area_lights", P(AreaLightDesc)), ("num_area_lights", c_int32),
                ("has_env_light", c_int32), ("env_luminance", c_float * 3),
                ("has_camera", c_int32), ("camera_eye", c_float * 3), ("camera_center", c_float * 3),
                ("camera_up", c_float * 3), ("camera_fovy_degrees", c_float),
                ("film_width", c_int32), ("film_height", c_int32),
                ("layout", c_int32), ("build_threads", c_int32), ("max_stack_entries", c_int32),
                ("render_tree", c_int32)]


class SceneInfo(ctypes.Structure):
    _fields_ = [("num_triangles", c_int64), ("num_nodes", c_int64), ("num_leaves", c_int64),
                ("max_depth", c_int32), ("layout", c_int32), ("device_bytes", c_int64),
                ("build_seconds", c_double), ("bounds_min", c_float * 3), ("bounds_max", c_float * 3),
                ("render_tree", c_int32), ("render_max_depth", c_int32), ("render_num_nodes", c_int64),
                ("render_num_leaves", c_int64), ("render_build_seconds", c_double)]


class RaysSoA(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("ox", "oy", "oz", "dx", "dy", "dz", "tmin", "tmax")]


class HitsSoA(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("tri_id", "t", "u", "v")]


class RenderParams(ctypes.Structure):
    _fields_ = [("technique", c_int32), ("rr_depth", c_int32), ("max_path_vertices", c_int32),
                ("sampling", c_int32), ("seed", c_uint64), ("num_samples", c_int64),
                ("sample_offset", c_int64), ("film_fp64", c_int32), ("wave_paths", c_int32)]


class DiffParams(ctypes.Structure):
    _fields_ = [("albedo", c_void_p), ("emission", c_void_p)]


class RenderStats(ctypes.Structure):
    _fields_ = [("rays_traced", c_int64), ("shadow_rays", c_int64), ("paths", c_int64),
                ("waves", c_int32), ("max_bounces_run", c_int32), ("device_ms", c_double)]


BATCH_WAVES, BATCH_STREAM, BATCH_OVERLAP = 0, 1, 2
EVAL_CONCENTRIC_DISK, EVAL_COSINE_HEMISPHERE = 0, 1


class BatchConfig(ctypes.Structure):
    _fields_ = [("layout", c_int32), ("wave_paths", c_int32), ("shade_blocks_per_sm", c_int32),
                ("use_graph", c_int32), ("mode", c_int32), ("overlap_bounce", c_int32)]


class TraceProfile(ctypes.Structure):
    _fields_ = [("rays", c_int64 * 2), ("launches", c_int64 * 2), ("trace_ms", c_double * 2),
                ("render_ms", c_double), ("node_tests", c_uint64 * 2), ("tri_tests", c_uint64 * 2)]


# Every symbol include/lmgpu.h declares, with (restype, argtypes).
SIGNATURES = {
    "lmgpu_abi_version": (c_int32, []),
    "lmgpu_last_error": (ctypes.c_char_p, []),
    "lmgpu_scene_create": (c_int32, [P(SceneDesc), P(c_void_p)]),
    "lmgpu_scene_destroy": (c_int32, [c_void_p]),
    "lmgpu_scene_info": (c_int32, [c_void_p, P(SceneInfo)]),
    "lmgpu_scene_build_host": (c_int32, [P(SceneDesc), P(SceneInfo), c_void_p, c_int64]),
    "lmgpu_intersect": (c_int32, [c_void_p, P(RaysSoA), c_int64, P(HitsSoA), c_void_p]),
    "lmgpu_intersect_host": (c_int32, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "lmgpu_occluded": (c_int32, [c_void_p, P(RaysSoA), c_int64, c_void_p, c_void_p]),
    "lmgpu_intersect_full_host": (c_int32, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "lmgpu_render": (c_int32, [c_void_p, P(RenderParams), c_void_p, P(RenderStats)]),
    "lmgpu_render_device": (c_int32, [c_void_p, P(RenderParams), c_void_p, c_void_p, P(RenderStats)]),
    "lmgpu_render_device_noalloc": (c_int32, [c_void_p, P(RenderParams), c_void_p, c_void_p]),
    "lmgpu_render_release": (c_int32, []),
    "lmgpu_scene_status": (c_int32, [c_void_p, c_void_p]),
    "lmgpu_adjoint_forward": (c_int32, [c_void_p, P(RenderParams), P(DiffParams), c_void_p, c_void_p, P(RenderStats)]),
    "lmgpu_adjoint_backward": (c_int32, [c_void_p, P(RenderParams), P(DiffParams), c_void_p, c_void_p, c_void_p,
                                         c_void_p, P(RenderStats)]),
    "lmgpu_intersect_counted": (c_int32, [c_void_p, P(RaysSoA), c_int64, P(HitsSoA), c_void_p, c_void_p]),
    "lmgpu_batch_create": (c_int32, [P(c_void_p), c_int32, P(c_void_p)]),
    "lmgpu_batch_destroy": (c_int32, [c_void_p]),
    "lmgpu_batch_get_config": (c_int32, [c_void_p, P(BatchConfig)]),
    "lmgpu_batch_set_config": (c_int32, [c_void_p, P(BatchConfig)]),
    "lmgpu_batch_render_device": (c_int32, [c_void_p, P(RenderParams), P(c_void_p), c_void_p, P(RenderStats)]),
    "lmgpu_batch_autotune": (c_int32, [c_void_p, P(RenderParams), c_double, c_void_p, P(BatchConfig),
                                       P(c_double)]),
    "lmgpu_batch_render": (c_int32, [c_void_p, P(RenderParams), P(c_void_p), P(RenderStats)]),
    "lmgpu_batch_profile": (c_int32, [c_void_p, P(RenderParams), P(c_void_p), c_void_p, c_int32, P(TraceProfile)]),
    "lmgpu_eval_sampling": (c_int32, [c_int32, c_void_p, c_int64, c_void_p]),
    "lmgpu_camera_sample_rays": (c_int32, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    "lmgpu_camera_raster_positions": (c_int32, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    "lmgpu_film_pixels": (c_int32, [c_void_p, c_void_p, c_int64, c_void_p]),
    "lmgpu_light_sample": (c_int32, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    "lmgpu_bsdf_sample": (c_int32, [c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p,
                                    c_void_p, c_void_p]),
    "lmgpu_bsdf_evaluate": (c_int32, [c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
}

_lib = None


class LmgpuError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"lmgpu {STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def lib():
    """Loads liblmgpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m lightmetrica_b200.build` "
                              "(the CUDA core has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != OK:
        msg = lib().lmgpu_last_error()
        raise LmgpuError(code, msg.decode() if msg else "")
