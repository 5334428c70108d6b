"""ctypes mirror of ``include/rkf_cuda.h`` and the loader of the CUDA library.

The library is built in-tree (``rkifield_b200/_lib/librkf_cuda.so``) by
``rkifield_b200/build.py``.  Loading fails loudly when it is missing: there
is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "librkf_cuda.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "rkf_cuda.h")

RKF_OK, RKF_INVALID_ARG, RKF_OOM, RKF_CUDA_ERROR, RKF_TIMEOUT = 0, 1, 2, 3, 4
RKF_BUSY, RKF_EPOCH_STALE, RKF_NOT_READY, RKF_UNSUPPORTED, RKF_CANCELLED = 5, 6, 7, 8, 9
STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA_ERROR", 4: "TIMEOUT", 5: "BUSY",
    6: "EPOCH_STALE", 7: "NOT_READY", 8: "UNSUPPORTED", 9: "CANCELLED",
}

EMPTY_SLOT = 0xFFFFFFFF
INTERIOR_SLOT = 0xFFFFFFFE
MAX_FLOAT = np.float32(3.402823e38)

RKF_SDF_NONE, RKF_SDF_ANALYTICAL, RKF_SDF_VOXELIZED = 0, 1, 2
RKF_PRIM_SPHERE, RKF_PRIM_BOX, RKF_PRIM_CAPSULE, RKF_PRIM_TORUS, RKF_PRIM_CYLINDER, RKF_PRIM_PLANE = range(6)
RKF_NO_PARENT = 0xFFFFFFFF
RKF_BLEND_SMOOTH_UNION, RKF_BLEND_UNION, RKF_BLEND_SUBTRACT, RKF_BLEND_INTERSECT = 0, 1, 2, 3
RKF_PRECISION_F16, RKF_PRECISION_F32, RKF_PRECISION_U8 = 0, 1, 2
RKF_MEM_HOST, RKF_MEM_DEVICE = 0, 1
RKF_BAND_VOXELS, RKF_BAND_REFERENCE = 0, 1
RKF_TRACE_CLOSEST, RKF_TRACE_ANY, RKF_TRACE_SHADOW = 0, 1, 2
RKF_FLAG_HIT, RKF_FLAG_BISECTED, RKF_FLAG_STEPS_OUT = 1, 2, 4
RKF_REQ_RENDER, RKF_REQ_RAYS, RKF_REQ_POINTS, RKF_REQ_EDIT = 0, 1, 2, 3
RKF_STRATEGY_BRUTE, RKF_STRATEGY_TILED, RKF_STRATEGY_BVH = 0, 1, 2
BVH_INVALID = 0xFFFFFFFF


class rkf_camera(C.Structure):
    _fields_ = [("position", C.c_float * 4), ("forward", C.c_float * 4),
                ("right", C.c_float * 4), ("up", C.c_float * 4),
                ("resolution", C.c_float * 2), ("jitter", C.c_float * 2),
                ("prev_vp", C.c_float * 16)]


class rkf_scene_uniforms(C.Structure):
    _fields_ = [("num_objects", C.c_uint32), ("max_steps", C.c_uint32),
                ("max_distance", C.c_float), ("hit_threshold", C.c_float)]


class rkf_gpu_object(C.Structure):
    _fields_ = [("inverse_world", C.c_float * 16), ("aabb_min", C.c_float * 4),
                ("aabb_max", C.c_float * 4), ("brick_map_offset", C.c_uint32),
                ("brick_map_dims", C.c_uint32 * 3), ("voxel_size", C.c_float),
                ("material_id", C.c_uint32), ("sdf_type", C.c_uint32),
                ("blend_mode", C.c_uint32), ("blend_radius", C.c_float),
                ("sdf_params", C.c_float * 4), ("accumulated_scale", C.c_float * 3),
                ("lod_level", C.c_uint32), ("object_id", C.c_uint32),
                ("primitive_type", C.c_uint32), ("geometry_aabb_min", C.c_float * 3),
                ("geometry_aabb_max", C.c_float * 3), ("_padding", C.c_float * 15)]


class rkf_march_params(C.Structure):
    _fields_ = [("scene", rkf_scene_uniforms), ("hard_max_steps", C.c_uint32),
                ("bisect_steps", C.c_uint32), ("min_step", C.c_float),
                ("near_surface_threshold", C.c_float), ("strategy", C.c_uint32),
                ("reserved", C.c_uint32)]


class rkf_config(C.Structure):
    _fields_ = [("device", C.c_int), ("pool_capacity_bricks", C.c_uint32),
                ("precision", C.c_uint32), ("keep_reference_pool", C.c_uint32),
                ("mem_budget_bytes", C.c_uint64), ("max_inflight", C.c_uint32),
                ("u8_band", C.c_float), ("u8_round", C.c_uint32), ("reserved", C.c_uint32 * 5)]


class rkf_scene_node(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("rotation", C.c_float * 4), ("scale", C.c_float * 3),
                ("parent", C.c_uint32), ("visible", C.c_uint32), ("sdf_type", C.c_uint32),
                ("primitive_type", C.c_uint32), ("params", C.c_float * 4), ("material_id", C.c_uint32),
                ("brick_map_offset", C.c_uint32), ("brick_map_dims", C.c_uint32 * 3),
                ("voxel_size", C.c_float), ("blend_mode", C.c_uint32), ("blend_radius", C.c_float)]


class rkf_flat_node(C.Structure):
    _fields_ = [("inverse_world", C.c_float * 16), ("accumulated_scale", C.c_float * 3),
                ("depth", C.c_uint32), ("parent_index", C.c_uint32), ("node", C.c_uint32)]


class rkf_bvh_node(C.Structure):
    """GpuBvhNode (gpu_bvh.rs:24-41): 32 bytes."""
    _fields_ = [("aabb_min", C.c_float * 3), ("left", C.c_uint32),
                ("aabb_max", C.c_float * 3), ("right_or_object", C.c_uint32)]


class rkf_bvh_item(C.Structure):
    _fields_ = [("object_index", C.c_uint32), ("aabb_min", C.c_float * 3), ("aabb_max", C.c_float * 3)]


class rkf_scene_info(C.Structure):
    _fields_ = [("num_objects", C.c_uint32), ("pool_bricks_used", C.c_uint32),
                ("pool_capacity", C.c_uint32), ("leaf_blocks", C.c_uint32),
                ("device_bytes", C.c_uint64), ("epoch", C.c_uint64)]


class rkf_prim(C.Structure):
    _fields_ = [("type", C.c_uint32), ("material", C.c_uint32), ("centre", C.c_float * 3),
                ("params", C.c_float * 3), ("rot", C.c_float * 9), ("bound_radius", C.c_float)]


PRIM_DTYPE = np.dtype([("type", "<u4"), ("material", "<u4"), ("centre", "<f4", 3),
                       ("params", "<f4", 3), ("rot", "<f4", 9), ("bound_radius", "<f4")])
assert PRIM_DTYPE.itemsize == C.sizeof(rkf_prim)


class rkf_voxelize_params(C.Structure):
    _fields_ = [("voxel_size", C.c_float), ("smooth_k", C.c_float),
                ("band_voxels", C.c_float), ("cut_distance", C.c_float),
                ("aabb_min", C.c_float * 3), ("aabb_max", C.c_float * 3),
                ("band_rule", C.c_uint32), ("object_id", C.c_uint32)]


class rkf_gbuffer(C.Structure):
    _fields_ = [("t", C.c_void_p), ("normal", C.c_void_p), ("slot", C.c_void_p),
                ("material", C.c_void_p), ("flags", C.c_void_p), ("position", C.c_void_p),
                ("packed_material", C.c_void_p), ("motion", C.c_void_p),
                ("mem", C.c_uint32), ("_pad", C.c_uint32)]


class rkf_hits(C.Structure):
    _fields_ = [("t", C.c_void_p), ("normal", C.c_void_p), ("slot", C.c_void_p),
                ("material", C.c_void_p), ("flags", C.c_void_p),
                ("mem", C.c_uint32), ("_pad", C.c_uint32)]


class rkf_edit_op(C.Structure):
    _fields_ = [("object_index", C.c_uint32), ("edit_type", C.c_uint32),
                ("shape_type", C.c_uint32), ("falloff", C.c_uint32),
                ("position", C.c_float * 3), ("rotation", C.c_float * 4),
                ("dimensions", C.c_float * 3), ("strength", C.c_float),
                ("blend_k", C.c_float), ("material_id", C.c_uint32),
                ("_pad", C.c_uint32 * 2)]


class rkf_view(C.Structure):
    _fields_ = [("camera", rkf_camera), ("width", C.c_uint32), ("height", C.c_uint32),
                ("out", rkf_gbuffer)]


class rkf_ray_batch(C.Structure):
    _fields_ = [("origins", C.c_void_p), ("dirs", C.c_void_p), ("tmax", C.c_void_p),
                ("n", C.c_uint32), ("mode", C.c_uint32), ("out", rkf_hits)]


class rkf_batch_tuning(C.Structure):
    _fields_ = [("tile_w", C.c_uint32), ("tile_h", C.c_uint32), ("step_budget", C.c_uint32),
                ("compact_interval", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("threads_per_block", C.c_uint32), ("refill_idle", C.c_uint32),
                ("probe_in_run", C.c_uint32), ("no_empty_path", C.c_uint32),
                ("order_tiles", C.c_uint32), ("tail_share", C.c_uint32)]


class rkf_request(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("mode", C.c_uint32), ("width", C.c_uint32),
                ("height", C.c_uint32), ("n", C.c_uint32), ("_pad", C.c_uint32),
                ("camera", rkf_camera), ("in0", C.c_void_p), ("in1", C.c_void_p),
                ("in2", C.c_void_p), ("edit", rkf_edit_op), ("out_t", C.c_void_p),
                ("out_normal", C.c_void_p), ("out_slot", C.c_void_p),
                ("out_material", C.c_void_p), ("out_flags", C.c_void_p)]


class rkf_result(C.Structure):
    _fields_ = [("status", C.c_int), ("kind", C.c_uint32), ("epoch", C.c_uint64),
                ("submit_us", C.c_double), ("start_us", C.c_double),
                ("done_us", C.c_double), ("device_ms", C.c_double)]


class rkf_world_pos(C.Structure):
    _fields_ = [("chunk", C.c_int32 * 3), ("local", C.c_float * 3)]


SIZES = {"rkf_camera": 144, "rkf_scene_uniforms": 16, "rkf_gpu_object": 256}
assert C.sizeof(rkf_camera) == 144 and C.sizeof(rkf_scene_uniforms) == 16
assert C.sizeof(rkf_gpu_object) == 256


def march_params_default(p: rkf_march_params) -> None:
    """Reference defaults (gpu_scene.rs:34-43, ray_march.wgsl:28-41), set
    host-side so that building march parameters needs no library."""
    p.scene.num_objects = 0
    p.scene.max_steps = 128
    p.scene.max_distance = 100.0
    p.scene.hit_threshold = 0.001
    p.hard_max_steps = 1024
    p.bisect_steps = 8
    p.min_step = 0.0005
    p.near_surface_threshold = 0.02
    p.strategy = RKF_STRATEGY_BRUTE


# Every function the header declares, with its ctypes signature.
_P, _U32, _U64, _I, _F = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_float
SIGNATURES = {
    "rkf_march_params_default": (None, [C.POINTER(rkf_march_params)]),
    "rkf_config_default": (None, [C.POINTER(rkf_config)]),
    "rkf_create": (_I, [C.POINTER(rkf_config), C.POINTER(_P)]),
    "rkf_destroy": (_I, [_P]),
    "rkf_last_error": (C.c_char_p, []),
    "rkf_pool_import_voxelsample": (_I, [_P, _P, _U32, _U32]),
    "rkf_brickmap_import": (_I, [_P, _P, _U64]),
    "rkf_objects_import": (_I, [_P, _P, _U32]),
    "rkf_bvh_import": (_I, [_P, _P, _U32]),
    "rkf_objects_update": (_I, [_P, _P, _U32, _P]),
    "rkf_flatten_object": (_I, [_P, _U32, _P, _P, _P, _P, C.POINTER(C.c_uint32)]),
    "rkf_gpu_object_from_flat_node": (_I, [_P, _P, _U32, _P, _P, _P, _P, _P]),
    "rkf_batch_graph_create": (_I, [_P, C.POINTER(rkf_view), _U32, C.POINTER(rkf_ray_batch), _U32,
                                    C.POINTER(rkf_march_params), C.POINTER(rkf_batch_tuning), C.POINTER(_P)]),
    "rkf_batch_graph_set_cameras": (_I, [_P, C.POINTER(rkf_camera), _U32]),
    "rkf_batch_graph_launch": (_I, [_P, _P]),
    "rkf_batch_graph_destroy": (_I, [_P]),
    "rkf_bvh_build": (_I, [_P, _U32, _P, _U32, C.POINTER(_U32)]),
    "rkf_scene_info_get": (_I, [_P, C.POINTER(rkf_scene_info)]),
    "rkf_pool_export_voxelsample": (_I, [_P, _U32, _U32, _P]),
    "rkf_brick_lookup": (_I, [_P, _U32, _P, _U32, _P]),
    "rkf_pool_export_planes": (_I, [_P, _U32, _U32, _P, _P, _P, _P]),
    "rkf_index_export": (_I, [_P, _P, C.POINTER(_U64), _P, C.POINTER(_U64), _P, C.POINTER(_U32)]),
    "rkf_voxelize_prims": (_I, [_P, _P, _U32, C.POINTER(rkf_voxelize_params), C.POINTER(_U32)]),
    "rkf_object_get": (_I, [_P, _U32, C.POINTER(rkf_gpu_object)]),
    "rkf_march": (_I, [_P, C.POINTER(rkf_camera), C.POINTER(rkf_march_params), _U32, _U32,
                       C.POINTER(rkf_gbuffer)]),
    "rkf_march_plain": (_I, [_P, C.POINTER(rkf_camera), C.POINTER(rkf_march_params), _U32,
                             _U32, C.POINTER(rkf_gbuffer)]),
    "rkf_march_async": (_I, [_P, C.POINTER(rkf_camera), C.POINTER(rkf_march_params), _U32, _U32,
                             C.POINTER(rkf_gbuffer), _P]),
    "rkf_march_plain_async": (_I, [_P, C.POINTER(rkf_camera), C.POINTER(rkf_march_params), _U32,
                                   _U32, C.POINTER(rkf_gbuffer), _P]),
    "rkf_trace_rays": (_I, [_P, _P, _P, _P, _U32, _U32, C.POINTER(rkf_march_params), _U32,
                            C.POINTER(rkf_hits)]),
    "rkf_secondary_rays": (_I, [_P, C.POINTER(rkf_camera), _U32, _U32, C.POINTER(rkf_gbuffer), _P, _U32,
                                _U32, C.c_float, _U32, _P, _P, _P, _P, _P, _P, C.POINTER(_U32), _P]),
    "rkf_query_points": (_I, [_P, _P, _U32, _P, _P, _P, _U32]),
    "rkf_edit_csg": (_I, [_P, C.POINTER(rkf_edit_op), C.POINTER(_U64)]),
    "rkf_march_batch": (_I, [_P, C.POINTER(rkf_view), _U32, C.POINTER(rkf_ray_batch), _U32,
                             C.POINTER(rkf_march_params), C.POINTER(rkf_batch_tuning)]),
    "rkf_march_batch_async": (_I, [_P, C.POINTER(rkf_view), _U32, C.POINTER(rkf_ray_batch), _U32,
                                   C.POINTER(rkf_march_params), C.POINTER(rkf_batch_tuning), _P]),
    "rkf_trace_rays_plain_async": (_I, [_P, _P, _P, _P, _U32, _U32, C.POINTER(rkf_march_params),
                                        C.POINTER(rkf_hits), _P]),
    "rkf_march_batch_noalloc": (_I, [_P, C.POINTER(rkf_view), _U32, C.POINTER(rkf_ray_batch), _U32,
                                     C.POINTER(rkf_march_params), C.POINTER(rkf_batch_tuning), _P]),
    "rkf_autotune": (_I, [_P, C.POINTER(rkf_view), _U32, C.POINTER(rkf_ray_batch), _U32,
                          C.POINTER(rkf_march_params), C.POINTER(rkf_batch_tuning)]),
    "rkf_tuning_set": (_I, [_P, C.POINTER(rkf_batch_tuning)]),
    "rkf_tuning_get": (_I, [_P, C.POINTER(rkf_batch_tuning)]),
    "rkf_serve_start": (_I, [_P, C.POINTER(rkf_march_params)]),
    "rkf_serve_stop": (_I, [_P]),
    "rkf_submit": (_I, [_P, C.POINTER(rkf_request), C.POINTER(_U64)]),
    "rkf_poll": (_I, [_P, _U64, C.POINTER(rkf_result), _U32]),
    "rkf_cancel": (_I, [_P, _U64]),
    "rkf_sdf_ao": (_I, [_P, _P, _P, _U32, _P, _U32]),
    "rkf_pool_import_soa": (_I, [_P, _P, _P, _P, _U32, _U32]),
    "rkf_testing_fail_allocation_after": (None, [C.c_longlong]),
    "rkf_testing_export_empty_dist": (_I, [_P, _P, C.POINTER(C.c_uint64)]),
    "rkf_testing_set_host_bands": (None, [C.c_int]),
    "rkf_testing_export_coarse": (_I, [_P, _P, _P, _P, C.POINTER(C.c_uint64)]),
    "rkf_testing_last_variant": (C.c_int, [_P]),
    "rkf_testing_far_ball": (C.c_int, [_P, C.c_float, _P]),
    "rkf_testing_far_plane": (C.c_int, [_P, C.c_float, _P]),
    "rkf_testing_pool_state": (_I, [_P, _P]),
    "rkf_testing_march_timing": (_I, [_P, C.c_uint32]),
    "rkf_testing_launch_stats": (_I, [_P, C.POINTER(C.c_uint64), _P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "rkf_world_relative": (None, [C.POINTER(rkf_world_pos), C.POINTER(rkf_world_pos),
                                  C.POINTER(C.c_double), C.POINTER(C.c_float)]),
    "rkf_scene_origin_set": (_I, [_P, C.POINTER(rkf_world_pos)]),
    "rkf_scene_origin_get": (_I, [_P, C.POINTER(rkf_world_pos)]),
    "rkf_march_world": (_I, [_P, C.POINTER(rkf_world_pos), C.POINTER(rkf_camera), C.POINTER(rkf_march_params),
                             _U32, _U32, C.POINTER(rkf_gbuffer)]),
    "rkf_trace_rays_world": (_I, [_P, _P, _P, _P, _U32, _U32, C.POINTER(rkf_march_params),
                                  C.POINTER(rkf_hits)]),
}

_lib = None


def load_library(path: str | None = None) -> C.CDLL:
    """Load the CUDA library; raise if it is missing (no fallback exists)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("RKF_CUDA_LIB", LIB_PATH)
    if not os.path.exists(p):
        raise RuntimeError(
            f"librkf_cuda.so not found at {p}; build it with `python -m rkifield_b200.build` "
            "(the march has no CPU fallback)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class RkfError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status: int, where: str) -> None:
    if status != RKF_OK:
        msg = load_library().rkf_last_error()
        raise RkfError(status, where, msg.decode() if msg else "")
