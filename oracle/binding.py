"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module, as the checker or as the timed CPU baseline.  The
product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from rkifield_b200 import _abi as abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle_rkf.so")


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


class orc_scene(C.Structure):
    _fields_ = [("pool_words", C.c_void_p), ("dist_f16", C.c_void_p), ("dist_f32", C.c_void_p),
                ("dist_u8", C.c_void_p), ("brick_scale", C.c_void_p), ("mat_plane", C.c_void_p),
                ("blend_plane", C.c_void_p), ("precision", C.c_uint32),
                ("brick_maps", C.c_void_p), ("top", C.c_void_p), ("leaves", C.c_void_p),
                ("obj_top_info", C.c_void_p), ("objects", C.c_void_p),
                ("num_objects", C.c_uint32), ("dist_f64", C.c_void_p),
                ("bvh", C.c_void_p), ("bvh_nodes", C.c_uint32)]

PRECISION_F64 = 3


class orc_stats(C.Structure):
    _fields_ = [("sectors", C.c_uint64), ("index_sectors", C.c_uint64),
                ("dist_sectors", C.c_uint64), ("mat_sectors", C.c_uint64),
                ("steps", C.c_uint64), ("evals", C.c_uint64)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, U32, I = C.c_void_p, C.c_uint32, C.c_int
        L.orc_f16_from_f32.restype = C.c_uint16
        L.orc_f16_from_f32.argtypes = [C.c_float]
        L.orc_coarse_field.restype = C.c_uint64
        L.orc_coarse_field.argtypes = [P, U32, P, P, P, C.c_uint64]
        L.orc_f16_to_f32.restype = C.c_float
        L.orc_f16_to_f32.argtypes = [C.c_uint16]
        L.orc_prim_sdf.restype = C.c_float
        L.orc_prim_sdf.argtypes = [P, P]
        L.orc_smin.restype = C.c_float
        L.orc_smin.argtypes = [C.c_float, C.c_float, C.c_float]
        L.orc_scene_eval.restype = C.c_float
        L.orc_scene_eval.argtypes = [P, U32, C.c_float, C.c_float, P, P, P, P]
        L.orc_voxelize.restype = P
        L.orc_voxelize.argtypes = [P, U32, P, I]
        L.orc_voxelized_info.argtypes = [P, P, P, P]
        L.orc_voxelized_copy.argtypes = [P, P, P]
        L.orc_voxelized_copy_f32.argtypes = [P, P]
        L.orc_voxelized_free.argtypes = [P]
        L.orc_voxelize_sparse.restype = P
        L.orc_voxelize_sparse.argtypes = [P, U32, P, I]
        L.orc_sparse_info.argtypes = [P, P, P, P, P, P]
        L.orc_sparse_copy.argtypes = [P, P, P, P, P, P, P]
        L.orc_sparse_free.argtypes = [P]
        L.orc_voxelize_bricks.argtypes = [P, U32, P, P, U32, P, P, I]
        L.orc_march.argtypes = [P, P, P, U32, U32, I, I, U32, U32] + [P] * 12 + [I, P]
        L.orc_trace_rays.argtypes = [P, P, P, P, U32, U32, P, I, I] + [P] * 7
        L.orc_query_points.argtypes = [P, P, U32, P, P, P, I]
        L.orc_shadow_shader.argtypes = [P, P, P, P, U32, P, I, P]
        L.orc_sdf_ao_shader.argtypes = [P, P, P, U32, P, I, P]
        L.orc_apply_edit_brick.restype = I
        L.orc_apply_edit_brick.argtypes = [P, P, C.c_float, P]
        L.orc_fill_brick_with_brush.argtypes = [P, P, C.c_float, P]
        L.orc_apply_edit_planes.restype = I
        L.orc_apply_edit_planes.argtypes = [P, P, P, P, C.c_float, P]
        L.orc_encode_u8.argtypes = [P, C.c_float, I, P, P]
        L.orc_evaluate_falloff.restype = C.c_float
        L.orc_evaluate_falloff.argtypes = [U32, C.c_float, C.c_float]
        L.orc_evaluate_shape.restype = C.c_float
        L.orc_evaluate_shape.argtypes = [U32, P, P]
        L.orc_sample_brick_trilinear.restype = C.c_float
        L.orc_sample_brick_trilinear.argtypes = [P, P, C.c_float]
        L.orc_march_params_default.argtypes = [P]
        L.orc_voxel_values_f64.argtypes = [P, U32, P, P, U32, P, I]
        L.orc_voxel_values_f64_bricks.argtypes = [P, U32, P, P, P, C.c_uint64, P, I]
        _lib = L
    return _lib


def ptr(a):
    return None if a is None else a.ctypes.data


def nthreads() -> int:
    return max(1, os.cpu_count() or 1)


class Voxelized:
    """Oracle voxelization of a primitive list into a fresh pool + flat map."""

    def __init__(self, prims: np.ndarray, vp: abi.rkf_voxelize_params, threads: int | None = None):
        L = lib()
        h = L.orc_voxelize(ptr(prims), len(prims), C.byref(vp), threads or nthreads())
        dims = np.zeros(3, np.uint32)
        nb = C.c_uint32()
        ni = C.c_uint32()
        L.orc_voxelized_info(h, ptr(dims), C.byref(nb), C.byref(ni))
        self.dims = dims
        self.n_bricks = nb.value
        self.n_interior = ni.value
        self.words = np.zeros(self.n_bricks * 1024, np.uint32)
        self.map = np.zeros(int(dims.prod()), np.uint32)
        L.orc_voxelized_copy(h, ptr(self.words), ptr(self.map))
        self.dist_f32 = np.zeros(self.n_bricks * 512, np.float32)
        L.orc_voxelized_copy_f32(h, ptr(self.dist_f32))
        L.orc_voxelized_free(h)
        self.voxel_size = vp.voxel_size

    def gpu_object(self, object_id: int = 1) -> abi.rkf_gpu_object:
        """The object's GpuObject (identity transform, unit scale) with the
        tight AABB of allocated bricks (brick_ops.rs:225-262)."""
        o = abi.rkf_gpu_object()
        for i in range(4):
            o.inverse_world[i * 4 + i] = 1.0
        vs = np.float32(self.voxel_size)
        be = vs * np.float32(8.0)
        gs = self.dims.astype(np.float32) * be
        for a in range(3):
            o.aabb_min[a] = float(-gs[a] * np.float32(0.5))
            o.aabb_max[a] = float(gs[a] * np.float32(0.5))
        o.brick_map_offset = 0
        for a in range(3):
            o.brick_map_dims[a] = int(self.dims[a])
        o.voxel_size = float(vs)
        o.sdf_type = abi.RKF_SDF_VOXELIZED
        o.accumulated_scale[0] = o.accumulated_scale[1] = o.accumulated_scale[2] = 1.0
        o.object_id = object_id
        # geometry AABB of allocated bricks
        m = self.map.reshape(int(self.dims[2]), int(self.dims[1]), int(self.dims[0]))
        alloc = m < abi.INTERIOR_SLOT
        if alloc.any():
            zz, yy, xx = np.nonzero(alloc)
            lo = np.array([xx.min(), yy.min(), zz.min()], np.float32)
            hi = np.array([xx.max() + 1, yy.max() + 1, zz.max() + 1], np.float32)
            gmin = lo * be - gs * np.float32(0.5)
            gmax = hi * be - gs * np.float32(0.5)
            for a in range(3):
                o.geometry_aabb_min[a] = float(gmin[a])
                o.geometry_aabb_max[a] = float(gmax[a])
        return o


def _object_of(dims, voxel_size, alloc_bxyz, object_id):
    """GpuObject of a voxelized grid (identity transform, unit scale) with the
    tight AABB of its allocated bricks (brick_ops.rs:225-262)."""
    o = abi.rkf_gpu_object()
    for i in range(4):
        o.inverse_world[i * 4 + i] = 1.0
    vs = np.float32(voxel_size)
    be = vs * np.float32(8.0)
    gs = np.asarray(dims).astype(np.float32) * be
    for a in range(3):
        o.aabb_min[a] = float(-gs[a] * np.float32(0.5))
        o.aabb_max[a] = float(gs[a] * np.float32(0.5))
        o.brick_map_dims[a] = int(dims[a])
    o.brick_map_offset = 0
    o.voxel_size = float(vs)
    o.sdf_type = abi.RKF_SDF_VOXELIZED
    o.accumulated_scale[0] = o.accumulated_scale[1] = o.accumulated_scale[2] = 1.0
    o.object_id = object_id
    if len(alloc_bxyz):
        lo = alloc_bxyz.min(axis=0).astype(np.float32)
        hi = (alloc_bxyz.max(axis=0) + 1).astype(np.float32)
        gmin = lo * be - gs * np.float32(0.5)
        gmax = hi * be - gs * np.float32(0.5)
        for a in range(3):
            o.geometry_aabb_min[a] = float(gmin[a])
            o.geometry_aabb_max[a] = float(gmax[a])
    return o


class SparseVoxelized:
    """Oracle voxelization into a two-level index and SoA planes (no flat
    map): the same slots and words as Voxelized, for grids whose flat map
    would not fit host memory."""

    def __init__(self, prims: np.ndarray, vp: abi.rkf_voxelize_params, threads: int | None = None):
        L = lib()
        h = L.orc_voxelize_sparse(ptr(prims), len(prims), C.byref(vp), threads or nthreads())
        self.dims = np.zeros(3, np.uint32)
        self.tdim = np.zeros(3, np.uint32)
        nb, ni, nl = C.c_uint32(), C.c_uint32(), C.c_uint32()
        L.orc_sparse_info(h, ptr(self.dims), ptr(self.tdim), C.byref(nb), C.byref(ni), C.byref(nl))
        self.n_bricks, self.n_interior, self.n_leaves = nb.value, ni.value, nl.value
        self.top = np.zeros(int(self.tdim.astype(np.int64).prod()), np.uint32)
        self.leaves = np.zeros(max(1, self.n_leaves) * 512, np.uint32)
        self.dist_f16 = np.zeros(self.n_bricks * 512, np.uint16)
        self.mat = np.zeros(self.n_bricks * 512, np.uint16)
        self.blend = np.zeros(self.n_bricks * 512, np.uint8)
        self.bxyz = np.zeros((self.n_bricks, 3), np.uint32)
        L.orc_sparse_copy(h, ptr(self.top), ptr(self.leaves), ptr(self.dist_f16), ptr(self.mat), ptr(self.blend),
                          ptr(self.bxyz))
        L.orc_sparse_free(h)
        self.voxel_size = vp.voxel_size
        self.obj_top_info = np.array([0, *self.tdim], np.uint32)

    def gpu_object(self, object_id: int = 1) -> abi.rkf_gpu_object:
        return _object_of(self.dims, self.voxel_size, self.bxyz, object_id)

    def scene(self, object_id: int = 1) -> "Scene":
        return Scene([self.gpu_object(object_id)], top=self.top, leaves=self.leaves, obj_top_info=self.obj_top_info,
                     dist_f16=self.dist_f16, mat_plane=self.mat, blend_plane=self.blend)


class Scene:
    """Keeps the arrays behind an orc_scene alive."""

    def __init__(self, objects, pool_words=None, brick_maps=None, top=None, leaves=None,
                 obj_top_info=None, dist_f16=None, dist_f32=None, dist_u8=None,
                 brick_scale=None, mat_plane=None, blend_plane=None,
                 precision=abi.RKF_PRECISION_F16, dist_f64=None, bvh=None):
        n = len(objects)
        self.objects = (abi.rkf_gpu_object * n)(*objects)
        self._keep = [pool_words, brick_maps, top, leaves, obj_top_info, dist_f16, dist_f32,
                      dist_u8, brick_scale, mat_plane, blend_plane, dist_f64, bvh]
        self.s = orc_scene(ptr(pool_words), ptr(dist_f16), ptr(dist_f32), ptr(dist_u8),
                           ptr(brick_scale), ptr(mat_plane), ptr(blend_plane), precision,
                           ptr(brick_maps), ptr(top), ptr(leaves), ptr(obj_top_info),
                           C.addressof(self.objects), n, ptr(dist_f64),
                           C.addressof(bvh) if bvh is not None and len(bvh) else None,
                           len(bvh) if bvh is not None else 0)


def coarse_field(objects):
    """orc_coarse_field: (origin float32[3], dims uint32[3], texels uint16[])."""
    n = len(objects)
    arr = (abi.rkf_gpu_object * max(n, 1))(*objects)
    origin = np.zeros(3, np.float32)
    dims = np.zeros(3, np.uint32)
    cnt = lib().orc_coarse_field(arr, n, ptr(origin), ptr(dims), None, 0)
    tex = np.zeros(cnt, np.uint16)
    lib().orc_coarse_field(arr, n, ptr(origin), ptr(dims), ptr(tex), cnt)
    return origin, dims, tex


def march(scene: Scene, cam, params, w: int, h: int, fp64: bool = False, threads: int | None = None,
          rows: tuple[int, int] | None = None, with_reference_planes: bool = False,
          with_margin: bool = False, with_root: bool = False, count_sectors: bool = False):
    r0, r1 = rows if rows else (0, 0)
    n = w * ((r1 - r0) if r1 > r0 else h)
    out = {
        "t": np.zeros(n, np.float32), "normal": np.zeros(3 * n, np.float32),
        "slot": np.zeros(n, np.uint32), "material": np.zeros(n, np.uint16),
        "flags": np.zeros(n, np.uint16),
    }
    if with_reference_planes:
        out["position"] = np.zeros(4 * n, np.float32)
        out["packed_material"] = np.zeros(n, np.uint32)
        out["motion"] = np.zeros(4 * n, np.float32)
    if fp64:
        out["t64"] = np.zeros(n, np.float64)
        out["normal64"] = np.zeros(3 * n, np.float64)
    if with_margin:
        out["margin"] = np.full(n, np.inf)
    if with_root and fp64:
        out["t_root"] = np.full(n, np.nan)
    st = orc_stats()
    lib().orc_march(C.byref(scene.s), C.byref(cam), C.byref(params), w, h, int(fp64),
                    threads or nthreads(), r0, r1, ptr(out["t"]), ptr(out["normal"]),
                    ptr(out["slot"]), ptr(out["material"]), ptr(out["flags"]),
                    ptr(out.get("position")), ptr(out.get("packed_material")),
                    ptr(out.get("motion")), ptr(out.get("t64")), ptr(out.get("normal64")),
                    ptr(out.get("margin")), ptr(out.get("t_root")), int(count_sectors),
                    C.byref(st))
    out["stats"] = {k: getattr(st, k) for k, _ in orc_stats._fields_}
    return out


def trace(scene: Scene, origins, dirs, tmax, mode: int, params, fp64: bool = False,
          threads: int | None = None, with_margin: bool = False):
    n = len(tmax)
    out = {"t": np.zeros(n, np.float32), "normal": np.zeros(3 * n, np.float32),
           "slot": np.zeros(n, np.uint32), "material": np.zeros(n, np.uint16),
           "flags": np.zeros(n, np.uint16)}
    if fp64:
        out["t64"] = np.zeros(n, np.float64)
    if with_margin:
        out["margin"] = np.full(n, np.inf)
    lib().orc_trace_rays(C.byref(scene.s), ptr(origins), ptr(dirs), ptr(tmax), n, mode,
                         C.byref(params), int(fp64), threads or nthreads(), ptr(out["t"]),
                         ptr(out["normal"]), ptr(out["slot"]), ptr(out["material"]),
                         ptr(out["flags"]), ptr(out.get("t64")), ptr(out.get("margin")))
    return out


def query_points(scene: Scene, points, threads: int | None = None):
    n = len(points) // 3
    d = np.zeros(n, np.float32)
    g = np.zeros(3 * n, np.float32)
    m = np.zeros(n, np.uint16)
    lib().orc_query_points(C.byref(scene.s), ptr(points), n, ptr(d), ptr(g), ptr(m),
                           threads or nthreads())
    return d, g, m


def sdf_ao(scene: Scene, pos, normal, threads: int | None = None):
    pos = np.ascontiguousarray(pos, np.float32).ravel()
    normal = np.ascontiguousarray(normal, np.float32).ravel()
    out = np.zeros(pos.size // 3, np.float32)
    lib().orc_sdf_ao(C.byref(scene.s), ptr(pos), ptr(normal), out.size, ptr(out), threads or nthreads())
    return out


def shadow_shader(scene: Scene, origins, dirs, tmax, cam_pos, threads: int | None = None):
    """soft_shadow through the shading pass's coarse-field sample_sdf, seen
    from the camera at cam_pos (orc_shadow_shader)."""
    origins = np.ascontiguousarray(origins, np.float32).ravel()
    dirs = np.ascontiguousarray(dirs, np.float32).ravel()
    tmax = np.ascontiguousarray(tmax, np.float32).ravel()
    cam = np.ascontiguousarray(cam_pos[:3], np.float32)
    out = np.zeros(tmax.size, np.float32)
    lib().orc_shadow_shader(C.byref(scene.s), ptr(origins), ptr(dirs), ptr(tmax), tmax.size, ptr(cam),
                            threads or nthreads(), ptr(out))
    return out


def sdf_ao_shader(scene: Scene, pos, normal, cam_pos, threads: int | None = None):
    """sdf_ao through the shading pass's coarse-field sample_sdf (orc_sdf_ao_shader)."""
    pos = np.ascontiguousarray(pos, np.float32).ravel()
    normal = np.ascontiguousarray(normal, np.float32).ravel()
    cam = np.ascontiguousarray(cam_pos[:3], np.float32)
    out = np.zeros(pos.size // 3, np.float32)
    lib().orc_sdf_ao_shader(C.byref(scene.s), ptr(pos), ptr(normal), out.size, ptr(cam), threads or nthreads(),
                            ptr(out))
    return out


def voxel_values_f64(prims, vp, brick_map, n_slots: int, threads: int | None = None):
    """FP64 scene SDF at the voxel centres of every allocated brick."""
    out = np.zeros(n_slots * 512, np.float64)
    lib().orc_voxel_values_f64(ptr(prims), len(prims), C.byref(vp), ptr(brick_map), n_slots, ptr(out),
                               threads or nthreads())
    return out


def voxel_values_f64_bricks(prims, vp, bxyz, slots, n_slots: int, threads: int | None = None):
    """FP64 scene SDF at the voxel centres of the listed bricks (coordinates
    bxyz (n,3), pool slots (n,)), into an array of n_slots bricks."""
    bxyz = np.ascontiguousarray(bxyz, np.uint32)
    slots = np.ascontiguousarray(slots, np.uint32)
    out = np.zeros(int(n_slots) * 512, np.float64)
    lib().orc_voxel_values_f64_bricks(ptr(prims), len(prims), C.byref(vp), ptr(bxyz), ptr(slots), slots.size,
                                      ptr(out), threads or nthreads())
    return out


def index_bricks(top, leaves, obj_top_info, obj: int = 0):
    """Brick coordinates and pool slots of every allocated brick of one object
    in a two-level index (top grid of 8^3-brick blocks, 512-entry leaves)."""
    off, tx, ty, tz = (int(x) for x in obj_top_info[4 * obj:4 * obj + 4])
    cells = np.asarray(top[off:off + tx * ty * tz], np.uint32)
    blk = np.nonzero(cells < abi.INTERIOR_SLOT)[0]
    leaf = cells[blk].astype(np.int64)
    kx, ky, kz = blk % tx, (blk // tx) % ty, blk // (tx * ty)
    j = np.arange(512)
    sl = np.asarray(leaves, np.uint32).reshape(-1, 512)[leaf]  # (nblk, 512)
    m = sl < abi.INTERIOR_SLOT
    bi, ji = np.nonzero(m)
    bx = kx[bi] * 8 + (j[ji] & 7)
    by = ky[bi] * 8 + ((j[ji] >> 3) & 7)
    bz = kz[bi] * 8 + (j[ji] >> 6)
    return np.stack([bx, by, bz], axis=1).astype(np.uint32), sl[bi, ji].astype(np.uint32)
