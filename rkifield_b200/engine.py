"""Host-side mirror of the reference's march interfaces over the C ABI.

The reference drives the march through ``GpuScene`` uploads
(``crates/rkf-render/src/gpu_scene.rs:141-234``), ``RayMarchPass::dispatch``
(``crates/rkf-render/src/ray_march.rs:96-118``) and physics point queries
through ``trait SdfQueryable`` (``crates/rkf-physics/src/sdf_collision.rs:38-44``).
This module offers the same operations, same names and argument meaning, on
top of ``librkf_cuda.so``.  Every call goes to the CUDA library; there is no
CPU path.  Errors raise :class:`RkfError` carrying the library status.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as abi
from ._abi import RkfError, check  # noqa: F401  (re-exported)

PRECISIONS = {"f16": abi.RKF_PRECISION_F16, "f32": abi.RKF_PRECISION_F32, "u8": abi.RKF_PRECISION_U8}


def _p(a):
    return None if a is None else a.ctypes.data


def build_bvh(pairs) -> C.Array:
    """``Bvh::build`` (crates/rkf-core/src/bvh.rs:66-260) over ``(object_index,
    aabb_min, aabb_max)`` triples, as the GPU node array ``upload_bvh`` takes
    (``GpuBvhNode::from_cpu``, gpu_bvh.rs:45-60); built on the host by the
    library."""
    pairs = list(pairs)
    items = (abi.rkf_bvh_item * max(1, len(pairs)))()
    for k, (oi, lo, hi) in enumerate(pairs):
        items[k].object_index = int(oi)
        for a in range(3):
            items[k].aabb_min[a] = float(lo[a])
            items[k].aabb_max[a] = float(hi[a])
    cap = max(1, 2 * len(pairs) - 1)
    nodes = (abi.rkf_bvh_node * cap)()
    n = C.c_uint32()
    check(abi.load_library().rkf_bvh_build(items, len(pairs), nodes, cap, C.byref(n)), "rkf_bvh_build")
    return (abi.rkf_bvh_node * n.value).from_buffer_copy(nodes, 0) if n.value else (abi.rkf_bvh_node * 0)()


def object_bvh(objects) -> C.Array:
    """The BVH the runtime uploads with its objects: one leaf per object
    index over the object's AABB (render.rs:79-140)."""
    return build_bvh((i, o.aabb_min, o.aabb_max) for i, o in enumerate(objects))


def scene_node(parent: int = abi.RKF_NO_PARENT, position=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0, 1.0),
               scale=(1.0, 1.0, 1.0), visible: bool = True, sdf_type: int = abi.RKF_SDF_NONE,
               primitive_type: int = 0, params=(0.0, 0.0, 0.0, 0.0), material_id: int = 0,
               brick_map_offset: int = 0, brick_map_dims=(0, 0, 0), voxel_size: float = 0.0,
               blend_mode: int = abi.RKF_BLEND_SMOOTH_UNION, blend_radius: float = 0.1) -> abi.rkf_scene_node:
    """One node of an object's tree (SceneNode, scene_node.rs); the defaults
    are SceneNode::new's: identity transform, visible, no SDF source, smooth
    union of radius 0.1 (BlendMode::default, scene_node.rs:124-128)."""
    nd = abi.rkf_scene_node()
    nd.position[:], nd.rotation[:], nd.scale[:] = list(position), list(rotation), list(scale)
    nd.parent, nd.visible, nd.sdf_type, nd.primitive_type = int(parent), int(bool(visible)), sdf_type, primitive_type
    nd.params[:], nd.material_id = list(params), material_id
    nd.brick_map_offset, nd.brick_map_dims[:], nd.voxel_size = brick_map_offset, list(brick_map_dims), voxel_size
    nd.blend_mode, nd.blend_radius = blend_mode, blend_radius
    return nd


def flatten_object(nodes, rotation=(0.0, 0.0, 0.0, 1.0), scale=(1.0, 1.0, 1.0),
                   position=(0.0, 0.0, 0.0)) -> list:
    """``flatten_object`` (transform_flatten.rs:56-110) of a tree given as
    scene nodes in depth-first pre-order, the object's own rotation and
    scale, and its baked (camera-relative) position: the flat nodes of the
    visible nodes, through rkf_flatten_object."""
    nodes = list(nodes)
    arr = (abi.rkf_scene_node * max(1, len(nodes)))(*nodes)
    out = (abi.rkf_flat_node * max(1, len(nodes)))()
    n = C.c_uint32()
    fl = lambda v: (C.c_float * len(v))(*[float(x) for x in v])  # noqa: E731
    check(abi.load_library().rkf_flatten_object(arr, len(nodes), fl(rotation), fl(scale), fl(position), out,
                                                C.byref(n)), "rkf_flatten_object")
    return [out[i] for i in range(n.value)]


def gpu_object_from_flat_node(flat: abi.rkf_flat_node, source: abi.rkf_scene_node, object_id: int,
                              aabb_min=(0.0,) * 4, aabb_max=(0.0,) * 4, geometry_aabb_min=(0.0,) * 3,
                              geometry_aabb_max=(0.0,) * 3) -> abi.rkf_gpu_object:
    """``GpuObject::from_flat_node`` (gpu_object.rs:141-220) through
    rkf_gpu_object_from_flat_node."""
    fl = lambda v: (C.c_float * len(v))(*[float(x) for x in v])  # noqa: E731
    o = abi.rkf_gpu_object()
    check(abi.load_library().rkf_gpu_object_from_flat_node(
        C.byref(flat), C.byref(source), int(object_id), fl(aabb_min), fl(aabb_max), fl(geometry_aabb_min),
        fl(geometry_aabb_max), C.byref(o)), "rkf_gpu_object_from_flat_node")
    return o


def gbuffer_host(n: int, reference_planes: bool = False) -> dict:
    out = {"t": np.zeros(n, np.float32), "normal": np.zeros(3 * n, np.float32),
           "slot": np.zeros(n, np.uint32), "material": np.zeros(n, np.uint16),
           "flags": np.zeros(n, np.uint16)}
    if reference_planes:
        out["position"] = np.zeros(4 * n, np.float32)
        out["packed_material"] = np.zeros(n, np.uint32)
        out["motion"] = np.zeros(4 * n, np.float32)
    return out


def _gb_struct(out: dict, mem: int = abi.RKF_MEM_HOST) -> abi.rkf_gbuffer:
    g = abi.rkf_gbuffer()
    for k in ("t", "normal", "slot", "material", "flags", "position", "packed_material", "motion"):
        v = out.get(k)
        setattr(g, k, None if v is None else (v if isinstance(v, int) else v.ctypes.data))
    g.mem = mem
    return g


class Context:
    """One device-resident scene (brick pool, brick index, object table)."""

    def __init__(self, device: int = 0, pool_capacity: int = 1 << 16, precision: str = "f16",
                 keep_reference_pool: bool = True, max_inflight: int = 64,
                 mem_budget_bytes: int = 0, u8_round: int = 0, u8_band: float = 0.0):
        self.lib = abi.load_library()
        cfg = abi.rkf_config()
        self.lib.rkf_config_default(C.byref(cfg))
        cfg.device = device
        cfg.pool_capacity_bricks = pool_capacity
        cfg.precision = PRECISIONS[precision]
        cfg.keep_reference_pool = int(keep_reference_pool)
        cfg.max_inflight = max_inflight
        cfg.mem_budget_bytes = mem_budget_bytes
        cfg.u8_round = u8_round
        cfg.u8_band = u8_band
        h = C.c_void_p()
        check(self.lib.rkf_create(C.byref(cfg), C.byref(h)), "rkf_create")
        self.h = h
        self.precision = precision

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if self.h:
            check(self.lib.rkf_destroy(self.h), "rkf_destroy")
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- import (GpuScene::set_brick_pool / upload_brick_maps / upload_objects)
    def set_brick_pool(self, words: np.ndarray, first_slot: int = 0):
        words = np.ascontiguousarray(words, np.uint32)
        assert words.size % 1024 == 0
        check(self.lib.rkf_pool_import_voxelsample(self.h, _p(words), first_slot, words.size // 1024),
              "rkf_pool_import_voxelsample")

    def set_brick_pool_planes(self, dist_f16: np.ndarray, mat: np.ndarray, blend: np.ndarray,
                              first_slot: int = 0):
        """Pool bricks as SoA planes (binary16 bits, material | secondary << 6, blend)."""
        d = np.ascontiguousarray(dist_f16, np.uint16)
        m = np.ascontiguousarray(mat, np.uint16)
        b = np.ascontiguousarray(blend, np.uint8)
        assert d.size == m.size == b.size and d.size % 512 == 0
        check(self.lib.rkf_pool_import_soa(self.h, _p(d), _p(m), _p(b), first_slot, d.size // 512),
              "rkf_pool_import_soa")

    def upload_brick_maps(self, packed: np.ndarray):
        packed = np.ascontiguousarray(packed, np.uint32)
        check(self.lib.rkf_brickmap_import(self.h, _p(packed), packed.size), "rkf_brickmap_import")

    def upload_objects(self, objects):
        arr = (abi.rkf_gpu_object * len(objects))(*objects)
        check(self.lib.rkf_objects_import(self.h, arr, len(objects)), "rkf_objects_import")

    def update_objects(self, objects, index_source=None):
        """Replace the object records, keeping the brick index (rkf_objects_update)."""
        arr = (abi.rkf_gpu_object * max(1, len(objects)))(*objects)
        src = None if index_source is None else np.ascontiguousarray(index_source, np.int32)
        check(self.lib.rkf_objects_update(self.h, arr, len(objects), _p(src)), "rkf_objects_update")

    def upload_bvh(self, nodes):
        """BVH nodes, root first (an ``rkf_bvh_node`` array); an empty one removes the BVH."""
        check(self.lib.rkf_bvh_import(self.h, nodes if len(nodes) else None, len(nodes)), "rkf_bvh_import")

    def voxelize(self, prims: np.ndarray, vp: abi.rkf_voxelize_params) -> int:
        prims = np.ascontiguousarray(prims)
        idx = C.c_uint32()
        check(self.lib.rkf_voxelize_prims(self.h, _p(prims), len(prims), C.byref(vp), C.byref(idx)),
              "rkf_voxelize_prims")
        return idx.value

    def info(self) -> dict:
        i = abi.rkf_scene_info()
        check(self.lib.rkf_scene_info_get(self.h, C.byref(i)), "rkf_scene_info_get")
        return {k: getattr(i, k) for k, _ in abi.rkf_scene_info._fields_}

    def object(self, i: int) -> abi.rkf_gpu_object:
        o = abi.rkf_gpu_object()
        check(self.lib.rkf_object_get(self.h, i, C.byref(o)), "rkf_object_get")
        return o

    def export_pool(self, first_slot: int, n_bricks: int) -> np.ndarray:
        w = np.zeros(n_bricks * 1024, np.uint32)
        check(self.lib.rkf_pool_export_voxelsample(self.h, first_slot, n_bricks, _p(w)),
              "rkf_pool_export_voxelsample")
        return w

    def export_planes(self, first_slot: int, n_bricks: int) -> dict:
        """SoA planes of the device pool (distance at the context precision)."""
        dt = {"f16": np.uint16, "f32": np.float32, "u8": np.int8}[self.precision]
        out = {"dist": np.zeros(n_bricks * 512, dt), "mat": np.zeros(n_bricks * 512, np.uint16),
               "blend": np.zeros(n_bricks * 512, np.uint8)}
        if self.precision == "u8":
            out["step"] = np.zeros(n_bricks, np.float32)
        check(self.lib.rkf_pool_export_planes(self.h, first_slot, n_bricks, _p(out["dist"]), _p(out.get("step")),
                                              _p(out["mat"]), _p(out["blend"])), "rkf_pool_export_planes")
        return out

    def export_index(self) -> dict:
        """Device brick index (top grids, leaves, per-object top info)."""
        tn, ln, no = C.c_uint64(), C.c_uint64(), C.c_uint32()
        check(self.lib.rkf_index_export(self.h, None, C.byref(tn), None, C.byref(ln), None, C.byref(no)),
              "rkf_index_export")
        top = np.zeros(max(1, tn.value), np.uint32)
        leaves = np.zeros(max(1, ln.value), np.uint32)
        info = np.zeros(4 * max(1, no.value), np.uint32)
        check(self.lib.rkf_index_export(self.h, _p(top), C.byref(tn), _p(leaves), C.byref(ln), _p(info),
                                        C.byref(no)), "rkf_index_export")
        return {"top": top, "leaves": leaves, "obj_top_info": info}

    def march_async(self, cam, params, width: int, height: int, dev_ptrs: dict, stream_ptr: int,
                    plain: bool = False):
        """Enqueue a march on a caller stream into device planes (no sync)."""
        g = _gb_struct(dev_ptrs, abi.RKF_MEM_DEVICE)
        fn = self.lib.rkf_march_plain_async if plain else self.lib.rkf_march_async
        check(fn(self.h, C.byref(cam), C.byref(params), width, height, C.byref(g), stream_ptr),
              "rkf_march_async")

    def set_tuning(self, tuning: abi.rkf_batch_tuning):
        """The launch tuning of the context's marches (rkf_tuning_set)."""
        check(self.lib.rkf_tuning_set(self.h, C.byref(tuning)), "rkf_tuning_set")

    def tuning(self) -> abi.rkf_batch_tuning:
        tu = abi.rkf_batch_tuning()
        check(self.lib.rkf_tuning_get(self.h, C.byref(tu)), "rkf_tuning_get")
        return tu

    def brick_lookup(self, obj: int, bxyz: np.ndarray) -> np.ndarray:
        bxyz = np.ascontiguousarray(bxyz, np.uint32)
        n = bxyz.size // 3
        out = np.zeros(n, np.uint32)
        check(self.lib.rkf_brick_lookup(self.h, obj, _p(bxyz), n, _p(out)), "rkf_brick_lookup")
        return out

    # -- march (RayMarchPass::dispatch) ------------------------------------
    def march(self, cam, params, width: int, height: int, reference_planes: bool = False,
              out: dict | None = None, plain: bool = False) -> dict:
        out = out if out is not None else gbuffer_host(width * height, reference_planes)
        g = _gb_struct(out)
        fn = self.lib.rkf_march_plain if plain else self.lib.rkf_march
        check(fn(self.h, C.byref(cam), C.byref(params), width, height, C.byref(g)),
              "rkf_march_plain" if plain else "rkf_march")
        return out

    def march_device(self, cam, params, width: int, height: int, dev_ptrs: dict, plain: bool = False):
        g = _gb_struct(dev_ptrs, abi.RKF_MEM_DEVICE)
        fn = self.lib.rkf_march_plain if plain else self.lib.rkf_march
        check(fn(self.h, C.byref(cam), C.byref(params), width, height, C.byref(g)), "march")

    # -- WorldPosition cameras and rays (FP64 rebasing, world_position.rs) --
    def set_scene_origin(self, chunk, local=(0.0, 0.0, 0.0)):
        """The WorldPosition the scene's f32 world space is relative to."""
        o = abi.rkf_world_pos()
        o.chunk[:] = [int(x) for x in chunk]
        o.local[:] = [float(x) for x in local]
        check(self.lib.rkf_scene_origin_set(self.h, C.byref(o)), "rkf_scene_origin_set")

    def march_world(self, cam_chunk, cam_local, cam, params, width: int, height: int,
                    reference_planes: bool = False) -> dict:
        """rkf_march with the camera at WorldPosition (cam_chunk, cam_local)."""
        wp = abi.rkf_world_pos()
        wp.chunk[:] = [int(x) for x in cam_chunk]
        wp.local[:] = [float(x) for x in cam_local]
        out = gbuffer_host(width * height, reference_planes)
        g = _gb_struct(out)
        check(self.lib.rkf_march_world(self.h, C.byref(wp), C.byref(cam), C.byref(params), width, height,
                                       C.byref(g)), "rkf_march_world")
        return out

    def trace_world(self, chunks, locals_, dirs, tmax, mode: int, params) -> dict:
        """rkf_trace_rays with origins given as WorldPositions (chunks int32
        (n,3), local offsets float32 (n,3))."""
        chunks = np.ascontiguousarray(chunks, np.int32).reshape(-1, 3)
        locals_ = np.ascontiguousarray(locals_, np.float32).reshape(-1, 3)
        n = chunks.shape[0]
        wp = (abi.rkf_world_pos * max(1, n))()
        buf = np.frombuffer(wp, dtype=np.dtype([("c", np.int32, 3), ("l", np.float32, 3)]), count=n)
        buf["c"], buf["l"] = chunks, locals_
        dirs = np.ascontiguousarray(dirs, np.float32).ravel()
        tmax = np.ascontiguousarray(tmax, np.float32).ravel()
        out = {"t": np.zeros(n, np.float32), "flags": np.zeros(n, np.uint16)}
        if mode == abi.RKF_TRACE_CLOSEST:
            out.update(normal=np.zeros(3 * n, np.float32), slot=np.zeros(n, np.uint32),
                       material=np.zeros(n, np.uint16))
        h = abi.rkf_hits()
        h.t, h.flags = _p(out["t"]), _p(out["flags"])
        h.normal, h.slot, h.material = _p(out.get("normal")), _p(out.get("slot")), _p(out.get("material"))
        h.mem = abi.RKF_MEM_HOST
        check(self.lib.rkf_trace_rays_world(self.h, wp, _p(dirs), _p(tmax), n, mode, C.byref(params), C.byref(h)),
              "rkf_trace_rays_world")
        return out

    # -- generic ray casts -------------------------------------------------
    def trace(self, origins, dirs, tmax, mode: int, params, closest_planes: bool = True) -> dict:
        origins = np.ascontiguousarray(origins, np.float32).ravel()
        dirs = np.ascontiguousarray(dirs, np.float32).ravel()
        tmax = np.ascontiguousarray(tmax, np.float32).ravel()
        n = tmax.size
        out = {"t": np.zeros(n, np.float32), "flags": np.zeros(n, np.uint16)}
        if mode == abi.RKF_TRACE_CLOSEST and closest_planes:
            out.update(normal=np.zeros(3 * n, np.float32), slot=np.zeros(n, np.uint32),
                       material=np.zeros(n, np.uint16))
        h = abi.rkf_hits()
        h.t = _p(out["t"])
        h.normal = _p(out.get("normal"))
        h.slot = _p(out.get("slot"))
        h.material = _p(out.get("material"))
        h.flags = _p(out["flags"])
        h.mem = abi.RKF_MEM_HOST
        check(self.lib.rkf_trace_rays(self.h, _p(origins), _p(dirs), _p(tmax), n, mode,
                                      C.byref(params), abi.RKF_MEM_HOST, C.byref(h)),
              "rkf_trace_rays")
        return out

    # -- point queries (SdfQueryable) --------------------------------------
    def query_points(self, points) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        pts = np.ascontiguousarray(points, np.float32).ravel()
        n = pts.size // 3
        d = np.zeros(n, np.float32)
        g = np.zeros(3 * n, np.float32)
        m = np.zeros(n, np.uint16)
        check(self.lib.rkf_query_points(self.h, _p(pts), n, _p(d), _p(g), _p(m), abi.RKF_MEM_HOST),
              "rkf_query_points")
        return d, g, m

    # -- edits ---------------------------------------------------------------
    def sdf_ao(self, pos, normal) -> np.ndarray:
        """sdf_ao at each position along its normal (host arrays)."""
        pos = np.ascontiguousarray(pos, np.float32).ravel()
        normal = np.ascontiguousarray(normal, np.float32).ravel()
        assert pos.size == normal.size and pos.size % 3 == 0
        out = np.zeros(pos.size // 3, np.float32)
        check(self.lib.rkf_sdf_ao(self.h, _p(pos), _p(normal), out.size, _p(out), abi.RKF_MEM_HOST), "rkf_sdf_ao")
        return out

    def edit(self, op: abi.rkf_edit_op) -> int:
        ep = C.c_uint64()
        check(self.lib.rkf_edit_csg(self.h, C.byref(op), C.byref(ep)), "rkf_edit_csg")
        return ep.value


class Server:
    """The resident request loop of a :class:`Context` (rkf_serve_start).

    submit_* admit one request and return its ticket; the arrays passed in
    (inputs and the output arrays the result is written to) must stay alive
    until poll returns the ticket.  Page-locked arrays let the loop copy
    asynchronously.  A refused admission raises RkfError(RKF_BUSY)."""

    def __init__(self, ctx: Context, params):
        self.ctx = ctx
        self.lib = ctx.lib
        self.params = params
        check(self.lib.rkf_serve_start(ctx.h, C.byref(params)), "rkf_serve_start")
        self._keep = {}

    def _submit(self, req, keep):
        t = C.c_uint64()
        check(self.lib.rkf_submit(self.ctx.h, C.byref(req), C.byref(t)), "rkf_submit")
        self._keep[t.value] = (req, keep)
        return t.value

    def submit_render(self, cam, width: int, height: int, out: dict) -> int:
        r = abi.rkf_request()
        r.kind = abi.RKF_REQ_RENDER
        r.width, r.height, r.n = width, height, width * height
        r.camera = cam
        r.out_t, r.out_normal = _p(out["t"]), _p(out["normal"])
        r.out_slot, r.out_material, r.out_flags = _p(out["slot"]), _p(out["material"]), _p(out["flags"])
        return self._submit(r, out)

    def submit_rays(self, o, d, tmax, mode: int, out: dict) -> int:
        r = abi.rkf_request()
        r.kind = abi.RKF_REQ_RAYS
        r.mode = mode
        r.n = tmax.size
        r.in0, r.in1, r.in2 = _p(o), _p(d), _p(tmax)
        r.out_t, r.out_flags = _p(out["t"]), _p(out["flags"])
        r.out_normal, r.out_slot, r.out_material = _p(out.get("normal")), _p(out.get("slot")), _p(out.get("material"))
        return self._submit(r, (o, d, tmax, out))

    def submit_points(self, pts, out: dict) -> int:
        r = abi.rkf_request()
        r.kind = abi.RKF_REQ_POINTS
        r.n = pts.size // 3
        r.in0 = _p(pts)
        r.out_t, r.out_normal, r.out_material = _p(out["dist"]), _p(out["grad"]), _p(out["material"])
        return self._submit(r, (pts, out))

    def submit_edit(self, op) -> int:
        r = abi.rkf_request()
        r.kind = abi.RKF_REQ_EDIT
        r.edit = op
        return self._submit(r, None)

    def poll(self, ticket: int, timeout_us: int = 0):
        """Returns the rkf_result as a dict, or None if not complete."""
        res = abi.rkf_result()
        st = self.lib.rkf_poll(self.ctx.h, ticket, C.byref(res), timeout_us)
        if st in (abi.RKF_NOT_READY, abi.RKF_TIMEOUT):
            return None
        check(st, "rkf_poll")
        self._keep.pop(ticket, None)
        return {k: getattr(res, k) for k, _ in abi.rkf_result._fields_}

    def cancel(self, ticket: int):
        check(self.lib.rkf_cancel(self.ctx.h, ticket), "rkf_cancel")

    def stop(self):
        check(self.lib.rkf_serve_stop(self.ctx.h), "rkf_serve_stop")


def render_out(n: int) -> dict:
    return gbuffer_host(n)


def rays_out(n: int, mode: int) -> dict:
    out = {"t": np.zeros(n, np.float32), "flags": np.zeros(n, np.uint16)}
    if mode == abi.RKF_TRACE_CLOSEST:
        out.update(normal=np.zeros(3 * n, np.float32), slot=np.zeros(n, np.uint32),
                   material=np.zeros(n, np.uint16))
    return out


def points_out(n: int) -> dict:
    return {"dist": np.zeros(n, np.float32), "grad": np.zeros(3 * n, np.float32),
            "material": np.zeros(n, np.uint16)}


class GpuScene:
    """``GpuScene`` upload surface (gpu_scene.rs:141-234) on a :class:`Context`."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def set_brick_pool(self, words):
        self.ctx.set_brick_pool(words)

    def upload_brick_maps(self, packed):
        self.ctx.upload_brick_maps(packed)

    def upload_objects(self, objects):
        self.ctx.upload_objects(objects)

    def upload_bvh(self, nodes):
        self.ctx.upload_bvh(nodes)


class BatchGraph:
    """A batched march captured once as a CUDA graph (rkf_batch_graph_*): the
    same views and ray batches (device outputs) launched again every frame,
    with new cameras set between launches.  Stale after a scene change
    (RkfError RKF_EPOCH_STALE on launch): make a new one."""

    def __init__(self, ctx: Context, views, batches, params, tuning=None):
        self.ctx = ctx
        self.h = C.c_void_p()
        self._keep = (views, batches, params, tuning)
        nv = len(views) if views is not None else 0
        nb = len(batches) if batches is not None else 0
        check(ctx.lib.rkf_batch_graph_create(ctx.h, views, nv, batches, nb, C.byref(params),
                                             C.byref(tuning) if tuning is not None else None, C.byref(self.h)),
              "rkf_batch_graph_create")
        self.n_views = nv

    def set_cameras(self, cams):
        arr = (abi.rkf_camera * len(cams))(*cams)
        check(self.ctx.lib.rkf_batch_graph_set_cameras(self.h, arr, len(cams)), "rkf_batch_graph_set_cameras")

    def launch(self, stream_ptr: int | None = None):
        check(self.ctx.lib.rkf_batch_graph_launch(self.h, stream_ptr), "rkf_batch_graph_launch")

    def close(self):
        if self.h.value:
            self.ctx.lib.rkf_batch_graph_destroy(self.h)
            self.h = C.c_void_p()


class RayMarchPass:
    """``RayMarchPass`` (ray_march.rs:29-119): dispatch marches one view into
    a G-buffer (SoA numpy planes)."""

    DEFAULT_INTERNAL = (960, 540)  # ray_march.rs:24-26

    def __init__(self, scene: GpuScene, width: int = 960, height: int = 540):
        self.scene = scene
        self.width, self.height = width, height

    def dispatch(self, camera, params, reference_planes: bool = False) -> dict:
        return self.scene.ctx.march(camera, params, self.width, self.height, reference_planes)


class BrickPoolSdf:
    """``SdfQueryable`` backed by the device brick pool: ``evaluate`` and
    ``gradient`` of sdf_collision.rs:38-44, batched."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def evaluate(self, pos) -> np.ndarray:
        return self.ctx.query_points(pos)[0]

    def gradient(self, pos) -> np.ndarray:
        return self.ctx.query_points(pos)[1].reshape(-1, 3)
