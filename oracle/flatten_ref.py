"""Test infrastructure: a CPU restatement of transform flattening and of the
GpuObject record of a flat node, the checker for rkf_flatten_object and
rkf_gpu_object_from_flat_node.  Never part of the product path.

flatten_object / flatten_node: crates/rkf-core/src/transform_flatten.rs:56-110.
GpuObject::from_flat_node: crates/rkf-render/src/gpu_object.rs:141-220, with
primitive_params (:233-256) and blend_mode_encode (:258-266).

Written independently of the library's version: the rotation here turns the
basis vectors by quaternion products (q v q*), matrices are numpy float64
and the inverse is numpy's.  The reference computes in f32 through glam
0.29 (Cargo.toml:31), whose operation order is not restated; its own tests
compare within 1e-3..1e-6, and so do the tests built on this restatement.
"""
import numpy as np

NO_PARENT = 0xFFFFFFFF


def _qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array([aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw,
                     aw * bw - ax * bx - ay * by - az * bz])


def trs_matrix(rotation, scale, translation):
    """Mat4::from_scale_rotation_translation (Transform::to_matrix,
    scene_node.rs:46-52): column j is the rotated basis vector e_j scaled by
    scale[j]; the last column is the translation.  The quaternion is used as
    given (q v q* with q* the conjugate), which for a non-unit q scales by
    |q|^2 as the closed-form matrix does."""
    q = np.asarray(rotation, np.float64)
    qc = np.array([-q[0], -q[1], -q[2], q[3]])
    m = np.eye(4)
    for j in range(3):
        e = np.zeros(4)
        e[j] = 1.0
        v = _qmul(_qmul(q, e), qc)[:3]
        # q v q* of a non-unit q scales by |q|^2; the closed form keeps the
        # diagonal's 1 - 2(..) terms, which differ from it by (|q|^2 - 1) on
        # the diagonal
        v[j] += 1.0 - float(q @ q)
        m[:3, j] = v * float(np.float64(scale[j]))
    m[:3, 3] = np.asarray(translation, np.float64)
    return m


def flatten_object(nodes, rotation, scale, position):
    """nodes: dicts with position, rotation, scale, parent, visible (pre-order,
    root first).  Returns dicts with inverse_world (4x4 float64, not rounded),
    accumulated_scale (float32 products, as glam's Vec3 mul), depth,
    parent_index and node."""
    obj_world = trs_matrix(rotation, scale, position)
    out = []
    # flatten_node recursion, restated over the pre-order list
    children = {i: [] for i in range(len(nodes))}
    for i, nd in enumerate(nodes[1:], start=1):
        children[nd["parent"]].append(i)

    def walk(i, parent_world, parent_scale, depth, parent_index):
        nd = nodes[i]
        world = parent_world @ trs_matrix(nd["rotation"], nd["scale"], nd["position"])
        acc = (np.asarray(parent_scale, np.float32) * np.asarray(nd["scale"], np.float32)).astype(np.float32)
        me = len(out)
        out.append({"inverse_world": np.linalg.inv(world), "accumulated_scale": acc, "depth": depth,
                    "parent_index": parent_index, "node": i})
        for c in children[i]:
            if nodes[c]["visible"]:
                walk(c, world, acc, depth + 1, me)

    walk(0, obj_world, np.asarray(scale, np.float32), 0, NO_PARENT)
    return out


def gpu_object_fields(flat, source, object_id, aabb_min, aabb_max, geom_min, geom_max):
    """The GpuObject fields of from_flat_node, as a dict."""
    sdf_type = source["sdf_type"]
    f = {"inverse_world": np.asarray(flat["inverse_world"], np.float32),
         "aabb_min": list(aabb_min), "aabb_max": list(aabb_max), "brick_map_offset": 0,
         "brick_map_dims": [0, 0, 0], "voxel_size": 0.0, "material_id": 0, "sdf_type": sdf_type,
         "sdf_params": [0.0] * 4, "primitive_type": 0,
         "accumulated_scale": list(flat["accumulated_scale"]), "lod_level": 0, "object_id": object_id,
         "geometry_aabb_min": list(geom_min), "geometry_aabb_max": list(geom_max)}
    if sdf_type == 1:
        f.update(material_id=source["material_id"], sdf_params=list(source["params"]),
                 primitive_type=source["primitive_type"])
    elif sdf_type == 2:
        f.update(brick_map_offset=source["brick_map_offset"], brick_map_dims=list(source["brick_map_dims"]),
                 voxel_size=source["voxel_size"])
    f["blend_mode"] = source["blend_mode"]
    f["blend_radius"] = source["blend_radius"] if source["blend_mode"] == 0 else 0.0
    return f
