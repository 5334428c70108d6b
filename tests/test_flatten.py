"""Transform flattening and object records (host only): rkf_flatten_object and
rkf_gpu_object_from_flat_node against the reference's own tests
(transform_flatten.rs:120-420, gpu_object.rs:322-470, ported with their
tolerances) and against an independent FP64 restatement
(oracle/flatten_ref.py) on seeded random trees."""
import math

import numpy as np
import pytest

from rkifield_b200 import _abi as abi
from rkifield_b200.engine import RkfError, flatten_object, gpu_object_from_flat_node, scene_node

NO = abi.RKF_NO_PARENT


def _mat(flat):
    return np.array(list(flat.inverse_world), np.float64).reshape(4, 4).T  # column-major


def _apply(m, p):
    return (m @ np.array([p[0], p[1], p[2], 1.0]))[:3]


def _sphere(parent, radius=0.1, material=1, **kw):
    return scene_node(parent, sdf_type=abi.RKF_SDF_ANALYTICAL, primitive_type=0, params=(radius, 0, 0, 0),
                      material_id=material, **kw)


# --- transform_flatten.rs tests ----------------------------------------------

def test_identity_transform_single_node():
    flat = flatten_object([_sphere(NO, 0.5)])
    assert len(flat) == 1
    assert np.abs(np.array(list(flat[0].accumulated_scale)) - 1.0).max() < 1e-6
    assert flat[0].depth == 0 and flat[0].parent_index == NO and flat[0].node == 0
    assert np.linalg.norm(_apply(_mat(flat[0]), (1, 2, 3)) - (1, 2, 3)) < 1e-4


def test_nested_transforms_propagate():
    nodes = [scene_node(NO), _sphere(0, position=(2.0, 0.0, 0.0))]
    flat = flatten_object(nodes)
    assert len(flat) == 2 and flat[1].node == 1
    assert flat[1].depth == 1 and flat[1].parent_index == 0
    world = np.linalg.inv(_mat(flat[1]))
    assert np.linalg.norm(_apply(world, (0, 0, 0)) - (2, 0, 0)) < 1e-4


def test_scale_accumulation():
    nodes = [scene_node(NO), scene_node(0, scale=(0.5, 0.5, 0.5))]
    flat = flatten_object(nodes, scale=(2.0, 2.0, 2.0))
    assert np.abs(np.array(list(flat[0].accumulated_scale)) - 2.0).max() < 1e-6
    assert np.abs(np.array(list(flat[1].accumulated_scale)) - 1.0).max() < 1e-6


def test_deep_scale_accumulation():
    nodes = [scene_node(NO), scene_node(0, scale=(3.0,) * 3), scene_node(1, scale=(0.5,) * 3)]
    flat = flatten_object(nodes, scale=(2.0, 2.0, 2.0))
    assert len(flat) == 3
    for f, want in zip(flat, (2.0, 6.0, 3.0)):
        assert np.abs(np.array(list(f.accumulated_scale)) - want).max() < 1e-6


def test_inverse_world_correctness():
    nodes = [scene_node(NO), _sphere(0, position=(3.0, 0.0, 0.0))]
    flat = flatten_object(nodes, position=(5.0, 0.0, 0.0))
    assert np.linalg.norm(_apply(_mat(flat[1]), (8, 0, 0))) < 1e-3


def test_camera_relative_precision():
    flat = flatten_object([_sphere(NO)], position=(1.0, 0.0, 0.0))
    assert np.linalg.norm(_apply(_mat(flat[0]), (1, 0, 0))) < 1e-3


def test_rotation_propagation():
    h = math.sin(math.pi / 4)
    nodes = [scene_node(NO), _sphere(0, position=(1.0, 0.0, 0.0))]
    flat = flatten_object(nodes, rotation=(0.0, 0.0, h, h))  # 90 degrees about z
    world = _apply(np.linalg.inv(_mat(flat[1])), (0, 0, 0))
    assert abs(world[0]) < 1e-3 and abs(world[1] - 1.0) < 1e-3


def test_invisible_children_skipped():
    nodes = [scene_node(NO), _sphere(0), _sphere(0, visible=False), _sphere(2)]  # the last under the invisible
    flat = flatten_object(nodes)
    assert [f.node for f in flat] == [0, 1]


def test_depth_first_order_and_parent_indices():
    # root -> [A -> [C], B], as the reference builds it
    nodes = [scene_node(NO), scene_node(0), scene_node(1), scene_node(0)]
    flat = flatten_object(nodes)
    assert [f.node for f in flat] == [0, 1, 2, 3]  # root, A, C, B
    assert [f.parent_index for f in flat] == [NO, 0, 1, 0]
    assert [f.depth for f in flat] == [0, 1, 2, 1]


def test_blend_modes_and_sources_preserved():
    nodes = [scene_node(NO), _sphere(0, 0.5, 42, blend_mode=abi.RKF_BLEND_SUBTRACT)]
    flat = flatten_object(nodes)
    g0 = gpu_object_from_flat_node(flat[0], nodes[flat[0].node], 1)
    g1 = gpu_object_from_flat_node(flat[1], nodes[flat[1].node], 1)
    assert g0.sdf_type == abi.RKF_SDF_NONE and g0.blend_mode == abi.RKF_BLEND_SMOOTH_UNION
    assert abs(g0.blend_radius - 0.1) < 1e-6
    assert g1.sdf_type == abi.RKF_SDF_ANALYTICAL and g1.blend_mode == abi.RKF_BLEND_SUBTRACT
    assert abs(g1.sdf_params[0] - 0.5) < 1e-6 and g1.material_id == 42 and g1.blend_radius == 0.0


# --- gpu_object.rs tests ------------------------------------------------------

def _flat_identity(scale=1.0, depth=0, parent=NO):
    f = abi.rkf_flat_node()
    f.inverse_world[:] = [1.0 if i % 5 == 0 else 0.0 for i in range(16)]
    f.accumulated_scale[:] = [scale] * 3
    f.depth, f.parent_index = depth, parent
    return f


def test_from_flat_node_analytical():
    src = _sphere(NO, 0.5, 3, blend_mode=abi.RKF_BLEND_SMOOTH_UNION, blend_radius=0.1)
    g = gpu_object_from_flat_node(_flat_identity(1.5), src, 42, (-0.5, -0.5, -0.5, 0.0), (0.5, 0.5, 0.5, 0.0))
    assert g.object_id == 42 and g.sdf_type == abi.RKF_SDF_ANALYTICAL and g.material_id == 3
    assert abs(g.sdf_params[0] - 0.5) < 1e-6 and abs(g.blend_radius - 0.1) < 1e-6
    assert g.blend_mode == abi.RKF_BLEND_SMOOTH_UNION and abs(g.accumulated_scale[0] - 1.5) < 1e-6
    assert list(g.aabb_min) == [-0.5, -0.5, -0.5, 0.0] and g.lod_level == 0


def test_from_flat_node_voxelized():
    src = scene_node(NO, sdf_type=abi.RKF_SDF_VOXELIZED, brick_map_offset=100, brick_map_dims=(8, 8, 8),
                     voxel_size=0.02, blend_mode=abi.RKF_BLEND_UNION)
    g = gpu_object_from_flat_node(_flat_identity(depth=1, parent=0), src, 7, (-1, -1, -1, 0), (1, 1, 1, 0))
    assert g.sdf_type == abi.RKF_SDF_VOXELIZED and g.brick_map_offset == 100
    assert list(g.brick_map_dims) == [8, 8, 8] and abs(g.voxel_size - 0.02) < 1e-6
    assert g.blend_mode == abi.RKF_BLEND_UNION and g.material_id == 0 and g.primitive_type == 0


def test_from_flat_node_none():
    g = gpu_object_from_flat_node(_flat_identity(), scene_node(NO, blend_mode=abi.RKF_BLEND_SUBTRACT), 1)
    assert g.sdf_type == abi.RKF_SDF_NONE and g.blend_mode == abi.RKF_BLEND_SUBTRACT


@pytest.mark.parametrize("prim,params", [(0, (1.5, 0, 0, 0)), (1, (1.0, 2.0, 3.0, 0)), (2, (0.5, 1.0, 0, 0)),
                                         (3, (1.0, 0.3, 0, 0)), (4, (0.5, 2.0, 0, 0)), (5, (0.0, 1.0, 0.0, 5.0))])
def test_primitive_params_all_types(prim, params):
    src = scene_node(NO, sdf_type=abi.RKF_SDF_ANALYTICAL, primitive_type=prim, params=params)
    g = gpu_object_from_flat_node(_flat_identity(), src, 0)
    assert g.primitive_type == prim and np.allclose(list(g.sdf_params), params, atol=1e-6)


@pytest.mark.parametrize("mode,radius,want", [(0, 0.2, 0.2), (1, 0.2, 0.0), (2, 0.2, 0.0), (3, 0.2, 0.0)])
def test_blend_mode_encoding(mode, radius, want):
    g = gpu_object_from_flat_node(_flat_identity(), scene_node(NO, blend_mode=mode, blend_radius=radius), 0)
    assert g.blend_mode == mode and abs(g.blend_radius - want) < 1e-6


# --- refusals -------------------------------------------------------------------

def test_refusals():
    with pytest.raises(RkfError):  # the root must come first
        flatten_object([scene_node(0)])
    with pytest.raises(RkfError):  # a parent after its child
        flatten_object([scene_node(NO), scene_node(2), scene_node(0)])
    with pytest.raises(RkfError):  # not pre-order: node 3's parent 1 is no longer on the path
        flatten_object([scene_node(NO), scene_node(0), scene_node(0), scene_node(1)])
    with pytest.raises(RkfError):  # two roots
        flatten_object([scene_node(NO), scene_node(NO)])
    with pytest.raises(RkfError):  # a zero scale makes the world matrix singular
        flatten_object([scene_node(NO), scene_node(0, scale=(1.0, 0.0, 1.0))])
    with pytest.raises(RkfError):
        gpu_object_from_flat_node(_flat_identity(), scene_node(NO, sdf_type=7), 0)
    with pytest.raises(RkfError):
        gpu_object_from_flat_node(_flat_identity(), scene_node(NO, blend_mode=4), 0)


# --- random trees against the FP64 restatement -------------------------------------

def _random_tree(rng, n):
    """A pre-order tree of n nodes: each node's parent is a node on the path
    from the root to the previous node."""
    specs, path = [], []
    for i in range(n):
        if i == 0:
            parent = NO
        else:
            path = path[:rng.integers(1, len(path) + 1)]
            parent = path[-1]
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        sc = rng.uniform(0.3, 3.0, 3) if rng.random() < 0.7 else np.full(3, rng.uniform(0.3, 3.0))
        specs.append({"parent": parent, "position": rng.uniform(-20, 20, 3).astype(np.float32),
                      "rotation": q.astype(np.float32), "scale": sc.astype(np.float32),
                      "visible": bool(i == 0 or rng.random() < 0.85)})
        path.append(i)
    return specs


def test_random_trees_match_fp64_restatement():
    from oracle import flatten_ref
    rng = np.random.default_rng(2024)
    for trial in range(60):
        specs = _random_tree(rng, int(rng.integers(1, 24)))
        q = rng.normal(size=4)
        q = (q / np.linalg.norm(q)).astype(np.float32)
        osc = rng.uniform(0.5, 2.0, 3).astype(np.float32)
        pos = rng.uniform(-500, 500, 3).astype(np.float32)
        nodes = [scene_node(s["parent"], s["position"], s["rotation"], s["scale"], s["visible"]) for s in specs]
        got = flatten_object(nodes, q, osc, pos)
        ref = flatten_ref.flatten_object(specs, q, osc, pos)
        assert [(f.node, f.parent_index, f.depth) for f in got] == \
               [(r["node"], r["parent_index"], r["depth"]) for r in ref], f"trial {trial}"
        for f, r in zip(got, ref):
            # f32 scale products: the same bits
            assert np.array_equal(np.array(list(f.accumulated_scale), np.float32), r["accumulated_scale"])
            # inverse rounded once from FP64: within an f32 rounding of each entry,
            # relative to the matrix's scale
            want = r["inverse_world"]
            tol = 4 * np.finfo(np.float32).eps * np.abs(want).max()
            assert np.abs(_mat(f) - want).max() <= tol, f"trial {trial} node {f.node}"


def test_records_match_restatement():
    from oracle import flatten_ref
    rng = np.random.default_rng(7)
    nodes = [scene_node(NO, blend_mode=abi.RKF_BLEND_UNION),
             _sphere(0, 0.25, 9, position=(1, 2, 3), blend_mode=abi.RKF_BLEND_SMOOTH_UNION, blend_radius=0.3),
             scene_node(0, sdf_type=abi.RKF_SDF_VOXELIZED, brick_map_offset=77, brick_map_dims=(4, 5, 6),
                        voxel_size=0.04, blend_mode=abi.RKF_BLEND_INTERSECT, blend_radius=0.5)]
    flat = flatten_object(nodes, position=(10.0, 0.0, -4.0))
    for f in flat:
        src = nodes[f.node]
        lo, hi = rng.uniform(-5, 0, 4).astype(np.float32), rng.uniform(0, 5, 4).astype(np.float32)
        glo, ghi = rng.uniform(-1, 0, 3).astype(np.float32), rng.uniform(0, 1, 3).astype(np.float32)
        g = gpu_object_from_flat_node(f, src, 5, lo, hi, glo, ghi)
        want = flatten_ref.gpu_object_fields(
            {"inverse_world": list(f.inverse_world), "accumulated_scale": list(f.accumulated_scale)},
            {k: (list(getattr(src, k)) if hasattr(getattr(src, k), "__len__") else getattr(src, k))
             for k, _ in abi.rkf_scene_node._fields_}, 5, lo, hi, glo, ghi)
        for k, v in want.items():
            got = getattr(g, k)
            got = list(got) if hasattr(got, "__len__") else got
            assert np.array_equal(np.asarray(got, np.float64).ravel(), np.asarray(v, np.float64).ravel()), k
