"""Object records made by transform flattening feed the march: an object's
node tree (rotated and non-uniformly scaled groups, analytic primitives, an
invisible subtree) is flattened with rkf_flatten_object, turned into records
with rkf_gpu_object_from_flat_node (the runtime's per-frame path,
render.rs:79-104 of the runtime crate), imported beside the voxelized small
scene, and the view is bit-exact against the oracle on the same records."""
import math

import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

PLANES = ("t", "normal", "slot", "material", "flags", "position", "packed_material", "motion")


def _quat(axis, angle):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    s = math.sin(angle / 2)
    return (float(a[0] * s), float(a[1] * s), float(a[2] * s), math.cos(angle / 2))


def _flattened_records():
    from rkifield_b200 import _abi as abi
    from rkifield_b200.engine import flatten_object, gpu_object_from_flat_node, scene_node
    NO, AN = abi.RKF_NO_PARENT, abi.RKF_SDF_ANALYTICAL
    nodes = [
        scene_node(NO),                                                                   # 0 group
        scene_node(0, sdf_type=AN, primitive_type=abi.RKF_PRIM_SPHERE, params=(2.5, 0, 0, 0),
                   material_id=100, position=(0.0, 8.0, 0.0)),                              # 1 sphere
        scene_node(0, rotation=_quat((0, 1, 1), 0.7), scale=(1.0, 1.5, 0.75),
                   position=(-6.0, 2.0, 3.0)),                                            # 2 group
        scene_node(2, sdf_type=AN, primitive_type=abi.RKF_PRIM_BOX, params=(1.5, 1.0, 2.0, 0),
                   material_id=101, rotation=_quat((1, 0, 0), 0.4)),                        # 3 box
        scene_node(2, sdf_type=AN, primitive_type=abi.RKF_PRIM_CAPSULE, params=(0.6, 1.8, 0, 0),
                   material_id=102, position=(0.0, 0.0, 4.0), blend_mode=abi.RKF_BLEND_UNION),  # 4 capsule
        scene_node(0, visible=False, sdf_type=AN, primitive_type=abi.RKF_PRIM_TORUS,
                   params=(3.0, 0.5, 0, 0), material_id=103),                               # 5 hidden torus
        scene_node(5, sdf_type=AN, primitive_type=abi.RKF_PRIM_SPHERE, params=(9.0, 0, 0, 0),
                   material_id=104),                                                        # 6 under it
    ]
    pos = (20.0, 4.0, -6.0)
    flat = flatten_object(nodes, rotation=_quat((0, 0, 1), 0.3), scale=(1.2, 1.2, 1.2), position=pos)
    assert [f.node for f in flat] == [0, 1, 2, 3, 4]
    lo = [pos[0] - 20.0, pos[1] - 20.0, pos[2] - 20.0, 0.0]
    hi = [pos[0] + 20.0, pos[1] + 20.0, pos[2] + 20.0, 0.0]
    return [gpu_object_from_flat_node(f, nodes[f.node], 3, lo, hi) for f in flat]


def test_flattened_objects_march_bit_exact(oracle, small_scene):
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    objs = [small_scene["obj"]] + _flattened_records()
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map)
    ctx = Context(pool_capacity=v.n_bricks + 1024)
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        ctx.upload_objects(objs)
        p = scenes.march_params(scenes.SCENE_SMALL)
        p.scene.max_distance = 200.0
        w, h = 200, 136
        seen = set()
        for eye, target in (((45.0, 18.0, 30.0), (16.0, 6.0, -4.0)), ((0.0, 40.0, 60.0), (8.0, 0.0, 0.0))):
            cam = scenes.camera_uniforms(eye, target, w, h)
            ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
            got = ctx.march(cam, p, w, h, reference_planes=True)
            for k in PLANES:
                assert_bits_equal(got[k], ref[k], f"eye {eye}: {k}")
            hit = (ref["flags"] & 1) != 0
            seen |= set(ref["material"][hit].tolist())
        # the flattened primitives are in view (materials 100-102; the voxelized
        # scene's are below 64); the hidden subtree (103, 104) is not there
        assert {100, 101, 102} <= seen, sorted(seen)
        assert not ({103, 104} & seen)
    finally:
        ctx.close()
