"""rkf_objects_update: object records replaced with the brick index kept, as
the runtime's per-frame upload_objects needs (render.rs:135-137).  On a
device-voxelized scene (no flat brick map to re-import): analytic objects
added beside the voxelized one, then the voxelized one moved; each march
bit-exact against the oracle reading the same planes and index.  Refused
records change nothing."""
import ctypes as C

import pytest

from conftest import assert_bits_equal
from test_tiled_gpu import PLANES, _analytic

pytestmark = pytest.mark.gpu


def _oracle_scene(oracle, ctx, n_bricks):
    pl = ctx.export_planes(0, n_bricks)
    idx = ctx.export_index()
    objs = [ctx.object(i) for i in range(ctx.info()["num_objects"])]
    return oracle.Scene(objs, top=idx["top"], leaves=idx["leaves"], obj_top_info=idx["obj_top_info"],
                        dist_f16=pl["dist"], mat_plane=pl["mat"], blend_plane=pl["blend"])


def _check(oracle, ctx, n_bricks, cam, p, w, h, what):
    sc = _oracle_scene(oracle, ctx, n_bricks)
    ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
    got = ctx.march(cam, p, w, h, reference_planes=True)
    assert ((ref["flags"] & 1) != 0).sum() > 200, what
    for k in PLANES:
        assert_bits_equal(got[k], ref[k], f"{what}: {k}")
    return got


def test_update_adds_objects_and_moves_the_voxelized_one(oracle, small_scene):
    from rkifield_b200 import _abi as abi, scenes
    from rkifield_b200.engine import Context, RkfError
    spec = small_scene["spec"]
    ctx = Context(pool_capacity=small_scene["vox"].n_bricks + 4096, keep_reference_pool=False)
    try:
        ctx.voxelize(small_scene["prims"], small_scene["vp"])
        n_bricks = ctx.info()["pool_bricks_used"]
        vox = ctx.object(0)
        w, h = 160, 120
        cam = scenes.seeded_camera(spec, w, h, seed=21)
        p = scenes.march_params(spec)
        p.scene.max_distance = 200.0

        extra = [_analytic(0, (14.0, 2.0, 0.0), (2.5,), (2.5, 2.5, 2.5), 5, 2),
                 _analytic(1, (-13.0, 0.0, 3.0), (1.5, 2.0, 1.5), (1.5, 2.0, 1.5), 6, 3),
                 _analytic(2, (0.0, 15.0, -2.0), (1.0, 2.0), (1.0, 3.0, 1.0), 7, 4)]
        ctx.update_objects([vox] + extra, index_source=[0, -1, -1, -1])
        assert ctx.info()["num_objects"] == 4
        _check(oracle, ctx, n_bricks, cam, p, w, h, "with analytic objects")

        # move the voxelized object (translation only: its empty-space path stays)
        moved = ctx.object(0)
        shift = (3.0, -2.0, 1.5)
        for a in range(3):
            moved.inverse_world[12 + a] = vox.inverse_world[12 + a] - shift[a]
            moved.aabb_min[a] = vox.aabb_min[a] + shift[a]
            moved.aabb_max[a] = vox.aabb_max[a] + shift[a]
        ctx.update_objects([moved])
        assert ctx.info()["num_objects"] == 1
        before = _check(oracle, ctx, n_bricks, cam, p, w, h, "moved")

        # refused: an index source that is not a voxelized object, another grid
        arr = (abi.rkf_gpu_object * 1)(moved)
        src = (C.c_int32 * 1)(3)
        assert ctx.lib.rkf_objects_update(ctx.h, arr, 1, src) == abi.RKF_INVALID_ARG
        other = ctx.object(0)
        other.brick_map_dims[0] += 8
        with pytest.raises(RkfError) as e:
            ctx.update_objects([other])
        assert e.value.status == abi.RKF_INVALID_ARG
        after = ctx.march(cam, p, w, h, reference_planes=True)
        for k in PLANES:
            assert_bits_equal(after[k], before[k], f"refused updates changed nothing: {k}")
    finally:
        ctx.close()
