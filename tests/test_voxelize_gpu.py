"""GPU voxelizer vs the oracle restatement of voxelize_sdf: identical brick
classification, slot order (z,y,x, lowest slots first) and voxel words."""
import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu


def _all_bricks(dims):
    z, y, x = np.meshgrid(np.arange(dims[2]), np.arange(dims[1]), np.arange(dims[0]), indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], 1).astype(np.uint32)


@pytest.mark.parametrize("rule", [0, 1], ids=["band3", "reference_rule"])
def test_voxelize_matches_oracle(oracle, small_scene, rule):
    from rkifield_b200 import _abi as abi
    from rkifield_b200.engine import Context
    prims = small_scene["prims"]
    vp = small_scene["vp"]
    vp2 = abi.rkf_voxelize_params.from_buffer_copy(bytes(vp))
    vp2.band_rule = rule
    ref = small_scene["vox"] if rule == 0 else oracle.Voxelized(prims, vp2)
    with Context(pool_capacity=ref.n_bricks + 1024) as ctx:
        oi = ctx.voxelize(prims, vp2)
        o = ctx.object(oi)
        assert list(o.brick_map_dims) == list(map(int, ref.dims))
        slots = ctx.brick_lookup(oi, _all_bricks(ref.dims))
        assert_bits_equal(slots, ref.map, "brick map")
        words = ctx.export_pool(0, ref.n_bricks)
        assert_bits_equal(words, ref.words, "voxel words")
        ro = ref.gpu_object()
        for f in ("geometry_aabb_min", "geometry_aabb_max", "aabb_min", "aabb_max"):
            assert list(getattr(o, f)) == list(getattr(ro, f)), f
        assert ctx.info()["pool_bricks_used"] == ref.n_bricks


def test_voxelized_scene_marches_like_imported(oracle, small_scene, small_ctx):
    """A scene built on the device marches bit-identically to the same scene
    imported through the reference upload path."""
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    spec = small_scene["spec"]
    cam = scenes.seeded_camera(spec, 128, 128, seed=3)
    p = scenes.march_params(spec)
    a = small_ctx.march(cam, p, 128, 128)
    with Context(pool_capacity=small_scene["vox"].n_bricks + 1024) as ctx:
        ctx.voxelize(small_scene["prims"], small_scene["vp"])
        b = ctx.march(cam, p, 128, 128)
        c = ctx.march(cam, p, 128, 128, plain=True)
    for k in a:
        assert_bits_equal(b[k], a[k], k)
        assert_bits_equal(c[k], a[k], "plain " + k)
