"""Pin the voxelizer restatement (and the GPU voxelizer and march) to output
of the reference itself: scenes/test_cross.rkf, the reference voxelize_sdf's
voxelization of five smooth-unioned spheres (gen_test_rkf.rs), decoded into
tests/golden/test_cross_rkf.npz by tests/golden/make_rkf_fixture.py."""
import os

import numpy as np
import pytest

from conftest import assert_bits_equal

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "test_cross_rkf.npz")


def fixture():
    return dict(np.load(FIX))


def cross_prims_and_params(f):
    from rkifield_b200 import _abi as abi
    n = len(f["sphere_radii"])
    prims = np.zeros(n, abi.PRIM_DTYPE)
    prims["type"] = 0
    prims["material"] = int(f["material"])
    prims["centre"] = f["sphere_centres"]
    prims["params"][:, 0] = f["sphere_radii"]
    prims["rot"] = np.eye(3, dtype=np.float32).ravel()
    prims["bound_radius"] = f["sphere_radii"]
    vs = np.float32(f["voxel_size"])
    margin = vs * np.float32(4.0)  # gen_test_rkf.rs:41-47
    lo = np.full(3, np.finfo(np.float32).max, np.float32)
    hi = np.full(3, -np.finfo(np.float32).max, np.float32)
    for c, r in zip(f["sphere_centres"], f["sphere_radii"]):
        e = np.float32(r) + margin
        lo = np.minimum(lo, c - e)
        hi = np.maximum(hi, c + e)
    vp = abi.rkf_voxelize_params()
    vp.voxel_size = float(vs)
    vp.smooth_k = float(f["smooth_k"])
    vp.band_voxels = 3.0
    vp.cut_distance = 1e30
    vp.aabb_min[:] = [float(x) for x in lo]
    vp.aabb_max[:] = [float(x) for x in hi]
    vp.band_rule = abi.RKF_BAND_REFERENCE
    vp.object_id = 1
    return prims, vp


def test_fixture_matches_reference_file_when_present():
    """The committed fixture equals the reference's own scenes/test_cross.rkf
    when a checkout of the reference is named by RKF_REFERENCE_ROOT."""
    root = os.environ.get("RKF_REFERENCE_ROOT", "")
    path = os.path.join(root, "scenes", "test_cross.rkf") if root else ""
    if not path or not os.path.exists(path):
        pytest.skip("no reference checkout (set RKF_REFERENCE_ROOT)")
    from rkifield_b200.rkf_asset import read_rkf
    lod = read_rkf(path).lods[-1]
    f = fixture()
    assert_bits_equal(lod.brick_map, f["brick_map"], "brick map")
    assert_bits_equal(lod.words, f["words"], "words")


def test_oracle_voxelizer_reproduces_reference_output(oracle):
    """voxelize_sdf restated: same bricks, same slot order, same f16 words as
    the reference wrote."""
    f = fixture()
    prims, vp = cross_prims_and_params(f)
    v = oracle.Voxelized(prims, vp)
    assert list(v.dims) == list(f["dims"])
    assert_bits_equal(v.map, f["brick_map"], "brick map")
    assert_bits_equal(v.words, f["words"], "VoxelSample words")


@pytest.mark.gpu
def test_gpu_voxelizer_and_march_on_reference_pool(oracle):
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    f = fixture()
    prims, vp = cross_prims_and_params(f)
    dims = f["dims"]
    with Context(pool_capacity=4096) as ctx:
        oi = ctx.voxelize(prims, vp)
        z, y, x = np.meshgrid(np.arange(dims[2]), np.arange(dims[1]), np.arange(dims[0]), indexing="ij")
        bxyz = np.stack([x.ravel(), y.ravel(), z.ravel()], 1).astype(np.uint32)
        assert_bits_equal(ctx.brick_lookup(oi, bxyz.ravel()), f["brick_map"], "GPU brick map")
        assert_bits_equal(ctx.export_pool(0, len(f["words"]) // 1024), f["words"], "GPU words")
    # march the reference's pool imported through the reference upload path
    from oracle.binding import Scene, march
    obj = None
    with Context(pool_capacity=4096) as ctx:
        ctx.set_brick_pool(f["words"])
        ctx.upload_brick_maps(f["brick_map"])
        from oracle.binding import Voxelized
        v = Voxelized(prims, vp)
        obj = v.gpu_object()
        ctx.upload_objects([obj])
        spec = scenes.SceneSpec("test_cross", 5, 2.0, float(f["voxel_size"]), max_steps=128)
        for seed in (1, 2, 3):
            cam = scenes.seeded_camera(spec, 200, 150, seed=seed, distance=2.5)
            p = scenes.march_params(spec)
            ref = march(Scene([obj], pool_words=f["words"], brick_maps=f["brick_map"]), cam, p, 200, 150,
                        with_reference_planes=True)
            assert (ref["flags"] & 1).sum() > 500
            for plain in (False, True):
                got = ctx.march(cam, p, 200, 150, reference_planes=True, plain=plain)
                for k in ("t", "normal", "slot", "material", "flags", "position", "packed_material", "motion"):
                    assert_bits_equal(got[k], ref[k], f"{k} plain={plain} seed={seed}")
