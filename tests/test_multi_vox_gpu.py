"""The multi-object empty-space path with several voxelized objects: four
objects voxelized on the device from their own seeded primitives and placed
apart by translations, beside four analytic objects.  Each voxelized object
runs EMPTY steps on its own field where the ray lies in one of its EMPTY
cubes and outside the balls of every other object -- analytic primitives'
bounding balls, and for the other voxelized objects the ball of their grid
box, beyond which their sampler returns the distance to that box (above every
EMPTY value).  Whole views from outside and from between the objects, and ray
batches in the three modes, are bit-exact against the oracle under the brute,
tiled and BVH strategies."""
import numpy as np
import pytest

from conftest import assert_bits_equal, oracle_scene_of
from test_tiled_gpu import PLANES, _analytic, _params

pytestmark = pytest.mark.gpu

VARIANT_MULTI_EMPTY, VARIANT_MULTI_EMPTY_TILED = 4, 5
OFFSETS = [(-9.0, 0.0, -9.0), (9.0, 1.0, -8.0), (-8.0, -1.0, 9.0), (10.0, 0.5, 9.5)]


def _moved(o, off, oid):
    """The object translated by off: inverse_world gains -off and the world
    AABB moves (the geometry AABB is in the object's local frame)."""
    from rkifield_b200 import _abi as abi
    m = abi.rkf_gpu_object.from_buffer_copy(o)
    for a in range(3):
        m.inverse_world[12 + a] = float(np.float32(m.inverse_world[12 + a]) - np.float32(off[a]))
        m.aabb_min[a] = float(np.float32(m.aabb_min[a]) + np.float32(off[a]))
        m.aabb_max[a] = float(np.float32(m.aabb_max[a]) + np.float32(off[a]))
    m.object_id = oid
    return m


@pytest.fixture(scope="module")
def four_vox():
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    ctx = Context(pool_capacity=1 << 17, keep_reference_pool=False)
    objs = []
    for i, off in enumerate(OFFSETS):
        spec = scenes.SceneSpec(f"mvox{i}_prims10_cube6m_vs4cm", 10, 6.0, 0.04, seed=40 + i)
        prims = scenes.make_prims(spec)
        idx = ctx.voxelize(prims, scenes.voxelize_params(spec, prims))
        assert idx == i
    for i, off in enumerate(OFFSETS):
        objs.append(_moved(ctx.object(i), off, 10 + i))
    objs += [_analytic(0, (0.0, 0.0, 0.0), (1.5,), (1.5, 1.5, 1.5), 5, 30),            # a sphere among them
             _analytic(1, (0.5, 6.0, -1.0), (1.0, 0.6, 1.2), (1.0, 0.6, 1.2), 6, 31),  # a box above
             _analytic(2, (-2.0, -5.0, 3.0), (0.8, 1.5), (0.8, 2.3, 0.8), 7, 32),     # a capsule below
             _analytic(0, (60.0, 40.0, -30.0), (2.0,), (2.0, 2.0, 2.0), 8, 33)]      # a lone sphere
    ctx.update_objects(objs, [0, 1, 2, 3, -1, -1, -1, -1])
    yield ctx, objs
    ctx.close()


def _cams():
    from rkifield_b200 import scenes
    rng = np.random.default_rng(5)
    out = []
    for k in range(2):  # from outside the group
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        out.append(("outside", scenes.camera_uniforms(45.0 * d, (0.0, 0.0, 0.0), 256, 144)))
    # from between the objects, looking at one of them
    out.append(("between", scenes.camera_uniforms((0.0, 3.5, 0.5), OFFSETS[1], 256, 144)))
    out.append(("between2", scenes.camera_uniforms((1.0, -3.0, 2.0), OFFSETS[2], 256, 144)))
    return out


@pytest.mark.parametrize("strategy", ["brute", "tiled", "bvh"])
def test_four_voxelized_objects_views_bit_exact(oracle, four_vox, strategy):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import engine
    ctx, objs = four_vox
    code = {"brute": abi.RKF_STRATEGY_BRUTE, "tiled": abi.RKF_STRATEGY_TILED, "bvh": abi.RKF_STRATEGY_BVH}[strategy]
    bvh = engine.object_bvh(objs) if strategy == "bvh" else None
    if bvh is not None:
        ctx.upload_bvh(bvh)
    sc = oracle_scene_of(oracle, ctx, bvh=bvh)
    p = _params(code)
    hits_vox = hits_ana = 0
    for name, cam in _cams():
        got = ctx.march(cam, p, 256, 144, reference_planes=True)
        want = VARIANT_MULTI_EMPTY_TILED if strategy == "tiled" else VARIANT_MULTI_EMPTY
        assert ctx.lib.rkf_testing_last_variant(ctx.h) == want, name
        ref = oracle.march(sc, cam, p, 256, 144, with_reference_planes=True)
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"{strategy} {name} {k}")
        hit = (ref["flags"] & 1) != 0
        oid = (ref["packed_material"][hit] >> 24) & 0xFF
        hits_vox += int(((oid >= 10) & (oid < 14)).sum())
        hits_ana += int((oid >= 30).sum())
    assert hits_vox > 1000 and hits_ana > 50, (hits_vox, hits_ana)
    if strategy == "bvh":
        ctx.upload_bvh([])


def test_four_voxelized_objects_rays_bit_exact(oracle, four_vox):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import scenes
    ctx, _ = four_vox
    sc = oracle_scene_of(oracle, ctx)
    rng = np.random.default_rng(21)
    n = 20000
    o = rng.uniform(-16.0, 16.0, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    tmax = rng.uniform(5.0, 60.0, n).astype(np.float32)
    p = _params(abi.RKF_STRATEGY_BRUTE)
    for mode in (abi.RKF_TRACE_CLOSEST, abi.RKF_TRACE_ANY, abi.RKF_TRACE_SHADOW):
        got = ctx.trace(o.ravel(), d.ravel(), tmax, mode, p)
        assert ctx.lib.rkf_testing_last_variant(ctx.h) == VARIANT_MULTI_EMPTY
        ref = oracle.trace(sc, o.ravel(), d.ravel(), tmax, mode, p)
        for k in got:
            assert_bits_equal(got[k], ref[k], f"mode {mode} {k}")
    del scenes
