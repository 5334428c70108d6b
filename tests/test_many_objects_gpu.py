"""Scenes with more objects than the launch parameters hold (32): the
multi-object kernel reads the records from the device table.  The voxelized
small scene beside 39 and 69 analytic primitives (spheres, boxes, capsules
and a plane scattered through and around its grid), views under the brute,
BVH and tiled strategies and ray casts in the three modes, bit-exact with
the oracle; the tiled strategy's object table holds 256 objects and refuses
more."""
import numpy as np
import pytest

from conftest import assert_bits_equal
from test_multi_empty_gpu import _plane
from test_tiled_gpu import PLANES, _analytic, _params
from test_trace_gpu import _rays

pytestmark = pytest.mark.gpu

VARIANT_MULTI = 0


def _objects(small_scene, n_extra, seed):
    rng = np.random.default_rng(seed)
    objs = [small_scene["obj"]]
    for i in range(n_extra - 1):
        c = rng.uniform(-30.0, 30.0, 3)
        kind = i % 3
        if kind == 0:
            r = float(rng.uniform(0.5, 2.5))
            objs.append(_analytic(0, tuple(c), (r,), (r, r, r), 1 + i % 60, 2 + i))
        elif kind == 1:
            b = rng.uniform(0.4, 2.0, 3)
            objs.append(_analytic(1, tuple(c), tuple(b), tuple(b), 1 + i % 60, 2 + i))
        else:
            r, hh = float(rng.uniform(0.3, 1.0)), float(rng.uniform(0.5, 2.0))
            objs.append(_analytic(2, tuple(c), (r, hh), (r, r + hh, r), 1 + i % 60, 2 + i))
    objs.append(_plane((0.0, 1.0, 0.0), (0.0, -20.0, 0.0), 9, 200))
    return objs


def _context(small_scene, objs):
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    ctx = Context(pool_capacity=v.n_bricks + 1024)
    ctx.set_brick_pool(v.words)
    ctx.upload_brick_maps(v.map)
    ctx.upload_objects(objs)
    return ctx


@pytest.mark.parametrize("n_extra", [39, 69, 299])
def test_many_objects_bit_exact(oracle, small_scene, n_extra):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import engine, scenes
    from rkifield_b200.engine import RkfError
    v = small_scene["vox"]
    objs = _objects(small_scene, n_extra, seed=n_extra)
    assert len(objs) == n_extra + 1 > 32
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map, bvh=engine.object_bvh(objs))
    ctx = _context(small_scene, objs)
    try:
        ctx.upload_bvh(engine.object_bvh(objs))
        w, h = 112, 80
        hits = 0
        for strategy in (abi.RKF_STRATEGY_BRUTE, abi.RKF_STRATEGY_BVH, abi.RKF_STRATEGY_TILED):
            p = _params(strategy)
            cam = scenes.camera_uniforms((45.0, 22.0, 55.0), (0.0, -4.0, 0.0), w, h)  # above the plane
            if strategy == abi.RKF_STRATEGY_TILED and len(objs) > 256:
                with pytest.raises(RkfError) as e:
                    ctx.march(cam, p, w, h)
                assert e.value.status == abi.RKF_UNSUPPORTED
                continue
            ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
            got = ctx.march(cam, p, w, h, reference_planes=True)
            assert ctx.lib.rkf_testing_last_variant(ctx.h) == VARIANT_MULTI
            for k in PLANES:
                assert_bits_equal(got[k], ref[k], f"{len(objs)} objects, strategy {strategy}: {k}")
            hits += int((((ref["packed_material"] >> 24) & 0xFF) >= 2).sum())
        assert hits > 100, "the views should see the analytic objects"
        o, d, tmax = _rays(4000, seed=3, box=30.0)
        for mode in (abi.RKF_TRACE_CLOSEST, abi.RKF_TRACE_ANY, abi.RKF_TRACE_SHADOW):
            ref = oracle.trace(sc, o.ravel(), d.ravel(), tmax, mode, _params(0))
            got = ctx.trace(o, d, tmax, mode, _params(0))
            for k in got:
                assert_bits_equal(got[k], ref[k], f"{len(objs)} objects, rays mode {mode}: {k}")
    finally:
        ctx.close()
