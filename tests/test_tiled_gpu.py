"""Multi-object scenes: the small scene's voxelized object with analytic
primitives around it, marched with the brute strategy (every object at every
step, ray_march.wgsl:776-858) and with the tiled strategy (coarse-field skips
and per-16x16-tile object lists, ray_march.wgsl:874-985), bit-exact against
the oracle's restatement of each."""
import numpy as np
import pytest

from conftest import assert_bits_equal

PLANES = ("t", "normal", "slot", "material", "flags", "position", "packed_material", "motion")


def _analytic(ptype, centre, params, half_extent, mat, oid):
    from rkifield_b200 import _abi as abi
    o = abi.rkf_gpu_object()
    for i in range(4):
        o.inverse_world[i * 4 + i] = 1.0
    for a in range(3):
        o.inverse_world[12 + a] = -float(centre[a])
        o.aabb_min[a] = float(centre[a] - half_extent[a])
        o.aabb_max[a] = float(centre[a] + half_extent[a])
        o.accumulated_scale[a] = 1.0
    o.sdf_type = abi.RKF_SDF_ANALYTICAL
    o.primitive_type = ptype
    for i, v in enumerate(params):
        o.sdf_params[i] = float(v)
    o.material_id = mat
    o.object_id = oid
    return o


def _objects(small_scene):
    return [small_scene["obj"],
            _analytic(0, (27.0, 0.0, 0.0), (3.0,), (3.0, 3.0, 3.0), 5, 2),               # sphere
            _analytic(1, (-26.0, 3.0, 1.0), (2.0, 3.0, 2.0), (2.0, 3.0, 2.0), 6, 3),      # box
            _analytic(2, (2.0, 25.0, -3.0), (1.5, 3.0), (1.5, 4.5, 1.5), 7, 4),           # capsule
            _analytic(0, (60.0, 40.0, -30.0), (2.0,), (2.0, 2.0, 2.0), 8, 5)]             # a lone sphere


def _camera(seed, w, h):
    from rkifield_b200 import scenes
    rng = np.random.default_rng(seed)
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    return scenes.camera_uniforms(70.0 * d, (0.0, 5.0, 0.0), w, h)


def _params(strategy):
    from rkifield_b200 import scenes
    p = scenes.march_params(scenes.SCENE_SMALL)
    p.scene.max_distance = 200.0
    p.strategy = strategy
    return p


def test_oracle_tiled_strategy_behaves(oracle, small_scene):
    """The restatement itself: empty tiles are sky, coarse skips change the
    trajectories (so t differs from the brute march in its low bits), and the
    two strategies agree on which rays hit."""
    from rkifield_b200 import _abi as abi
    v = small_scene["vox"]
    sc = oracle.Scene(_objects(small_scene), pool_words=v.words, brick_maps=v.map)
    w, h = 192, 128
    cam = _camera(3, w, h)
    b = oracle.march(sc, cam, _params(abi.RKF_STRATEGY_BRUTE), w, h)
    t = oracle.march(sc, cam, _params(abi.RKF_STRATEGY_TILED), w, h)
    hb, ht = (b["flags"] & 1) != 0, (t["flags"] & 1) != 0
    assert hb.sum() > 500
    assert (hb == ht).mean() > 0.99
    both = hb & ht
    assert (b["t"][both] != t["t"][both]).any(), "coarse skips should move the sample points"
    # a hit is declared anywhere inside the hit threshold (half a voxel), so
    # different sample points may stop up to that far apart
    assert np.abs(b["t"][both] - t["t"][both]).max() <= 0.5 * 0.04


@pytest.mark.gpu
@pytest.mark.parametrize("strategy", [0, 1], ids=["brute", "tiled"])
@pytest.mark.parametrize("seed", [3, 4])
def test_multi_object_views_bit_exact(oracle, small_scene, strategy, seed):
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    objs = _objects(small_scene)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map)
    ctx = Context(pool_capacity=v.n_bricks + 1024)
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        ctx.upload_objects(objs)
        w, h = 200, 136  # not a multiple of the 16-pixel tiles
        cam = _camera(seed, w, h)
        p = _params(strategy)
        ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
        got = ctx.march(cam, p, w, h, reference_planes=True)
        hit = (ref["flags"] & 1) != 0
        assert hit.sum() > 500
        ids = (ref["packed_material"][hit] >> 24) & 0xFF
        assert len(set(ids.tolist())) >= 2, "the view should see several objects"
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"strategy {strategy} {k}")
        if strategy == 1:
            # the same march through the batched entry point
            from rkifield_b200 import _abi as abi, cudart
            import ctypes as C
            g = cudart.device_gbuffer(w * h, reference_planes=True)
            vw = (abi.rkf_view * 1)()
            vw[0].camera = cam
            vw[0].width, vw[0].height = w, h
            for kk, a in g.items():
                setattr(vw[0].out, kk, a.ptr)
            vw[0].out.mem = abi.RKF_MEM_DEVICE
            abi.check(ctx.lib.rkf_march_batch(ctx.h, vw, 1, None, 0, C.byref(p), None), "batch")
            for kk in ("t", "flags", "slot"):
                assert_bits_equal(g[kk].download(), ref[kk], f"batched tiled {kk}")
    finally:
        ctx.close()


@pytest.mark.gpu
def test_tiled_after_scene_change_bit_exact(oracle, small_scene):
    """The coarse field follows the scene: march, add an object, march again."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    objs = _objects(small_scene)
    ctx = Context(pool_capacity=v.n_bricks + 1024)
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        w, h = 160, 96
        cam = _camera(5, w, h)
        p = _params(abi.RKF_STRATEGY_TILED)
        for k in (3, 5):
            ctx.upload_objects(objs[:k])
            sc = oracle.Scene(objs[:k], pool_words=v.words, brick_maps=v.map)
            ref = oracle.march(sc, cam, p, w, h)
            got = ctx.march(cam, p, w, h)
            for name in ("t", "normal", "slot", "material", "flags"):
                assert_bits_equal(got[name], ref[name], f"{k} objects {name}")
    finally:
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [11, 12])
def test_single_object_tiled_bit_exact(oracle, small_scene, small_ctx, seed):
    """One voxelized object seen from outside its box: the tiled march takes
    coarse-field skips outside the box and EMPTY runs inside it (on the field
    of blocks no coarse skip can reach), bit-exact against the oracle's tiled
    march, which differs from the brute march in the low bits of t."""
    from rkifield_b200 import _abi as abi, scenes
    spec = small_scene["spec"]
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    w, h = 192, 160
    cam = scenes.seeded_camera(spec, w, h, seed=seed)
    p = scenes.march_params(spec)
    p.strategy = abi.RKF_STRATEGY_TILED
    ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
    got = small_ctx.march(cam, p, w, h, reference_planes=True)
    hit = (ref["flags"] & 1) != 0
    assert hit.sum() > 500
    for k in PLANES:
        assert_bits_equal(got[k], ref[k], f"single-object tiled {k}")
    brute = oracle.march(sc, cam, scenes.march_params(spec), w, h)
    assert (brute["t"][hit] != ref["t"][hit]).any(), "the coarse field should move some sample points"


@pytest.mark.gpu
def test_device_coarse_field_equals_oracle(oracle, small_scene):
    """The coarse field the device builds (one thread per cell) is the
    oracle's, which the golden tests pin to coarse_field.rs: same origin,
    dims and binary16 texels."""
    import ctypes as C
    from rkifield_b200 import _abi as abi
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    ctx = Context(pool_capacity=v.n_bricks + 1024)
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        for objs in (_objects(small_scene), [small_scene["obj"]]):
            ctx.upload_objects(objs)
            origin = np.zeros(3, np.float32)
            dims = np.zeros(3, np.uint32)
            n = C.c_uint64()
            abi.check(ctx.lib.rkf_testing_export_coarse(ctx.h, origin.ctypes.data, dims.ctypes.data, None,
                                                        C.byref(n)), "export coarse")
            tex = np.zeros(n.value, np.uint16)
            abi.check(ctx.lib.rkf_testing_export_coarse(ctx.h, origin.ctypes.data, dims.ctypes.data,
                                                        tex.ctypes.data, C.byref(n)), "export coarse")
            o_ref, d_ref, t_ref = oracle.coarse_field(objs)
            assert_bits_equal(origin, o_ref, "coarse origin")
            assert dims.tolist() == d_ref.tolist()
            assert_bits_equal(tex, t_ref, "coarse texels")
    finally:
        ctx.close()
