"""The full-size workload: 512 seeded primitives in a 256 m cube voxelized at
2 cm on the device (about 1.1 M bricks), one view from inside the grid at
1920x1080 and 960x540.  Whole frames are compared bit for bit with the FP32
oracle reading the same pool planes and index, and a repeat of the march is
identical.  Ray batches whose tmax falls around the distance a ray covers in
its step budget exercise both ways a miss can end (out of steps, or past tmax)
where the march settles rays without stepping them."""
import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

PLANES = ("t", "normal", "slot", "material", "flags", "position", "packed_material", "motion")
W, H = 1920, 1080


@pytest.mark.parametrize("w,h", [(1920, 1080), (960, 540)], ids=["1080p", "540p"])
def test_large_view_full_frame_bit_exact(oracle, large, large_oracle, w, h):
    """The headline view at both sizes, every pixel, every output plane,
    against the FP32 oracle (all host threads) on the same planes and index."""
    from rkifield_b200 import scenes
    ctx, spec, _, p = large
    cam = scenes.seeded_camera(spec, w, h, seed=100, inside=True, distance=spec.cube * 0.18)
    got = ctx.march(cam, p, w, h, reference_planes=True)
    ref = oracle.march(large_oracle, cam, p, w, h, with_reference_planes=True)
    for k in PLANES:
        assert_bits_equal(got[k], ref[k], f"{w}x{h} {k}")
    flags = ref["flags"]
    assert (flags & 1).sum() > 0.01 * w * h, "the view should hit geometry"
    assert (flags & 4).sum() > 0.5 * w * h, "most rays should run out of steps in empty space"
    # heaviest tiles first, one launch and in three bands of host outputs;
    # warp-shared EMPTY runs in the launch's tail (with 32, every warp that
    # has no work left shares)
    from rkifield_b200 import _abi as abi
    tu0 = ctx.tuning()
    try:
        for order, share, bands in ((1, 0, 1), (1, 0, 3), (1, 4, 1), (0, 32, 3), (1, 32, 1)):
            tu = abi.rkf_batch_tuning.from_buffer_copy(tu0)
            tu.order_tiles, tu.tail_share = order, share
            ctx.set_tuning(tu)
            ctx.lib.rkf_testing_set_host_bands(bands)
            got = ctx.march(cam, p, w, h, reference_planes=True)
            for k in PLANES:
                assert_bits_equal(got[k], ref[k], f"{w}x{h} order {order} tail share {share}, {bands} bands, {k}")
    finally:
        ctx.lib.rkf_testing_set_host_bands(-1)
        ctx.set_tuning(tu0)


def test_large_view_repeat_identical(large):
    ctx, spec, cam, p = large
    a = ctx.march(cam, p, W, H)
    b = ctx.march(cam, p, W, H)
    for k in a:
        assert_bits_equal(a[k], b[k], k)
    flags = a["flags"]
    # most rays run out of steps in empty space; some hit
    assert (flags & 1).sum() > 10_000


def test_large_rays_around_the_step_budget_bit_exact(oracle, large, large_oracle):
    """Rays from inside the cube with tmax near the distance 1024 steps of
    EMPTY space cover (about 164 m): some run out of steps, some pass tmax,
    some are too close to call and are stepped; shadow rays with long tmax."""
    from rkifield_b200 import _abi as abi
    ctx, spec, cam, p = large
    rng = np.random.default_rng(12)
    n = 6000
    o = rng.uniform(-60.0, 60.0, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    span = np.float32(1024 * 8 * spec.voxel_size)
    tmax = (span * rng.uniform(0.97, 1.03, n)).astype(np.float32)
    tmax[:200] = span  # on the boundary itself
    tu0 = ctx.tuning()
    for mode in (abi.RKF_TRACE_CLOSEST, abi.RKF_TRACE_ANY, abi.RKF_TRACE_SHADOW):
        ref = oracle.trace(large_oracle, o.ravel(), d.ravel(), tmax, mode, p)
        got = ctx.trace(o.ravel(), d.ravel(), tmax, mode, p)
        for k in ("t", "flags"):
            assert_bits_equal(got[k], ref[k], f"mode {mode} {k}")
        # every warp that has no work left takes its lanes' EMPTY runs together
        tu = abi.rkf_batch_tuning.from_buffer_copy(tu0)
        tu.tail_share = 32
        try:
            ctx.set_tuning(tu)
            got = ctx.trace(o.ravel(), d.ravel(), tmax, mode, p)
        finally:
            ctx.set_tuning(tu0)
        for k in ("t", "flags"):
            assert_bits_equal(got[k], ref[k], f"mode {mode} tail share {k}")
        if mode == abi.RKF_TRACE_CLOSEST:
            steps_out = (ref["flags"] & 4) != 0
            assert steps_out.sum() > 200 and (ref["flags"] == 0).sum() > 200, "both miss endings must occur"


def test_large_view_tiled_rows_bit_exact(oracle, large, large_oracle):
    """The tiled strategy on the single-object scene (EMPTY runs on the field
    of blocks no coarse skip can reach, tiled steps elsewhere): sampled rows
    bit-exact against the oracle's tiled march."""
    from rkifield_b200 import _abi as abi, scenes
    ctx, spec, cam, _ = large
    p = scenes.march_params(spec)
    p.strategy = abi.RKF_STRATEGY_TILED
    got = ctx.march(cam, p, W, H, reference_planes=True)
    for r in (0, 389, 541, 1079):
        ref = oracle.march(large_oracle, cam, p, W, H, rows=(r, r + 1), with_reference_planes=True)
        for k in PLANES:
            assert_bits_equal(got[k].reshape(H, -1)[r], ref[k].reshape(1, -1)[0], f"tiled row {r} {k}")


def test_large_view_with_analytic_objects_rows_bit_exact(oracle, large):
    """The multi-object empty-space path at full size: analytic objects in
    front of the camera (spheres, a rotated and scaled box), one far away and
    a ground plane below the cube, beside the voxelized object; EMPTY runs and
    settling chains stop at each object's ball or the plane's half-space.  The whole frame (brute strategy) and sampled rows (tiled
    strategy) bit-exact against the oracle reading the same planes and index.
    The scene is restored afterwards."""
    from test_multi_empty_gpu import _rotation, _transformed
    from test_tiled_gpu import _analytic
    ctx, spec, cam, p = large
    vox = ctx.object(0)
    pos = np.array(cam.position[:3], np.float64)
    fwd = np.array(cam.forward[:3], np.float64)
    right = np.array(cam.right[:3], np.float64)
    up = np.array(cam.up[:3], np.float64)
    fwd, right, up = (v / np.linalg.norm(v) for v in (fwd, right, up))
    props = []
    for i, (dist, x, y, r) in enumerate([(12, -3, 1, 1.0), (25, 4, -2, 2.0), (40, 0, 0, 3.0), (60, -10, 5, 2.5),
                                         (90, 12, -6, 4.0)]):
        c = pos + fwd * dist + right * x + up * y
        props.append(_analytic(0, tuple(float(v) for v in c), (r,), (r, r, r), 5, 10 + i))
    c = pos + fwd * 30 + right * 8
    props.append(_transformed(1, tuple(float(v) for v in c), (2.0, 1.0, 1.5), _rotation((1, 2, 3), 0.7),
                              (1.5, 0.7, 1.2), 7, 20))
    props.append(_analytic(0, (0.0, 0.0, 500.0), (1.0,), (1.0, 1.0, 1.0), 5, 21))
    # a ground plane just below the cube: the runs stop at its half-space
    from test_multi_empty_gpu import _plane
    props.append(_plane((0.0, 1.0, 0.0), (0.0, -spec.cube * 0.5 - 1.0, 0.0), 9, 22))
    try:
        ctx.update_objects([vox] + props, [0] + [-1] * len(props))
        n = ctx.info()["pool_bricks_used"]
        pl = ctx.export_planes(0, n)
        idx = ctx.export_index()
        objs = [ctx.object(i) for i in range(ctx.info()["num_objects"])]
        sc = oracle.Scene(objs, top=idx["top"], leaves=idx["leaves"], obj_top_info=idx["obj_top_info"],
                          dist_f16=pl["dist"], mat_plane=pl["mat"], blend_plane=pl["blend"])
        got = ctx.march(cam, p, W, H, reference_planes=True)
        assert ctx.lib.rkf_testing_last_variant(ctx.h) == 4
        ref = oracle.march(sc, cam, p, W, H, with_reference_planes=True)
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"with objects, full frame {k}")
        hit = (ref["flags"] & 1) != 0
        prop_hits = int((((ref["packed_material"][hit] >> 24) & 0xFF) >= 10).sum())
        assert prop_hits > 0, "the view should see the analytic objects"
        # the same under the tiled strategy (EMPTY runs on the tiled empty-space field)
        from rkifield_b200 import _abi as abi, scenes
        pt = scenes.march_params(spec)
        pt.strategy = abi.RKF_STRATEGY_TILED
        got = ctx.march(cam, pt, W, H, reference_planes=True)
        assert ctx.lib.rkf_testing_last_variant(ctx.h) == 5
        for r in (0, 480, 541, 1079):
            ref = oracle.march(sc, cam, pt, W, H, rows=(r, r + 1), with_reference_planes=True)
            for k in PLANES:
                assert_bits_equal(got[k].reshape(H, -1)[r], ref[k].reshape(1, -1)[0], f"tiled, row {r} {k}")
    finally:
        ctx.update_objects([vox])


def test_large_view_with_voxelized_props_bit_exact(oracle, large):
    """Several voxelized objects at full size: the 1.1 M-brick object plus
    three small voxelized objects and two analytic ones in front of the
    camera (the multi-object empty-space path: EMPTY runs on each voxelized
    object's own field, outside every other object's ball).  The whole
    1920x1080 frame bit-exact against the oracle (brute strategy) and sampled
    rows under the tiled strategy.  Own context: the shared scene is not
    touched."""
    from test_multi_vox_gpu import _moved
    from test_tiled_gpu import _analytic
    from rkifield_b200 import _abi as abi, scenes
    from rkifield_b200.engine import Context
    from conftest import oracle_scene_of
    _, spec, cam, p = large
    prims = scenes.make_prims(spec)
    ctx = Context(pool_capacity=1_300_000, keep_reference_pool=False)
    try:
        ctx.voxelize(prims, scenes.voxelize_params(spec, prims))
        pos = np.array(cam.position[:3], np.float64)
        fwd, right, up = (np.array(v[:3], np.float64) for v in (cam.forward, cam.right, cam.up))
        fwd, right, up = (v / np.linalg.norm(v) for v in (fwd, right, up))
        objs = [ctx.object(0)]
        for i, (dist, x, y) in enumerate([(14.0, -4.0, 1.0), (30.0, 6.0, -2.0), (55.0, -9.0, 3.0)]):
            s2 = scenes.SceneSpec(f"prop{i}_prims8_cube4m_vs2cm", 8, 4.0, 0.02, seed=70 + i)
            pr = scenes.make_prims(s2)
            assert ctx.voxelize(pr, scenes.voxelize_params(s2, pr)) == i + 1
            objs.append(_moved(ctx.object(i + 1), pos + fwd * dist + right * x + up * y, 40 + i))
        objs.append(_analytic(0, tuple(float(v) for v in pos + fwd * 20 + right * 5), (1.5,), (1.5, 1.5, 1.5), 5, 50))
        objs.append(_analytic(1, tuple(float(v) for v in pos + fwd * 40 - up * 4), (2.0, 1.0, 1.5), (2.0, 1.0, 1.5),
                              6, 51))
        ctx.update_objects(objs, [0, 1, 2, 3, -1, -1])
        sc = oracle_scene_of(oracle, ctx)
        got = ctx.march(cam, p, W, H, reference_planes=True)
        assert ctx.lib.rkf_testing_last_variant(ctx.h) == 4
        ref = oracle.march(sc, cam, p, W, H, with_reference_planes=True)
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"voxelized props, full frame {k}")
        hit = (ref["flags"] & 1) != 0
        oid = (ref["packed_material"][hit] >> 24) & 0xFF
        assert ((oid >= 40) & (oid < 43)).sum() > 1000, "the view should see the voxelized props"
        pt = scenes.march_params(spec)
        pt.strategy = abi.RKF_STRATEGY_TILED
        got = ctx.march(cam, pt, W, H, reference_planes=True)
        assert ctx.lib.rkf_testing_last_variant(ctx.h) == 5
        for r in (0, 480, 541, 1079):
            ref = oracle.march(sc, cam, pt, W, H, rows=(r, r + 1), with_reference_planes=True)
            for k in PLANES:
                assert_bits_equal(got[k].reshape(H, -1)[r], ref[k].reshape(1, -1)[0], f"tiled, row {r} {k}")
    finally:
        ctx.close()
