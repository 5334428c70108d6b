"""The multi-object empty-space path: one voxelized object beside analytic
objects and objects of no type.  EMPTY runs and settling chains stay outside
each analytic object's ball (its primitive's bounding radius mapped to world
space, widened by the largest EMPTY value and every rounding bound), so the
minimum over the scene there is the voxelized object's EMPTY value, and every
output stays bit-exact against the oracle: views, and ray casts in the three
modes (closest, any hit, soft shadow), with analytic objects outside the
grid, just beyond it and inside it, rotated and non-uniformly scaled, and the
voxelized object not first in the list, under the brute, tiled and BVH
strategies.  A plane bounds the runs by the half-space where its value may
fall to an EMPTY value.  A tuning without the empty path marches the
full sampler only, with the same outputs, and the autotuner may pick it."""
import ctypes as C

import numpy as np
import pytest

from conftest import assert_bits_equal
from test_tiled_gpu import PLANES, _analytic, _camera, _params
from test_trace_gpu import _rays

pytestmark = pytest.mark.gpu


VARIANT_MULTI, VARIANT_MULTI_EMPTY, VARIANT_MULTI_EMPTY_TILED = 0, 4, 5


def _rotation(axis, angle):
    a = np.asarray(axis, np.float64)
    a /= np.linalg.norm(a)
    k = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(angle) * k + (1 - np.cos(angle)) * (k @ k)


def _transformed(ptype, centre, params, rot, scale, mat, oid):
    """An analytic object whose local frame is scaled by `scale`, rotated by
    `rot` and moved to `centre`: inverse_world maps world to local,
    l = S^-1 R^T (p - c)."""
    o = _analytic(ptype, centre, params, (1.0, 1.0, 1.0), mat, oid)
    a = np.diag(1.0 / np.asarray(scale, np.float64)) @ rot.T
    t = -a @ np.asarray(centre, np.float64)
    for i in range(3):
        for k in range(3):
            o.inverse_world[4 * k + i] = float(a[i, k])
        o.inverse_world[12 + i] = float(t[i])
        o.accumulated_scale[i] = float(scale[i])
    ext = float(np.linalg.norm(params[:3])) * float(max(scale)) + 1.0
    for i in range(3):
        o.aabb_min[i] = float(centre[i] - ext)
        o.aabb_max[i] = float(centre[i] + ext)
    return o


def _none_object(oid):
    o = _analytic(0, (0.0, 0.0, 0.0), (1.0,), (1.0, 1.0, 1.0), 0, oid)
    from rkifield_b200 import _abi as abi
    o.sdf_type = abi.RKF_SDF_NONE
    return o


def _scene_objects(small_scene):
    return [_analytic(0, (30.0, 0.0, 0.0), (3.0,), (3.0, 3.0, 3.0), 5, 2),                     # sphere beyond the grid
            small_scene["obj"],                                                                 # voxelized (index 1)
            _analytic(3, (0.0, 19.5, 0.0), (4.0, 1.0), (5.0, 1.0, 5.0), 6, 3),                  # torus just above it
            _transformed(1, (-10.0, 2.0, 8.0), (2.0, 1.0, 1.5), _rotation((1, 2, 3), 0.7),
                         (1.5, 0.7, 1.2), 7, 4),                                                # rotated, scaled box
            _none_object(5),
            _analytic(2, (12.0, -5.0, -9.0), (1.0, 2.5), (1.0, 3.5, 1.0), 8, 6),                # capsule inside the grid
            _analytic(4, (-5.0, 12.0, -14.0), (2.0, 1.5), (2.0, 1.5, 2.0), 9, 7)]               # cylinder inside the grid


def _context(small_scene, objs):
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    ctx = Context(pool_capacity=v.n_bricks + 1024)
    ctx.set_brick_pool(v.words)
    ctx.upload_brick_maps(v.map)
    ctx.upload_objects(objs)
    return ctx


@pytest.mark.parametrize("seed", [3, 5, 8])
def test_views_bit_exact(oracle, small_scene, seed):
    v = small_scene["vox"]
    objs = _scene_objects(small_scene)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map)
    ctx = _context(small_scene, objs)
    try:
        w, h = 200, 136
        cam = _camera(seed, w, h)
        p = _params(0)
        ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
        got = ctx.march(cam, p, w, h, reference_planes=True)
        assert ctx.lib.rkf_testing_last_variant(ctx.h) == VARIANT_MULTI_EMPTY
        hit = (ref["flags"] & 1) != 0
        assert hit.sum() > 500
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"seed {seed}: {k}")
    finally:
        ctx.close()


def test_views_see_the_analytic_objects(oracle, small_scene):
    """A camera close to the torus and the box: rays graze the balls."""
    from rkifield_b200 import scenes
    v = small_scene["vox"]
    objs = _scene_objects(small_scene)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map)
    ctx = _context(small_scene, objs)
    try:
        w, h = 160, 120
        p = _params(0)
        seen = set()
        for eye, target in (((0.0, 32.0, 18.0), (0.0, 19.5, 0.0)), ((-22.0, 6.0, 24.0), (-10.0, 2.0, 8.0))):
            cam = scenes.camera_uniforms(eye, target, w, h)
            ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
            got = ctx.march(cam, p, w, h, reference_planes=True)
            assert ctx.lib.rkf_testing_last_variant(ctx.h) == VARIANT_MULTI_EMPTY
            for k in PLANES:
                assert_bits_equal(got[k], ref[k], f"eye {eye}: {k}")
            hit = (ref["flags"] & 1) != 0
            seen |= set(((ref["packed_material"][hit] >> 24) & 0xFF).tolist())
        assert {3, 4} <= seen, f"object ids seen: {sorted(seen)}"
    finally:
        ctx.close()


@pytest.mark.parametrize("mode", [0, 1, 2], ids=["closest", "any", "shadow"])
def test_rays_bit_exact(oracle, small_scene, mode):
    from rkifield_b200 import scenes
    v = small_scene["vox"]
    objs = _scene_objects(small_scene)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map)
    ctx = _context(small_scene, objs)
    try:
        o, d, tmax = _rays(20000, seed=40 + mode, box=24.0)
        p = scenes.march_params(small_scene["spec"])
        ref = oracle.trace(sc, o.ravel(), d.ravel(), tmax, mode, p)
        got = ctx.trace(o, d, tmax, mode, p)
        assert ctx.lib.rkf_testing_last_variant(ctx.h) == VARIANT_MULTI_EMPTY
        assert_bits_equal(got["t"], ref["t"], "t")
        assert_bits_equal(got["flags"], ref["flags"], "flags")
        if mode == 0:
            for k in ("normal", "slot", "material"):
                assert_bits_equal(got[k], ref[k], k)
        assert 100 < int((ref["flags"] & 1).sum()) < 20000
    finally:
        ctx.close()


def _plane(normal, point, mat, oid, rot=None):
    """An analytic plane through `point` (world) with local normal `normal`,
    optionally rotated: inverse_world maps world to local, l = R^T (p - point)."""
    o = _analytic(5, point, tuple(normal), (60.0, 60.0, 60.0), mat, oid)
    if rot is not None:
        a = rot.T
        t = -a @ np.asarray(point, np.float64)
        for i in range(3):
            for k in range(3):
                o.inverse_world[4 * k + i] = float(a[i, k])
            o.inverse_world[12 + i] = float(t[i])
    return o


@pytest.mark.parametrize("case", ["ground_below", "tilted_through", "above_camera_side"])
def test_scenes_with_a_plane_take_the_multi_object_path(oracle, small_scene, case):
    """A plane (ray_march.wgsl:206-208, 257-258) bounds the EMPTY runs by the
    half-space where its value may drop to an EMPTY value; views under the
    brute and tiled strategies and ray casts in the three modes, bit-exact
    with the oracle: a ground plane below the grid, a tilted plane through
    it, and a plane whose near side holds the camera."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import scenes
    v = small_scene["vox"]
    w, h = 120, 80
    plane = {"ground_below": _plane((0.0, 1.0, 0.0), (0.0, -17.0, 0.0), 3, 8),
             "tilted_through": _plane((0.0, 1.0, 0.0), (2.0, -3.0, 1.0), 3, 8, rot=_rotation((1.0, 0.0, 0.4), 0.5)),
             "above_camera_side": _plane((0.0, -1.0, 0.0), (0.0, 24.0, 0.0), 3, 8)}[case]
    objs = _scene_objects(small_scene) + [plane]
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map)
    ctx = _context(small_scene, objs)
    try:
        hits = 0
        for strategy, variant in ((0, VARIANT_MULTI_EMPTY), (abi.RKF_STRATEGY_TILED, VARIANT_MULTI_EMPTY_TILED)):
            p = _params(strategy)
            for seed in (4, 6):
                cam = _camera(seed, w, h)
                ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
                got = ctx.march(cam, p, w, h, reference_planes=True)
                assert ctx.lib.rkf_testing_last_variant(ctx.h) == variant
                for k in PLANES:
                    assert_bits_equal(got[k], ref[k], f"{case} strategy {strategy} seed {seed}: {k}")
                hits += int(((ref["packed_material"] >> 24) & 0xFF == 8).sum())
        # a camera inside the grid looking down at the ground plane
        cam = scenes.camera_uniforms((3.0, 6.0, 9.0), (0.0, -17.0, 0.0), w, h)
        p = _params(0)
        ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
        got = ctx.march(cam, p, w, h, reference_planes=True)
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"{case} looking down: {k}")
        hits += int(((ref["packed_material"] >> 24) & 0xFF == 8).sum())
        assert hits > 50, "the views should see the plane"
        o, d, tmax = _rays(6000, seed=9)
        for mode in (abi.RKF_TRACE_CLOSEST, abi.RKF_TRACE_ANY, abi.RKF_TRACE_SHADOW):
            ref = oracle.trace(sc, o.ravel(), d.ravel(), tmax, mode, _params(0))
            got = ctx.trace(o, d, tmax, mode, _params(0))
            assert ctx.lib.rkf_testing_last_variant(ctx.h) == VARIANT_MULTI_EMPTY
            for k in got:
                assert_bits_equal(got[k], ref[k], f"{case} rays mode {mode}: {k}")
    finally:
        ctx.close()


def test_tiled_strategy_marches_the_multi_object_path(oracle, small_scene):
    """The tiled strategy (coarse skips, per-tile object lists): EMPTY runs
    on the tiled empty-space field for rays whose tile lists the voxelized
    object, tiled steps elsewhere; bit-exact against the oracle's tiled march
    from afar (coarse skips active) and close to the objects."""
    from rkifield_b200 import _abi as abi, scenes
    v = small_scene["vox"]
    objs = _scene_objects(small_scene)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map)
    ctx = _context(small_scene, objs)
    try:
        p = _params(abi.RKF_STRATEGY_TILED)
        views = [(_camera(seed, 200, 136), 200, 136) for seed in (3, 5, 8)]
        views += [(scenes.camera_uniforms(eye, target, 160, 120), 160, 120)
                  for eye, target in (((0.0, 32.0, 18.0), (0.0, 19.5, 0.0)), ((-22.0, 6.0, 24.0), (-10.0, 2.0, 8.0)),
                                      ((5.0, 3.0, 4.0), (20.0, -2.0, -9.0)))]
        for i, (cam, w, h) in enumerate(views):
            ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
            got = ctx.march(cam, p, w, h, reference_planes=True)
            assert ctx.lib.rkf_testing_last_variant(ctx.h) == VARIANT_MULTI_EMPTY_TILED
            assert int((ref["flags"] & 1).sum()) > 300
            for k in PLANES:
                assert_bits_equal(got[k], ref[k], f"tiled view {i}: {k}")
    finally:
        ctx.close()


def test_tuning_without_the_empty_path(oracle, small_scene):
    from rkifield_b200 import _abi as abi, cudart
    v = small_scene["vox"]
    w, h = 160, 120
    cam = _camera(5, w, h)
    p = _params(0)
    for objs, plain in (([small_scene["obj"]], 1), (_scene_objects(small_scene), VARIANT_MULTI)):
        sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map)
        ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
        ctx = _context(small_scene, objs)
        try:
            g = cudart.device_gbuffer(w * h, reference_planes=True)
            vw = (abi.rkf_view * 1)()
            vw[0].camera = cam
            vw[0].width, vw[0].height = w, h
            for k, a in g.items():
                setattr(vw[0].out, k, a.ptr)
            vw[0].out.mem = abi.RKF_MEM_DEVICE
            tu = abi.rkf_batch_tuning(4, 8, 32, 64, 0, 256, 32, 0, 1)
            abi.check(ctx.lib.rkf_march_batch(ctx.h, vw, 1, None, 0, C.byref(p), C.byref(tu)), "rkf_march_batch")
            assert ctx.lib.rkf_testing_last_variant(ctx.h) == plain
            for k, a in g.items():
                assert_bits_equal(a.download(), ref[k], f"{len(objs)} objects, no empty path: {k}")
            out = abi.rkf_batch_tuning()
            abi.check(ctx.lib.rkf_autotune(ctx.h, vw, 1, None, 0, C.byref(p), C.byref(out)), "rkf_autotune")
            assert out.no_empty_path in (0, 1)
            got = ctx.march(cam, p, w, h, reference_planes=True)  # with the tuning the context keeps
            for k in PLANES:
                assert_bits_equal(got[k], ref[k], f"{len(objs)} objects, autotuned: {k}")
        finally:
            ctx.close()


def test_graph_marches_the_multi_object_path(oracle, small_scene):
    """A batch graph captured over the multi-object scene: its launch writes
    the oracle's planes."""
    from rkifield_b200 import _abi as abi, cudart
    v = small_scene["vox"]
    objs = _scene_objects(small_scene)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map)
    ctx = _context(small_scene, objs)
    graph = C.c_void_p()
    try:
        w, h = 160, 120
        cam = _camera(8, w, h)
        p = _params(0)
        ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
        g = cudart.device_gbuffer(w * h, reference_planes=True)
        vw = (abi.rkf_view * 1)()
        vw[0].camera = cam
        vw[0].width, vw[0].height = w, h
        for k, a in g.items():
            setattr(vw[0].out, k, a.ptr)
        vw[0].out.mem = abi.RKF_MEM_DEVICE
        abi.check(ctx.lib.rkf_batch_graph_create(ctx.h, vw, 1, None, 0, C.byref(p), None, C.byref(graph)),
                  "rkf_batch_graph_create")
        abi.check(ctx.lib.rkf_batch_graph_launch(graph, None), "rkf_batch_graph_launch")
        cudart.synchronize()
        assert int((ref["flags"] & 1).sum()) > 200
        for k, a in g.items():
            assert_bits_equal(a.download(), ref[k], f"graph: {k}")
    finally:
        if graph.value:
            ctx.lib.rkf_batch_graph_destroy(graph)
        ctx.close()


def test_serving_marches_the_multi_object_path(oracle, small_scene):
    """Renders and ray batches served by the resident loop over the
    multi-object scene equal the oracle's."""
    from rkifield_b200 import engine, scenes
    from rkifield_b200.engine import Server
    v = small_scene["vox"]
    objs = _scene_objects(small_scene)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map)
    ctx = _context(small_scene, objs)
    p = scenes.march_params(small_scene["spec"])
    p.scene.max_distance = 200.0
    srv = Server(ctx, p)
    try:
        w, h = 160, 120
        cam = _camera(3, w, h)
        o, d, tmax = _rays(5000, seed=77, box=24.0)
        out_r = engine.render_out(w * h)
        out_b = engine.rays_out(5000, 0)
        tickets = [srv.submit_render(cam, w, h, out_r), srv.submit_rays(o, d, tmax, 0, out_b)]
        for t in tickets:
            res = srv.poll(t, 10_000_000)
            assert res is not None and res["status"] == 0, res
        ref = oracle.march(sc, cam, p, w, h)
        for k in out_r:
            if k in ref:
                assert_bits_equal(out_r[k], ref[k], f"served render: {k}")
        ref_b = oracle.trace(sc, o.ravel(), d.ravel(), tmax, 0, p)
        for k in out_b:
            assert_bits_equal(out_b[k], ref_b[k], f"served rays: {k}")
        assert int((ref["flags"] & 1).sum()) > 200
    finally:
        srv.stop()
        ctx.close()


def test_bvh_strategy_marches_the_multi_object_path(oracle, small_scene):
    """The BVH strategy over the runtime's tree (one leaf per object AABB):
    its walk reaches the voxelized object everywhere in its grid, so the
    multi-object empty-space variant marches it, bit-exact against the
    oracle's walk; a tree whose leaf for the voxelized object does not hold
    its grid marches the plain kernel, also bit-exact."""
    from rkifield_b200 import _abi as abi, engine, scenes
    v = small_scene["vox"]
    objs = _scene_objects(small_scene)
    nodes = engine.object_bvh(objs)
    shrunk = (abi.rkf_bvh_node * len(nodes))(*nodes)
    leaf = [i for i, n in enumerate(shrunk) if n.left == abi.BVH_INVALID and n.right_or_object == 1]
    assert len(leaf) == 1
    shrunk[leaf[0]].aabb_min[0] += 1.0
    ctx = _context(small_scene, objs)
    try:
        w, h = 200, 136
        p = _params(abi.RKF_STRATEGY_BVH)
        for tree, variant in ((nodes, VARIANT_MULTI_EMPTY), (shrunk, VARIANT_MULTI)):
            ctx.upload_bvh(tree)
            sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map, bvh=tree)
            for seed in (3, 5):
                cam = _camera(seed, w, h)
                ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
                got = ctx.march(cam, p, w, h, reference_planes=True)
                assert ctx.lib.rkf_testing_last_variant(ctx.h) == variant
                assert int((ref["flags"] & 1).sum()) > 500
                for k in PLANES:
                    assert_bits_equal(got[k], ref[k], f"variant {variant} seed {seed}: {k}")
            o, d, tmax = _rays(8000, seed=91, box=24.0)
            pr = scenes.march_params(small_scene["spec"])
            pr.strategy = abi.RKF_STRATEGY_BVH
            ref = oracle.trace(sc, o.ravel(), d.ravel(), tmax, 0, pr)
            got = ctx.trace(o, d, tmax, 0, pr)
            assert ctx.lib.rkf_testing_last_variant(ctx.h) == variant
            for k in ("t", "flags", "normal", "slot", "material"):
                assert_bits_equal(got[k], ref[k], f"variant {variant} rays: {k}")
    finally:
        ctx.close()
