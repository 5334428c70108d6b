"""The BVH strategy (ray_march_bvh, ray_march.wgsl:641-773) and its inputs:
the host-side SAH build (Bvh::build, crates/rkf-core/src/bvh.rs:66-260) and
the node import (GpuScene::upload_bvh, gpu_scene.rs:186).

CPU: the library's build against the reference's own build tests
(bvh.rs:407-440) and node for node against a float32 restatement written
here; the oracle's BVH march against its brute march.  GPU: views and ray
batches marched through the imported BVH, bit-exact against the oracle, a
tree deeper than the shader's 32-entry stack, and the import's checks."""
import ctypes as C

import numpy as np
import pytest

from conftest import assert_bits_equal
from test_tiled_gpu import PLANES, _camera, _objects, _params

F = np.float32
INVALID = 0xFFFFFFFF


# ---- a float32 restatement of build_recursive (bvh.rs:153-250) -------------
def _area(lo, hi):
    x, y, z = hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]
    return F(2.0) * ((x * y + y * z) + z * x)


def _py_build(boxes, ids):
    nodes = []

    def enclosing(idx):
        lo, hi = boxes[idx[0]][0].copy(), boxes[idx[0]][1].copy()
        for i in idx[1:]:
            lo, hi = np.fmin(lo, boxes[i][0]), np.fmax(hi, boxes[i][1])
        return lo, hi

    def reserve(e):
        nodes.append([e[0], INVALID, e[1], INVALID])
        return len(nodes) - 1

    def cent(i, axis):
        return (boxes[i][0][axis] + boxes[i][1][axis]) * F(0.5)

    def build(idx):
        e = enclosing(idx)
        if len(idx) == 1:
            k = reserve(e)
            nodes[k][3] = ids[idx[0]]
            return k
        if len(idx) == 2:
            k = reserve(e)
            nodes[k][1] = build(idx[:1])
            nodes[k][3] = build(idx[1:])
            return k
        esa = np.fmax(_area(*e), F(1e-10))
        best_cost, best_axis, best_split = F(np.finfo(np.float32).max), 0, len(idx) // 2
        for axis in range(3):
            idx.sort(key=lambda i: cent(i, axis))  # stable, like sort_by
            for split in range(1, len(idx)):
                la, ra = _area(*enclosing(idx[:split])), _area(*enclosing(idx[split:]))
                cost = F(1.0) + (F(1.0) * (la * F(split) + ra * F(len(idx) - split))) / esa
                if cost < best_cost:
                    best_cost, best_axis, best_split = cost, axis, split
        idx.sort(key=lambda i: cent(i, best_axis))
        k = reserve(e)
        nodes[k][1] = build(idx[:best_split])
        nodes[k][3] = build(idx[best_split:])
        return k

    if boxes:
        build(list(range(len(boxes))))
    return nodes


def _lib_build(boxes, ids):
    from rkifield_b200 import engine
    return engine.build_bvh((ids[k], boxes[k][0], boxes[k][1]) for k in range(len(boxes)))


def _unit_box(c):
    c = np.asarray(c, F)
    return (c - F(0.5), c + F(0.5))


def test_build_matches_reference_build_tests():
    """bvh.rs:407-440: empty, one object, two objects, twenty in a row."""
    assert len(_lib_build([], [])) == 0
    n = _lib_build([_unit_box((0, 0, 0))], [1])
    assert len(n) == 1 and n[0].left == INVALID and n[0].right_or_object == 1
    n = _lib_build([_unit_box((-2, 0, 0)), _unit_box((2, 0, 0))], [1, 2])
    assert len(n) == 3 and n[0].left != INVALID
    assert sum(1 for x in n if x.left == INVALID) == 2
    boxes = [_unit_box((i * 3.0, 0, 0)) for i in range(20)]
    n = _lib_build(boxes, list(range(20)))
    assert sum(1 for x in n if x.left == INVALID) == 20 and len(n) >= 20
    # build_root_aabb_encloses_all
    n = _lib_build([(np.array([-5, -1, -1], F), np.array([-4, 1, 1], F)),
                    (np.array([4, -1, -1], F), np.array([5, 1, 1], F))], [0, 1])
    assert n[0].aabb_min[0] <= -5.0 and n[0].aabb_max[0] >= 5.0


@pytest.mark.parametrize("seed", range(6))
def test_build_node_for_node(seed):
    """The library's build equals the restatement above bit for bit,
    including ties of centroids (the stable sorts decide those)."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 48))
    boxes = []
    for _ in range(n):
        c = rng.normal(size=3).astype(F) * F(20)
        if rng.random() < 0.3:
            c[rng.integers(0, 3)] = F(2.5)  # shared centroids along one axis
        h = rng.uniform(0.1, 4.0, size=3).astype(F)
        boxes.append((c - h, c + h))
    ids = [int(x) for x in rng.permutation(1000)[:n]]
    got = _lib_build(boxes, ids)
    ref = _py_build(boxes, ids)
    assert len(got) == len(ref) == 2 * n - 1
    for k, (g, r) in enumerate(zip(got, ref)):
        assert np.array(g.aabb_min, F).tobytes() == np.asarray(r[0], F).tobytes(), k
        assert np.array(g.aabb_max, F).tobytes() == np.asarray(r[2], F).tobytes(), k
        assert (g.left, g.right_or_object) == (r[1], r[3]), k
        if g.left != INVALID:
            assert k < g.left < len(got) and k < g.right_or_object < len(got)


def test_build_rejects_bad_input():
    from rkifield_b200 import _abi as abi
    lib = abi.load_library()
    items = (abi.rkf_bvh_item * 2)()
    nodes = (abi.rkf_bvh_node * 3)()
    n = C.c_uint32()
    assert lib.rkf_bvh_build(items, 2, nodes, 2, C.byref(n)) == abi.RKF_INVALID_ARG  # room for 2 of 3
    items[1].aabb_min[1] = float("nan")
    assert lib.rkf_bvh_build(items, 2, nodes, 3, C.byref(n)) == abi.RKF_INVALID_ARG


def _scene_bvh(objs):
    from rkifield_b200 import engine
    return engine.object_bvh(objs)


def test_oracle_bvh_equals_brute(oracle, small_scene):
    """Every object here has an SDF no smaller than the distance to its AABB,
    so skipping far nodes never drops the nearest object; with no exact ties
    between objects the BVH march equals the brute march bit for bit."""
    from rkifield_b200 import _abi as abi
    v = small_scene["vox"]
    objs = _objects(small_scene)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map, bvh=_scene_bvh(objs))
    w, h = 128, 96
    cam = _camera(3, w, h)
    b = oracle.march(sc, cam, _params(abi.RKF_STRATEGY_BRUTE), w, h)
    t = oracle.march(sc, cam, _params(abi.RKF_STRATEGY_BVH), w, h)
    assert ((b["flags"] & 1) != 0).sum() > 300
    for k in ("t", "normal", "slot", "material", "flags"):
        assert_bits_equal(t[k], b[k], f"bvh vs brute {k}")


def _chain_bvh(objs, depth=40):
    """A right-leaning chain: internal node k has a leaf on the left and the
    next internal node on the right, so the stack grows by one per level.
    The shader pushes children only while fewer than 31 entries are on the
    stack, so the walk stops descending at level 31: leaves 0..30 are
    reached, deeper ones never.  Object 0 is named only by leaves 34 and 39,
    so a march that respects the limit never evaluates it; the last node
    names an index beyond the object count."""
    from rkifield_b200 import _abi as abi
    lo = np.min([o.aabb_min[:] for o in objs], axis=0)
    hi = np.max([o.aabb_max[:] for o in objs], axis=0)
    nodes = (abi.rkf_bvh_node * (2 * depth + 1))()
    for k in range(depth):
        inner, leaf = 2 * k, 2 * k + 1
        oi = (depth - 1 - k) % len(objs)
        if oi == 0 and k <= 30:
            oi = 1
        for a in range(3):
            nodes[inner].aabb_min[a], nodes[inner].aabb_max[a] = lo[a], hi[a]
            nodes[leaf].aabb_min[a] = objs[oi].aabb_min[a]
            nodes[leaf].aabb_max[a] = objs[oi].aabb_max[a]
        nodes[inner].left, nodes[inner].right_or_object = leaf, 2 * k + 2
        nodes[leaf].left, nodes[leaf].right_or_object = INVALID, oi
    last = 2 * depth
    for a in range(3):
        nodes[last].aabb_min[a], nodes[last].aabb_max[a] = lo[a], hi[a]
    nodes[last].left, nodes[last].right_or_object = INVALID, 7  # beyond the object count: skipped
    return nodes


def test_oracle_stack_limit_drops_deep_levels(oracle, small_scene):
    """The restatement keeps the shader's stack rule: the voxelized object,
    named only below the limit of a 40-level chain, is never hit, while the
    brute march hits it."""
    from rkifield_b200 import _abi as abi
    v = small_scene["vox"]
    objs = _objects(small_scene)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map, bvh=_chain_bvh(objs))
    w, h = 96, 64
    cam = _camera(3, w, h)
    t = oracle.march(sc, cam, _params(abi.RKF_STRATEGY_BVH), w, h, with_reference_planes=True)
    b = oracle.march(sc, cam, _params(abi.RKF_STRATEGY_BRUTE), w, h, with_reference_planes=True)

    def ids(g):
        hit = (g["flags"] & 1) != 0
        return set(((g["packed_material"][hit] >> 24) & 0xFF).tolist())
    assert objs[0].object_id in ids(b)
    assert objs[0].object_id not in ids(t), "object 0 sits only below the stack limit"


# ---- GPU -------------------------------------------------------------------
def _ctx(small_scene, objs):
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    ctx = Context(pool_capacity=v.n_bricks + 1024)
    ctx.set_brick_pool(v.words)
    ctx.upload_brick_maps(v.map)
    ctx.upload_objects(objs)
    return ctx


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [3, 4])
def test_bvh_views_bit_exact(oracle, small_scene, seed):
    from rkifield_b200 import _abi as abi
    v = small_scene["vox"]
    objs = _objects(small_scene)
    bvh = _scene_bvh(objs)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map, bvh=bvh)
    ctx = _ctx(small_scene, objs)
    try:
        ctx.upload_bvh(bvh)
        w, h = 200, 136
        cam = _camera(seed, w, h)
        p = _params(abi.RKF_STRATEGY_BVH)
        ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
        got = ctx.march(cam, p, w, h, reference_planes=True)
        assert ((ref["flags"] & 1) != 0).sum() > 500
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"bvh {k}")
    finally:
        ctx.close()


@pytest.mark.gpu
def test_bvh_stack_limit_bit_exact(oracle, small_scene):
    """A 40-level chain: the kernel drops the levels beyond the 32-entry
    stack exactly as the shader and the oracle do, and skips leaves whose
    object index is beyond the object count."""
    from rkifield_b200 import _abi as abi
    v = small_scene["vox"]
    objs = _objects(small_scene)
    nodes = _chain_bvh(objs)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map, bvh=nodes)
    ctx = _ctx(small_scene, objs)
    try:
        ctx.upload_bvh(nodes)
        w, h = 128, 96
        cam = _camera(4, w, h)
        p = _params(abi.RKF_STRATEGY_BVH)
        ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
        got = ctx.march(cam, p, w, h, reference_planes=True)
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"chain {k}")
    finally:
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["closest", "any"])
def test_bvh_ray_batches_bit_exact(oracle, small_scene, mode):
    from rkifield_b200 import _abi as abi
    v = small_scene["vox"]
    objs = _objects(small_scene)
    bvh = _scene_bvh(objs)
    sc = oracle.Scene(objs, pool_words=v.words, brick_maps=v.map, bvh=bvh)
    rng = np.random.default_rng(9)
    n = 20000
    org = rng.uniform(-40, 40, size=(n, 3)).astype(F)
    tgt = rng.uniform(-20, 20, size=(n, 3)).astype(F)
    d = tgt - org
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d = d.astype(F)
    tmax = np.full(n, 150.0, F)
    m = abi.RKF_TRACE_CLOSEST if mode == "closest" else abi.RKF_TRACE_ANY
    p = _params(abi.RKF_STRATEGY_BVH)
    ref = oracle.trace(sc, org.ravel(), d.ravel(), tmax, m, p)
    ctx = _ctx(small_scene, objs)
    try:
        ctx.upload_bvh(bvh)
        got = ctx.trace(org, d, tmax, m, p)
        assert ((ref["flags"] & 1) != 0).sum() > 1000
        for k in got:
            assert_bits_equal(got[k], ref[k], f"bvh {mode} {k}")
    finally:
        ctx.close()


@pytest.mark.gpu
def test_bvh_import_checks(small_scene):
    """Nodes that are not one tree with children after their parent are
    refused and the previous BVH stays; the BVH strategy needs a BVH; the
    brute-only launch paths refuse the strategy."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200.engine import RkfError
    objs = _objects(small_scene)
    ctx = _ctx(small_scene, objs)
    try:
        cam = _camera(3, 64, 48)
        p = _params(abi.RKF_STRATEGY_BVH)
        with pytest.raises(RkfError) as e:
            ctx.march(cam, p, 64, 48)
        assert e.value.status == abi.RKF_INVALID_ARG
        good = _scene_bvh(objs)
        ctx.upload_bvh(good)
        before = ctx.march(cam, p, 64, 48)

        def refused(nodes):
            with pytest.raises(RkfError) as e:
                ctx.upload_bvh(nodes)
            assert e.value.status == abi.RKF_INVALID_ARG

        def edited(k, field, value):
            nodes = (abi.rkf_bvh_node * len(good))(*good)
            setattr(nodes[k], field, value)
            return nodes

        inner = [k for k in range(len(good)) if good[k].left != INVALID]
        assert len(inner) >= 2
        k = inner[1]
        refused(edited(k, "left", 0))                                    # back to the root: a cycle
        refused(edited(0, "right_or_object", good[0].left))              # one child named twice
        refused(edited(0, "right_or_object", len(good)))                 # past the end
        refused(edited(k, "left", k - 1 if k - 1 != good[k].right_or_object else k))  # not after its parent
        orphan = (abi.rkf_bvh_node * 3)(*good[:1])
        orphan[0].left = INVALID                                         # nodes 1, 2 named by no one
        refused(orphan)
        after = ctx.march(cam, p, 64, 48)
        for k in before:
            assert_bits_equal(after[k], before[k], f"previous BVH kept: {k}")
        with pytest.raises(RkfError) as e:
            ctx.march(cam, p, 64, 48, plain=True)
        assert e.value.status == abi.RKF_UNSUPPORTED
        ctx.upload_bvh((abi.rkf_bvh_node * 0)())
        with pytest.raises(RkfError) as e:
            ctx.march(cam, p, 64, 48)
        assert e.value.status == abi.RKF_INVALID_ARG
    finally:
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f32", "u8"])
@pytest.mark.parametrize("strategy", ["bvh", "tiled"])
def test_strategies_over_precision_planes_bit_exact(oracle, small_scene, precision, strategy):
    """The BVH and tiled marches over the f32 and u8 distance planes, against
    the oracle reading the same planes and index; the BVH march also through
    three bands of host-output rows."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    objs = _objects(small_scene)
    bvh = _scene_bvh(objs)
    ctx = Context(pool_capacity=v.n_bricks + 1024, precision=precision)
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        ctx.upload_objects(objs)
        ctx.upload_bvh(bvh)
        pl = ctx.export_planes(0, v.n_bricks)
        idx = ctx.export_index()
        if precision == "f32":
            kw = {"dist_f32": pl["dist"], "precision": abi.RKF_PRECISION_F32}
        else:
            kw = {"dist_u8": pl["dist"], "brick_scale": pl["step"], "precision": abi.RKF_PRECISION_U8}
        sc = oracle.Scene(objs, top=idx["top"], leaves=idx["leaves"], obj_top_info=idx["obj_top_info"],
                          mat_plane=pl["mat"], blend_plane=pl["blend"], bvh=bvh, **kw)
        w, h = 200, 136
        cam = _camera(4, w, h)
        p = _params(abi.RKF_STRATEGY_BVH if strategy == "bvh" else abi.RKF_STRATEGY_TILED)
        ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
        got = ctx.march(cam, p, w, h, reference_planes=True)
        assert ((ref["flags"] & 1) != 0).sum() > 500
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"{strategy} {precision} {k}")
        if strategy == "bvh":
            lib = abi.load_library()
            lib.rkf_testing_set_host_bands(3)
            try:
                banded = ctx.march(cam, p, w, h, reference_planes=True)
            finally:
                lib.rkf_testing_set_host_bands(-1)
            for k in PLANES:
                assert_bits_equal(banded[k], ref[k], f"banded {strategy} {precision} {k}")
    finally:
        ctx.close()


@pytest.mark.gpu
def test_bvh_single_leaf_bit_exact(oracle, small_scene):
    """A BVH of one leaf over the one voxelized object (which the library
    marches as the brute march it equals), against the oracle's stack walk."""
    from rkifield_b200 import _abi as abi, engine, scenes
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    spec = small_scene["spec"]
    obj = small_scene["obj"]
    bvh = engine.object_bvh([obj])
    assert len(bvh) == 1 and bvh[0].left == INVALID and bvh[0].right_or_object == 0
    sc = oracle.Scene([obj], pool_words=v.words, brick_maps=v.map, bvh=bvh)
    ctx = Context(pool_capacity=v.n_bricks + 1024)
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        ctx.upload_objects([obj])
        ctx.upload_bvh(bvh)
        w, h = 160, 128
        cam = scenes.seeded_camera(spec, w, h, seed=13)
        p = scenes.march_params(spec)
        p.strategy = abi.RKF_STRATEGY_BVH
        ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
        got = ctx.march(cam, p, w, h, reference_planes=True)
        assert ((ref["flags"] & 1) != 0).sum() > 300
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"one-leaf bvh {k}")
    finally:
        ctx.close()
