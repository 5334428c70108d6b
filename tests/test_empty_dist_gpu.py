"""The empty-space distance field and the march path that uses it.

The field (one byte per top-grid block) must be the capped Chebyshev
distance to the nearest non-EMPTY block after a build, and never above it
after edits (which lower it around the blocks they turn into leaf blocks).
The march that skips the sampler inside EMPTY cubes must stay bit-exact:
views from inside the grid (long runs through empty space, many cube exits)
and from outside, against the FP32 oracle."""
import ctypes as C

import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

CAP = 64
EMPTY = 0xFFFFFFFF
PLANES = ("t", "normal", "slot", "material", "flags", "position", "packed_material", "motion")


def _field(ctx):
    from rkifield_b200 import _abi as abi
    n = C.c_uint64()
    lib = abi.load_library()
    abi.check(lib.rkf_testing_export_empty_dist(ctx.h, None, C.byref(n)), "export_empty_dist")
    out = np.zeros(max(1, n.value), np.uint8)
    abi.check(lib.rkf_testing_export_empty_dist(ctx.h, out.ctypes.data, C.byref(n)), "export_empty_dist")
    return out[:n.value]


def _chebyshev(top, info):
    """Brute-force field of every object's top grid."""
    want = np.zeros(top.size, np.uint8)
    for i in range(info.size // 4):
        off, nx, ny, nz = (int(v) for v in info[4 * i:4 * i + 4])
        g = top[off:off + nx * ny * nz].reshape(nz, ny, nx)
        z, y, x = np.nonzero(g != EMPTY)
        zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        d = np.full((nz, ny, nx), CAP, np.int64)
        for bz, by, bx in zip(z, y, x):
            d = np.minimum(d, np.maximum(np.maximum(abs(zz - bz), abs(yy - by)), abs(xx - bx)))
        want[off:off + nx * ny * nz] = d.ravel()
    return want


def test_field_exact_after_build(small_scene):
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    spec = small_scene["spec"]
    ctx = Context(pool_capacity=small_scene["vox"].n_bricks * 2 + 4096, keep_reference_pool=False)
    try:
        ctx.voxelize(small_scene["prims"], small_scene["vp"])
        prims2 = small_scene["prims"][:5].copy()
        ctx.voxelize(prims2, scenes.voxelize_params(spec, prims2, object_id=2))
        idx = ctx.export_index()
        got = _field(ctx)
        want = _chebyshev(idx["top"], idx["obj_top_info"])
        assert (want == 0).sum() > 0 and (want > 1).sum() > 0
        assert_bits_equal(got, want, "empty-space distance field")
    finally:
        ctx.close()


def test_field_after_import_matches_build(small_scene, small_ctx):
    idx = small_ctx.export_index()
    assert_bits_equal(_field(small_ctx), _chebyshev(idx["top"], idx["obj_top_info"]), "imported scene field")


def test_field_conservative_after_edits(oracle, small_scene):
    from rkifield_b200 import _abi as abi, scenes
    from rkifield_b200.engine import Context
    spec = small_scene["spec"]
    ctx = Context(pool_capacity=small_scene["vox"].n_bricks * 2 + 8192, keep_reference_pool=False)
    try:
        ctx.voxelize(small_scene["prims"], small_scene["vp"])
        rng = np.random.default_rng(7)
        lo = np.array(small_scene["vp"].aabb_min[:], np.float32)
        hi = np.array(small_scene["vp"].aabb_max[:], np.float32)
        for _ in range(6):  # additive blobs in empty space create leaf blocks there
            op = abi.rkf_edit_op()
            op.object_index, op.edit_type, op.shape_type, op.falloff = 0, 0, 0, 1
            op.position[:] = [float(v) for v in rng.uniform(lo + 2, hi - 2)]
            op.rotation[:] = (0.0, 0.0, 0.0, 1.0)
            op.dimensions[:] = (0.5, 0.0, 0.0)
            op.strength, op.blend_k, op.material_id = 1.0, 0.05, 9
            ctx.edit(op)
        idx = ctx.export_index()
        got = _field(ctx).astype(np.int64)
        want = _chebyshev(idx["top"], idx["obj_top_info"]).astype(np.int64)
        assert (got <= want).all(), "the field overstates a distance after edits"
        assert ((got == 0) == (want == 0)).all(), "EMPTY and non-EMPTY blocks must stay distinguished"
        # the march of the edited scene still matches the oracle on the same index
        cam = scenes.seeded_camera(spec, 160, 120, seed=31, inside=True)
        p = scenes.march_params(spec)
        pl = ctx.export_planes(0, ctx.info()["pool_capacity"])
        sc = oracle.Scene([ctx.object(0)], top=idx["top"], leaves=idx["leaves"], obj_top_info=idx["obj_top_info"],
                          dist_f16=pl["dist"], mat_plane=pl["mat"], blend_plane=pl["blend"])
        ref = oracle.march(sc, cam, p, 160, 120, with_reference_planes=True)
        got_m = ctx.march(cam, p, 160, 120, reference_planes=True)
        for k in PLANES:
            assert_bits_equal(got_m[k], ref[k], f"edited scene {k}")
    finally:
        ctx.close()


@pytest.mark.parametrize("seed", [21, 22, 23])
def test_inside_views_bit_exact(oracle, small_scene, small_ctx, seed):
    """Cameras inside the grid: rays start in empty space and cross many
    EMPTY cubes before hitting or running out of steps."""
    from rkifield_b200 import scenes
    spec = small_scene["spec"]
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    cam = scenes.seeded_camera(spec, 224, 160, seed=seed, inside=True)
    p = scenes.march_params(spec)
    ref = oracle.march(sc, cam, p, 224, 160, with_reference_planes=True)
    got = small_ctx.march(cam, p, 224, 160, reference_planes=True)
    assert (ref["flags"] & 1).sum() > 200
    for k in PLANES:
        assert_bits_equal(got[k], ref[k], k)


def test_shadow_and_any_rays_bit_exact(oracle, small_scene, small_ctx):
    """Soft-shadow and any-hit rays through empty space (the same cubes,
    stepped along the raw direction)."""
    from rkifield_b200 import _abi as abi
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    rng = np.random.default_rng(3)
    n = 20000
    lo = np.array(small_scene["vp"].aabb_min[:], np.float32)
    hi = np.array(small_scene["vp"].aabb_max[:], np.float32)
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d[:100, 1] = 0.0  # axis-parallel components
    d[100:200, 0] = 0.0
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    tmax = rng.uniform(1.0, 40.0, n).astype(np.float32)
    from rkifield_b200 import scenes
    p = scenes.march_params(small_scene["spec"])
    for mode in (abi.RKF_TRACE_SHADOW, abi.RKF_TRACE_ANY, abi.RKF_TRACE_CLOSEST):
        ref = oracle.trace(sc, o.ravel(), d.ravel(), tmax, mode, p)
        got = small_ctx.trace(o.ravel(), d.ravel(), tmax, mode, p)
        for k in ("t", "flags"):
            assert_bits_equal(got[k], ref[k], f"mode {mode} {k}")


@pytest.mark.parametrize("bands", [0, 3])
def test_inside_views_heaviest_tiles_first_bit_exact(oracle, small_scene, bands):
    """The same inside views with the views' tiles handed out heaviest first
    (rkf_batch_tuning.order_tiles): identical to the oracle through device
    outputs and through host outputs marched in bands (each band ordered
    among its own rows)."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import cudart, scenes
    from rkifield_b200.engine import Context
    spec = small_scene["spec"]
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    ctx = Context(pool_capacity=max(v.n_bricks + 4096, 1 << 15))
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        ctx.upload_objects([small_scene["obj"]])
        tu = abi.rkf_batch_tuning()
        tu.tile_w, tu.tile_h, tu.compact_interval, tu.order_tiles = 8, 4, 128, 1
        ctx.set_tuning(tu)
        assert ctx.tuning().order_tiles == 1
        p = scenes.march_params(spec)
        if bands:
            ctx.lib.rkf_testing_set_host_bands(bands)
        for seed in (21, 24):
            w, h = 240, 136
            cam = scenes.seeded_camera(spec, w, h, seed=seed, inside=True)
            ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
            got = ctx.march(cam, p, w, h, reference_planes=True)
            assert ctx.lib.rkf_testing_last_variant(ctx.h) == 2
            for k in PLANES:
                assert_bits_equal(got[k], ref[k], f"seed {seed} bands {bands} {k}")
            if not bands:
                g = cudart.device_gbuffer(w * h, reference_planes=True)
                ctx.march_device(cam, p, w, h, cudart.gbuffer_ptrs(g))
                for k in PLANES:
                    assert_bits_equal(g[k].download(), ref[k], f"device outputs seed {seed} {k}")
    finally:
        ctx.lib.rkf_testing_set_host_bands(-1)
        ctx.close()
