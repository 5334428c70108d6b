"""GPU parity of the march kernels against the FP32 oracle (bit-exact).

The oracle restates ray_march.wgsl (brute strategy, bisection, normals,
material/blend lookups, G-buffer packing); both CUDA kernels must reproduce
every output plane bit for bit on the same seeded scene and camera.
"""
import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

PLANES = ("t", "normal", "slot", "material", "flags", "position", "packed_material", "motion")


def _oracle_march(oracle, small_scene, cam, p, w, h):
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    return oracle.march(sc, cam, p, w, h, with_reference_planes=True)


@pytest.mark.parametrize("plain", [False, True], ids=["b200", "plain"])
@pytest.mark.parametrize("cam_seed", [11, 12])
def test_small_scene_view_bit_exact(oracle, small_scene, small_ctx, plain, cam_seed):
    from rkifield_b200 import scenes
    spec = small_scene["spec"]
    w, h = 256, 256
    cam = scenes.seeded_camera(spec, w, h, seed=cam_seed)
    p = scenes.march_params(spec)
    ref = _oracle_march(oracle, small_scene, cam, p, w, h)
    got = small_ctx.march(cam, p, w, h, reference_planes=True, plain=plain)
    hits = int((ref["flags"] & 1).sum())
    assert hits > 1000, "view should hit geometry"
    for k in PLANES:
        assert_bits_equal(got[k], ref[k], k)


def test_small_scene_non_square_and_ragged(oracle, small_scene, small_ctx):
    """Resolutions that are not multiples of the tile shape (edge tiles)."""
    from rkifield_b200 import scenes
    spec = small_scene["spec"]
    for (w, h) in [(97, 61), (1, 1), (33, 7)]:
        cam = scenes.seeded_camera(spec, w, h, seed=5)
        p = scenes.march_params(spec)
        ref = _oracle_march(oracle, small_scene, cam, p, w, h)
        got = small_ctx.march(cam, p, w, h, reference_planes=True)
        for k in PLANES:
            assert_bits_equal(got[k], ref[k], f"{k} @ {w}x{h}")


@pytest.mark.parametrize("precision", ["f16", "u8"])
def test_soa_import_matches_voxelsample_import(oracle, small_scene, small_ctx, precision):
    """The same pool given as SoA planes: identical planes, reference words
    and march (f16), and the same u8 codes as the word import (u8)."""
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    w = v.words.reshape(-1, 2)
    d16 = (w[:, 0] & 0xFFFF).astype(np.uint16)
    mat = (((w[:, 0] >> 16) & 0x3F) | (((w[:, 0] >> 22) & 0x3F) << 6)).astype(np.uint16)
    blend = (w[:, 1] >> 24).astype(np.uint8)
    cap = v.n_bricks + 1024
    a = Context(pool_capacity=cap, precision=precision)
    b = Context(pool_capacity=cap, precision=precision)
    try:
        for ctx in (a, b):
            ctx.upload_brick_maps(v.map)
        a.set_brick_pool_planes(d16, mat, blend)
        b.set_brick_pool(v.words)
        for ctx in (a, b):
            ctx.upload_objects([small_scene["obj"]])
        pa, pb = a.export_planes(0, v.n_bricks), b.export_planes(0, v.n_bricks)
        for k in pa:
            assert_bits_equal(pa[k], pb[k], f"{precision} plane {k}")
        assert a.info()["pool_bricks_used"] == b.info()["pool_bricks_used"] == v.n_bricks
        if precision == "f16":
            assert_bits_equal(a.export_pool(0, v.n_bricks), v.words, "reference words rebuilt from planes")
        spec = small_scene["spec"]
        cam = scenes.seeded_camera(spec, 128, 128, seed=17)
        p = scenes.march_params(spec)
        ga, gb = a.march(cam, p, 128, 128, reference_planes=True), b.march(cam, p, 128, 128, reference_planes=True)
        for k in PLANES:
            assert_bits_equal(ga[k], gb[k], f"{precision} march {k}")
    finally:
        a.close()
        b.close()


def test_objects_reimport_replaces_the_index(oracle, small_scene):
    """A second rkf_objects_import builds the index afresh: its top grid names
    leaf blocks of the new leaf buffer only, and the index and the march equal
    those of a context that imported the objects once."""
    from rkifield_b200 import _abi as abi, scenes
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    cap = v.n_bricks + 1024
    a = Context(pool_capacity=cap)
    b = Context(pool_capacity=cap)
    try:
        for ctx in (a, b):
            ctx.set_brick_pool(v.words)
            ctx.upload_brick_maps(v.map)
        a.upload_objects([small_scene["obj"]])
        a.upload_objects([small_scene["obj"]])
        b.upload_objects([small_scene["obj"]])
        ia, ib = a.export_index(), b.export_index()
        n_leaves = a.info()["leaf_blocks"]
        assert n_leaves == b.info()["leaf_blocks"] > 0
        leaf = ia["top"][ia["top"] < abi.INTERIOR_SLOT]
        assert leaf.size and int(leaf.max()) < n_leaves
        for k in ia:
            assert_bits_equal(ia[k], ib[k], f"index {k}")
        spec = small_scene["spec"]
        cam = scenes.seeded_camera(spec, 128, 96, seed=23)
        p = scenes.march_params(spec)
        ga, gb = a.march(cam, p, 128, 96), b.march(cam, p, 128, 96)
        for k in ga:
            assert_bits_equal(ga[k], gb[k], f"march {k}")
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("bands", [1, 2, 3, 8])
def test_host_output_bands_bit_exact(oracle, small_scene, small_ctx, bands):
    """rkf_march with host outputs marches large views in bands of tile rows
    whose copies overlap the next band: every band count gives the oracle's
    planes, on a height that is not a multiple of the tile height."""
    from rkifield_b200 import _abi as abi, scenes
    lib = abi.load_library()
    spec = small_scene["spec"]
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    w, h = 640, 429
    cam = scenes.seeded_camera(spec, w, h, seed=31)
    p = scenes.march_params(spec)
    lib.rkf_testing_set_host_bands(bands)
    try:
        got = small_ctx.march(cam, p, w, h, reference_planes=True)
    finally:
        lib.rkf_testing_set_host_bands(-1)
    ref = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
    assert ((ref["flags"] & 1) != 0).sum() > 1000
    for k in PLANES:
        assert_bits_equal(got[k], ref[k], f"{bands} bands {k}")
