"""Cameras and ray origins as WorldPositions far from the world origin.

The scene is uploaded relative to a scene origin a million chunks (8,000 km)
from the world origin, where an f32 coordinate resolves only about 1 m.  The
march entry points that take WorldPositions rebase them against the scene
origin in FP64 on the host (WorldPosition::relative_to_f64,
crates/rkf-core/src/world_position.rs:107-120) and round to f32 once: the
results equal the FP32 oracle's march from the rebased f32 camera and
origins bit for bit, while the naive route (absolute f32 metres, then a
subtraction) misplaces the camera by metres."""
import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

PLANES = ("t", "normal", "slot", "material", "flags", "position", "packed_material", "motion")
ORIGIN_CHUNK = (1_000_000, -1_000_000, 300_000)
ORIGIN_LOCAL = (1.5, 2.25, -3.0)


def _rebase(chunk, local):
    """relative_to_f64 against the scene origin, rounded to f32 (the library's
    rule: f32 difference of the local offsets, f64 sum with the chunk metres)."""
    chunk = np.asarray(chunk, np.int64).reshape(-1, 3)
    local = np.asarray(local, np.float32).reshape(-1, 3)
    dc = (chunk - np.asarray(ORIGIN_CHUNK, np.int64)).astype(np.float64) * 8.0
    dl = (local - np.asarray(ORIGIN_LOCAL, np.float32)).astype(np.float32).astype(np.float64)
    return (dc + dl).astype(np.float32)


def _world_of(rel):
    """A WorldPosition whose rebased f32 is close to rel: chunk offset by
    floor(rel / 8) from the origin's, local offset the rest."""
    rel = np.asarray(rel, np.float64).reshape(-1, 3)
    k = np.floor(rel / 8.0).astype(np.int64)
    chunk = np.asarray(ORIGIN_CHUNK, np.int64) + k
    local = (np.asarray(ORIGIN_LOCAL, np.float64) + rel - 8.0 * k).astype(np.float32)
    return chunk.astype(np.int32), local


def test_world_camera_and_rays_bit_exact(oracle, small_scene):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    spec = small_scene["spec"]
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    ctx = Context(pool_capacity=max(v.n_bricks + 4096, 1 << 15))
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        ctx.upload_objects([small_scene["obj"]])
        ctx.set_scene_origin(ORIGIN_CHUNK, ORIGIN_LOCAL)
        p = scenes.march_params(spec)
        w, h = 200, 120
        for seed in (11, 31):
            cam = scenes.seeded_camera(spec, w, h, seed=seed, inside=(seed == 31))
            chunk, local = _world_of(np.array(cam.position[:3], np.float64))
            rel = _rebase(chunk, local)[0]
            got = ctx.march_world(chunk[0], local[0], cam, p, w, h, reference_planes=True)
            cam_rel = abi.rkf_camera.from_buffer_copy(cam)
            cam_rel.position[0], cam_rel.position[1], cam_rel.position[2] = (float(x) for x in rel)
            ref = oracle.march(sc, cam_rel, p, w, h, with_reference_planes=True)
            assert (ref["flags"] & 1).sum() > 100
            for k in PLANES:
                assert_bits_equal(got[k], ref[k], f"seed {seed} {k}")
            # absolute f32 metres 8,000 km out resolve about a metre: the naive
            # camera lands far from the rebased one
            absolute = (np.asarray(chunk[0], np.float64) * 8.0 + local[0]).astype(np.float32)
            origin_abs = (np.asarray(ORIGIN_CHUNK, np.float64) * 8.0 + np.asarray(ORIGIN_LOCAL)).astype(np.float32)
            naive = (absolute - origin_abs).astype(np.float32)
            assert np.abs(naive.astype(np.float64) - rel).max() > 0.05
        # ray origins as WorldPositions
        rng = np.random.default_rng(9)
        n = 4000
        rel_o = rng.uniform(-14.0, 14.0, (n, 3))
        chunks, locals_ = _world_of(rel_o)
        d = rng.standard_normal((n, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        tmax = np.full(n, 30.0, np.float32)
        o32 = _rebase(chunks, locals_)
        for mode in (abi.RKF_TRACE_CLOSEST, abi.RKF_TRACE_ANY, abi.RKF_TRACE_SHADOW):
            got = ctx.trace_world(chunks, locals_, d, tmax, mode, p)
            ref = oracle.trace(sc, o32.ravel(), d.ravel(), tmax, mode, p)
            for k in got:
                assert_bits_equal(got[k], ref[k], f"world rays mode {mode} {k}")
        # the origin round-trips
        o = abi.rkf_world_pos()
        abi.check(ctx.lib.rkf_scene_origin_get(ctx.h, o), "origin")
        assert tuple(o.chunk) == ORIGIN_CHUNK and tuple(o.local) == ORIGIN_LOCAL
    finally:
        ctx.close()
