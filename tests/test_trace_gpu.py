"""GPU parity of ray casts, point queries and the batched march.

Ray casts in the three modes (closest hit = the full march of
ray_march.wgsl:776-858 with normals and material; any hit; soft shadow of
shade_common_shading.wgsl:9-33) and point queries (SdfQueryable over the
pool, sdf_collision.rs:38-56) are compared bit for bit with the FP32 oracle.
The batched launch must return exactly what separate calls return.
"""
import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu


def _rays(n, seed, box=18.0, zero_components=True):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-box, box, (n, 3)).astype(np.float32)
    d = rng.standard_normal((n, 3)).astype(np.float32)
    if zero_components:  # axis-aligned rays exercise the 1e-10 safe direction
        d[: n // 16, 1] = 0.0
        d[n // 16: n // 8, 0] = 0.0
        d[n // 8: n // 8 + 8] = np.float32([0, 0, 1])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = rng.uniform(1.0, 60.0, n).astype(np.float32)
    return o, d, tmax


@pytest.mark.parametrize("mode", [0, 1, 2], ids=["closest", "any", "shadow"])
def test_trace_rays_bit_exact(oracle, small_scene, small_ctx, mode):
    from rkifield_b200 import scenes
    spec = small_scene["spec"]
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    o, d, tmax = _rays(20000, seed=mode + 1)
    p = scenes.march_params(spec)
    ref = oracle.trace(sc, o.ravel(), d.ravel(), tmax, mode, p)
    got = small_ctx.trace(o, d, tmax, mode, p)
    assert_bits_equal(got["t"], ref["t"], "t")
    assert_bits_equal(got["flags"], ref["flags"], "flags")
    if mode == 0:
        for k in ("normal", "slot", "material"):
            assert_bits_equal(got[k], ref[k], k)
    hits = int((ref["flags"] & 1).sum())
    assert 100 < hits < 20000


@pytest.mark.parametrize("mode", [0, 1, 2], ids=["closest", "any", "shadow"])
@pytest.mark.parametrize("max_steps", [None, 0], ids=["default", "no_near_steps"])
def test_rays_ending_at_their_first_check(oracle, small_scene, small_ctx, mode, max_steps):
    """Rays whose tmax lies below their starting t (0, or 0.005 for soft
    shadows) end unhit at their first check; the kernel writes their outputs
    while refilling and hands the lane the next id.  Mixed with live rays
    (many such rays in a row, as the secondary rays of pixels that missed),
    with tmax just around the starting t, -0, NaN and infinity, and with a
    near-step limit of 0 (every ray then ends with STEPS_OUT): bit-exact
    with the oracle in every mode."""
    from rkifield_b200 import scenes
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    o, d, tmax = _rays(12000, seed=40 + mode)
    rng = np.random.default_rng(77)
    dead = rng.random(tmax.size) < 0.85
    tmax[dead] = -1.0
    special = np.float32([0.0, -0.0, 1e-30, -1e-30, 0.003, 0.005, 0.0051, np.nan, np.inf, -np.inf])
    tmax[:special.size] = special
    tmax[5000:8000] = -1.0  # a long run of them
    p = scenes.march_params(scenes.SCENE_SMALL)
    if max_steps is not None:
        p.scene.max_steps = max_steps
    ref = oracle.trace(sc, o.ravel(), d.ravel(), tmax, mode, p)
    got = small_ctx.trace(o, d, tmax, mode, p)
    for k in ref:
        if k in got:
            assert_bits_equal(got[k], ref[k], k)
    # also alone: every ray of a batch ends at once
    ref = oracle.trace(sc, o[:512].ravel(), d[:512].ravel(), np.full(512, -2.0, np.float32), mode, p)
    got = small_ctx.trace(o[:512], d[:512], np.full(512, -2.0, np.float32), mode, p)
    for k in ref:
        if k in got:
            assert_bits_equal(got[k], ref[k], "all ending at once " + k)


def test_trace_zero_rays(small_ctx):
    from rkifield_b200 import scenes
    out = small_ctx.trace(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32),
                          np.zeros(0, np.float32), 0, scenes.march_params(scenes.SCENE_SMALL))
    assert out["t"].size == 0


def test_query_points_bit_exact(oracle, small_scene, small_ctx):
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    rng = np.random.default_rng(9)
    pts = rng.uniform(-20, 20, (50000, 3)).astype(np.float32)
    # also points right on the band around surfaces: march hits
    d_ref, g_ref, m_ref = oracle.query_points(sc, pts.ravel())
    d, g, m = small_ctx.query_points(pts)
    assert_bits_equal(d, d_ref, "distance")
    assert_bits_equal(g, g_ref, "gradient")
    assert_bits_equal(m, m_ref, "material")
    assert (np.abs(d) < 0.5).sum() > 10


def test_batch_equals_separate_calls(small_scene, small_ctx):
    """Several uneven views and ray batches in one persistent launch give the
    same bits as separate calls."""
    import ctypes as C

    from rkifield_b200 import _abi as abi
    from rkifield_b200 import cudart, scenes
    spec = small_scene["spec"]
    p = scenes.march_params(spec)
    sizes = [(128, 72), (31, 200), (256, 256)]
    views = (abi.rkf_view * len(sizes))()
    gb = []
    refs = []
    for i, (w, h) in enumerate(sizes):
        cam = scenes.seeded_camera(spec, w, h, seed=60 + i)
        refs.append(small_ctx.march(cam, p, w, h))
        g = cudart.device_gbuffer(w * h)
        gb.append(g)
        views[i].camera = cam
        views[i].width, views[i].height = w, h
        for k, a in g.items():
            setattr(views[i].out, k, a.ptr)
        views[i].out.mem = abi.RKF_MEM_DEVICE
    o, d, tmax = _rays(5000, seed=77)
    ray_ref = [small_ctx.trace(o, d, tmax, m, p) for m in (0, 2)]
    ins = [cudart.DeviceArray(o.size, np.float32).upload(o.ravel()),
           cudart.DeviceArray(d.size, np.float32).upload(d.ravel()),
           cudart.DeviceArray(tmax.size, np.float32).upload(tmax)]
    batches = (abi.rkf_ray_batch * 2)()
    hb = []
    for j, m in enumerate((0, 2)):
        h = {"t": cudart.DeviceArray(5000, np.float32), "flags": cudart.DeviceArray(5000, np.uint16)}
        if m == 0:
            h.update(normal=cudart.DeviceArray(15000, np.float32), slot=cudart.DeviceArray(5000, np.uint32),
                     material=cudart.DeviceArray(5000, np.uint16))
        hb.append(h)
        batches[j].origins, batches[j].dirs, batches[j].tmax = ins[0].ptr, ins[1].ptr, ins[2].ptr
        batches[j].n, batches[j].mode = 5000, m
        for k, a in h.items():
            setattr(batches[j].out, k, a.ptr)
        batches[j].out.mem = abi.RKF_MEM_DEVICE
    # (tile_w, tile_h, step_budget, compact_interval, blocks_per_sm, threads_per_block, refill_idle,
    #  probe_in_run, no_empty_path, order_tiles, tail_share)
    for tu in (None, (16, 2, 0, 4, 0, 128, 0, 0), (4, 8, 0, 64, 1, 256, 0, 1), (8, 4, 3, 16, 0, 256, 32, 0),
               (4, 8, 200, 8, 0, 64, 1, 1), (8, 4, 0, 128, 0, 256, 0, 0, 0, 1), (16, 2, 24, 32, 0, 128, 8, 1, 0, 1),
               (8, 4, 32, 128, 0, 256, 32, 0, 0, 1, 4), (4, 8, 5, 16, 0, 128, 8, 0, 0, 0, 32),
               (8, 4, 0, 64, 0, 256, 0, 1, 0, 1, 32)):
        tuning = None
        if tu is not None:
            tuning = abi.rkf_batch_tuning(*tu)
        abi.check(small_ctx.lib.rkf_march_batch(small_ctx.h, views, len(sizes), batches, 2, C.byref(p),
                                                None if tuning is None else C.byref(tuning)), "batch")
        for g, r in zip(gb, refs):
            for k in r:
                assert_bits_equal(g[k].download(), r[k], f"view {k} tuning {tu}")
        for h, r in zip(hb, ray_ref):
            for k in h:
                assert_bits_equal(h[k].download(), r[k], f"rays {k} tuning {tu}")


def test_sdf_ao_bit_exact(oracle, small_scene, small_ctx):
    """sdf_ao (shade_common_shading.wgsl:37-47) at hit points offset by
    SHADOW_BIAS along their normals, as the shading pass calls it, and at
    random points of the scene box."""
    from rkifield_b200 import scenes
    v = small_scene["vox"]
    sc = oracle.Scene([small_scene["obj"]], pool_words=v.words, brick_maps=v.map)
    spec = small_scene["spec"]
    cam = scenes.seeded_camera(spec, 160, 120, seed=41)
    g = small_ctx.march(cam, scenes.march_params(spec), 160, 120, reference_planes=True)
    hit = (g["flags"] & 1) != 0
    assert hit.sum() > 500
    n = g["normal"].reshape(-1, 3)[hit]
    pos = g["position"].reshape(-1, 4)[hit, :3]
    pos = (pos + (n * np.float32(0.08)).astype(np.float32)).astype(np.float32)
    rng = np.random.default_rng(9)
    lo = np.array(small_scene["vp"].aabb_min[:], np.float32)
    hi = np.array(small_scene["vp"].aabb_max[:], np.float32)
    rp = rng.uniform(lo, hi, size=(4000, 3)).astype(np.float32)
    rn = rng.normal(size=(4000, 3))
    rn = (rn / np.linalg.norm(rn, axis=1, keepdims=True)).astype(np.float32)
    P = np.concatenate([pos, rp]).astype(np.float32)
    N = np.concatenate([n, rn]).astype(np.float32)
    ref = oracle.sdf_ao(sc, P, N)
    got = small_ctx.sdf_ao(P, N)
    assert ((ref > 0.0) & (ref < 1.0)).sum() > 100, "AO should vary"
    assert_bits_equal(got, ref, "sdf_ao")
