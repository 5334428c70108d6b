"""How far the library's SHADOW mode and rkf_sdf_ao sit from the shading
pass's own sample_sdf (shade_common.wgsl:521-572), which reads the coarse
field wherever it exceeds 0.5 m and the objects' exact minimum elsewhere.

The library takes the exact minimum everywhere (the coarse value comes from
a texture unit's filter and cannot be pinned), and its outputs equal the
oracle's exact forms bit for bit (the -m gpu trace and AO tests).  Here the
oracle's two forms are compared on the multi-object scene, at the hit points
of views (offset by SHADOW_BIAS along the normal, as the shading pass calls
them) with shadow rays toward three lights: the penumbra term only reacts
to distances below 0.02 m and blocking to 0.005 m, both inside the 0.5 m
band where the two forms agree, so the coarse field only changes the step
lengths in open space.  Bounds: the same blocked/lit decision for every
ray, shadow values within 5e-3, AO within 1e-5."""
import numpy as np

from test_tiled_gpu import _camera, _objects


def test_shadow_and_ao_bounded_against_the_coarse_sample_sdf(oracle, small_scene):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import scenes
    v = small_scene["vox"]
    sc = oracle.Scene(_objects(small_scene), pool_words=v.words, brick_maps=v.map)
    p = scenes.march_params(scenes.SCENE_SMALL)
    p.scene.max_distance = 200.0
    n_rays = worst_shadow = worst_ao = 0.0
    for seed in (3, 5):
        w, h = 160, 108
        cam = _camera(seed, w, h)
        g = oracle.march(sc, cam, p, w, h, with_reference_planes=True)
        hit = (g["flags"] & 1) != 0
        assert hit.sum() > 400
        nrm = g["normal"].reshape(-1, 3)[hit]
        q = (g["position"].reshape(-1, 4)[hit][:, :3] + nrm * np.float32(0.08)).astype(np.float32)
        cp = np.array(cam.position[:3], np.float32)
        worst_ao = max(worst_ao, float(np.abs(oracle.sdf_ao(sc, q, nrm) - oracle.sdf_ao_shader(sc, q, nrm, cp)).max()))
        for light in ((0.4, 0.8, 0.3), (-0.9, 0.2, 0.1), (0.95, 0.1, -0.2)):
            ld = np.array(light, np.float32)
            ld /= np.linalg.norm(ld)
            dirs = np.tile(ld, (len(q), 1)).astype(np.float32)
            tmax = np.full(len(q), 150.0, np.float32)
            exact = oracle.trace(sc, q.ravel(), dirs.ravel(), tmax, abi.RKF_TRACE_SHADOW, p)["t"]
            shader = oracle.shadow_shader(sc, q, dirs, tmax, cp)
            assert ((exact == 0) == (shader == 0)).all(), f"seed {seed} light {light}: blocked rays differ"
            assert 0.02 < (exact > 0).mean() < 0.98, "both lit and blocked rays"
            worst_shadow = max(worst_shadow, float(np.abs(exact - shader).max()))
            n_rays += len(q)
    assert n_rays > 3000
    assert worst_shadow <= 5e-3, worst_shadow
    assert worst_ao <= 1e-5, worst_ao
