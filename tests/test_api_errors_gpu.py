"""Argument checks of the march entry points: each bad call returns its
documented status (and a message) before anything reaches the device, and
the context keeps working: a valid march after the refused calls gives the
same planes as before them."""
import ctypes as C

import pytest

from conftest import assert_bits_equal
from test_tiled_gpu import _analytic, _camera, _objects, _params

pytestmark = pytest.mark.gpu


def _status(fn):
    from rkifield_b200.engine import RkfError
    with pytest.raises(RkfError) as e:
        fn()
    assert str(e.value).split(": ")[-1], "a refused call carries a message"
    return e.value.status


def _view(cam, w, h, g):
    from rkifield_b200 import _abi as abi
    vw = (abi.rkf_view * 1)()
    vw[0].camera = cam
    vw[0].width, vw[0].height = w, h
    for k, a in g.items():
        setattr(vw[0].out, k, a.ptr)
    vw[0].out.mem = abi.RKF_MEM_DEVICE
    return vw


def test_march_argument_checks_leave_the_context_usable(small_scene):
    from rkifield_b200 import _abi as abi, cudart
    from rkifield_b200.engine import Context, Server, gbuffer_host
    v = small_scene["vox"]
    objs = _objects(small_scene)
    ctx = Context(pool_capacity=v.n_bricks + 1024)
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        w, h = 96, 64
        cam = _camera(3, w, h)
        p = _params(abi.RKF_STRATEGY_BRUTE)
        # no objects yet
        assert _status(lambda: ctx.march(cam, p, w, h)) == abi.RKF_INVALID_ARG
        ctx.upload_objects(objs)
        before = ctx.march(cam, p, w, h)

        small = gbuffer_host(16)  # the sizes are refused before any plane is touched
        assert _status(lambda: ctx.march(cam, p, 0, h, out=small)) == abi.RKF_INVALID_ARG
        assert _status(lambda: ctx.march(cam, p, 70000, 70000, out=small)) == abi.RKF_INVALID_ARG
        out = gbuffer_host(w * h)
        del out["normal"]
        assert _status(lambda: ctx.march(cam, p, w, h, out=out)) == abi.RKF_INVALID_ARG
        for field, value in (("hard_max_steps", 0), ("hard_max_steps", (1 << 20) + 1), ("bisect_steps", 65),
                             ("strategy", 7)):
            bad = _params(abi.RKF_STRATEGY_BRUTE)
            setattr(bad, field, value)
            assert _status(lambda: ctx.march(cam, bad, w, h)) == abi.RKF_INVALID_ARG, field

        # launch tuning of the batched entry point
        g = cudart.device_gbuffer(w * h)
        vw = _view(cam, w, h, g)
        for tile_w, tile_h, threads in ((0, 4, 256), (128, 64, 256), (8, 4, 100), (8, 4, 512)):
            tu = abi.rkf_batch_tuning(tile_w, tile_h, 32, 64, 0, threads, 32, 0)
            st = ctx.lib.rkf_march_batch(ctx.h, vw, 1, None, 0, C.byref(p), C.byref(tu))
            assert st == abi.RKF_INVALID_ARG, (tile_w, tile_h, threads)

        # paths that run the brute strategy only
        tiled = _params(abi.RKF_STRATEGY_TILED)
        assert _status(lambda: ctx.march(cam, tiled, w, h, plain=True)) == abi.RKF_UNSUPPORTED
        assert ctx.lib.rkf_march_batch_noalloc(ctx.h, vw, 1, None, 0, C.byref(tiled), None, None) \
            == abi.RKF_UNSUPPORTED
        assert _status(lambda: Server(ctx, tiled)) == abi.RKF_UNSUPPORTED

        after = ctx.march(cam, p, w, h)
        for k in before:
            assert_bits_equal(after[k], before[k], f"after refused calls: {k}")

        # more objects than the launch parameters hold: marched from the
        # device object table (tests/test_many_objects_gpu.py checks the
        # values), and the tiled strategy refuses more than its 256
        many = list(objs) + [_analytic(0, (40.0 + 3 * i, 0.0, 0.0), (1.0,), (1.0, 1.0, 1.0), 5, 10 + i)
                             for i in range(33 - len(objs))]
        ctx.upload_objects(many)
        g33 = ctx.march(cam, p, w, h)
        assert ctx.lib.rkf_testing_last_variant(ctx.h) == 0
        assert (g33["flags"] & 1).any()
        many = list(objs) + [_analytic(0, (40.0 + 3 * (i % 40), 3.0 * (i // 40), 0.0), (1.0,), (1.0, 1.0, 1.0), 5,
                                       10 + i % 200) for i in range(257 - len(objs))]
        ctx.upload_objects(many)
        assert _status(lambda: ctx.march(cam, tiled, w, h)) == abi.RKF_UNSUPPORTED
        ctx.upload_objects(objs)
        again = ctx.march(cam, p, w, h)
        for k in before:
            assert_bits_equal(again[k], before[k], f"after re-import: {k}")
    finally:
        ctx.close()
