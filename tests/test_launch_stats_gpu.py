"""Launch accounting of a context (rkf_testing_launch_stats).

Every kernel the library launches is counted: a view marched into device
planes is one persistent march launch, plus the three kernels of the
heaviest-first tile order (cost, scan, place) when that order is on.  With
march timing on, each persistent march launch is bracketed by CUDA events on
its stream; the benchmark divides the kernel's algorithmic bytes by those
times."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _stats(ctx, cap=0):
    n_launch, n_timed = C.c_uint64(0), C.c_uint32(0)
    ms = (C.c_float * max(cap, 1))()
    from rkifield_b200 import _abi as abi
    abi.check(ctx.lib.rkf_testing_launch_stats(ctx.h, C.byref(n_launch), ms, cap, C.byref(n_timed)), "stats")
    return int(n_launch.value), int(n_timed.value), [float(ms[i]) for i in range(min(cap, n_timed.value))]


def test_launch_counts_and_march_timing(small_scene):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import cudart, scenes
    from rkifield_b200.engine import Context
    spec = small_scene["spec"]
    v = small_scene["vox"]
    ctx = Context(pool_capacity=max(v.n_bricks + 4096, 1 << 15))
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        ctx.upload_objects([small_scene["obj"]])
        p = scenes.march_params(spec)
        w, h = 240, 136
        cam = scenes.seeded_camera(spec, w, h, seed=21, inside=True)
        g = cudart.device_gbuffer(w * h)
        ptrs = cudart.gbuffer_ptrs(g)
        per_view = {}
        for order in (0, 1):
            tu = abi.rkf_batch_tuning()
            tu.tile_w, tu.tile_h, tu.compact_interval, tu.order_tiles = 8, 4, 128, order
            ctx.set_tuning(tu)
            ctx.march_device(cam, p, w, h, ptrs)  # first march: any lazy set-up
            n0, _, _ = _stats(ctx)
            for _ in range(3):
                ctx.march_device(cam, p, w, h, ptrs)
            n1, _, _ = _stats(ctx)
            assert ctx.lib.rkf_testing_last_variant(ctx.h) == 2  # the empty-space path
            per_view[order] = (n1 - n0) / 3
        assert per_view == {0: 1.0, 1: 4.0}
        # timing: one event pair per persistent march launch, nothing before
        # it is switched on, and the list restarts when it is switched on again
        abi.check(ctx.lib.rkf_testing_march_timing(ctx.h, 1), "timing on")
        _, n_timed, _ = _stats(ctx)
        assert n_timed == 0
        for _ in range(5):
            ctx.march_device(cam, p, w, h, ptrs)
        _, n_timed, ms = _stats(ctx, 8)
        assert n_timed == 5 and len(ms) == 5
        assert all(0.0 < m < 1000.0 for m in ms), ms
        _, _, ms2 = _stats(ctx, 2)  # fewer than timed: the first ones
        assert ms2 == ms[:2]
        abi.check(ctx.lib.rkf_testing_march_timing(ctx.h, 1), "timing restart")
        ctx.march_device(cam, p, w, h, ptrs)
        assert _stats(ctx, 8)[1] == 1
        abi.check(ctx.lib.rkf_testing_march_timing(ctx.h, 0), "timing off")
        ctx.march_device(cam, p, w, h, ptrs)
        assert _stats(ctx, 8)[1] == 0
        assert ctx.lib.rkf_testing_march_timing(ctx.h, 2) == abi.RKF_INVALID_ARG
        # the plain march counts too (one launch per view)
        n0, _, _ = _stats(ctx)
        ctx.march_device(cam, p, w, h, ptrs, plain=True)
        assert _stats(ctx)[0] - n0 == 1
    finally:
        ctx.close()
