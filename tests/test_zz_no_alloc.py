"""The allocation-free batched march, through the C ABI.

rkf_march_batch_noalloc exists for callers that must not allocate device
memory when they call: a renderer on a fixed per-frame time budget (cudaMalloc
synchronises the whole device) or an application whose framework owns every
device allocation.  It keeps its launch scratch in one fixed static device
array instead of context-owned buffers.  These tests check that it returns
exactly what rkf_march_batch returns on the same inputs, on two calls in a
row (the second call reuses the shared scratch left by the first), for one
voxelized object alone and beside analytic objects; that the device's free
memory is the same before and after those calls; and that it refuses more
work than its scratch can describe, refuses bad tunings and strategies,
and leaves a later call still exact.

The file is named to run last in a full test session and builds everything
it needs itself, so it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(with_analytic=False):
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    spec = scenes.SceneSpec("noalloc_prims16_cube8m_vs4cm", 16, 8.0, 0.04, seed=21)
    prims = scenes.make_prims(spec)
    ctx = Context(pool_capacity=1 << 15)
    ctx.voxelize(prims, scenes.voxelize_params(spec, prims))
    if with_analytic:
        # one voxelized object beside analytic ones: the multi-object kernels
        from test_tiled_gpu import _analytic
        ctx.update_objects([ctx.object(0),
                            _analytic(0, (6.0, 0.5, 0.0), (1.0,), (1.0, 1.0, 1.0), 5, 2),
                            _analytic(1, (-5.5, 1.0, 1.0), (0.8, 1.2, 0.6), (0.8, 1.2, 0.6), 6, 3),
                            _analytic(0, (40.0, 30.0, -20.0), (2.0,), (2.0, 2.0, 2.0), 8, 4)],
                           [0, -1, -1, -1])
    return spec, ctx


def _work(spec, ctx):
    """Two views of uneven size and two ray batches, all in device memory."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import cudart, scenes
    sizes = [(96, 40), (33, 65)]
    views = (abi.rkf_view * len(sizes))()
    gbufs = []
    for i, (w, h) in enumerate(sizes):
        g = cudart.device_gbuffer(w * h)
        gbufs.append(g)
        views[i].camera = scenes.seeded_camera(spec, w, h, seed=40 + i)
        views[i].width, views[i].height = w, h
        for k, v in g.items():
            setattr(views[i].out, k, v.ptr)
        views[i].out.mem = abi.RKF_MEM_DEVICE
    rng = np.random.default_rng(5)
    n = 3000
    o = rng.uniform(-5, 5, (n, 3)).astype(np.float32)
    d = rng.standard_normal((n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.full(n, 20.0, np.float32)
    inputs = [cudart.DeviceArray(3 * n, np.float32).upload(o.ravel()),
              cudart.DeviceArray(3 * n, np.float32).upload(d.ravel()),
              cudart.DeviceArray(n, np.float32).upload(tmax)]
    batches = (abi.rkf_ray_batch * 2)()
    hit_bufs = []
    for j, mode in enumerate((abi.RKF_TRACE_CLOSEST, abi.RKF_TRACE_SHADOW)):
        hb = {"t": cudart.DeviceArray(n, np.float32), "flags": cudart.DeviceArray(n, np.uint16)}
        if mode == abi.RKF_TRACE_CLOSEST:  # shadow rays return only t (the factor) and flags
            hb.update(normal=cudart.DeviceArray(3 * n, np.float32), slot=cudart.DeviceArray(n, np.uint32),
                      material=cudart.DeviceArray(n, np.uint16))
        hit_bufs.append(hb)
        b = batches[j]
        b.origins, b.dirs, b.tmax = inputs[0].ptr, inputs[1].ptr, inputs[2].ptr
        b.n, b.mode = n, mode
        for k, v in hb.items():
            setattr(b.out, k, v.ptr)
        b.out.mem = abi.RKF_MEM_DEVICE
    return views, batches, gbufs + hit_bufs, inputs


def _snapshot(bufs):
    return [{k: v.download() for k, v in b.items()} for b in bufs]


def _scramble(bufs):
    for b in bufs:
        for v in b.values():
            v.memset(0xA5)


def _free_bytes():
    from cuda.bindings import runtime as rt
    err, free, _total = rt.cudaMemGetInfo()
    assert err == rt.cudaError_t.cudaSuccess
    return int(free)


def _same_bits(a, b):
    if a.dtype.kind == "f":
        return (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    return a == b


@pytest.mark.parametrize("with_analytic", [False, True], ids=["one_object", "with_analytic_objects"])
def test_noalloc_batch_matches_allocating_batch_on_two_calls(with_analytic):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import cudart, scenes
    spec, ctx = _scene(with_analytic)
    try:
        views, batches, bufs, _keep = _work(spec, ctx)
        p = scenes.march_params(spec)
        lib = ctx.lib
        abi.check(lib.rkf_march_batch(ctx.h, views, len(views), batches, len(batches), C.byref(p), None),
                  "rkf_march_batch")
        ref = _snapshot(bufs)
        assert any((r["flags"] & 1).any() for r in ref), "the work should hit geometry"
        stream = cudart.Stream()
        free_before = None
        for call in range(2):
            _scramble(bufs)
            cudart.synchronize()
            abi.check(lib.rkf_march_batch_noalloc(ctx.h, views, len(views), batches, len(batches), C.byref(p),
                                                  None, stream.ptr), "rkf_march_batch_noalloc")
            stream.synchronize()
            if call == 0:
                # the first call on the device resolved the scratch's address;
                # from here on a call must leave the free memory unchanged
                free_before = _free_bytes()
            got = _snapshot(bufs)
            for r, g in zip(ref, got):
                for k in r:
                    same = _same_bits(r[k], g[k])
                    assert same.all(), f"call {call}: plane {k} differs in {int((~same).sum())} entries"
        assert _free_bytes() == free_before, "a call allocated device memory"
        if with_analytic:
            assert ctx.lib.rkf_testing_last_variant(ctx.h) == 4  # the multi-object empty-space kernel
    finally:
        ctx.close()


def test_noalloc_batch_rejects_more_segments_than_its_scratch():
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import scenes
    spec, ctx = _scene()
    try:
        n = abi_max = 64
        views = (abi.rkf_view * (n + 1))()
        p = scenes.march_params(spec)
        st = ctx.lib.rkf_march_batch_noalloc(ctx.h, views, abi_max + 1, None, 0, C.byref(p), None, None)
        assert st == abi.RKF_INVALID_ARG
        assert b"64" in ctx.lib.rkf_last_error()
    finally:
        ctx.close()


def test_noalloc_refused_calls_then_exact_again():
    """Calls refused for their block size or strategy return their status
    (they are checked before anything is enqueued on the shared scratch), and
    the next accepted call still returns exactly the first call's results."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import cudart, scenes
    spec, ctx = _scene()
    try:
        views, batches, bufs, _keep = _work(spec, ctx)
        p = scenes.march_params(spec)
        lib = ctx.lib
        abi.check(lib.rkf_march_batch_noalloc(ctx.h, views, len(views), batches, len(batches), C.byref(p),
                                              None, None), "rkf_march_batch_noalloc")
        cudart.synchronize()
        ref = _snapshot(bufs)
        bad = abi.rkf_batch_tuning()
        bad.tile_w, bad.tile_h, bad.threads_per_block = 8, 4, 48
        st = lib.rkf_march_batch_noalloc(ctx.h, views, 1, None, 0, C.byref(p), C.byref(bad), None)
        assert st == abi.RKF_INVALID_ARG
        ps = scenes.march_params(spec)
        ps.strategy = abi.RKF_STRATEGY_TILED
        st = lib.rkf_march_batch_noalloc(ctx.h, views, 1, None, 0, C.byref(ps), None, None)
        assert st == abi.RKF_UNSUPPORTED
        cudart.synchronize()
        _scramble(bufs)
        abi.check(lib.rkf_march_batch_noalloc(ctx.h, views, len(views), batches, len(batches), C.byref(p),
                                              None, None), "rkf_march_batch_noalloc")
        cudart.synchronize()
        for r, g in zip(ref, _snapshot(bufs)):
            for k in r:
                assert _same_bits(r[k], g[k]).all(), k
    finally:
        ctx.close()
