"""A batched march captured as a CUDA graph (rkf_batch_graph_*): each launch
writes the same planes as rkf_march_batch on the same views and ray batches,
bit for bit; new cameras between launches take effect; a scene change makes
the graph stale; strategies other than brute are refused."""
import ctypes as C

import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

SIZES = [(96, 64), (0, 0), (200, 136), (33, 17)]  # one empty view


def _views(cams):
    from rkifield_b200 import _abi as abi, cudart
    vs = (abi.rkf_view * len(SIZES))()
    bufs = []
    for i, ((w, h), cam) in enumerate(zip(SIZES, cams)):
        g = cudart.device_gbuffer(max(1, w * h), reference_planes=True)
        bufs.append(g)
        vs[i].camera = cam
        vs[i].width, vs[i].height = w, h
        for k, a in g.items():
            setattr(vs[i].out, k, a.ptr)
        vs[i].out.mem = abi.RKF_MEM_DEVICE
    return vs, bufs


def _rays(seed):
    from rkifield_b200 import _abi as abi, cudart
    rng = np.random.default_rng(seed)
    n = 5000
    o = rng.uniform(-20, 20, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    tm = np.full(n, 40.0, np.float32)
    ins = [cudart.DeviceArray(3 * n, np.float32).upload(o), cudart.DeviceArray(3 * n, np.float32).upload(d),
           cudart.DeviceArray(n, np.float32).upload(tm)]
    bs = (abi.rkf_ray_batch * 2)()
    outs = []
    for j, mode in enumerate((abi.RKF_TRACE_CLOSEST, abi.RKF_TRACE_SHADOW)):
        out = {"t": cudart.DeviceArray(n, np.float32), "flags": cudart.DeviceArray(n, np.uint16)}
        if mode == abi.RKF_TRACE_CLOSEST:
            out.update(normal=cudart.DeviceArray(3 * n, np.float32), slot=cudart.DeviceArray(n, np.uint32),
                       material=cudart.DeviceArray(n, np.uint16))
        outs.append(out)
        b = bs[j]
        b.origins, b.dirs, b.tmax, b.n, b.mode = ins[0].ptr, ins[1].ptr, ins[2].ptr, n, mode
        b.out.t, b.out.flags, b.out.mem = out["t"].ptr, out["flags"].ptr, abi.RKF_MEM_DEVICE
        if mode == abi.RKF_TRACE_CLOSEST:
            b.out.normal, b.out.slot, b.out.material = out["normal"].ptr, out["slot"].ptr, out["material"].ptr
    return bs, outs, ins


def _download(bufs, outs):
    got = []
    for (w, h), g in zip(SIZES, bufs):
        if w * h:
            got.append({k: a.download() for k, a in g.items()})
    for out in outs:
        got.append({k: a.download() for k, a in out.items()})
    return got


def _same(a, b, what):
    for x, y in zip(a, b):
        for k in x:
            assert_bits_equal(x[k], y[k], f"{what}: {k}")


def test_graph_launches_equal_the_batched_march(small_scene):
    from rkifield_b200 import _abi as abi, cudart, scenes
    from rkifield_b200.engine import Context, check
    v = small_scene["vox"]
    spec = small_scene["spec"]
    ctx = Context(pool_capacity=v.n_bricks + 1024)
    graph = C.c_void_p()
    try:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        ctx.upload_objects([small_scene["obj"]])
        lib = ctx.lib
        p = scenes.march_params(spec)
        cams_a = [scenes.seeded_camera(spec, max(w, 1), max(h, 1), seed=40 + i) for i, (w, h) in enumerate(SIZES)]
        cams_b = [scenes.seeded_camera(spec, max(w, 1), max(h, 1), seed=60 + i) for i, (w, h) in enumerate(SIZES)]
        gv, gbufs = _views(cams_a)
        gb, gouts, gins = _rays(7)
        rv, rbufs = _views(cams_a)
        rb, routs, _ = _rays(7)

        check(lib.rkf_batch_graph_create(ctx.h, gv, len(SIZES), gb, 2, C.byref(p), None, C.byref(graph)),
              "rkf_batch_graph_create")
        check(lib.rkf_batch_graph_launch(graph, None), "rkf_batch_graph_launch")
        check(lib.rkf_march_batch(ctx.h, rv, len(SIZES), rb, 2, C.byref(p), None), "rkf_march_batch")
        cudart.synchronize()
        first = _download(gbufs, gouts)
        _same(first, _download(rbufs, routs), "graph vs batch")
        assert ((first[0]["flags"] & 1) != 0).sum() > 100

        # a second launch with nothing changed writes the same planes
        for a in gbufs[0].values():
            a.memset(0)
        cudart.synchronize()
        check(lib.rkf_batch_graph_launch(graph, None), "rkf_batch_graph_launch")
        cudart.synchronize()
        _same(_download(gbufs, gouts), first, "second launch")

        # new cameras take effect on the next launch
        cams = (abi.rkf_camera * len(SIZES))(*cams_b)
        check(lib.rkf_batch_graph_set_cameras(graph, cams, len(SIZES)), "rkf_batch_graph_set_cameras")
        check(lib.rkf_batch_graph_launch(graph, None), "rkf_batch_graph_launch")
        rv2, rbufs2 = _views(cams_b)
        check(lib.rkf_march_batch(ctx.h, rv2, len(SIZES), rb, 2, C.byref(p), None), "rkf_march_batch")
        cudart.synchronize()
        moved = _download(gbufs, gouts)
        _same(moved, _download(rbufs2, routs), "graph vs batch, new cameras")
        assert not np.array_equal(moved[0]["t"], first[0]["t"]), "the cameras changed the views"
        assert lib.rkf_batch_graph_set_cameras(graph, cams, 2) == abi.RKF_INVALID_ARG

        # a scene change makes the graph stale
        ctx.upload_objects([small_scene["obj"]])
        assert lib.rkf_batch_graph_launch(graph, None) == abi.RKF_EPOCH_STALE
        lib.rkf_batch_graph_destroy(graph)
        graph = C.c_void_p()

        tiled = scenes.march_params(spec)
        tiled.strategy = abi.RKF_STRATEGY_TILED
        assert lib.rkf_batch_graph_create(ctx.h, gv, len(SIZES), gb, 2, C.byref(tiled), None,
                                          C.byref(graph)) == abi.RKF_UNSUPPORTED
        assert not graph.value
    finally:
        if graph.value:
            ctx.lib.rkf_batch_graph_destroy(graph)
        ctx.close()
