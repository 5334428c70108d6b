"""The batching workload at full size: the 64 uneven views of the benchmark
(pixel area log-uniform between 128^2 and 2048^2, each looking at a seeded
primitive of the 1.1 M-brick scene) with their soft-shadow and ambient-
occlusion rays.  Three of the views -- the smallest, the median and the
largest -- and their secondary rays go through one batched launch
(rkf_march_batch) and through the same batch captured as a CUDA graph.  Every
pixel of the three views and 20,000 of their secondary rays are compared bit
for bit with the FP32 oracle on the same pool planes and index; the graph's
outputs must equal the direct call's."""
import ctypes as C

import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

PLANES = ("t", "normal", "slot", "material", "flags")


def _device_view(abi, cudart, v):
    g = cudart.device_gbuffer(v.width * v.height)
    rv = abi.rkf_view()
    rv.camera = v.cam
    rv.width, rv.height = v.width, v.height
    for k, a in g.items():
        setattr(rv.out, k, a.ptr)
    rv.out.mem = abi.RKF_MEM_DEVICE
    return rv, g


def test_batch_views_and_secondaries_bit_exact(oracle, large, large_oracle):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import cudart, scenes, workloads
    from rkifield_b200.engine import BatchGraph
    ctx, spec, _, p = large
    prims = scenes.make_prims(spec)
    views = workloads.make_views(spec, prims, 64, seed=300)  # the benchmark's batching views
    areas = np.array([v.width * v.height for v in views])
    order = np.argsort(areas, kind="stable")
    pick = [views[i] for i in (order[0], order[len(order) // 2], order[-1])]
    assert pick[-1].width * pick[-1].height > 1_000_000
    lib = ctx.lib
    vs = (abi.rkf_view * 3)()
    gbufs = []
    for i, v in enumerate(pick):
        vs[i], g = _device_view(abi, cudart, v)
        gbufs.append(g)
    # primaries first: the secondary rays start at their hits
    abi.check(lib.rkf_march_batch(ctx.h, vs, 3, None, 0, C.byref(p), None), "primaries")
    rng = np.random.default_rng(17)
    batches = (abi.rkf_ray_batch * 6)()
    keep, outs, rays = [], [], []
    for i, v in enumerate(pick):
        npx = v.width * v.height
        g = gbufs[i]
        target = np.array(v.cam.position[:3], np.float64) + 8.0 * np.array(v.cam.forward[:3], np.float64)
        lights = (target[None] + rng.uniform(-10, 10, (4, 3)) + np.array([0.0, 8.0, 0.0])).astype(np.float32)
        arrs = [cudart.DeviceArray(3 * 4 * npx, np.float32), cudart.DeviceArray(3 * 4 * npx, np.float32),
                cudart.DeviceArray(4 * npx, np.float32), cudart.DeviceArray(3 * 8 * npx, np.float32),
                cudart.DeviceArray(3 * 8 * npx, np.float32), cudart.DeviceArray(8 * npx, np.float32)]
        keep.append(arrs)
        hits = C.c_uint32()
        gb = abi.rkf_gbuffer()
        gb.t, gb.normal, gb.flags, gb.mem = g["t"].ptr, g["normal"].ptr, g["flags"].ptr, abi.RKF_MEM_DEVICE
        abi.check(lib.rkf_secondary_rays(ctx.h, C.byref(v.cam), v.width, v.height, C.byref(gb), lights.ctypes.data,
                                         4, 8, 1.0, 300 * 1000 + i, *[a.ptr for a in arrs], C.byref(hits), None),
                  "secondary rays")
        assert hits.value > 0
        for j, (o, d, t, nper, mode) in enumerate(((arrs[0], arrs[1], arrs[2], 4, abi.RKF_TRACE_SHADOW),
                                                   (arrs[3], arrs[4], arrs[5], 8, abi.RKF_TRACE_ANY))):
            out = {"t": cudart.DeviceArray(nper * npx, np.float32), "flags": cudart.DeviceArray(nper * npx, np.uint16)}
            outs.append(out)
            rays.append((o, d, t, mode))
            b = batches[2 * i + j]
            b.origins, b.dirs, b.tmax, b.n, b.mode = o.ptr, d.ptr, t.ptr, nper * npx, mode
            b.out.t, b.out.flags, b.out.mem = out["t"].ptr, out["flags"].ptr, abi.RKF_MEM_DEVICE
    prim_ref = [{k: a.download() for k, a in g.items()} for g in gbufs]
    for g in gbufs:
        for a in g.values():
            a.memset(0xA5)
    # the whole batch: three views and six secondary batches in one launch
    abi.check(lib.rkf_march_batch(ctx.h, vs, 3, batches, 6, C.byref(p), None), "batch")
    got_views = [{k: a.download() for k, a in g.items()} for g in gbufs]
    got_rays = [{k: a.download() for k, a in o.items()} for o in outs]
    for i, v in enumerate(pick):
        for k in PLANES:
            assert_bits_equal(got_views[i][k], prim_ref[i][k], f"view {i} {k}: batch vs primaries alone")
        ref = oracle.march(large_oracle, v.cam, p, v.width, v.height)
        for k in PLANES:
            assert_bits_equal(got_views[i][k], ref[k], f"view {i} ({v.width}x{v.height}) {k}")
    # 20,000 live secondary rays against the oracle: 10,000 shadow, 10,000 AO
    for mode, quota in ((abi.RKF_TRACE_SHADOW, 10_000), (abi.RKF_TRACE_ANY, 10_000)):
        idx = [j for j, r in enumerate(rays) if r[3] == mode]  # smallest view first
        checked = 0
        for n_left, j in zip(range(len(idx), 0, -1), idx):
            o, d, t, _ = rays[j]
            tm = t.download()
            live = np.nonzero(tm > 0)[0]
            per = (quota - checked) // n_left  # what a smaller view lacks, a larger one makes up
            sel = live if live.size <= per else np.sort(rng.choice(live, per, replace=False))
            oo = o.download().reshape(-1, 3)[sel]
            dd = d.download().reshape(-1, 3)[sel]
            ref = oracle.trace(large_oracle, oo.ravel(), dd.ravel(), tm[sel], mode, p)
            for k in ("t", "flags"):
                assert_bits_equal(got_rays[j][k][sel], ref[k], f"batch {j} mode {mode} {k}")
            checked += sel.size
        assert checked >= quota * 0.9
    # the same batch replayed from a CUDA graph: identical outputs
    for g in gbufs:
        for a in g.values():
            a.memset(0x5A)
    for o in outs:
        for a in o.values():
            a.memset(0x5A)
    stream = cudart.Stream()
    graph = BatchGraph(ctx, vs, batches, p)
    try:
        graph.launch(stream.ptr)
        stream.synchronize()
    finally:
        graph.close()
    for i in range(3):
        for k, a in gbufs[i].items():
            assert_bits_equal(a.download(), got_views[i][k], f"graph view {i} {k}")
    for j in range(6):
        for k, a in outs[j].items():
            assert_bits_equal(a.download(), got_rays[j][k], f"graph batch {j} {k}")
