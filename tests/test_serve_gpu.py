"""The resident request loop: continuous batching with interleaved edits.

A mixed stream of renders, ray batches and point queries with CSG edits
between them is submitted as fast as admission allows, so requests overlap on
the device.  Every request's result must equal, bit for bit, its result when
run alone at the same index epoch (a fresh context replaying the same
admissions one at a time)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(spec, prims, n, seed):
    from rkifield_b200 import workloads
    reqs = workloads.make_request_stream(spec, prims, n, seed, rate_hz=1e9, edit_every=7, ray_tmax=20.0,
                                         max_rays=20000, max_points=20000, render_area=(16 ** 2, 160 * 90))
    return reqs


def _fresh_ctx(small_scene):
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    ctx = Context(pool_capacity=v.n_bricks + 60000, mem_budget_bytes=256 << 20)
    ctx.set_brick_pool(v.words)
    ctx.upload_brick_maps(v.map)
    ctx.upload_objects([small_scene["obj"]])
    return ctx


def _submit(srv, r):
    from rkifield_b200 import engine
    if r.kind == 0:
        out = engine.render_out(r.width * r.height)
        return srv.submit_render(r.cam, r.width, r.height, out), out
    if r.kind == 1:
        out = engine.rays_out(r.n, 0)
        return srv.submit_rays(r.o, r.d, r.tmax, 0, out), out
    if r.kind == 2:
        out = engine.points_out(r.n)
        return srv.submit_points(r.points, out), out
    return srv.submit_edit(r.edit), None


def _run(small_scene, reqs, concurrent: bool):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import scenes
    from rkifield_b200.engine import RkfError, Server
    ctx = _fresh_ctx(small_scene)
    srv = Server(ctx, scenes.march_params(small_scene["spec"]))
    results = [None] * len(reqs)
    outs = [None] * len(reqs)
    live = {}
    i = 0
    while i < len(reqs) or live:
        while i < len(reqs):
            try:
                t, out = _submit(srv, reqs[i])
            except RkfError as e:
                assert e.status == abi.RKF_BUSY
                break
            live[t] = i
            outs[i] = out
            i += 1
            if not concurrent:
                break
        for t in list(live):
            res = srv.poll(t, 0 if concurrent else 10_000_000)
            if res is not None:
                assert res["status"] == 0, res
                results[live.pop(t)] = res
    srv.stop()
    ctx.close()
    return results, outs


def test_results_alone_equal_results_in_the_mix(small_scene):
    spec, prims = small_scene["spec"], small_scene["prims"]
    reqs = _requests(spec, prims, 60, seed=123)
    assert any(r.kind == 3 for r in reqs)
    mixed, mo = _run(small_scene, reqs, concurrent=True)
    alone, ao = _run(small_scene, reqs, concurrent=False)
    for i, r in enumerate(reqs):
        assert mixed[i]["epoch"] == alone[i]["epoch"], f"request {i} epoch"
        if r.kind == 3:
            continue
        for k in mo[i]:
            a, b = mo[i][k], ao[i][k]
            same = (a.view(np.uint8) == b.view(np.uint8)).all()
            assert same, f"request {i} (kind {r.kind}) plane {k} differs alone vs in the mix"
    # the mix overlapped: some request started before an earlier one finished
    starts = [m["start_us"] for m in mixed]
    ends = [m["done_us"] for m in mixed]
    assert any(starts[j] < ends[i] for i in range(len(reqs)) for j in range(i + 1, len(reqs)))


def test_admission_budget_and_cancel(small_scene):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import engine, scenes
    from rkifield_b200.engine import RkfError, Server
    ctx = _fresh_ctx(small_scene)
    srv = Server(ctx, scenes.march_params(small_scene["spec"]))
    try:
        big = 4096 * 4096  # 24 B/px of outputs: beyond the 256 MiB budget
        with pytest.raises(RkfError) as e:
            srv.submit_render(scenes.seeded_camera(small_scene["spec"], 4096, 4096, seed=1), 4096, 4096,
                              engine.render_out(1))
        assert e.value.status == abi.RKF_BUSY
        # a malformed request is refused without touching the loop
        with pytest.raises(RkfError) as e:
            srv.submit_rays(np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(1, np.float32), 7,
                            engine.rays_out(1, 0))
        assert e.value.status == abi.RKF_INVALID_ARG
        del big
    finally:
        srv.stop()
        ctx.close()
