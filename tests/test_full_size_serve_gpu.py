"""The serving workload at full size: 200 requests of the benchmark's mix
(renders, ray batches, point queries) on the 1.1 M-brick scene with a CSG
sphere edit every 50th request.  Run once one request at a time and once as
fast as admission allows (requests overlapping on the device): every result
must be bit-identical between the two, and every 10th request's result must
equal the FP32 oracle's on the pool planes and index of that request's epoch
(exported from the one-at-a-time session after each edit)."""
import numpy as np
import pytest

from conftest import assert_bits_equal, oracle_scene_of

pytestmark = pytest.mark.gpu


def _start(spec, prims):
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context, Server
    ctx = Context(pool_capacity=3_000_000, keep_reference_pool=False, mem_budget_bytes=2 << 30)
    ctx.voxelize(prims, scenes.voxelize_params(spec, prims))
    return ctx, Server(ctx, scenes.march_params(spec))


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


def _check(oracle, sc, p, k, r, out):
    from rkifield_b200 import _abi as abi
    if r.kind == 0:
        ref = oracle.march(sc, r.cam, p, r.width, r.height)
        for name in ("t", "normal", "slot", "material", "flags"):
            assert_bits_equal(out[name], ref[name], f"request {k} render {name}")
    elif r.kind == 1:
        ref = oracle.trace(sc, r.o.ravel(), r.d.ravel(), r.tmax, abi.RKF_TRACE_CLOSEST, p)
        for name in ("t", "normal", "slot", "material", "flags"):
            assert_bits_equal(out[name], ref[name], f"request {k} rays {name}")
    else:
        d, g, m = oracle.query_points(sc, r.points.ravel())
        assert_bits_equal(out["dist"], d, f"request {k} points dist")
        assert_bits_equal(out["grad"], g, f"request {k} points grad")
        assert_bits_equal(out["material"], m, f"request {k} points material")


def test_large_serving_alone_equals_mix_and_oracle(oracle, large):
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import scenes, workloads
    from rkifield_b200.engine import RkfError
    _, spec, _, p = large
    prims = scenes.make_prims(spec)
    reqs = workloads.make_request_stream(spec, prims, 200, seed=500, rate_hz=1e9, edit_every=50,
                                         max_rays=100_000, max_points=65_536, render_area=(64 ** 2, 480 * 270))
    assert sum(r.kind == 3 for r in reqs) == 4

    # one request at a time; the oracle scene follows the session's epochs
    ctx, srv = _start(spec, prims)
    res_alone, outs_alone, checked = [], [], 0
    try:
        sc, epoch = oracle_scene_of(oracle, ctx), ctx.info()["epoch"]
        epoch0 = epoch
        for k, r in enumerate(reqs):
            t, out = _submit(srv, r)
            res = srv.poll(t, 120_000_000)
            assert res is not None and res["status"] == 0, (k, res)
            res_alone.append(res)
            outs_alone.append(out)
            if r.kind == 3:
                sc = None
                sc, epoch = oracle_scene_of(oracle, ctx), res["epoch"]
            elif k % 10 == 0:
                assert res["epoch"] == epoch, k
                _check(oracle, sc, p, k, r, out)
                checked += 1
        assert epoch == epoch0 + 4
    finally:
        srv.stop()
        ctx.close()
    assert checked >= 15

    # the same requests overlapping on the device
    ctx, srv = _start(spec, prims)
    res_mix, outs_mix, live, i = [None] * len(reqs), [None] * len(reqs), {}, 0
    try:
        while i < len(reqs) or live:
            while i < len(reqs):
                try:
                    t, out = _submit(srv, reqs[i])
                except RkfError as e:
                    assert e.status == abi.RKF_BUSY
                    break
                live[t], outs_mix[i] = i, out
                i += 1
            for t in list(live):
                res = srv.poll(t, 0)
                if res is not None:
                    assert res["status"] == 0, res
                    res_mix[live.pop(t)] = res
    finally:
        srv.stop()
        ctx.close()
    for k, r in enumerate(reqs):
        assert res_mix[k]["epoch"] == res_alone[k]["epoch"], k
        if r.kind == 3:
            continue
        for name in outs_mix[k]:
            assert (outs_mix[k][name].view(np.uint8) == outs_alone[k][name].view(np.uint8)).all(), \
                f"request {k} (kind {r.kind}) plane {name}: alone vs mix"
    starts = [m["start_us"] for m in res_mix]
    ends = [m["done_us"] for m in res_mix]
    assert any(starts[j] < ends[i] for i in range(len(reqs)) for j in range(i + 1, len(reqs))), \
        "the mixed session should overlap requests"
