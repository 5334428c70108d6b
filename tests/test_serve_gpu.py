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


def _pool_state(ctx):
    import ctypes as C
    out = (C.c_uint32 * 5)()
    from rkifield_b200 import _abi as abi
    abi.check(ctx.lib.rkf_testing_pool_state(ctx.h, out), "rkf_testing_pool_state")
    cap, used, free, leaves, free_leaves = list(out)
    return {"capacity": cap, "used": used, "free": free, "held": cap - used - free, "leaves": leaves,
            "free_leaves": free_leaves}


def _run_soak(small_scene, reqs, concurrent: bool):
    """The stream through one session; returns the outputs, the results and
    the pool bookkeeping seen after every edit completes."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import scenes
    from rkifield_b200.engine import RkfError, Server
    ctx = _fresh_ctx(small_scene)
    srv = Server(ctx, scenes.march_params(small_scene["spec"]))
    results, outs, states = [None] * len(reqs), [None] * len(reqs), []
    live = {}
    i = 0
    try:
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
                    k = live.pop(t)
                    assert res["status"] == 0, (k, res)
                    results[k] = res
                    if not concurrent and reqs[k].kind == 3:
                        states.append(_pool_state(ctx))
        srv.stop()
        after = _pool_state(ctx)
    finally:
        ctx.close()
    return results, outs, states, after


def test_soak_reclaims_slots_and_leaves(small_scene):
    """5,000 requests with a CSG edit every 50th (100 edits, each retiring the
    bricks it rewrites).  Retired slots and leaves come back two edits later,
    so the slots held for older epochs stay within a few edits' worth while
    the session retires many times that; every request still equals its
    result alone (the reuse points depend on the order of edits only)."""
    from rkifield_b200 import workloads
    spec, prims = small_scene["spec"], small_scene["prims"]
    reqs = workloads.make_request_stream(spec, prims, 5000, seed=321, rate_hz=1e9, edit_every=50, ray_tmax=20.0,
                                         max_rays=1024, max_points=1024, render_area=(16 ** 2, 48 * 27))
    n_edits = sum(1 for r in reqs if r.kind == 3)
    assert n_edits == 100
    alone, ao, states, after_alone = _run_soak(small_scene, reqs, concurrent=False)
    mixed, mo, _, after_mixed = _run_soak(small_scene, reqs, concurrent=True)
    for i, r in enumerate(reqs):
        assert mixed[i]["epoch"] == alone[i]["epoch"], f"request {i} epoch"
        if r.kind == 3:
            continue
        for k in mo[i]:
            assert (mo[i][k].view(np.uint8) == ao[i][k].view(np.uint8)).all(), f"request {i} plane {k}"
    assert after_alone == after_mixed
    # A brush of radius <= 1 m plus its 0.05 m blend reaches at most 9 bricks
    # (0.32 m) and 2 index blocks (2.56 m) per axis.  Held slots are those the
    # last two edits retired, so at most 2 * 9^3; without reuse they would add
    # up over all 100 edits.  Leaves are appended only when none is free: a
    # handful of edits' worth in the whole session.
    held = [s["held"] for s in states]
    assert len(held) == n_edits
    assert 0 < max(held) <= 2 * 9 ** 3, held
    assert sum(1 for a, b in zip(held, held[1:]) if b < a) >= 10, held
    leaves = [s["leaves"] for s in states]
    assert leaves[-1] - leaves[0] <= 3 * 2 ** 3, leaves
    # after the session nothing is held
    assert after_alone["held"] == 0


def test_cancel_and_poll_timeout(small_scene):
    """rkf_cancel takes back a request that has not started (its result is
    RKF_CANCELLED and its budget returns); a running or finished request
    cannot be cancelled; rkf_poll with a timeout on an unfinished request
    returns RKF_TIMEOUT (None here) and the request still completes."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import engine, scenes
    from rkifield_b200.engine import RkfError, Server
    ctx = _fresh_ctx(small_scene)
    srv = Server(ctx, scenes.march_params(small_scene["spec"]))
    try:
        spec = small_scene["spec"]
        # a long request ahead keeps the next ones queued
        big_w, big_h = 1920, 1080
        big_out = engine.render_out(big_w * big_h)
        t_big = srv.submit_render(scenes.seeded_camera(spec, big_w, big_h, seed=3), big_w, big_h, big_out)
        rng = np.random.default_rng(4)
        pts = rng.uniform(-5, 5, (4096, 3)).astype(np.float32)
        queued = []
        for _ in range(40):
            out = engine.points_out(4096)
            queued.append((srv.submit_points(pts, out), out))
        cancelled = 0
        for t, _ in reversed(queued):
            try:
                srv.cancel(t)
                cancelled += 1
            except RkfError as e:
                assert e.status == abi.RKF_BUSY  # already running
        assert cancelled > 0, "some queued request should still be cancellable"
        # a poll with a 1 microsecond timeout on the long render: not done yet,
        # or done; either way the ticket stays valid until it is collected
        r0 = srv.poll(t_big, 1)
        res = r0 if r0 is not None else srv.poll(t_big, 60_000_000)
        assert res is not None and res["status"] == 0
        statuses = []
        for t, _ in queued:
            r = srv.poll(t, 60_000_000)
            assert r is not None
            statuses.append(r["status"])
        assert statuses.count(abi.RKF_CANCELLED) == cancelled
        assert all(s in (0, abi.RKF_CANCELLED) for s in statuses)
        # finished and collected tickets are unknown now
        with pytest.raises(RkfError) as e:
            srv.cancel(t_big)
        assert e.value.status == abi.RKF_INVALID_ARG
    finally:
        srv.stop()
        ctx.close()


def test_poll_timeout_status(small_scene):
    """rkf_poll returns RKF_TIMEOUT (not a result) when its wait ends before
    the request completes: a render queued behind another is polled with a
    1 microsecond limit right after submission."""
    import ctypes as C
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import engine, scenes
    from rkifield_b200.engine import Server
    ctx = _fresh_ctx(small_scene)
    srv = Server(ctx, scenes.march_params(small_scene["spec"]))
    try:
        spec = small_scene["spec"]
        outs, tks = [], []
        for s in range(3):
            o = engine.render_out(1920 * 1080)
            outs.append(o)
            tks.append(srv.submit_render(scenes.seeded_camera(spec, 1920, 1080, seed=5 + s), 1920, 1080, o))
        res = abi.rkf_result()
        st = ctx.lib.rkf_poll(ctx.h, tks[-1], C.byref(res), 1)
        assert st in (abi.RKF_TIMEOUT, abi.RKF_OK)
        if st == abi.RKF_OK:
            pytest.skip("the request completed within a microsecond")
        assert st == abi.RKF_TIMEOUT
        st = ctx.lib.rkf_poll(ctx.h, tks[-1], C.byref(res), 0)
        assert st in (abi.RKF_NOT_READY, abi.RKF_OK)
        for t in tks:
            if st == abi.RKF_OK and t == tks[-1]:
                continue
            assert srv.poll(t, 60_000_000)["status"] == 0
    finally:
        srv.stop()
        ctx.close()


def test_objects_update_between_sessions(small_scene):
    """The runtime's per-frame object upload (rkf_objects_update) is refused
    while a serving session runs (RKF_BUSY, nothing changes), and is taken
    between sessions: the next session renders the moved object exactly as
    the direct march does, and differently from before the move."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import engine, scenes
    from rkifield_b200.engine import RkfError, Server
    spec = small_scene["spec"]
    ctx = _fresh_ctx(small_scene)
    p = scenes.march_params(spec)
    w, h = 160, 96
    cam = scenes.seeded_camera(spec, w, h, seed=11)

    def served():
        srv = Server(ctx, p)
        try:
            out = engine.render_out(w * h)
            t = srv.submit_render(cam, w, h, out)
            res = srv.poll(t, 60_000_000)
            assert res is not None and res["status"] == 0
            return out
        finally:
            srv.stop()

    try:
        before = served()
        moved = abi.rkf_gpu_object.from_buffer_copy(small_scene["obj"])
        for a, d in enumerate((0.75, -0.5, 0.25)):  # inverse_world translation: the object moves by -d
            moved.inverse_world[12 + a] += d
            moved.aabb_min[a] -= d
            moved.aabb_max[a] -= d
        srv = Server(ctx, p)
        try:
            with pytest.raises(RkfError) as e:
                ctx.update_objects([moved])
            assert e.value.status == abi.RKF_BUSY
        finally:
            srv.stop()
        assert all((served()[k].view(np.uint8) == before[k].view(np.uint8)).all() for k in before)
        ctx.update_objects([moved])
        after = served()
        direct = ctx.march(cam, p, w, h)
        for k in after:
            assert (after[k].view(np.uint8) == direct[k].view(np.uint8)).all(), k
        assert not (after["t"].view(np.uint8) == before["t"].view(np.uint8)).all()
    finally:
        ctx.close()
