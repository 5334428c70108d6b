"""Error paths under injected allocation failures.

The failure is made on the host: ``rkf_testing_fail_allocation_after(n)``
lets n more device allocations through and makes the next one report
out-of-memory without calling cudaMalloc, so no GPU fault is involved.  Each
failing call must return RKF_OOM with a message and leave the context as it
was: after the failures, the same call succeeding produces a pool, an index
and a march that are bit-identical to a context that never failed."""
import ctypes as C

import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

MAX_INJECTIONS = 64


@pytest.fixture
def inject():
    from rkifield_b200 import _abi as abi
    lib = abi.load_library()
    yield lambda n: lib.rkf_testing_fail_allocation_after(C.c_longlong(n))
    lib.rkf_testing_fail_allocation_after(C.c_longlong(-1))


def _state(ctx, n_bricks):
    idx = ctx.export_index()
    info = ctx.info()
    pl = ctx.export_planes(0, n_bricks)
    return {"top": idx["top"], "leaves": idx["leaves"], "obj_top_info": idx["obj_top_info"],
            "dist": pl["dist"], "mat": pl["mat"], "blend": pl["blend"],
            "used": np.array([info["pool_bricks_used"], info["leaf_blocks"], info["num_objects"]])}


def _march(ctx, spec, seed=21):
    from rkifield_b200 import scenes
    cam = scenes.seeded_camera(spec, 128, 96, seed=seed)
    return ctx.march(cam, scenes.march_params(spec), 128, 96)


def _same(a, b, what):
    for k in a:
        assert_bits_equal(a[k], b[k], f"{what}: {k}")


def _new_ctx(small_scene):
    from rkifield_b200.engine import Context
    ctx = Context(pool_capacity=small_scene["vox"].n_bricks * 2 + 4096, keep_reference_pool=False)
    ctx.voxelize(small_scene["prims"], small_scene["vp"])
    return ctx


def _retry_until_ok(inject, call, check_unchanged):
    """Inject a failure at the 0th, 1st, ... allocation of ``call`` until it
    succeeds; every failure must be RKF_OOM and leave the context unchanged."""
    from rkifield_b200 import _abi as abi
    failures = 0
    for k in range(MAX_INJECTIONS):
        inject(k)
        try:
            result = call()
        except abi.RkfError as e:
            inject(-1)
            assert e.status == abi.RKF_OOM, str(e)
            assert "allocation" in str(e)
            failures += 1
            check_unchanged()
            continue
        inject(-1)
        return result, failures
    raise AssertionError(f"call still failing after {MAX_INJECTIONS} injected failures")


def test_create_reports_oom(inject, small_scene):
    from rkifield_b200 import _abi as abi
    from rkifield_b200.engine import Context
    n = small_scene["vox"].n_bricks + 1024
    _, failures = _retry_until_ok(inject, lambda: Context(pool_capacity=n).close(), lambda: None)
    assert failures >= 3  # every pool plane is its own allocation
    with pytest.raises(abi.RkfError):
        inject(0)
        Context(pool_capacity=n)
    inject(-1)
    Context(pool_capacity=n).close()


def test_voxelize_failure_rolls_back(inject, small_scene):
    from rkifield_b200 import scenes
    spec = small_scene["spec"]
    prims2 = small_scene["prims"][:12].copy()
    vp2 = scenes.voxelize_params(spec, prims2, object_id=2)
    n = small_scene["vox"].n_bricks * 2 + 1024
    ctx, fresh = _new_ctx(small_scene), _new_ctx(small_scene)
    try:
        # a failed call may have written free slots; compare the slots in use
        used0 = ctx.info()["pool_bricks_used"]
        before, img0 = _state(ctx, used0), _march(ctx, spec)
        assert (img0["flags"] & 1).sum() > 500

        def unchanged():
            _same(_state(ctx, used0), before, "after a failed voxelize")
            _same(_march(ctx, spec), img0, "march after a failed voxelize")

        _, failures = _retry_until_ok(inject, lambda: ctx.voxelize(prims2, vp2), unchanged)
        assert failures >= 5
        fresh.voxelize(prims2, vp2)
        _same(_state(ctx, n), _state(fresh, n), "voxelize after failures vs never failed")
        _same(_march(ctx, spec, 22), _march(fresh, spec, 22), "march after failures vs never failed")
    finally:
        ctx.close()
        fresh.close()


@pytest.mark.parametrize("kind", [0, 1])  # additive (new bricks), subtractive (copy-on-write)
def test_edit_failure_rolls_back(inject, small_scene, kind):
    from rkifield_b200 import _abi as abi
    spec = small_scene["spec"]
    n = small_scene["vox"].n_bricks * 2 + 1024
    prim = small_scene["prims"][3]
    p = prim["centre"]
    # additive: a sphere across the primitive's bound; subtractive: carve its centre
    dx = float(prim["bound_radius"]) + 0.3 if kind == 0 else 0.0
    op = abi.rkf_edit_op()
    op.object_index, op.edit_type, op.shape_type, op.falloff = 0, kind, 0, 1
    op.position[:] = [float(p[0]) + dx, float(p[1]), float(p[2])]
    op.rotation[:] = (0.0, 0.0, 0.0, 1.0)
    op.dimensions[:] = (0.6, 0.0, 0.0)
    op.strength, op.blend_k, op.material_id = 1.0, 0.05, 7
    ctx, fresh = _new_ctx(small_scene), _new_ctx(small_scene)
    try:
        used0 = ctx.info()["pool_bricks_used"]
        before, img0 = _state(ctx, used0), _march(ctx, spec)
        epoch0 = ctx.info()["epoch"]

        def unchanged():
            assert ctx.info()["epoch"] == epoch0
            _same(_state(ctx, used0), before, "after a failed edit")
            _same(_march(ctx, spec), img0, "march after a failed edit")

        _, failures = _retry_until_ok(inject, lambda: ctx.edit(op), unchanged)
        assert failures >= 2
        fresh.edit(op)
        after = _state(ctx, n)
        assert ctx.info()["epoch"] == epoch0 + 1, "the edit changed nothing"
        _same(after, _state(fresh, n), "edit after failures vs never failed")
        _same(_march(ctx, spec, 23), _march(fresh, spec, 23), "march after failures vs never failed")
    finally:
        ctx.close()
        fresh.close()
