"""pytest configuration: the `gpu` marker and shared fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import binding
    binding.lib()
    return binding


@pytest.fixture(scope="session")
def small_scene(oracle):
    """The 64-primitive, 4 cm scene voxelized by the oracle (reference layouts)."""
    from rkifield_b200 import scenes
    spec = scenes.SCENE_SMALL
    prims = scenes.make_prims(spec)
    vp = scenes.voxelize_params(spec, prims)
    vox = oracle.Voxelized(prims, vp)
    obj = vox.gpu_object()
    return {"spec": spec, "prims": prims, "vp": vp, "vox": vox, "obj": obj}


@pytest.fixture(scope="session")
def small_ctx(small_scene):
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    ctx = Context(pool_capacity=max(v.n_bricks + 4096, 1 << 15))
    ctx.set_brick_pool(v.words)
    ctx.upload_brick_maps(v.map)
    ctx.upload_objects([small_scene["obj"]])
    yield ctx
    ctx.close()


@pytest.fixture(scope="session")
def large():
    """The full-size workload: 512 seeded primitives in a 256 m cube voxelized
    at 2 cm on the device (about 1.1 M bricks, two-level index), the headline
    camera inside the grid and the march parameters of that scene."""
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    spec = scenes.SCENE_LARGE
    prims = scenes.make_prims(spec)
    ctx = Context(pool_capacity=3_000_000, keep_reference_pool=False)
    ctx.voxelize(prims, scenes.voxelize_params(spec, prims))
    cam = scenes.seeded_camera(spec, 1920, 1080, seed=100, inside=True, distance=spec.cube * 0.18)
    p = scenes.march_params(spec)
    yield ctx, spec, cam, p
    ctx.close()


def oracle_scene_of(oracle, ctx, objects=None, bvh=None):
    """An oracle scene reading the context's own pool planes and index (the
    inputs the device march reads), with its objects (and BVH nodes)."""
    idx = ctx.export_index()
    leaves = idx["leaves"]
    live = leaves[leaves < 0xFFFFFFFE]
    n = int(live.max()) + 1 if live.size else 1
    pl = ctx.export_planes(0, n)
    if objects is None:
        objects = [ctx.object(i) for i in range(ctx.info()["num_objects"])]
    return oracle.Scene(objects, top=idx["top"], leaves=leaves, obj_top_info=idx["obj_top_info"],
                        dist_f16=pl["dist"], mat_plane=pl["mat"], blend_plane=pl["blend"], bvh=bvh)


@pytest.fixture(scope="session")
def large_oracle(oracle, large):
    ctx = large[0]
    assert ctx.info()["pool_bricks_used"] > 1_000_000
    return oracle_scene_of(oracle, ctx, [ctx.object(0)])


def assert_bits_equal(a: np.ndarray, b: np.ndarray, what: str):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape, what
    if a.dtype.kind == "f":
        ai = a.view(np.uint32 if a.itemsize == 4 else np.uint64)
        bi = b.view(np.uint32 if b.itemsize == 4 else np.uint64)
        both_nan = np.isnan(a) & np.isnan(b)
        bad = (ai != bi) & ~both_nan
    else:
        bad = a != b
    n = int(bad.sum())
    if n:
        i = np.nonzero(bad.ravel())[0][:5]
        raise AssertionError(f"{what}: {n} of {a.size} differ; first at {i}: {a.ravel()[i]} vs {b.ravel()[i]}")
