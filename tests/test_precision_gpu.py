"""Storage precisions of the distance plane: f32 and band-normalised u8 (f16
is the default covered elsewhere).  The march over each plane is bit-exact
against the FP32 oracle reading the same plane, and the u8 code is checked
against its definition: normalised by the +-3-voxel narrow band with a
per-brick scale, B = min(3 voxels, largest finite |d| in the brick),
step = B/127, |code| = min(floor(|d|/step), 127) (toward zero, |d| clamped to
B), less one where code*step would round above |d|, with the sign of d, so a
decoded |d| never exceeds the true one; or, with rounding to nearest,
|code| = min(rint(|d|/step), 127), within half a step."""
import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu


def _ctx(small_scene, precision, u8_round=0):
    from rkifield_b200.engine import Context
    ctx = Context(pool_capacity=small_scene["vox"].n_bricks + 1024, precision=precision,
                  keep_reference_pool=False, u8_round=u8_round)
    ctx.voxelize(small_scene["prims"], small_scene["vp"])
    return ctx


def _oracle_scene(oracle, ctx, precision, n):
    from rkifield_b200 import _abi as abi
    pl = ctx.export_planes(0, n)
    idx = ctx.export_index()
    code = {"f32": abi.RKF_PRECISION_F32, "u8": abi.RKF_PRECISION_U8}[precision]
    kw = {"dist_f32": pl["dist"]} if precision == "f32" else {"dist_u8": pl["dist"], "brick_scale": pl["step"]}
    return oracle.Scene([ctx.object(0)], top=idx["top"], leaves=idx["leaves"], obj_top_info=idx["obj_top_info"],
                        mat_plane=pl["mat"], blend_plane=pl["blend"], precision=code, **kw), pl


@pytest.mark.parametrize("precision,u8_round", [("f32", 0), ("u8", 0), ("u8", 1)],
                         ids=["f32", "u8_toward_zero", "u8_nearest"])
def test_precision_march_bit_exact(oracle, small_scene, precision, u8_round):
    from rkifield_b200 import scenes
    spec = small_scene["spec"]
    n = small_scene["vox"].n_bricks
    ctx = _ctx(small_scene, precision, u8_round)
    try:
        sc, pl = _oracle_scene(oracle, ctx, precision, n)
        for seed in (11, 12):
            cam = scenes.seeded_camera(spec, 192, 160, seed=seed)
            p = scenes.march_params(spec)
            ref = oracle.march(sc, cam, p, 192, 160, with_reference_planes=True)
            got = ctx.march(cam, p, 192, 160, reference_planes=True)
            assert (ref["flags"] & 1).sum() > 500
            for k in ("t", "normal", "slot", "material", "flags", "position", "packed_material", "motion"):
                assert_bits_equal(got[k], ref[k], f"{precision} {k}")
        if precision == "f32":
            assert_bits_equal(pl["dist"], small_scene["vox"].dist_f32, "f32 plane = voxelizer distances")
        else:
            d = small_scene["vox"].dist_f32.reshape(-1, 512)
            fin = np.where(np.isfinite(d), np.abs(d), 0.0).astype(np.float32)
            band = np.float32(3.0) * np.float32(spec.voxel_size)
            rng = np.maximum(np.minimum(fin.max(axis=1), band), np.float32(1e-6)).astype(np.float32)
            step = (rng / np.float32(127.0)).astype(np.float32)
            assert_bits_equal(pl["step"], step, "u8 step")
            a = np.abs(d).astype(np.float32)
            qa = (a / step[:, None]).astype(np.float32)
            q = np.rint(qa) if u8_round else np.floor(qa)
            c = np.where(q >= 127, 127, np.nan_to_num(q, posinf=127)).astype(np.int32)
            if not u8_round:
                over = (c > 0) & ((c.astype(np.float32) * step[:, None]).astype(np.float32) > a)
                c = np.where(over, c - 1, c)
            code = np.where(d < 0, -c, c).astype(np.int8).ravel()
            assert_bits_equal(pl["dist"], code, "u8 codes")
            dec = pl["dist"].astype(np.float32).reshape(-1, 512) * pl["step"][:, None]
            ok = np.isfinite(d)
            inb = ok & (np.abs(d) <= rng[:, None])
            stp = np.broadcast_to(step[:, None], d.shape)[inb]
            err = (np.abs(d) - np.abs(dec))[inb]
            if u8_round:
                # to nearest: within half a step (plus the product's rounding)
                assert (np.abs(err) <= stp * 0.5001).all()
            else:
                assert (np.abs(dec[ok]) <= np.abs(d[ok]) + 0).all(), "u8 must never overstate |d|"
                # inside the band the code is within one step of the true distance
                assert (err <= stp * 1.0001).all()
    finally:
        ctx.close()
