"""Device CSG edits against the oracle's restatement of apply_edit_cpu
(crates/rkf-edit/src/cpu_apply.rs:28-200), brick by brick, then the march of
the edited scene against the oracle march."""
import ctypes as C

import numpy as np
import pytest

from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu


def _op(kind, pos, radius, mat, blend_k=0.05, falloff=1, shape=0, dims=None):
    from rkifield_b200 import _abi as abi
    op = abi.rkf_edit_op()
    op.object_index = 0
    op.edit_type = kind
    op.shape_type = shape
    op.falloff = falloff
    op.position[:] = [float(x) for x in pos]
    op.rotation[:] = (0.0, 0.0, 0.0, 1.0)
    op.dimensions[:] = dims if dims is not None else (radius, 0.0, 0.0)
    op.strength = 1.0
    op.blend_k = blend_k
    op.material_id = mat
    return op


def _bricks_in_range(op, dims, vs):
    """find_affected_bricks' brick range (edit_op.rs:97-118)."""
    be = np.float32(vs) * np.float32(8)
    origin = -(dims.astype(np.float32) * be * np.float32(0.5))
    mx = max(op.dimensions[0], op.dimensions[1], op.dimensions[2])
    ext = np.float32(mx) + np.float32(op.blend_k)
    pos = np.array(op.position[:], np.float32)
    lo = np.floor((pos - ext - origin) / be).astype(int)
    hi = np.ceil((pos + ext - origin) / be - np.float32(0.001)).astype(int)
    lo = np.maximum(lo, 0)
    hi = np.minimum(np.maximum(hi, 0), dims.astype(int) - 1)
    out = []
    for z in range(lo[2], hi[2] + 1):
        for y in range(lo[1], hi[1] + 1):
            for x in range(lo[0], hi[0] + 1):
                out.append((x, y, z))
    return np.array(out, np.uint32), origin, be


def _expected(oracle, ctx, op, dims, vs, words_by_slot):
    """For every brick in range: (old slot, expected words or None if unchanged)."""
    bxyz, origin, be = _bricks_in_range(op, dims, vs)
    slots = ctx.brick_lookup(0, bxyz.ravel())
    additive = op.edit_type in (0, 3)
    exp = []
    for b, s in zip(bxyz, slots):
        if op.edit_type >= 5 and s >= 0xFFFFFFFE:  # smooth, flatten, paint: allocated bricks only
            exp.append((b, s, None))
            continue
        if s == 0xFFFFFFFF:
            if not additive:
                exp.append((b, s, None))
                continue
            w = np.zeros(1024, np.uint32)
            w[0::2] = oracle.lib().orc_f16_from_f32(float(np.float32(vs) * np.float32(8)))
        elif s == 0xFFFFFFFE:
            if additive:
                exp.append((b, s, None))
                continue
            w = np.zeros(1024, np.uint32)
            w[0::2] = oracle.lib().orc_f16_from_f32(float(-(np.float32(vs) * np.float32(2))))
        else:
            w = words_by_slot(int(s)).copy()
        bmin = (origin + b.astype(np.float32) * be).astype(np.float32)
        changed = oracle.lib().orc_apply_edit_brick(w.ctypes.data, bmin.ctypes.data, float(vs), C.byref(op))
        exp.append((b, s, w if changed else None))
    return exp


def test_csg_edits_match_oracle_and_march(oracle, small_scene):
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    v = small_scene["vox"]
    spec = small_scene["spec"]
    prims = small_scene["prims"]
    cap = v.n_bricks + 20000
    with Context(pool_capacity=cap) as ctx:
        ctx.set_brick_pool(v.words)
        ctx.upload_brick_maps(v.map)
        ctx.upload_objects([small_scene["obj"]])
        p0 = prims[3]
        c = p0["centre"].astype(np.float64)
        r = float(p0["bound_radius"])
        ops = [_op(0, c + np.array([r, 0, 0]), 0.6, 7),          # union bump on a surface
               _op(1, c + np.array([0, r * 0.8, 0]), 0.5, 0),    # carve
               _op(3, c + np.array([0, 0, r + 0.3]), 0.4, 9, blend_k=0.1, falloff=2),
               _op(4, c - np.array([r * 0.5, 0, 0]), 0.7, 0, blend_k=0.1),
               _op(0, c + np.array([-3.0, 2.0, 1.0]), 0.3, 11, shape=1, dims=(0.3, 0.2, 0.4)),
               _op(5, c + np.array([r, 0, 0]), 0.5, 0),                      # smooth brush
               _op(6, c + np.array([0, r, 0]), 0.6, 0, falloff=0),          # flatten
               _op(7, c + np.array([0, 0, -r]), 0.3, 13)]                    # paint
        for op in ops:
            words = ctx.export_pool(0, cap)
            exp = _expected(oracle, ctx, op, v.dims, spec.voxel_size,
                            lambda s: words[1024 * s:1024 * (s + 1)])
            assert any(e[2] is not None for e in exp), "the edit should change bricks"
            e0 = ctx.info()["epoch"]
            ep = ctx.edit(op)
            assert ep == e0 + 1
            bxyz = np.array([e[0] for e in exp], np.uint32)
            after = ctx.brick_lookup(0, bxyz.ravel())
            words2 = ctx.export_pool(0, cap)
            for (b, s_old, w_exp), s_new in zip(exp, after):
                if w_exp is None:
                    assert s_new == s_old, f"brick {b} should be untouched"
                else:
                    assert s_new < 0xFFFFFFFE and s_new != s_old, f"brick {b} should move to a fresh slot"
                    assert_bits_equal(words2[1024 * s_new:1024 * (s_new + 1)], w_exp, f"brick {b} words")
        # march the edited scene: device index vs oracle on the exported scene
        z, y, x = np.meshgrid(np.arange(v.dims[2]), np.arange(v.dims[1]), np.arange(v.dims[0]), indexing="ij")
        allb = np.stack([x.ravel(), y.ravel(), z.ravel()], 1).astype(np.uint32)
        fmap = ctx.brick_lookup(0, allb.ravel())
        words = ctx.export_pool(0, cap)
        sc = oracle.Scene([small_scene["obj"]], pool_words=words, brick_maps=fmap)
        cam = scenes.camera_uniforms(c + np.array([4.0, 2.0, 5.0]), c, 160, 120)
        p = scenes.march_params(spec)
        ref = oracle.march(sc, cam, p, 160, 120, with_reference_planes=True)
        got = ctx.march(cam, p, 160, 120, reference_planes=True)
        plain = ctx.march(cam, p, 160, 120, reference_planes=True, plain=True)
        assert (ref["flags"] & 1).sum() > 1000
        for k in ref:
            if k == "stats":
                continue
            assert_bits_equal(got[k], ref[k], k)
            assert_bits_equal(plain[k], ref[k], "plain " + k)
        # color paint writes a companion color pool this library does not keep
        from rkifield_b200 import _abi as abi
        from rkifield_b200.engine import RkfError
        e0 = ctx.info()["epoch"]
        for kind, status in ((8, abi.RKF_UNSUPPORTED), (9, abi.RKF_INVALID_ARG)):
            with pytest.raises(RkfError) as e:
                ctx.edit(_op(kind, c, 0.3, 1))
            assert e.value.status == status
        assert ctx.info()["epoch"] == e0


@pytest.mark.parametrize("precision,u8_round", [("f32", 0), ("u8", 0), ("u8", 1)],
                         ids=["f32", "u8_toward_zero", "u8_nearest"])
def test_csg_edits_on_f32_and_u8_pools(oracle, small_scene, precision, u8_round):
    """The same edits on pools stored in f32 and in band-normalised u8: the
    brush blends with the decoded distance (apply_edit_cpu's arithmetic,
    cpu_apply.rs:28-200) and an edited u8 brick is encoded again with its own
    step.  Brick by brick against the oracle's restatement, then the march of
    the edited scene against the oracle march over the exported planes."""
    from rkifield_b200 import _abi as abi
    from rkifield_b200 import scenes
    from rkifield_b200.engine import Context
    spec, prims, vp = small_scene["spec"], small_scene["prims"], small_scene["vp"]
    vs = np.float32(spec.voxel_size)
    cap = small_scene["vox"].n_bricks + 20000
    ctx = Context(pool_capacity=cap, precision=precision, keep_reference_pool=False, u8_round=u8_round)
    try:
        ctx.voxelize(prims, vp)
        obj = ctx.object(0)
        dims = np.array(obj.brick_map_dims[:], np.uint32)
        p0 = prims[3]
        c = p0["centre"].astype(np.float64)
        r = float(p0["bound_radius"])
        ops = [_op(0, c + np.array([r, 0, 0]), 0.6, 7),
               _op(1, c + np.array([0, r * 0.8, 0]), 0.5, 0),
               _op(3, c + np.array([0, 0, r + 0.3]), 0.4, 9, blend_k=0.1, falloff=2),
               _op(4, c - np.array([r * 0.5, 0, 0]), 0.7, 0, blend_k=0.1),
               _op(5, c + np.array([r, 0, 0]), 0.5, 0),
               _op(6, c + np.array([0, r, 0]), 0.6, 0, falloff=0),
               _op(7, c + np.array([0, 0, -r]), 0.3, 13)]
        L = oracle.lib()
        for op in ops:
            pl = ctx.export_planes(0, cap)
            bxyz, origin, be = _bricks_in_range(op, dims, vs)
            slots = ctx.brick_lookup(0, bxyz.ravel())
            additive = op.edit_type in (0, 3)
            exp = []
            for b, s in zip(bxyz, slots):
                if (s == abi.EMPTY_SLOT and not additive) or (s == abi.INTERIOR_SLOT and additive) or \
                        (op.edit_type >= 5 and s >= abi.INTERIOR_SLOT):
                    exp.append((b, s, None))
                    continue
                if s >= abi.INTERIOR_SLOT:
                    d = np.full(512, vs * np.float32(8) if s == abi.EMPTY_SLOT else -(vs * np.float32(2)), np.float32)
                    m = np.zeros(512, np.uint16)
                    bl = np.zeros(512, np.uint8)
                else:
                    sl = slice(512 * int(s), 512 * (int(s) + 1))
                    d = (pl["dist"][sl].astype(np.float32) * pl["step"][int(s)]).astype(np.float32) \
                        if precision == "u8" else pl["dist"][sl].copy()
                    m = pl["mat"][sl].copy()
                    bl = pl["blend"][sl].copy()
                bmin = (origin + b.astype(np.float32) * be).astype(np.float32)
                changed = L.orc_apply_edit_planes(d.ctypes.data, m.ctypes.data, bl.ctypes.data, bmin.ctypes.data,
                                                  float(vs), C.byref(op))
                if not changed:
                    exp.append((b, s, None))
                    continue
                e = {"mat": m, "blend": bl}
                if precision == "u8":
                    code = np.zeros(512, np.int8)
                    step = np.zeros(1, np.float32)
                    L.orc_encode_u8(d.ctypes.data, float(np.float32(3.0) * vs), u8_round, code.ctypes.data,
                                    step.ctypes.data)
                    e.update(dist=code, step=step)
                else:
                    e["dist"] = d
                exp.append((b, s, e))
            assert any(x[2] is not None for x in exp), "the edit should change bricks"
            ctx.edit(op)
            after = ctx.brick_lookup(0, bxyz.ravel())
            pl2 = ctx.export_planes(0, cap)
            for (b, s_old, e), s_new in zip(exp, after):
                if e is None:
                    assert s_new == s_old, f"brick {b} should be untouched"
                    continue
                assert s_new < abi.INTERIOR_SLOT and s_new != s_old, f"brick {b} should move to a fresh slot"
                sl = slice(512 * int(s_new), 512 * (int(s_new) + 1))
                for k in ("dist", "mat", "blend"):
                    assert_bits_equal(pl2[k][sl], e[k], f"brick {b} {k}")
                if precision == "u8":
                    assert_bits_equal(pl2["step"][int(s_new):int(s_new) + 1], e["step"], f"brick {b} step")
        # the edited scene marches as the oracle does over the exported planes
        idx = ctx.export_index()
        pl = ctx.export_planes(0, cap)
        code = {"f32": abi.RKF_PRECISION_F32, "u8": abi.RKF_PRECISION_U8}[precision]
        kw = {"dist_f32": pl["dist"]} if precision == "f32" else {"dist_u8": pl["dist"], "brick_scale": pl["step"]}
        sc = oracle.Scene([obj], top=idx["top"], leaves=idx["leaves"], obj_top_info=idx["obj_top_info"],
                          mat_plane=pl["mat"], blend_plane=pl["blend"], precision=code, **kw)
        cam = scenes.camera_uniforms(c + np.array([4.0, 2.0, 5.0]), c, 160, 120)
        p = scenes.march_params(spec)
        ref = oracle.march(sc, cam, p, 160, 120, with_reference_planes=True)
        got = ctx.march(cam, p, 160, 120, reference_planes=True)
        assert (ref["flags"] & 1).sum() > 1000
        for k in ("t", "normal", "slot", "material", "flags", "position", "packed_material", "motion"):
            assert_bits_equal(got[k], ref[k], f"{precision} edited march {k}")
    finally:
        ctx.close()
