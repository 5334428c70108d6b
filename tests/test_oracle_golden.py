"""Pin the CPU oracle against the known answers the reference's own unit
tests assert for the pieces of the march path (read from the reference's
test modules; each case cites the test it restates).

These are CPU tests: they exercise only the oracle (the checker) and host
logic, never the product library's compute entry points.
"""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import assert_bits_equal

from rkifield_b200 import _abi as abi


def f16(oracle, x):
    return oracle.lib().orc_f16_from_f32(x)


def f32(oracle, h):
    return oracle.lib().orc_f16_to_f32(h)


# ---- binary16 conversion (the `half` crate, RNE) ---------------------------

def test_f16_conversion_matches_numpy_rne(oracle):
    rng = np.random.default_rng(0)
    xs = np.concatenate([
        rng.standard_normal(20000).astype(np.float32) * np.float32(10.0) ** rng.integers(-9, 6, 20000),
        np.float32([0.0, -0.0, 65504.0, 65519.996, 65520.0, 1e-8, 5.96e-8, 2.98e-8, 2.9802322e-08,
                    6.1035156e-05, np.inf, -np.inf, 1.5, -0.5, 0.32, -0.08]),
    ]).astype(np.float32)
    L = oracle.lib()
    got = np.array([L.orc_f16_from_f32(float(x)) for x in xs], np.uint16)
    want = xs.astype(np.float16).view(np.uint16)  # IEEE RNE
    assert (got == want).all()
    back = np.array([L.orc_f16_to_f32(int(h)) for h in got], np.float32)
    assert (back.view(np.uint32) == want.view(np.float16).astype(np.float32).view(np.uint32)).all()


def test_f16_all_bit_patterns_decode_exactly(oracle):
    L = oracle.lib()
    hs = np.arange(0, 65536, 7, dtype=np.uint32)
    got = np.array([L.orc_f16_to_f32(int(h)) for h in hs], np.float32)
    want = hs.astype(np.uint16).view(np.float16).astype(np.float32)
    nan = np.isnan(want)
    assert (np.isnan(got) == nan).all()
    assert (got[~nan].view(np.uint32) == want[~nan].view(np.uint32)).all()


# ---- VoxelSample packing (crates/rkf-core/src/voxel.rs:124-276) -----------

def pack(oracle, d, mat, sec=0, blend=0):
    w0 = f16(oracle, d) | ((mat & 0x3F) << 16) | ((sec & 0x3F) << 22)
    return w0, blend << 24


def test_voxel_sample_roundtrip_typical(oracle):  # roundtrip_typical_values
    w0, w1 = pack(oracle, 1.5, 42)
    assert f32(oracle, w0 & 0xFFFF) == 1.5 and (w0 >> 16) & 0x3F == 42 and w1 >> 24 == 0


def test_voxel_sample_negative_and_blend(oracle):  # roundtrip_negative_distance, new_with_blend_weight
    w0, w1 = pack(oracle, -0.5, 1, blend=200)
    assert f32(oracle, w0 & 0xFFFF) == -0.5 and (w0 >> 16) & 0x3F == 1 and w1 >> 24 == 200


def test_voxel_sample_material_masked(oracle):  # material_id_masked_to_6_bits
    w0, _ = pack(oracle, 0.0, 0xFF)
    assert (w0 >> 16) & 0x3F == 63 and (w0 >> 22) & 0x3F == 0  # must not bleed into secondary


def test_voxel_sample_blended(oracle):  # new_blended_roundtrip
    w0, w1 = pack(oracle, -0.5, 3, 7, 128)
    assert (w0 >> 16) & 0x3F == 3 and (w0 >> 22) & 0x3F == 7 and w1 >> 24 == 128


def test_voxel_sample_default_is_infinity(oracle):  # default_has_infinity_distance_and_zero_blend
    w0, w1 = pack(oracle, float("inf"), 0)
    assert math.isinf(f32(oracle, w0 & 0xFFFF)) and w1 == 0
    assert f16(oracle, 65504.0) == 0x7BFF  # edge_case_f16_max_distance (f16::MAX)


# ---- brick / brick map indexing (brick.rs:194-338, brick_map.rs:285-528) ---

def test_brick_index_corners():
    idx = lambda x, y, z: x + 8 * y + 64 * z  # noqa: E731  (brick.rs:28-42)
    assert [idx(0, 0, 0), idx(7, 0, 0), idx(0, 7, 0), idx(0, 0, 7), idx(7, 7, 7)] == [0, 7, 56, 448, 511]


def test_brick_map_flatten():
    dims = (3, 4, 5)
    flat = lambda x, y, z: x + y * dims[0] + z * dims[0] * dims[1]  # noqa: E731  (brick_map.rs:80-85)
    assert flat(2, 0, 0) == 2 and flat(0, 1, 0) == 3 and flat(0, 0, 1) == 12 and flat(2, 3, 4) == 59


# ---- analytic SDFs (crates/rkf-core/src/sdf.rs:63-166) ----------------------

def prim(kind, centre=(0, 0, 0), params=(1, 0, 0)):
    p = np.zeros(1, abi.PRIM_DTYPE)
    p["type"] = kind
    p["centre"] = centre
    p["params"] = params
    p["rot"] = np.eye(3, dtype=np.float32).ravel()
    p["bound_radius"] = 10.0
    return p


def sdf(oracle, p, pos):
    q = np.array(pos, np.float32)
    return oracle.lib().orc_prim_sdf(p.ctypes.data, q.ctypes.data)


def test_sphere_sdf(oracle):
    s = prim(0, params=(1, 0, 0))
    assert abs(sdf(oracle, s, (0, 0, 0)) + 1.0) < 1e-6
    assert abs(sdf(oracle, s, (1, 0, 0))) < 1e-6
    assert abs(sdf(oracle, s, (2, 0, 0)) - 1.0) < 1e-6
    assert abs(sdf(oracle, s, (0.5, 0, 0)) + 0.5) < 1e-6


def test_box_sdf(oracle):
    b = prim(1, params=(1, 1, 1))
    assert abs(sdf(oracle, b, (0, 0, 0)) + 1.0) < 1e-6
    assert abs(sdf(oracle, b, (1, 0, 0))) < 1e-6
    assert abs(sdf(oracle, b, (2, 0, 0)) - 1.0) < 1e-6
    assert abs(sdf(oracle, b, (2, 2, 2)) - math.sqrt(3)) < 1e-5
    assert abs(sdf(oracle, b, (0.5, 0, 0)) + 0.5) < 1e-6


def test_capsule_sdf(oracle):
    # capsule_sdf(a=(0,0,0), b=(0,1,0), r=0.5): centred form a=(0,-h,0),b=(0,h,0), h=0.5
    c = prim(2, centre=(0, 0.5, 0), params=(0.5, 0.5, 0))
    for y in (0.0, 0.5, 1.0):
        assert abs(sdf(oracle, c, (0, y, 0)) + 0.5) < 1e-6
    assert abs(sdf(oracle, c, (0.5, 0.5, 0))) < 1e-6
    assert abs(sdf(oracle, c, (1.5, 0.5, 0)) - 1.0) < 1e-6


def test_smin(oracle):  # sdf.rs:48-51 doc: |a-b| >= k -> min exactly; else below min
    L = oracle.lib()
    assert L.orc_smin(1.0, 3.0, 0.5) == 1.0
    assert L.orc_smin(1.0, 1.0, 0.5) < 1.0
    assert abs(L.orc_smin(1.0, 1.0, 0.5) - (1.0 - 0.125)) < 1e-7


# ---- single-brick trilinear (crates/rkf-core/src/sampling.rs:134-290) -------

def brick_words(oracle, dist_fn, mat_fn=lambda x, y, z: 1):
    w = np.zeros(1024, np.uint32)
    for z in range(8):
        for y in range(8):
            for x in range(8):
                w0, w1 = pack(oracle, dist_fn(x, y, z), mat_fn(x, y, z))
                i = x + 8 * y + 64 * z
                w[2 * i], w[2 * i + 1] = w0, w1
    return w


def tri(oracle, w, pos):
    q = np.array(pos, np.float32)
    return oracle.lib().orc_sample_brick_trilinear(w.ctypes.data, q.ctypes.data, 0.0)


def test_trilinear_at_voxel_centres(oracle):  # trilinear_at_voxel_centers_matches_stored_value
    w = brick_words(oracle, lambda x, y, z: (x + y * 8 + z * 64) * 0.01)
    for (x, y, z) in [(0, 0, 0), (3, 4, 5), (6, 6, 6), (1, 6, 2)]:
        pos = ((x + 0.5) / 8, (y + 0.5) / 8, (z + 0.5) / 8)
        stored = f32(oracle, f16(oracle, (x + y * 8 + z * 64) * 0.01))
        assert abs(tri(oracle, w, pos) - stored) < 0.02


def test_trilinear_uniform_and_midpoint(oracle):
    w = brick_words(oracle, lambda x, y, z: 3.5)  # trilinear_uniform_brick_returns_constant
    for pos in [(0.1, 0.2, 0.3), (0.5, 0.5, 0.5), (0.9, 0.9, 0.9)]:
        assert abs(tri(oracle, w, pos) - 3.5) < 1e-3
    w = brick_words(oracle, lambda x, y, z: 0.0 if x < 4 else 2.0)  # trilinear_midpoint_interpolation
    assert abs(tri(oracle, w, ((3.5 + 0.5) / 8, 0.5, 0.5)) - 1.0) < 0.15


def test_trilinear_monotone_along_x(oracle):  # trilinear_is_smooth
    w = brick_words(oracle, lambda x, y, z: float(x))
    prev = tri(oracle, w, (0.0, 0.5, 0.5))
    for i in range(1, 21):
        cur = tri(oracle, w, (i / 20, 0.5, 0.5))
        assert cur >= prev - 1e-4
        prev = cur


# ---- CSG edit (crates/rkf-edit/src/cpu_apply.rs:343-475) --------------------

def edit_op(edit_type, pos, radius, blend_k, material, falloff=1):
    op = abi.rkf_edit_op()
    op.edit_type = edit_type
    op.shape_type = 0
    op.falloff = falloff
    op.position[:] = pos
    op.rotation[:] = (0.0, 0.0, 0.0, 1.0)
    op.dimensions[:] = (radius, 0.0, 0.0)
    op.strength = 1.0
    op.blend_k = blend_k
    op.material_id = material
    return op


def test_edit_sphere_union_adds_material(oracle):  # sphere_union_adds_material
    w = brick_words(oracle, lambda x, y, z: 1.0, lambda x, y, z: 0)
    op = edit_op(3, (0.2, 0.2, 0.2), 0.15, 0.15 * 0.3, 5)
    bmin = np.zeros(3, np.float32)
    mod = oracle.lib().orc_apply_edit_brick(w.ctypes.data, bmin.ctypes.data, 0.05, C.byref(op))
    assert mod == 1
    i = 4 + 4 * 8 + 4 * 64
    assert f32(oracle, int(w[2 * i]) & 0xFFFF) < 1.0


def test_edit_sphere_subtract_carves(oracle):  # sphere_subtract_carves
    w = brick_words(oracle, lambda x, y, z: -0.5, lambda x, y, z: 2)
    op = edit_op(4, (0.2, 0.2, 0.2), 0.15, 0.05, 0)
    bmin = np.zeros(3, np.float32)
    mod = oracle.lib().orc_apply_edit_brick(w.ctypes.data, bmin.ctypes.data, 0.05, C.byref(op))
    assert mod == 1
    i = 4 + 4 * 8 + 4 * 64
    assert f32(oracle, int(w[2 * i]) & 0xFFFF) > -0.5


def test_edit_paint_sets_material_near_surface(oracle):  # paint_sets_material_near_surface
    """Paint (cpu_apply.rs:166-173): voxels with |d| < 2 dims.x take the
    brush material as VoxelSample::new(d, material, 0) -- secondary material
    and blend weight cleared, distance kept -- and the brick counts as
    modified; the others keep everything."""
    w = brick_words(oracle, lambda x, y, z: 0.01 if (y == 4 and z == 4) else 1.0, lambda x, y, z: 1)
    w[0::2] |= np.uint32(9 << 22)
    w[1::2] = np.uint32(200 << 24)
    before = w.copy()
    op = edit_op(7, (0.2, 0.2, 0.2), 0.5, 0.0, 42)
    mod = oracle.lib().orc_apply_edit_brick(w.ctypes.data, np.zeros(3, np.float32).ctypes.data, 0.05, C.byref(op))
    assert mod == 1
    i = 4 + 4 * 8 + 4 * 64
    assert (int(w[2 * i]) >> 16) & 0x3F == 42 and (int(w[2 * i]) >> 22) & 0x3F == 0 and int(w[2 * i + 1]) == 0
    assert int(w[2 * i]) & 0xFFFF == int(before[2 * i]) & 0xFFFF
    j = 1 + 2 * 8 + 3 * 64  # |d| = 1.0, not below 2 * 0.5
    assert w[2 * j] == before[2 * j] and w[2 * j + 1] == before[2 * j + 1]


def test_edit_smooth_scales_distance(oracle):  # smooth_operation_reduces_distance
    w = brick_words(oracle, lambda x, y, z: (x - 3.5) * 0.1, lambda x, y, z: 1)
    before = w.copy()
    op = edit_op(5, (0.2, 0.2, 0.2), 0.5, 0.0, 0)
    mod = oracle.lib().orc_apply_edit_brick(w.ctypes.data, np.zeros(3, np.float32).ctypes.data, 0.05, C.byref(op))
    assert mod == 1
    for x in (0, 7):
        i = x + 4 * 8 + 4 * 64
        assert abs(f32(oracle, int(w[2 * i]) & 0xFFFF)) < abs(f32(oracle, int(before[2 * i]) & 0xFFFF))


def test_edit_flatten_pulls_toward_plane(oracle):
    """Flatten (cpu_apply.rs:158-165): d moves toward the brush's local
    plane distance (edit-local y) by half the strength at the voxel."""
    w = brick_words(oracle, lambda x, y, z: 1.0, lambda x, y, z: 1)
    op = edit_op(6, (0.2, 0.2, 0.2), 0.5, 0.0, 0)
    mod = oracle.lib().orc_apply_edit_brick(w.ctypes.data, np.zeros(3, np.float32).ctypes.data, 0.05, C.byref(op))
    assert mod == 1
    for y in (0, 7):
        i = 4 + y * 8 + 4 * 64
        plane = (y + 0.5) * 0.05 - 0.2
        d = f32(oracle, int(w[2 * i]) & 0xFFFF)
        assert plane < d < 1.0


def test_edit_shape_and_falloff(oracle):
    L = oracle.lib()
    z = np.zeros(3, np.float32)
    assert abs(L.orc_evaluate_shape(0, np.float32([1, 0, 0]).ctypes.data, z.ctypes.data) + 1.0) < 1e-5
    assert abs(L.orc_evaluate_shape(1, np.float32([0.5, 0.5, 0.5]).ctypes.data, z.ctypes.data) + 0.5) < 1e-5
    assert abs(L.orc_evaluate_falloff(1, 0.0, 1.0) - 1.0) < 1e-5
    assert abs(L.orc_evaluate_falloff(1, 1.0, 1.0)) < 1e-5
    assert abs(L.orc_evaluate_falloff(0, 1.5, 1.0)) < 1e-5


# ---- voxelizer (crates/rkf-core/src/voxelize_object.rs:489-700) -------------

def test_voxelizer_grid_is_centred_and_band_limited(oracle):
    """dims = ceil(aabb/brick), grid centred at the origin, narrow band only
    (voxelize_object.rs:61-81, narrow_band_skips_interior)."""
    p = prim(0, params=(1.0, 0, 0))
    p["bound_radius"] = 1.001
    vp = abi.rkf_voxelize_params()
    vp.voxel_size, vp.smooth_k, vp.band_voxels, vp.cut_distance = 0.1, 0.1, 3.0, 1.0
    vp.aabb_min[:] = (-1.5, -1.5, -1.5)
    vp.aabb_max[:] = (1.5, 1.5, 1.5)
    v = oracle.Voxelized(p, vp)
    assert list(v.dims) == [4, 4, 4]  # ceil(3.0 / 0.8)
    # reference band rule allocates more than the +-3 voxel band
    vp.band_rule = 1
    vr = oracle.Voxelized(p, vp)
    assert vr.n_bricks >= v.n_bricks and v.n_bricks > 0
    # every allocated voxel's stored distance is the sphere SDF at its centre
    d = v.dist_f32.reshape(-1, 512)
    m = v.map.reshape(4, 4, 4)
    for (bz, by, bx) in zip(*np.nonzero(m < abi.INTERIOR_SLOT)):
        s = m[bz, by, bx]
        for (x, y, zz) in [(0, 0, 0), (7, 7, 7), (3, 5, 1)]:
            c = np.float32(-1.6) + np.float32(bx) * np.float32(0.8) + (np.float32(x) * np.float32(0.1) + np.float32(0.05))
            cy = np.float32(-1.6) + np.float32(by) * np.float32(0.8) + (np.float32(y) * np.float32(0.1) + np.float32(0.05))
            cz = np.float32(-1.6) + np.float32(bz) * np.float32(0.8) + (np.float32(zz) * np.float32(0.1) + np.float32(0.05))
            r = math.sqrt(c * c + cy * cy + cz * cz)
            if r - 1.001 >= 1.0:  # beyond the cut distance no primitive contributes
                assert math.isinf(d[s, x + 8 * y + 64 * zz])
            else:
                assert abs(d[s, x + 8 * y + 64 * zz] - (r - 1.0)) < 1e-5


# ---- coarse field of the tiled strategy (coarse_field.rs) -------------------
def _aabb_distance(q, lo, hi):
    """aabb_unsigned_distance (coarse_field.rs): length of max(lo - q, q - hi, 0), in float32."""
    F = np.float32
    d = np.maximum(np.maximum(F(lo) - F(q), F(q) - F(hi)), F(0))
    return np.sqrt((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]).astype(F)


def _box(lo, hi):
    from rkifield_b200 import _abi as abi
    o = abi.rkf_gpu_object()
    for a in range(3):
        o.aabb_min[a], o.aabb_max[a] = lo[a], hi[a]
        o.accumulated_scale[a] = 1.0
    o.sdf_type = abi.RKF_SDF_ANALYTICAL
    return o


def test_coarse_aabb_distance_matches_reference_tests():
    """aabb_distance_outside / _inside / _corner (coarse_field.rs:471-500)."""
    F = np.float32
    assert abs(_aabb_distance(np.array([3, 0, 0], F), [-1] * 3, [1] * 3) - 2.0) < 1e-5
    assert _aabb_distance(np.zeros(3, F), [-1] * 3, [1] * 3) == 0.0
    assert abs(_aabb_distance(np.array([2, 2, 2], F), [0] * 3, [1] * 3) - np.sqrt(F(3))) < 1e-5


def test_coarse_field_dims_match_reference_test(oracle):
    """dims_calculation (coarse_field.rs:502-527): an extent of (4, 2, 6) at
    0.32 m cells is 13 x 7 x 19 = 1729 cells; here it is an object box of
    (2, 0, 4) grown by the 1 m margin, origin (-2, -1, -3) as in that test."""
    origin, dims, tex = oracle.coarse_field([_box((-1.0, 0.0, -2.0), (1.0, 0.0, 2.0))])
    assert origin.tolist() == [-2.0, -1.0, -3.0]
    assert dims.tolist() == [13, 7, 19] and tex.size == 1729
    assert all(dims[a] * np.float32(0.32) >= [4.0, 2.0, 6.0][a] for a in range(3))


@pytest.mark.parametrize("boxes", [
    [((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5))],
    [((-3.0, 0.0, 1.0), (-1.0, 2.5, 4.0)), ((2.0, -1.0, -1.0), (5.0, 0.5, 0.25)), ((0.0, 3.0, -2.0), (0.5, 3.5, 6.0))],
])
def test_coarse_field_texels_match_populate(oracle, boxes):
    """populate (coarse_field.rs:240-266, as its populate_one_object test runs
    it): each texel is the binary16 of the smallest distance from the cell
    centre to an object AABB, starting from cell size x the largest dim."""
    F = np.float32
    origin, dims, tex = oracle.coarse_field([_box(lo, hi) for lo, hi in boxes])
    vs = F(0.32)
    start = vs * F(dims.max())
    z, y, x = np.meshgrid(*[np.arange(d, dtype=F) for d in dims[::-1]], indexing="ij")
    q = np.stack([origin[0] + (x + F(0.5)) * vs, origin[1] + (y + F(0.5)) * vs, origin[2] + (z + F(0.5)) * vs],
                 axis=-1).astype(F)
    best = np.full(q.shape[:-1], start, F)
    for lo, hi in boxes:
        best = np.minimum(best, _aabb_distance(q, lo, hi))
    want = best.astype(np.float16).view(np.uint16).ravel()
    assert_bits_equal(tex, want, "coarse texels")
    assert (tex == 0).any(), "cells inside a box hold 0"
