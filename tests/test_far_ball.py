"""The multi-object empty-space path rests on one bound: outside an analytic
object's ball (its primitive's bounding radius mapped through inverse_world,
widened by the largest EMPTY value and rounding bounds, rkf_testing_far_ball)
every FP32 value of evaluate_object exceeds the EMPTY values.  Checked here
with the oracle's FP32 evaluation (bit-identical to the device's) at points
just outside the balls of random spheres, boxes, capsules, tori and
cylinders, rotated, non-uniformly scaled and moved; planes, singular
transforms and non-positive scales have no ball.  Host only: no GPU."""
import ctypes as C

import numpy as np

from test_multi_empty_gpu import _rotation, _transformed

EMPTY_HI = np.float32(0.16 * (1.0 + 2.0 ** -16))  # 8 voxels of 2 cm, widened as the launch widens it


def _ball(lib, obj, empty_hi=EMPTY_HI):
    out = (C.c_float * 5)()
    ok = lib.rkf_testing_far_ball(C.byref(obj), C.c_float(empty_hi), out)
    return ok, np.array(out[:3], np.float64), float(out[3]), float(out[4])


def _points_outside(rng, c, a, b, n):
    """Points at the ball's radius a + b*P (P = the L1 magnitude of the point,
    which bounds |o| + |d| |tmax| for a ray through it from the origin),
    in random directions, rounded to FP32."""
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    r = np.full(n, a)
    for _ in range(4):  # r = a + b * |c + r u|_1, by fixed point (b is tiny)
        r = a + b * np.abs(c + r[:, None] * u).sum(axis=1)
    return (c + (r * (1.0 + 1e-7))[:, None] * u).astype(np.float32)


def test_values_outside_the_ball_exceed_the_empty_values(oracle):
    from rkifield_b200 import _abi as abi
    lib = abi.load_library()
    rng = np.random.default_rng(2024)
    params = {0: 1, 1: 3, 2: 2, 3: 2, 4: 2}  # sphere, box, capsule, torus, cylinder
    worst = np.inf
    for trial in range(150):
        ptype = trial % 5
        prm = tuple(float(x) for x in rng.uniform(0.05, 3.0, params[ptype]))
        centre = tuple(float(x) for x in rng.uniform(-60.0, 60.0, 3))
        scale = tuple(float(x) for x in rng.uniform(0.3, 3.0, 3)) if trial % 3 else (1.0, 1.0, 1.0)
        rot = _rotation(rng.normal(size=3), rng.uniform(0, np.pi)) if trial % 2 else np.eye(3)
        obj = _transformed(ptype, centre, prm, rot, scale, 1, 1)
        ok, c, a, b = _ball(lib, obj)
        assert ok, f"trial {trial}: no ball"
        # the centre is the local origin in world space; the radius is not absurd
        assert np.abs(c - np.asarray(centre)).max() < 1e-4 * (1 + np.abs(centre).max())
        reach = np.linalg.norm(prm) * max(scale) + 1.0
        assert reach * 0.2 < a < 10 * reach, (trial, a, reach)
        pts = _points_outside(rng, c, a, b, 4000)
        d, _, _ = oracle.query_points(oracle.Scene([obj]), pts.ravel())
        assert (d > EMPTY_HI).all(), (trial, float(d.min()))
        worst = min(worst, float(d.min()))
    assert worst < 1.0  # some balls are tight enough for the check to bite


def test_objects_without_a_ball(oracle):
    from rkifield_b200 import _abi as abi
    lib = abi.load_library()
    plane = _transformed(5, (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), np.eye(3), (1.0, 1.0, 1.0), 1, 1)
    assert _ball(lib, plane)[0] == 0
    flat = _transformed(0, (1.0, 2.0, 3.0), (1.0,), np.eye(3), (1.0, 1.0, 1.0), 1, 1)
    for i in range(3):
        flat.inverse_world[4 * i + 1] = 0.0  # a singular linear part
    assert _ball(lib, flat)[0] == 0
    neg = _transformed(0, (1.0, 2.0, 3.0), (1.0,), np.eye(3), (1.0, -1.0, 1.0), 1, 1)
    assert _ball(lib, neg)[0] == 0  # min_scale <= 0
    inf = _transformed(1, (1.0, 2.0, 3.0), (np.inf, 1.0, 1.0), np.eye(3), (1.0, 1.0, 1.0), 1, 1)
    assert _ball(lib, inf)[0] == 0
