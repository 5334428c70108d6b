"""Seeded synthetic scenes and cameras for the march workloads.

A scene is a list of analytic primitives (spheres, boxes, capsules with
random rotations) whose smooth union (polynomial smin, ``sdf.rs:48-51``) is
voxelized into one object, the way ``World::voxelize`` turns an SDF closure
into a brick map (``crates/rkf-core/src/voxelize_object.rs:53-182``).

The camera follows the reference fly camera: yaw/pitch give
``forward = (-sin(yaw)cos(pitch), sin(pitch), -cos(yaw)cos(pitch))``,
``right = (cos(yaw), 0, -sin(yaw))`` and ``up = normalize(right x forward)``
(``crates/rkf-render/src/camera.rs:76-93``); the uniforms pre-scale right by
``tan(fov/2)*aspect`` and up by ``tan(fov/2)`` (``camera.rs:161-184``).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import _abi as abi

PRIM_SPHERE, PRIM_BOX, PRIM_CAPSULE = 0, 1, 2


@dataclasses.dataclass
class SceneSpec:
    """Definition of one seeded workload scene."""

    name: str
    n_prims: int
    cube: float          # edge of the cube the centres are drawn from (m)
    voxel_size: float    # m
    size_lo: float = 0.2
    size_hi: float = 2.0
    smooth_k: float = 0.1
    band_voxels: float = 3.0
    cut_distance: float = 1.0
    seed: int = 1
    max_steps: int = 128


# The workloads: the CPU-runnable plain scene (64 primitives in a 32 m cube at
# 4 cm, ~20k bricks) and the large single-GPU scene (512 primitives in a 256 m
# cube at 2 cm, ~500k bricks).
SCENE_SMALL = SceneSpec("prims64_cube32m_vs4cm", 64, 32.0, 0.04, seed=1, max_steps=128)
SCENE_LARGE = SceneSpec("prims512_cube256m_vs2cm", 512, 256.0, 0.02, seed=2, max_steps=256)


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniform random rotation (Shoemake's quaternion method) as a row-major 3x3."""
    u1, u2, u3 = rng.random(3)
    q = np.array([
        math.sqrt(1 - u1) * math.sin(2 * math.pi * u2),
        math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
        math.sqrt(u1) * math.sin(2 * math.pi * u3),
        math.sqrt(u1) * math.cos(2 * math.pi * u3),
    ])
    x, y, z, w = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ], dtype=np.float64)


def make_prims(spec: SceneSpec) -> np.ndarray:
    """Seeded primitive list as an ``rkf_prim`` structured array."""
    rng = np.random.default_rng(spec.seed)
    prims = np.zeros(spec.n_prims, dtype=abi.PRIM_DTYPE)
    half = spec.cube * 0.5
    for i in range(spec.n_prims):
        kind = int(rng.integers(0, 3))
        centre = rng.uniform(-half, half, 3)
        p = prims[i]
        p["type"] = kind
        p["material"] = 1 + (i % 63)
        p["centre"] = centre.astype(np.float32)
        if kind == PRIM_SPHERE:
            r = rng.uniform(spec.size_lo, spec.size_hi)
            p["params"] = np.float32([r, 0.0, 0.0])
            p["rot"] = np.eye(3, dtype=np.float32).ravel()
            bound = r
        elif kind == PRIM_BOX:
            h = rng.uniform(spec.size_lo, spec.size_hi, 3)
            p["params"] = h.astype(np.float32)
            p["rot"] = _random_rotation(rng).astype(np.float32).ravel()
            bound = float(np.linalg.norm(h))
        else:
            r = rng.uniform(spec.size_lo, spec.size_hi)
            hh = rng.uniform(spec.size_lo, spec.size_hi)
            p["params"] = np.float32([r, hh, 0.0])
            p["rot"] = _random_rotation(rng).astype(np.float32).ravel()
            bound = r + hh
        # bounding radius with a relative margin so float rounding never
        # makes a primitive reach outside it
        p["bound_radius"] = np.float32(bound * 1.001 + 1e-4)
    return prims


def scene_aabb(prims: np.ndarray, margin: float) -> tuple[np.ndarray, np.ndarray]:
    c = prims["centre"].astype(np.float64)
    b = prims["bound_radius"].astype(np.float64)[:, None]
    lo = (c - b).min(axis=0) - margin
    hi = (c + b).max(axis=0) + margin
    return lo.astype(np.float32), hi.astype(np.float32)


def voxelize_params(spec: SceneSpec, prims: np.ndarray, object_id: int = 1):
    vp = abi.rkf_voxelize_params()
    vp.voxel_size = spec.voxel_size
    vp.smooth_k = spec.smooth_k
    vp.band_voxels = spec.band_voxels
    vp.cut_distance = spec.cut_distance
    lo, hi = scene_aabb(prims, margin=2 * 8 * spec.voxel_size)
    for a in range(3):
        vp.aabb_min[a] = float(lo[a])
        vp.aabb_max[a] = float(hi[a])
    vp.band_rule = abi.RKF_BAND_VOXELS
    vp.object_id = object_id
    return vp


def camera_uniforms(position, target, width: int, height: int, fov_degrees: float = 60.0):
    """``Camera::uniforms`` for a camera at ``position`` looking at ``target``."""
    pos = np.asarray(position, dtype=np.float32)
    d = np.asarray(target, dtype=np.float64) - pos.astype(np.float64)
    d /= np.linalg.norm(d)
    pitch = np.float32(math.asin(max(-1.0, min(1.0, d[1]))))
    yaw = np.float32(math.atan2(-d[0], -d[2]))
    sy, cy = np.float32(math.sin(yaw)), np.float32(math.cos(yaw))
    sp, cp = np.float32(math.sin(pitch)), np.float32(math.cos(pitch))
    fwd = np.array([-sy * cp, sp, -cy * cp], dtype=np.float32)
    right = np.array([cy, 0.0, -sy], dtype=np.float32)
    up = np.cross(right, fwd).astype(np.float32)
    up = (up / np.float32(np.sqrt(np.dot(up, up)))).astype(np.float32)
    half_fov_tan = np.float32(math.tan(math.radians(fov_degrees) * 0.5))
    aspect = np.float32(width) / np.float32(height)
    r = right * half_fov_tan * aspect
    u = up * half_fov_tan
    cam = abi.rkf_camera()
    for a in range(3):
        cam.position[a] = float(pos[a])
        cam.forward[a] = float(fwd[a])
        cam.right[a] = float(r[a])
        cam.up[a] = float(u[a])
    cam.resolution[0] = float(width)
    cam.resolution[1] = float(height)
    for c in range(4):  # prev_vp = identity (column-major)
        cam.prev_vp[c * 4 + c] = 1.0
    return cam


def seeded_camera(spec: SceneSpec, width: int, height: int, seed: int, inside: bool = False,
                  distance: float | None = None):
    """Camera at a seeded pose looking at the scene centre (outside the cube
    by default, at 0.6 of the half-extent when ``inside``)."""
    rng = np.random.default_rng(seed)
    az = rng.uniform(0, 2 * math.pi)
    el = rng.uniform(-0.35, 0.6)
    if distance is None:
        distance = spec.cube * (0.3 if inside else 1.25)
    pos = distance * np.array([math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az)])
    return camera_uniforms(pos, (0.0, 0.0, 0.0), width, height)


def march_params(spec: SceneSpec, max_distance: float | None = None):
    p = abi.rkf_march_params()
    abi.march_params_default(p)
    p.scene.max_steps = spec.max_steps
    p.scene.hit_threshold = np.float32(0.5) * np.float32(spec.voxel_size)
    p.scene.max_distance = max_distance if max_distance is not None else spec.cube * 3.0
    return p
