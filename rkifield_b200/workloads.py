"""Seeded synthetic workloads for the batched and served march.

Batching workload: views of uneven size (pixel area log-uniform between
128^2 and 2048^2, 16:9), each camera placed a few metres from a seeded
primitive and looking at it, plus incoherent secondary rays built from each
view's primary hits: shadow rays towards seeded point lights (soft-shadow
mode, the reference's soft_shadow, shade_common_shading.wgsl:9-33) and
cosine-weighted hemisphere ambient-occlusion rays (any-hit mode, 1 m).

Serving workload: a Poisson stream of requests mixing point-distance
queries, ray-cast batches and camera renders, with a CSG sphere add or
subtract every 50th request.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import scenes

SHADOW_BIAS = 0.08   # shade_common.wgsl:276
AO_BIAS = 0.02
AO_RADIUS = 1.0


@dataclasses.dataclass
class View:
    cam: object
    width: int
    height: int


def make_views(spec, prims, n_views: int, seed: int, area_lo: float = 128 ** 2,
               area_hi: float = 2048 ** 2) -> list[View]:
    rng = np.random.default_rng(seed)
    views = []
    for _ in range(n_views):
        area = math.exp(rng.uniform(math.log(area_lo), math.log(area_hi)))
        w = max(16, int(round(math.sqrt(area * 16.0 / 9.0))))
        h = max(9, int(round(w * 9.0 / 16.0)))
        p = prims[int(rng.integers(0, len(prims)))]
        c = p["centre"].astype(np.float64)
        dist = float(p["bound_radius"]) + rng.uniform(2.0, 8.0)
        u = rng.standard_normal(3)
        u /= np.linalg.norm(u)
        pos = c + dist * u
        views.append(View(scenes.camera_uniforms(pos, c, w, h), w, h))
    return views


def secondary_rays(gbuf: dict, width: int, height: int, cam, rng: np.random.Generator,
                   n_lights: int = 4, ao_per_hit: int = 8):
    """Shadow and AO rays for the hit pixels of one view's G-buffer.

    Returns (shadow_o, shadow_d, shadow_tmax), (ao_o, ao_d, ao_tmax) as
    float32 arrays (n,3)/(n,)."""
    hit = (gbuf["flags"] & 1) != 0
    idx = np.nonzero(hit)[0]
    n = idx.size
    if n == 0:
        z3 = np.zeros((0, 3), np.float32)
        z = np.zeros(0, np.float32)
        return (z3, z3, z), (z3, z3, z)
    t = gbuf["t"][idx].astype(np.float64)
    nrm = gbuf["normal"].reshape(-1, 3)[idx].astype(np.float64)
    # hit position from the camera ray of each pixel (ray_march.wgsl:1046-1068)
    px = (idx % width).astype(np.float64)
    py = (idx // width).astype(np.float64)
    u = (px + 0.5) / width
    v = (py + 0.5) / height
    fwd = np.array(cam.forward[:3], np.float64)
    right = np.array(cam.right[:3], np.float64)
    up = np.array(cam.up[:3], np.float64)
    d = fwd[None] + (u * 2 - 1)[:, None] * right[None] + (1 - v * 2)[:, None] * up[None]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pos = np.array(cam.position[:3], np.float64)[None] + d * t[:, None]
    # point lights around the view target
    target = np.array(cam.position[:3], np.float64) + fwd * float(np.median(t))
    lights = target[None] + rng.uniform(-10.0, 10.0, (n_lights, 3)) + np.array([0.0, 8.0, 0.0])
    so = pos + nrm * SHADOW_BIAS
    sd = lights[None, :, :] - so[:, None, :]
    st = np.linalg.norm(sd, axis=2)
    sd /= st[:, :, None]
    shadow = (so.repeat(n_lights, 0).astype(np.float32), sd.reshape(-1, 3).astype(np.float32),
              st.reshape(-1).astype(np.float32))
    # cosine-weighted hemisphere about the normal (Malley's method)
    r1 = rng.random((n, ao_per_hit))
    r2 = rng.random((n, ao_per_hit))
    rr = np.sqrt(r1)
    phi = 2 * np.pi * r2
    lx, ly, lz = rr * np.cos(phi), rr * np.sin(phi), np.sqrt(np.maximum(0.0, 1 - r1))
    a = np.where(np.abs(nrm[:, 0:1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    tx = np.cross(a, nrm)
    tx /= np.linalg.norm(tx, axis=1, keepdims=True)
    ty = np.cross(nrm, tx)
    ad = (lx[..., None] * tx[:, None] + ly[..., None] * ty[:, None] + lz[..., None] * nrm[:, None])
    ao_o = (pos + nrm * AO_BIAS).repeat(ao_per_hit, 0)
    ao = (ao_o.astype(np.float32), ad.reshape(-1, 3).astype(np.float32),
          np.full(n * ao_per_hit, AO_RADIUS, np.float32))
    return shadow, ao


@dataclasses.dataclass
class Request:
    kind: int            # 0 render, 1 rays, 2 points, 3 edit
    arrival_s: float
    n: int = 0
    width: int = 0
    height: int = 0
    cam: object = None
    o: np.ndarray | None = None
    d: np.ndarray | None = None
    tmax: np.ndarray | None = None
    points: np.ndarray | None = None
    edit: object = None


def make_request_stream(spec, prims, n_requests: int, seed: int, rate_hz: float = 2000.0,
                        edit_every: int = 50, ray_tmax: float = 32.0,
                        max_rays: int = 1 << 20, max_points: int = 65536,
                        render_area=(64 ** 2, 1920 * 1080)) -> list[Request]:
    """Poisson arrivals; request kinds drawn uniformly among points, rays and
    renders; sizes log-uniform; every `edit_every`-th request a CSG sphere."""
    from . import _abi as abi
    rng = np.random.default_rng(seed)
    half = spec.cube * 0.5
    t = 0.0
    reqs = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate_hz)
        if edit_every and (i + 1) % edit_every == 0:
            op = abi.rkf_edit_op()
            op.object_index = 0
            op.edit_type = int(rng.integers(0, 2))  # union / subtract
            op.shape_type = 0
            op.falloff = 1
            p = prims[int(rng.integers(0, len(prims)))]
            c = p["centre"] + rng.uniform(-1, 1, 3) * float(p["bound_radius"])
            op.position[:] = [float(x) for x in c]
            op.rotation[:] = (0.0, 0.0, 0.0, 1.0)
            op.dimensions[:] = (float(rng.uniform(0.1, 1.0)), 0.0, 0.0)
            op.strength = 1.0
            op.blend_k = 0.05
            op.material_id = int(rng.integers(1, 63))
            reqs.append(Request(3, t, edit=op))
            continue
        kind = int(rng.integers(0, 3))
        if kind == 2:
            n = int(round(math.exp(rng.uniform(0.0, math.log(max_points)))))
            reqs.append(Request(2, t, n=n, points=rng.uniform(-half, half, (n, 3)).astype(np.float32)))
        elif kind == 1:
            n = int(round(math.exp(rng.uniform(0.0, math.log(max_rays)))))
            o = rng.uniform(-half, half, (n, 3)).astype(np.float32)
            d = rng.standard_normal((n, 3))
            d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
            reqs.append(Request(1, t, n=n, o=o, d=d, tmax=np.full(n, ray_tmax, np.float32)))
        else:
            area = math.exp(rng.uniform(math.log(render_area[0]), math.log(render_area[1])))
            w = max(16, int(round(math.sqrt(area * 16.0 / 9.0))))
            h = max(9, int(round(w * 9.0 / 16.0)))
            p = prims[int(rng.integers(0, len(prims)))]
            c = p["centre"].astype(np.float64)
            u = rng.standard_normal(3)
            u /= np.linalg.norm(u)
            cam = scenes.camera_uniforms(c + (float(p["bound_radius"]) + rng.uniform(2, 8)) * u, c, w, h)
            reqs.append(Request(0, t, width=w, height=h, n=w * h, cam=cam))
    return reqs
