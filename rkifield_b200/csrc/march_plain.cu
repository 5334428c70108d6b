// march_plain.cu — the plain march: a direct port of ray_march.wgsl's main
// (:1036-1112) with ray_march_brute (:776-858), one thread per pixel in 8x8
// blocks like the shader's workgroup, reading the reference layouts: the AoS
// VoxelSample pool (8 bytes per voxel) and the packed flat brick maps
// (brick_maps[offset + bx + by*dx + bz*dx*dy]).  Every step performs the
// shader's 8 map reads and 8 pool reads and its material lookup.  This is the
// one-launch-per-request baseline the batched march is measured against.
#include <cstring>

#include "ctx.h"
#include "march.h"

namespace rkf {

namespace detail {

struct PlainParams {
  SceneDev s;
  rkf_march_params p;
  float pos[3], fwd[3], right[3], up[3], jitter[2];
  float prev_vp[16];
  uint32_t w, h;
  float* t;
  float* normal;
  uint32_t* slot;
  uint16_t* material;
  uint16_t* flags;
  float* position;
  uint32_t* packed;
  float* motion;
};

__device__ __forceinline__ uint32_t plain_lookup(const PlainParams& kp, const ObjDev& o, uint32_t bx,
                                                 uint32_t by, uint32_t bz) {
  if (o.has_flat)
    return kp.s.flat_maps[static_cast<size_t>(o.map_off) + bx + static_cast<size_t>(by) * o.bdims[0] +
                          static_cast<size_t>(bz) * o.bdims[0] * o.bdims[1]];
  return lookup2(kp.s, o, bx, by, bz);
}

// sample_voxel_at / sample_voxel_at_grad (ray_march.wgsl:270-315)
__device__ __forceinline__ float plain_voxel(const PlainParams& kp, const ObjDev& o, int vx, int vy,
                                             int vz, bool grad) {
  const int cx = clampi(vx, 0, o.tv[0] - 1), cy = clampi(vy, 0, o.tv[1] - 1),
            cz = clampi(vz, 0, o.tv[2] - 1);
  const uint32_t slot = plain_lookup(kp, o, cx / 8, cy / 8, cz / 8);
  if (slot == RKF_EMPTY_SLOT) return o.be;
  if (slot == RKF_INTERIOR_SLOT) return grad ? -o.be : -(o.vs * 2.0f);
  const size_t i = static_cast<size_t>(slot) * 512 + (cx % 8) + (cy % 8) * 8 + (cz % 8) * 64;
  return __half2float(__ushort_as_half(static_cast<uint16_t>(kp.s.aos[i].x & 0xFFFFu)));
}

// sample_voxelized / sample_voxelized_grad (ray_march.wgsl:353-498)
__device__ float plain_sample(const PlainParams& kp, const ObjDev& o, float lx, float ly, float lz,
                              bool grad) {
  const float gpx = __fadd_rn(lx, o.half_gs[0]), gpy = __fadd_rn(ly, o.half_gs[1]),
              gpz = __fadd_rn(lz, o.half_gs[2]);
  const float clx = clampf(gpx, o.lo, o.hi[0]), cly = clampf(gpy, o.lo, o.hi[1]),
              clz = clampf(gpz, o.lo, o.hi[2]);
  const float outside = len3(__fsub_rn(gpx, clx), __fsub_rn(gpy, cly), __fsub_rn(gpz, clz));
  if (outside > o.be2) return outside;
  if (!grad && o.has_geom) {
    const float gd = len3(__fsub_rn(lx, clampf(lx, o.gmin[0], o.gmax[0])),
                          __fsub_rn(ly, clampf(ly, o.gmin[1], o.gmax[1])),
                          __fsub_rn(lz, clampf(lz, o.gmin[2], o.gmax[2])));
    if (gd > o.be) return gd;
  }
  const float vcx = __fsub_rn(__fdiv_rn(clx, o.vs), 0.5f);
  const float vcy = __fsub_rn(__fdiv_rn(cly, o.vs), 0.5f);
  const float vcz = __fsub_rn(__fdiv_rn(clz, o.vs), 0.5f);
  const int x0 = static_cast<int>(floorf(vcx)), y0 = static_cast<int>(floorf(vcy)),
            z0 = static_cast<int>(floorf(vcz));
  const float tx = __fsub_rn(vcx, static_cast<float>(x0)), ty = __fsub_rn(vcy, static_cast<float>(y0)),
              tz = __fsub_rn(vcz, static_cast<float>(z0));
  const float c000 = plain_voxel(kp, o, x0, y0, z0, grad);
  const float c100 = plain_voxel(kp, o, x0 + 1, y0, z0, grad);
  const float c010 = plain_voxel(kp, o, x0, y0 + 1, z0, grad);
  const float c110 = plain_voxel(kp, o, x0 + 1, y0 + 1, z0, grad);
  const float c001 = plain_voxel(kp, o, x0, y0, z0 + 1, grad);
  const float c101 = plain_voxel(kp, o, x0 + 1, y0, z0 + 1, grad);
  const float c011 = plain_voxel(kp, o, x0, y0 + 1, z0 + 1, grad);
  const float c111 = plain_voxel(kp, o, x0 + 1, y0 + 1, z0 + 1, grad);
  const float c00 = mixf(c000, c100, tx), c10 = mixf(c010, c110, tx);
  const float c01 = mixf(c001, c101, tx), c11 = mixf(c011, c111, tx);
  const float c0 = mixf(c00, c10, ty), c1 = mixf(c01, c11, ty);
  return __fadd_rn(mixf(c0, c1, tz), outside);
}

// nearest voxel (ray_march.wgsl:540-596); returns slot or sentinel
__device__ uint32_t plain_nearest(const PlainParams& kp, const ObjDev& o, float lx, float ly, float lz,
                                  size_t* vi) {
  const float gpx = __fadd_rn(lx, o.half_gs[0]), gpy = __fadd_rn(ly, o.half_gs[1]),
              gpz = __fadd_rn(lz, o.half_gs[2]);
  if (gpx < 0.0f || gpy < 0.0f || gpz < 0.0f || gpx >= o.gs[0] || gpy >= o.gs[1] || gpz >= o.gs[2])
    return RKF_EMPTY_SLOT;
  const int x = clampi(static_cast<int>(floorf(__fdiv_rn(gpx, o.vs))), 0, o.tv[0] - 1);
  const int y = clampi(static_cast<int>(floorf(__fdiv_rn(gpy, o.vs))), 0, o.tv[1] - 1);
  const int z = clampi(static_cast<int>(floorf(__fdiv_rn(gpz, o.vs))), 0, o.tv[2] - 1);
  const uint32_t slot = plain_lookup(kp, o, x / 8, y / 8, z / 8);
  *vi = static_cast<size_t>(slot) * 512 + (x % 8) + (y % 8) * 8 + (z % 8) * 64;
  return slot;
}

// evaluate_object (ray_march.wgsl:600-634) with the eager material read
__device__ float plain_eval(const PlainParams& kp, const ObjDev& o, float wx, float wy, float wz,
                            uint32_t* mat) {
  if (o.sdf_type == RKF_SDF_NONE) {
    *mat = 0;
    return kMaxFloat;
  }
  float lx, ly, lz;
  to_local(o, wx, wy, wz, lx, ly, lz);
  float d;
  if (o.sdf_type == RKF_SDF_ANALYTICAL) {
    d = analytic_sdf(o, lx, ly, lz);
    *mat = o.material_id;
  } else {
    d = plain_sample(kp, o, lx, ly, lz, false);
    *mat = 0;
    if (d < o.vs16) {
      size_t vi;
      const uint32_t slot = plain_nearest(kp, o, lx, ly, lz, &vi);
      if (slot < RKF_INTERIOR_SLOT) *mat = (kp.s.aos[vi].x >> 16) & 0x3Fu;
    }
  }
  return __fmul_rn(d, o.min_scale);
}

__global__ void __launch_bounds__(64) k_march_plain(PlainParams kp) {
  extern __shared__ ObjDev objs[];
  const uint32_t tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (uint32_t i = tid; i < kp.s.n_objs; i += blockDim.x * blockDim.y) objs[i] = kp.s.objs[i];
  __syncthreads();
  const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= kp.w || py >= kp.h) return;
  const rkf_march_params& p = kp.p;
  const uint32_t idx = py * kp.w + px;
  // ray generation (ray_march.wgsl:1046-1053)
  const float u = __fdiv_rn(__fadd_rn(__fadd_rn(static_cast<float>(px), 0.5f), kp.jitter[0]), static_cast<float>(kp.w));
  const float v = __fdiv_rn(__fadd_rn(__fadd_rn(static_cast<float>(py), 0.5f), kp.jitter[1]), static_cast<float>(kp.h));
  const float nx = __fsub_rn(__fmul_rn(u, 2.0f), 1.0f), ny = __fsub_rn(1.0f, __fmul_rn(v, 2.0f));
  const float vx = __fadd_rn(__fadd_rn(kp.fwd[0], __fmul_rn(kp.right[0], nx)), __fmul_rn(kp.up[0], ny));
  const float vy = __fadd_rn(__fadd_rn(kp.fwd[1], __fmul_rn(kp.right[1], nx)), __fmul_rn(kp.up[1], ny));
  const float vz = __fadd_rn(__fadd_rn(kp.fwd[2], __fmul_rn(kp.right[2], nx)), __fmul_rn(kp.up[2], ny));
  const float dl = len3(vx, vy, vz);
  const float dx = __fdiv_rn(vx, dl), dy = __fdiv_rn(vy, dl), dz = __fdiv_rn(vz, dl);
  const float ox = kp.pos[0], oy = kp.pos[1], oz = kp.pos[2];
  const float sx = fabsf(dx) < 1e-10f ? 1e-10f : dx, sy = fabsf(dy) < 1e-10f ? 1e-10f : dy,
              sz = fabsf(dz) < 1e-10f ? 1e-10f : dz;
  // ray_march_brute (:776-858)
  float t = 0.0f, prev_t = 0.0f, prev_dist = kMaxFloat, rt = kMaxFloat;
  uint32_t near = 0, step = 0, rmat = 0, robj = 0;
  bool hit = false, bisected = false;
  for (; step < p.hard_max_steps; ++step) {
    if (t > p.scene.max_distance || near >= p.scene.max_steps) break;
    const float qx = __fadd_rn(ox, __fmul_rn(sx, t)), qy = __fadd_rn(oy, __fmul_rn(sy, t)),
                qz = __fadd_rn(oz, __fmul_rn(sz, t));
    float md = kMaxFloat;
    uint32_t bm = 0, bi = 0;
    for (uint32_t i = 0; i < kp.s.n_objs; ++i) {
      uint32_t m;
      const float d = plain_eval(kp, objs[i], qx, qy, qz, &m);
      if (d < md) {
        md = d;
        bm = m;
        bi = i;
      }
    }
    if (md < 0.0f && prev_dist > p.scene.hit_threshold) {
      float lo = prev_t, hi = t;
      uint32_t bmat = bm;
      for (uint32_t b = 0; b < p.bisect_steps; ++b) {
        const float mid = __fmul_rn(__fadd_rn(lo, hi), 0.5f);
        uint32_t m;
        const float d = plain_eval(kp, objs[bi], __fadd_rn(ox, __fmul_rn(sx, mid)),
                                   __fadd_rn(oy, __fmul_rn(sy, mid)), __fadd_rn(oz, __fmul_rn(sz, mid)), &m);
        if (d < 0.0f) {
          hi = mid;
        } else {
          lo = mid;
          bmat = m;
        }
      }
      rt = __fmul_rn(__fadd_rn(lo, hi), 0.5f);
      hit = bisected = true;
      rmat = bmat;
      robj = bi;
      break;
    }
    if (md < p.scene.hit_threshold) {
      rt = t;
      hit = true;
      rmat = bm;
      robj = bi;
      break;
    }
    if (md < p.near_surface_threshold) near++;
    prev_t = t;
    prev_dist = md;
    t = __fadd_rn(t, fmax_(md, p.min_step));
  }
  uint16_t flags = 0;
  float nxo = 0, nyo = 0, nzo = 0, hx = 0, hy = 0, hz = 0, sdf_hit = 0;
  uint32_t slot = RKF_EMPTY_SLOT, sec = 0, blend = 0;
  if (hit) {
    flags |= RKF_FLAG_HIT;
    if (bisected) flags |= RKF_FLAG_BISECTED;
    const ObjDev& o = objs[robj];
    hx = __fadd_rn(ox, __fmul_rn(dx, rt));
    hy = __fadd_rn(oy, __fmul_rn(dy, rt));
    hz = __fadd_rn(oz, __fmul_rn(dz, rt));
    // compute_normal_for_object (:1003-1032)
    if (o.sdf_type == RKF_SDF_VOXELIZED) {
      float lx, ly, lz;
      to_local(o, hx, hy, hz, lx, ly, lz);
      const float e = __fmul_rn(o.vs, 2.0f);
      const float g0 = __fsub_rn(plain_sample(kp, o, __fadd_rn(lx, e), ly, lz, true),
                                 plain_sample(kp, o, __fsub_rn(lx, e), ly, lz, true));
      const float g1 = __fsub_rn(plain_sample(kp, o, lx, __fadd_rn(ly, e), lz, true),
                                 plain_sample(kp, o, lx, __fsub_rn(ly, e), lz, true));
      const float g2 = __fsub_rn(plain_sample(kp, o, lx, ly, __fadd_rn(lz, e), true),
                                 plain_sample(kp, o, lx, ly, __fsub_rn(lz, e), true));
      const float wx = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[0], g0), __fmul_rn(o.m[1], g1)), __fmul_rn(o.m[2], g2)), __fmul_rn(o.m[3], 0.0f));
      const float wy = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[4], g0), __fmul_rn(o.m[5], g1)), __fmul_rn(o.m[6], g2)), __fmul_rn(o.m[7], 0.0f));
      const float wz = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[8], g0), __fmul_rn(o.m[9], g1)), __fmul_rn(o.m[10], g2)), __fmul_rn(o.m[11], 0.0f));
      const float l = len3(wx, wy, wz);
      if (l < 1e-10f) {
        nyo = 1.0f;
      } else {
        nxo = __fdiv_rn(wx, l); nyo = __fdiv_rn(wy, l); nzo = __fdiv_rn(wz, l);
      }
      size_t vi;
      slot = plain_nearest(kp, o, lx, ly, lz, &vi);
      if (slot < RKF_INTERIOR_SLOT) {
        const uint2 w = kp.s.aos[vi];
        sec = (w.x >> 22) & 0x3Fu;
        blend = (w.y >> 24) & 0xFFu;
      }
      sdf_hit = plain_sample(kp, o, lx, ly, lz, false);
    } else {
      const float e = __fmul_rn(p.scene.hit_threshold, 10.0f);
      uint32_t m;
      const float a = __fsub_rn(plain_eval(kp, o, __fadd_rn(hx, e), hy, hz, &m), plain_eval(kp, o, __fsub_rn(hx, e), hy, hz, &m));
      const float b = __fsub_rn(plain_eval(kp, o, hx, __fadd_rn(hy, e), hz, &m), plain_eval(kp, o, hx, __fsub_rn(hy, e), hz, &m));
      const float c = __fsub_rn(plain_eval(kp, o, hx, hy, __fadd_rn(hz, e), &m), plain_eval(kp, o, hx, hy, __fsub_rn(hz, e), &m));
      const float l = len3(a, b, c);
      nxo = __fdiv_rn(a, l); nyo = __fdiv_rn(b, l); nzo = __fdiv_rn(c, l);
    }
  } else if (step >= p.hard_max_steps || near >= p.scene.max_steps) {
    flags |= RKF_FLAG_STEPS_OUT;
  }
  kp.t[idx] = hit ? rt : kMaxFloat;
  kp.normal[3 * static_cast<size_t>(idx)] = nxo;
  kp.normal[3 * static_cast<size_t>(idx) + 1] = nyo;
  kp.normal[3 * static_cast<size_t>(idx) + 2] = nzo;
  kp.slot[idx] = slot;
  kp.material[idx] = static_cast<uint16_t>(hit ? rmat : 0u);
  kp.flags[idx] = flags;
  if (kp.position)
    reinterpret_cast<float4*>(kp.position)[idx] = hit ? make_float4(hx, hy, hz, rt) : make_float4(0.f, 0.f, 0.f, kMaxFloat);
  if (kp.packed)
    kp.packed[idx] = hit ? ((rmat & 0x3Fu) | (sec << 6) | (blend << 12) | (objs[robj].object_id << 24)) : 0u;
  if (kp.motion) {
    float4 mv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (hit) {
      const float* m = kp.prev_vp;
      const float cx = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], hx), __fmul_rn(m[4], hy)), __fmul_rn(m[8], hz)), __fmul_rn(m[12], 1.0f));
      const float cy = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[1], hx), __fmul_rn(m[5], hy)), __fmul_rn(m[9], hz)), __fmul_rn(m[13], 1.0f));
      const float cw = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[3], hx), __fmul_rn(m[7], hy)), __fmul_rn(m[11], hz)), __fmul_rn(m[15], 1.0f));
      float mox = 0.f, moy = 0.f;
      if (cw > 0.0f) {
        const float ndx = __fdiv_rn(cx, cw), ndy = __fdiv_rn(cy, cw);
        const float pu = __fadd_rn(__fmul_rn(ndx, 0.5f), 0.5f), pv = __fsub_rn(0.5f, __fmul_rn(ndy, 0.5f));
        const float cu = __fdiv_rn(__fadd_rn(static_cast<float>(px), 0.5f), static_cast<float>(kp.w));
        const float cv = __fdiv_rn(__fadd_rn(static_cast<float>(py), 0.5f), static_cast<float>(kp.h));
        mox = __fsub_rn(cu, pu);
        moy = __fsub_rn(cv, pv);
      }
      mv = make_float4(mox, moy, 1.0f, sdf_hit);
    }
    reinterpret_cast<float4*>(kp.motion)[idx] = mv;
  }
}

struct PlainRays {
  PlainParams kp;  // scene, parameters (view fields unused)
  const float* o;
  const float* d;
  const float* tmax;
  uint32_t n, mode;
};

// One thread per ray: the same reference loop for generic ray casts
// (closest hit, any hit, soft shadow of shade_common_shading.wgsl:9-33).
__global__ void __launch_bounds__(128) k_trace_plain(PlainRays r) {
  extern __shared__ ObjDev objs[];
  for (uint32_t i = threadIdx.x; i < r.kp.s.n_objs; i += blockDim.x) objs[i] = r.kp.s.objs[i];
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.n) return;
  const PlainParams& kp = r.kp;
  const rkf_march_params& p = kp.p;
  const float ox = r.o[3 * static_cast<size_t>(i)], oy = r.o[3 * static_cast<size_t>(i) + 1],
              oz = r.o[3 * static_cast<size_t>(i) + 2];
  const float dx = r.d[3 * static_cast<size_t>(i)], dy = r.d[3 * static_cast<size_t>(i) + 1],
              dz = r.d[3 * static_cast<size_t>(i) + 2];
  const float tmax = r.tmax[i];
  if (r.mode == RKF_TRACE_SHADOW) {
    float shadow = 1.0f, t = 0.005f;
    uint32_t near = 0, it = 0;
    bool occluded = false;
    for (; it < 256u; ++it) {
      if (near >= 32u || t > tmax) break;
      const float qx = __fadd_rn(ox, __fmul_rn(dx, t)), qy = __fadd_rn(oy, __fmul_rn(dy, t)),
                  qz = __fadd_rn(oz, __fmul_rn(dz, t));
      float d = kMaxFloat;
      for (uint32_t k = 0; k < kp.s.n_objs; ++k) {
        uint32_t m;
        d = fmin_(d, plain_eval(kp, objs[k], qx, qy, qz, &m));
      }
      if (d < 0.005f) {
        occluded = true;
        break;
      }
      if (d < 0.02f) {
        shadow = fmin_(shadow, __fdiv_rn(__fmul_rn(16.0f, d), t));
        near++;
      }
      t = __fadd_rn(t, fmax_(d, 0.005f));
    }
    kp.t[i] = occluded ? 0.0f : clampf(shadow, 0.0f, 1.0f);
    if (kp.flags) kp.flags[i] = occluded ? RKF_FLAG_HIT : 0;
    return;
  }
  const float sx = fabsf(dx) < 1e-10f ? 1e-10f : dx, sy = fabsf(dy) < 1e-10f ? 1e-10f : dy,
              sz = fabsf(dz) < 1e-10f ? 1e-10f : dz;
  float t = 0.0f, prev_t = 0.0f, prev_dist = kMaxFloat, rt = kMaxFloat;
  uint32_t near = 0, step = 0, rmat = 0, robj = 0;
  bool hit = false, bisected = false;
  for (; step < p.hard_max_steps; ++step) {
    if (t > tmax || near >= p.scene.max_steps) break;
    const float qx = __fadd_rn(ox, __fmul_rn(sx, t)), qy = __fadd_rn(oy, __fmul_rn(sy, t)),
                qz = __fadd_rn(oz, __fmul_rn(sz, t));
    float md = kMaxFloat;
    uint32_t bm = 0, bi = 0;
    for (uint32_t k = 0; k < kp.s.n_objs; ++k) {
      uint32_t m;
      const float d = plain_eval(kp, objs[k], qx, qy, qz, &m);
      if (d < md) {
        md = d;
        bm = m;
        bi = k;
      }
    }
    if (md < 0.0f && prev_dist > p.scene.hit_threshold) {
      if (r.mode == RKF_TRACE_ANY) {
        rt = t;
        hit = true;
        robj = bi;
        break;
      }
      float lo = prev_t, hi = t;
      uint32_t bmat = bm;
      for (uint32_t b = 0; b < p.bisect_steps; ++b) {
        const float mid = __fmul_rn(__fadd_rn(lo, hi), 0.5f);
        uint32_t m;
        const float d = plain_eval(kp, objs[bi], __fadd_rn(ox, __fmul_rn(sx, mid)),
                                   __fadd_rn(oy, __fmul_rn(sy, mid)), __fadd_rn(oz, __fmul_rn(sz, mid)), &m);
        if (d < 0.0f) {
          hi = mid;
        } else {
          lo = mid;
          bmat = m;
        }
      }
      rt = __fmul_rn(__fadd_rn(lo, hi), 0.5f);
      hit = bisected = true;
      rmat = bmat;
      robj = bi;
      break;
    }
    if (md < p.scene.hit_threshold) {
      rt = t;
      hit = true;
      rmat = bm;
      robj = bi;
      break;
    }
    if (md < p.near_surface_threshold) near++;
    prev_t = t;
    prev_dist = md;
    t = __fadd_rn(t, fmax_(md, p.min_step));
  }
  const bool steps_out = !hit && (step >= p.hard_max_steps || near >= p.scene.max_steps);
  kp.t[i] = hit ? rt : kMaxFloat;
  if (r.mode == RKF_TRACE_ANY) {
    if (kp.flags) kp.flags[i] = hit ? RKF_FLAG_HIT : (steps_out ? RKF_FLAG_STEPS_OUT : 0);
    return;
  }
  uint16_t flags = hit ? static_cast<uint16_t>(RKF_FLAG_HIT | (bisected ? RKF_FLAG_BISECTED : 0))
                       : static_cast<uint16_t>(steps_out ? RKF_FLAG_STEPS_OUT : 0);
  float nxo = 0, nyo = 0, nzo = 0;
  uint32_t slot = RKF_EMPTY_SLOT;
  if (hit) {
    const ObjDev& o = objs[robj];
    const float hx = __fadd_rn(ox, __fmul_rn(dx, rt)), hy = __fadd_rn(oy, __fmul_rn(dy, rt)),
                hz = __fadd_rn(oz, __fmul_rn(dz, rt));
    if (o.sdf_type == RKF_SDF_VOXELIZED) {
      float lx, ly, lz;
      to_local(o, hx, hy, hz, lx, ly, lz);
      const float e = __fmul_rn(o.vs, 2.0f);
      const float g0 = __fsub_rn(plain_sample(kp, o, __fadd_rn(lx, e), ly, lz, true),
                                 plain_sample(kp, o, __fsub_rn(lx, e), ly, lz, true));
      const float g1 = __fsub_rn(plain_sample(kp, o, lx, __fadd_rn(ly, e), lz, true),
                                 plain_sample(kp, o, lx, __fsub_rn(ly, e), lz, true));
      const float g2 = __fsub_rn(plain_sample(kp, o, lx, ly, __fadd_rn(lz, e), true),
                                 plain_sample(kp, o, lx, ly, __fsub_rn(lz, e), true));
      const float wx = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[0], g0), __fmul_rn(o.m[1], g1)), __fmul_rn(o.m[2], g2)), __fmul_rn(o.m[3], 0.0f));
      const float wy = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[4], g0), __fmul_rn(o.m[5], g1)), __fmul_rn(o.m[6], g2)), __fmul_rn(o.m[7], 0.0f));
      const float wz = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[8], g0), __fmul_rn(o.m[9], g1)), __fmul_rn(o.m[10], g2)), __fmul_rn(o.m[11], 0.0f));
      const float l = len3(wx, wy, wz);
      if (l < 1e-10f) {
        nyo = 1.0f;
      } else {
        nxo = __fdiv_rn(wx, l); nyo = __fdiv_rn(wy, l); nzo = __fdiv_rn(wz, l);
      }
      size_t vi;
      slot = plain_nearest(kp, o, lx, ly, lz, &vi);
    } else {
      const float e = __fmul_rn(p.scene.hit_threshold, 10.0f);
      uint32_t m;
      const float a = __fsub_rn(plain_eval(kp, o, __fadd_rn(hx, e), hy, hz, &m), plain_eval(kp, o, __fsub_rn(hx, e), hy, hz, &m));
      const float b = __fsub_rn(plain_eval(kp, o, hx, __fadd_rn(hy, e), hz, &m), plain_eval(kp, o, hx, __fsub_rn(hy, e), hz, &m));
      const float c = __fsub_rn(plain_eval(kp, o, hx, hy, __fadd_rn(hz, e), &m), plain_eval(kp, o, hx, hy, __fsub_rn(hz, e), &m));
      const float l = len3(a, b, c);
      nxo = __fdiv_rn(a, l); nyo = __fdiv_rn(b, l); nzo = __fdiv_rn(c, l);
    }
  }
  if (kp.normal) {
    kp.normal[3 * static_cast<size_t>(i)] = nxo;
    kp.normal[3 * static_cast<size_t>(i) + 1] = nyo;
    kp.normal[3 * static_cast<size_t>(i) + 2] = nzo;
  }
  if (kp.slot) kp.slot[i] = slot;
  if (kp.material) kp.material[i] = static_cast<uint16_t>(hit ? rmat : 0u);
  if (kp.flags) kp.flags[i] = flags;
}

}  // namespace detail

rkf_status launch_trace_plain(Ctx* c, const float* o, const float* d, const float* tmax, uint32_t n,
                              uint32_t mode, const rkf_march_params* p, const rkf_hits& out,
                              cudaStream_t st) {
  if (!c->aos.p) return fail(RKF_UNSUPPORTED, "rkf_trace_rays_plain: context keeps no reference (AoS) pool");
  if (n == 0) return RKF_OK;
  detail::PlainRays r;
  std::memset(&r, 0, sizeof(r));
  r.kp.s = c->scene_dev();
  r.kp.p = *p;
  r.kp.p.scene.num_objects = c->obj_count();
  r.kp.t = out.t;
  r.kp.normal = out.normal;
  r.kp.slot = out.slot;
  r.kp.material = out.material;
  r.kp.flags = out.flags;
  r.o = o;
  r.d = d;
  r.tmax = tmax;
  r.n = n;
  r.mode = mode;
  const size_t smem = sizeof(ObjDev) * (c->obj_count() ? c->obj_count() : 1);
  detail::k_trace_plain<<<(n + 127) / 128, 128, smem, st>>>(r);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  return RKF_OK;
}

rkf_status launch_plain(Ctx* c, const rkf_camera* cam, const rkf_march_params* p, uint32_t w,
                        uint32_t h, const rkf_gbuffer& out, cudaStream_t st) {
  if (!c->aos.p) return fail(RKF_UNSUPPORTED, "rkf_march_plain: context keeps no reference (AoS) pool");
  if (p->strategy != RKF_STRATEGY_BRUTE)
    return fail(RKF_UNSUPPORTED, "rkf_march_plain: the baseline runs the brute strategy only");
  detail::PlainParams kp;
  kp.s = c->scene_dev();
  kp.p = *p;
  kp.p.scene.num_objects = c->obj_count();
  for (int a = 0; a < 3; ++a) {
    kp.pos[a] = cam->position[a];
    kp.fwd[a] = cam->forward[a];
    kp.right[a] = cam->right[a];
    kp.up[a] = cam->up[a];
  }
  kp.jitter[0] = cam->jitter[0];
  kp.jitter[1] = cam->jitter[1];
  for (int i = 0; i < 16; ++i) kp.prev_vp[i] = cam->prev_vp[i];
  kp.w = w;
  kp.h = h;
  kp.t = out.t;
  kp.normal = out.normal;
  kp.slot = out.slot;
  kp.material = out.material;
  kp.flags = out.flags;
  kp.position = out.position;
  kp.packed = out.packed_material;
  kp.motion = out.motion;
  const dim3 block(8, 8);
  const dim3 grid((w + 7) / 8, (h + 7) / 8);
  const size_t smem = sizeof(ObjDev) * (c->obj_count() ? c->obj_count() : 1);
  detail::k_march_plain<<<grid, block, smem, st>>>(kp);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  return RKF_OK;
}

}  // namespace rkf
