// sampler.cuh — sample_voxelized / evaluate_object for the B200 march
// (SoA distance plane, two-level index, per-lane brick cache).
//
// ray_march.wgsl:270-413 (sample_voxel_at, sample_voxel_at_grad,
// sample_voxelized, sample_voxelized_grad), :540-596 (nearest-voxel
// material/blend), :600-634 (evaluate_object).  Results are bit-identical
// to the shader's arithmetic; the only differences are which memory reads
// happen: corners that resolve to the same brick share one index lookup, the
// last brick and top-grid block a lane resolved are reused, and EMPTY /
// INTERIOR corners read nothing.
#pragma once

#include "device_common.cuh"

namespace rkf {

// Per-lane memo of the last resolved brick and top-grid block.
struct LaneCache {
  uint32_t obj = 0xFFFFFFFFu;
  uint32_t bx = 0xFFFFFFFFu, by = 0, bz = 0;
  uint32_t slot = 0;
  uint32_t blk = 0xFFFFFFFFu;
  uint32_t topv = 0;
};

__device__ __forceinline__ uint32_t lookup_cached(const SceneDev& s, const ObjDev& o, uint32_t oi,
                                                  uint32_t bx, uint32_t by, uint32_t bz,
                                                  LaneCache& lc) {
  if (bx == lc.bx && by == lc.by && bz == lc.bz && oi == lc.obj) return lc.slot;
  const uint32_t blk = top_index(o, bx, by, bz);
  uint32_t tv;
  if (blk == lc.blk) {
    tv = lc.topv;
  } else {
    tv = __ldg(s.top + blk);
    lc.blk = blk;
    lc.topv = tv;
  }
  uint32_t slot = tv;
  if (tv < RKF_INTERIOR_SLOT)
    slot = __ldg(s.leaves + static_cast<size_t>(tv) * 512 + (bx & 7) + (by & 7) * 8 + (bz & 7) * 64);
  lc.obj = oi;
  lc.bx = bx;
  lc.by = by;
  lc.bz = bz;
  lc.slot = slot;
  return slot;
}

template <int PREC>
__device__ __forceinline__ float corner(const SceneDev& s, const ObjDev& o, uint32_t slot,
                                        uint32_t idx, bool grad) {
  if (slot == RKF_EMPTY_SLOT) return o.be;                         // vs * 8
  if (slot == RKF_INTERIOR_SLOT) return grad ? -o.be : -(o.vs * 2.0f);  // -(vs*8) / -(vs*2)
  return pool_dist<PREC>(s, slot, idx);
}

// sample_voxelized (grad=false) / sample_voxelized_grad (grad=true)
template <int PREC>
__device__ __forceinline__ float sample_vox(const SceneDev& s, const ObjDev& o, uint32_t oi,
                                            float lx, float ly, float lz, bool grad,
                                            LaneCache& lc) {
  const float gpx = __fadd_rn(lx, o.half_gs[0]);
  const float gpy = __fadd_rn(ly, o.half_gs[1]);
  const float gpz = __fadd_rn(lz, o.half_gs[2]);
  const float clx = clampf(gpx, o.lo, o.hi[0]);
  const float cly = clampf(gpy, o.lo, o.hi[1]);
  const float clz = clampf(gpz, o.lo, o.hi[2]);
  const float ox = __fsub_rn(gpx, clx), oy = __fsub_rn(gpy, cly), oz = __fsub_rn(gpz, clz);
  // sqrt((0*0+0*0)+0*0) == 0 exactly, so the square root is only taken when needed
  const float outside = (ox == 0.0f && oy == 0.0f && oz == 0.0f) ? 0.0f : len3(ox, oy, oz);
  if (outside > o.be2) return outside;
  if (!grad && o.has_geom) {
    const float gdx = __fsub_rn(lx, clampf(lx, o.gmin[0], o.gmax[0]));
    const float gdy = __fsub_rn(ly, clampf(ly, o.gmin[1], o.gmax[1]));
    const float gdz = __fsub_rn(lz, clampf(lz, o.gmin[2], o.gmax[2]));
    if (!(gdx == 0.0f && gdy == 0.0f && gdz == 0.0f)) {
      const float gd = len3(gdx, gdy, gdz);
      if (gd > o.be) return gd;
    }
  }
  const float vcx = __fsub_rn(__fdiv_rn(clx, o.vs), 0.5f);
  const float vcy = __fsub_rn(__fdiv_rn(cly, o.vs), 0.5f);
  const float vcz = __fsub_rn(__fdiv_rn(clz, o.vs), 0.5f);
  const float fx = floorf(vcx), fy = floorf(vcy), fz = floorf(vcz);
  const float tx = __fsub_rn(vcx, fx), ty = __fsub_rn(vcy, fy), tz = __fsub_rn(vcz, fz);
  const int x0 = static_cast<int>(fx), y0 = static_cast<int>(fy), z0 = static_cast<int>(fz);
  const int cx0 = clampi(x0, 0, o.tv[0] - 1), cx1 = clampi(x0 + 1, 0, o.tv[0] - 1);
  const int cy0 = clampi(y0, 0, o.tv[1] - 1), cy1 = clampi(y0 + 1, 0, o.tv[1] - 1);
  const int cz0 = clampi(z0, 0, o.tv[2] - 1), cz1 = clampi(z0 + 1, 0, o.tv[2] - 1);
  const uint32_t bx0 = cx0 >> 3, bx1 = cx1 >> 3, by0 = cy0 >> 3, by1 = cy1 >> 3;
  const uint32_t bz0 = cz0 >> 3, bz1 = cz1 >> 3;
  const uint32_t ix0 = cx0 & 7, ix1 = cx1 & 7, iy0 = (cy0 & 7) * 8, iy1 = (cy1 & 7) * 8;
  const uint32_t iz0 = (cz0 & 7) * 64, iz1 = (cz1 & 7) * 64;
  const bool sx = bx0 == bx1, sy = by0 == by1, sz = bz0 == bz1;
  // distinct bricks of the 8 corners, each resolved once
  const uint32_t s000 = lookup_cached(s, o, oi, bx0, by0, bz0, lc);
  const uint32_t s100 = sx ? s000 : lookup_cached(s, o, oi, bx1, by0, bz0, lc);
  const uint32_t s010 = sy ? s000 : lookup_cached(s, o, oi, bx0, by1, bz0, lc);
  const uint32_t s110 = sy ? s100 : (sx ? s010 : lookup_cached(s, o, oi, bx1, by1, bz0, lc));
  uint32_t s001 = s000, s101 = s100, s011 = s010, s111 = s110;
  if (!sz) {
    s001 = lookup_cached(s, o, oi, bx0, by0, bz1, lc);
    s101 = sx ? s001 : lookup_cached(s, o, oi, bx1, by0, bz1, lc);
    s011 = sy ? s001 : lookup_cached(s, o, oi, bx0, by1, bz1, lc);
    s111 = sy ? s101 : (sx ? s011 : lookup_cached(s, o, oi, bx1, by1, bz1, lc));
  }
  const float c000 = corner<PREC>(s, o, s000, ix0 + iy0 + iz0, grad);
  const float c100 = corner<PREC>(s, o, s100, ix1 + iy0 + iz0, grad);
  const float c010 = corner<PREC>(s, o, s010, ix0 + iy1 + iz0, grad);
  const float c110 = corner<PREC>(s, o, s110, ix1 + iy1 + iz0, grad);
  const float c001 = corner<PREC>(s, o, s001, ix0 + iy0 + iz1, grad);
  const float c101 = corner<PREC>(s, o, s101, ix1 + iy0 + iz1, grad);
  const float c011 = corner<PREC>(s, o, s011, ix0 + iy1 + iz1, grad);
  const float c111 = corner<PREC>(s, o, s111, ix1 + iy1 + iz1, grad);
  const float c00 = mixf(c000, c100, tx);
  const float c10 = mixf(c010, c110, tx);
  const float c01 = mixf(c001, c101, tx);
  const float c11 = mixf(c011, c111, tx);
  const float c0 = mixf(c00, c10, ty);
  const float c1 = mixf(c01, c11, ty);
  return __fadd_rn(mixf(c0, c1, tz), outside);
}

// Nearest-voxel slot lookup of sample_voxelized_material / _blend_data.
__device__ __forceinline__ uint32_t nearest_slot(const SceneDev& s, const ObjDev& o, uint32_t oi,
                                                 float lx, float ly, float lz, uint32_t& idx,
                                                 LaneCache& lc) {
  const float gpx = __fadd_rn(lx, o.half_gs[0]);
  const float gpy = __fadd_rn(ly, o.half_gs[1]);
  const float gpz = __fadd_rn(lz, o.half_gs[2]);
  if (gpx < 0.0f || gpy < 0.0f || gpz < 0.0f || gpx >= o.gs[0] || gpy >= o.gs[1] || gpz >= o.gs[2])
    return RKF_EMPTY_SLOT;
  const int x = clampi(static_cast<int>(floorf(__fdiv_rn(gpx, o.vs))), 0, o.tv[0] - 1);
  const int y = clampi(static_cast<int>(floorf(__fdiv_rn(gpy, o.vs))), 0, o.tv[1] - 1);
  const int z = clampi(static_cast<int>(floorf(__fdiv_rn(gpz, o.vs))), 0, o.tv[2] - 1);
  idx = (x & 7) + (y & 7) * 8 + (z & 7) * 64;
  return lookup_cached(s, o, oi, x >> 3, y >> 3, z >> 3, lc);
}

// evaluate_object without the material read.  Returns the scaled distance;
// *unscaled receives the sampler's value (the material-lookup test of
// ray_march.wgsl:621 compares it with vs*16).
template <int PREC>
__device__ __forceinline__ float eval_obj(const SceneDev& s, const ObjDev& o, uint32_t oi, float wx,
                                          float wy, float wz, float* unscaled, LaneCache& lc) {
  if (o.sdf_type == RKF_SDF_NONE) {
    *unscaled = kMaxFloat;
    return kMaxFloat;
  }
  float lx, ly, lz;
  to_local(o, wx, wy, wz, lx, ly, lz);
  const float d = o.sdf_type == RKF_SDF_ANALYTICAL ? analytic_sdf(o, lx, ly, lz)
                                                   : sample_vox<PREC>(s, o, oi, lx, ly, lz, false, lc);
  *unscaled = d;
  return __fmul_rn(d, o.min_scale);
}

// Material evaluate_object would report at world position w for object oi
// (ray_march.wgsl:613-626).
__device__ __forceinline__ uint32_t material_at(const SceneDev& s, const ObjDev& o, uint32_t oi,
                                                float wx, float wy, float wz, LaneCache& lc) {
  if (o.sdf_type == RKF_SDF_ANALYTICAL) return o.material_id;
  if (o.sdf_type != RKF_SDF_VOXELIZED) return 0u;
  float lx, ly, lz;
  to_local(o, wx, wy, wz, lx, ly, lz);
  uint32_t idx = 0;
  const uint32_t slot = nearest_slot(s, o, oi, lx, ly, lz, idx, lc);
  if (slot >= RKF_INTERIOR_SLOT) return 0u;
  return __ldg(s.mat + static_cast<size_t>(slot) * 512 + idx) & 0x3Fu;
}

}  // namespace rkf
