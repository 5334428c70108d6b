// sampler.cuh — sample_voxelized / evaluate_object for the B200 march
// (SoA distance plane, two-level index, per-lane block/brick memo).
//
// ray_march.wgsl:270-413 (sample_voxel_at, sample_voxel_at_grad,
// sample_voxelized, sample_voxelized_grad), :540-596 (nearest-voxel
// material/blend), :600-634 (evaluate_object).  Every value returned is
// bit-identical to the shader's arithmetic.  What differs is the work done to
// get it:
//   * a trilinear cell whose 8 corners resolve to one sentinel (an EMPTY or
//     INTERIOR 8^3-brick block, or one sentinel brick) reads nothing and mixes
//     the constant with 3 lerps: mix(c,c,t) repeated gives the same bits as
//     the 7 lerps of 8 equal corners;
//   * corners in one allocated brick are read from one base address;
//   * the last block and brick a lane resolved are memoised;
//   * x / vs uses the verified exact quotient when the object allows it;
//   * sqrt is skipped when its argument is exactly 0 (sqrt(+0) = +0).
#pragma once

#include "device_common.cuh"

namespace rkf {

// Per-lane memo of the last resolved top-grid block and brick.
struct LaneCache {
  uint32_t blk = 0xFFFFFFFFu;
  uint32_t topv = 0;
  uint32_t brick = 0xFFFFFFFFu;  // packed (leaf number, brick within leaf)
  uint32_t slot = 0;
};

__device__ __forceinline__ float mix3_const(float c, float tx, float ty, float tz) {
  const float c00 = mixf(c, c, tx);
  const float c0 = mixf(c00, c00, ty);
  return mixf(c0, c0, tz);
}

template <int PREC>
__device__ __forceinline__ float corner(const SceneDev& s, const ObjDev& o, uint32_t slot,
                                        uint32_t idx, bool grad) {
  if (slot == RKF_EMPTY_SLOT) return o.be;                      // vs * 8
  if (slot == RKF_INTERIOR_SLOT) return grad ? -o.be : -o.vs2;  // -(vs*8) / -(vs*2)
  return pool_dist<PREC>(s, slot, idx);
}

__device__ __forceinline__ uint32_t resolve_top(const SceneDev& s, uint32_t blk, LaneCache& lc) {
  if (blk != lc.blk) {
    lc.blk = blk;
    lc.topv = __ldg(s.top + blk);
  }
  return lc.topv;
}

// slot of brick (bx,by,bz) (or a sentinel) through the memo
__device__ __forceinline__ uint32_t lookup_cached(const SceneDev& s, const ObjDev& o, uint32_t bx,
                                                  uint32_t by, uint32_t bz, LaneCache& lc) {
  const uint32_t tv = resolve_top(s, top_index(o, bx, by, bz), lc);
  if (tv >= RKF_INTERIOR_SLOT) return tv;
  const uint32_t key = (tv << 9) | ((bx & 7) + (by & 7) * 8 + (bz & 7) * 64);
  if (key != lc.brick) {
    lc.brick = key;
    lc.slot = __ldg(s.leaves + static_cast<size_t>(tv) * 512 + (key & 511u));
  }
  return lc.slot;
}

// sample_voxelized (grad=false) / sample_voxelized_grad (grad=true) at an
// object-local position.
template <int PREC>
__device__ __forceinline__ float sample_vox(const SceneDev& s, const ObjDev& o, float lx, float ly,
                                            float lz, bool grad, LaneCache& lc) {
  const float gpx = __fadd_rn(lx, o.half_gs[0]);
  const float gpy = __fadd_rn(ly, o.half_gs[1]);
  const float gpz = __fadd_rn(lz, o.half_gs[2]);
  // lo > 0, so IEEE min/max give the shader's clamp bit for bit
  const float clx = fminf(fmaxf(gpx, o.lo), o.hi[0]);
  const float cly = fminf(fmaxf(gpy, o.lo), o.hi[1]);
  const float clz = fminf(fmaxf(gpz, o.lo), o.hi[2]);
  const float ox = __fsub_rn(gpx, clx), oy = __fsub_rn(gpy, cly), oz = __fsub_rn(gpz, clz);
  float outside = 0.0f;
  if (ox != 0.0f || oy != 0.0f || oz != 0.0f) {
    outside = len3(ox, oy, oz);
    if (outside > o.be2) return outside;
  }
  if (!grad && o.has_geom) {
    // only the squares of these differences reach the result, so the sign of
    // a zero difference (the one place IEEE min/max and the shader's select
    // form can differ) is irrelevant
    const float gdx = __fsub_rn(lx, fminf(fmaxf(lx, o.gmin[0]), o.gmax[0]));
    const float gdy = __fsub_rn(ly, fminf(fmaxf(ly, o.gmin[1]), o.gmax[1]));
    const float gdz = __fsub_rn(lz, fminf(fmaxf(lz, o.gmin[2]), o.gmax[2]));
    if (gdx != 0.0f || gdy != 0.0f || gdz != 0.0f) {
      const float gd = len3(gdx, gdy, gdz);
      if (gd > o.be) return gd;
    }
  }
  float qx, qy, qz;
  if (o.div_ok) {
    qx = exact_div_vs(clx, o.vs, o.rcp_vs);
    qy = exact_div_vs(cly, o.vs, o.rcp_vs);
    qz = exact_div_vs(clz, o.vs, o.rcp_vs);
  } else {
    qx = __fdiv_rn(clx, o.vs);
    qy = __fdiv_rn(cly, o.vs);
    qz = __fdiv_rn(clz, o.vs);
  }
  const float vcx = __fsub_rn(qx, 0.5f), vcy = __fsub_rn(qy, 0.5f), vcz = __fsub_rn(qz, 0.5f);
  const float fx = floorf(vcx), fy = floorf(vcy), fz = floorf(vcz);
  const float tx = __fsub_rn(vcx, fx), ty = __fsub_rn(vcy, fy), tz = __fsub_rn(vcz, fz);
  const int x0 = static_cast<int>(fx), y0 = static_cast<int>(fy), z0 = static_cast<int>(fz);
  // cl lies in [vs*0.01, grid - vs*0.01] (never NaN: the clamp maps NaN to a
  // bound), so the lower corner x0 is in [-1, tv-1]: clamping x0 from below
  // and x0+1 from above is the shader's two-sided clamp of both
  const int cx0 = max(x0, 0), cx1 = min(x0 + 1, o.tv[0] - 1);
  const int cy0 = max(y0, 0), cy1 = min(y0 + 1, o.tv[1] - 1);
  const int cz0 = max(z0, 0), cz1 = min(z0 + 1, o.tv[2] - 1);
  // ---- blocks (8^3 bricks = 64 voxels per axis) holding the corners --------
  const uint32_t kx0 = cx0 >> 6, ky0 = cy0 >> 6, kz0 = cz0 >> 6;
  const uint32_t txy = o.tdim[0] * o.tdim[1];
  const uint32_t b000 = o.top_off + kx0 + ky0 * o.tdim[0] + kz0 * txy;
  const uint32_t tv = resolve_top(s, b000, lc);
  const uint32_t kdx = (cx1 >> 6) - kx0, kdy = ((cy1 >> 6) - ky0) * o.tdim[0],
                 kdz = ((cz1 >> 6) - kz0) * txy;
  if ((kdx | kdy | kdz) != 0u) {
    // the cell straddles blocks: it is still one constant when every block
    // it touches holds the same sentinel
    if (tv >= RKF_INTERIOR_SLOT) {
      const uint32_t* tp = s.top + b000;
      const bool same = __ldg(tp + kdx) == tv && __ldg(tp + kdy) == tv && __ldg(tp + kdx + kdy) == tv &&
                        __ldg(tp + kdz) == tv && __ldg(tp + kdx + kdz) == tv && __ldg(tp + kdy + kdz) == tv &&
                        __ldg(tp + kdx + kdy + kdz) == tv;
      if (same) {
        const float c = tv == RKF_EMPTY_SLOT ? o.be : (grad ? -o.be : -o.vs2);
        return __fadd_rn(mix3_const(c, tx, ty, tz), outside);
      }
    }
  } else {
    // ---- all corners in one block -------------------------------------------
    if (tv >= RKF_INTERIOR_SLOT) {
      const float c = tv == RKF_EMPTY_SLOT ? o.be : (grad ? -o.be : -o.vs2);
      return __fadd_rn(mix3_const(c, tx, ty, tz), outside);
    }
    if ((cx0 >> 3) == (cx1 >> 3) && (cy0 >> 3) == (cy1 >> 3) && (cz0 >> 3) == (cz1 >> 3)) {
      // ---- all corners in one brick ----------------------------------------
      const uint32_t key = (tv << 9) | (((cx0 >> 3) & 7) + ((cy0 >> 3) & 7) * 8 + ((cz0 >> 3) & 7) * 64);
      if (key != lc.brick) {
        lc.brick = key;
        lc.slot = __ldg(s.leaves + static_cast<size_t>(tv) * 512 + (key & 511u));
      }
      const uint32_t slot = lc.slot;
      if (slot >= RKF_INTERIOR_SLOT) {
        const float c = slot == RKF_EMPTY_SLOT ? o.be : (grad ? -o.be : -o.vs2);
        return __fadd_rn(mix3_const(c, tx, ty, tz), outside);
      }
      const uint32_t i0 = (cx0 & 7) + (cy0 & 7) * 8 + (cz0 & 7) * 64;
      const uint32_t dx = (cx1 & 7) - (cx0 & 7), dy = ((cy1 & 7) - (cy0 & 7)) * 8,
                     dz = ((cz1 & 7) - (cz0 & 7)) * 64;
      const float c000 = pool_dist<PREC>(s, slot, i0);
      const float c100 = pool_dist<PREC>(s, slot, i0 + dx);
      const float c010 = pool_dist<PREC>(s, slot, i0 + dy);
      const float c110 = pool_dist<PREC>(s, slot, i0 + dx + dy);
      const float c001 = pool_dist<PREC>(s, slot, i0 + dz);
      const float c101 = pool_dist<PREC>(s, slot, i0 + dx + dz);
      const float c011 = pool_dist<PREC>(s, slot, i0 + dy + dz);
      const float c111 = pool_dist<PREC>(s, slot, i0 + dx + dy + dz);
      const float c00 = mixf(c000, c100, tx), c10 = mixf(c010, c110, tx);
      const float c01 = mixf(c001, c101, tx), c11 = mixf(c011, c111, tx);
      const float c0 = mixf(c00, c10, ty), c1 = mixf(c01, c11, ty);
      return __fadd_rn(mixf(c0, c1, tz), outside);
    } else {
      // ---- one leaf block, corners across bricks: constant when every brick
      // they touch holds the same sentinel
      const uint32_t lb = ((cx0 >> 3) & 7) + ((cy0 >> 3) & 7) * 8 + ((cz0 >> 3) & 7) * 64;
      const uint32_t ldx = (cx1 >> 3) - (cx0 >> 3), ldy = ((cy1 >> 3) - (cy0 >> 3)) * 8,
                     ldz = ((cz1 >> 3) - (cz0 >> 3)) * 64;
      const uint32_t* lp = s.leaves + static_cast<size_t>(tv) * 512 + lb;
      const uint32_t s0 = __ldg(lp);
      if (s0 >= RKF_INTERIOR_SLOT && __ldg(lp + ldx) == s0 && __ldg(lp + ldy) == s0 &&
          __ldg(lp + ldx + ldy) == s0 && __ldg(lp + ldz) == s0 && __ldg(lp + ldx + ldz) == s0 &&
          __ldg(lp + ldy + ldz) == s0 && __ldg(lp + ldx + ldy + ldz) == s0) {
        const float c = s0 == RKF_EMPTY_SLOT ? o.be : (grad ? -o.be : -o.vs2);
        return __fadd_rn(mix3_const(c, tx, ty, tz), outside);
      }
    }
  }
  // ---- general: corners across bricks, each distinct brick resolved once --
  const uint32_t bx0 = cx0 >> 3, bx1 = cx1 >> 3, by0 = cy0 >> 3, by1 = cy1 >> 3;
  const uint32_t bz0 = cz0 >> 3, bz1 = cz1 >> 3;
  const uint32_t ix0 = cx0 & 7, ix1 = cx1 & 7, iy0 = (cy0 & 7) * 8, iy1 = (cy1 & 7) * 8;
  const uint32_t iz0 = (cz0 & 7) * 64, iz1 = (cz1 & 7) * 64;
  const bool sx = bx0 == bx1, sy = by0 == by1, sz = bz0 == bz1;
  const uint32_t s000 = lookup_cached(s, o, bx0, by0, bz0, lc);
  const uint32_t s100 = sx ? s000 : lookup_cached(s, o, bx1, by0, bz0, lc);
  const uint32_t s010 = sy ? s000 : lookup_cached(s, o, bx0, by1, bz0, lc);
  const uint32_t s110 = sy ? s100 : (sx ? s010 : lookup_cached(s, o, bx1, by1, bz0, lc));
  uint32_t s001 = s000, s101 = s100, s011 = s010, s111 = s110;
  if (!sz) {
    s001 = lookup_cached(s, o, bx0, by0, bz1, lc);
    s101 = sx ? s001 : lookup_cached(s, o, bx1, by0, bz1, lc);
    s011 = sy ? s001 : lookup_cached(s, o, bx0, by1, bz1, lc);
    s111 = sy ? s101 : (sx ? s011 : lookup_cached(s, o, bx1, by1, bz1, lc));
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
__device__ __forceinline__ uint32_t nearest_slot(const SceneDev& s, const ObjDev& o, float lx,
                                                 float ly, float lz, uint32_t& idx, LaneCache& lc) {
  const float gpx = __fadd_rn(lx, o.half_gs[0]);
  const float gpy = __fadd_rn(ly, o.half_gs[1]);
  const float gpz = __fadd_rn(lz, o.half_gs[2]);
  if (gpx < 0.0f || gpy < 0.0f || gpz < 0.0f || gpx >= o.gs[0] || gpy >= o.gs[1] || gpz >= o.gs[2])
    return RKF_EMPTY_SLOT;
  const int x = clampi(static_cast<int>(floorf(__fdiv_rn(gpx, o.vs))), 0, o.tv[0] - 1);
  const int y = clampi(static_cast<int>(floorf(__fdiv_rn(gpy, o.vs))), 0, o.tv[1] - 1);
  const int z = clampi(static_cast<int>(floorf(__fdiv_rn(gpz, o.vs))), 0, o.tv[2] - 1);
  idx = (x & 7) + (y & 7) * 8 + (z & 7) * 64;
  return lookup_cached(s, o, x >> 3, y >> 3, z >> 3, lc);
}

// world -> local for a translation-only inverse_world.  ((1*x + 0*y) + 0*z)
// equals x up to the sign of a zero, and every consumer of the local
// coordinate adds a nonzero offset to it or compares it, so x + m12 gives the
// same downstream bits as the full product.
__device__ __forceinline__ void to_local_fast(const ObjDev& o, float wx, float wy, float wz,
                                              float& lx, float& ly, float& lz) {
  if (o.translate_only) {
    lx = __fadd_rn(wx, o.m[12]);
    ly = __fadd_rn(wy, o.m[13]);
    lz = __fadd_rn(wz, o.m[14]);
  } else {
    to_local(o, wx, wy, wz, lx, ly, lz);
  }
}

// evaluate_object without the material read.  Returns the scaled distance;
// *unscaled receives the sampler's value (the material-lookup test of
// ray_march.wgsl:621 compares it with vs*16).
template <int PREC>
__device__ __forceinline__ float eval_obj(const SceneDev& s, const ObjDev& o, float wx, float wy,
                                          float wz, float* unscaled, LaneCache& lc) {
  if (o.sdf_type == RKF_SDF_NONE) {
    *unscaled = kMaxFloat;
    return kMaxFloat;
  }
  float lx, ly, lz;
  to_local_fast(o, wx, wy, wz, lx, ly, lz);
  const float d = o.sdf_type == RKF_SDF_ANALYTICAL ? analytic_sdf(o, lx, ly, lz)
                                                   : sample_vox<PREC>(s, o, lx, ly, lz, false, lc);
  *unscaled = d;
  return __fmul_rn(d, o.min_scale);
}

// Material evaluate_object would report at world position w for object o
// (ray_march.wgsl:613-626).
__device__ __forceinline__ uint32_t material_at(const SceneDev& s, const ObjDev& o, float wx,
                                                float wy, float wz, LaneCache& lc) {
  if (o.sdf_type == RKF_SDF_ANALYTICAL) return o.material_id;
  if (o.sdf_type != RKF_SDF_VOXELIZED) return 0u;
  float lx, ly, lz;
  to_local_fast(o, wx, wy, wz, lx, ly, lz);
  uint32_t idx = 0;
  const uint32_t slot = nearest_slot(s, o, lx, ly, lz, idx, lc);
  if (slot >= RKF_INTERIOR_SLOT) return 0u;
  return __ldg(s.mat + static_cast<size_t>(slot) * 512 + idx) & 0x3Fu;
}

}  // namespace rkf
