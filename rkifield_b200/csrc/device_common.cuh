// device_common.cuh — device-side scene layout and the exact-arithmetic
// samplers shared by the march kernels.
//
// Arithmetic follows crates/rkf-render/shaders/ray_march.wgsl operation by
// operation: the library is compiled with --fmad=false and IEEE division and
// square root, and every expression below keeps the shader's evaluation order
// (mix(a,b,t) = a*(1-t) + b*t, length = sqrt((x*x + y*y) + z*z), mat4*vec4
// summed column by column).  This makes every kernel bit-identical to the
// FP32 restatement of the shader.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>

#include "../../include/rkf_cuda.h"

namespace rkf {

constexpr float kMaxFloat = 3.402823e+38f;  // ray_march.wgsl:27

// ---------------------------------------------------------------------------
// Layout of a scene in HBM
// ---------------------------------------------------------------------------
// Pool: structure-of-arrays planes, 512 voxels per brick in x+8y+64z order.
//   dist_f16  [cap*512] u16   (RKF_PRECISION_F16)
//   dist_f32  [cap*512] f32   (RKF_PRECISION_F32)
//   dist_u8   [cap*512] s8 + brick_step[cap] f32 (RKF_PRECISION_U8)
//   mat       [cap*512] u16   material | secondary << 6
//   blend     [cap*512] u8
//   aos       [cap*512] uint2 reference VoxelSample (plain march only)
// Index: per object a top grid over 8^3-brick blocks (u32: EMPTY, INTERIOR or
// a leaf number) and leaves of 512 u32 slots in x+8y+64z brick order.

struct ObjDev {
  float m[16];          // inverse_world, column-major
  float vs, be, be2;    // voxel size, brick extent, 2*brick extent
  float gs[3];          // grid size = dims * be
  float half_gs[3];     // gs * 0.5
  float lo;             // vs * 0.01
  float hi[3];          // gs - lo
  float vs16;           // vs * 16 (material lookup threshold)
  float gmin[3], gmax[3];
  float min_scale;
  float params[4];
  int tv[3];            // total voxels per axis = dims*8
  uint32_t bdims[3];    // brick dims
  uint32_t top_off;     // offset of this object's top grid
  uint32_t tdim[3];     // top grid dims (blocks)
  uint32_t map_off;     // reference flat map offset (brick_map_offset)
  uint32_t sdf_type, prim_type, object_id, material_id;
  uint32_t has_geom;
  uint32_t has_flat;    // brick map lives in the reference flat buffer
  float rcp_vs;         // RN(1/vs), for the exact quotient below
  uint32_t div_ok;      // 1: exact_div_vs == IEEE x/vs verified on [lo, max(hi)]
  uint32_t translate_only;  // inverse_world is identity in its linear part
  float vs2;            // vs * 2 (INTERIOR value of the stepping sampler)
};

// x / vs rounded to nearest even, by one Markstein correction step of the
// product with the rounded reciprocal (q0 = x*r, e = x - q0*vs exactly by
// FMA, q = q0 + e*r).  An object uses it only after every float of its
// clamped sampling domain has been checked against the IEEE quotient on the
// device (ObjDev::div_ok); otherwise the IEEE division is used.
__device__ __forceinline__ float exact_div_vs(float x, float vs, float rcp) {
  const float q0 = __fmul_rn(x, rcp);
  const float e = __fmaf_rn(-q0, vs, x);
  return __fmaf_rn(e, rcp, q0);
}

struct SceneDev {
  const uint16_t* __restrict__ dist_f16;
  const float* __restrict__ dist_f32;
  const int8_t* __restrict__ dist_u8;
  const float* __restrict__ brick_step;
  const uint16_t* __restrict__ mat;
  const uint8_t* __restrict__ blend;
  const uint2* __restrict__ aos;
  const uint32_t* __restrict__ top;
  const uint8_t* __restrict__ empty_dist;  // per top cell, see empty_dist.h
  const uint32_t* __restrict__ leaves;
  const uint32_t* __restrict__ flat_maps;
  const ObjDev* __restrict__ objs;
  uint32_t n_objs;
  uint32_t precision;
};

// ---------------------------------------------------------------------------
// Arithmetic helpers with the shader's semantics (non-NaN operands)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fmin_(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float fmax_(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) {
  return fmin_(fmax_(x, lo), hi);
}
__device__ __forceinline__ float mixf(float a, float b, float t) {
  return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}
__device__ __forceinline__ float len3(float x, float y, float z) {
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

__device__ __forceinline__ float f16_load(const uint16_t* p) {
  return __half2float(__ushort_as_half(__ldg(p)));
}

// world -> object-local: r_i = ((m0i*x + m1i*y) + m2i*z) + m3i*1
__device__ __forceinline__ void to_local(const ObjDev& o, float wx, float wy, float wz,
                                         float& lx, float& ly, float& lz) {
  lx = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[0], wx), __fmul_rn(o.m[4], wy)),
                           __fmul_rn(o.m[8], wz)), __fmul_rn(o.m[12], 1.0f));
  ly = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[1], wx), __fmul_rn(o.m[5], wy)),
                           __fmul_rn(o.m[9], wz)), __fmul_rn(o.m[13], 1.0f));
  lz = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[2], wx), __fmul_rn(o.m[6], wy)),
                           __fmul_rn(o.m[10], wz)), __fmul_rn(o.m[14], 1.0f));
}

// analytic primitives (ray_march.wgsl:182-264)
__device__ __forceinline__ float analytic_sdf(const ObjDev& o, float x, float y, float z) {
  const float a0 = o.params[0], a1 = o.params[1], a2 = o.params[2];
  switch (o.prim_type) {
    case RKF_PRIM_SPHERE:
      return __fsub_rn(len3(x, y, z), a0);
    case RKF_PRIM_BOX: {
      const float qx = __fsub_rn(fabsf(x), a0), qy = __fsub_rn(fabsf(y), a1),
                  qz = __fsub_rn(fabsf(z), a2);
      return __fadd_rn(len3(fmax_(qx, 0.f), fmax_(qy, 0.f), fmax_(qz, 0.f)),
                       fmin_(fmax_(qx, fmax_(qy, qz)), 0.f));
    }
    case RKF_PRIM_CAPSULE:
      return __fsub_rn(len3(x, fmax_(__fsub_rn(fabsf(y), a1), 0.f), z), a0);
    case RKF_PRIM_TORUS: {
      const float qx = __fsub_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(z, z))), a0);
      return __fsub_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(qx, qx), __fmul_rn(y, y))), a1);
    }
    case RKF_PRIM_CYLINDER: {
      const float dx = __fsub_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(z, z))), a0);
      const float dy = __fsub_rn(fabsf(y), a1);
      const float mx = fmax_(dx, 0.f), my = fmax_(dy, 0.f);
      return __fadd_rn(fmin_(fmax_(dx, dy), 0.f),
                       __fsqrt_rn(__fadd_rn(__fmul_rn(mx, mx), __fmul_rn(my, my))));
    }
    case RKF_PRIM_PLANE: {
      const float l = len3(a0, a1, a2);
      const float nx = __fdiv_rn(a0, l), ny = __fdiv_rn(a1, l), nz = __fdiv_rn(a2, l);
      return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, nx), __fmul_rn(y, ny)), __fmul_rn(z, nz)),
                       0.f);
    }
    default:
      return kMaxFloat;
  }
}

// ---------------------------------------------------------------------------
// Index lookup
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t top_index(const ObjDev& o, uint32_t bx, uint32_t by,
                                              uint32_t bz) {
  return o.top_off + (bx >> 3) + (by >> 3) * o.tdim[0] + (bz >> 3) * o.tdim[0] * o.tdim[1];
}

__device__ __forceinline__ uint32_t lookup2(const SceneDev& s, const ObjDev& o, uint32_t bx,
                                            uint32_t by, uint32_t bz) {
  const uint32_t t = __ldg(s.top + top_index(o, bx, by, bz));
  if (t >= RKF_INTERIOR_SLOT) return t;
  return __ldg(s.leaves + static_cast<size_t>(t) * 512 + (bx & 7) + (by & 7) * 8 + (bz & 7) * 64);
}

// ---------------------------------------------------------------------------
// Sample of the SoA distance plane at the context precision
// ---------------------------------------------------------------------------
template <int PREC>
__device__ __forceinline__ float pool_dist(const SceneDev& s, uint32_t slot, uint32_t idx) {
  const size_t v = static_cast<size_t>(slot) * 512 + idx;
  if (PREC == RKF_PRECISION_F32) return __ldg(s.dist_f32 + v);
  if (PREC == RKF_PRECISION_U8)
    return __fmul_rn(static_cast<float>(__ldg(s.dist_u8 + v)), __ldg(s.brick_step + slot));
  return f16_load(s.dist_f16 + v);
}

}  // namespace rkf
