// edit.cu — CSG brush edits on the device with copy-on-write bricks.
//
// Per-voxel arithmetic: apply_edit_cpu (crates/rkf-edit/src/cpu_apply.rs:
// 28-200) for CsgUnion / CsgSubtract / CsgIntersect / SmoothUnion /
// SmoothSubtract with the sphere, box and capsule brushes
// (evaluate_shape :231-262) and the falloff curves (evaluate_falloff
// :265-283).  Brick selection follows find_affected_bricks
// (crates/rkf-edit/src/edit_op.rs:97-140) over the brush's local AABB, and
// extends it the way an editor has to for a narrow-band pool: an EMPTY brick
// the brush can reach is materialised (every voxel at the EMPTY sampling
// value vs*8) for additive edits, an INTERIOR brick (vs*2 below zero, the
// stepping value) for subtractive ones.
//
// Copy-on-write: every touched brick is written to a fresh pool slot and a
// new epoch of the two-level index (a copy of the top grid plus new leaves
// for the touched blocks) points at the new slots.  Work launched on the old
// epoch keeps reading the old slots and leaves, which return to their free
// lists once no work holds that epoch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "edit.h"
#include "empty_dist.h"

namespace rkf {
namespace detail {

__device__ __forceinline__ float edit_shape(uint32_t shape, const float* dims, float x, float y, float z) {
  if (shape == 0) return __fsub_rn(len3(x, y, z), dims[0]);
  if (shape == 1) {
    const float qx = __fsub_rn(fabsf(x), dims[0]), qy = __fsub_rn(fabsf(y), dims[1]),
                qz = __fsub_rn(fabsf(z), dims[2]);
    return __fadd_rn(len3(fmax_(qx, 0.f), fmax_(qy, 0.f), fmax_(qz, 0.f)), fmin_(fmax_(qx, fmax_(qy, qz)), 0.f));
  }
  // capsule a=(0,-h,0), b=(0,h,0)
  const float h = dims[1];
  const float pax = __fsub_rn(x, 0.0f), pay = __fsub_rn(y, -h), paz = __fsub_rn(z, 0.0f);
  const float bax = 0.0f, bay = __fsub_rn(h, -h), baz = 0.0f;
  const float dpb = __fadd_rn(__fadd_rn(__fmul_rn(pax, bax), __fmul_rn(pay, bay)), __fmul_rn(paz, baz));
  const float dbb = __fadd_rn(__fadd_rn(__fmul_rn(bax, bax), __fmul_rn(bay, bay)), __fmul_rn(baz, baz));
  const float hh = clampf(__fdiv_rn(dpb, dbb), 0.0f, 1.0f);
  return __fsub_rn(len3(__fsub_rn(pax, __fmul_rn(bax, hh)), __fsub_rn(pay, __fmul_rn(bay, hh)),
                        __fsub_rn(paz, __fmul_rn(baz, hh))),
                   dims[0]);
}

__device__ __forceinline__ float edit_falloff(uint32_t curve, float d, float r) {
  if (r <= 0.0f || d >= r) return 0.0f;
  const float t = __fdiv_rn(d, r);
  if (curve == 0) return __fsub_rn(1.0f, t);
  if (curve == 1) return __fsub_rn(1.0f, __fmul_rn(__fmul_rn(t, t), __fsub_rn(3.0f, __fmul_rn(2.0f, t))));
  const float f = __fsub_rn(1.0f, t);
  return __fmul_rn(__fmul_rn(f, f), f);
}

__device__ __forceinline__ float smin_e(float a, float b, float k) {
  const float h = __fdiv_rn(fmax_(__fsub_rn(k, fabsf(__fsub_rn(a, b))), 0.0f), k);
  return __fsub_rn(fmin_(a, b), __fmul_rn(__fmul_rn(__fmul_rn(h, h), k), 0.25f));
}

struct EditKernelArgs {
  rkf_edit_op op;
  float iq[4];        // inverse rotation (conjugate)
  float max_extent;   // max(dimensions)
  float vs;
  const uint32_t* src;        // per candidate: source slot or sentinel
  const uint32_t* dst;        // per candidate: destination slot
  const float* bmin;          // per candidate: brick_local_min (3 floats)
  uint16_t* dist_f16;
  uint16_t* mat;
  uint8_t* blend;
  uint2* aos;
  uint8_t* changed;
  // the f32 and u8 pools: the brush blends with the decoded distance; an
  // edited u8 brick is encoded again (band-normalised, per-brick step)
  float* dist_f32;
  int8_t* dist_u8;
  float* brick_step;
  uint32_t precision;
  float u8_band;
  uint32_t u8_nearest;
};

// One 512-thread block per candidate brick.
__global__ void __launch_bounds__(512) k_edit(EditKernelArgs a) {
  const uint32_t c = blockIdx.x;
  const uint32_t v = threadIdx.x;
  const uint32_t vx = v & 7, vy = (v >> 3) & 7, vz = v >> 6;
  const uint32_t src = a.src[c], dst = a.dst[c];
  const float vs = a.vs;
  // existing voxel (a sentinel brick is materialised at its sampling value,
  // at the pool's precision)
  const bool f16 = a.precision == RKF_PRECISION_F16;
  uint32_t w0, w1;
  float existing_plane = 0.0f;  // f32 / u8 pools: the decoded distance
  if (src == RKF_EMPTY_SLOT || src == RKF_INTERIOR_SLOT) {
    const float d = src == RKF_EMPTY_SLOT ? __fmul_rn(vs, 8.0f) : -__fmul_rn(vs, 2.0f);
    w0 = __half_as_ushort(__float2half_rn(d));
    w1 = 0;
    existing_plane = d;
  } else {
    const size_t i = static_cast<size_t>(src) * 512 + v;
    const uint16_t m = a.mat[i];
    const uint32_t dbits = f16 ? static_cast<uint32_t>(a.dist_f16[i]) : 0u;
    w0 = dbits | ((m & 0x3Fu) << 16) | (((m >> 6) & 0x3Fu) << 22);
    w1 = static_cast<uint32_t>(a.blend[i]) << 24;
    if (a.precision == RKF_PRECISION_F32) existing_plane = a.dist_f32[i];
    if (a.precision == RKF_PRECISION_U8)
      existing_plane = __fmul_rn(static_cast<float>(a.dist_u8[i]), a.brick_step[src]);
  }
  const rkf_edit_op& op = a.op;
  // voxel_pos = brick_min + (v * vs) + splat(vs*0.5)  (cpu_apply.rs:52-55)
  const float hv = __fmul_rn(vs, 0.5f);
  const float px = __fadd_rn(__fadd_rn(a.bmin[3 * c], __fmul_rn(static_cast<float>(vx), vs)), hv);
  const float py = __fadd_rn(__fadd_rn(a.bmin[3 * c + 1], __fmul_rn(static_cast<float>(vy), vs)), hv);
  const float pz = __fadd_rn(__fadd_rn(a.bmin[3 * c + 2], __fmul_rn(static_cast<float>(vz), vs)), hv);
  const float rx = __fsub_rn(px, op.position[0]), ry = __fsub_rn(py, op.position[1]),
              rz = __fsub_rn(pz, op.position[2]);
  // inverse rotation: v*(w*w - b.b) + b*(2 b.v) + (b x v)*(2w)
  const float bx = a.iq[0], by = a.iq[1], bz = a.iq[2], w = a.iq[3];
  const float b2 = __fadd_rn(__fadd_rn(__fmul_rn(bx, bx), __fmul_rn(by, by)), __fmul_rn(bz, bz));
  const float s0 = __fsub_rn(__fmul_rn(w, w), b2);
  const float bv2 = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(rx, bx), __fmul_rn(ry, by)), __fmul_rn(rz, bz)), 2.0f);
  const float w2 = __fmul_rn(w, 2.0f);
  const float cx = __fsub_rn(__fmul_rn(by, rz), __fmul_rn(bz, ry));
  const float cy = __fsub_rn(__fmul_rn(bz, rx), __fmul_rn(bx, rz));
  const float cz = __fsub_rn(__fmul_rn(bx, ry), __fmul_rn(by, rx));
  const float ex = __fadd_rn(__fadd_rn(__fmul_rn(rx, s0), __fmul_rn(bx, bv2)), __fmul_rn(cx, w2));
  const float ey = __fadd_rn(__fadd_rn(__fmul_rn(ry, s0), __fmul_rn(by, bv2)), __fmul_rn(cy, w2));
  const float ez = __fadd_rn(__fadd_rn(__fmul_rn(rz, s0), __fmul_rn(bz, bv2)), __fmul_rn(cz, w2));
  const float shape_d = edit_shape(op.shape_type, op.dimensions, ex, ey, ez);
  const float dc = len3(rx, ry, rz);
  const float fw = edit_falloff(op.falloff, dc, __fadd_rn(a.max_extent, op.blend_k));
  int changed = 0;
  float out_d = f16 ? 0.0f : existing_plane;  // f32 / u8 pools: the voxel's new distance
  if (fw > 0.0f) {
    const float existing = f16 ? __half2float(__ushort_as_half(static_cast<uint16_t>(w0 & 0xFFFFu))) : existing_plane;
    const uint32_t smat = (w0 >> 16) & 0x3Fu, ssec = (w0 >> 22) & 0x3Fu, sbl = w1 >> 24;
    const float strength = __fmul_rn(op.strength, fw);
    const float thr = __fmul_rn(vs, 0.1f);
    const float shift = __fmul_rn(__fsub_rn(1.0f, strength), a.max_extent);
    float nd = existing;
    uint32_t mat = smat;
    switch (op.edit_type) {
      case 0: {
        const float e = __fadd_rn(shape_d, shift);
        nd = fmin_(existing, e);
        mat = e < existing ? op.material_id : ((nd < 0.0f && smat == 0) ? op.material_id : smat);
        break;
      }
      case 1:
        nd = fmax_(existing, -__fadd_rn(shape_d, shift));
        break;
      case 2:
        nd = fmax_(existing, __fsub_rn(shape_d, shift));
        break;
      case 3: {
        const float k = fmax_(op.blend_k, 0.001f);
        const float e = __fadd_rn(shape_d, shift);
        nd = smin_e(existing, e, k);
        mat = e < existing ? op.material_id : ((nd < 0.0f && smat == 0) ? op.material_id : smat);
        break;
      }
      case 4: {
        const float k = fmax_(op.blend_k, 0.001f);
        nd = -smin_e(-existing, __fadd_rn(shape_d, shift), k);
        break;
      }
      case 5:  // Smooth (cpu_apply.rs:151-157): d * (1 - 0.3 strength)
        nd = __fmul_rn(existing, __fsub_rn(1.0f, __fmul_rn(strength, 0.3f)));
        break;
      case 6:  // Flatten (:158-165): lerp toward the brush's local plane y = 0
        nd = __fadd_rn(existing, __fmul_rn(__fsub_rn(ey, existing), __fmul_rn(strength, 0.5f)));
        break;
      default:
        break;
    }
    // Paint (:166-173): near-surface voxels take the brush material as
    // VoxelSample::new(d, material, 0) -- secondary and blend cleared
    const bool paint = op.edit_type == 7 && fabsf(existing) < __fmul_rn(op.dimensions[0], 2.0f);
    if (paint) mat = op.material_id;
    const uint32_t sec_out = paint ? 0u : ssec, blend_out = paint ? 0u : sbl;
    w0 = static_cast<uint32_t>(__half_as_ushort(__float2half_rn(nd))) | ((mat & 0x3Fu) << 16) | (sec_out << 22);
    w1 = blend_out << 24;
    changed = paint || fabsf(__fsub_rn(nd, existing)) > thr;
    out_d = nd;
  } else if (!f16) {
    // an untouched voxel of an f32 / u8 brick: the reference words carry
    // its distance in binary16
    w0 = (w0 & 0xFFFF0000u) | static_cast<uint32_t>(__half_as_ushort(__float2half_rn(existing_plane)));
  }
  const size_t o = static_cast<size_t>(dst) * 512 + v;
  if (f16) a.dist_f16[o] = static_cast<uint16_t>(w0 & 0xFFFFu);
  if (a.precision == RKF_PRECISION_F32) a.dist_f32[o] = out_d;
  a.mat[o] = static_cast<uint16_t>(((w0 >> 16) & 0x3Fu) | (((w0 >> 22) & 0x3Fu) << 6));
  a.blend[o] = static_cast<uint8_t>(w1 >> 24);
  if (a.aos) a.aos[o] = make_uint2(w0, w1);
  if (a.precision == RKF_PRECISION_U8) {
    // the brick's code: B = min(band, largest finite |d|), step = B/127
    // (the encoding of the u8 pool, k_encode_u8)
    __shared__ float red[16];
    const float ad = fabsf(out_d);
    float m = ad <= 3.0e38f ? ad : 0.0f;
    for (int off = 16; off; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, off));
    if ((v & 31) == 0) red[v >> 5] = m;
    __syncthreads();
    float mx = 0.0f;
    for (int k = 0; k < 16; ++k) mx = fmaxf(mx, red[k]);
    const float range = fmaxf(fminf(mx, a.u8_band), 1e-6f);
    const float st = __fdiv_rn(range, 127.0f);
    const float qa = __fdiv_rn(ad, st);
    const float q = a.u8_nearest ? rintf(qa) : floorf(qa);
    int code = q >= 127.0f ? 127 : static_cast<int>(q);
    if (!a.u8_nearest && code > 0 && __fmul_rn(static_cast<float>(code), st) > ad) --code;
    a.dist_u8[o] = static_cast<int8_t>(out_d < 0.0f ? -code : code);
    if (v == 0) a.brick_step[dst] = st;
  }
  const int any = __syncthreads_or(changed);
  if (v == 0) a.changed[c] = static_cast<uint8_t>(any != 0);
}

// Gather top entries and leaf contents of the given blocks.
__global__ void k_gather_blocks(const uint32_t* top, const uint32_t* leaves, const uint32_t* blocks,
                                uint32_t n, uint32_t* top_out, uint32_t* leaf_out) {
  const uint32_t b = blockIdx.x;
  if (b >= n) return;
  const uint32_t tv = top[blocks[b]];
  if (threadIdx.x == 0) top_out[b] = tv;
  for (uint32_t i = threadIdx.x; i < 512; i += blockDim.x)
    leaf_out[static_cast<size_t>(b) * 512 + i] = tv < RKF_INTERIOR_SLOT ? leaves[static_cast<size_t>(tv) * 512 + i] : tv;
}

__global__ void k_scatter_top(uint32_t* top, const uint32_t* blocks, const uint32_t* vals, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) top[blocks[i]] = vals[i];
}

}  // namespace detail

namespace {
// A temporary device buffer: caller scratch when given, else an allocation.
struct Temp {
  DevBuf own;
  void* p = nullptr;
  rkf_status get(const EditScratch* scratch, size_t bytes) {
    if (scratch) {
      p = (*scratch)(bytes);
      return p ? RKF_OK : fail(RKF_OOM, "rkf_edit_csg: no scratch room for the edit");
    }
    rkf_status st = own.alloc(bytes);
    p = own.p;
    return st;
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};
}  // namespace

rkf_status apply_edit(Ctx* c, const rkf_edit_op& op, cudaStream_t st, EditOutcome* out,
                      const EditScratch* scratch) {
  out->changed_bricks = 0;
  out->new_epoch = false;
  out->new_top.release();
  out->retired.clear();
  out->retired_leaves.clear();
  if (op.object_index >= c->obj_count()) return fail(RKF_INVALID_ARG, "rkf_edit_csg: object index out of range");
  if (op.edit_type == 8)
    return fail(RKF_UNSUPPORTED, "rkf_edit_csg: color paint writes a companion color pool this library does not keep");
  if (op.edit_type > 8 || op.shape_type > 2 || op.falloff > 2)
    return fail(RKF_INVALID_ARG, "rkf_edit_csg: unsupported edit, shape or falloff type");
  const rkf_gpu_object& go = c->objects[op.object_index];
  if (go.sdf_type != RKF_SDF_VOXELIZED) return fail(RKF_INVALID_ARG, "rkf_edit_csg: object is not voxelized");
  const ObjDev& od = c->objdev_host[op.object_index];
  const float vs = go.voxel_size;
  const float be = vs * 8.0f;
  const float max_dim = std::max(op.dimensions[0], std::max(op.dimensions[1], op.dimensions[2]));
  const float extent = max_dim + op.blend_k;  // EditOp::local_aabb (edit_op.rs:82-92)
  const float falloff_r = max_dim + op.blend_k;
  int bmin[3], bmax[3];
  float origin[3];
  for (int a = 0; a < 3; ++a) {
    origin[a] = -od.half_gs[a];  // grid minimum = object AABB minimum
    const float emin = op.position[a] - extent, emax = op.position[a] + extent;
    const int lo = static_cast<int>(std::floor((emin - origin[a]) / be));
    const int hi = static_cast<int>(std::ceil((emax - origin[a]) / be - 0.001f));
    bmin[a] = std::max(lo, 0);
    bmax[a] = std::min(std::max(hi, 0), static_cast<int>(go.brick_map_dims[a]) - 1);
  }
  // bricks whose box the falloff sphere reaches (outside it no voxel changes)
  std::vector<uint32_t> bxyz;
  std::vector<float> bmins;
  for (int z = bmin[2]; z <= bmax[2]; ++z)
    for (int y = bmin[1]; y <= bmax[1]; ++y)
      for (int x = bmin[0]; x <= bmax[0]; ++x) {
        const float m[3] = {origin[0] + static_cast<float>(x) * be, origin[1] + static_cast<float>(y) * be,
                            origin[2] + static_cast<float>(z) * be};
        double d2 = 0.0;
        for (int a = 0; a < 3; ++a) {
          const double p = op.position[a], lo = m[a], hi = static_cast<double>(m[a]) + be;
          const double e = p < lo ? lo - p : (p > hi ? p - hi : 0.0);
          d2 += e * e;
        }
        const double r = static_cast<double>(falloff_r) + 1e-4;
        if (d2 >= r * r) continue;
        bxyz.push_back(x);
        bxyz.push_back(y);
        bxyz.push_back(z);
        bmins.insert(bmins.end(), m, m + 3);
      }
  const uint32_t ncand_all = static_cast<uint32_t>(bxyz.size() / 3);
  if (ncand_all == 0) return RKF_OK;
  // current slots through the device index
  std::vector<uint32_t> cur(ncand_all);
  {
    Temp b;
    rkf_status s2 = b.get(scratch, static_cast<size_t>(ncand_all) * 16);
    if (s2 != RKF_OK) return s2;
    RKF_CUDA_TRY(cudaMemcpyAsync(b.p, bxyz.data(), bxyz.size() * 4, cudaMemcpyHostToDevice, st));
    rkf_status s3 = lookup_bricks(c, op.object_index, b.as<uint32_t>(), ncand_all,
                                  b.as<uint32_t>() + 3 * static_cast<size_t>(ncand_all), st);
    if (s3 != RKF_OK) return s3;
    RKF_CUDA_TRY(cudaMemcpyAsync(cur.data(), b.as<uint32_t>() + 3 * static_cast<size_t>(ncand_all),
                                 ncand_all * 4, cudaMemcpyDeviceToHost, st));
    RKF_CUDA_TRY(cudaStreamSynchronize(st));
  }
  const bool additive = op.edit_type == 0 || op.edit_type == 3;
  // smooth, flatten and paint act on allocated bricks only, the bricks
  // find_affected_bricks hands apply_edit_cpu (edit_op.rs:97-141)
  const bool allocated_only = op.edit_type >= 5;
  std::vector<uint32_t> src, dst, cidx;
  std::vector<float> cmin;
  for (uint32_t i = 0; i < ncand_all; ++i) {
    const uint32_t s = cur[i];
    if (allocated_only && (s == RKF_EMPTY_SLOT || s == RKF_INTERIOR_SLOT)) continue;
    if (s == RKF_EMPTY_SLOT && !additive) continue;
    if (s == RKF_INTERIOR_SLOT && additive) continue;
    src.push_back(s);
    cidx.push_back(i);
    cmin.insert(cmin.end(), &bmins[3 * i], &bmins[3 * i] + 3);
  }
  const uint32_t n = static_cast<uint32_t>(src.size());
  if (n == 0) return RKF_OK;
  if (c->free_slots.size() < n) return fail(RKF_OOM, "rkf_edit_csg: brick pool has too few free slots");
  for (uint32_t i = 0; i < n; ++i) {
    dst.push_back(c->free_slots.back());
    c->free_slots.pop_back();
  }
  // Until the new top grid exists, a failure restores the free list exactly
  // (order included) and leaves the index untouched (the copies went to
  // slots nothing references).
  const size_t free_kept = c->free_slots.size();
  const uint32_t used0 = c->used_slots, leaves0 = c->n_leaves;
  const std::vector<uint32_t> free_leaves0 = c->free_leaves;
  Rollback undo([&] {
    c->free_slots.resize(free_kept);
    for (size_t i = dst.size(); i-- > 0;) c->free_slots.push_back(dst[i]);
    c->used_slots = used0;
    c->n_leaves = leaves0;
    c->free_leaves = free_leaves0;
    out->retired.clear();
    out->retired_leaves.clear();
    out->changed_bricks = 0;
    out->new_top.release();
    out->new_empty_dist.release();
  });
  Temp dargs;
  rkf_status s2 = dargs.get(scratch, static_cast<size_t>(n) * 24 + 256);
  if (s2 != RKF_OK) return s2;
  uint32_t* d_src = dargs.as<uint32_t>();
  uint32_t* d_dst = d_src + n;
  float* d_min = reinterpret_cast<float*>(d_dst + n);
  uint8_t* d_changed = reinterpret_cast<uint8_t*>(d_min + 3 * static_cast<size_t>(n));
  RKF_CUDA_TRY(cudaMemcpyAsync(d_src, src.data(), n * 4ull, cudaMemcpyHostToDevice, st));
  RKF_CUDA_TRY(cudaMemcpyAsync(d_dst, dst.data(), n * 4ull, cudaMemcpyHostToDevice, st));
  RKF_CUDA_TRY(cudaMemcpyAsync(d_min, cmin.data(), n * 12ull, cudaMemcpyHostToDevice, st));
  detail::EditKernelArgs ka;
  std::memset(&ka, 0, sizeof(ka));
  ka.op = op;
  ka.iq[0] = -op.rotation[0];
  ka.iq[1] = -op.rotation[1];
  ka.iq[2] = -op.rotation[2];
  ka.iq[3] = op.rotation[3];
  ka.max_extent = max_dim;
  ka.vs = vs;
  ka.src = d_src;
  ka.dst = d_dst;
  ka.bmin = d_min;
  ka.dist_f16 = c->dist_f16.as<uint16_t>();
  ka.mat = c->mat.as<uint16_t>();
  ka.blend = c->blend.as<uint8_t>();
  ka.aos = c->aos.as<uint2>();
  ka.changed = d_changed;
  ka.dist_f32 = c->dist_f32.as<float>();
  ka.dist_u8 = c->dist_u8.as<int8_t>();
  ka.brick_step = c->brick_step.as<float>();
  ka.precision = c->cfg.precision;
  ka.u8_band = c->cfg.u8_band > 0.0f ? c->cfg.u8_band : 3.0f * vs;
  ka.u8_nearest = c->cfg.u8_round == 1 ? 1u : 0u;
  detail::k_edit<<<n, 512, 0, st>>>(ka);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  std::vector<uint8_t> changed(n);
  RKF_CUDA_TRY(cudaMemcpyAsync(changed.data(), d_changed, n, cudaMemcpyDeviceToHost, st));
  RKF_CUDA_TRY(cudaStreamSynchronize(st));
  // unchanged bricks keep their entry; their fresh slots go back
  std::vector<uint32_t> ch_brick, ch_slot;
  for (uint32_t i = 0; i < n; ++i) {
    if (changed[i]) {
      ch_brick.push_back(cidx[i]);
      ch_slot.push_back(dst[i]);
      if (src[i] < RKF_INTERIOR_SLOT) out->retired.push_back(src[i]);
    } else {
      c->free_slots.push_back(dst[i]);
    }
  }
  c->used_slots += static_cast<uint32_t>(ch_slot.size()) - static_cast<uint32_t>(out->retired.size());
  out->changed_bricks = static_cast<uint32_t>(ch_slot.size());
  if (ch_slot.empty()) {
    undo.dismiss();
    return RKF_OK;
  }

  // ---- new epoch of the index: copy the top grid, new leaves for the blocks
  std::vector<uint32_t> blocks;  // global top indices of touched blocks
  std::vector<uint32_t> local_of(ch_slot.size());
  for (size_t i = 0; i < ch_brick.size(); ++i) {
    const uint32_t* b = &bxyz[3 * ch_brick[i]];
    const uint32_t blk = od.top_off + (b[0] >> 3) + (b[1] >> 3) * od.tdim[0] + (b[2] >> 3) * od.tdim[0] * od.tdim[1];
    auto it = std::find(blocks.begin(), blocks.end(), blk);
    local_of[i] = static_cast<uint32_t>(it - blocks.begin());
    if (it == blocks.end()) blocks.push_back(blk);
  }
  const uint32_t nb = static_cast<uint32_t>(blocks.size());
  // leaf numbers of the new epoch's touched blocks: freed leaves first (the
  // last freed on top), then new ones after n_leaves
  std::vector<uint32_t> newtop(nb);
  uint32_t appended = 0;
  for (uint32_t i = 0; i < nb; ++i) {
    if (!c->free_leaves.empty()) {
      newtop[i] = c->free_leaves.back();
      c->free_leaves.pop_back();
    } else {
      newtop[i] = c->n_leaves + appended++;
    }
  }
  if ((s2 = c->ensure_leaf_capacity(c->n_leaves + appended)) != RKF_OK) return s2;
  Temp g;
  if ((s2 = g.get(scratch, static_cast<size_t>(nb) * (4 + 4 + 2048) + 256)) != RKF_OK) return s2;
  uint32_t* d_blocks = g.as<uint32_t>();
  uint32_t* d_topv = d_blocks + nb;
  uint32_t* d_leafs = d_topv + nb;
  RKF_CUDA_TRY(cudaMemcpyAsync(d_blocks, blocks.data(), nb * 4ull, cudaMemcpyHostToDevice, st));
  detail::k_gather_blocks<<<nb, 128, 0, st>>>(c->top.as<uint32_t>(), c->leaves.as<uint32_t>(), d_blocks, nb,
                                              d_topv, d_leafs);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  std::vector<uint32_t> leafv(static_cast<size_t>(nb) * 512), oldtop(nb);
  RKF_CUDA_TRY(cudaMemcpyAsync(leafv.data(), d_leafs, leafv.size() * 4, cudaMemcpyDeviceToHost, st));
  RKF_CUDA_TRY(cudaMemcpyAsync(oldtop.data(), d_topv, nb * 4ull, cudaMemcpyDeviceToHost, st));
  RKF_CUDA_TRY(cudaStreamSynchronize(st));
  // the leaves these blocks pointed at belong to the old epoch only
  for (uint32_t i = 0; i < nb; ++i)
    if (oldtop[i] < RKF_INTERIOR_SLOT) out->retired_leaves.push_back(oldtop[i]);
  for (size_t i = 0; i < ch_brick.size(); ++i) {
    const uint32_t* b = &bxyz[3 * ch_brick[i]];
    leafv[static_cast<size_t>(local_of[i]) * 512 + (b[0] & 7) + (b[1] & 7) * 8 + (b[2] & 7) * 64] = ch_slot[i];
  }
  // the new leaves (runs of consecutive numbers in one copy each); a new top
  // grid points the touched blocks at them
  for (uint32_t i = 0; i < nb;) {
    uint32_t j = i + 1;
    while (j < nb && newtop[j] == newtop[j - 1] + 1) ++j;
    RKF_CUDA_TRY(cudaMemcpyAsync(c->leaves.as<uint32_t>() + static_cast<size_t>(newtop[i]) * 512,
                                 leafv.data() + static_cast<size_t>(i) * 512, static_cast<size_t>(j - i) * 2048,
                                 cudaMemcpyHostToDevice, st));
    i = j;
  }
  const bool into = out->top_dst && out->field_dst;
  if (!into && (s2 = out->new_top.alloc(std::max<uint64_t>(c->top_len, 1) * 4)) != RKF_OK) return s2;
  uint32_t* ntop = into ? out->top_dst : out->new_top.as<uint32_t>();
  RKF_CUDA_TRY(cudaMemcpyAsync(ntop, c->top.p, c->top_len * 4, cudaMemcpyDeviceToDevice, st));
  RKF_CUDA_TRY(cudaMemcpyAsync(d_topv, newtop.data(), nb * 4ull, cudaMemcpyHostToDevice, st));
  detail::k_scatter_top<<<(nb + 127) / 128, 128, 0, st>>>(ntop, d_blocks, d_topv, nb);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  // the touched blocks are leaf blocks now: lower the field around them
  if (!into && (s2 = out->new_empty_dist.alloc(std::max<uint64_t>(c->top_len, 1))) != RKF_OK) return s2;
  uint8_t* nfield = into ? out->field_dst : out->new_empty_dist.as<uint8_t>();
  RKF_CUDA_TRY(cudaMemcpyAsync(nfield, c->empty_dist.p, c->top_len, cudaMemcpyDeviceToDevice, st));
  if ((s2 = lower_empty_dist(od, nfield, d_blocks, blocks, st)) != RKF_OK) return s2;
  c->counted(1);
  c->n_leaves += appended;
  // the reference flat map (read only by the plain march) is updated in place
  if (od.has_flat && !c->flat_host.empty()) {
    for (size_t i = 0; i < ch_brick.size(); ++i) {
      const uint32_t* b = &bxyz[3 * ch_brick[i]];
      const uint64_t f = od.map_off + b[0] + static_cast<uint64_t>(b[1]) * od.bdims[0] +
                         static_cast<uint64_t>(b[2]) * od.bdims[0] * od.bdims[1];
      c->flat_host[f] = ch_slot[i];
      RKF_CUDA_TRY(cudaMemcpyAsync(c->flat_maps.as<uint32_t>() + f, &c->flat_host[f], 4, cudaMemcpyHostToDevice, st));
    }
  }
  RKF_CUDA_TRY(cudaStreamSynchronize(st));
  undo.dismiss();
  out->new_epoch = true;
  return RKF_OK;
}

}  // namespace rkf

using namespace rkf;

extern "C" rkf_status rkf_edit_csg(rkf_ctx* ctx, const rkf_edit_op* op, uint64_t* new_epoch) {
  if (!ctx || !op) return fail(RKF_INVALID_ARG, "rkf_edit_csg: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_edit_csg: the context is serving; submit edits as requests");
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  // direct edits: nothing else holds the old epoch once the context stream is idle
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  EditOutcome r;
  rkf_status st = apply_edit(c, *op, c->stream, &r);
  if (st != RKF_OK) return st;
  if (r.new_top.p) {
    std::swap(c->top.p, r.new_top.p);
    std::swap(c->top.bytes, r.new_top.bytes);
    std::swap(c->empty_dist.p, r.new_empty_dist.p);
    std::swap(c->empty_dist.bytes, r.new_empty_dist.bytes);
    c->epoch++;
    for (uint32_t s : r.retired) c->free_slots.push_back(s);
    for (uint32_t l : r.retired_leaves) c->free_leaves.push_back(l);
  }
  if (new_epoch) *new_epoch = c->epoch;
  return RKF_OK;
}
