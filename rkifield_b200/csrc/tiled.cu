// tiled.cu — the coarse acceleration field and the per-tile object lists of
// the tiled strategy (ray_march_tiled, ray_march.wgsl:874-985).
//
// Coarse field (crates/rkf-render/src/coarse_field.rs): 0.32 m cells
// (COARSE_VOXEL_SIZE, :21) over the union of the object AABBs grown by the
// runtime's 1 m margin (from_scene_aabbs, :211-232; the runtime call at
// rkf-runtime/src/api/renderer/render.rs:257-263), at most 128 per axis
// (:24, :93-97); each texel is the binary16 of the smallest unsigned distance
// from the cell centre to an object AABB, starting from vs * max(dims)
// (populate, :240-266).  The reference fills it on the CPU every frame; here
// one thread per cell fills it on the device when the objects change.
//
// Tile lists (tile_object_cull.wgsl:90-205): per 16x16-pixel tile the objects
// whose projected AABB overlaps it, at most 32.  The shader appends with a
// shared-memory atomic, so its order is unspecified; here one warp per tile
// appends in ascending object index (a ballot per 32 objects).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "ctx.h"
#include "march.h"
#include "../../include/rkf_cuda_testing.h"
#include "empty_dist.h"
#include "tiled.h"

namespace rkf {

namespace detail {

constexpr uint32_t kMaxAabbs = 256;  // objects of a tiled launch (28 B each in the launch parameters)

struct Aabbs {
  float lo[kMaxAabbs][3], hi[kMaxAabbs][3];
  uint32_t none[kMaxAabbs];  // sdf_type NONE (skipped by the cull, kept by the field)
  uint32_t n;
};
static_assert(sizeof(Aabbs) <= 16384, "the AABB table must fit the kernel parameter space with room to spare");

__global__ void k_coarse_build(const __grid_constant__ Aabbs a, float ox, float oy, float oz, uint32_t dx,
                               uint32_t dy, uint32_t dz, float vs, float start, uint16_t* __restrict__ tex) {
  const uint64_t n = static_cast<uint64_t>(dx) * dy * dz;
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t x = static_cast<uint32_t>(i % dx), y = static_cast<uint32_t>((i / dx) % dy),
                 z = static_cast<uint32_t>(i / (static_cast<uint64_t>(dx) * dy));
  const float q[3] = {__fadd_rn(ox, __fmul_rn(__fadd_rn(static_cast<float>(x), 0.5f), vs)),
                      __fadd_rn(oy, __fmul_rn(__fadd_rn(static_cast<float>(y), 0.5f), vs)),
                      __fadd_rn(oz, __fmul_rn(__fadd_rn(static_cast<float>(z), 0.5f), vs))};
  float best = start;
  for (uint32_t k = 0; k < a.n; ++k) {
    float d3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      d3[c] = fmaxf(fmaxf(__fsub_rn(a.lo[k][c], q[c]), __fsub_rn(q[c], a.hi[k][c])), 0.0f);
    best = fminf(best, len3(d3[0], d3[1], d3[2]));
  }
  tex[i] = __half_as_ushort(__float2half_rn(best));
}

struct CullView {
  float pos[3], fwd[3], right[3], up[3];
  float resx, resy;
  uint32_t tiles_x, tile_off;
};

__device__ __forceinline__ float dot3(const float* a, const float* b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1])), __fmul_rn(a[2], b[2]));
}

// One warp per tile of one view.
__global__ void k_tile_cull(const __grid_constant__ Aabbs a, CullView v, uint32_t* __restrict__ cnt,
                            uint32_t* __restrict__ list) {
  const uint32_t tile = blockIdx.x, lane = threadIdx.x;
  const uint32_t tx = tile % v.tiles_x, ty = tile / v.tiles_x;
  const float tminx = static_cast<float>(tx * 16), tminy = static_cast<float>(ty * 16);
  const float tmaxx = __fadd_rn(tminx, 16.0f), tmaxy = __fadd_rn(tminy, 16.0f);
  const float r_sq = dot3(v.right, v.right), u_sq = dot3(v.up, v.up);
  uint32_t count = 0;
  for (uint32_t base = 0; base < a.n; base += 32) {
    const uint32_t i = base + lane;
    bool overlaps = false;
    if (i < a.n && !a.none[i]) {
      float smin_x = v.resx, smin_y = v.resy, smax_x = 0.0f, smax_y = 0.0f;
      bool front = false, behind = false;
      for (uint32_t c = 0; c < 8; ++c) {
        const float rel[3] = {__fsub_rn((c & 1u) ? a.hi[i][0] : a.lo[i][0], v.pos[0]),
                              __fsub_rn((c & 2u) ? a.hi[i][1] : a.lo[i][1], v.pos[1]),
                              __fsub_rn((c & 4u) ? a.hi[i][2] : a.lo[i][2], v.pos[2])};
        const float depth = dot3(rel, v.fwd);
        if (depth > 0.0f) {  // project_to_pixel (:90-113)
          const float ndc_x = __fdiv_rn(dot3(rel, v.right), __fmul_rn(depth, r_sq));
          const float ndc_y = __fdiv_rn(dot3(rel, v.up), __fmul_rn(depth, u_sq));
          const float px = __fmul_rn(__fadd_rn(__fmul_rn(ndc_x, 0.5f), 0.5f), v.resx);
          const float py = __fmul_rn(__fsub_rn(0.5f, __fmul_rn(ndc_y, 0.5f)), v.resy);
          front = true;
          smin_x = fmin_(smin_x, px);
          smin_y = fmin_(smin_y, py);
          smax_x = fmax_(smax_x, px);
          smax_y = fmax_(smax_y, py);
        } else {
          behind = true;
        }
      }
      if (behind && front) overlaps = true;
      else if (!behind && front)
        overlaps = smax_x >= tminx && smin_x < tmaxx && smax_y >= tminy && smin_y < tmaxy;
    }
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, overlaps);
    const uint32_t at = count + __popc(m & ((1u << lane) - 1u));
    if (overlaps && at < kTileObjects) list[(static_cast<size_t>(v.tile_off) + tile) * kTileObjects + at] = i;
    count += __popc(m);
  }
  if (lane == 0) cnt[v.tile_off + tile] = min(count, kTileObjects);
}

}  // namespace detail

rkf_status prepare_tiled(Ctx* c, std::vector<Segment>& segs, cudaStream_t st, TiledDev* out) {
  const uint32_t n = c->obj_count();
  if (n > detail::kMaxAabbs) return fail(RKF_UNSUPPORTED, "tiled march: too many objects");
  detail::Aabbs a;
  std::memset(&a, 0, sizeof(a));
  a.n = n;
  for (uint32_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      a.lo[i][k] = c->objects[i].aabb_min[k];
      a.hi[i][k] = c->objects[i].aabb_max[k];
    }
    a.none[i] = c->objects[i].sdf_type == RKF_SDF_NONE ? 1u : 0u;
  }
  // ---- coarse field, rebuilt when the scene changed ----------------------
  const float vs = 0.32f, margin = 1.0f;
  if (!c->coarse_tex.p || c->coarse_epoch != c->epoch) {
    float lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
      lo[k] = n ? 3.402823466e+38f : 0.0f;
      hi[k] = n ? -3.402823466e+38f : vs;
    }
    for (uint32_t i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::fmin(lo[k], a.lo[i][k]);
        hi[k] = std::fmax(hi[k], a.hi[i][k]);
      }
    for (int k = 0; k < 3; ++k) {
      c->coarse_origin[k] = lo[k] - margin;
      const float extent = (hi[k] + margin) - c->coarse_origin[k];
      const float cells = std::fmin(std::ceil(extent / vs), 128.0f);
      c->coarse_dims[k] = std::max<uint32_t>(1u, cells > 0.0f ? static_cast<uint32_t>(cells) : 0u);
    }
    const uint64_t cells = static_cast<uint64_t>(c->coarse_dims[0]) * c->coarse_dims[1] * c->coarse_dims[2];
    DevBuf nt;
    rkf_status s2 = nt.alloc(cells * 2);
    if (s2 != RKF_OK) return s2;
    const uint32_t dmax = std::max(c->coarse_dims[0], std::max(c->coarse_dims[1], c->coarse_dims[2]));
    detail::k_coarse_build<<<static_cast<unsigned>((cells + 255) / 256), 256, 0, st>>>(
        a, c->coarse_origin[0], c->coarse_origin[1], c->coarse_origin[2], c->coarse_dims[0], c->coarse_dims[1],
        c->coarse_dims[2], vs, vs * static_cast<float>(dmax), nt.as<uint16_t>());
    c->counted();
    RKF_CUDA_TRY(cudaGetLastError());
    RKF_CUDA_TRY(cudaStreamSynchronize(st));
    std::swap(c->coarse_tex.p, nt.p);
    std::swap(c->coarse_tex.bytes, nt.bytes);
    c->coarse_epoch = c->epoch;
  }
  // ---- tile lists of every view ------------------------------------------
  uint64_t tiles = 0;
  for (const Segment& sg : segs)
    if (sg.kind == 0) tiles += static_cast<uint64_t>((sg.w + 15) / 16) * ((sg.h + 15) / 16);
  const size_t need = (tiles ? tiles : 1) * (kTileObjects + 1) * 4;
  if (c->tile_buf.bytes < need) {
    rkf_status s2 = c->tile_buf.alloc(need);
    if (s2 != RKF_OK) return s2;
  }
  uint32_t* cnt = c->tile_buf.as<uint32_t>();
  uint32_t* list = cnt + (tiles ? tiles : 1);
  uint64_t off = 0;
  for (Segment& sg : segs) {
    if (sg.kind != 0) continue;
    detail::CullView v;
    for (int k = 0; k < 3; ++k) {
      v.pos[k] = sg.pos[k];
      v.fwd[k] = sg.fwd[k];
      v.right[k] = sg.right[k];
      v.up[k] = sg.up[k];
      sg.coarse_ocr[k] = c->coarse_origin[k] - sg.pos[k];  // CoarseField::upload (:297-305)
    }
    v.resx = static_cast<float>(sg.w);
    v.resy = static_cast<float>(sg.h);
    v.tiles_x = (sg.w + 15) / 16;
    v.tile_off = static_cast<uint32_t>(off);
    sg.tile_off = static_cast<uint32_t>(off);
    const uint32_t nt = v.tiles_x * ((sg.h + 15) / 16);
    if (nt) {
      detail::k_tile_cull<<<nt, 32, 0, st>>>(a, v, cnt, list);
      c->counted();
    }
    RKF_CUDA_TRY(cudaGetLastError());
    off += nt;
  }
  out->coarse = c->coarse_tex.as<uint16_t>();
  for (int k = 0; k < 3; ++k) out->cdims[k] = c->coarse_dims[k];
  out->cinv_vs = 1.0f / vs;
  out->tile_cnt = cnt;
  out->tile_list = list;
  return RKF_OK;
}

namespace detail {

// 1 for a texel whose value exceeds kCoarseSafe
__global__ void k_coarse_unsafe(const uint16_t* __restrict__ tex, uint32_t n, uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __half2float(__ushort_as_half(tex[i])) > kCoarseSafe ? 1u : 0u;
}

// inclusive prefix sum along one axis of a dx x dy x dz array (one thread per line)
__global__ void k_prefix_axis(uint32_t* __restrict__ a, uint32_t dx, uint32_t dy, uint32_t dz, uint32_t axis) {
  const uint32_t line = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t len = axis == 0 ? dx : axis == 1 ? dy : dz;
  const uint32_t lines = axis == 0 ? dy * dz : axis == 1 ? dx * dz : dx * dy;
  if (line >= lines) return;
  size_t base, stride;
  if (axis == 0) {
    base = static_cast<size_t>(line) * dx;
    stride = 1;
  } else if (axis == 1) {
    base = static_cast<size_t>(line % dx) + static_cast<size_t>(line / dx) * dx * dy;
    stride = dx;
  } else {
    base = line;
    stride = static_cast<size_t>(dx) * dy;
  }
  uint32_t acc = 0;
  for (uint32_t k = 0; k < len; ++k) {
    acc += a[base + k * stride];
    a[base + k * stride] = acc;
  }
}

struct SafeArgs {
  const uint32_t* top;   // the object's top grid (global indices)
  const uint32_t* pre;   // 3D prefix count of unsafe texels
  uint32_t* masked;      // out: top with unsafe EMPTY blocks made INTERIOR
  uint32_t off, tx, ty, tz;
  uint32_t cd[3];        // coarse field dims
  double lo[3];          // world position of grid coordinate 0 (-half_gs - translation)
  double block;          // block edge (64 voxels)
  double corg[3];        // coarse field origin
  double cvs;            // coarse cell
};

__device__ __forceinline__ uint32_t pre_at(const SafeArgs& a, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0) return 0u;
  return a.pre[static_cast<size_t>(x) + static_cast<size_t>(y) * a.cd[0] +
               static_cast<size_t>(z) * a.cd[0] * a.cd[1]];
}

// One thread per top block: the texels a sample in the block (widened by a
// voxel) can interpolate lie in [floor(xmin) - 1, floor(xmax) + 2] per axis
// of x = (world - origin) / cell - 0.5 (one texel of margin each side covers
// the float rounding of the camera-relative coordinates); the block stays
// EMPTY only if none of them is unsafe.  Positions outside the field sample 0.
__global__ void k_tiled_mask(const __grid_constant__ SafeArgs a) {
  const uint64_t n = static_cast<uint64_t>(a.tx) * a.ty * a.tz;
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t k[3] = {static_cast<uint32_t>(i % a.tx), static_cast<uint32_t>((i / a.tx) % a.ty),
                         static_cast<uint32_t>(i / (static_cast<uint64_t>(a.tx) * a.ty))};
  const uint32_t v = a.top[a.off + i];
  uint32_t out = v;
  if (v == RKF_EMPTY_SLOT) {
    int r0[3], r1[3];
    bool any = true;
    for (int d = 0; d < 3; ++d) {
      const double vox = a.block / 64.0;
      const double w0 = a.lo[d] + k[d] * a.block - vox, w1 = a.lo[d] + (k[d] + 1) * a.block + vox;
      const double x0 = (w0 - a.corg[d]) / a.cvs - 0.5, x1 = (w1 - a.corg[d]) / a.cvs - 0.5;
      r0[d] = max(static_cast<int>(floor(x0)) - 1, 0);
      r1[d] = min(static_cast<int>(floor(x1)) + 2, static_cast<int>(a.cd[d]) - 1);
      if (r1[d] < r0[d]) any = false;  // the block lies wholly outside the field
    }
    uint32_t cnt = 0;
    if (any) {
      const int x0 = r0[0] - 1, y0 = r0[1] - 1, z0 = r0[2] - 1, x1 = r1[0], y1 = r1[1], z1 = r1[2];
      cnt = pre_at(a, x1, y1, z1) - pre_at(a, x0, y1, z1) - pre_at(a, x1, y0, z1) - pre_at(a, x1, y1, z0) +
            pre_at(a, x0, y0, z1) + pre_at(a, x0, y1, z0) + pre_at(a, x1, y0, z0) - pre_at(a, x0, y0, z0);
    }
    if (cnt) out = RKF_INTERIOR_SLOT;
  }
  a.masked[a.off + i] = out;
}

}  // namespace detail

rkf_status prepare_tiled_empty(Ctx* c, cudaStream_t st, const std::vector<uint32_t>& objs) {
  if (c->tiled_epoch == c->epoch && c->tiled_empty_dist.p) return RKF_OK;
  if (c->coarse_epoch != c->epoch || !c->coarse_tex.p)
    return fail(RKF_CUDA_ERROR, "tiled march: coarse field missing for the empty-space field");
  const uint32_t cd[3] = {c->coarse_dims[0], c->coarse_dims[1], c->coarse_dims[2]};
  const uint32_t nt = cd[0] * cd[1] * cd[2];
  DevBuf pre, masked, field;
  rkf_status s2 = pre.alloc(static_cast<size_t>(nt) * 4);
  if (s2 == RKF_OK) s2 = masked.alloc(std::max<uint64_t>(c->top_len, 1) * 4);
  if (s2 == RKF_OK) s2 = field.alloc(std::max<uint64_t>(c->top_len, 1));
  if (s2 != RKF_OK) return s2;
  detail::k_coarse_unsafe<<<(nt + 255) / 256, 256, 0, st>>>(c->coarse_tex.as<uint16_t>(), nt, pre.as<uint32_t>());
  c->counted();
  for (uint32_t axis = 0; axis < 3; ++axis) {
    const uint32_t lines = axis == 0 ? cd[1] * cd[2] : axis == 1 ? cd[0] * cd[2] : cd[0] * cd[1];
    detail::k_prefix_axis<<<(lines + 127) / 128, 128, 0, st>>>(pre.as<uint32_t>(), cd[0], cd[1], cd[2], axis);
    c->counted();
  }
  RKF_CUDA_TRY(cudaMemsetAsync(field.p, 0, std::max<uint64_t>(c->top_len, 1), st));
  for (uint32_t vi : objs) {
    const ObjDev& o = c->objdev_host[vi];
    detail::SafeArgs a;
    a.top = c->top.as<uint32_t>();
    a.pre = pre.as<uint32_t>();
    a.masked = masked.as<uint32_t>();
    a.off = o.top_off;
    a.tx = o.tdim[0];
    a.ty = o.tdim[1];
    a.tz = o.tdim[2];
    for (int d = 0; d < 3; ++d) {
      a.cd[d] = cd[d];
      a.lo[d] = -static_cast<double>(o.half_gs[d]) - static_cast<double>(o.m[12 + d]);
      a.corg[d] = c->coarse_origin[d];
    }
    a.block = 64.0 * static_cast<double>(o.vs);
    a.cvs = 0.32;
    const uint64_t nb = static_cast<uint64_t>(a.tx) * a.ty * a.tz;
    detail::k_tiled_mask<<<static_cast<unsigned>((nb + 255) / 256), 256, 0, st>>>(a);
    c->counted();
    RKF_CUDA_TRY(cudaGetLastError());
    if ((s2 = build_empty_dist(o, masked.as<uint32_t>(), field.as<uint8_t>(), st)) != RKF_OK) return s2;
    c->counted(3);
  }
  RKF_CUDA_TRY(cudaStreamSynchronize(st));
  std::swap(c->tiled_empty_dist.p, field.p);
  std::swap(c->tiled_empty_dist.bytes, field.bytes);
  c->tiled_epoch = c->epoch;
  return RKF_OK;
}

}  // namespace rkf

extern "C" rkf_status rkf_testing_export_coarse(rkf_ctx* ctx, float origin[3], uint32_t dims[3], uint16_t* tex,
                                                 uint64_t* n) {
  using namespace rkf;
  if (!ctx || !origin || !dims || !n) return fail(RKF_INVALID_ARG, "rkf_testing_export_coarse: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  std::vector<Segment> none;
  TiledDev td;
  rkf_status st = prepare_tiled(c, none, c->stream, &td);  // builds the field for the current epoch
  if (st != RKF_OK) return st;
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 3; ++k) {
    origin[k] = c->coarse_origin[k];
    dims[k] = c->coarse_dims[k];
  }
  *n = static_cast<uint64_t>(dims[0]) * dims[1] * dims[2];
  if (tex) RKF_CUDA_TRY(cudaMemcpy(tex, c->coarse_tex.p, *n * 2, cudaMemcpyDeviceToHost));
  return RKF_OK;
}
