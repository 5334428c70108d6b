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
#include "tiled.h"

namespace rkf {

namespace detail {

constexpr uint32_t kMaxAabbs = 64;

struct Aabbs {
  float lo[kMaxAabbs][3], hi[kMaxAabbs][3];
  uint32_t none[kMaxAabbs];  // sdf_type NONE (skipped by the cull, kept by the field)
  uint32_t n;
};

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
    if (nt) detail::k_tile_cull<<<nt, 32, 0, st>>>(a, v, cnt, list);
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

}  // namespace rkf
