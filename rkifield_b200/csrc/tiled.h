// tiled.h — inputs of the tiled march strategy (tiled.cu).
#pragma once

#include <cuda_fp16.h>

#include <vector>

#include "device_common.cuh"

namespace rkf {

struct Ctx;
struct Segment;

constexpr uint32_t kTileObjects = 32;           // TILE_MAX_OBJECTS (ray_march.wgsl:48)
constexpr uint32_t kNoTiles = 0xFFFFFFFFu;      // a ray that marches every object
constexpr float kCoarseNear = 0.5f;             // COARSE_NEAR_THRESHOLD (ray_march.wgsl:863)

// What the march reads for the tiled strategy.
struct TiledDev {
  const uint16_t* coarse;       // binary16 texels, x + y*dx + z*dx*dy
  uint32_t cdims[3];
  float cinv_vs;                // 1 / COARSE_VOXEL_SIZE
  const uint32_t* tile_cnt;     // per tile (all view segments, segment-relative offsets)
  const uint32_t* tile_list;    // kTileObjects object indices per tile
};

// Build the coarse field (when the objects changed since the last build) and
// the tile lists of every view segment; sets each view segment's tile offset
// and field origin relative to its camera.  Enqueued on st.
rkf_status prepare_tiled(Ctx* c, std::vector<Segment>& segs, cudaStream_t st, TiledDev* out);

// The empty-space field the tiled march of voxelized objects (translation-
// only objects, the empty-space path's kind) runs its EMPTY runs on: each
// listed object's field with every block treated as occupied that a sample
// inside it could see a coarse value above kCoarseSafe through (so there the
// tiled step evaluates the object, as the brute step does); the regions of
// other objects hold 0 (no run).  Built into c->tiled_empty_dist when the
// scene epoch changed; needs the coarse field of the same epoch.  Enqueued on
// st and synchronised.
constexpr float kCoarseSafe = 0.49f;  // below COARSE_NEAR_THRESHOLD with room for mix() rounding
rkf_status prepare_tiled_empty(Ctx* c, cudaStream_t st, const std::vector<uint32_t>& objs);

// sample_coarse_field (ray_march.wgsl:228-235) at a camera-relative position:
// 0 outside the field, else a linear, clamp-to-edge read of the texture, with
// the texture unit modelled as 1/256 weight steps and mix() along x, y, z.
__device__ __forceinline__ float coarse_sample(const TiledDev& td, const float* ocr, float cx, float cy,
                                               float cz) {
  const float cr[3] = {cx, cy, cz};
  int i0[3], i1[3];
  float w[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float n = static_cast<float>(td.cdims[a]);
    const float u = __fdiv_rn(__fmul_rn(__fsub_rn(cr[a], ocr[a]), td.cinv_vs), n);
    if (u < 0.0f || u > 1.0f) return 0.0f;
    const float x = __fsub_rn(__fmul_rn(u, n), 0.5f);
    const float f = floorf(x);
    w[a] = __fmul_rn(rintf(__fmul_rn(__fsub_rn(x, f), 256.0f)), 0.00390625f);
    const int k = static_cast<int>(f), last = static_cast<int>(td.cdims[a]) - 1;
    i0[a] = min(max(k, 0), last);
    i1[a] = min(max(k + 1, 0), last);
  }
  const size_t sy = td.cdims[0], sz = static_cast<size_t>(td.cdims[0]) * td.cdims[1];
  auto T = [&](int x, int y, int z) {
    return __half2float(__ushort_as_half(__ldg(td.coarse + x + y * sy + z * sz)));
  };
  const float c00 = mixf(T(i0[0], i0[1], i0[2]), T(i1[0], i0[1], i0[2]), w[0]);
  const float c10 = mixf(T(i0[0], i1[1], i0[2]), T(i1[0], i1[1], i0[2]), w[0]);
  const float c01 = mixf(T(i0[0], i0[1], i1[2]), T(i1[0], i0[1], i1[2]), w[0]);
  const float c11 = mixf(T(i0[0], i1[1], i1[2]), T(i1[0], i1[1], i1[2]), w[0]);
  return mixf(mixf(c00, c10, w[1]), mixf(c01, c11, w[1]), w[2]);
}

}  // namespace rkf
