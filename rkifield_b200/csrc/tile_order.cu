// tile_order.cu — heaviest-first order of the ray tiles of views.
//
// A persistent march hands out a view's ray tiles (tile_w x tile_h pixels per
// work item) from a global counter.  In row order the tiles whose rays take
// longest -- rays that cross a hundred metres of empty space before they meet
// or graze geometry, and step through all of it -- are often handed out last,
// and the launch ends on a tail where a few warps march alone.  Handing the
// heaviest tiles out first lets the cheap ones fill that tail.  The order
// changes which warp marches a tile and when, never what a ray computes, so
// every output is the same in any order.
//
// The estimate walks each tile's centre ray through the empty-space distance
// field (one byte per 8^3-brick block: radius of the cube of EMPTY blocks
// around it, empty_dist.h) from cube exit to cube exit, and counts the EMPTY
// steps before the last block that is not EMPTY within the ray's reach, plus
// a few steps per such block; eight lanes walk the eight stretches of a ray
// side by side.  A counting sort (64 cost classes, heaviest
// first, separately within each group of tile rows) writes the permutation.
#include <cmath>
#include <cstring>

#include "ctx.h"
#include "tile_order.h"

namespace rkf {
namespace detail {

constexpr uint32_t kOrderKeys = kOrderMaxGroups * kOrderBuckets;

__device__ __forceinline__ uint32_t order_view_of(const OrderTable& t, uint32_t gi) {
  uint32_t lo = 0, hi = t.n_views;  // last view with tile_base <= gi
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (t.v[mid].tile_base <= gi) lo = mid; else hi = mid;
  }
  return lo;
}

// Lanes that walk one tile's centre ray, each over its own stretch of the
// ray's reach: the walk is a chain of dependent loads of the field (cold in
// L2 at the start of a frame), so splitting it cuts the kernel's longest
// chain by this factor.
constexpr uint32_t kOrderLanes = 8;
constexpr int kOrderLaneSteps = 32;  // cube jumps a lane takes at most

// Part `lane` of the walk of a tile's centre ray (see above): the number of
// non-EMPTY blocks it meets and the distance of the last of them (0: none).
__device__ void tile_walk(const OrderTable& t, const Segment& sg, uint32_t col, uint32_t row, uint32_t lane,
                          uint32_t* blocks_out, float* t_last_out) {
  const ObjDev& o = t.o;
  *blocks_out = 0;
  *t_last_out = 0.0f;
  const uint32_t px = min(col * t.tile_w + t.tile_w / 2, sg.w - 1);
  const uint32_t py = min(row * t.tile_h + t.tile_h / 2, sg.h - 1);
  const float u = (static_cast<float>(px) + 0.5f + sg.jitter[0]) / static_cast<float>(sg.w);
  const float v = (static_cast<float>(py) + 0.5f + sg.jitter[1]) / static_cast<float>(sg.h);
  const float nx = 2.0f * u - 1.0f, ny = 1.0f - 2.0f * v;
  float d[3];
  for (int a = 0; a < 3; ++a) d[a] = sg.fwd[a] + sg.right[a] * nx + sg.up[a] * ny;
  const float il = rsqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  // grid voxel coordinate along the ray: g(t) = a0 + a1 * t (t in metres)
  float a0[3], a1[3], ia[3];
  float t0 = 0.0f, t1 = t.reach;
  for (int a = 0; a < 3; ++a) {
    a0[a] = (sg.pos[a] + o.m[12 + a] + o.half_gs[a]) * o.rcp_vs - 0.5f;
    a1[a] = d[a] * il * o.rcp_vs;
    ia[a] = a1[a] != 0.0f ? 1.0f / a1[a] : 0.0f;
    const float tv = static_cast<float>(o.tv[a]);
    if (a1[a] != 0.0f) {
      const float ta = -a0[a] * ia[a], tb = (tv - a0[a]) * ia[a];
      t0 = fmaxf(t0, fminf(ta, tb));
      t1 = fminf(t1, fmaxf(ta, tb));
    } else if (!(a0[a] >= 0.0f && a0[a] < tv)) {
      t1 = -1.0f;
    }
  }
  if (!(t0 < t1)) return;  // the ray misses the grid
  const float len = (t1 - t0) * (1.0f / static_cast<float>(kOrderLanes));
  const float s1 = lane + 1 == kOrderLanes ? t1 : t0 + len * static_cast<float>(lane + 1);
  const float eps = 0.01f * o.vs;
  float tt = t0 + len * static_cast<float>(lane) + eps, t_last = 0.0f;
  uint32_t blocks = 0;
  for (int it = 0; it < kOrderLaneSteps && tt < s1; ++it) {
    int k[3];
    for (int a = 0; a < 3; ++a) {
      const float g = fminf(fmaxf(a0[a] + a1[a] * tt, 0.0f), static_cast<float>(o.tv[a] - 1));
      k[a] = static_cast<int>(g) >> 6;
    }
    const uint32_t r = __ldg(t.field + o.top_off + k[0] + k[1] * o.tdim[0] + k[2] * o.tdim[0] * o.tdim[1]);
    const int rad = r ? static_cast<int>(r) - 1 : 0;
    float te = INFINITY;
    for (int a = 0; a < 3; ++a) {
      const float lo = static_cast<float>((k[a] - rad) * 64), hi = static_cast<float>((k[a] + rad + 1) * 64);
      if (a1[a] > 0.0f) te = fminf(te, (hi - a0[a]) * ia[a]);
      else if (a1[a] < 0.0f) te = fminf(te, (lo - a0[a]) * ia[a]);
    }
    if (r == 0) {
      ++blocks;
      t_last = tt;
    }
    tt = fmaxf(te, tt) + eps;
  }
  *blocks_out = blocks;
  *t_last_out = t_last;
}

// Adds n to *addr once per distinct address among the active lanes that
// pass want (the counters are few and every tile hits one of them: one
// atomic per tile serialises on the busiest address).  Returns, to every
// wanting lane, the counter's old value plus the count of lanes below it
// with the same address: a distinct slot per lane.
__device__ __forceinline__ uint32_t warp_add(uint32_t* addr, bool want) {
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned long long key = want ? reinterpret_cast<unsigned long long>(addr) : ~0ull;
  const uint32_t peers = __match_any_sync(0xffffffffu, key);
  const uint32_t leader = __ffs(peers) - 1;
  uint32_t base = 0;
  if (want && lane == leader) base = atomicAdd(addr, static_cast<uint32_t>(__popc(peers)));
  base = __shfl_sync(0xffffffffu, base, leader);
  return base + static_cast<uint32_t>(__popc(peers & ((1u << lane) - 1u)));
}

// kOrderLanes lanes per tile (a warp holds whole tiles): the tile's cost,
// EMPTY steps before its last non-EMPTY block plus 6 per such block, gives
// its class; the first lane keys the tile and counts it.
__global__ void k_tile_cost(const __grid_constant__ OrderTable t) {
  const uint64_t th = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint32_t lane = static_cast<uint32_t>(th % kOrderLanes);
  const uint64_t tile = th / kOrderLanes;
  const bool live = tile < t.total_tiles;  // every lane takes part in the shuffles
  const uint32_t gi = live ? static_cast<uint32_t>(tile) : 0u;
  const uint32_t vi = order_view_of(t, gi);
  const OrderView& v = t.v[vi];
  const uint32_t li = gi - v.tile_base;
  const uint32_t row = li / v.tiles_x, col = li % v.tiles_x;
  uint32_t blocks = 0;
  float t_last = 0.0f;
  if (live) tile_walk(t, t.segs[v.seg], col, row, lane, &blocks, &t_last);
  for (uint32_t m = kOrderLanes / 2; m; m >>= 1) {
    blocks += __shfl_xor_sync(0xffffffffu, blocks, m, kOrderLanes);
    t_last = fmaxf(t_last, __shfl_xor_sync(0xffffffffu, t_last, m, kOrderLanes));
  }
  const bool first = live && lane == 0;
  const float cost = t_last / t.step + 6.0f * static_cast<float>(blocks);
  const uint32_t cls = kOrderBuckets - 1 - min(kOrderBuckets - 1, static_cast<uint32_t>(cost * (1.0f / 16.0f)));
  uint32_t g = 0;
  while (g + 1 < v.n_groups && row >= v.group_row[g + 1]) ++g;
  const uint32_t key = g * kOrderBuckets + cls;
  if (first) t.key[gi] = key;
  warp_add(t.count + static_cast<size_t>(vi) * 2 * kOrderKeys + key, first);
}

// One thread per view: exclusive prefix of the counters (groups in order,
// heaviest class first within each), so group g's tiles land in its own rows.
__global__ void k_tile_scan(const __grid_constant__ OrderTable t) {
  const uint32_t vi = blockIdx.x * blockDim.x + threadIdx.x;
  if (vi >= t.n_views) return;
  const uint32_t* cnt = t.count + static_cast<size_t>(vi) * 2 * kOrderKeys;
  uint32_t* off = t.count + static_cast<size_t>(vi) * 2 * kOrderKeys + kOrderKeys;
  uint32_t s = 0;
  for (uint32_t k = 0; k < t.v[vi].n_groups * kOrderBuckets; ++k) {
    off[k] = s;
    s += cnt[k];
  }
}

__global__ void k_tile_place(const __grid_constant__ OrderTable t) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = tid < t.total_tiles;  // every lane takes part in warp_add
  const uint32_t gi = live ? tid : 0u;
  const uint32_t vi = order_view_of(t, gi);
  const OrderView& v = t.v[vi];
  uint32_t* off = t.count + static_cast<size_t>(vi) * 2 * kOrderKeys + kOrderKeys;
  const uint32_t pos = warp_add(off + (live ? t.key[gi] : 0u), live);
  if (live) t.perm[v.tile_base + pos] = gi - v.tile_base;
}

}  // namespace detail

rkf_status tile_order_prepare(Ctx* c, std::vector<Segment>& segs, uint32_t tile_w, uint32_t tile_h,
                              const uint32_t* band_rows, uint32_t n_bands, OrderTable* tbl, bool* any) {
  std::memset(tbl, 0, sizeof(*tbl));
  *any = false;
  if (!tile_w) tile_w = 8;
  if (!tile_h) tile_h = 4;
  if (band_rows && (n_bands == 0 || n_bands > kOrderMaxGroups))
    return fail(RKF_INVALID_ARG, "tile order: bad band count");
  tbl->tile_w = tile_w;
  tbl->tile_h = tile_h;
  uint64_t total = 0;
  for (size_t i = 0; i < segs.size() && tbl->n_views < kOrderMaxViews; ++i) {
    const Segment& sg = segs[i];
    if (sg.kind != 0) continue;
    const uint32_t rows = (sg.h + tile_h - 1) / tile_h;
    OrderView& v = tbl->v[tbl->n_views++];
    v.seg = static_cast<uint32_t>(i);
    v.tile_base = static_cast<uint32_t>(total);
    v.tiles_x = sg.tiles_x;
    v.n_tiles = sg.tiles_x * rows;
    if (band_rows) {
      v.n_groups = n_bands;
      for (uint32_t b = 0; b <= n_bands; ++b) v.group_row[b] = band_rows[b];
    } else {
      v.n_groups = 1;
      v.group_row[0] = 0;
      v.group_row[1] = rows;
    }
    total += v.n_tiles;
  }
  if (tbl->n_views == 0 || total == 0) return RKF_OK;
  if (total > (1ull << 31)) return fail(RKF_INVALID_ARG, "tile order: too many tiles");
  tbl->total_tiles = static_cast<uint32_t>(total);
  const size_t tiles_b = (total * 4 + 255) & ~static_cast<size_t>(255);
  const size_t count_b = static_cast<size_t>(tbl->n_views) * 2 * detail::kOrderKeys * 4;
  const size_t need = 2 * tiles_b + count_b;
  if (c->order_buf.bytes < need) {
    const rkf_status st = c->order_buf.alloc(need + need / 4);
    if (st != RKF_OK) return st;
  }
  char* base = c->order_buf.as<char>();
  tbl->key = reinterpret_cast<uint32_t*>(base);
  tbl->perm = reinterpret_cast<uint32_t*>(base + tiles_b);
  tbl->count = reinterpret_cast<uint32_t*>(base + 2 * tiles_b);
  for (uint32_t i = 0; i < tbl->n_views; ++i) segs[tbl->v[i].seg].tile_perm = tbl->perm + tbl->v[i].tile_base;
  *any = true;
  return RKF_OK;
}

rkf_status tile_order_enqueue(Ctx* c, OrderTable& tbl, const Segment* dev_segs, const ObjDev& o,
                              const uint8_t* field, float reach, float step, cudaStream_t st) {
  (void)c;
  tbl.o = o;
  tbl.field = field;
  tbl.segs = dev_segs;
  tbl.reach = reach;
  tbl.step = step;
  RKF_CUDA_TRY(cudaMemsetAsync(tbl.count, 0,
                               static_cast<size_t>(tbl.n_views) * 2 * detail::kOrderKeys * 4, st));
  const unsigned blocks = (tbl.total_tiles + 255) / 256;
  const unsigned cost_blocks =
      static_cast<unsigned>((static_cast<uint64_t>(tbl.total_tiles) * detail::kOrderLanes + 255) / 256);
  detail::k_tile_cost<<<cost_blocks, 256, 0, st>>>(tbl);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  detail::k_tile_scan<<<1, 64, 0, st>>>(tbl);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  detail::k_tile_place<<<blocks, 256, 0, st>>>(tbl);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  return RKF_OK;
}

}  // namespace rkf
