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
// a few steps per such block.  A counting sort (64 cost classes, heaviest
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

// EMPTY steps a tile's centre ray is expected to take (see above).
__device__ float tile_cost(const OrderTable& t, const Segment& sg, uint32_t col, uint32_t row) {
  const ObjDev& o = t.o;
  const uint32_t px = min(col * t.tile_w + t.tile_w / 2, sg.w - 1);
  const uint32_t py = min(row * t.tile_h + t.tile_h / 2, sg.h - 1);
  const float u = (static_cast<float>(px) + 0.5f + sg.jitter[0]) / static_cast<float>(sg.w);
  const float v = (static_cast<float>(py) + 0.5f + sg.jitter[1]) / static_cast<float>(sg.h);
  const float nx = 2.0f * u - 1.0f, ny = 1.0f - 2.0f * v;
  float d[3];
  for (int a = 0; a < 3; ++a) d[a] = sg.fwd[a] + sg.right[a] * nx + sg.up[a] * ny;
  const float il = rsqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  // grid voxel coordinate along the ray: g(t) = a0 + a1 * t (t in metres)
  float a0[3], a1[3];
  float t0 = 0.0f, t1 = t.reach;
  for (int a = 0; a < 3; ++a) {
    a0[a] = (sg.pos[a] + o.m[12 + a] + o.half_gs[a]) * o.rcp_vs - 0.5f;
    a1[a] = d[a] * il * o.rcp_vs;
    const float tv = static_cast<float>(o.tv[a]);
    if (a1[a] != 0.0f) {
      const float ta = -a0[a] / a1[a], tb = (tv - a0[a]) / a1[a];
      t0 = fmaxf(t0, fminf(ta, tb));
      t1 = fminf(t1, fmaxf(ta, tb));
    } else if (!(a0[a] >= 0.0f && a0[a] < tv)) {
      t1 = -1.0f;
    }
  }
  if (!(t0 < t1)) return 0.0f;  // the ray misses the grid
  const float eps = 0.01f * o.vs;
  float tt = t0 + eps, t_last = 0.0f;
  uint32_t blocks = 0;
  for (int it = 0; it < 128 && tt < t1; ++it) {
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
      if (a1[a] > 0.0f) te = fminf(te, (hi - a0[a]) / a1[a]);
      else if (a1[a] < 0.0f) te = fminf(te, (lo - a0[a]) / a1[a]);
    }
    if (r == 0) {
      ++blocks;
      t_last = tt;
    }
    tt = fmaxf(te, tt) + eps;
  }
  return t_last / t.step + 6.0f * static_cast<float>(blocks);
}

__global__ void k_tile_cost(const __grid_constant__ OrderTable t) {
  const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= t.total_tiles) return;
  const uint32_t vi = order_view_of(t, gi);
  const OrderView& v = t.v[vi];
  const uint32_t li = gi - v.tile_base;
  const uint32_t row = li / v.tiles_x, col = li % v.tiles_x;
  const float cost = tile_cost(t, t.segs[v.seg], col, row);
  const uint32_t cls = kOrderBuckets - 1 - min(kOrderBuckets - 1, static_cast<uint32_t>(cost * (1.0f / 16.0f)));
  uint32_t g = 0;
  while (g + 1 < v.n_groups && row >= v.group_row[g + 1]) ++g;
  const uint32_t key = g * kOrderBuckets + cls;
  t.key[gi] = key;
  atomicAdd(t.count + static_cast<size_t>(vi) * 2 * kOrderKeys + key, 1u);
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
  const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= t.total_tiles) return;
  const uint32_t vi = order_view_of(t, gi);
  const OrderView& v = t.v[vi];
  uint32_t* off = t.count + static_cast<size_t>(vi) * 2 * kOrderKeys + kOrderKeys;
  const uint32_t pos = atomicAdd(off + t.key[gi], 1u);
  t.perm[v.tile_base + pos] = gi - v.tile_base;
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
  detail::k_tile_cost<<<blocks, 256, 0, st>>>(tbl);
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
