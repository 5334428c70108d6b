// tile_order.h — heaviest-first order of the ray tiles of views (tile_order.cu).
#pragma once

#include <vector>

#include "march.h"

namespace rkf {

constexpr uint32_t kOrderMaxViews = 64;   // views of one launch that are ordered
constexpr uint32_t kOrderMaxGroups = 8;   // groups of tile rows ordered separately
constexpr uint32_t kOrderBuckets = 64;    // cost classes of the counting sort

struct OrderView {
  uint32_t seg;         // the view's segment in the launch's table
  uint32_t tile_base;   // first entry of the view in the order buffer
  uint32_t n_tiles, tiles_x;
  uint32_t n_groups;    // rows [group_row[g], group_row[g+1]) are ordered among themselves
  uint32_t group_row[kOrderMaxGroups + 1];
};

struct OrderTable {
  uint32_t n_views, total_tiles, tile_w, tile_h;
  float reach;          // distance the estimate walks along a ray
  float step;           // length of one EMPTY step
  uint32_t _pad[2];
  ObjDev o;             // the object of the empty-space path
  const uint8_t* field; // its empty-space distance field
  const Segment* segs;  // the launch's segment table (device)
  uint32_t* key;        // per tile: group * kOrderBuckets + cost class (descending)
  uint32_t* count;      // per view: kOrderMaxGroups * kOrderBuckets counters, then as many offsets
  uint32_t* perm;       // per tile: the tile handed out at that position
  OrderView v[kOrderMaxViews];
};

// Plans the order of the view segments in segs (at most kOrderMaxViews are
// ordered): points their tile_perm at slices of the context's order buffer,
// grown as needed.  band_rows (n_bands + 1 tile-row boundaries, or null for
// one group per view) splits every view into groups whose tiles stay within
// the group's work ids.  *any = false when there is nothing to order.
rkf_status tile_order_prepare(Ctx* c, std::vector<Segment>& segs, uint32_t tile_w, uint32_t tile_h,
                              const uint32_t* band_rows, uint32_t n_bands, OrderTable* tbl, bool* any);

// Enqueues on st the cost estimate of every planned tile and the counting
// sort that writes the permutations; dev_segs holds the launch's segment table.
rkf_status tile_order_enqueue(Ctx* c, OrderTable& tbl, const Segment* dev_segs, const ObjDev& o,
                              const uint8_t* field, float reach, float step, cudaStream_t st);

}  // namespace rkf
