// march.h — work segments of the persistent march and its launchers.
#pragma once

#include <vector>

#include "ctx.h"

namespace rkf {

constexpr uint32_t kMaxObjectsFast = 32;

// One unit of batched work: a view (kind 0, primary rays over w x h pixels
// walked in tile order) or a ray batch (kind 1).  Device pointers only.
struct Segment {
  uint64_t first;     // first global work id of the segment
  uint64_t n_ids;     // work ids the segment spans
  uint32_t kind, mode;
  uint32_t w, h, tiles_x, tile_off;  // tile_off: first object tile of the view (tiled strategy)
  float pos[3], fwd[3], right[3], up[3], jitter[2];
  float coarse_ocr[3];                // coarse field origin relative to the camera (tiled strategy)
  uint32_t _pad;
  const uint32_t* tile_perm;          // view: the tile handed out at each position (null: row order)
  float prev_vp[16];
  const float* origins;
  const float* dirs;
  const float* tmax;
  float* t;
  float* normal;
  uint32_t* slot;
  uint16_t* material;
  uint16_t* flags;
  float* position;
  uint32_t* packed;
  float* motion;
};

Segment view_segment(const rkf_camera* cam, uint32_t w, uint32_t h, uint32_t tile_w,
                     uint32_t tile_h, const rkf_gbuffer& out);
Segment ray_segment(const float* o, const float* d, const float* tmax, uint32_t n, uint32_t mode,
                    const rkf_hits& out);
// Marches work ids id0 .. id0 + total - 1 of the segments (id0 > 0: a part
// of the work, e.g. one band of tile rows of a view; not with the tiled
// strategy, whose tile lists cover whole views).  segs_resident: seg_buf
// already holds this segment table (a later part of the same work), so it
// is not uploaded again.
rkf_status launch_persistent(Ctx* c, const std::vector<Segment>& segs, uint64_t total,
                             const rkf_march_params* p, const rkf_batch_tuning& tu,
                             cudaStream_t st, DevBuf* seg_buf, unsigned long long* counter,
                             uint64_t id0 = 0, bool segs_resident = false);
// Same launch as launch_persistent, with the segment table and work counter
// in caller-provided device memory (it allocates nothing).  segs_uploaded:
// the caller has already queued the copy of the table into dev_segs on st
// (from page-locked memory, so that enqueueing never waits on the stream).
// multi_empty: a scene of one voxelized object beside analytic objects
// marches the multi-object empty-space variant (else the plain multi-object
// kernel).
// The refusals of launch_persistent_scratch (strategy, object count, block
// size), without enqueueing anything.
rkf_status check_persistent_scratch(const Ctx* c, const rkf_march_params* p, const rkf_batch_tuning& tu);
rkf_status launch_persistent_scratch(Ctx* c, const Segment* segs_host, uint32_t nseg, uint64_t total,
                                     const rkf_march_params* p, const rkf_batch_tuning& tu,
                                     cudaStream_t st, Segment* dev_segs, unsigned long long* dev_counter,
                                     bool segs_uploaded = false, bool multi_empty = false);
// Whether a launch over this context's objects with these parameters marches
// the empty-space path (the condition for ordering its views' tiles), and
// the object whose empty-space field it reads.
bool empty_order_source(const Ctx* c, const rkf_march_params* p, const rkf_batch_tuning& tu, ObjDev* o);
// Distance the tile-order estimate walks along a ray.
float order_reach(const ObjDev& o, const rkf_march_params* p);
rkf_status launch_trace_plain(Ctx* c, const float* o, const float* d, const float* tmax, uint32_t n,
                              uint32_t mode, const rkf_march_params* p, const rkf_hits& out,
                              cudaStream_t st);
rkf_status launch_ao(Ctx* c, const float* pos, const float* nrm, uint32_t n, float* ao, cudaStream_t st);
rkf_status launch_query(Ctx* c, const float* pts, uint32_t n, float* d, float* g, uint16_t* m,
                        cudaStream_t st);

}  // namespace rkf
