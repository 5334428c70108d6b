// ctx.h — host-side state of an rkf_ctx (one device, one resident scene).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rkf_cuda.h"
#include "device_common.cuh"

namespace rkf {

// Thread-local message for rkf_last_error().
void set_error(const std::string& msg);
rkf_status fail(rkf_status st, const std::string& msg);

#define RKF_CUDA_TRY(expr)                                                        \
  do {                                                                            \
    cudaError_t e_ = (expr);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      return ::rkf::fail(e_ == cudaErrorMemoryAllocation ? RKF_OOM : RKF_CUDA_ERROR, \
                         std::string(#expr) + ": " + cudaGetErrorString(e_));    \
    }                                                                             \
  } while (0)

// A device allocation owned by the context.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf();
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  rkf_status alloc(size_t n);  // frees any previous allocation
  void release();
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

// Allocation hook used by every context allocation (tests replace it to
// simulate an out-of-memory device without touching the GPU).
using alloc_hook_fn = cudaError_t (*)(void** p, size_t bytes);
extern alloc_hook_fn g_alloc_hook;

// Runs its function when the scope ends unless dismissed: undoes a
// multi-step change of the context that failed part-way.
template <class F>
struct Rollback {
  F f;
  bool armed = true;
  explicit Rollback(F fn) : f(fn) {}
  Rollback(const Rollback&) = delete;
  Rollback& operator=(const Rollback&) = delete;
  ~Rollback() {
    if (armed) f();
  }
  void dismiss() { armed = false; }
};

struct ServeState;  // serve.cu

struct Ctx {
  int device = 0;
  rkf_config cfg{};
  cudaStream_t stream = nullptr;
  int sm_count = 0;

  // pool planes
  uint32_t capacity = 0;
  DevBuf dist_f16, dist_f32, dist_u8, brick_step, mat, blend, aos;
  std::vector<uint32_t> free_slots;  // LIFO, low slots on top (brick_pool.rs:37-42)
  uint32_t used_slots = 0;

  // reference flat maps (kept for the plain march when imported)
  DevBuf flat_maps;
  uint64_t flat_len = 0;
  std::vector<uint32_t> flat_host;  // host copy used to build the index

  // two-level index
  DevBuf top;
  uint64_t top_len = 0;
  DevBuf empty_dist;  // u8 per top cell: empty-space distance field (empty_dist.h)
  DevBuf leaves;
  uint32_t n_leaves = 0, leaf_cap = 0;
  std::vector<uint32_t> free_leaves;  // leaf numbers below n_leaves that no epoch references
  bool leaves_frozen = false;  // set while serving: the leaf buffer must not move

  // tiled strategy (tiled.h): coarse field (rebuilt when epoch changes) and tile lists
  DevBuf coarse_tex, tile_buf;
  // empty-space field of the tiled strategy for a single object: EMPTY
  // blocks that no coarse skip can reach (tiled.cu); built for tiled_epoch
  DevBuf tiled_empty_dist;
  uint64_t tiled_epoch = ~0ull;
  int last_variant = -1;  // kernel variant of the last persistent march launch
  float coarse_origin[3] = {0.0f, 0.0f, 0.0f};
  uint32_t coarse_dims[3] = {0, 0, 0};
  uint64_t coarse_epoch = ~0ull;

  // BVH of the BVH strategy (bvh.cu): rkf_bvh_node records, root first, and
  // per node the walk's next node and whether it descends (bvh.cu)
  DevBuf bvh, bvh_next;
  uint32_t bvh_n = 0;
  bool bvh_one_leaf0 = false;  // the tree is one leaf naming object 0
  std::vector<rkf_bvh_node> bvh_host;  // the imported tree, root first
  std::vector<uint32_t> bvh_next_host;  // its walk links (bvh_next)

  // objects
  std::vector<rkf_gpu_object> objects;
  std::vector<ObjDev> objdev_host;
  DevBuf objdev;

  uint64_t epoch = 0;
  rkf_world_pos origin{};  // WorldPosition the scene's f32 world space is relative to

  // scratch reused by march calls (host-pointer outputs staged here)
  DevBuf stage;
  // host-output views: band b marches on band_stream[b % 2] (so a band's
  // launch fills the SMs its predecessor's last rays leave idle), and its
  // rows go back on copy_stream once band_ev[b] has completed
  static constexpr int kMaxBands = 8;
  cudaStream_t copy_stream = nullptr;
  cudaStream_t band_stream = nullptr;  // the second band stream; the first is `stream`
  cudaEvent_t band_ev[kMaxBands] = {};
  cudaEvent_t segs_ev = nullptr;
  DevBuf order_buf;  // heaviest-first tile order of views (tile_order.h)
  DevBuf counters;   // work counters of the persistent kernels
  DevBuf seg_buf;    // segment table of the persistent kernel

  // batching
  rkf_batch_tuning tuning{};
  bool tuned = false;

  ServeState* serve = nullptr;  // owned; created by rkf_serve_start

  // launch accounting (rkf_testing_launch_stats): every kernel the context
  // launches is counted; while march timing is on, each persistent march
  // launch is bracketed by a pair of events on its stream
  static constexpr uint32_t kMaxTimed = 4096;
  std::atomic<uint64_t> launches{0};
  bool time_march = false;
  std::vector<cudaEvent_t> march_ev;  // start, end of each timed launch
  uint32_t march_timed = 0;           // launches timed since timing was switched on
  void counted(uint32_t n = 1) { launches.fetch_add(n, std::memory_order_relaxed); }
  // records the start (end = false) or end event of a timed march launch
  rkf_status march_event(cudaStream_t st, bool end);

  SceneDev scene_dev() const;
  uint32_t obj_count() const { return static_cast<uint32_t>(objects.size()); }
  rkf_status upload_objects();
  rkf_status verify_exact_div();
  std::map<uint32_t, std::pair<uint32_t, uint32_t>> div_checked;  // vs bits -> verified bit range
  rkf_status ensure_leaf_capacity(uint32_t need);
  rkf_status stage_bytes(size_t bytes);
};

// Builds ObjDev (precomputed per-object constants) from a GpuObject.
ObjDev make_objdev(const rkf_gpu_object& o, uint32_t top_off, uint32_t has_flat);

// Marches (march_fast.cu / march_plain.cu)
struct Segment;
rkf_status launch_plain(Ctx* c, const rkf_camera* cam, const rkf_march_params* p, uint32_t w,
                        uint32_t h, const rkf_gbuffer& dev_out, cudaStream_t st);

}  // namespace rkf
