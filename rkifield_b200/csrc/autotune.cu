// autotune.cu — pick the persistent march's launch tuning for a workload.
//
// The batched march has nine knobs that change speed but never results:
// the ray-tile shape that orders a view's work ids (the spatial coherence of
// the rays a warp holds), the compaction interval (march iterations between
// lane refills), the step budget (empty-space steps a lane runs before its
// warp re-converges), the refill threshold (idle lanes that make a warp
// refill), where a lane probes its next EMPTY cube (inside a run or between
// runs), the block size, whether it runs EMPTY runs at all, whether views
// hand out their heaviest ray tiles first and whether the warps of the
// launch's tail share their EMPTY runs.  rkf_autotune times candidates on
// the caller's sample of the work with CUDA events: every tile x interval x
// block size at the default budget and threshold, then the heaviest-first
// tile order, then every budget, then every threshold, then the other probe
// placement, then warp-shared EMPTY runs in the launch's tail, then the march
// without EMPTY runs, each at the best so far.
// Each timed launch starts with the L2 cache flushed (a write of twice its
// size, outside the timed events), as a frame does after other work: with
// the index left in L2 by the previous trial, the knobs that cut DRAM
// traffic (tile shape, tile order) would look worth less than they are.
// The fastest is kept in the context, where rkf_march and rkf_march_batch
// use it.
#include <cfloat>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "march.h"

using namespace rkf;

extern "C" rkf_status rkf_autotune(rkf_ctx* ctx, const rkf_view* views, uint32_t n_views,
                                   const rkf_ray_batch* batches, uint32_t n_batches,
                                   const rkf_march_params* p, rkf_batch_tuning* out) {
  if (!ctx || !p || (n_views && !views) || (n_batches && !batches))
    return fail(RKF_INVALID_ARG, "rkf_autotune: null argument");
  if (n_views + n_batches == 0) return fail(RKF_INVALID_ARG, "rkf_autotune: no work to tune on");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  static const uint32_t tiles[][2] = {{4, 8}, {8, 4}, {16, 2}};
  static const uint32_t intervals[] = {16, 32, 64, 128};
  static const uint32_t threads[] = {128, 256};
  static const uint32_t budgets[] = {16, 64};
  static const uint32_t refills[] = {8, 16, 24};
  cudaEvent_t e0, e1;
  RKF_CUDA_TRY(cudaEventCreate(&e0));
  RKF_CUDA_TRY(cudaEventCreate(&e1));
  rkf_batch_tuning best = c->tuning;
  float best_ms = FLT_MAX;
  rkf_status st = RKF_OK;
  // the flush buffer lives for this call only (no flush when the device has
  // no room for it)
  int l2_bytes = 0;
  cudaDeviceGetAttribute(&l2_bytes, cudaDevAttrL2CacheSize, c->device);
  DevBuf flush;
  if (l2_bytes > 0 && flush.alloc(2 * static_cast<size_t>(l2_bytes)) != RKF_OK) {
    flush.release();
    cudaGetLastError();
    set_error("");  // not an error of this call: it tunes without the flush
  }
  // one untimed launch, then the best of two timed ones, each after a flush
  auto trial = [&](const rkf_batch_tuning& tu) {
    st = rkf_march_batch_async(ctx, views, n_views, batches, n_batches, p, &tu, nullptr);
    if (st != RKF_OK) return;
    float ms = FLT_MAX;
    for (int r = 0; r < 2; ++r) {
      if (flush.p && cudaMemsetAsync(flush.p, r + 1, flush.bytes, c->stream) != cudaSuccess) {
        st = fail(RKF_CUDA_ERROR, "rkf_autotune: L2 flush failed");
        return;
      }
      cudaEventRecord(e0, c->stream);
      st = rkf_march_batch_async(ctx, views, n_views, batches, n_batches, p, &tu, nullptr);
      if (st != RKF_OK) return;
      cudaEventRecord(e1, c->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        st = fail(RKF_CUDA_ERROR, "rkf_autotune: launch failed");
        return;
      }
      float m = 0.0f;
      cudaEventElapsedTime(&m, e0, e1);
      if (m < ms) ms = m;
    }
    if (ms < best_ms) {
      best_ms = ms;
      best = tu;
    }
  };
  for (const auto& tl : tiles)
    for (uint32_t iv : intervals)
      for (uint32_t th : threads)
        if (st == RKF_OK) trial(rkf_batch_tuning{tl[0], tl[1], 32, iv, 0, th, 32, 0, 0});
  // heaviest tiles first (views on the empty-space path), before the
  // finer knobs so that they are tuned with the order that wins
  if (st == RKF_OK && n_views) {
    rkf_batch_tuning tu = best;
    tu.order_tiles = 1;
    trial(tu);
  }
  const rkf_batch_tuning base = best;
  for (uint32_t b : budgets) {
    if (st != RKF_OK) break;
    rkf_batch_tuning tu = base;
    tu.step_budget = b;
    trial(tu);
  }
  const rkf_batch_tuning base2 = best;
  for (uint32_t r : refills) {
    if (st != RKF_OK) break;
    rkf_batch_tuning tu = base2;
    tu.refill_idle = r;
    trial(tu);
  }
  if (st == RKF_OK) {
    rkf_batch_tuning tu = best;
    tu.probe_in_run = 1;
    trial(tu);
  }
  // the warp-shared EMPTY runs of the launch's tail
  if (st == RKF_OK) {
    rkf_batch_tuning tu = best;
    tu.tail_share = 2;
    trial(tu);
  }
  // where EMPTY runs do not pay (a camera outside a dense grid: short runs,
  // probes that mostly fail), the full sampler alone is faster
  if (st == RKF_OK) {
    rkf_batch_tuning tu = best;
    tu.no_empty_path = 1;
    trial(tu);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != RKF_OK) return st;
  c->tuning = best;
  c->tuned = true;
  if (out) *out = best;
  return RKF_OK;
}

extern "C" rkf_status rkf_tuning_set(rkf_ctx* ctx, const rkf_batch_tuning* tuning) {
  if (!ctx || !tuning) return fail(RKF_INVALID_ARG, "rkf_tuning_set: null argument");
  const rkf_batch_tuning& tu = *tuning;
  const uint32_t threads = tu.threads_per_block ? tu.threads_per_block : 256;
  if ((tu.tile_w == 0) != (tu.tile_h == 0) || tu.tile_w * tu.tile_h > 4096 || threads > 256 || threads % 32 ||
      tu.refill_idle > 32 || tu.probe_in_run > 1 || tu.no_empty_path > 1 || tu.order_tiles > 1 ||
      tu.tail_share > 32)
    return fail(RKF_INVALID_ARG, "rkf_tuning_set: bad tuning");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_tuning_set: the context is serving");
  c->tuning = tu;
  c->tuned = true;
  return RKF_OK;
}

extern "C" rkf_status rkf_tuning_get(rkf_ctx* ctx, rkf_batch_tuning* out) {
  if (!ctx || !out) return fail(RKF_INVALID_ARG, "rkf_tuning_get: null argument");
  *out = reinterpret_cast<Ctx*>(ctx)->tuning;
  return RKF_OK;
}
