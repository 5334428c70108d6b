// api.cu — public march / trace / query / batch entry points.
//
// Host-pointer outputs are staged in a context-owned device buffer and copied
// back on the context stream; device-pointer outputs are written in place.
// A large view with host outputs is marched in bands of tile rows, each
// band's rows copied back on a second stream while the next band marches.
#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstring>
#include <vector>

#include "../../include/rkf_cuda_testing.h"
#include "ctx.h"
#include "march.h"
#include "tile_order.h"

using namespace rkf;

namespace detail {

// Band count of host-output views: < 0 chooses by size (rkf_testing_*).
std::atomic<int> g_host_bands{-1};

// Whether every given host plane is page-locked: only then do the banded
// copies run asynchronously (a copy into pageable memory holds the host until
// it is done, which would hold back the next band's launch).
bool all_page_locked(const rkf_gbuffer& g) {
  const void* planes[] = {g.t, g.normal, g.slot, g.material, g.flags, g.position, g.packed_material, g.motion};
  for (const void* p : planes) {
    if (!p) continue;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (a.type != cudaMemoryTypeHost) return false;
  }
  return true;
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Device staging for a G-buffer of n elements; fills dev with device pointers.
rkf_status stage_gbuffer(Ctx* c, const rkf_gbuffer& host, uint64_t n, rkf_gbuffer* dev) {
  const size_t sz[8] = {n * 4, n * 12, n * 4, n * 2, n * 2, host.position ? n * 16 : 0,
                        host.packed_material ? n * 4 : 0, host.motion ? n * 16 : 0};
  size_t total = 0;
  for (size_t s : sz) total += align256(s);
  rkf_status st = c->stage_bytes(total);
  if (st != RKF_OK) return st;
  char* b = c->stage.as<char>();
  void* ptrs[8];
  for (int i = 0; i < 8; ++i) {
    ptrs[i] = sz[i] ? b : nullptr;
    b += align256(sz[i]);
  }
  *dev = host;
  dev->t = static_cast<float*>(ptrs[0]);
  dev->normal = static_cast<float*>(ptrs[1]);
  dev->slot = static_cast<uint32_t*>(ptrs[2]);
  dev->material = static_cast<uint16_t*>(ptrs[3]);
  dev->flags = static_cast<uint16_t*>(ptrs[4]);
  dev->position = static_cast<float*>(ptrs[5]);
  dev->packed_material = static_cast<uint32_t*>(ptrs[6]);
  dev->motion = static_cast<float*>(ptrs[7]);
  dev->mem = RKF_MEM_DEVICE;
  return RKF_OK;
}

rkf_status copy_back_gbuffer(Ctx* c, const rkf_gbuffer& host, const rkf_gbuffer& dev, uint64_t n) {
  auto cp = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    if (!dst || !src || !bytes) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
  };
  RKF_CUDA_TRY(cp(host.t, dev.t, n * 4));
  RKF_CUDA_TRY(cp(host.normal, dev.normal, n * 12));
  RKF_CUDA_TRY(cp(host.slot, dev.slot, n * 4));
  RKF_CUDA_TRY(cp(host.material, dev.material, n * 2));
  RKF_CUDA_TRY(cp(host.flags, dev.flags, n * 2));
  RKF_CUDA_TRY(cp(host.position, dev.position, n * 16));
  RKF_CUDA_TRY(cp(host.packed_material, dev.packed_material, n * 4));
  RKF_CUDA_TRY(cp(host.motion, dev.motion, n * 16));
  return RKF_OK;
}

// Bands of a host-output view of n rays: band b's copy overlaps the march
// of the bands after it; only the last band's copy stays exposed.
int host_bands(uint64_t n) {
  const int forced = g_host_bands.load();
  if (forced >= 0) return std::min(std::max(forced, 1), Ctx::kMaxBands);
  return n >= (1u << 20) ? 3 : n >= (1u << 18) ? 2 : 1;  // measured best on a 1080p view
}

// rkf_march into host planes, band by band: tile rows [r0, r1) of the view
// are the work ids [r0, r1) x tiles_x x tile area and write pixel rows
// [r0 * tile_h, min(r1 * tile_h, h)), contiguous in every plane.  Bands
// weigh 2 : 2 : ... : 1, so the last (exposed) copy is the smallest.  Bands
// alternate between two streams with a work counter each: the launches do
// not wait on one another, so band b + 1's blocks take the SMs that band
// b's blocks free while its last rays finish.
rkf_status march_host_banded(Ctx* c, const rkf_camera* cam, const rkf_march_params* p, uint32_t w,
                             uint32_t h, const rkf_gbuffer& host, int bands) {
  const uint64_t n = static_cast<uint64_t>(w) * h;
  rkf_gbuffer dev;
  rkf_status st = stage_gbuffer(c, host, n, &dev);
  if (st != RKF_OK) return st;
  for (cudaStream_t* s : {&c->copy_stream, &c->band_stream})
    if (!*s) RKF_CUDA_TRY(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
  for (int b = 0; b < bands; ++b)
    if (!c->band_ev[b]) RKF_CUDA_TRY(cudaEventCreateWithFlags(&c->band_ev[b], cudaEventDisableTiming));
  if (!c->segs_ev) RKF_CUDA_TRY(cudaEventCreateWithFlags(&c->segs_ev, cudaEventDisableTiming));
  const rkf_batch_tuning& tu = c->tuning;
  std::vector<Segment> segs{view_segment(cam, w, h, tu.tile_w, tu.tile_h, dev)};
  segs[0].first = 0;
  const uint32_t tile_w = tu.tile_w ? tu.tile_w : 8, tile_h = tu.tile_h ? tu.tile_h : 4;
  const uint64_t row_ids = static_cast<uint64_t>(segs[0].tiles_x) * tile_w * tile_h;
  const uint32_t rows = (h + tile_h - 1) / tile_h;
  const uint32_t weight = 2u * static_cast<uint32_t>(bands) - 1u;
  // tile rows of each band: band b marches rows [band_rows[b], band_rows[b+1])
  std::vector<uint32_t> band_rows{0};
  for (int b = 0; b < bands && band_rows.back() < rows; ++b) {
    const uint32_t r1 = b == bands - 1 ? rows
                                       : std::min(rows, static_cast<uint32_t>(
                                                            (static_cast<uint64_t>(rows) * 2u * (b + 1)) / weight));
    if (r1 > band_rows.back()) band_rows.push_back(r1);
  }
  // heaviest-first order within each band, planned once for all bands
  ObjDev order_obj;
  OrderTable order_tbl;
  bool ordered = false;
  if (tu.order_tiles && p->strategy != RKF_STRATEGY_TILED && empty_order_source(c, p, tu, &order_obj) &&
      (st = tile_order_prepare(c, segs, tile_w, tile_h, band_rows.data(),
                               static_cast<uint32_t>(band_rows.size() - 1), &order_tbl, &ordered)) != RKF_OK)
    return st;
  const size_t sb = sizeof(Segment);
  if (c->seg_buf.bytes < sb && (st = c->seg_buf.alloc(sb)) != RKF_OK) return st;
  RKF_CUDA_TRY(cudaMemcpyAsync(c->seg_buf.p, segs.data(), sb, cudaMemcpyHostToDevice, c->stream));
  if (ordered &&
      (st = tile_order_enqueue(c, order_tbl, c->seg_buf.as<Segment>(), order_obj, c->empty_dist.as<uint8_t>(),
                               order_reach(order_obj, p), order_obj.be * order_obj.min_scale, c->stream)) != RKF_OK)
    return st;
  RKF_CUDA_TRY(cudaEventRecord(c->segs_ev, c->stream));
  RKF_CUDA_TRY(cudaStreamWaitEvent(c->band_stream, c->segs_ev, 0));
  // on an error, work already queued must finish before the caller's
  // buffers are handed back
  struct Drain {
    Ctx* c;
    ~Drain() {
      cudaStreamSynchronize(c->copy_stream);
      cudaStreamSynchronize(c->band_stream);
      cudaStreamSynchronize(c->stream);
    }
  } drain{c};
  // one counter per band, 64 bytes apart, past the counters other launches use
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(c->counters.as<char>() + 1024);
  for (size_t b = 0; b + 1 < band_rows.size(); ++b) {
    const uint32_t r0 = band_rows[b], r1 = band_rows[b + 1];
    cudaStream_t bs = (b & 1) ? c->band_stream : c->stream;
    st = launch_persistent(c, segs, (r1 - r0) * row_ids, p, tu, bs, &c->seg_buf, counters + 8 * b,
                           r0 * row_ids, true);
    if (st != RKF_OK) return st;
    RKF_CUDA_TRY(cudaEventRecord(c->band_ev[b], bs));
    RKF_CUDA_TRY(cudaStreamWaitEvent(c->copy_stream, c->band_ev[b], 0));
    const uint64_t p0 = static_cast<uint64_t>(r0) * tile_h * w;
    const uint64_t p1 = std::min<uint64_t>(static_cast<uint64_t>(r1) * tile_h, h) * w;
    auto cp = [&](void* dst, const void* src, size_t elem) -> cudaError_t {
      if (!dst || !src) return cudaSuccess;
      return cudaMemcpyAsync(static_cast<char*>(dst) + p0 * elem, static_cast<const char*>(src) + p0 * elem,
                             (p1 - p0) * elem, cudaMemcpyDeviceToHost, c->copy_stream);
    };
    RKF_CUDA_TRY(cp(host.t, dev.t, 4));
    RKF_CUDA_TRY(cp(host.normal, dev.normal, 12));
    RKF_CUDA_TRY(cp(host.slot, dev.slot, 4));
    RKF_CUDA_TRY(cp(host.material, dev.material, 2));
    RKF_CUDA_TRY(cp(host.flags, dev.flags, 2));
    RKF_CUDA_TRY(cp(host.position, dev.position, 16));
    RKF_CUDA_TRY(cp(host.packed_material, dev.packed_material, 4));
    RKF_CUDA_TRY(cp(host.motion, dev.motion, 16));
  }
  RKF_CUDA_TRY(cudaStreamSynchronize(c->copy_stream));
  RKF_CUDA_TRY(cudaStreamSynchronize(c->band_stream));
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return RKF_OK;
}

rkf_status check_common(rkf_ctx* ctx, const void* a, const rkf_march_params* p, const char* fn) {
  if (!ctx || !a || !p) return fail(RKF_INVALID_ARG, std::string(fn) + ": null argument");
  if (p->hard_max_steps == 0 || p->hard_max_steps > (1u << 20))
    return fail(RKF_INVALID_ARG, std::string(fn) + ": hard_max_steps out of range");
  if (p->bisect_steps > 64) return fail(RKF_INVALID_ARG, std::string(fn) + ": bisect_steps out of range");
  if (p->strategy > RKF_STRATEGY_BVH) return fail(RKF_INVALID_ARG, std::string(fn) + ": unknown strategy");
  return RKF_OK;
}

rkf_status check_gbuffer(const rkf_gbuffer* out, const char* fn) {
  if (!out || !out->t || !out->normal || !out->slot || !out->material || !out->flags)
    return fail(RKF_INVALID_ARG, std::string(fn) + ": G-buffer plane missing");
  if (out->mem > RKF_MEM_DEVICE) return fail(RKF_INVALID_ARG, std::string(fn) + ": bad mem kind");
  return RKF_OK;
}

template <class F>
rkf_status run_gbuffer(Ctx* c, const rkf_gbuffer* out, uint64_t n, F&& launch) {
  if (out->mem == RKF_MEM_DEVICE) {
    rkf_status st = launch(*out);
    if (st != RKF_OK) return st;
    RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return RKF_OK;
  }
  rkf_gbuffer dev;
  rkf_status st = stage_gbuffer(c, *out, n, &dev);
  if (st != RKF_OK) return st;
  st = launch(dev);
  if (st != RKF_OK) return st;
  st = copy_back_gbuffer(c, *out, dev, n);
  if (st != RKF_OK) return st;
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return RKF_OK;
}

}  // namespace detail

using namespace detail;

extern "C" {

rkf_status rkf_march(rkf_ctx* ctx, const rkf_camera* cam, const rkf_march_params* p, uint32_t width,
                     uint32_t height, rkf_gbuffer* out) {
  rkf_status st = check_common(ctx, cam, p, "rkf_march");
  if (st != RKF_OK) return st;
  if ((st = check_gbuffer(out, "rkf_march")) != RKF_OK) return st;
  if (width == 0 || height == 0 || static_cast<uint64_t>(width) * height > (1ull << 31))
    return fail(RKF_INVALID_ARG, "rkf_march: bad resolution");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  const uint64_t n = static_cast<uint64_t>(width) * height;
  const int bands = host_bands(n);
  if (out->mem == RKF_MEM_HOST && bands > 1 && p->strategy != RKF_STRATEGY_TILED &&
      (g_host_bands.load() >= 0 || all_page_locked(*out)))
    return march_host_banded(c, cam, p, width, height, *out, bands);
  return run_gbuffer(c, out, n, [&](const rkf_gbuffer& dev) {
    const rkf_batch_tuning& tu = c->tuning;
    std::vector<Segment> segs{view_segment(cam, width, height, tu.tile_w, tu.tile_h, dev)};
    segs[0].first = 0;
    return launch_persistent(c, segs, segs[0].n_ids, p, tu, c->stream, &c->seg_buf,
                             c->counters.as<unsigned long long>());
  });
}

rkf_status rkf_march_plain(rkf_ctx* ctx, const rkf_camera* cam, const rkf_march_params* p,
                           uint32_t width, uint32_t height, rkf_gbuffer* out) {
  rkf_status st = check_common(ctx, cam, p, "rkf_march_plain");
  if (st != RKF_OK) return st;
  if ((st = check_gbuffer(out, "rkf_march_plain")) != RKF_OK) return st;
  if (width == 0 || height == 0 || static_cast<uint64_t>(width) * height > (1ull << 31))
    return fail(RKF_INVALID_ARG, "rkf_march_plain: bad resolution");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  const uint64_t n = static_cast<uint64_t>(width) * height;
  return run_gbuffer(c, out, n, [&](const rkf_gbuffer& dev) {
    return launch_plain(c, cam, p, width, height, dev, c->stream);
  });
}

rkf_status rkf_march_async(rkf_ctx* ctx, const rkf_camera* cam, const rkf_march_params* p,
                           uint32_t width, uint32_t height, const rkf_gbuffer* out, void* stream) {
  rkf_status st = check_common(ctx, cam, p, "rkf_march_async");
  if (st != RKF_OK) return st;
  if ((st = check_gbuffer(out, "rkf_march_async")) != RKF_OK) return st;
  if (out->mem != RKF_MEM_DEVICE) return fail(RKF_INVALID_ARG, "rkf_march_async: device G-buffer required");
  if (width == 0 || height == 0 || static_cast<uint64_t>(width) * height > (1ull << 31))
    return fail(RKF_INVALID_ARG, "rkf_march_async: bad resolution");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  const rkf_batch_tuning& tu = c->tuning;
  std::vector<Segment> segs{view_segment(cam, width, height, tu.tile_w, tu.tile_h, *out)};
  segs[0].first = 0;
  return launch_persistent(c, segs, segs[0].n_ids, p, tu, s, &c->seg_buf, c->counters.as<unsigned long long>());
}

rkf_status rkf_march_plain_async(rkf_ctx* ctx, const rkf_camera* cam, const rkf_march_params* p,
                                 uint32_t width, uint32_t height, const rkf_gbuffer* out, void* stream) {
  rkf_status st = check_common(ctx, cam, p, "rkf_march_plain_async");
  if (st != RKF_OK) return st;
  if ((st = check_gbuffer(out, "rkf_march_plain_async")) != RKF_OK) return st;
  if (out->mem != RKF_MEM_DEVICE) return fail(RKF_INVALID_ARG, "rkf_march_plain_async: device G-buffer required");
  if (width == 0 || height == 0 || static_cast<uint64_t>(width) * height > (1ull << 31))
    return fail(RKF_INVALID_ARG, "rkf_march_plain_async: bad resolution");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  return launch_plain(c, cam, p, width, height, *out, stream ? static_cast<cudaStream_t>(stream) : c->stream);
}

rkf_status rkf_trace_rays(rkf_ctx* ctx, const float* origins, const float* dirs, const float* tmax,
                          uint32_t n, uint32_t mode, const rkf_march_params* p, uint32_t in_mem,
                          rkf_hits* out) {
  rkf_status st = check_common(ctx, p, p, "rkf_trace_rays");
  if (st != RKF_OK) return st;
  if (!out || !out->t || (n && (!origins || !dirs || !tmax)))
    return fail(RKF_INVALID_ARG, "rkf_trace_rays: null argument");
  if (mode > RKF_TRACE_SHADOW) return fail(RKF_INVALID_ARG, "rkf_trace_rays: bad mode");
  if (in_mem > RKF_MEM_DEVICE || out->mem > RKF_MEM_DEVICE)
    return fail(RKF_INVALID_ARG, "rkf_trace_rays: bad mem kind");
  if (n == 0) return RKF_OK;
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  // stage inputs and outputs as needed: [o 12n][d 12n][tmax 4n] + outputs
  const size_t in_b = in_mem == RKF_MEM_HOST ? align256(12ull * n) * 2 + align256(4ull * n) : 0;
  const size_t out_b = out->mem == RKF_MEM_HOST
                           ? align256(4ull * n) + align256(12ull * n) + align256(4ull * n) +
                                 align256(2ull * n) * 2
                           : 0;
  if ((st = c->stage_bytes(in_b + out_b)) != RKF_OK) return st;
  char* b = c->stage.as<char>();
  const float *d_o = origins, *d_d = dirs, *d_t = tmax;
  if (in_mem == RKF_MEM_HOST) {
    RKF_CUDA_TRY(cudaMemcpyAsync(b, origins, 12ull * n, cudaMemcpyHostToDevice, c->stream));
    d_o = reinterpret_cast<float*>(b);
    b += align256(12ull * n);
    RKF_CUDA_TRY(cudaMemcpyAsync(b, dirs, 12ull * n, cudaMemcpyHostToDevice, c->stream));
    d_d = reinterpret_cast<float*>(b);
    b += align256(12ull * n);
    RKF_CUDA_TRY(cudaMemcpyAsync(b, tmax, 4ull * n, cudaMemcpyHostToDevice, c->stream));
    d_t = reinterpret_cast<float*>(b);
    b += align256(4ull * n);
  }
  rkf_hits dev = *out;
  if (out->mem == RKF_MEM_HOST) {
    dev.t = reinterpret_cast<float*>(b);
    b += align256(4ull * n);
    dev.normal = out->normal ? reinterpret_cast<float*>(b) : nullptr;
    b += align256(12ull * n);
    dev.slot = out->slot ? reinterpret_cast<uint32_t*>(b) : nullptr;
    b += align256(4ull * n);
    dev.material = out->material ? reinterpret_cast<uint16_t*>(b) : nullptr;
    b += align256(2ull * n);
    dev.flags = out->flags ? reinterpret_cast<uint16_t*>(b) : nullptr;
    dev.mem = RKF_MEM_DEVICE;
  }
  std::vector<Segment> segs{ray_segment(d_o, d_d, d_t, n, mode, dev)};
  segs[0].first = 0;
  st = launch_persistent(c, segs, n, p, c->tuning, c->stream, &c->seg_buf,
                         c->counters.as<unsigned long long>());
  if (st != RKF_OK) return st;
  if (out->mem == RKF_MEM_HOST) {
    RKF_CUDA_TRY(cudaMemcpyAsync(out->t, dev.t, 4ull * n, cudaMemcpyDeviceToHost, c->stream));
    if (out->normal) RKF_CUDA_TRY(cudaMemcpyAsync(out->normal, dev.normal, 12ull * n, cudaMemcpyDeviceToHost, c->stream));
    if (out->slot) RKF_CUDA_TRY(cudaMemcpyAsync(out->slot, dev.slot, 4ull * n, cudaMemcpyDeviceToHost, c->stream));
    if (out->material) RKF_CUDA_TRY(cudaMemcpyAsync(out->material, dev.material, 2ull * n, cudaMemcpyDeviceToHost, c->stream));
    if (out->flags) RKF_CUDA_TRY(cudaMemcpyAsync(out->flags, dev.flags, 2ull * n, cudaMemcpyDeviceToHost, c->stream));
  }
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return RKF_OK;
}

rkf_status rkf_query_points(rkf_ctx* ctx, const float* points, uint32_t n, float* dist, float* grad,
                            uint16_t* material, uint32_t mem) {
  if (!ctx || (n && !points)) return fail(RKF_INVALID_ARG, "rkf_query_points: null argument");
  if (mem > RKF_MEM_DEVICE) return fail(RKF_INVALID_ARG, "rkf_query_points: bad mem kind");
  if (n == 0) return RKF_OK;
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  if (mem == RKF_MEM_DEVICE) {
    rkf_status st = launch_query(c, points, n, dist, grad, material, c->stream);
    if (st != RKF_OK) return st;
    RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return RKF_OK;
  }
  const size_t b_in = align256(12ull * n), b_d = align256(4ull * n), b_g = align256(12ull * n),
               b_m = align256(2ull * n);
  rkf_status st = c->stage_bytes(b_in + b_d + b_g + b_m);
  if (st != RKF_OK) return st;
  char* b = c->stage.as<char>();
  float* dp = reinterpret_cast<float*>(b);
  float* dd = reinterpret_cast<float*>(b + b_in);
  float* dg = reinterpret_cast<float*>(b + b_in + b_d);
  uint16_t* dm = reinterpret_cast<uint16_t*>(b + b_in + b_d + b_g);
  RKF_CUDA_TRY(cudaMemcpyAsync(dp, points, 12ull * n, cudaMemcpyHostToDevice, c->stream));
  st = launch_query(c, dp, n, dist ? dd : nullptr, grad ? dg : nullptr, material ? dm : nullptr, c->stream);
  if (st != RKF_OK) return st;
  if (dist) RKF_CUDA_TRY(cudaMemcpyAsync(dist, dd, 4ull * n, cudaMemcpyDeviceToHost, c->stream));
  if (grad) RKF_CUDA_TRY(cudaMemcpyAsync(grad, dg, 12ull * n, cudaMemcpyDeviceToHost, c->stream));
  if (material) RKF_CUDA_TRY(cudaMemcpyAsync(material, dm, 2ull * n, cudaMemcpyDeviceToHost, c->stream));
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return RKF_OK;
}

rkf_status rkf_sdf_ao(rkf_ctx* ctx, const float* pos, const float* normal, uint32_t n, float* ao,
                      uint32_t mem) {
  if (!ctx || (n && (!pos || !normal || !ao))) return fail(RKF_INVALID_ARG, "rkf_sdf_ao: null argument");
  if (mem > RKF_MEM_DEVICE) return fail(RKF_INVALID_ARG, "rkf_sdf_ao: bad mem kind");
  if (n == 0) return RKF_OK;
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  if (mem == RKF_MEM_DEVICE) {
    rkf_status st = launch_ao(c, pos, normal, n, ao, c->stream);
    if (st != RKF_OK) return st;
    RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return RKF_OK;
  }
  const size_t b_in = align256(12ull * n), b_ao = align256(4ull * n);
  rkf_status st = c->stage_bytes(2 * b_in + b_ao);
  if (st != RKF_OK) return st;
  char* b = c->stage.as<char>();
  float* dp = reinterpret_cast<float*>(b);
  float* dn = reinterpret_cast<float*>(b + b_in);
  float* da = reinterpret_cast<float*>(b + 2 * b_in);
  RKF_CUDA_TRY(cudaMemcpyAsync(dp, pos, 12ull * n, cudaMemcpyHostToDevice, c->stream));
  RKF_CUDA_TRY(cudaMemcpyAsync(dn, normal, 12ull * n, cudaMemcpyHostToDevice, c->stream));
  if ((st = launch_ao(c, dp, dn, n, da, c->stream)) != RKF_OK) return st;
  RKF_CUDA_TRY(cudaMemcpyAsync(ao, da, 4ull * n, cudaMemcpyDeviceToHost, c->stream));
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return RKF_OK;
}

rkf_status rkf_march_batch(rkf_ctx* ctx, const rkf_view* views, uint32_t n_views,
                           const rkf_ray_batch* batches, uint32_t n_batches,
                           const rkf_march_params* p, const rkf_batch_tuning* tuning) {
  rkf_status st = rkf_march_batch_async(ctx, views, n_views, batches, n_batches, p, tuning, nullptr);
  if (st != RKF_OK) return st;
  RKF_CUDA_TRY(cudaStreamSynchronize(reinterpret_cast<Ctx*>(ctx)->stream));
  return RKF_OK;
}

rkf_status rkf_trace_rays_plain_async(rkf_ctx* ctx, const float* origins, const float* dirs,
                                      const float* tmax, uint32_t n, uint32_t mode,
                                      const rkf_march_params* p, const rkf_hits* out, void* stream) {
  rkf_status st = check_common(ctx, p, p, "rkf_trace_rays_plain_async");
  if (st != RKF_OK) return st;
  if (!out || !out->t || (n && (!origins || !dirs || !tmax)))
    return fail(RKF_INVALID_ARG, "rkf_trace_rays_plain_async: null argument");
  if (mode > RKF_TRACE_SHADOW || out->mem != RKF_MEM_DEVICE)
    return fail(RKF_INVALID_ARG, "rkf_trace_rays_plain_async: bad mode or host outputs");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  return launch_trace_plain(c, origins, dirs, tmax, n, mode, p, *out,
                            stream ? static_cast<cudaStream_t>(stream) : c->stream);
}

rkf_status rkf_march_batch_async(rkf_ctx* ctx, const rkf_view* views, uint32_t n_views,
                                 const rkf_ray_batch* batches, uint32_t n_batches,
                                 const rkf_march_params* p, const rkf_batch_tuning* tuning,
                                 void* stream) {
  if (!ctx || !p || (n_views && !views) || (n_batches && !batches))
    return fail(RKF_INVALID_ARG, "rkf_march_batch: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  const cudaStream_t strm = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  const rkf_batch_tuning tu = tuning ? *tuning : c->tuning;
  if (tu.tile_w == 0 || tu.tile_h == 0 || tu.tile_w * tu.tile_h > 4096)
    return fail(RKF_INVALID_ARG, "rkf_march_batch: bad tile shape");
  std::vector<Segment> segs;
  segs.reserve(n_views + n_batches);
  uint64_t first = 0;
  for (uint32_t i = 0; i < n_views; ++i) {
    const rkf_view& v = views[i];
    if (v.width == 0 || v.height == 0) continue;
    if (v.out.mem != RKF_MEM_DEVICE || !v.out.t || !v.out.normal || !v.out.slot || !v.out.material || !v.out.flags)
      return fail(RKF_INVALID_ARG, "rkf_march_batch: views need device G-buffers");
    Segment sg = view_segment(&v.camera, v.width, v.height, tu.tile_w, tu.tile_h, v.out);
    sg.first = first;
    first += sg.n_ids;
    segs.push_back(sg);
  }
  for (uint32_t i = 0; i < n_batches; ++i) {
    const rkf_ray_batch& r = batches[i];
    if (r.n == 0) continue;
    if (r.out.mem != RKF_MEM_DEVICE || !r.out.t || !r.origins || !r.dirs || !r.tmax || r.mode > RKF_TRACE_SHADOW)
      return fail(RKF_INVALID_ARG, "rkf_march_batch: bad ray batch");
    Segment sg = ray_segment(r.origins, r.dirs, r.tmax, r.n, r.mode, r.out);
    sg.first = first;
    first += sg.n_ids;
    segs.push_back(sg);
  }
  if (segs.empty()) return RKF_OK;
  return launch_persistent(c, segs, first, p, tu, strm, &c->seg_buf, c->counters.as<unsigned long long>());
}

void rkf_testing_set_host_bands(int bands) { detail::g_host_bands.store(bands < 0 ? -1 : bands); }

rkf_status rkf_scene_origin_set(rkf_ctx* ctx, const rkf_world_pos* origin) {
  if (!ctx || !origin) return fail(RKF_INVALID_ARG, "rkf_scene_origin_set: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_scene_origin_set: the context is serving");
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(origin->local[a])) return fail(RKF_INVALID_ARG, "rkf_scene_origin_set: non-finite offset");
  c->origin = *origin;
  return RKF_OK;
}

rkf_status rkf_scene_origin_get(rkf_ctx* ctx, rkf_world_pos* out) {
  if (!ctx || !out) return fail(RKF_INVALID_ARG, "rkf_scene_origin_get: null argument");
  *out = reinterpret_cast<Ctx*>(ctx)->origin;
  return RKF_OK;
}

rkf_status rkf_march_world(rkf_ctx* ctx, const rkf_world_pos* cam_pos, const rkf_camera* cam,
                           const rkf_march_params* p, uint32_t width, uint32_t height, rkf_gbuffer* out) {
  if (!ctx || !cam_pos || !cam) return fail(RKF_INVALID_ARG, "rkf_march_world: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  rkf_camera rel = *cam;
  float pos[3];
  rkf_world_relative(cam_pos, &c->origin, nullptr, pos);
  for (int a = 0; a < 3; ++a) rel.position[a] = pos[a];
  return rkf_march(ctx, &rel, p, width, height, out);
}

rkf_status rkf_trace_rays_world(rkf_ctx* ctx, const rkf_world_pos* origins, const float* dirs,
                                const float* tmax, uint32_t n, uint32_t mode, const rkf_march_params* p,
                                rkf_hits* out) {
  if (!ctx || (n && (!origins || !dirs || !tmax))) return fail(RKF_INVALID_ARG, "rkf_trace_rays_world: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  std::vector<float> rel(3ull * n);
  for (uint32_t i = 0; i < n; ++i) rkf_world_relative(origins + i, &c->origin, nullptr, rel.data() + 3ull * i);
  return rkf_trace_rays(ctx, rel.data(), dirs, tmax, n, mode, p, RKF_MEM_HOST, out);
}

}  // extern "C"
