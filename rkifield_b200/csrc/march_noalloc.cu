// march_noalloc.cu — the batched march for callers that cannot allocate
// device memory at call time.
//
// rkf_march_batch sizes its launch scratch (the segment table the kernel
// reads and the work counter its warps draw rays from) on demand, which may
// call cudaMalloc.  cudaMalloc synchronises the device, so callers that run
// on a fixed per-frame time budget, or inside a host framework that owns
// every device allocation through its own allocator, cannot call an entry
// point that might allocate.  rkf_march_batch_noalloc does the same work
// with that scratch in one fixed file-scope device array instead.
//
// The segment table reaches the array through a small staging kernel that
// takes the whole table as a kernel parameter (at most 64 segments, under
// 17 KB): enqueueing a launch never waits on the stream, where a copy from
// pageable host memory can, and the table's bytes travel with the launch, so
// no host buffer has to outlive the call.
#include <cstring>
#include <mutex>

#include "ctx.h"
#include "march.h"

namespace rkf {
namespace {

// Scratch of the allocation-free launch: the work counter, then the segment
// table.  It occupies RKF_NOALLOC_MAX_SEGMENTS * sizeof(Segment) + 256 bytes
// (about 17 KB) on every device that loads the library, until the process
// exits.  Every call shares it.
struct NoAllocScratch {
  unsigned long long counter;
  unsigned long long pad[31];  // keeps the table 256-byte aligned
  Segment segs[RKF_NOALLOC_MAX_SEGMENTS];
};
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// The segment table of one call, passed by value to the staging kernel.
struct NoAllocTable {
  uint32_t nseg;
  uint32_t pad;
  Segment segs[RKF_NOALLOC_MAX_SEGMENTS];
};
static_assert(sizeof(NoAllocTable) <= 32000, "the table must fit the kernel parameter space");
static_assert(sizeof(Segment) % 8 == 0, "segments are copied as 8-byte words");

// Writes the call's segments into the scratch array and clears the work
// counter.  One block; each thread copies 8-byte words.
__global__ void k_noalloc_stage(const __grid_constant__ NoAllocTable tbl, NoAllocScratch* dst) {
  const uint32_t words = tbl.nseg * static_cast<uint32_t>(sizeof(Segment) / 8);
  const auto* src = reinterpret_cast<const unsigned long long*>(tbl.segs);
  auto* out = reinterpret_cast<unsigned long long*>(dst->segs);
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) out[i] = src[i];
  if (threadIdx.x == 0) dst->counter = 0ull;
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
NoAllocScratch* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current).
// Host code may only use the symbol through this address: the name itself
// is a host-side stand-in.  Resolved once per device, on its first call.
rkf_status scratch_for(int device, NoAllocScratch** out) {
  if (device < 0 || device >= kMaxDevices) return fail(RKF_INVALID_ARG, "rkf_march_batch_noalloc: device ordinal too large");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(RKF_CUDA_ERROR, std::string("rkf_march_batch_noalloc: cudaGetSymbolAddress failed: ") +
                                      cudaGetErrorString(e));
    g_scratch_addr[device] = static_cast<NoAllocScratch*>(p);
  }
  *out = g_scratch_addr[device];
  return RKF_OK;
}

}  // namespace
}  // namespace rkf

using namespace rkf;

extern "C" rkf_status rkf_march_batch_noalloc(rkf_ctx* ctx, const rkf_view* views, uint32_t n_views,
                                              const rkf_ray_batch* batches, uint32_t n_batches,
                                              const rkf_march_params* p, const rkf_batch_tuning* tuning,
                                              void* stream) {
  if (!ctx || !p || (n_views && !views) || (n_batches && !batches))
    return fail(RKF_INVALID_ARG, "rkf_march_batch_noalloc: null argument");
  if (static_cast<uint64_t>(n_views) + n_batches > RKF_NOALLOC_MAX_SEGMENTS)
    return fail(RKF_INVALID_ARG, "rkf_march_batch_noalloc: more than " +
                                     std::to_string(RKF_NOALLOC_MAX_SEGMENTS) +
                                     " views and ray batches in one call (the fixed scratch holds that many)");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  NoAllocScratch* scratch = nullptr;
  rkf_status st = scratch_for(c->device, &scratch);
  if (st != RKF_OK) return st;
  const rkf_batch_tuning tu = tuning ? *tuning : c->tuning;
  if (tu.tile_w == 0 || tu.tile_h == 0 || tu.tile_w * tu.tile_h > 4096)
    return fail(RKF_INVALID_ARG, "rkf_march_batch_noalloc: bad tile shape");
  // every refusal of the launch itself, before anything touches the shared
  // scratch (a refused call must not overwrite a table another call uses)
  st = check_persistent_scratch(c, p, tu);
  if (st != RKF_OK) return st;
  NoAllocTable tbl;
  std::memset(&tbl, 0, sizeof(tbl));
  uint32_t nseg = 0;
  uint64_t first = 0;
  for (uint32_t i = 0; i < n_views; ++i) {
    const rkf_view& v = views[i];
    if (v.width == 0 || v.height == 0) continue;
    if (v.out.mem != RKF_MEM_DEVICE || !v.out.t || !v.out.normal || !v.out.slot || !v.out.material || !v.out.flags)
      return fail(RKF_INVALID_ARG, "rkf_march_batch_noalloc: views need device G-buffers");
    Segment sg = view_segment(&v.camera, v.width, v.height, tu.tile_w, tu.tile_h, v.out);
    sg.first = first;
    first += sg.n_ids;
    tbl.segs[nseg++] = sg;
  }
  for (uint32_t i = 0; i < n_batches; ++i) {
    const rkf_ray_batch& r = batches[i];
    if (r.n == 0) continue;
    if (r.out.mem != RKF_MEM_DEVICE || !r.out.t || !r.origins || !r.dirs || !r.tmax || r.mode > RKF_TRACE_SHADOW)
      return fail(RKF_INVALID_ARG, "rkf_march_batch_noalloc: bad ray batch");
    Segment sg = ray_segment(r.origins, r.dirs, r.tmax, r.n, r.mode, r.out);
    sg.first = first;
    first += sg.n_ids;
    tbl.segs[nseg++] = sg;
  }
  if (nseg == 0) return RKF_OK;
  tbl.nseg = nseg;
  const cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  // the table and a cleared counter go in by value; the march then reads them
  k_noalloc_stage<<<1, 256, 0, s>>>(tbl, scratch);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  return launch_persistent_scratch(c, tbl.segs, nseg, first, p, tu, s, scratch->segs, &scratch->counter,
                                   /*segs_uploaded=*/true, /*multi_empty=*/true);
}
