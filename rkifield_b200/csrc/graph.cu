// graph.cu — a batched march captured once as a CUDA graph and replayed.
//
// A renderer that marches the same set of views and ray batches every frame
// (same sizes, same output buffers, new cameras) pays, per rkf_march_batch
// call, the host work of building the segment table, its copy and the
// launch.  Here that work is captured once on a private stream into a graph
// of three nodes -- the segment table's copy from page-locked memory the
// graph owns to device memory it owns, the reset of the work counter, and the
// persistent march kernel -- and each frame only rewrites the cameras in the
// page-locked table and launches the graph.
//
// The kernel node holds the scene as it was at capture (object table, index
// pointers), so a graph belongs to one epoch of its context: after an object
// import, a voxelization or an edit, launching it returns RKF_EPOCH_STALE and
// the caller creates it again.
#include <cstring>
#include <vector>

#include "ctx.h"
#include "march.h"

namespace rkf {

struct BatchGraph {
  Ctx* c = nullptr;
  uint64_t epoch = 0;
  rkf_batch_tuning tu{};
  std::vector<rkf_view> views;        // as given (cameras are replaced per frame)
  std::vector<uint32_t> view_seg;     // segment of view i, or ~0u for an empty view
  std::vector<Segment> segs;          // host copy of the table
  Segment* pinned = nullptr;          // page-locked table the copy node reads
  DevBuf dev;                         // 256 B of counter, then the device table
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t done = nullptr;         // recorded after each launch
  bool launched = false;

  ~BatchGraph() {
    if (launched) cudaEventSynchronize(done);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (done) cudaEventDestroy(done);
    if (pinned) cudaFreeHost(pinned);
  }
};

}  // namespace rkf

using namespace rkf;

extern "C" {

rkf_status rkf_batch_graph_create(rkf_ctx* ctx, const rkf_view* views, uint32_t n_views,
                                  const rkf_ray_batch* batches, uint32_t n_batches, const rkf_march_params* p,
                                  const rkf_batch_tuning* tuning, rkf_batch_graph** out) {
  if (!ctx || !p || !out || (n_views && !views) || (n_batches && !batches))
    return fail(RKF_INVALID_ARG, "rkf_batch_graph_create: null argument");
  *out = nullptr;
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  if (p->strategy != RKF_STRATEGY_BRUTE)
    return fail(RKF_UNSUPPORTED, "rkf_batch_graph_create: graphs run the brute strategy only");
  auto g = std::make_unique<BatchGraph>();
  g->c = c;
  g->epoch = c->epoch;
  g->tu = tuning ? *tuning : c->tuning;
  const rkf_batch_tuning& tu = g->tu;
  if (tu.tile_w == 0 || tu.tile_h == 0 || tu.tile_w * tu.tile_h > 4096)
    return fail(RKF_INVALID_ARG, "rkf_batch_graph_create: bad tile shape");
  uint64_t first = 0;
  g->views.assign(views, views + n_views);
  g->view_seg.assign(n_views, ~0u);
  for (uint32_t i = 0; i < n_views; ++i) {
    const rkf_view& v = views[i];
    if (v.width == 0 || v.height == 0) continue;
    if (v.out.mem != RKF_MEM_DEVICE || !v.out.t || !v.out.normal || !v.out.slot || !v.out.material || !v.out.flags)
      return fail(RKF_INVALID_ARG, "rkf_batch_graph_create: views need device G-buffers");
    Segment sg = view_segment(&v.camera, v.width, v.height, tu.tile_w, tu.tile_h, v.out);
    sg.first = first;
    first += sg.n_ids;
    g->view_seg[i] = static_cast<uint32_t>(g->segs.size());
    g->segs.push_back(sg);
  }
  for (uint32_t i = 0; i < n_batches; ++i) {
    const rkf_ray_batch& r = batches[i];
    if (r.n == 0) continue;
    if (r.out.mem != RKF_MEM_DEVICE || !r.out.t || !r.origins || !r.dirs || !r.tmax || r.mode > RKF_TRACE_SHADOW)
      return fail(RKF_INVALID_ARG, "rkf_batch_graph_create: bad ray batch");
    Segment sg = ray_segment(r.origins, r.dirs, r.tmax, r.n, r.mode, r.out);
    sg.first = first;
    first += sg.n_ids;
    g->segs.push_back(sg);
  }
  if (g->segs.empty()) return fail(RKF_INVALID_ARG, "rkf_batch_graph_create: no work");
  const size_t sb = sizeof(Segment) * g->segs.size();
  RKF_CUDA_TRY(cudaHostAlloc(reinterpret_cast<void**>(&g->pinned), sb, cudaHostAllocDefault));
  std::memcpy(g->pinned, g->segs.data(), sb);
  rkf_status st = g->dev.alloc(256 + sb);
  if (st != RKF_OK) return st;
  auto* counter = g->dev.as<unsigned long long>();
  auto* dev_segs = reinterpret_cast<Segment*>(g->dev.as<char>() + 256);
  RKF_CUDA_TRY(cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming));
  cudaStream_t cap = nullptr;
  RKF_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) {
    e = cudaMemcpyAsync(dev_segs, g->pinned, sb, cudaMemcpyHostToDevice, cap);
    if (e == cudaSuccess)
      st = launch_persistent_scratch(c, g->segs.data(), static_cast<uint32_t>(g->segs.size()), first, p, tu, cap,
                                     dev_segs, counter, true, true);
    const cudaError_t e2 = cudaStreamEndCapture(cap, &g->graph);
    if (e == cudaSuccess) e = e2;
  }
  cudaStreamDestroy(cap);
  if (st != RKF_OK) return st;
  if (e != cudaSuccess)
    return fail(RKF_CUDA_ERROR, std::string("rkf_batch_graph_create: capture failed: ") + cudaGetErrorString(e));
  RKF_CUDA_TRY(cudaGraphInstantiate(&g->exec, g->graph, 0));
  *out = reinterpret_cast<rkf_batch_graph*>(g.release());
  return RKF_OK;
}

rkf_status rkf_batch_graph_set_cameras(rkf_batch_graph* graph, const rkf_camera* cameras, uint32_t n) {
  if (!graph || (n && !cameras)) return fail(RKF_INVALID_ARG, "rkf_batch_graph_set_cameras: null argument");
  auto* g = reinterpret_cast<BatchGraph*>(graph);
  if (n != g->views.size())
    return fail(RKF_INVALID_ARG, "rkf_batch_graph_set_cameras: one camera per view of the graph");
  RKF_CUDA_TRY(cudaSetDevice(g->c->device));
  // the previous launch's copy node reads the table: let it finish first
  if (g->launched) RKF_CUDA_TRY(cudaEventSynchronize(g->done));
  for (uint32_t i = 0; i < n; ++i) {
    g->views[i].camera = cameras[i];
    const uint32_t k = g->view_seg[i];
    if (k == ~0u) continue;
    const rkf_view& v = g->views[i];
    Segment sg = view_segment(&v.camera, v.width, v.height, g->tu.tile_w, g->tu.tile_h, v.out);
    sg.first = g->segs[k].first;
    g->segs[k] = sg;
    g->pinned[k] = sg;
  }
  return RKF_OK;
}

rkf_status rkf_batch_graph_launch(rkf_batch_graph* graph, void* stream) {
  if (!graph) return fail(RKF_INVALID_ARG, "rkf_batch_graph_launch: null argument");
  auto* g = reinterpret_cast<BatchGraph*>(graph);
  if (g->c->epoch != g->epoch)
    return fail(RKF_EPOCH_STALE, "rkf_batch_graph_launch: the scene changed since the graph was made");
  RKF_CUDA_TRY(cudaSetDevice(g->c->device));
  const cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g->c->stream;
  RKF_CUDA_TRY(cudaGraphLaunch(g->exec, st));
  RKF_CUDA_TRY(cudaEventRecord(g->done, st));
  g->launched = true;
  return RKF_OK;
}

rkf_status rkf_batch_graph_destroy(rkf_batch_graph* graph) {
  if (!graph) return RKF_OK;
  auto* g = reinterpret_cast<BatchGraph*>(graph);
  cudaSetDevice(g->c->device);
  delete g;
  return RKF_OK;
}

}  // extern "C"
