// ctx.cu — context lifetime, scene import (the reference upload path), the
// two-level brick index, and small query entry points.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/rkf_cuda_testing.h"
#include "ctx.h"
#include "edit.h"
#include "empty_dist.h"

namespace rkf {

namespace {
thread_local std::string t_last_error;
// >= 0: that many more context allocations succeed, then one reports
// cudaErrorMemoryAllocation without calling cudaMalloc (rkf_testing_*).
std::atomic<long long> g_fail_after{-1};
cudaError_t default_alloc(void** p, size_t bytes) {
  long long n = g_fail_after.load();
  while (n >= 0) {
    if (n == 0) {
      g_fail_after.store(-1);
      return cudaErrorMemoryAllocation;
    }
    if (g_fail_after.compare_exchange_weak(n, n - 1)) break;
  }
  return cudaMalloc(p, bytes);
}
}  // namespace

alloc_hook_fn g_alloc_hook = default_alloc;

void set_error(const std::string& msg) { t_last_error = msg; }
rkf_status fail(rkf_status st, const std::string& msg) {
  t_last_error = msg;
  return st;
}

DevBuf::~DevBuf() { release(); }
void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}
rkf_status DevBuf::alloc(size_t n) {
  release();
  if (n == 0) return RKF_OK;
  cudaError_t e = g_alloc_hook(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? RKF_OOM : RKF_CUDA_ERROR,
                std::string("device allocation of ") + std::to_string(n) +
                    " bytes failed: " + cudaGetErrorString(e));
  }
  bytes = n;
  return RKF_OK;
}

ObjDev make_objdev(const rkf_gpu_object& o, uint32_t top_off, uint32_t has_flat) {
  ObjDev d;
  std::memset(&d, 0, sizeof(d));
  std::memcpy(d.m, o.inverse_world, sizeof(d.m));
  // Every constant below is the value the shader recomputes per sample, in the
  // same float operations (ray_march.wgsl:354-363, :621, :630).
  d.vs = o.voxel_size;
  d.be = d.vs * 8.0f;
  d.be2 = d.be * 2.0f;
  for (int a = 0; a < 3; ++a) {
    d.gs[a] = static_cast<float>(o.brick_map_dims[a]) * d.be;
    d.half_gs[a] = d.gs[a] * 0.5f;
  }
  d.lo = d.vs * 0.01f;
  for (int a = 0; a < 3; ++a) d.hi[a] = d.gs[a] - d.lo;
  d.vs16 = d.vs * 16.0f;
  for (int a = 0; a < 3; ++a) {
    d.gmin[a] = o.geometry_aabb_min[a];
    d.gmax[a] = o.geometry_aabb_max[a];
  }
  d.has_geom = o.geometry_aabb_max[0] > o.geometry_aabb_min[0] ? 1u : 0u;
  const float sx = o.accumulated_scale[0], sy = o.accumulated_scale[1],
              sz = o.accumulated_scale[2];
  const float myz = sz < sy ? sz : sy;
  d.min_scale = myz < sx ? myz : sx;
  for (int a = 0; a < 4; ++a) d.params[a] = o.sdf_params[a];
  for (int a = 0; a < 3; ++a) {
    d.tv[a] = static_cast<int>(o.brick_map_dims[a]) * 8;
    d.bdims[a] = o.brick_map_dims[a];
    d.tdim[a] = (o.brick_map_dims[a] + 7) / 8;
  }
  d.top_off = top_off;
  d.map_off = o.brick_map_offset;
  d.has_flat = has_flat;
  d.vs2 = d.vs * 2.0f;
  d.rcp_vs = d.vs > 0.0f ? static_cast<float>(1.0 / static_cast<double>(d.vs)) : 0.0f;
  d.div_ok = 0;  // set after the device check (verify_exact_div)
  const float* m = o.inverse_world;
  d.translate_only = (m[0] == 1.0f && m[1] == 0.0f && m[2] == 0.0f && m[3] == 0.0f && m[4] == 0.0f &&
                      m[5] == 1.0f && m[6] == 0.0f && m[7] == 0.0f && m[8] == 0.0f && m[9] == 0.0f &&
                      m[10] == 1.0f && m[11] == 0.0f && m[15] == 1.0f)
                         ? 1u
                         : 0u;
  d.sdf_type = o.sdf_type;
  d.prim_type = o.primitive_type;
  d.object_id = o.object_id;
  d.material_id = o.material_id;
  return d;
}

SceneDev Ctx::scene_dev() const {
  SceneDev s;
  s.dist_f16 = dist_f16.as<uint16_t>();
  s.dist_f32 = dist_f32.as<float>();
  s.dist_u8 = dist_u8.as<int8_t>();
  s.brick_step = brick_step.as<float>();
  s.mat = mat.as<uint16_t>();
  s.blend = blend.as<uint8_t>();
  s.aos = aos.as<uint2>();
  s.top = top.as<uint32_t>();
  s.empty_dist = empty_dist.as<uint8_t>();
  s.leaves = leaves.as<uint32_t>();
  s.flat_maps = flat_maps.as<uint32_t>();
  s.objs = objdev.as<ObjDev>();
  s.n_objs = obj_count();
  s.precision = cfg.precision;
  return s;
}

namespace detail {
// Counts the floats x in [b0, b0+n) (as bit patterns) whose exact_div_vs
// differs from the IEEE quotient x/vs.
__global__ void k_verify_div(float vs, float rcp, uint32_t b0, uint32_t n, unsigned int* bad) {
  const uint32_t stride = gridDim.x * blockDim.x;
  unsigned int local = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float x = __uint_as_float(b0 + i);
    if (__float_as_uint(exact_div_vs(x, vs, rcp)) != __float_as_uint(__fdiv_rn(x, vs))) ++local;
  }
  if (local) atomicAdd(bad, local);
}
}  // namespace detail

// Decide ObjDev::div_ok for every voxelized object: exhaustively compare the
// fast quotient with IEEE division over every float of the object's clamped
// sampling domain [vs*0.01, max(grid size) - vs*0.01].
rkf_status Ctx::verify_exact_div() {
  for (ObjDev& d : objdev_host) {
    if (d.sdf_type != RKF_SDF_VOXELIZED || d.div_ok) continue;
    const float hi = std::max(d.hi[0], std::max(d.hi[1], d.hi[2]));
    if (!(d.lo > 0.0f) || !(hi > d.lo)) continue;
    uint32_t b0, b1;
    std::memcpy(&b0, &d.lo, 4);
    std::memcpy(&b1, &hi, 4);
    uint32_t vsb;
    std::memcpy(&vsb, &d.vs, 4);
    auto it = div_checked.find(vsb);
    if (it != div_checked.end() && it->second.first <= b0 && it->second.second >= b1) {
      d.div_ok = 1;
      continue;
    }
    DevBuf bad;
    rkf_status st = bad.alloc(4);
    if (st != RKF_OK) return st;
    RKF_CUDA_TRY(cudaMemsetAsync(bad.p, 0, 4, stream));
    detail::k_verify_div<<<sm_count * 8, 256, 0, stream>>>(d.vs, d.rcp_vs, b0, b1 - b0 + 1,
                                                          bad.as<unsigned int>());
    counted();
    RKF_CUDA_TRY(cudaGetLastError());
    unsigned int nbad = 0;
    RKF_CUDA_TRY(cudaMemcpyAsync(&nbad, bad.p, 4, cudaMemcpyDeviceToHost, stream));
    RKF_CUDA_TRY(cudaStreamSynchronize(stream));
    if (nbad == 0) {
      d.div_ok = 1;
      div_checked[vsb] = {b0, b1};
    }
  }
  return RKF_OK;
}

rkf_status Ctx::upload_objects() {
  if (objdev_host.empty()) return RKF_OK;
  rkf_status vst = verify_exact_div();
  if (vst != RKF_OK) return vst;
  const size_t bytes = objdev_host.size() * sizeof(ObjDev);
  if (objdev.bytes < bytes) {
    DevBuf nb;  // the old table stays valid if this allocation fails
    rkf_status st = nb.alloc(bytes);
    if (st != RKF_OK) return st;
    std::swap(objdev.p, nb.p);
    std::swap(objdev.bytes, nb.bytes);
  }
  RKF_CUDA_TRY(cudaMemcpyAsync(objdev.p, objdev_host.data(), bytes, cudaMemcpyHostToDevice, stream));
  RKF_CUDA_TRY(cudaStreamSynchronize(stream));
  return RKF_OK;
}

rkf_status Ctx::ensure_leaf_capacity(uint32_t need) {
  if (need <= leaf_cap) return RKF_OK;
  // while serving, in-flight launches hold the leaf buffer's address
  if (leaves_frozen) return fail(RKF_OOM, "index leaf capacity reserved for the serving session is exhausted");
  uint32_t cap = leaf_cap ? leaf_cap : 64;
  while (cap < need) cap *= 2;
  DevBuf nb;
  rkf_status st = nb.alloc(static_cast<size_t>(cap) * 512 * 4);
  if (st != RKF_OK) return st;
  if (n_leaves)
    RKF_CUDA_TRY(cudaMemcpyAsync(nb.p, leaves.p, static_cast<size_t>(n_leaves) * 2048,
                                 cudaMemcpyDeviceToDevice, stream));
  RKF_CUDA_TRY(cudaStreamSynchronize(stream));
  std::swap(leaves.p, nb.p);
  std::swap(leaves.bytes, nb.bytes);
  leaf_cap = cap;
  return RKF_OK;
}

rkf_status Ctx::stage_bytes(size_t bytes) {
  if (stage.bytes >= bytes) return RKF_OK;
  return stage.alloc(bytes + bytes / 4);
}

rkf_status Ctx::march_event(cudaStream_t st, bool end) {
  // (the serving loop's launches are not timed: its worker thread would
  // share the event list with the caller)
  if (!time_march || serve || march_timed >= kMaxTimed) return RKF_OK;
  const size_t k = 2 * static_cast<size_t>(march_timed) + (end ? 1 : 0);
  if (k >= march_ev.size()) {
    cudaEvent_t e = nullptr;
    RKF_CUDA_TRY(cudaEventCreate(&e));
    march_ev.push_back(e);
  }
  RKF_CUDA_TRY(cudaEventRecord(march_ev[k], st));
  if (end) ++march_timed;
  return RKF_OK;
}

namespace detail {

// VoxelSample words -> SoA planes (+ optional AoS copy).  One thread per voxel.
__global__ void k_import_words(const uint2* __restrict__ words, uint64_t nvox, uint64_t first_vox,
                               uint16_t* dist_f16, float* dist_f32, uint16_t* mat, uint8_t* blend,
                               uint2* aos) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= nvox) return;
  const uint2 w = words[i];
  const uint64_t v = first_vox + i;
  const uint16_t d = static_cast<uint16_t>(w.x & 0xFFFFu);
  if (dist_f16) dist_f16[v] = d;
  if (dist_f32) dist_f32[v] = __half2float(__ushort_as_half(d));
  mat[v] = static_cast<uint16_t>(((w.x >> 16) & 0x3Fu) | (((w.x >> 22) & 0x3Fu) << 6));
  blend[v] = static_cast<uint8_t>(w.y >> 24);
  if (aos) aos[v] = w;
}

// SoA planes (f16 distance, material | secondary << 6, blend) -> the context
// planes (+ the reference word pair, packed as VoxelSample::new_blended packs
// it, voxel.rs:43-54).  One thread per voxel.
__global__ void k_import_soa(const uint16_t* __restrict__ d16, const uint16_t* __restrict__ m16,
                             const uint8_t* __restrict__ bl, uint64_t nvox, uint64_t first_vox, uint16_t* dist_f16,
                             float* dist_f32, uint16_t* mat, uint8_t* blend, uint2* aos) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= nvox) return;
  const uint64_t v = first_vox + i;
  const uint16_t d = d16[i];
  const uint32_t mm = m16[i] & 0xFFFu;
  const uint8_t b = bl[i];
  if (dist_f16) dist_f16[v] = d;
  if (dist_f32) dist_f32[v] = __half2float(__ushort_as_half(d));
  mat[v] = static_cast<uint16_t>(mm);
  blend[v] = b;
  if (aos) aos[v] = make_uint2(d | ((mm & 0x3Fu) << 16) | (((mm >> 6) & 0x3Fu) << 22), static_cast<uint32_t>(b) << 24);
}

__global__ void k_lookup(SceneDev s, uint32_t obj, const uint32_t* bxyz, uint32_t n, uint32_t* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const ObjDev& o = s.objs[obj];
  const uint32_t bx = bxyz[3 * i], by = bxyz[3 * i + 1], bz = bxyz[3 * i + 2];
  if (bx >= o.bdims[0] || by >= o.bdims[1] || bz >= o.bdims[2]) {
    out[i] = RKF_EMPTY_SLOT;
    return;
  }
  out[i] = lookup2(s, o, bx, by, bz);
}

}  // namespace detail

rkf_status lookup_bricks(Ctx* c, uint32_t obj, const uint32_t* d_bxyz, uint32_t n, uint32_t* d_out,
                         cudaStream_t st) {
  if (n == 0) return RKF_OK;
  detail::k_lookup<<<(n + 255) / 256, 256, 0, st>>>(c->scene_dev(), obj, d_bxyz, n, d_out);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  return RKF_OK;
}

// Band-normalised signed u8 code of one brick.  The brick's band is
// B = min(band, largest finite |d| in the brick) -- band is the narrow band's
// half-width (3 voxels for a voxelized object), so B / band is the brick's
// scale s_b <= 1 -- and step = B/127.  |code| = min(floor(|d|/step), 127),
// rounding toward zero and clamping |d| to B, less one when the decoded
// product code*step would round above |d|: a decoded |d| never exceeds the
// true one (sphere tracing never overshoots).  band = +inf: B is the brick's
// largest |d|.  nearest: |code| = min(rint(|d|/step), 127) instead -- each
// code within half a step of |d| (clamped to B), errors of either sign, so
// they do not add up along a ray's steps the way a one-sided bias does.
__global__ void k_encode_u8(const float* __restrict__ src_f32, const uint16_t* __restrict__ src_f16,
                            uint32_t first_slot, uint32_t n_bricks, int8_t* code, float* step, float band,
                            bool nearest) {
  const uint32_t b = blockIdx.x;
  if (b >= n_bricks) return;
  const uint64_t base = (static_cast<uint64_t>(first_slot) + b) * 512;
  __shared__ float red[256];
  float m = 0.0f;
  for (int i = threadIdx.x; i < 512; i += blockDim.x) {
    const float d = src_f32 ? src_f32[base + i] : __half2float(__ushort_as_half(src_f16[base + i]));
    const float a = fabsf(d);
    if (a <= 3.0e38f && a > m) m = a;
  }
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  const float range = fmaxf(fminf(red[0], band), 1e-6f);
  const float st = __fdiv_rn(range, 127.0f);
  if (threadIdx.x == 0) step[first_slot + b] = st;
  for (int i = threadIdx.x; i < 512; i += blockDim.x) {
    const float d = src_f32 ? src_f32[base + i] : __half2float(__ushort_as_half(src_f16[base + i]));
    const float a = fabsf(d);
    const float qa = __fdiv_rn(a, st);
    const float q = nearest ? rintf(qa) : floorf(qa);
    int c = q >= 127.0f ? 127 : static_cast<int>(q);
    // toward zero: the decoder's product RN(c*step) must not exceed |d| (the
    // quotient may round up to the next integer)
    if (!nearest && c > 0 && __fmul_rn(static_cast<float>(c), st) > a) --c;
    code[base + i] = static_cast<int8_t>(d < 0.0f ? -c : c);
  }
}

}  // namespace rkf

using namespace rkf;

extern "C" {

const char* rkf_last_error(void) { return t_last_error.c_str(); }

void rkf_testing_fail_allocation_after(long long n) { g_fail_after.store(n < 0 ? -1 : n); }

void rkf_march_params_default(rkf_march_params* p) {
  if (!p) return;
  p->scene.num_objects = 0;
  p->scene.max_steps = 128;         // gpu_scene.rs:38
  p->scene.max_distance = 100.0f;   // gpu_scene.rs:39
  p->scene.hit_threshold = 0.001f;  // gpu_scene.rs:40
  p->hard_max_steps = 1024;         // ray_march.wgsl:36
  p->bisect_steps = 8;              // ray_march.wgsl:31
  p->min_step = 0.0005f;            // ray_march.wgsl:30
  p->near_surface_threshold = 0.02f;  // ray_march.wgsl:41
  p->strategy = RKF_STRATEGY_BRUTE;
  p->reserved = 0;
}

void rkf_config_default(rkf_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->device = 0;
  cfg->pool_capacity_bricks = 1u << 16;
  cfg->precision = RKF_PRECISION_F16;
  cfg->keep_reference_pool = 1;
  cfg->max_inflight = 64;
}

rkf_status rkf_create(const rkf_config* cfg, rkf_ctx** out) {
  if (!cfg || !out) return fail(RKF_INVALID_ARG, "rkf_create: null argument");
  if (cfg->precision > RKF_PRECISION_U8) return fail(RKF_INVALID_ARG, "rkf_create: bad precision");
  if (!(cfg->u8_band >= 0.0f) || cfg->u8_round > 1) return fail(RKF_INVALID_ARG, "rkf_create: bad u8 encoding");
  if (cfg->pool_capacity_bricks == 0 || cfg->pool_capacity_bricks > (RKF_INTERIOR_SLOT - 1))
    return fail(RKF_INVALID_ARG, "rkf_create: pool_capacity_bricks out of range");
  int ndev = 0;
  RKF_CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (cfg->device < 0 || cfg->device >= ndev)
    return fail(RKF_INVALID_ARG, "rkf_create: no CUDA device " + std::to_string(cfg->device));
  RKF_CUDA_TRY(cudaSetDevice(cfg->device));
  auto c = std::make_unique<Ctx>();
  c->device = cfg->device;
  c->cfg = *cfg;
  if (c->cfg.max_inflight == 0) c->cfg.max_inflight = 64;
  RKF_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  RKF_CUDA_TRY(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device));
  const size_t cap = cfg->pool_capacity_bricks;
  c->capacity = cfg->pool_capacity_bricks;
  const size_t nv = cap * 512;
  rkf_status st = RKF_OK;
  switch (cfg->precision) {
    case RKF_PRECISION_F32:
      st = c->dist_f32.alloc(nv * 4);
      break;
    case RKF_PRECISION_U8:
      if ((st = c->dist_u8.alloc(nv)) == RKF_OK) st = c->brick_step.alloc(cap * 4);
      // the f16 plane stays the import staging source for the u8 encoder
      if (st == RKF_OK) st = c->dist_f16.alloc(nv * 2);
      break;
    default:
      st = c->dist_f16.alloc(nv * 2);
  }
  if (st == RKF_OK) st = c->mat.alloc(nv * 2);
  if (st == RKF_OK) st = c->blend.alloc(nv);
  if (st == RKF_OK && cfg->keep_reference_pool) st = c->aos.alloc(nv * 8);
  if (st == RKF_OK) st = c->counters.alloc(4096);
  if (st != RKF_OK) {
    cudaStreamDestroy(c->stream);
    return st;
  }
  c->free_slots.resize(cap);
  for (size_t i = 0; i < cap; ++i) c->free_slots[i] = static_cast<uint32_t>(cap - 1 - i);
  c->tuning = rkf_batch_tuning{4, 8, 32, 64, 0, 256, 32, 0, 0};
  *out = reinterpret_cast<rkf_ctx*>(c.release());
  return RKF_OK;
}

rkf_status rkf_serve_stop(rkf_ctx* ctx);

rkf_status rkf_destroy(rkf_ctx* ctx) {
  if (!ctx) return fail(RKF_INVALID_ARG, "rkf_destroy: null ctx");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  cudaSetDevice(c->device);
  if (c->serve) rkf_serve_stop(ctx);
  cudaStreamSynchronize(c->stream);
  cudaStreamDestroy(c->stream);
  for (cudaStream_t s : {c->copy_stream, c->band_stream})
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  for (cudaEvent_t e : c->band_ev)
    if (e) cudaEventDestroy(e);
  if (c->segs_ev) cudaEventDestroy(c->segs_ev);
  for (cudaEvent_t e : c->march_ev) cudaEventDestroy(e);
  delete c;
  return RKF_OK;
}

namespace {
// Tail of a pool import into slots [first_slot, first_slot + n_bricks): the u8
// encoding when the context stores codes, then the slots leave the free list.
rkf_status finish_pool_import(Ctx* c, uint32_t first_slot, uint32_t n_bricks) {
  if (c->cfg.precision == RKF_PRECISION_U8) {
    // the pool does not know the voxel size of its bricks: the configured
    // band, else each brick's own largest |d|
    const float band = c->cfg.u8_band > 0.0f ? c->cfg.u8_band : INFINITY;
    k_encode_u8<<<n_bricks, 256, 0, c->stream>>>(nullptr, c->dist_f16.as<uint16_t>(), first_slot, n_bricks,
                                                 c->dist_u8.as<int8_t>(), c->brick_step.as<float>(), band,
                                                 c->cfg.u8_round == 1);
    c->counted();
    RKF_CUDA_TRY(cudaGetLastError());
  }
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  std::vector<uint32_t> keep;
  keep.reserve(c->free_slots.size());
  for (uint32_t s : c->free_slots)
    if (s < first_slot || s >= first_slot + n_bricks) keep.push_back(s);
  c->used_slots += static_cast<uint32_t>(c->free_slots.size() - keep.size());
  c->free_slots.swap(keep);
  return RKF_OK;
}
}  // namespace

rkf_status rkf_pool_import_soa(rkf_ctx* ctx, const uint16_t* dist_f16, const uint16_t* mat, const uint8_t* blend,
                               uint32_t first_slot, uint32_t n_bricks) {
  if (!ctx || (n_bricks && (!dist_f16 || !mat || !blend)))
    return fail(RKF_INVALID_ARG, "rkf_pool_import_soa: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_pool_import_soa: the context is serving");
  if (static_cast<uint64_t>(first_slot) + n_bricks > c->capacity)
    return fail(RKF_INVALID_ARG, "rkf_pool_import_soa: slots beyond pool capacity");
  if (n_bricks == 0) return RKF_OK;
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  const uint64_t nvox = static_cast<uint64_t>(n_bricks) * 512;
  const size_t b16 = (nvox * 2 + 255) & ~static_cast<size_t>(255);
  rkf_status st = c->stage_bytes(2 * b16 + nvox);
  if (st != RKF_OK) return st;
  char* b = c->stage.as<char>();
  RKF_CUDA_TRY(cudaMemcpyAsync(b, dist_f16, nvox * 2, cudaMemcpyHostToDevice, c->stream));
  RKF_CUDA_TRY(cudaMemcpyAsync(b + b16, mat, nvox * 2, cudaMemcpyHostToDevice, c->stream));
  RKF_CUDA_TRY(cudaMemcpyAsync(b + 2 * b16, blend, nvox, cudaMemcpyHostToDevice, c->stream));
  const unsigned blocks = static_cast<unsigned>((nvox + 255) / 256);
  detail::k_import_soa<<<blocks, 256, 0, c->stream>>>(
      reinterpret_cast<const uint16_t*>(b), reinterpret_cast<const uint16_t*>(b + b16),
      reinterpret_cast<const uint8_t*>(b + 2 * b16), nvox, static_cast<uint64_t>(first_slot) * 512,
      c->dist_f16.as<uint16_t>(), c->dist_f32.as<float>(), c->mat.as<uint16_t>(), c->blend.as<uint8_t>(),
      c->aos.as<uint2>());
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  return finish_pool_import(c, first_slot, n_bricks);
}

rkf_status rkf_pool_import_voxelsample(rkf_ctx* ctx, const uint32_t* words, uint32_t first_slot,
                                       uint32_t n_bricks) {
  if (!ctx || (!words && n_bricks)) return fail(RKF_INVALID_ARG, "rkf_pool_import_voxelsample: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_pool_import_voxelsample: the context is serving");
  if (static_cast<uint64_t>(first_slot) + n_bricks > c->capacity)
    return fail(RKF_INVALID_ARG, "rkf_pool_import_voxelsample: slots beyond pool capacity");
  if (n_bricks == 0) return RKF_OK;
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  const uint64_t nvox = static_cast<uint64_t>(n_bricks) * 512;
  rkf_status st = c->stage_bytes(nvox * 8);
  if (st != RKF_OK) return st;
  RKF_CUDA_TRY(cudaMemcpyAsync(c->stage.p, words, nvox * 8, cudaMemcpyHostToDevice, c->stream));
  const uint64_t first_vox = static_cast<uint64_t>(first_slot) * 512;
  const unsigned blocks = static_cast<unsigned>((nvox + 255) / 256);
  detail::k_import_words<<<blocks, 256, 0, c->stream>>>(c->stage.as<uint2>(), nvox, first_vox,
                                                c->dist_f16.as<uint16_t>(), c->dist_f32.as<float>(),
                                                c->mat.as<uint16_t>(), c->blend.as<uint8_t>(),
                                                c->aos.as<uint2>());
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  return finish_pool_import(c, first_slot, n_bricks);
}

rkf_status rkf_pool_export_voxelsample(rkf_ctx* ctx, uint32_t first_slot, uint32_t n_bricks,
                                       uint32_t* words) {
  if (!ctx || !words) return fail(RKF_INVALID_ARG, "rkf_pool_export_voxelsample: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c->aos.p) return fail(RKF_UNSUPPORTED, "rkf_pool_export_voxelsample: context keeps no reference pool");
  if (static_cast<uint64_t>(first_slot) + n_bricks > c->capacity)
    return fail(RKF_INVALID_ARG, "rkf_pool_export_voxelsample: range beyond capacity");
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  RKF_CUDA_TRY(cudaMemcpyAsync(words, c->aos.as<uint2>() + static_cast<size_t>(first_slot) * 512,
                               static_cast<size_t>(n_bricks) * 4096, cudaMemcpyDeviceToHost, c->stream));
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return RKF_OK;
}

rkf_status rkf_brickmap_import(rkf_ctx* ctx, const uint32_t* packed, uint64_t n) {
  if (!ctx || (!packed && n)) return fail(RKF_INVALID_ARG, "rkf_brickmap_import: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_brickmap_import: the context is serving");
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  DevBuf nb;  // the previous maps stay if this fails
  rkf_status st = nb.alloc(n * 4);
  if (st != RKF_OK) return st;
  if (n) RKF_CUDA_TRY(cudaMemcpy(nb.p, packed, n * 4, cudaMemcpyHostToDevice));
  std::swap(c->flat_maps.p, nb.p);
  std::swap(c->flat_maps.bytes, nb.bytes);
  c->flat_host.assign(packed, packed + n);
  c->flat_len = n;
  return RKF_OK;
}

rkf_status rkf_objects_import(rkf_ctx* ctx, const rkf_gpu_object* objects, uint32_t n) {
  if (!ctx || (!objects && n)) return fail(RKF_INVALID_ARG, "rkf_objects_import: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_objects_import: the context is serving");
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  // validate and build the two-level index of every voxelized object
  std::vector<uint32_t> top;
  std::vector<uint32_t> leaf_host;
  std::vector<ObjDev> od;
  for (uint32_t i = 0; i < n; ++i) {
    const rkf_gpu_object& o = objects[i];
    if (o.sdf_type > RKF_SDF_VOXELIZED) return fail(RKF_INVALID_ARG, "rkf_objects_import: bad sdf_type");
    uint32_t top_off = static_cast<uint32_t>(top.size());
    if (o.sdf_type == RKF_SDF_VOXELIZED) {
      const uint64_t dx = o.brick_map_dims[0], dy = o.brick_map_dims[1], dz = o.brick_map_dims[2];
      if (dx == 0 || dy == 0 || dz == 0 || !(o.voxel_size > 0.0f))
        return fail(RKF_INVALID_ARG, "rkf_objects_import: voxelized object with empty grid");
      if (o.brick_map_offset + dx * dy * dz > c->flat_host.size())
        return fail(RKF_INVALID_ARG, "rkf_objects_import: brick map extends past the imported buffer");
      const uint32_t tx = static_cast<uint32_t>((dx + 7) / 8), ty = static_cast<uint32_t>((dy + 7) / 8),
                     tz = static_cast<uint32_t>((dz + 7) / 8);
      top.resize(top.size() + static_cast<size_t>(tx) * ty * tz, RKF_EMPTY_SLOT);
      for (uint32_t kz = 0; kz < tz; ++kz)
        for (uint32_t ky = 0; ky < ty; ++ky)
          for (uint32_t kx = 0; kx < tx; ++kx) {
            bool any = false, all_int = true;
            for (uint32_t l = 0; l < 512; ++l) {
              const uint64_t bx = kx * 8 + (l & 7), by = ky * 8 + ((l >> 3) & 7), bz = kz * 8 + (l >> 6);
              uint32_t s = RKF_EMPTY_SLOT;
              if (bx < dx && by < dy && bz < dz)
                s = c->flat_host[o.brick_map_offset + bx + by * dx + bz * dx * dy];
              if (s != RKF_EMPTY_SLOT) any = true;
              if (s != RKF_INTERIOR_SLOT) all_int = false;
              if (s < RKF_INTERIOR_SLOT && s >= c->capacity)
                return fail(RKF_INVALID_ARG, "rkf_objects_import: brick map names a slot beyond the pool");
            }
            uint32_t entry = RKF_EMPTY_SLOT;
            if (all_int) {
              entry = RKF_INTERIOR_SLOT;
            } else if (any) {
              // the import replaces the leaf buffer: entries count from 0
              entry = static_cast<uint32_t>(leaf_host.size() / 512);
              for (uint32_t l = 0; l < 512; ++l) {
                const uint64_t bx = kx * 8 + (l & 7), by = ky * 8 + ((l >> 3) & 7), bz = kz * 8 + (l >> 6);
                uint32_t s = RKF_EMPTY_SLOT;
                if (bx < dx && by < dy && bz < dz)
                  s = c->flat_host[o.brick_map_offset + bx + by * dx + bz * dx * dy];
                leaf_host.push_back(s);
              }
            }
            top[top_off + kx + ky * tx + kz * tx * ty] = entry;
          }
    }
    od.push_back(make_objdev(o, top_off, o.sdf_type == RKF_SDF_VOXELIZED ? 1u : 0u));
  }
  // replace the index wholesale: build it in fresh buffers, so a failure
  // leaves the previous scene in place
  const uint32_t nl = static_cast<uint32_t>(leaf_host.size() / 512);
  uint32_t cap = 64;
  while (cap < nl) cap *= 2;
  DevBuf nleaves, ntop, nfield;
  rkf_status st = nleaves.alloc(static_cast<size_t>(cap) * 2048);
  if (st == RKF_OK) st = ntop.alloc(std::max<size_t>(top.size(), 1) * 4);
  if (st == RKF_OK) st = nfield.alloc(std::max<size_t>(top.size(), 1));
  if (st != RKF_OK) return st;
  if (nl)
    RKF_CUDA_TRY(cudaMemcpy(nleaves.p, leaf_host.data(), leaf_host.size() * 4, cudaMemcpyHostToDevice));
  if (!top.empty()) RKF_CUDA_TRY(cudaMemcpy(ntop.p, top.data(), top.size() * 4, cudaMemcpyHostToDevice));
  for (const ObjDev& d : od)
    if ((st = build_empty_dist(d, ntop.as<uint32_t>(), nfield.as<uint8_t>(), c->stream)) != RKF_OK) return st;
    c->counted(3);
  std::vector<rkf_gpu_object> objects0(objects, objects + n);
  std::swap(c->objects, objects0);
  std::swap(c->objdev_host, od);
  if ((st = c->upload_objects()) != RKF_OK) {
    std::swap(c->objects, objects0);
    std::swap(c->objdev_host, od);
    return st;
  }
  std::swap(c->leaves.p, nleaves.p);
  std::swap(c->leaves.bytes, nleaves.bytes);
  c->leaf_cap = cap;
  c->n_leaves = nl;
  c->free_leaves.clear();
  std::swap(c->top.p, ntop.p);
  std::swap(c->top.bytes, ntop.bytes);
  std::swap(c->empty_dist.p, nfield.p);
  std::swap(c->empty_dist.bytes, nfield.bytes);
  c->top_len = top.size();
  c->epoch++;
  return RKF_OK;
}

rkf_status rkf_objects_update(rkf_ctx* ctx, const rkf_gpu_object* objects, uint32_t n,
                              const int32_t* index_source) {
  if (!ctx || (!objects && n)) return fail(RKF_INVALID_ARG, "rkf_objects_update: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_objects_update: the context is serving");
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  std::vector<rkf_gpu_object> recs(objects, objects + n);
  std::vector<ObjDev> od;
  od.reserve(n);
  for (uint32_t i = 0; i < n; ++i) {
    rkf_gpu_object& o = recs[i];
    if (o.sdf_type > RKF_SDF_VOXELIZED) return fail(RKF_INVALID_ARG, "rkf_objects_update: bad sdf_type");
    if (o.sdf_type != RKF_SDF_VOXELIZED) {
      od.push_back(make_objdev(o, 0, 0));
      continue;
    }
    const int64_t s = index_source ? index_source[i] : static_cast<int64_t>(i);
    if (s < 0 || s >= static_cast<int64_t>(c->obj_count()) ||
        c->objects[static_cast<size_t>(s)].sdf_type != RKF_SDF_VOXELIZED)
      return fail(RKF_INVALID_ARG, "rkf_objects_update: a voxelized record names no voxelized object's index");
    const rkf_gpu_object& e = c->objects[static_cast<size_t>(s)];
    const ObjDev& ed = c->objdev_host[static_cast<size_t>(s)];
    if (o.brick_map_dims[0] != e.brick_map_dims[0] || o.brick_map_dims[1] != e.brick_map_dims[1] ||
        o.brick_map_dims[2] != e.brick_map_dims[2] || o.voxel_size != e.voxel_size)
      return fail(RKF_INVALID_ARG, "rkf_objects_update: the record's grid differs from its index source");
    o.brick_map_offset = e.brick_map_offset;  // the brick map the index was built from
    od.push_back(make_objdev(o, ed.top_off, ed.has_flat));
  }
  std::swap(c->objects, recs);
  std::swap(c->objdev_host, od);
  rkf_status st = c->upload_objects();
  if (st != RKF_OK) {
    std::swap(c->objects, recs);
    std::swap(c->objdev_host, od);
    return st;
  }
  c->epoch++;
  return RKF_OK;
}

rkf_status rkf_object_get(rkf_ctx* ctx, uint32_t i, rkf_gpu_object* out) {
  if (!ctx || !out) return fail(RKF_INVALID_ARG, "rkf_object_get: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (i >= c->obj_count()) return fail(RKF_INVALID_ARG, "rkf_object_get: index out of range");
  *out = c->objects[i];
  return RKF_OK;
}

rkf_status rkf_scene_info_get(rkf_ctx* ctx, rkf_scene_info* out) {
  if (!ctx || !out) return fail(RKF_INVALID_ARG, "rkf_scene_info_get: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  out->num_objects = c->obj_count();
  out->pool_bricks_used = c->used_slots;
  out->pool_capacity = c->capacity;
  out->leaf_blocks = c->n_leaves;
  out->device_bytes = c->dist_f16.bytes + c->dist_f32.bytes + c->dist_u8.bytes + c->brick_step.bytes +
                      c->mat.bytes + c->blend.bytes + c->aos.bytes + c->top.bytes + c->empty_dist.bytes + c->leaves.bytes +
                      c->flat_maps.bytes + c->objdev.bytes;
  out->epoch = c->epoch;
  return RKF_OK;
}

rkf_status rkf_pool_export_planes(rkf_ctx* ctx, uint32_t first_slot, uint32_t n_bricks, void* dist,
                                  float* step, uint16_t* mat, uint8_t* blend) {
  if (!ctx) return fail(RKF_INVALID_ARG, "rkf_pool_export_planes: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (static_cast<uint64_t>(first_slot) + n_bricks > c->capacity)
    return fail(RKF_INVALID_ARG, "rkf_pool_export_planes: range beyond capacity");
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  const size_t v0 = static_cast<size_t>(first_slot) * 512, nv = static_cast<size_t>(n_bricks) * 512;
  if (dist) {
    switch (c->cfg.precision) {
      case RKF_PRECISION_F32:
        RKF_CUDA_TRY(cudaMemcpy(dist, c->dist_f32.as<float>() + v0, nv * 4, cudaMemcpyDeviceToHost));
        break;
      case RKF_PRECISION_U8:
        RKF_CUDA_TRY(cudaMemcpy(dist, c->dist_u8.as<int8_t>() + v0, nv, cudaMemcpyDeviceToHost));
        break;
      default:
        RKF_CUDA_TRY(cudaMemcpy(dist, c->dist_f16.as<uint16_t>() + v0, nv * 2, cudaMemcpyDeviceToHost));
    }
  }
  if (step && c->cfg.precision == RKF_PRECISION_U8)
    RKF_CUDA_TRY(cudaMemcpy(step, c->brick_step.as<float>() + first_slot, n_bricks * 4ull, cudaMemcpyDeviceToHost));
  if (mat) RKF_CUDA_TRY(cudaMemcpy(mat, c->mat.as<uint16_t>() + v0, nv * 2, cudaMemcpyDeviceToHost));
  if (blend) RKF_CUDA_TRY(cudaMemcpy(blend, c->blend.as<uint8_t>() + v0, nv, cudaMemcpyDeviceToHost));
  return RKF_OK;
}

rkf_status rkf_index_export(rkf_ctx* ctx, uint32_t* top, uint64_t* top_n, uint32_t* leaves,
                            uint64_t* leaf_entries, uint32_t* obj_top_info, uint32_t* n_objects) {
  if (!ctx || !top_n || !leaf_entries || !n_objects)
    return fail(RKF_INVALID_ARG, "rkf_index_export: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  *top_n = c->top_len;
  *leaf_entries = static_cast<uint64_t>(c->n_leaves) * 512;
  *n_objects = c->obj_count();
  if (top && c->top_len)
    RKF_CUDA_TRY(cudaMemcpy(top, c->top.p, c->top_len * 4, cudaMemcpyDeviceToHost));
  if (leaves && c->n_leaves)
    RKF_CUDA_TRY(cudaMemcpy(leaves, c->leaves.p, static_cast<size_t>(c->n_leaves) * 2048, cudaMemcpyDeviceToHost));
  if (obj_top_info)
    for (uint32_t i = 0; i < c->obj_count(); ++i) {
      obj_top_info[4 * i] = c->objdev_host[i].top_off;
      for (int a = 0; a < 3; ++a) obj_top_info[4 * i + 1 + a] = c->objdev_host[i].tdim[a];
    }
  return RKF_OK;
}

rkf_status rkf_testing_export_empty_dist(rkf_ctx* ctx, uint8_t* out, uint64_t* n) {
  if (!ctx || !n) return fail(RKF_INVALID_ARG, "rkf_testing_export_empty_dist: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  *n = c->top_len;
  if (out && c->top_len) RKF_CUDA_TRY(cudaMemcpy(out, c->empty_dist.p, c->top_len, cudaMemcpyDeviceToHost));
  return RKF_OK;
}

rkf_status rkf_testing_march_timing(rkf_ctx* ctx, uint32_t enable) {
  if (!ctx || enable > 1) return fail(RKF_INVALID_ARG, "rkf_testing_march_timing: bad argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_testing_march_timing: the context is serving");
  c->time_march = enable != 0;
  c->march_timed = 0;
  return RKF_OK;
}

rkf_status rkf_testing_launch_stats(rkf_ctx* ctx, uint64_t* launches, float* march_ms, uint32_t cap,
                                    uint32_t* n_timed) {
  if (!ctx || (!march_ms && cap)) return fail(RKF_INVALID_ARG, "rkf_testing_launch_stats: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (launches) *launches = c->launches.load();
  if (n_timed) *n_timed = c->march_timed;
  if (cap) RKF_CUDA_TRY(cudaSetDevice(c->device));
  for (uint32_t i = 0; i < std::min(cap, c->march_timed); ++i) {
    RKF_CUDA_TRY(cudaEventSynchronize(c->march_ev[2 * i + 1]));
    RKF_CUDA_TRY(cudaEventElapsedTime(&march_ms[i], c->march_ev[2 * i], c->march_ev[2 * i + 1]));
  }
  return RKF_OK;
}

rkf_status rkf_brick_lookup(rkf_ctx* ctx, uint32_t obj, const uint32_t* bxyz, uint32_t n,
                            uint32_t* slots) {
  if (!ctx || ((!bxyz || !slots) && n)) return fail(RKF_INVALID_ARG, "rkf_brick_lookup: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (obj >= c->obj_count() || c->objects[obj].sdf_type != RKF_SDF_VOXELIZED)
    return fail(RKF_INVALID_ARG, "rkf_brick_lookup: not a voxelized object");
  if (n == 0) return RKF_OK;
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  DevBuf buf;
  rkf_status st = buf.alloc(static_cast<size_t>(n) * 16);
  if (st != RKF_OK) return st;
  uint32_t* din = buf.as<uint32_t>();
  uint32_t* dout = din + 3 * static_cast<size_t>(n);
  RKF_CUDA_TRY(cudaMemcpyAsync(din, bxyz, static_cast<size_t>(n) * 12, cudaMemcpyHostToDevice, c->stream));
  detail::k_lookup<<<(n + 255) / 256, 256, 0, c->stream>>>(c->scene_dev(), obj, din, n, dout);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  RKF_CUDA_TRY(cudaMemcpyAsync(slots, dout, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost, c->stream));
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return RKF_OK;
}

void rkf_world_relative(const rkf_world_pos* pos, const rkf_world_pos* origin, double out_f64[3],
                        float out_f32[3]) {
  // WorldPosition::relative_to_f64 (world_position.rs:107-120), CHUNK_SIZE 8 m
  for (int a = 0; a < 3; ++a) {
    const double chunk_m = static_cast<double>(pos->chunk[a] - origin->chunk[a]) * 8.0;
    const double local = static_cast<double>(pos->local[a] - origin->local[a]);
    const double v = chunk_m + local;
    if (out_f64) out_f64[a] = v;
    if (out_f32) out_f32[a] = static_cast<float>(v);
  }
}

}  // extern "C"
