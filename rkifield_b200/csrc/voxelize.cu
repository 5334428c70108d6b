// voxelize.cu — build a voxelized object on the device from analytic
// primitives: voxelize_sdf (crates/rkf-core/src/voxelize_object.rs:53-182)
// with the scene SDF of a seeded primitive list.
//
// Scene SDF (same definition as the CPU restatement used to check it): the
// polynomial smooth-min fold (crates/rkf-core/src/sdf.rs:48-51), in ascending
// primitive order, over the primitives whose bounding sphere is nearer than
// `cut_distance`; material = the nearest primitive's, secondary material and
// blend weight from the runner-up when it is within k.
//
// Pipeline:
//   1. host: brick grid (dims, centred origin) exactly as voxelize_sdf
//      computes it; a uniform cell grid listing, per cell, every primitive
//      that can pass the cut test anywhere in the cell (a superset, so the
//      per-point test keeps the fold identical to one over all primitives)
//   2. k_classify_centres: one thread per brick; the brick-centre distance
//      decides EMPTY / INTERIOR / candidate (count pass, then list pass)
//   3. k_populate: one 512-thread block per candidate brick evaluates every
//      voxel centre and decides allocated / EMPTY / INTERIOR
//   4. host: allocated bricks get pool slots in ascending flat order (the
//      reference's z,y,x loop, lowest free slots first); the two-level index
//      and the GpuObject are built
//   5. k_scatter: candidate voxels -> pool planes (f16/f32/u8, material,
//      blend, reference VoxelSample)
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "empty_dist.h"

namespace rkf {
namespace detail {

struct VoxGrid {
  uint32_t dims[3];
  float vs, bws, hb, origin[3];
  float k, cut, band, thr, ref_band;
  uint32_t rule;
  // cell grid of primitive lists
  float cmin[3], cinv;
  int cdims[3];
};

__device__ __forceinline__ float prim_sdf_dev(const rkf_prim& p, float px, float py, float pz) {
  const float dx = __fsub_rn(px, p.centre[0]), dy = __fsub_rn(py, p.centre[1]),
              dz = __fsub_rn(pz, p.centre[2]);
  if (p.type == RKF_PRIM_SPHERE) return __fsub_rn(len3(dx, dy, dz), p.params[0]);
  const float* m = p.rot;
  const float lx = __fadd_rn(__fadd_rn(__fmul_rn(m[0], dx), __fmul_rn(m[3], dy)), __fmul_rn(m[6], dz));
  const float ly = __fadd_rn(__fadd_rn(__fmul_rn(m[1], dx), __fmul_rn(m[4], dy)), __fmul_rn(m[7], dz));
  const float lz = __fadd_rn(__fadd_rn(__fmul_rn(m[2], dx), __fmul_rn(m[5], dy)), __fmul_rn(m[8], dz));
  if (p.type == RKF_PRIM_BOX) {
    const float qx = __fsub_rn(fabsf(lx), p.params[0]), qy = __fsub_rn(fabsf(ly), p.params[1]),
                qz = __fsub_rn(fabsf(lz), p.params[2]);
    const float outside = len3(fmax_(qx, 0.0f), fmax_(qy, 0.0f), fmax_(qz, 0.0f));
    const float inside = fmin_(fmax_(qx, fmax_(qy, qz)), 0.0f);
    return __fadd_rn(outside, inside);
  }
  // capsule a=(0,-h,0), b=(0,h,0)
  const float h = p.params[1];
  const float pax = __fsub_rn(lx, 0.0f), pay = __fsub_rn(ly, -h), paz = __fsub_rn(lz, 0.0f);
  const float bax = __fsub_rn(0.0f, 0.0f), bay = __fsub_rn(h, -h), baz = __fsub_rn(0.0f, 0.0f);
  const float dpb = __fadd_rn(__fadd_rn(__fmul_rn(pax, bax), __fmul_rn(pay, bay)), __fmul_rn(paz, baz));
  const float dbb = __fadd_rn(__fadd_rn(__fmul_rn(bax, bax), __fmul_rn(bay, bay)), __fmul_rn(baz, baz));
  const float hh = clampf(__fdiv_rn(dpb, dbb), 0.0f, 1.0f);
  return __fsub_rn(len3(__fsub_rn(pax, __fmul_rn(bax, hh)), __fsub_rn(pay, __fmul_rn(bay, hh)),
                        __fsub_rn(paz, __fmul_rn(baz, hh))),
                   p.params[0]);
}

__device__ __forceinline__ float smin_dev(float a, float b, float k) {
  const float h = __fdiv_rn(fmax_(__fsub_rn(k, fabsf(__fsub_rn(a, b))), 0.0f), k);
  return __fsub_rn(fmin_(a, b), __fmul_rn(__fmul_rn(__fmul_rn(h, h), k), 0.25f));
}

struct VoxArgs {
  VoxGrid g;
  const rkf_prim* prims;
  const uint32_t* cell_start;
  const uint32_t* cell_items;
};

__device__ __forceinline__ float scene_eval_dev(const VoxArgs& a, float px, float py, float pz,
                                                uint32_t* mat, uint32_t* sec, uint32_t* blend) {
  const VoxGrid& g = a.g;
  int c[3];
  const float pp[3] = {px, py, pz};
  for (int i = 0; i < 3; ++i) {
    const int ci = static_cast<int>(floorf((pp[i] - g.cmin[i]) * g.cinv));
    c[i] = min(max(ci, 0), g.cdims[i] - 1);
  }
  const uint32_t cell = c[0] + c[1] * g.cdims[0] + c[2] * g.cdims[0] * g.cdims[1];
  const uint32_t b = __ldg(a.cell_start + cell), e = __ldg(a.cell_start + cell + 1);
  float acc = INFINITY, best = INFINITY, second = INFINITY;
  int bi = -1, si = -1;
  for (uint32_t j = b; j < e; ++j) {
    const uint32_t i = __ldg(a.cell_items + j);
    const rkf_prim& p = a.prims[i];
    const float lb = __fsub_rn(len3(__fsub_rn(px, p.centre[0]), __fsub_rn(py, p.centre[1]),
                                    __fsub_rn(pz, p.centre[2])),
                               p.bound_radius);
    if (!(lb < g.cut)) continue;
    const float d = prim_sdf_dev(p, px, py, pz);
    acc = smin_dev(acc, d, g.k);
    if (d < best) {
      second = best;
      si = bi;
      best = d;
      bi = static_cast<int>(i);
    } else if (d < second) {
      second = d;
      si = static_cast<int>(i);
    }
  }
  if (mat) {
    *mat = bi >= 0 ? a.prims[bi].material : 0u;
    *sec = 0u;
    *blend = 0u;
    if (si >= 0 && __fsub_rn(second, best) < g.k) {
      const float w = __fmul_rn(0.5f, __fsub_rn(1.0f, __fdiv_rn(__fsub_rn(second, best), g.k)));
      *sec = a.prims[si].material;
      *blend = static_cast<uint32_t>(floorf(__fadd_rn(__fmul_rn(w, 255.0f), 0.5f)));
    }
  }
  return acc;
}

// brick-centre classification: 0 candidate, 1 EMPTY, 2 INTERIOR
__device__ __forceinline__ uint32_t classify_centre(const VoxArgs& a, uint32_t bx, uint32_t by,
                                                    uint32_t bz) {
  const VoxGrid& g = a.g;
  const float mx = __fadd_rn(g.origin[0], __fmul_rn(static_cast<float>(bx), g.bws));
  const float my = __fadd_rn(g.origin[1], __fmul_rn(static_cast<float>(by), g.bws));
  const float mz = __fadd_rn(g.origin[2], __fmul_rn(static_cast<float>(bz), g.bws));
  const float dc = scene_eval_dev(a, __fadd_rn(mx, g.hb), __fadd_rn(my, g.hb), __fadd_rn(mz, g.hb),
                                  nullptr, nullptr, nullptr);
  if (g.rule == RKF_BAND_REFERENCE) return fabsf(dc) < g.ref_band ? 0u : 1u;
  if (fabsf(dc) <= g.thr) return 0u;
  return dc > 0.0f ? 1u : 2u;
}

// pass 0 counts, pass 1 writes the candidate / interior flat-id lists
__global__ void k_classify_centres(VoxArgs a, int pass, unsigned long long* counts,
                                   uint64_t* cand, uint64_t cand_cap, uint64_t* inter,
                                   uint64_t inter_cap) {
  const uint32_t bx = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t by = blockIdx.y, bz = blockIdx.z;
  uint32_t cls = 1;
  if (bx < a.g.dims[0]) cls = classify_centre(a, bx, by, bz);
  const uint64_t flat = bx + static_cast<uint64_t>(by) * a.g.dims[0] +
                        static_cast<uint64_t>(bz) * a.g.dims[0] * a.g.dims[1];
  // warp-aggregated appends
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t want = 0; want < 3; want += 2) {
    const bool mine = bx < a.g.dims[0] && cls == want;
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, mine);
    if (!m) continue;
    const uint32_t leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(counts + (want == 0 ? 0 : 1), static_cast<unsigned long long>(__popc(m)));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (pass == 1 && mine) {
      const uint64_t pos = base + __popc(m & ((1u << lane) - 1u));
      if (want == 0 && pos < cand_cap) cand[pos] = flat;
      if (want == 2 && pos < inter_cap) inter[pos] = flat;
    }
  }
}

// One block (512 threads) per candidate brick.
__global__ void __launch_bounds__(512) k_populate(VoxArgs a, const uint64_t* __restrict__ cand,
                                                  uint64_t n, float* dist, uint16_t* mat,
                                                  uint8_t* blend, uint8_t* cls_out) {
  const uint64_t ci = blockIdx.x;
  if (ci >= n) return;
  const VoxGrid& g = a.g;
  const uint64_t flat = cand[ci];
  const uint32_t bx = static_cast<uint32_t>(flat % g.dims[0]);
  const uint32_t by = static_cast<uint32_t>((flat / g.dims[0]) % g.dims[1]);
  const uint32_t bz = static_cast<uint32_t>(flat / (static_cast<uint64_t>(g.dims[0]) * g.dims[1]));
  const uint32_t v = threadIdx.x;
  const uint32_t vx = v & 7, vy = (v >> 3) & 7, vz = v >> 6;
  const float mx = __fadd_rn(g.origin[0], __fmul_rn(static_cast<float>(bx), g.bws));
  const float my = __fadd_rn(g.origin[1], __fmul_rn(static_cast<float>(by), g.bws));
  const float mz = __fadd_rn(g.origin[2], __fmul_rn(static_cast<float>(bz), g.bws));
  const float hv = __fmul_rn(g.vs, 0.5f);
  // voxel centre = brick_min + (v*vs + half_voxel)   (voxelize_object.rs:170-176)
  const float px = __fadd_rn(mx, __fadd_rn(__fmul_rn(static_cast<float>(vx), g.vs), hv));
  const float py = __fadd_rn(my, __fadd_rn(__fmul_rn(static_cast<float>(vy), g.vs), hv));
  const float pz = __fadd_rn(mz, __fadd_rn(__fmul_rn(static_cast<float>(vz), g.vs), hv));
  uint32_t m, s, b;
  float d = scene_eval_dev(a, px, py, pz, &m, &s, &b);
  if (g.rule == RKF_BAND_REFERENCE) s = b = 0;  // VoxelSample::new(d, mat, 0) (voxelize_object.rs:180)
  const size_t o = ci * 512 + v;
  dist[o] = d;
  mat[o] = static_cast<uint16_t>((m & 0x3Fu) | ((s & 0x3Fu) << 6));
  blend[o] = static_cast<uint8_t>(b);
  const int in_band = fabsf(d) <= g.band;
  const int not_pos = !(d > 0.0f);
  const int not_neg = !(d < 0.0f);
  const int any_band = __syncthreads_or(in_band);
  const int any_not_pos = __syncthreads_or(not_pos);
  const int any_not_neg = __syncthreads_or(not_neg);
  if (v == 0) {
    uint8_t c;
    if (g.rule == RKF_BAND_REFERENCE || any_band) c = 0;
    else if (!any_not_pos) c = 1;
    else if (!any_not_neg) c = 2;
    else c = 0;
    cls_out[ci] = c;
  }
}

// candidate voxels -> pool planes at their slots
__global__ void k_scatter(const float* __restrict__ dist, const uint16_t* __restrict__ mat,
                          const uint8_t* __restrict__ blend, const uint32_t* __restrict__ cand_idx,
                          const uint32_t* __restrict__ slots, uint32_t n, uint16_t* dist_f16,
                          float* dist_f32, uint16_t* pmat, uint8_t* pblend, uint2* aos) {
  const uint32_t i = blockIdx.x;
  if (i >= n) return;
  const size_t src = static_cast<size_t>(cand_idx[i]) * 512 + threadIdx.x;
  const size_t dst = static_cast<size_t>(slots[i]) * 512 + threadIdx.x;
  const float d = dist[src];
  const uint16_t h = __half_as_ushort(__float2half_rn(d));
  const uint16_t m = mat[src];
  const uint8_t b = blend[src];
  if (dist_f16) dist_f16[dst] = h;
  if (dist_f32) dist_f32[dst] = d;
  pmat[dst] = m;
  pblend[dst] = b;
  // VoxelSample::new_blended packing (voxel.rs:44-52)
  if (aos) aos[dst] = make_uint2(static_cast<uint32_t>(h) | ((m & 0x3Fu) << 16) | (((m >> 6) & 0x3Fu) << 22),
                                 static_cast<uint32_t>(b) << 24);
}

}  // namespace detail

// u8 encoder (ctx.cu)
__global__ void k_encode_u8(const float* __restrict__ src_f32, const uint16_t* __restrict__ src_f16,
                            uint32_t first_slot, uint32_t n_bricks, int8_t* code, float* step, float band,
                            bool nearest);

}  // namespace rkf

using namespace rkf;
using namespace rkf::detail;

extern "C" rkf_status rkf_voxelize_prims(rkf_ctx* ctx, const rkf_prim* prims, uint32_t n_prims,
                                         const rkf_voxelize_params* vp, uint32_t* out_object_index) {
  if (!ctx || !vp || (n_prims && !prims)) return fail(RKF_INVALID_ARG, "rkf_voxelize_prims: null argument");
  if (!(vp->voxel_size > 0.0f) || !(vp->smooth_k > 0.0f) || vp->band_rule > RKF_BAND_REFERENCE)
    return fail(RKF_INVALID_ARG, "rkf_voxelize_prims: bad parameters");
  for (uint32_t i = 0; i < n_prims; ++i)
    if (prims[i].type > RKF_PRIM_CAPSULE) return fail(RKF_INVALID_ARG, "rkf_voxelize_prims: bad primitive type");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->obj_count() + 1 > 64) return fail(RKF_UNSUPPORTED, "rkf_voxelize_prims: object table full");
  RKF_CUDA_TRY(cudaSetDevice(c->device));

  // ---- 1. grid exactly as voxelize_sdf (voxelize_object.rs:61-81) -----------
  VoxGrid g;
  std::memset(&g, 0, sizeof(g));
  g.vs = vp->voxel_size;
  g.bws = vp->voxel_size * 8.0f;
  g.hb = g.bws * 0.5f;
  for (int a = 0; a < 3; ++a) {
    const float size = vp->aabb_max[a] - vp->aabb_min[a];
    uint32_t d = static_cast<uint32_t>(std::ceil(size / g.bws));
    g.dims[a] = d < 1 ? 1 : d;
    g.origin[a] = -((static_cast<float>(g.dims[a]) * g.bws) * 0.5f);
  }
  if (g.dims[1] > 65535 || g.dims[2] > 65535 || static_cast<uint64_t>(g.dims[0]) * g.dims[1] * g.dims[2] > (1ull << 36))
    return fail(RKF_INVALID_ARG, "rkf_voxelize_prims: grid too large");
  g.k = vp->smooth_k;
  g.cut = vp->cut_distance;
  g.band = vp->band_voxels * g.vs;
  g.thr = (g.band + g.bws * 0.8660254f) + g.vs;
  g.ref_band = g.bws * 1.8f;
  g.rule = vp->band_rule;

  // cell grid over the brick grid's extent
  const double ext[3] = {g.dims[0] * static_cast<double>(g.bws), g.dims[1] * static_cast<double>(g.bws),
                         g.dims[2] * static_cast<double>(g.bws)};
  const double maxext = std::max(ext[0], std::max(ext[1], ext[2]));
  double cell = std::max(2.0 * static_cast<double>(g.cut), maxext / 128.0);
  for (int a = 0; a < 3; ++a) {
    g.cmin[a] = g.origin[a];
    g.cdims[a] = std::max(1, static_cast<int>(std::ceil(ext[a] / cell)));
  }
  g.cinv = static_cast<float>(1.0 / cell);
  const size_t ncell = static_cast<size_t>(g.cdims[0]) * g.cdims[1] * g.cdims[2];
  std::vector<std::vector<uint32_t>> lists(ncell);
  for (uint32_t i = 0; i < n_prims; ++i) {
    const double reach = static_cast<double>(prims[i].bound_radius) + g.cut + 0.02 * cell + 1e-3;
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::max(0, static_cast<int>(std::floor((prims[i].centre[a] - reach - g.cmin[a]) / cell)) - 1);
      hi[a] = std::min(g.cdims[a] - 1, static_cast<int>(std::floor((prims[i].centre[a] + reach - g.cmin[a]) / cell)) + 1);
    }
    for (int z = lo[2]; z <= hi[2]; ++z)
      for (int y = lo[1]; y <= hi[1]; ++y)
        for (int x = lo[0]; x <= hi[0]; ++x) {
          double d2 = 0.0;
          const int cc[3] = {x, y, z};
          for (int a = 0; a < 3; ++a) {
            const double b0 = g.cmin[a] + cc[a] * cell - 0.01 * cell, b1 = g.cmin[a] + (cc[a] + 1) * cell + 0.01 * cell;
            const double v = prims[i].centre[a];
            const double e = v < b0 ? b0 - v : (v > b1 ? v - b1 : 0.0);
            d2 += e * e;
          }
          if (d2 <= reach * reach) lists[x + y * g.cdims[0] + static_cast<size_t>(z) * g.cdims[0] * g.cdims[1]].push_back(i);
        }
  }
  std::vector<uint32_t> cstart(ncell + 1, 0), citems;
  for (size_t i = 0; i < ncell; ++i) {
    cstart[i] = static_cast<uint32_t>(citems.size());
    citems.insert(citems.end(), lists[i].begin(), lists[i].end());  // ascending primitive order
  }
  cstart[ncell] = static_cast<uint32_t>(citems.size());

  DevBuf d_prims, d_cstart, d_citems, d_counts;
  rkf_status st;
  if ((st = d_prims.alloc(std::max<size_t>(1, n_prims) * sizeof(rkf_prim))) != RKF_OK) return st;
  if ((st = d_cstart.alloc(cstart.size() * 4)) != RKF_OK) return st;
  if ((st = d_citems.alloc(std::max<size_t>(1, citems.size()) * 4)) != RKF_OK) return st;
  if ((st = d_counts.alloc(64)) != RKF_OK) return st;
  if (n_prims) RKF_CUDA_TRY(cudaMemcpyAsync(d_prims.p, prims, n_prims * sizeof(rkf_prim), cudaMemcpyHostToDevice, c->stream));
  RKF_CUDA_TRY(cudaMemcpyAsync(d_cstart.p, cstart.data(), cstart.size() * 4, cudaMemcpyHostToDevice, c->stream));
  if (!citems.empty()) RKF_CUDA_TRY(cudaMemcpyAsync(d_citems.p, citems.data(), citems.size() * 4, cudaMemcpyHostToDevice, c->stream));
  VoxArgs va{g, d_prims.as<rkf_prim>(), d_cstart.as<uint32_t>(), d_citems.as<uint32_t>()};

  // ---- 2. centre classification: count, then list ---------------------------
  const dim3 cblock(128);
  const dim3 cgrid((g.dims[0] + 127) / 128, g.dims[1], g.dims[2]);
  unsigned long long counts[2] = {0, 0};
  RKF_CUDA_TRY(cudaMemsetAsync(d_counts.p, 0, 16, c->stream));
  k_classify_centres<<<cgrid, cblock, 0, c->stream>>>(va, 0, d_counts.as<unsigned long long>(), nullptr, 0, nullptr, 0);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  RKF_CUDA_TRY(cudaMemcpyAsync(counts, d_counts.p, 16, cudaMemcpyDeviceToHost, c->stream));
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  const uint64_t n_cand = counts[0], n_int = counts[1];
  DevBuf d_cand, d_inter;
  if ((st = d_cand.alloc(std::max<uint64_t>(1, n_cand) * 8)) != RKF_OK) return st;
  if ((st = d_inter.alloc(std::max<uint64_t>(1, n_int) * 8)) != RKF_OK) return st;
  RKF_CUDA_TRY(cudaMemsetAsync(d_counts.p, 0, 16, c->stream));
  k_classify_centres<<<cgrid, cblock, 0, c->stream>>>(va, 1, d_counts.as<unsigned long long>(),
                                                      d_cand.as<uint64_t>(), n_cand, d_inter.as<uint64_t>(), n_int);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());

  // ---- 3. populate candidates --------------------------------------------------
  DevBuf d_dist, d_mat, d_blend, d_cls;
  if ((st = d_dist.alloc(std::max<uint64_t>(1, n_cand) * 512 * 4)) != RKF_OK) return st;
  if ((st = d_mat.alloc(std::max<uint64_t>(1, n_cand) * 512 * 2)) != RKF_OK) return st;
  if ((st = d_blend.alloc(std::max<uint64_t>(1, n_cand) * 512)) != RKF_OK) return st;
  if ((st = d_cls.alloc(std::max<uint64_t>(1, n_cand))) != RKF_OK) return st;
  if (n_cand) {
    k_populate<<<static_cast<unsigned>(n_cand), 512, 0, c->stream>>>(va, d_cand.as<uint64_t>(), n_cand,
                                                                     d_dist.as<float>(), d_mat.as<uint16_t>(),
                                                                     d_blend.as<uint8_t>(), d_cls.as<uint8_t>());
    c->counted();
    RKF_CUDA_TRY(cudaGetLastError());
  }
  std::vector<uint64_t> cand(n_cand), inter(n_int);
  std::vector<uint8_t> cls(n_cand);
  if (n_cand) {
    RKF_CUDA_TRY(cudaMemcpyAsync(cand.data(), d_cand.p, n_cand * 8, cudaMemcpyDeviceToHost, c->stream));
    RKF_CUDA_TRY(cudaMemcpyAsync(cls.data(), d_cls.p, n_cand, cudaMemcpyDeviceToHost, c->stream));
  }
  if (n_int) RKF_CUDA_TRY(cudaMemcpyAsync(inter.data(), d_inter.p, n_int * 8, cudaMemcpyDeviceToHost, c->stream));
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));

  // ---- 4. slots in ascending flat order, the index and the GpuObject ---------
  std::vector<std::pair<uint64_t, uint32_t>> alloc;  // (flat, candidate index)
  for (uint64_t i = 0; i < n_cand; ++i) {
    if (cls[i] == 0) alloc.emplace_back(cand[i], static_cast<uint32_t>(i));
    else if (cls[i] == 2) inter.push_back(cand[i]);
  }
  std::sort(alloc.begin(), alloc.end());
  const uint32_t n_alloc = static_cast<uint32_t>(alloc.size());
  if (n_alloc > c->free_slots.size()) return fail(RKF_OOM, "rkf_voxelize_prims: brick pool has too few free slots");
  std::vector<uint32_t> slots(n_alloc), cidx(n_alloc);
  for (uint32_t i = 0; i < n_alloc; ++i) {
    slots[i] = c->free_slots.back();  // Pool::allocate_range pops lowest slots first
    c->free_slots.pop_back();
    cidx[i] = alloc[i].second;
  }
  c->used_slots += n_alloc;
  // Until the object is committed, a failure gives the slots back (in the
  // order they were taken) and leaves the index and object table as they were;
  // bytes already written past top_len / n_leaves are unreferenced.
  Rollback undo([&, leaves0 = c->n_leaves, top_len0 = c->top_len, nobj0 = c->objects.size()] {
    for (uint32_t i = n_alloc; i-- > 0;) c->free_slots.push_back(slots[i]);
    c->used_slots -= n_alloc;
    c->n_leaves = leaves0;
    c->top_len = top_len0;
    c->objects.resize(nobj0);
    c->objdev_host.resize(nobj0);
  });

  const uint32_t tdim[3] = {(g.dims[0] + 7) / 8, (g.dims[1] + 7) / 8, (g.dims[2] + 7) / 8};
  const size_t ntop = static_cast<size_t>(tdim[0]) * tdim[1] * tdim[2];
  std::vector<uint32_t> top(ntop, RKF_EMPTY_SLOT);
  std::vector<uint16_t> n_nonempty(ntop, 0), n_interior(ntop, 0);
  auto block_of = [&](uint64_t f, uint32_t* b3) {
    b3[0] = static_cast<uint32_t>(f % g.dims[0]);
    b3[1] = static_cast<uint32_t>((f / g.dims[0]) % g.dims[1]);
    b3[2] = static_cast<uint32_t>(f / (static_cast<uint64_t>(g.dims[0]) * g.dims[1]));
    return (b3[0] >> 3) + (b3[1] >> 3) * static_cast<size_t>(tdim[0]) + (b3[2] >> 3) * static_cast<size_t>(tdim[0]) * tdim[1];
  };
  uint32_t b3[3];
  uint32_t gl[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, gh[3] = {0, 0, 0};
  for (auto& a : alloc) {
    const size_t blk = block_of(a.first, b3);
    n_nonempty[blk]++;
    for (int q = 0; q < 3; ++q) {
      gl[q] = std::min(gl[q], b3[q]);
      gh[q] = std::max(gh[q], b3[q] + 1);
    }
  }
  for (uint64_t f : inter) {
    const size_t blk = block_of(f, b3);
    n_nonempty[blk]++;
    n_interior[blk]++;
  }
  auto block_full = [&](size_t blk) {
    const uint32_t kx = static_cast<uint32_t>(blk % tdim[0]), ky = static_cast<uint32_t>((blk / tdim[0]) % tdim[1]),
                   kz = static_cast<uint32_t>(blk / (static_cast<size_t>(tdim[0]) * tdim[1]));
    return kx * 8 + 8 <= g.dims[0] && ky * 8 + 8 <= g.dims[1] && kz * 8 + 8 <= g.dims[2];
  };
  uint32_t n_new_leaves = 0;
  for (size_t blk = 0; blk < ntop; ++blk) {
    if (!n_nonempty[blk]) continue;
    if (n_interior[blk] == 512 && block_full(blk)) {
      top[blk] = RKF_INTERIOR_SLOT;
    } else {
      top[blk] = c->n_leaves + n_new_leaves++;
    }
  }
  std::vector<uint32_t> leaves(static_cast<size_t>(n_new_leaves) * 512, RKF_EMPTY_SLOT);
  auto put = [&](uint64_t f, uint32_t v) {
    const size_t blk = block_of(f, b3);
    const uint32_t t = top[blk];
    if (t >= RKF_INTERIOR_SLOT) return;
    leaves[static_cast<size_t>(t - c->n_leaves) * 512 + (b3[0] & 7) + (b3[1] & 7) * 8 + (b3[2] & 7) * 64] = v;
  };
  for (uint32_t i = 0; i < n_alloc; ++i) put(alloc[i].first, slots[i]);
  for (uint64_t f : inter) put(f, RKF_INTERIOR_SLOT);

  // upload slots / scatter voxels
  if (n_alloc) {
    DevBuf d_slots, d_cidx;
    if ((st = d_slots.alloc(n_alloc * 4ull)) != RKF_OK) return st;
    if ((st = d_cidx.alloc(n_alloc * 4ull)) != RKF_OK) return st;
    RKF_CUDA_TRY(cudaMemcpyAsync(d_slots.p, slots.data(), n_alloc * 4ull, cudaMemcpyHostToDevice, c->stream));
    RKF_CUDA_TRY(cudaMemcpyAsync(d_cidx.p, cidx.data(), n_alloc * 4ull, cudaMemcpyHostToDevice, c->stream));
    k_scatter<<<n_alloc, 512, 0, c->stream>>>(d_dist.as<float>(), d_mat.as<uint16_t>(), d_blend.as<uint8_t>(),
                                              d_cidx.as<uint32_t>(), d_slots.as<uint32_t>(), n_alloc,
                                              c->dist_f16.as<uint16_t>(), c->dist_f32.as<float>(),
                                              c->mat.as<uint16_t>(), c->blend.as<uint8_t>(), c->aos.as<uint2>());
    c->counted();
    RKF_CUDA_TRY(cudaGetLastError());
    if (c->cfg.precision == RKF_PRECISION_U8) {
      // encode each new brick from its f32 distances (staged per slot)
      DevBuf tmp;
      if ((st = tmp.alloc(static_cast<size_t>(c->capacity) * 512 * 4)) != RKF_OK) return st;
      k_scatter<<<n_alloc, 512, 0, c->stream>>>(d_dist.as<float>(), d_mat.as<uint16_t>(), d_blend.as<uint8_t>(),
                                                d_cidx.as<uint32_t>(), d_slots.as<uint32_t>(), n_alloc, nullptr,
                                                tmp.as<float>(), c->mat.as<uint16_t>(), c->blend.as<uint8_t>(), nullptr);
      c->counted();
      RKF_CUDA_TRY(cudaGetLastError());
      // the codes cover the narrow band: +-3 voxels unless configured
      const float band = c->cfg.u8_band > 0.0f ? c->cfg.u8_band : 3.0f * g.vs;
      // slots of one voxelization are not necessarily contiguous: encode per slot
      for (uint32_t i = 0; i < n_alloc;) {
        uint32_t j = i + 1;
        while (j < n_alloc && slots[j] == slots[j - 1] + 1) ++j;
        k_encode_u8<<<j - i, 256, 0, c->stream>>>(tmp.as<float>(), nullptr, slots[i], j - i,
                                                  c->dist_u8.as<int8_t>(), c->brick_step.as<float>(), band,
                                                  c->cfg.u8_round == 1);
        c->counted();
        RKF_CUDA_TRY(cudaGetLastError());
        i = j;
      }
      RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
  }
  // append index
  if ((st = c->ensure_leaf_capacity(c->n_leaves + std::max<uint32_t>(n_new_leaves, 1))) != RKF_OK) return st;
  if (n_new_leaves)
    RKF_CUDA_TRY(cudaMemcpyAsync(c->leaves.as<uint32_t>() + static_cast<size_t>(c->n_leaves) * 512, leaves.data(),
                                 leaves.size() * 4, cudaMemcpyHostToDevice, c->stream));
  const uint64_t top_off = c->top_len;
  rkf_gpu_object o;
  std::memset(&o, 0, sizeof(o));
  for (int i = 0; i < 4; ++i) o.inverse_world[i * 4 + i] = 1.0f;
  const float be = g.vs * 8.0f;
  float gs[3];
  for (int a = 0; a < 3; ++a) {
    gs[a] = static_cast<float>(g.dims[a]) * be;
    o.aabb_min[a] = -(gs[a] * 0.5f);
    o.aabb_max[a] = gs[a] * 0.5f;
    o.brick_map_dims[a] = g.dims[a];
    o.accumulated_scale[a] = 1.0f;
  }
  o.voxel_size = g.vs;
  o.sdf_type = RKF_SDF_VOXELIZED;
  o.object_id = vp->object_id;
  if (n_alloc) {  // compute_geometry_aabb_for_flat_node (brick_ops.rs:225-262)
    for (int a = 0; a < 3; ++a) {
      o.geometry_aabb_min[a] = static_cast<float>(gl[a]) * be - gs[a] * 0.5f;
      o.geometry_aabb_max[a] = static_cast<float>(gh[a]) * be - gs[a] * 0.5f;
    }
  }
  const ObjDev od = make_objdev(o, static_cast<uint32_t>(top_off), 0u);
  {
    DevBuf nt, nf;
    if ((st = nt.alloc((top_off + ntop) * 4)) != RKF_OK) return st;
    if ((st = nf.alloc(top_off + ntop)) != RKF_OK) return st;
    if (top_off) RKF_CUDA_TRY(cudaMemcpyAsync(nt.p, c->top.p, top_off * 4, cudaMemcpyDeviceToDevice, c->stream));
    if (top_off) RKF_CUDA_TRY(cudaMemcpyAsync(nf.p, c->empty_dist.p, top_off, cudaMemcpyDeviceToDevice, c->stream));
    RKF_CUDA_TRY(cudaMemcpyAsync(nt.as<uint32_t>() + top_off, top.data(), ntop * 4, cudaMemcpyHostToDevice, c->stream));
    if ((st = build_empty_dist(od, nt.as<uint32_t>(), nf.as<uint8_t>(), c->stream)) != RKF_OK) return st;
    c->counted(3);
    std::swap(c->top.p, nt.p);
    std::swap(c->top.bytes, nt.bytes);
    std::swap(c->empty_dist.p, nf.p);
    std::swap(c->empty_dist.bytes, nf.bytes);
  }
  c->top_len = top_off + ntop;
  c->n_leaves += n_new_leaves;
  c->objects.push_back(o);
  c->objdev_host.push_back(od);
  if ((st = c->upload_objects()) != RKF_OK) return st;
  undo.dismiss();
  c->epoch++;
  if (out_object_index) *out_object_index = c->obj_count() - 1;
  return RKF_OK;
}
