// oracle.cpp — CPU oracle for the RKIField SDF ray-march path.
//
// TEST INFRASTRUCTURE ONLY: this is the checker (and the timed CPU baseline)
// for the CUDA kernels.  The product library never links or calls it.
//
// Build: g++ -O2 -ffp-contract=off -fno-fast-math (see oracle/Makefile).  No
// contraction and IEEE single precision on x86-64 SSE give the exact FP32
// operation sequence the reference shader states.
//
// Operation order rules used throughout (the WGSL spec definitions):
//   mix(a,b,t)   = a*(1-t) + b*t
//   clamp(x,l,h) = min(max(x,l),h)
//   length(v)    = sqrt((v.x*v.x + v.y*v.y) + v.z*v.z)
//   dot(a,b)     = (a.x*b.x + a.y*b.y) + a.z*b.z
//   normalize(v) = v / length(v)
//   M * v (mat4, column-major m[c][r]) : r_i = ((m0i*x + m1i*y) + m2i*z) + m3i*w
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr float kMaxFloat = 3.402823e+38f;  // ray_march.wgsl:27

// ---------------------------------------------------------------------------
// binary16 (IEEE-754), round-to-nearest-even — the `half` crate's from_f32 /
// to_f32 used by VoxelSample::new (crates/rkf-core/src/voxel.rs:33).
// ---------------------------------------------------------------------------
uint16_t f16_from_f32(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) {  // inf / nan
    if (ax == 0x7f800000u) return static_cast<uint16_t>(sign | 0x7c00u);
    return static_cast<uint16_t>(sign | 0x7e00u | ((ax >> 13) & 0x3ffu));
  }
  if (ax >= 0x47800000u) return static_cast<uint16_t>(sign | 0x7c00u);  // >= 65536
  if (ax >= 0x38800000u) {  // normal half range (>= 2^-14)
    const uint32_t e = (ax >> 23) - 127 + 15;
    const uint32_t mant = ax & 0x7fffffu;
    uint32_t h = (e << 10) | (mant >> 13);
    const uint32_t rem = mant & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;  // carry may reach inf
    return static_cast<uint16_t>(sign | h);
  }
  // subnormal half: value / 2^-24 rounded to nearest even
  const int e = static_cast<int>(ax >> 23);
  if (e == 0) return static_cast<uint16_t>(sign);
  const uint32_t m = (ax & 0x7fffffu) | 0x800000u;
  const int shift = 126 - e;
  if (shift > 24) return static_cast<uint16_t>(sign);
  uint32_t h = m >> shift;
  const uint32_t rem = m & ((1u << shift) - 1u);
  const uint32_t half = 1u << (shift - 1);
  if (rem > half || (rem == half && (h & 1u))) h++;
  return static_cast<uint16_t>(sign | h);
}

float f16_to_f32(uint16_t h) {
  const uint32_t sign = (static_cast<uint32_t>(h) & 0x8000u) << 16;
  const uint32_t e = (h >> 10) & 0x1fu;
  const uint32_t m = h & 0x3ffu;
  uint32_t x;
  if (e == 0) {
    if (m == 0) {
      x = sign;
    } else {  // subnormal: m * 2^-24, exact in f32
      float v = static_cast<float>(m) * 5.9604644775390625e-08f;
      std::memcpy(&x, &v, 4);
      x |= sign;
    }
  } else if (e == 31) {
    x = sign | 0x7f800000u | (m << 13);
  } else {
    x = sign | ((e - 15 + 127) << 23) | (m << 13);
  }
  float f;
  std::memcpy(&f, &x, 4);
  return f;
}

// ---------------------------------------------------------------------------
// Small vector helpers with the stated operation order.
// ---------------------------------------------------------------------------
template <class R>
struct V3 {
  R x, y, z;
};
template <class R>
inline V3<R> v3(R x, R y, R z) { return V3<R>{x, y, z}; }
template <class R>
inline V3<R> add(V3<R> a, V3<R> b) { return v3<R>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class R>
inline V3<R> sub(V3<R> a, V3<R> b) { return v3<R>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class R>
inline V3<R> mul(V3<R> a, R s) { return v3<R>(a.x * s, a.y * s, a.z * s); }
template <class R>
inline R dot(V3<R> a, V3<R> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class R>
inline R length(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R>
inline R fmin_(R a, R b) { return b < a ? b : a; }  // WGSL min on non-NaN
template <class R>
inline R fmax_(R a, R b) { return a < b ? b : a; }
template <class R>
inline R clampf(R x, R lo, R hi) { return fmin_(fmax_(x, lo), hi); }
template <class R>
inline R mixf(R a, R b, R t) { return a * (R(1) - t) + b * t; }

// ---------------------------------------------------------------------------
// Analytic SDFs of the synthetic scene (crates/rkf-core/src/sdf.rs:12-51).
// ---------------------------------------------------------------------------
template <class R>
R prim_sdf(const rkf_prim& p, R px, R py, R pz) {
  const R dx = px - R(p.centre[0]);
  const R dy = py - R(p.centre[1]);
  const R dz = pz - R(p.centre[2]);
  if (p.type == RKF_PRIM_SPHERE) {  // sphere_sdf, sdf.rs:12-15
    return std::sqrt((dx * dx + dy * dy) + dz * dz) - R(p.params[0]);
  }
  // local = R^T (p - c); rot is row-major
  const float* m = p.rot;
  const R lx = (R(m[0]) * dx + R(m[3]) * dy) + R(m[6]) * dz;
  const R ly = (R(m[1]) * dx + R(m[4]) * dy) + R(m[7]) * dz;
  const R lz = (R(m[2]) * dx + R(m[5]) * dy) + R(m[8]) * dz;
  if (p.type == RKF_PRIM_BOX) {  // box_sdf, sdf.rs:33-38
    const R qx = std::fabs(lx) - R(p.params[0]);
    const R qy = std::fabs(ly) - R(p.params[1]);
    const R qz = std::fabs(lz) - R(p.params[2]);
    const R ox = fmax_(qx, R(0)), oy = fmax_(qy, R(0)), oz = fmax_(qz, R(0));
    const R outside = std::sqrt((ox * ox + oy * oy) + oz * oz);
    const R inside = fmin_(fmax_(qx, fmax_(qy, qz)), R(0));
    return outside + inside;
  }
  // capsule_sdf(a=(0,-h,0), b=(0,h,0), r), sdf.rs:21-26
  const R h = R(p.params[1]);
  const V3<R> a = v3<R>(R(0), -h, R(0));
  const V3<R> b = v3<R>(R(0), h, R(0));
  const V3<R> pa = sub(v3<R>(lx, ly, lz), a);
  const V3<R> ba = sub(b, a);
  const R hh = clampf(dot(pa, ba) / dot(ba, ba), R(0), R(1));
  return length(sub(pa, mul(ba, hh))) - R(p.params[0]);
}

template <class R>
R smin(R a, R b, R k) {  // sdf.rs:48-51
  const R h = fmax_(k - std::fabs(a - b), R(0)) / k;
  return fmin_(a, b) - h * h * k * R(0.25);
}

// Scene distance: smooth-min fold, in ascending primitive order, over the
// primitives whose bounding sphere is nearer than `cut`.  Material = the
// nearest primitive's; secondary/blend from the runner-up when within k.
template <class R>
R scene_eval(const rkf_prim* prims, const uint32_t* cand, uint32_t ncand, R k, R cut,
             R px, R py, R pz, uint32_t* mat, uint32_t* sec, uint32_t* blend) {
  R acc = R(INFINITY);
  R best = R(INFINITY), second = R(INFINITY);
  int bi = -1, si = -1;
  for (uint32_t c = 0; c < ncand; ++c) {
    const uint32_t i = cand ? cand[c] : c;
    const rkf_prim& p = prims[i];
    const R dx = px - R(p.centre[0]);
    const R dy = py - R(p.centre[1]);
    const R dz = pz - R(p.centre[2]);
    const R lb = std::sqrt((dx * dx + dy * dy) + dz * dz) - R(p.bound_radius);
    if (!(lb < cut)) continue;
    const R d = prim_sdf<R>(p, px, py, pz);
    acc = smin<R>(acc, d, k);
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
  if (mat) *mat = bi >= 0 ? prims[bi].material : 0u;
  if (sec) {
    *sec = 0u;
    *blend = 0u;
    if (si >= 0 && second - best < k) {
      const R w = R(0.5) * (R(1) - (second - best) / k);
      *sec = prims[si].material;
      *blend = static_cast<uint32_t>(std::floor(w * R(255) + R(0.5)));
    }
  }
  return acc;
}

uint32_t pack_word0(float d, uint32_t mat, uint32_t sec) {  // voxel.rs:44-52
  return static_cast<uint32_t>(f16_from_f32(d)) | ((mat & 0x3Fu) << 16) | ((sec & 0x3Fu) << 22);
}

// ---------------------------------------------------------------------------
// Voxelizer (crates/rkf-core/src/voxelize_object.rs:53-182)
// ---------------------------------------------------------------------------
struct Grid {
  uint32_t dims[3];
  float vs, bws, origin[3];
};

Grid make_grid(const rkf_voxelize_params* vp) {
  Grid g;
  g.vs = vp->voxel_size;
  g.bws = vp->voxel_size * 8.0f;  // voxelize_object.rs:63
  for (int a = 0; a < 3; ++a) {
    const float size = vp->aabb_max[a] - vp->aabb_min[a];
    uint32_t d = static_cast<uint32_t>(std::ceil(size / g.bws));
    g.dims[a] = d < 1 ? 1 : d;  // :67-71
    g.origin[a] = -((static_cast<float>(g.dims[a]) * g.bws) * 0.5f);  // :77-81
  }
  return g;
}

// Candidate primitives of a brick: every primitive whose bounding sphere
// grown by `cut` reaches the brick's box (plus a margin).  The per-point cut
// test inside scene_eval keeps the result identical to a fold over all
// primitives.
void brick_candidates(const rkf_prim* prims, uint32_t n, const float bmin[3], float bws,
                      float cut, std::vector<uint32_t>& out) {
  out.clear();
  for (uint32_t i = 0; i < n; ++i) {
    double d2 = 0.0;
    for (int a = 0; a < 3; ++a) {
      const double lo = bmin[a], hi = static_cast<double>(bmin[a]) + bws;
      const double c = prims[i].centre[a];
      const double e = c < lo ? lo - c : (c > hi ? c - hi : 0.0);
      d2 += e * e;
    }
    const double reach = static_cast<double>(prims[i].bound_radius) + cut + 0.05 * bws + 1e-3;
    if (d2 < reach * reach) out.push_back(i);
  }
}

struct BrickResult {
  uint32_t cls;  // 0 allocated, 1 EMPTY, 2 INTERIOR
  uint32_t words[1024];
  float dist[512];
};

void brick_min_of(const Grid& g, uint32_t bx, uint32_t by, uint32_t bz, float out[3]) {
  // brick_min = grid_origin + (b * bws)   (voxelize_object.rs:92-97)
  out[0] = g.origin[0] + static_cast<float>(bx) * g.bws;
  out[1] = g.origin[1] + static_cast<float>(by) * g.bws;
  out[2] = g.origin[2] + static_cast<float>(bz) * g.bws;
}

void classify_brick(const rkf_prim* prims, uint32_t n, const rkf_voxelize_params* vp,
                    const Grid& g, uint32_t bx, uint32_t by, uint32_t bz,
                    std::vector<uint32_t>& cand, BrickResult& r) {
  float bmin[3];
  brick_min_of(g, bx, by, bz, bmin);
  const float k = vp->smooth_k, cut = vp->cut_distance;
  brick_candidates(prims, n, bmin, g.bws, cut, cand);
  const float hb = g.bws * 0.5f;
  const float cx = bmin[0] + hb, cy = bmin[1] + hb, cz = bmin[2] + hb;  // :98
  const float dc = scene_eval<float>(prims, cand.data(), static_cast<uint32_t>(cand.size()), k,
                                     cut, cx, cy, cz, nullptr, nullptr, nullptr);
  if (vp->band_rule == RKF_BAND_REFERENCE) {
    if (!(std::fabs(dc) < g.bws * 1.8f)) {  // :86,100-101
      r.cls = 1;
      return;
    }
  } else {
    const float band = vp->band_voxels * g.vs;
    const float thr = (band + g.bws * 0.8660254f) + g.vs;
    if (!(std::fabs(dc) <= thr)) {
      r.cls = dc > 0.0f ? 1u : 2u;
      return;
    }
  }
  // populate_brick (voxelize_object.rs:160-182): voxel centres
  const float half_voxel = g.vs * 0.5f;
  bool any_band = false, all_pos = true, all_neg = true;
  const float band = vp->band_voxels * g.vs;
  for (uint32_t vz = 0; vz < 8; ++vz)
    for (uint32_t vy = 0; vy < 8; ++vy)
      for (uint32_t vx = 0; vx < 8; ++vx) {
        const float px = bmin[0] + (static_cast<float>(vx) * g.vs + half_voxel);
        const float py = bmin[1] + (static_cast<float>(vy) * g.vs + half_voxel);
        const float pz = bmin[2] + (static_cast<float>(vz) * g.vs + half_voxel);
        uint32_t mat, sec, blend;
        const float d = scene_eval<float>(prims, cand.data(), static_cast<uint32_t>(cand.size()),
                                          k, cut, px, py, pz, &mat, &sec, &blend);
        const uint32_t idx = vx + vy * 8 + vz * 64;
        r.dist[idx] = d;
        if (vp->band_rule == RKF_BAND_REFERENCE) {  // VoxelSample::new(d, mat, 0) (:180)
          sec = 0;
          blend = 0;
        }
        r.words[2 * idx] = pack_word0(d, mat, sec);
        r.words[2 * idx + 1] = blend << 24;
        if (std::fabs(d) <= band) any_band = true;
        if (!(d > 0.0f)) all_pos = false;
        if (!(d < 0.0f)) all_neg = false;
      }
  if (vp->band_rule == RKF_BAND_REFERENCE || any_band) {
    r.cls = 0;
  } else if (all_pos) {
    r.cls = 1;
  } else if (all_neg) {
    r.cls = 2;
  } else {
    r.cls = 0;
  }
}

template <class F>
void parallel_for(uint64_t n, int threads, F&& f) {
  if (threads <= 1 || n < 64) {
    for (uint64_t i = 0; i < n; ++i) f(i, 0);
    return;
  }
  std::atomic<uint64_t> next{0};
  const uint64_t chunk = std::max<uint64_t>(1, n / (static_cast<uint64_t>(threads) * 64));
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&, t] {
      for (;;) {
        const uint64_t b = next.fetch_add(chunk);
        if (b >= n) break;
        const uint64_t e = std::min(n, b + chunk);
        for (uint64_t i = b; i < e; ++i) f(i, t);
      }
    });
  }
  for (auto& th : pool) th.join();
}

}  // namespace

struct orc_voxelized {
  Grid g;
  std::vector<uint32_t> map;
  std::vector<uint32_t> words;
  std::vector<float> dist;
  uint32_t n_bricks = 0, n_interior = 0;
};

// ---------------------------------------------------------------------------
// March restatement (crates/rkf-render/shaders/ray_march.wgsl)
// ---------------------------------------------------------------------------
namespace {

struct Tracker {  // distinct 32-byte sectors touched by one ray
  std::vector<uint64_t> keys;
  bool on = false;
  void touch(uint64_t plane, uint64_t byte_addr) {
    if (on) keys.push_back((plane << 56) | (byte_addr >> 5));
  }
};

// ---------------------------------------------------------------------------
// Tiled strategy inputs: the coarse acceleration field and the per-tile object
// lists.
// ---------------------------------------------------------------------------
// CoarseField (crates/rkf-render/src/coarse_field.rs): cells of 0.32 m
// (COARSE_VOXEL_SIZE, :21) over the union of the objects' AABBs grown by the
// runtime's 1 m margin (from_scene_aabbs, :211-232; render.rs:257-263), at
// most 128 per axis (:24, :93-97); each texel is the binary16 of the smallest
// unsigned distance from the cell centre to an object AABB, starting from
// vs * max(dims) (populate, :240-266; aabb_unsigned_distance, :72-79).
struct CoarseField {
  float origin[3];
  uint32_t dims[3];
  float vs, inv_vs;
  std::vector<uint16_t> tex;  // x + y*dx + z*dx*dy
};

CoarseField coarse_build(const orc_scene* s) {
  CoarseField c;
  c.vs = 0.32f;
  const float margin = 1.0f;
  float lo[3], hi[3];
  if (s->num_objects == 0) {
    for (int a = 0; a < 3; ++a) lo[a] = 0.0f, hi[a] = c.vs;
  } else {
    for (int a = 0; a < 3; ++a) lo[a] = FLT_MAX, hi[a] = -FLT_MAX;
    for (uint32_t i = 0; i < s->num_objects; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::fmin(lo[a], s->objects[i].aabb_min[a]);
        hi[a] = std::fmax(hi[a], s->objects[i].aabb_max[a]);
      }
  }
  for (int a = 0; a < 3; ++a) {
    c.origin[a] = lo[a] - margin;
    const float extent = (hi[a] + margin) - c.origin[a];
    const float cells = std::fmin(std::ceil(extent / c.vs), 128.0f);  // ceil() as u32, .min(128).max(1)
    c.dims[a] = std::max<uint32_t>(1u, cells > 0.0f ? static_cast<uint32_t>(cells) : 0u);
  }
  c.inv_vs = 1.0f / c.vs;
  const uint32_t dmax = std::max(c.dims[0], std::max(c.dims[1], c.dims[2]));
  const float start = c.vs * static_cast<float>(dmax);
  c.tex.resize(static_cast<size_t>(c.dims[0]) * c.dims[1] * c.dims[2]);
  for (uint32_t z = 0; z < c.dims[2]; ++z)
    for (uint32_t y = 0; y < c.dims[1]; ++y)
      for (uint32_t x = 0; x < c.dims[0]; ++x) {
        const float q[3] = {c.origin[0] + (static_cast<float>(x) + 0.5f) * c.vs,
                            c.origin[1] + (static_cast<float>(y) + 0.5f) * c.vs,
                            c.origin[2] + (static_cast<float>(z) + 0.5f) * c.vs};
        float best = start;
        for (uint32_t i = 0; i < s->num_objects; ++i) {
          const rkf_gpu_object& o = s->objects[i];
          float d3[3];
          for (int a = 0; a < 3; ++a) {
            const float e = std::fmax(o.aabb_min[a] - q[a], q[a] - o.aabb_max[a]);
            d3[a] = std::fmax(e, 0.0f);
          }
          const float d = std::sqrt((d3[0] * d3[0] + d3[1] * d3[1]) + d3[2] * d3[2]);
          best = std::fmin(best, d);
        }
        c.tex[x + y * static_cast<size_t>(c.dims[0]) + z * static_cast<size_t>(c.dims[0]) * c.dims[1]] =
            f16_from_f32(best);
      }
  return c;
}

// sample_coarse_field (ray_march.wgsl:228-235): uvw = (cam_rel - origin_cam_rel)
// * inv_voxel_size / dims, 0 outside [0,1]^3, else a linearly filtered,
// clamp-to-edge read of the R16Float texture.  The filter is a model of the
// texture unit: texel coordinate u*N - 0.5, its fraction quantised to 1/256
// (the 8 fractional weight bits NVIDIA documents for linear filtering), then
// mix(a, b, w) along x, y and z.  The reference's value comes from that
// hardware and cannot be pinned here.
float coarse_sample(const CoarseField& c, const float ocr[3], float cx, float cy, float cz) {
  const float cr[3] = {cx, cy, cz};
  int i0[3], i1[3];
  float w[3];
  for (int a = 0; a < 3; ++a) {
    const float u = ((cr[a] - ocr[a]) * c.inv_vs) / static_cast<float>(c.dims[a]);
    if (u < 0.0f || u > 1.0f) return 0.0f;
    const float x = u * static_cast<float>(c.dims[a]) - 0.5f;
    const float f = std::floor(x);
    w[a] = std::nearbyint((x - f) * 256.0f) * 0.00390625f;
    const int n = static_cast<int>(c.dims[a]);
    const int k = static_cast<int>(f);
    i0[a] = std::min(std::max(k, 0), n - 1);
    i1[a] = std::min(std::max(k + 1, 0), n - 1);
  }
  const size_t sx = 1, sy = c.dims[0], sz = static_cast<size_t>(c.dims[0]) * c.dims[1];
  auto T = [&](int x, int y, int z) { return f16_to_f32(c.tex[x * sx + y * sy + z * sz]); };
  const float c00 = mixf(T(i0[0], i0[1], i0[2]), T(i1[0], i0[1], i0[2]), w[0]);
  const float c10 = mixf(T(i0[0], i1[1], i0[2]), T(i1[0], i1[1], i0[2]), w[0]);
  const float c01 = mixf(T(i0[0], i0[1], i1[2]), T(i1[0], i0[1], i1[2]), w[0]);
  const float c11 = mixf(T(i0[0], i1[1], i1[2]), T(i1[0], i1[1], i1[2]), w[0]);
  return mixf(mixf(c00, c10, w[1]), mixf(c01, c11, w[1]), w[2]);
}

// tile_object_cull.wgsl:90-205: per 16x16-pixel tile, the objects whose
// projected AABB overlaps it (all 8 corners in front: screen rectangle test;
// straddling the camera plane: always; all behind: never), at most 32.  The
// shader appends with a shared-memory atomic, so its order (and, beyond 32,
// its choice) is unspecified; here it is ascending object index.  The screen
// is the view's size (the reference sizes its tiles and its G-buffer from
// the same resolution).
void tile_cull(const orc_scene* s, const rkf_camera* cam, uint32_t w, uint32_t h, std::vector<uint32_t>& cnt,
               std::vector<uint32_t>& list, uint32_t* tiles_x) {
  const float resx = static_cast<float>(w), resy = static_cast<float>(h);
  const uint32_t ntx = static_cast<uint32_t>(std::ceil(resx / 16.0f));
  const uint32_t nty = static_cast<uint32_t>(std::ceil(resy / 16.0f));
  *tiles_x = ntx;
  cnt.assign(static_cast<size_t>(ntx) * nty, 0);
  list.assign(static_cast<size_t>(ntx) * nty * 32, 0);
  const V3<float> fwd = v3<float>(cam->forward[0], cam->forward[1], cam->forward[2]);
  const V3<float> rt = v3<float>(cam->right[0], cam->right[1], cam->right[2]);
  const V3<float> up = v3<float>(cam->up[0], cam->up[1], cam->up[2]);
  const V3<float> cp = v3<float>(cam->position[0], cam->position[1], cam->position[2]);
  const float r_sq = dot(rt, rt), u_sq = dot(up, up);
  for (uint32_t ty = 0; ty < nty; ++ty)
    for (uint32_t tx = 0; tx < ntx; ++tx) {
      const float tminx = static_cast<float>(tx * 16), tminy = static_cast<float>(ty * 16);
      const float tmaxx = tminx + 16.0f, tmaxy = tminy + 16.0f;
      uint32_t n = 0;
      const size_t tile = static_cast<size_t>(ty) * ntx + tx;
      for (uint32_t i = 0; i < s->num_objects; ++i) {
        const rkf_gpu_object& o = s->objects[i];
        if (o.sdf_type == RKF_SDF_NONE) continue;
        float smin_x = resx, smin_y = resy, smax_x = 0.0f, smax_y = 0.0f;
        bool front = false, behind = false;
        for (uint32_t c = 0; c < 8; ++c) {
          const V3<float> corner = v3<float>((c & 1u) ? o.aabb_max[0] : o.aabb_min[0],
                                             (c & 2u) ? o.aabb_max[1] : o.aabb_min[1],
                                             (c & 4u) ? o.aabb_max[2] : o.aabb_min[2]);
          const V3<float> rel = sub(corner, cp);
          const float depth = dot(rel, fwd);
          if (depth > 0.0f) {
            const float ndc_x = dot(rel, rt) / (depth * r_sq);
            const float ndc_y = dot(rel, up) / (depth * u_sq);
            const float px = (ndc_x * 0.5f + 0.5f) * resx;
            const float py = (0.5f - ndc_y * 0.5f) * resy;
            front = true;
            smin_x = fmin_(smin_x, px), smin_y = fmin_(smin_y, py);
            smax_x = fmax_(smax_x, px), smax_y = fmax_(smax_y, py);
          } else {
            behind = true;
          }
        }
        bool overlaps = false;
        if (behind && front) overlaps = true;
        else if (!behind && front)
          overlaps = smax_x >= tminx && smin_x < tmaxx && smax_y >= tminy && smin_y < tmaxy;
        if (overlaps && n < 32) list[tile * 32 + n++] = i;
      }
      cnt[tile] = n;
    }
}

// The tiled strategy's per-ray inputs.
struct TiledRay {
  const CoarseField* cf;
  float ocr[3];        // field origin relative to the camera (CoarseField::upload, :297-305)
  float cam[3];        // camera.position
  const uint32_t* list;
  uint32_t count;
};

template <class R>
struct Marcher {
  const orc_scene* s;
  Tracker* tr;
  double* margin;  // smallest distance of an FP decision to its threshold

  void note(R a, R b) {
    if (margin) {
      const double m = std::fabs(static_cast<double>(a) - static_cast<double>(b));
      if (m < *margin) *margin = m;
    }
  }

  uint32_t lookup(const rkf_gpu_object& o, uint32_t oi, uint32_t bx, uint32_t by, uint32_t bz) {
    if (s->brick_maps) {  // brick_maps[offset + bx + by*dx + bz*dx*dy] (ray_march.wgsl:276-277)
      const uint64_t a = static_cast<uint64_t>(o.brick_map_offset) + bx +
                         static_cast<uint64_t>(by) * o.brick_map_dims[0] +
                         static_cast<uint64_t>(bz) * o.brick_map_dims[0] * o.brick_map_dims[1];
      tr->touch(0, a * 4);
      return s->brick_maps[a];
    }
    // two-level: top grid of 8^3-brick blocks, then a 512-entry leaf
    const uint32_t* info = s->obj_top_info + 4 * oi;
    const uint64_t ti = static_cast<uint64_t>(info[0]) + (bx >> 3) +
                        static_cast<uint64_t>(by >> 3) * info[1] +
                        static_cast<uint64_t>(bz >> 3) * info[1] * info[2];
    tr->touch(0, ti * 4);
    const uint32_t t = s->top[ti];
    if (t == RKF_EMPTY_SLOT || t == RKF_INTERIOR_SLOT) return t;
    const uint64_t li = static_cast<uint64_t>(t) * 512 + (bx & 7) + (by & 7) * 8 + (bz & 7) * 64;
    tr->touch(3, li * 4);
    return s->leaves[li];
  }

  R dist(uint32_t slot, uint32_t idx) {
    const uint64_t v = static_cast<uint64_t>(slot) * 512 + idx;
    if (s->pool_words) {
      tr->touch(1, v * 2);
      return R(f16_to_f32(static_cast<uint16_t>(s->pool_words[2 * v] & 0xFFFFu)));
    }
    switch (s->precision) {
      case RKF_PRECISION_F32:
        tr->touch(1, v * 4);
        return R(s->dist_f32[v]);
      case RKF_PRECISION_U8:
        tr->touch(1, v);
        return R(static_cast<float>(s->dist_u8[v])) * R(s->brick_scale[slot]);
      case ORC_PRECISION_F64:  // analytic values at voxel centres (error reference)
        tr->touch(1, v * 8);
        return R(s->dist_f64[v]);
      default:
        tr->touch(1, v * 2);
        return R(f16_to_f32(s->dist_f16[v]));
    }
  }
  uint32_t mat_word(uint32_t slot, uint32_t idx) {  // mat | sec<<6
    const uint64_t v = static_cast<uint64_t>(slot) * 512 + idx;
    tr->touch(2, v * 2);
    if (s->pool_words) {
      const uint32_t w0 = s->pool_words[2 * v];
      return ((w0 >> 16) & 0x3Fu) | (((w0 >> 22) & 0x3Fu) << 6);
    }
    return s->mat_plane[v];
  }
  uint32_t blend_of(uint32_t slot, uint32_t idx) {
    const uint64_t v = static_cast<uint64_t>(slot) * 512 + idx;
    if (s->pool_words) return (s->pool_words[2 * v + 1] >> 24) & 0xFFu;
    return s->blend_plane[v];
  }

  // sample_voxel_at / sample_voxel_at_grad (ray_march.wgsl:270-315)
  R voxel_at(const rkf_gpu_object& o, uint32_t oi, int vx, int vy, int vz, int tx, int ty,
             int tz, R vs, bool grad) {
    const int cx = std::min(std::max(vx, 0), tx - 1);
    const int cy = std::min(std::max(vy, 0), ty - 1);
    const int cz = std::min(std::max(vz, 0), tz - 1);
    const uint32_t slot = lookup(o, oi, cx / 8, cy / 8, cz / 8);
    if (slot == RKF_EMPTY_SLOT) return vs * R(8);
    if (slot == RKF_INTERIOR_SLOT) return -(vs * (grad ? R(8) : R(2)));
    return dist(slot, static_cast<uint32_t>((cx % 8) + (cy % 8) * 8 + (cz % 8) * 64));
  }

  // sample_voxelized (:353-413) and sample_voxelized_grad (:463-498)
  R voxelized(const rkf_gpu_object& o, uint32_t oi, V3<R> lp, bool grad) {
    const R vs = R(o.voxel_size);
    const R be = vs * R(8);
    const V3<R> gs = v3<R>(R(static_cast<float>(o.brick_map_dims[0])) * be,
                           R(static_cast<float>(o.brick_map_dims[1])) * be,
                           R(static_cast<float>(o.brick_map_dims[2])) * be);
    const V3<R> gp = add(lp, mul(gs, R(0.5)));
    const R lo = vs * R(0.01f);
    const V3<R> cl = v3<R>(clampf(gp.x, lo, gs.x - lo), clampf(gp.y, lo, gs.y - lo),
                           clampf(gp.z, lo, gs.z - lo));
    const R outside = length(sub(gp, cl));
    note(outside, be * R(2));
    if (outside > be * R(2)) return outside;
    if (!grad && o.geometry_aabb_max[0] > o.geometry_aabb_min[0]) {
      const V3<R> gc = v3<R>(clampf(lp.x, R(o.geometry_aabb_min[0]), R(o.geometry_aabb_max[0])),
                             clampf(lp.y, R(o.geometry_aabb_min[1]), R(o.geometry_aabb_max[1])),
                             clampf(lp.z, R(o.geometry_aabb_min[2]), R(o.geometry_aabb_max[2])));
      const R gd = length(sub(lp, gc));
      note(gd, be);
      if (gd > be) return gd;
    }
    const V3<R> vc = v3<R>(cl.x / vs - R(0.5), cl.y / vs - R(0.5), cl.z / vs - R(0.5));
    const int x0 = static_cast<int>(std::floor(vc.x));
    const int y0 = static_cast<int>(std::floor(vc.y));
    const int z0 = static_cast<int>(std::floor(vc.z));
    const R tx = vc.x - R(static_cast<float>(x0));
    const R ty = vc.y - R(static_cast<float>(y0));
    const R tz = vc.z - R(static_cast<float>(z0));
    const int TX = static_cast<int>(o.brick_map_dims[0]) * 8;
    const int TY = static_cast<int>(o.brick_map_dims[1]) * 8;
    const int TZ = static_cast<int>(o.brick_map_dims[2]) * 8;
    const R c000 = voxel_at(o, oi, x0, y0, z0, TX, TY, TZ, vs, grad);
    const R c100 = voxel_at(o, oi, x0 + 1, y0, z0, TX, TY, TZ, vs, grad);
    const R c010 = voxel_at(o, oi, x0, y0 + 1, z0, TX, TY, TZ, vs, grad);
    const R c110 = voxel_at(o, oi, x0 + 1, y0 + 1, z0, TX, TY, TZ, vs, grad);
    const R c001 = voxel_at(o, oi, x0, y0, z0 + 1, TX, TY, TZ, vs, grad);
    const R c101 = voxel_at(o, oi, x0 + 1, y0, z0 + 1, TX, TY, TZ, vs, grad);
    const R c011 = voxel_at(o, oi, x0, y0 + 1, z0 + 1, TX, TY, TZ, vs, grad);
    const R c111 = voxel_at(o, oi, x0 + 1, y0 + 1, z0 + 1, TX, TY, TZ, vs, grad);
    const R c00 = mixf(c000, c100, tx);
    const R c10 = mixf(c010, c110, tx);
    const R c01 = mixf(c001, c101, tx);
    const R c11 = mixf(c011, c111, tx);
    const R c0 = mixf(c00, c10, ty);
    const R c1 = mixf(c01, c11, ty);
    return mixf(c0, c1, tz) + outside;
  }

  // nearest-voxel lookup shared by sample_voxelized_material (:540-566) and
  // sample_voxelized_blend_data (:570-596); returns the slot or a sentinel.
  uint32_t nearest(const rkf_gpu_object& o, uint32_t oi, V3<R> lp, uint32_t* idx_out) {
    const R vs = R(o.voxel_size);
    const R be = vs * R(8);
    const V3<R> gs = v3<R>(R(static_cast<float>(o.brick_map_dims[0])) * be,
                           R(static_cast<float>(o.brick_map_dims[1])) * be,
                           R(static_cast<float>(o.brick_map_dims[2])) * be);
    const V3<R> gp = add(lp, mul(gs, R(0.5)));
    if (gp.x < R(0) || gp.y < R(0) || gp.z < R(0) || gp.x >= gs.x || gp.y >= gs.y ||
        gp.z >= gs.z)
      return RKF_EMPTY_SLOT;
    const int TX = static_cast<int>(o.brick_map_dims[0]) * 8;
    const int TY = static_cast<int>(o.brick_map_dims[1]) * 8;
    const int TZ = static_cast<int>(o.brick_map_dims[2]) * 8;
    const int x = std::min(std::max(static_cast<int>(std::floor(gp.x / vs)), 0), TX - 1);
    const int y = std::min(std::max(static_cast<int>(std::floor(gp.y / vs)), 0), TY - 1);
    const int z = std::min(std::max(static_cast<int>(std::floor(gp.z / vs)), 0), TZ - 1);
    const uint32_t slot = lookup(o, oi, x / 8, y / 8, z / 8);
    *idx_out = static_cast<uint32_t>((x % 8) + (y % 8) * 8 + (z % 8) * 64);
    return slot;
  }

  uint32_t material(const rkf_gpu_object& o, uint32_t oi, V3<R> lp) {
    uint32_t idx = 0;
    const uint32_t slot = nearest(o, oi, lp, &idx);
    if (slot == RKF_EMPTY_SLOT || slot == RKF_INTERIOR_SLOT) return 0u;
    return mat_word(slot, idx) & 0x3Fu;
  }

  static R analytic(const rkf_gpu_object& o, V3<R> p) {  // ray_march.wgsl:182-264
    const R a0 = R(o.sdf_params[0]), a1 = R(o.sdf_params[1]), a2 = R(o.sdf_params[2]);
    switch (o.primitive_type) {
      case RKF_PRIM_SPHERE:
        return length(p) - a0;
      case RKF_PRIM_BOX: {
        const V3<R> q = v3<R>(std::fabs(p.x) - a0, std::fabs(p.y) - a1, std::fabs(p.z) - a2);
        const V3<R> mq = v3<R>(fmax_(q.x, R(0)), fmax_(q.y, R(0)), fmax_(q.z, R(0)));
        return length(mq) + fmin_(fmax_(q.x, fmax_(q.y, q.z)), R(0));
      }
      case RKF_PRIM_CAPSULE: {
        const V3<R> q = v3<R>(p.x, fmax_(std::fabs(p.y) - a1, R(0)), p.z);
        return length(q) - a0;
      }
      case RKF_PRIM_TORUS: {
        const R qx = std::sqrt(p.x * p.x + p.z * p.z) - a0;
        return std::sqrt(qx * qx + p.y * p.y) - a1;
      }
      case RKF_PRIM_CYLINDER: {
        const R dx = std::sqrt(p.x * p.x + p.z * p.z) - a0;
        const R dy = std::fabs(p.y) - a1;
        const R mx = fmax_(dx, R(0)), my = fmax_(dy, R(0));
        return fmin_(fmax_(dx, dy), R(0)) + std::sqrt(mx * mx + my * my);
      }
      case RKF_PRIM_PLANE: {
        const V3<R> n = v3<R>(a0, a1, a2);
        const R l = length(n);
        const V3<R> nn = v3<R>(n.x / l, n.y / l, n.z / l);
        return dot(p, nn) + R(0);
      }
      default:
        return R(kMaxFloat);
    }
  }

  static V3<R> to_local(const rkf_gpu_object& o, V3<R> w) {
    const float* m = o.inverse_world;  // column-major m[c*4 + r]
    return v3<R>(((R(m[0]) * w.x + R(m[4]) * w.y) + R(m[8]) * w.z) + R(m[12]) * R(1),
                 ((R(m[1]) * w.x + R(m[5]) * w.y) + R(m[9]) * w.z) + R(m[13]) * R(1),
                 ((R(m[2]) * w.x + R(m[6]) * w.y) + R(m[10]) * w.z) + R(m[14]) * R(1));
  }

  // evaluate_object (:600-634).  with_mat=false is evaluate_object_dist
  // (shade_common.wgsl:486-500).
  R evaluate(V3<R> wp, uint32_t oi, uint32_t* mat, bool with_mat = true) {
    const rkf_gpu_object& o = s->objects[oi];
    if (o.sdf_type == RKF_SDF_NONE) {
      *mat = 0;
      return R(kMaxFloat);
    }
    const V3<R> lp = to_local(o, wp);
    R d;
    if (o.sdf_type == RKF_SDF_ANALYTICAL) {
      d = analytic(o, lp);
      *mat = o.material_id;
    } else {
      d = voxelized(o, oi, lp, false);
      *mat = 0;
      if (with_mat) {
        note(d, R(o.voxel_size) * R(16));
        if (d < R(o.voxel_size) * R(16)) *mat = material(o, oi, lp);
      }
    }
    const R ms = fmin_(R(o.accumulated_scale[0]),
                       fmin_(R(o.accumulated_scale[1]), R(o.accumulated_scale[2])));
    return d * ms;
  }

  struct Result {
    R t;
    bool hit;
    bool bisected;
    bool out_of_steps;
    uint32_t mat, obj_id, obj_idx;
  };

  // ray_march_brute (:776-858), or ray_march_bvh (:641-773) when the
  // strategy is BVH, or ray_march_tiled (:874-985) when tl is given.  The
  // three differ only in the objects a step evaluates and their order.
  // any_hit stops at the first surface contact without bisecting.
  Result march(V3<R> origin, V3<R> dir, const rkf_march_params* p, R max_distance,
               bool any_hit, uint64_t* steps_out, const TiledRay* tl = nullptr) {
    Result r{R(kMaxFloat), false, false, false, 0, 0, 0};
    // ray_march_tiled (:874-985): a tile with no objects is sky
    if (tl && tl->count == 0) return r;
    const V3<R> sd = v3<R>(std::fabs(dir.x) < R(1e-10f) ? R(1e-10f) : dir.x,
                           std::fabs(dir.y) < R(1e-10f) ? R(1e-10f) : dir.y,
                           std::fabs(dir.z) < R(1e-10f) ? R(1e-10f) : dir.z);
    const R hit_thr = R(p->scene.hit_threshold);
    const R near_thr = R(p->near_surface_threshold);
    const R min_step = R(p->min_step);
    const bool use_bvh = p->strategy == RKF_STRATEGY_BVH && s->bvh && s->bvh_nodes;
    R t = R(0), prev_t = R(0), prev_dist = R(kMaxFloat);
    uint32_t near_steps = 0;
    uint32_t step = 0;
    for (; step < p->hard_max_steps; ++step) {
      note(t, max_distance);
      if (t > max_distance || near_steps >= p->scene.max_steps) break;
      const V3<R> pos = add(origin, mul(sd, t));
      if (tl) {
        // coarse empty-space skip (:907-921): forget the previous sample
        const R cd = R(coarse_sample(*tl->cf, tl->ocr, static_cast<float>(pos.x - R(tl->cam[0])),
                                     static_cast<float>(pos.y - R(tl->cam[1])),
                                     static_cast<float>(pos.z - R(tl->cam[2]))));
        if (cd > R(0.5f)) {  // COARSE_NEAR_THRESHOLD (:863)
          prev_dist = R(kMaxFloat);
          t += cd;
          continue;
        }
      }
      R min_dist = R(kMaxFloat);
      uint32_t best_mat = 0, best_id = 0, best_idx = 0;
      auto consider = [&](uint32_t i) {
        uint32_t m;
        const R d = evaluate(pos, i, &m, !any_hit);
        if (d < min_dist) {
          min_dist = d;
          best_mat = m;
          best_id = s->objects[i].object_id;
          best_idx = i;
        }
      };
      if (!tl && use_bvh) {
        // BVH traversal (:672-721): skip nodes whose AABB is farther than
        // the best distance so far; push left then right (right is visited
        // first) while the 32-entry stack has room for both
        uint32_t stack[32];
        uint32_t sp = 1;
        stack[0] = 0;
        while (sp > 0) {
          const uint32_t ni = stack[--sp];
          if (ni >= s->bvh_nodes) continue;  // the import admits no such tree
          const rkf_bvh_node& nd = s->bvh[ni];
          const V3<R> c = v3<R>(std::fmin(std::fmax(pos.x, R(nd.aabb_min[0])), R(nd.aabb_max[0])),
                                std::fmin(std::fmax(pos.y, R(nd.aabb_min[1])), R(nd.aabb_max[1])),
                                std::fmin(std::fmax(pos.z, R(nd.aabb_min[2])), R(nd.aabb_max[2])));
          const R box_dist = length(sub(c, pos));
          if (box_dist > min_dist) continue;
          if (nd.left == RKF_BVH_INVALID) {
            if (nd.right_or_object < s->num_objects) consider(nd.right_or_object);
          } else if (sp < 31) {
            stack[sp++] = nd.left;
            stack[sp++] = nd.right_or_object;
          }
        }
      } else {
        const uint32_t n_eval = tl ? tl->count : s->num_objects;
        for (uint32_t j = 0; j < n_eval; ++j) consider(tl ? tl->list[j] : j);
      }
      note(min_dist, R(0));
      note(min_dist, hit_thr);
      if (min_dist < R(0) && prev_dist > hit_thr) {
        if (any_hit) {
          r.t = t;
          r.hit = true;
          r.obj_idx = best_idx;
          break;
        }
        R lo = prev_t, hi = t;
        uint32_t bmat = best_mat;
        for (uint32_t b = 0; b < p->bisect_steps; ++b) {
          const R mid = (lo + hi) * R(0.5);
          uint32_t m;
          const R md = evaluate(add(origin, mul(sd, mid)), best_idx, &m);
          note(md, R(0));
          if (md < R(0)) {
            hi = mid;
          } else {
            lo = mid;
            bmat = m;
          }
        }
        r.t = (lo + hi) * R(0.5);
        r.hit = true;
        r.bisected = true;
        r.mat = bmat;
        r.obj_id = best_id;
        r.obj_idx = best_idx;
        break;
      }
      if (min_dist < hit_thr) {
        r.t = t;
        r.hit = true;
        r.mat = best_mat;
        r.obj_id = best_id;
        r.obj_idx = best_idx;
        break;
      }
      note(min_dist, near_thr);
      if (min_dist < near_thr) near_steps++;
      prev_t = t;
      prev_dist = min_dist;
      t += fmax_(min_dist, min_step);
    }
    if (!r.hit) r.out_of_steps = (step >= p->hard_max_steps) || near_steps >= p->scene.max_steps;
    if (steps_out) *steps_out += step;
    return r;
  }

  // compute_normal_for_object (:1003-1032)
  V3<R> normal(V3<R> pos, uint32_t oi, const rkf_march_params* p) {
    const rkf_gpu_object& o = s->objects[oi];
    if (o.sdf_type == RKF_SDF_VOXELIZED) {
      const V3<R> lp = to_local(o, pos);
      const R e = R(o.voxel_size) * R(2);  // :505
      const R gx = voxelized(o, oi, v3<R>(lp.x + e, lp.y, lp.z), true) -
                   voxelized(o, oi, v3<R>(lp.x - e, lp.y, lp.z), true);
      const R gy = voxelized(o, oi, v3<R>(lp.x, lp.y + e, lp.z), true) -
                   voxelized(o, oi, v3<R>(lp.x, lp.y - e, lp.z), true);
      const R gz = voxelized(o, oi, v3<R>(lp.x, lp.y, lp.z + e), true) -
                   voxelized(o, oi, v3<R>(lp.x, lp.y, lp.z - e), true);
      const float* m = o.inverse_world;  // transpose(M) * (g, 0)
      const V3<R> wg = v3<R>(((R(m[0]) * gx + R(m[1]) * gy) + R(m[2]) * gz) + R(m[3]) * R(0),
                             ((R(m[4]) * gx + R(m[5]) * gy) + R(m[6]) * gz) + R(m[7]) * R(0),
                             ((R(m[8]) * gx + R(m[9]) * gy) + R(m[10]) * gz) + R(m[11]) * R(0));
      const R len = length(wg);
      if (len < R(1e-10f)) return v3<R>(R(0), R(1), R(0));
      return v3<R>(wg.x / len, wg.y / len, wg.z / len);
    }
    const R e = R(p->scene.hit_threshold) * R(10);
    uint32_t m;
    const R nx = evaluate(v3<R>(pos.x + e, pos.y, pos.z), oi, &m) -
                 evaluate(v3<R>(pos.x - e, pos.y, pos.z), oi, &m);
    const R ny = evaluate(v3<R>(pos.x, pos.y + e, pos.z), oi, &m) -
                 evaluate(v3<R>(pos.x, pos.y - e, pos.z), oi, &m);
    const R nz = evaluate(v3<R>(pos.x, pos.y, pos.z + e), oi, &m) -
                 evaluate(v3<R>(pos.x, pos.y, pos.z - e), oi, &m);
    const V3<R> n = v3<R>(nx, ny, nz);
    const R l = length(n);
    return v3<R>(n.x / l, n.y / l, n.z / l);
  }

  // soft_shadow (shade_common_shading.wgsl:9-33) with sample_sdf as the
  // min over objects (shade_common.wgsl:521-572 without the coarse field).
  R soft_shadow(V3<R> origin, V3<R> ld, R max_dist, uint64_t* steps_out) {
    const R eps = R(0.005f), k = R(16);
    R shadow = R(1), t = eps;
    uint32_t near_steps = 0, i = 0;
    for (; i < 256u; ++i) {
      note(t, max_dist);
      if (near_steps >= 32u || t > max_dist) break;
      const V3<R> pos = add(origin, mul(ld, t));
      R d = R(kMaxFloat);
      for (uint32_t oi = 0; oi < s->num_objects; ++oi) {
        uint32_t m;
        d = fmin_(d, evaluate(pos, oi, &m, false));
      }
      note(d, eps);
      if (d < eps) {
        if (steps_out) *steps_out += i;
        return R(0);
      }
      note(d, R(0.02f));
      if (d < R(0.02f)) {
        shadow = fmin_(shadow, k * d / t);
        near_steps++;
      }
      t += fmax_(d, eps);
    }
    if (steps_out) *steps_out += i;
    return clampf(shadow, R(0), R(1));
  }

  // Refine the trilinear surface crossing near a hit in FP64: march forward
  // in small steps to bracket a sign change of the object's field, then
  // bisect to convergence.  Returns NaN when no crossing is found.
  double refine_root(V3<R> origin, V3<R> dir, R t_hit, uint32_t oi) {
    const rkf_gpu_object& o = s->objects[oi];
    const double step = static_cast<double>(o.voxel_size) * 0.0625;
    auto f = [&](double t) {
      uint32_t m;
      return static_cast<double>(evaluate(add(origin, mul(dir, R(t))), oi, &m, false));
    };
    double lo = static_cast<double>(t_hit) - 2.0 * static_cast<double>(o.voxel_size);
    if (lo < 0) lo = 0;
    double flo = f(lo);
    if (!(flo > 0)) return NAN;
    const double t_end = static_cast<double>(t_hit) + 4.0 * static_cast<double>(o.voxel_size);
    for (double t = lo + step; t <= t_end; t += step) {
      const double ft = f(t);
      if (ft <= 0) {
        double a = t - step, b = t;
        for (int it = 0; it < 80; ++it) {
          const double m = 0.5 * (a + b);
          if (f(m) > 0) a = m; else b = m;
        }
        return 0.5 * (a + b);
      }
    }
    return NAN;
  }
};

struct RayOut {
  float* t;
  float* normal;
  uint32_t* slot;
  uint16_t* material;
  uint16_t* flags;
  double* t64;
  double* normal64;
  double* margin;
};

template <class R>
void shade_epilogue(Marcher<R>& mc, const typename Marcher<R>::Result& res, V3<R> origin,
                    V3<R> dir, const rkf_march_params* p, uint64_t i, const RayOut& o,
                    V3<R>* hit_pos_out, V3<R>* n_out, uint32_t* sec_out, uint32_t* blend_out,
                    R* sdf_at_hit) {
  uint16_t flags = 0;
  V3<R> n = v3<R>(R(0), R(0), R(0));
  uint32_t slot = RKF_EMPTY_SLOT;
  *sec_out = 0;
  *blend_out = 0;
  *sdf_at_hit = R(0);
  V3<R> hp = v3<R>(R(0), R(0), R(0));
  if (res.hit) {
    flags |= RKF_FLAG_HIT;
    if (res.bisected) flags |= RKF_FLAG_BISECTED;
    hp = add(origin, mul(dir, res.t));  // ray_march.wgsl:1068 (unsafe dir)
    n = mc.normal(hp, res.obj_idx, p);
    const rkf_gpu_object& ob = mc.s->objects[res.obj_idx];
    if (ob.sdf_type == RKF_SDF_VOXELIZED) {
      const V3<R> lh = Marcher<R>::to_local(ob, hp);
      uint32_t idx = 0;
      slot = mc.nearest(ob, res.obj_idx, lh, &idx);
      if (slot != RKF_EMPTY_SLOT && slot != RKF_INTERIOR_SLOT) {
        *sec_out = (mc.mat_word(slot, idx) >> 6) & 0x3Fu;
        *blend_out = mc.blend_of(slot, idx);
      }
      *sdf_at_hit = mc.voxelized(ob, res.obj_idx, lh, false);
    }
  } else if (res.out_of_steps) {
    flags |= RKF_FLAG_STEPS_OUT;
  }
  if (o.t) o.t[i] = res.hit ? static_cast<float>(res.t) : kMaxFloat;
  if (o.t64) o.t64[i] = res.hit ? static_cast<double>(res.t) : static_cast<double>(kMaxFloat);
  if (o.normal) {
    o.normal[3 * i] = static_cast<float>(n.x);
    o.normal[3 * i + 1] = static_cast<float>(n.y);
    o.normal[3 * i + 2] = static_cast<float>(n.z);
  }
  if (o.normal64) {
    o.normal64[3 * i] = static_cast<double>(n.x);
    o.normal64[3 * i + 1] = static_cast<double>(n.y);
    o.normal64[3 * i + 2] = static_cast<double>(n.z);
  }
  if (o.slot) o.slot[i] = slot;
  if (o.material) o.material[i] = static_cast<uint16_t>(res.hit ? res.mat : 0u);
  if (o.flags) o.flags[i] = flags;
  *hit_pos_out = hp;
  *n_out = n;
}

// Sector accounting per ray: sort+unique the touched sectors.  Material
// reads made during the march are not algorithmic; the hit's nearest-voxel
// material sector is.
void finish_sectors(Tracker& tr, orc_stats* st, bool hit_material) {
  if (!tr.on) return;
  std::sort(tr.keys.begin(), tr.keys.end());
  tr.keys.erase(std::unique(tr.keys.begin(), tr.keys.end()), tr.keys.end());
  uint64_t idx = 0, dst = 0, mat = 0;
  for (uint64_t k : tr.keys) {
    const uint64_t plane = k >> 56;
    if (plane == 0 || plane == 3) idx++;
    else if (plane == 1) dst++;
  }
  mat = hit_material ? 1 : 0;
  st->index_sectors += idx;
  st->dist_sectors += dst;
  st->mat_sectors += mat;
  st->sectors += idx + dst + mat;
  tr.keys.clear();
}

template <class R>
void march_view(const orc_scene* s, const rkf_camera* cam, const rkf_march_params* p,
                uint32_t w, uint32_t h, int threads, uint32_t row0, uint32_t row1,
                const RayOut& out, float* position, uint32_t* packed, float* motion,
                double* t_root, int count_sectors, orc_stats* stats) {
  if (row1 <= row0) {
    row0 = 0;
    row1 = h;
  }
  const uint64_t n = static_cast<uint64_t>(row1 - row0) * w;
  std::vector<orc_stats> per(std::max(threads, 1));
  std::memset(per.data(), 0, sizeof(orc_stats) * per.size());
  const bool tiled = p->strategy == RKF_STRATEGY_TILED;
  CoarseField cf;
  std::vector<uint32_t> tcnt, tlist;
  uint32_t tiles_x = 0;
  float ocr[3] = {0.0f, 0.0f, 0.0f};
  if (tiled) {
    cf = coarse_build(s);
    tile_cull(s, cam, w, h, tcnt, tlist, &tiles_x);
    for (int a = 0; a < 3; ++a) ocr[a] = cf.origin[a] - cam->position[a];
  }
  parallel_for(n, threads, [&](uint64_t li, int th) {
    Tracker tr;
    tr.on = count_sectors != 0;
    double marg = 1e300;
    Marcher<R> mc{s, &tr, out.margin ? &marg : nullptr};
    const uint32_t px = static_cast<uint32_t>(li % w);
    const uint32_t py = row0 + static_cast<uint32_t>(li / w);
    const uint64_t i = li;  // outputs hold rows [row0, row1) only
    // ray generation (ray_march.wgsl:1046-1053)
    const R u = ((R(static_cast<float>(px)) + R(0.5)) + R(cam->jitter[0])) / R(static_cast<float>(w));
    const R v = ((R(static_cast<float>(py)) + R(0.5)) + R(cam->jitter[1])) / R(static_cast<float>(h));
    const R nx = u * R(2) - R(1);
    const R ny = R(1) - v * R(2);
    const V3<R> f = v3<R>(R(cam->forward[0]), R(cam->forward[1]), R(cam->forward[2]));
    const V3<R> rt = v3<R>(R(cam->right[0]), R(cam->right[1]), R(cam->right[2]));
    const V3<R> up = v3<R>(R(cam->up[0]), R(cam->up[1]), R(cam->up[2]));
    const V3<R> dv = add(add(f, mul(rt, nx)), mul(up, ny));
    const R dl = length(dv);
    const V3<R> dir = v3<R>(dv.x / dl, dv.y / dl, dv.z / dl);
    const V3<R> org = v3<R>(R(cam->position[0]), R(cam->position[1]), R(cam->position[2]));
    TiledRay tr_{};
    if (tiled) {
      // the march's tile grid: dims from the view, (w + 15) / 16 tiles per row (:884-888)
      const size_t tile = static_cast<size_t>(py / 16) * ((w + 15) / 16) + px / 16;
      tr_.cf = &cf;
      for (int a = 0; a < 3; ++a) tr_.ocr[a] = ocr[a], tr_.cam[a] = cam->position[a];
      tr_.list = tlist.data() + tile * 32;
      tr_.count = tcnt[tile];
    }
    const auto res = mc.march(org, dir, p, R(p->scene.max_distance), false, &per[th].steps,
                              tiled ? &tr_ : nullptr);
    V3<R> hp, nn;
    uint32_t sec, blend;
    R sdf_hit;
    shade_epilogue(mc, res, org, dir, p, i, out, &hp, &nn, &sec, &blend, &sdf_hit);
    if (out.margin) out.margin[i] = marg;
    if (t_root) t_root[i] = res.hit ? mc.refine_root(org, dir, res.t, res.obj_idx) : NAN;
    if (position) {
      position[4 * i] = res.hit ? static_cast<float>(hp.x) : 0.0f;
      position[4 * i + 1] = res.hit ? static_cast<float>(hp.y) : 0.0f;
      position[4 * i + 2] = res.hit ? static_cast<float>(hp.z) : 0.0f;
      position[4 * i + 3] = res.hit ? static_cast<float>(res.t) : kMaxFloat;
    }
    if (packed) {
      packed[i] = res.hit ? ((res.mat & 0x3Fu) | (sec << 6) | (blend << 12) | (res.obj_id << 24))
                          : 0u;
    }
    if (motion) {  // ray_march.wgsl:1094-1105
      float mx = 0.0f, my = 0.0f, mz = 0.0f, mw = 0.0f;
      if (res.hit) {
        const float* m = cam->prev_vp;
        const R cx = ((R(m[0]) * hp.x + R(m[4]) * hp.y) + R(m[8]) * hp.z) + R(m[12]) * R(1);
        const R cy = ((R(m[1]) * hp.x + R(m[5]) * hp.y) + R(m[9]) * hp.z) + R(m[13]) * R(1);
        const R cw = ((R(m[3]) * hp.x + R(m[7]) * hp.y) + R(m[11]) * hp.z) + R(m[15]) * R(1);
        R ox = R(0), oy = R(0);
        if (cw > R(0)) {
          const R ndx = cx / cw, ndy = cy / cw;
          const R pu = ndx * R(0.5) + R(0.5), pv = R(0.5) - ndy * R(0.5);
          const R cu = (R(static_cast<float>(px)) + R(0.5)) / R(static_cast<float>(w));
          const R cv = (R(static_cast<float>(py)) + R(0.5)) / R(static_cast<float>(h));
          ox = cu - pu;
          oy = cv - pv;
        }
        mx = static_cast<float>(ox);
        my = static_cast<float>(oy);
        mz = 1.0f;
        mw = static_cast<float>(sdf_hit);
      }
      motion[4 * i] = mx;
      motion[4 * i + 1] = my;
      motion[4 * i + 2] = mz;
      motion[4 * i + 3] = mw;
    }
    finish_sectors(tr, &per[th], res.hit && s->objects[res.obj_idx].sdf_type == RKF_SDF_VOXELIZED);
  });
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    for (auto& q : per) {
      stats->sectors += q.sectors;
      stats->index_sectors += q.index_sectors;
      stats->dist_sectors += q.dist_sectors;
      stats->mat_sectors += q.mat_sectors;
      stats->steps += q.steps;
      stats->evals += q.evals;
    }
  }
}

template <class R>
void trace_impl(const orc_scene* s, const float* origins, const float* dirs, const float* tmax,
                uint32_t n, uint32_t mode, const rkf_march_params* p, int threads,
                const RayOut& out) {
  parallel_for(n, threads, [&](uint64_t i, int) {
    Tracker tr;
    double marg = 1e300;
    Marcher<R> mc{s, &tr, out.margin ? &marg : nullptr};
    const V3<R> o = v3<R>(R(origins[3 * i]), R(origins[3 * i + 1]), R(origins[3 * i + 2]));
    const V3<R> d = v3<R>(R(dirs[3 * i]), R(dirs[3 * i + 1]), R(dirs[3 * i + 2]));
    if (mode == RKF_TRACE_SHADOW) {
      const R f = mc.soft_shadow(o, d, R(tmax[i]), nullptr);
      if (out.t) out.t[i] = static_cast<float>(f);
      if (out.t64) out.t64[i] = static_cast<double>(f);
      if (out.flags) out.flags[i] = f == R(0) ? RKF_FLAG_HIT : 0;
    } else if (mode == RKF_TRACE_ANY) {
      const auto res = mc.march(o, d, p, R(tmax[i]), true, nullptr);
      if (out.t) out.t[i] = res.hit ? static_cast<float>(res.t) : kMaxFloat;
      if (out.t64) out.t64[i] = res.hit ? static_cast<double>(res.t) : static_cast<double>(kMaxFloat);
      if (out.flags) out.flags[i] = res.hit ? RKF_FLAG_HIT : (res.out_of_steps ? RKF_FLAG_STEPS_OUT : 0);
    } else {
      const auto res = mc.march(o, d, p, R(tmax[i]), false, nullptr);
      V3<R> hp, nn;
      uint32_t sec, blend;
      R sh;
      shade_epilogue(mc, res, o, d, p, i, out, &hp, &nn, &sec, &blend, &sh);
    }
    if (out.margin) out.margin[i] = marg;
  });
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

uint16_t orc_f16_from_f32(float f) { return f16_from_f32(f); }
float orc_f16_to_f32(uint16_t h) { return f16_to_f32(h); }

float orc_prim_sdf(const rkf_prim* p, const float pos[3]) {
  return prim_sdf<float>(*p, pos[0], pos[1], pos[2]);
}
float orc_smin(float a, float b, float k) { return smin<float>(a, b, k); }
float orc_scene_eval(const rkf_prim* prims, uint32_t n, float k, float cut, const float pos[3],
                     uint32_t* material, uint32_t* secondary, uint32_t* blend) {
  return scene_eval<float>(prims, nullptr, n, k, cut, pos[0], pos[1], pos[2], material,
                           secondary, blend);
}

orc_voxelized* orc_voxelize(const rkf_prim* prims, uint32_t n_prims,
                            const rkf_voxelize_params* vp, int threads) {
  auto* v = new orc_voxelized;
  v->g = make_grid(vp);
  const Grid& g = v->g;
  const uint64_t nb = static_cast<uint64_t>(g.dims[0]) * g.dims[1] * g.dims[2];
  std::vector<uint8_t> cls(nb, 1);
  std::vector<BrickResult*> res(nb, nullptr);
  std::vector<std::vector<uint32_t>> cands(std::max(threads, 1));
  parallel_for(nb, threads, [&](uint64_t f, int th) {
    const uint32_t bx = static_cast<uint32_t>(f % g.dims[0]);
    const uint32_t by = static_cast<uint32_t>((f / g.dims[0]) % g.dims[1]);
    const uint32_t bz = static_cast<uint32_t>(f / (static_cast<uint64_t>(g.dims[0]) * g.dims[1]));
    BrickResult r;
    classify_brick(prims, n_prims, vp, g, bx, by, bz, cands[th], r);
    cls[f] = static_cast<uint8_t>(r.cls);
    if (r.cls == 0) {
      res[f] = new BrickResult(r);
    }
  });
  v->map.assign(nb, RKF_EMPTY_SLOT);
  // slots in z,y,x loop order (== ascending flat index), lowest first
  // (brick_pool.rs:37-42, voxelize_object.rs:123-158)
  uint32_t slot = 0;
  for (uint64_t f = 0; f < nb; ++f) {
    if (cls[f] == 0) {
      v->map[f] = slot++;
    } else if (cls[f] == 2) {
      v->map[f] = RKF_INTERIOR_SLOT;
      v->n_interior++;
    }
  }
  v->n_bricks = slot;
  v->words.resize(static_cast<uint64_t>(slot) * 1024);
  v->dist.resize(static_cast<uint64_t>(slot) * 512);
  for (uint64_t f = 0; f < nb; ++f) {
    if (res[f]) {
      const uint32_t s = v->map[f];
      std::memcpy(&v->words[static_cast<uint64_t>(s) * 1024], res[f]->words, 4096);
      std::memcpy(&v->dist[static_cast<uint64_t>(s) * 512], res[f]->dist, 2048);
      delete res[f];
    }
  }
  return v;
}

// The same voxelization into a two-level index (top grid of 8^3-brick
// blocks, 512-entry leaves) and SoA planes, for grids whose flat brick map
// would not fit host memory.  A brick no primitive's candidate test reaches
// has no candidates, so classify_brick finds it EMPTY; only the bricks near
// some primitive are classified, in ascending flat order, which keeps the slot
// order and every word of orc_voxelize.
struct orc_sparse {
  Grid g;
  uint32_t tdim[3] = {0, 0, 0};
  std::vector<uint32_t> top, leaves;
  std::vector<uint16_t> dist_f16, mat;
  std::vector<uint8_t> blend;
  std::vector<uint32_t> bxyz;  // coordinates of each allocated brick, by slot
  uint32_t n_bricks = 0, n_interior = 0, n_leaves = 0;
};

orc_sparse* orc_voxelize_sparse(const rkf_prim* prims, uint32_t n_prims, const rkf_voxelize_params* vp,
                                int threads) {
  auto* v = new orc_sparse;
  v->g = make_grid(vp);
  const Grid& g = v->g;
  const uint64_t dx = g.dims[0], dy = g.dims[1];
  // 1. bricks some primitive's candidate test reaches (brick_candidates)
  std::vector<std::vector<uint64_t>> per(n_prims);
  parallel_for(n_prims, threads, [&](uint64_t i, int) {
    const rkf_prim& pr = prims[i];
    const double reach = static_cast<double>(pr.bound_radius) + vp->cut_distance + 0.05 * g.bws + 1e-3;
    int64_t lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = static_cast<int64_t>(std::floor((pr.centre[a] - reach - g.origin[a]) / g.bws)) - 1;
      hi[a] = static_cast<int64_t>(std::ceil((pr.centre[a] + reach - g.origin[a]) / g.bws)) + 1;
      lo[a] = std::max<int64_t>(lo[a], 0);
      hi[a] = std::min<int64_t>(hi[a], static_cast<int64_t>(g.dims[a]) - 1);
    }
    for (int64_t z = lo[2]; z <= hi[2]; ++z)
      for (int64_t y = lo[1]; y <= hi[1]; ++y)
        for (int64_t x = lo[0]; x <= hi[0]; ++x) {
          float bmin[3];
          brick_min_of(g, static_cast<uint32_t>(x), static_cast<uint32_t>(y), static_cast<uint32_t>(z), bmin);
          double d2 = 0.0;
          for (int a = 0; a < 3; ++a) {
            const double l = bmin[a], h = static_cast<double>(bmin[a]) + g.bws;
            const double c = pr.centre[a];
            const double e = c < l ? l - c : (c > h ? c - h : 0.0);
            d2 += e * e;
          }
          if (d2 < reach * reach) per[i].push_back(static_cast<uint64_t>(x) + y * dx + z * dx * dy);
        }
  });
  std::vector<uint64_t> cand;
  for (auto& p : per) {
    cand.insert(cand.end(), p.begin(), p.end());
    std::vector<uint64_t>().swap(p);
  }
  std::sort(cand.begin(), cand.end());
  cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
  // 2. classify the candidates
  std::vector<uint8_t> cls(cand.size(), 1);
  std::vector<std::vector<uint32_t>> cands(std::max(threads, 1));
  parallel_for(cand.size(), threads, [&](uint64_t k, int th) {
    const uint64_t f = cand[k];
    BrickResult r;
    classify_brick(prims, n_prims, vp, g, static_cast<uint32_t>(f % dx), static_cast<uint32_t>((f / dx) % dy),
                   static_cast<uint32_t>(f / (dx * dy)), cands[th], r);
    cls[k] = static_cast<uint8_t>(r.cls);
  });
  // 3. slots in ascending flat order; index blocks
  for (int a = 0; a < 3; ++a) v->tdim[a] = (g.dims[a] + 7) / 8;
  const uint64_t tx = v->tdim[0], ty = v->tdim[1], tz = v->tdim[2];
  v->top.assign(tx * ty * tz, RKF_EMPTY_SLOT);
  std::vector<uint64_t> alloc;
  std::vector<uint32_t> slot_of(cand.size(), RKF_EMPTY_SLOT);
  for (uint64_t k = 0; k < cand.size(); ++k) {
    if (cls[k] == 1) continue;
    const uint64_t f = cand[k];
    const uint64_t blk = (f % dx) / 8 + ((f / dx) % dy) / 8 * tx + (f / (dx * dy)) / 8 * tx * ty;
    if (v->top[blk] == RKF_EMPTY_SLOT) v->top[blk] = v->n_leaves++;
    if (cls[k] == 0) {
      slot_of[k] = v->n_bricks++;
      alloc.push_back(k);
    } else {
      slot_of[k] = RKF_INTERIOR_SLOT;
      v->n_interior++;
    }
  }
  v->leaves.assign(static_cast<uint64_t>(v->n_leaves) * 512, RKF_EMPTY_SLOT);
  for (uint64_t k = 0; k < cand.size(); ++k) {
    if (cls[k] == 1) continue;
    const uint64_t f = cand[k];
    const uint64_t x = f % dx, y = (f / dx) % dy, z = f / (dx * dy);
    const uint64_t blk = x / 8 + y / 8 * tx + z / 8 * tx * ty;
    v->leaves[static_cast<uint64_t>(v->top[blk]) * 512 + (x & 7) + (y & 7) * 8 + (z & 7) * 64] = slot_of[k];
  }
  // 4. the allocated bricks' planes
  const uint64_t nb = v->n_bricks;
  v->dist_f16.resize(nb * 512);
  v->mat.resize(nb * 512);
  v->blend.resize(nb * 512);
  v->bxyz.resize(nb * 3);
  parallel_for(nb, threads, [&](uint64_t s, int th) {
    const uint64_t f = cand[alloc[s]];
    const uint32_t x = static_cast<uint32_t>(f % dx), y = static_cast<uint32_t>((f / dx) % dy),
                   z = static_cast<uint32_t>(f / (dx * dy));
    BrickResult r;
    classify_brick(prims, n_prims, vp, g, x, y, z, cands[th], r);
    for (uint32_t i = 0; i < 512; ++i) {
      const uint32_t w0 = r.words[2 * i];
      v->dist_f16[s * 512 + i] = static_cast<uint16_t>(w0 & 0xFFFFu);
      v->mat[s * 512 + i] = static_cast<uint16_t>(((w0 >> 16) & 0x3Fu) | (((w0 >> 22) & 0x3Fu) << 6));
      v->blend[s * 512 + i] = static_cast<uint8_t>(r.words[2 * i + 1] >> 24);
    }
    v->bxyz[3 * s] = x;
    v->bxyz[3 * s + 1] = y;
    v->bxyz[3 * s + 2] = z;
  });
  return v;
}

void orc_sparse_info(const orc_sparse* v, uint32_t dims[3], uint32_t tdim[3], uint32_t* n_bricks,
                     uint32_t* n_interior, uint32_t* n_leaves) {
  for (int a = 0; a < 3; ++a) {
    dims[a] = v->g.dims[a];
    tdim[a] = v->tdim[a];
  }
  *n_bricks = v->n_bricks;
  *n_interior = v->n_interior;
  *n_leaves = v->n_leaves;
}

void orc_sparse_copy(const orc_sparse* v, uint32_t* top, uint32_t* leaves, uint16_t* dist_f16, uint16_t* mat,
                     uint8_t* blend, uint32_t* bxyz) {
  std::memcpy(top, v->top.data(), v->top.size() * 4);
  std::memcpy(leaves, v->leaves.data(), v->leaves.size() * 4);
  std::memcpy(dist_f16, v->dist_f16.data(), v->dist_f16.size() * 2);
  std::memcpy(mat, v->mat.data(), v->mat.size() * 2);
  std::memcpy(blend, v->blend.data(), v->blend.size());
  std::memcpy(bxyz, v->bxyz.data(), v->bxyz.size() * 4);
}

void orc_sparse_free(orc_sparse* v) { delete v; }

void orc_voxelized_info(const orc_voxelized* v, uint32_t dims[3], uint32_t* n_bricks,
                        uint32_t* n_interior) {
  for (int a = 0; a < 3; ++a) dims[a] = v->g.dims[a];
  *n_bricks = v->n_bricks;
  *n_interior = v->n_interior;
}
void orc_voxelized_copy(const orc_voxelized* v, uint32_t* words, uint32_t* map) {
  if (words) std::memcpy(words, v->words.data(), v->words.size() * 4);
  if (map) std::memcpy(map, v->map.data(), v->map.size() * 4);
}
void orc_voxelized_copy_f32(const orc_voxelized* v, float* dist) {
  std::memcpy(dist, v->dist.data(), v->dist.size() * 4);
}
void orc_voxelized_free(orc_voxelized* v) { delete v; }

void orc_voxel_values_f64(const rkf_prim* prims, uint32_t n_prims, const rkf_voxelize_params* vp,
                          const uint32_t* map, uint32_t n_slots, double* dist, int threads) {
  const Grid g = make_grid(vp);
  const uint64_t nb = static_cast<uint64_t>(g.dims[0]) * g.dims[1] * g.dims[2];
  std::vector<std::vector<uint32_t>> cands(std::max(threads, 1));
  parallel_for(nb, threads, [&](uint64_t f, int th) {
    const uint32_t slot = map[f];
    if (slot >= RKF_INTERIOR_SLOT || slot >= n_slots) return;
    const uint32_t bx = static_cast<uint32_t>(f % g.dims[0]);
    const uint32_t by = static_cast<uint32_t>((f / g.dims[0]) % g.dims[1]);
    const uint32_t bz = static_cast<uint32_t>(f / (static_cast<uint64_t>(g.dims[0]) * g.dims[1]));
    float bmin[3];
    brick_min_of(g, bx, by, bz, bmin);
    brick_candidates(prims, n_prims, bmin, g.bws, vp->cut_distance, cands[th]);
    const float hv = g.vs * 0.5f;
    for (uint32_t v = 0; v < 512; ++v) {
      // the voxel centre the reference samples (voxelize_object.rs:170-176), evaluated in FP64
      const double px = bmin[0] + (static_cast<float>(v & 7) * g.vs + hv);
      const double py = bmin[1] + (static_cast<float>((v >> 3) & 7) * g.vs + hv);
      const double pz = bmin[2] + (static_cast<float>(v >> 6) * g.vs + hv);
      dist[static_cast<uint64_t>(slot) * 512 + v] =
          scene_eval<double>(prims, cands[th].data(), static_cast<uint32_t>(cands[th].size()), vp->smooth_k,
                             vp->cut_distance, px, py, pz, nullptr, nullptr, nullptr);
    }
  });
}

void orc_voxel_values_f64_bricks(const rkf_prim* prims, uint32_t n_prims, const rkf_voxelize_params* vp,
                                 const uint32_t* bxyz, const uint32_t* slots, uint64_t n, double* dist,
                                 int threads) {
  // the same values as orc_voxel_values_f64, for bricks listed with their
  // slots (a two-level index has no flat map to walk)
  const Grid g = make_grid(vp);
  std::vector<std::vector<uint32_t>> cands(std::max(threads, 1));
  parallel_for(n, threads, [&](uint64_t i, int th) {
    float bmin[3];
    brick_min_of(g, bxyz[3 * i], bxyz[3 * i + 1], bxyz[3 * i + 2], bmin);
    brick_candidates(prims, n_prims, bmin, g.bws, vp->cut_distance, cands[th]);
    const float hv = g.vs * 0.5f;
    for (uint32_t v = 0; v < 512; ++v) {
      const double px = bmin[0] + (static_cast<float>(v & 7) * g.vs + hv);
      const double py = bmin[1] + (static_cast<float>((v >> 3) & 7) * g.vs + hv);
      const double pz = bmin[2] + (static_cast<float>(v >> 6) * g.vs + hv);
      dist[static_cast<uint64_t>(slots[i]) * 512 + v] =
          scene_eval<double>(prims, cands[th].data(), static_cast<uint32_t>(cands[th].size()), vp->smooth_k,
                             vp->cut_distance, px, py, pz, nullptr, nullptr, nullptr);
    }
  });
}

void orc_voxelize_bricks(const rkf_prim* prims, uint32_t n_prims, const rkf_voxelize_params* vp,
                         const uint32_t* bxyz, uint32_t n, uint32_t* cls, uint32_t* words,
                         int threads) {
  const Grid g = make_grid(vp);
  std::vector<std::vector<uint32_t>> cands(std::max(threads, 1));
  parallel_for(n, threads, [&](uint64_t i, int th) {
    BrickResult r;
    classify_brick(prims, n_prims, vp, g, bxyz[3 * i], bxyz[3 * i + 1], bxyz[3 * i + 2],
                   cands[th], r);
    cls[i] = r.cls;
    if (words && r.cls == 0) std::memcpy(words + i * 1024, r.words, 4096);
  });
}

void orc_march(const orc_scene* s, const rkf_camera* cam, const rkf_march_params* p, uint32_t w,
               uint32_t h, int fp64, int threads, uint32_t row0, uint32_t row1, float* t,
               float* normal, uint32_t* slot, uint16_t* material, uint16_t* flags,
               float* position, uint32_t* packed, float* motion, double* t64, double* normal64,
               double* margin, double* t_root, int count_sectors, orc_stats* stats) {
  RayOut o{t, normal, slot, material, flags, t64, normal64, margin};
  if (fp64)
    march_view<double>(s, cam, p, w, h, threads, row0, row1, o, position, packed, motion,
                       t_root, count_sectors, stats);
  else
    march_view<float>(s, cam, p, w, h, threads, row0, row1, o, position, packed, motion,
                      nullptr, count_sectors, stats);
}

void orc_trace_rays(const orc_scene* s, const float* origins, const float* dirs,
                    const float* tmax, uint32_t n, uint32_t mode, const rkf_march_params* p,
                    int fp64, int threads, float* t, float* normal, uint32_t* slot,
                    uint16_t* material, uint16_t* flags, double* t64, double* margin) {
  RayOut o{t, normal, slot, material, flags, t64, nullptr, margin};
  if (fp64)
    trace_impl<double>(s, origins, dirs, tmax, n, mode, p, threads, o);
  else
    trace_impl<float>(s, origins, dirs, tmax, n, mode, p, threads, o);
}

void orc_query_points(const orc_scene* s, const float* points, uint32_t n, float* dist,
                      float* grad, uint16_t* material, int threads) {
  rkf_march_params p;
  orc_march_params_default(&p);
  parallel_for(n, threads, [&](uint64_t i, int) {
    Tracker tr;
    Marcher<float> mc{s, &tr, nullptr};
    const V3<float> q = v3<float>(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
    float best = kMaxFloat;
    uint32_t bm = 0, bi = 0;
    for (uint32_t oi = 0; oi < s->num_objects; ++oi) {
      uint32_t m;
      const float d = mc.evaluate(q, oi, &m);
      if (d < best) {
        best = d;
        bm = m;
        bi = oi;
      }
    }
    if (dist) dist[i] = best;
    if (material) material[i] = static_cast<uint16_t>(bm);
    if (grad) {
      V3<float> n3 = v3<float>(0.0f, 1.0f, 0.0f);
      if (s->num_objects) n3 = mc.normal(q, bi, &p);
      grad[3 * i] = n3.x;
      grad[3 * i + 1] = n3.y;
      grad[3 * i + 2] = n3.z;
    }
  });
}

// sdf_ao (shade_common_shading.wgsl:37-47) through sample_sdf
// (shade_common.wgsl:521-572: inside the objects' bounds, the minimum of
// evaluate_object over the objects).
void orc_sdf_ao(const orc_scene* s, const float* pos, const float* normal, uint32_t n, float* ao,
                int threads) {
  parallel_for(n, threads, [&](uint64_t i, int) {
    Tracker tr;
    Marcher<float> mc{s, &tr, nullptr};
    const V3<float> p = v3<float>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    const V3<float> nv = v3<float>(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]);
    float acc = 0.0f, scale = 1.0f;
    for (uint32_t k = 1; k <= 4; ++k) {
      const float dist = 0.12f * static_cast<float>(k);  // AO_STEP_SIZE * f32(i)
      const V3<float> q = add(p, mul(nv, dist));
      float d = kMaxFloat;
      for (uint32_t oi = 0; oi < s->num_objects; ++oi) {
        uint32_t m;
        const float e = mc.evaluate(q, oi, &m);
        d = e < d ? e : d;
      }
      acc = acc + scale * (dist - d);
      scale = scale * 0.5f;
    }
    const float v = 1.0f - 0.7f * acc;  // AO_STRENGTH
    const float lo = v < 0.0f ? 0.0f : v;
    ao[i] = lo > 1.0f ? 1.0f : lo;
  });
}

// The shading pass's own sample_sdf (shade_common.wgsl:521-572): the coarse
// field at the camera-relative position first (sample_coarse_field, :504-511,
// the filter model of coarse_sample), its value where above
// COARSE_NEAR_THRESHOLD 0.5 (:291), else the minimum of evaluate_object over
// the objects (the shader walks the BVH for it; on scenes whose objects'
// distances are at least their box distances the walk's minimum is the
// same).  The library's SHADOW mode and rkf_sdf_ao use the minimum
// everywhere (the coarse value comes from a texture unit and cannot be
// pinned); these two let the tests bound the difference.
static float shader_sample_sdf(Marcher<float>& mc, const orc_scene* s, const CoarseField& cf, const float ocr[3],
                               const float cam[3], V3<float> q) {
  const float cd = coarse_sample(cf, ocr, q.x - cam[0], q.y - cam[1], q.z - cam[2]);
  if (cd > 0.5f) return cd;
  float d = kMaxFloat;
  for (uint32_t oi = 0; oi < s->num_objects; ++oi) {
    uint32_t m;
    const float e = mc.evaluate(q, oi, &m, false);
    d = e < d ? e : d;
  }
  return d;
}

// soft_shadow (shade_common_shading.wgsl:9-33) through the shader's sample_sdf.
void orc_shadow_shader(const orc_scene* s, const float* origins, const float* dirs, const float* tmax, uint32_t n,
                       const float cam[3], int threads, float* shadow) {
  const CoarseField cf = coarse_build(s);
  float ocr[3];
  for (int a = 0; a < 3; ++a) ocr[a] = cf.origin[a] - cam[a];
  parallel_for(n, threads, [&](uint64_t i, int) {
    Tracker tr;
    Marcher<float> mc{s, &tr, nullptr};
    const V3<float> o = v3<float>(origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]);
    const V3<float> ld = v3<float>(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
    float sh = 1.0f, t = 0.005f;
    uint32_t near_steps = 0;
    bool blocked = false;
    for (uint32_t k = 0; k < 256u; ++k) {
      if (near_steps >= 32u || t > tmax[i]) break;
      const float d = shader_sample_sdf(mc, s, cf, ocr, cam, add(o, mul(ld, t)));
      if (d < 0.005f) {
        blocked = true;
        break;
      }
      if (d < 0.02f) {
        sh = fmin_(sh, 16.0f * d / t);
        near_steps++;
      }
      t += fmax_(d, 0.005f);
    }
    shadow[i] = blocked ? 0.0f : clampf(sh, 0.0f, 1.0f);
  });
}

// sdf_ao (shade_common_shading.wgsl:37-47) through the shader's sample_sdf.
void orc_sdf_ao_shader(const orc_scene* s, const float* pos, const float* normal, uint32_t n, const float cam[3],
                       int threads, float* ao) {
  const CoarseField cf = coarse_build(s);
  float ocr[3];
  for (int a = 0; a < 3; ++a) ocr[a] = cf.origin[a] - cam[a];
  parallel_for(n, threads, [&](uint64_t i, int) {
    Tracker tr;
    Marcher<float> mc{s, &tr, nullptr};
    const V3<float> p = v3<float>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    const V3<float> nv = v3<float>(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]);
    float acc = 0.0f, scale = 1.0f;
    for (uint32_t k = 1; k <= 4; ++k) {
      const float dist = 0.12f * static_cast<float>(k);
      const float d = shader_sample_sdf(mc, s, cf, ocr, cam, add(p, mul(nv, dist)));
      acc = acc + scale * (dist - d);
      scale = scale * 0.5f;
    }
    const float v = 1.0f - 0.7f * acc;
    const float lo = v < 0.0f ? 0.0f : v;
    ao[i] = lo > 1.0f ? 1.0f : lo;
  });
}

// ---------------------------------------------------------------------------
// CSG edits (crates/rkf-edit/src/cpu_apply.rs)
// ---------------------------------------------------------------------------
static V3<float> quat_rotate(const float q[4], V3<float> v) {
  // unit quaternion rotation: v*(w*w - b.b) + b*(2 b.v) + (b x v)*(2w)
  const V3<float> b = v3<float>(q[0], q[1], q[2]);
  const float w = q[3];
  const float b2 = dot(b, b);
  const V3<float> cr = v3<float>(b.y * v.z - b.z * v.y, b.z * v.x - b.x * v.z, b.x * v.y - b.y * v.x);
  return add(add(mul(v, w * w - b2), mul(b, dot(v, b) * 2.0f)), mul(cr, w * 2.0f));
}

float orc_evaluate_shape(uint32_t shape, const float dims[3], const float pos[3]) {
  const V3<float> p = v3<float>(pos[0], pos[1], pos[2]);
  switch (shape) {  // cpu_apply.rs:231-262
    case 0:
      return length(p) - dims[0];
    case 1: {
      const float qx = std::fabs(p.x) - dims[0], qy = std::fabs(p.y) - dims[1],
                  qz = std::fabs(p.z) - dims[2];
      const V3<float> o = v3<float>(fmax_(qx, 0.0f), fmax_(qy, 0.0f), fmax_(qz, 0.0f));
      return length(o) + fmin_(fmax_(qx, fmax_(qy, qz)), 0.0f);
    }
    case 2: {
      const V3<float> a = v3<float>(0.0f, -dims[1], 0.0f), b = v3<float>(0.0f, dims[1], 0.0f);
      const V3<float> pa = sub(p, a), ba = sub(b, a);
      const float h = clampf(dot(pa, ba) / dot(ba, ba), 0.0f, 1.0f);
      return length(sub(pa, mul(ba, h))) - dims[0];
    }
    default:
      return kMaxFloat;
  }
}

float orc_evaluate_falloff(uint32_t curve, float distance, float radius) {  // cpu_apply.rs:265-283
  if (radius <= 0.0f || distance >= radius) return 0.0f;
  const float t = distance / radius;
  if (curve == 0) return 1.0f - t;
  if (curve == 1) return 1.0f - t * t * (3.0f - 2.0f * t);
  const float f = 1.0f - t;
  return f * f * f;
}

// One voxel of apply_edit_cpu (cpu_apply.rs:28-200): the brush's value at
// the voxel centre vp blended into the existing distance and material.
// Returns false where the falloff is zero (the voxel keeps its values).
static bool edit_voxel(const rkf_edit_op* op, float max_extent, const float iq[4], V3<float> vp,
                       float existing, uint32_t smat, float* nd_out, uint32_t* mat_out, bool* painted) {
  const V3<float> pos = v3<float>(op->position[0], op->position[1], op->position[2]);
  const V3<float> el = quat_rotate(iq, sub(vp, pos));
  const float ela[3] = {el.x, el.y, el.z};
  const float shape_d = orc_evaluate_shape(op->shape_type, op->dimensions, ela);
  const float dc = length(sub(vp, pos));
  const float fw = orc_evaluate_falloff(op->falloff, dc, max_extent + op->blend_k);
  if (fw <= 0.0f) return false;
  const float strength = op->strength * fw;
  float nd = existing;
  uint32_t mat = smat;
  switch (op->edit_type) {
    case 0: {  // CsgUnion
      const float e = shape_d + (1.0f - strength) * max_extent;
      nd = fmin_(existing, e);
      mat = e < existing ? op->material_id : ((nd < 0.0f && smat == 0) ? op->material_id : smat);
      break;
    }
    case 1: {  // CsgSubtract
      const float e = shape_d + (1.0f - strength) * max_extent;
      nd = fmax_(existing, -e);
      break;
    }
    case 2: {  // CsgIntersect
      const float e = shape_d - (1.0f - strength) * max_extent;
      nd = fmax_(existing, e);
      break;
    }
    case 3: {  // SmoothUnion
      const float k = fmax_(op->blend_k, 0.001f);
      const float e = shape_d + (1.0f - strength) * max_extent;
      nd = smin<float>(existing, e, k);
      mat = e < existing ? op->material_id : ((nd < 0.0f && smat == 0) ? op->material_id : smat);
      break;
    }
    case 4: {  // SmoothSubtract
      const float k = fmax_(op->blend_k, 0.001f);
      const float e = shape_d + (1.0f - strength) * max_extent;
      nd = -smin<float>(-existing, e, k);
      break;
    }
    case 5:  // Smooth (:151-157)
      nd = existing * (1.0f - strength * 0.3f);
      break;
    case 6:  // Flatten (:158-165): lerp(a, b, t) = a + (b - a) * t (:285-288) toward the plane y = 0
      nd = existing + (el.y - existing) * (strength * 0.5f);
      break;
    default:
      break;
  }
  // Paint (:166-173): VoxelSample::new(existing, material, 0) near the surface
  *painted = op->edit_type == 7 && std::fabs(existing) < op->dimensions[0] * 2.0f;
  if (*painted) mat = op->material_id;
  *nd_out = nd;
  *mat_out = mat;
  return true;
}

static V3<float> edit_voxel_centre(const float bmin[3], float vs, uint32_t vx, uint32_t vy, uint32_t vz) {
  // voxel_pos = brick_min + (v * vs) + splat(vs*0.5)   (cpu_apply.rs:52-55)
  return add(add(v3<float>(bmin[0], bmin[1], bmin[2]),
                 mul(v3<float>(static_cast<float>(vx), static_cast<float>(vy), static_cast<float>(vz)), vs)),
             v3<float>(vs * 0.5f, vs * 0.5f, vs * 0.5f));
}

int orc_apply_edit_brick(uint32_t* words, const float bmin[3], float vs, const rkf_edit_op* op) {
  const float iq[4] = {-op->rotation[0], -op->rotation[1], -op->rotation[2], op->rotation[3]};
  const float max_extent = fmax_(fmax_(op->dimensions[0], op->dimensions[1]), op->dimensions[2]);
  bool any_changed = false;
  for (uint32_t vz = 0; vz < 8; ++vz)
    for (uint32_t vy = 0; vy < 8; ++vy)
      for (uint32_t vx = 0; vx < 8; ++vx) {
        const uint32_t idx = vx + vy * 8 + vz * 64;
        const uint32_t w0 = words[2 * idx], w1 = words[2 * idx + 1];
        const float existing = f16_to_f32(static_cast<uint16_t>(w0 & 0xFFFFu));
        const uint32_t smat = (w0 >> 16) & 0x3Fu, ssec = (w0 >> 22) & 0x3Fu, sbl = w1 >> 24;
        float nd;
        uint32_t mat;
        bool painted;
        if (!edit_voxel(op, max_extent, iq, edit_voxel_centre(bmin, vs, vx, vy, vz), existing, smat, &nd, &mat,
                        &painted))
          continue;
        words[2 * idx] = pack_word0(nd, mat, painted ? 0u : ssec);
        words[2 * idx + 1] = painted ? 0u : sbl << 24;
        if (painted || std::fabs(nd - existing) > vs * 0.1f) any_changed = true;
      }
  return any_changed ? 1 : 0;
}

// The same edit on a brick stored as planes with f32 distances (the f32 and
// u8 pools: the distance the brush blends with is the decoded one, and the
// result is kept unrounded).  mat holds material | secondary << 6; blend
// (may be null) changes only where paint clears it.  Returns 1 when some
// voxel moved by more than vs/10 or was painted.
int orc_apply_edit_planes(float* dist, uint16_t* mat, uint8_t* blend, const float bmin[3], float vs,
                          const rkf_edit_op* op) {
  const float iq[4] = {-op->rotation[0], -op->rotation[1], -op->rotation[2], op->rotation[3]};
  const float max_extent = fmax_(fmax_(op->dimensions[0], op->dimensions[1]), op->dimensions[2]);
  bool any_changed = false;
  for (uint32_t vz = 0; vz < 8; ++vz)
    for (uint32_t vy = 0; vy < 8; ++vy)
      for (uint32_t vx = 0; vx < 8; ++vx) {
        const uint32_t idx = vx + vy * 8 + vz * 64;
        const float existing = dist[idx];
        const uint32_t smat = mat[idx] & 0x3Fu, ssec = (mat[idx] >> 6) & 0x3Fu;
        float nd;
        uint32_t m;
        bool painted;
        if (!edit_voxel(op, max_extent, iq, edit_voxel_centre(bmin, vs, vx, vy, vz), existing, smat, &nd, &m,
                        &painted))
          continue;
        dist[idx] = nd;
        mat[idx] = static_cast<uint16_t>((m & 0x3Fu) | ((painted ? 0u : ssec) << 6));
        if (painted && blend) blend[idx] = 0;
        if (painted || std::fabs(nd - existing) > vs * 0.1f) any_changed = true;
      }
  return any_changed ? 1 : 0;
}

// Band-normalised u8 code of one brick's 512 distances: B = min(band,
// largest finite |d|) (at least 1e-6), step = B/127; toward zero:
// |code| = min(floor(|d|/step), 127), less one where code*step rounds above
// |d|; to nearest: min(rint(|d|/step), 127); with the sign of d.
void orc_encode_u8(const float* dist, float band, int nearest, int8_t* code, float* step) {
  float m = 0.0f;
  for (int i = 0; i < 512; ++i) {
    const float a = std::fabs(dist[i]);
    if (a <= 3.0e38f && a > m) m = a;
  }
  const float range = std::fmax(std::fmin(m, band), 1e-6f);
  const float st = range / 127.0f;
  *step = st;
  for (int i = 0; i < 512; ++i) {
    const float a = std::fabs(dist[i]);
    const float qa = a / st;
    const float q = nearest ? std::nearbyint(qa) : std::floor(qa);
    int c = q >= 127.0f ? 127 : static_cast<int>(q);
    if (!nearest && c > 0 && static_cast<float>(c) * st > a) --c;
    code[i] = static_cast<int8_t>(dist[i] < 0.0f ? -c : c);
  }
}

void orc_fill_brick_with_brush(uint32_t* words, const float bmin[3], float vs,
                               const rkf_edit_op* op) {
  const float iq[4] = {-op->rotation[0], -op->rotation[1], -op->rotation[2], op->rotation[3]};
  const float max_d = vs * 8.0f;
  const V3<float> pos = v3<float>(op->position[0], op->position[1], op->position[2]);
  for (uint32_t vz = 0; vz < 8; ++vz)
    for (uint32_t vy = 0; vy < 8; ++vy)
      for (uint32_t vx = 0; vx < 8; ++vx) {
        const V3<float> vc = add(add(v3<float>(bmin[0], bmin[1], bmin[2]),
                                     mul(v3<float>(static_cast<float>(vx), static_cast<float>(vy),
                                                   static_cast<float>(vz)), vs)),
                                 v3<float>(vs * 0.5f, vs * 0.5f, vs * 0.5f));
        const V3<float> el = quat_rotate(iq, sub(vc, pos));
        const float ela[3] = {el.x, el.y, el.z};
        const float d = fmin_(orc_evaluate_shape(op->shape_type, op->dimensions, ela), max_d);
        const uint32_t idx = vx + vy * 8 + vz * 64;
        words[2 * idx] = pack_word0(d, d < 0.0f ? op->material_id : 0u, 0u);
        words[2 * idx + 1] = 0u;
      }
}

float orc_sample_brick_trilinear(const uint32_t* words, const float lp[3], float /*vs*/) {
  // sampling.rs:23-66 (single brick, clamped inside the brick)
  const float dim = 8.0f;
  float f[3];
  uint32_t i0[3], i1[3];
  float tt[3];
  for (int a = 0; a < 3; ++a) {
    f[a] = clampf(lp[a] * dim - 0.5f, 0.0f, dim - 1.0001f);
    i0[a] = static_cast<uint32_t>(std::floor(f[a]));
    i1[a] = std::min(i0[a] + 1, 7u);
    tt[a] = f[a] - static_cast<float>(i0[a]);
  }
  auto d = [&](uint32_t x, uint32_t y, uint32_t z) {
    return f16_to_f32(static_cast<uint16_t>(words[2 * (x + y * 8 + z * 64)] & 0xFFFFu));
  };
  const float c00 = d(i0[0], i0[1], i0[2]) * (1.0f - tt[0]) + d(i1[0], i0[1], i0[2]) * tt[0];
  const float c10 = d(i0[0], i1[1], i0[2]) * (1.0f - tt[0]) + d(i1[0], i1[1], i0[2]) * tt[0];
  const float c01 = d(i0[0], i0[1], i1[2]) * (1.0f - tt[0]) + d(i1[0], i0[1], i1[2]) * tt[0];
  const float c11 = d(i0[0], i1[1], i1[2]) * (1.0f - tt[0]) + d(i1[0], i1[1], i1[2]) * tt[0];
  const float c0 = c00 * (1.0f - tt[1]) + c10 * tt[1];
  const float c1 = c01 * (1.0f - tt[1]) + c11 * tt[1];
  return c0 * (1.0f - tt[2]) + c1 * tt[2];
}

// Reference defaults (gpu_scene.rs:34-43, ray_march.wgsl:28-41).
uint64_t orc_coarse_field(const rkf_gpu_object* objects, uint32_t n, float origin[3], uint32_t dims[3],
                          uint16_t* tex, uint64_t cap) {
  orc_scene sc;
  std::memset(&sc, 0, sizeof(sc));
  sc.objects = objects;
  sc.num_objects = n;
  const CoarseField c = coarse_build(&sc);
  for (int a = 0; a < 3; ++a) {
    origin[a] = c.origin[a];
    dims[a] = c.dims[a];
  }
  if (tex && cap >= c.tex.size()) std::memcpy(tex, c.tex.data(), c.tex.size() * 2);
  return c.tex.size();
}

void orc_march_params_default(rkf_march_params* p) {
  p->scene.num_objects = 0;
  p->scene.max_steps = 128;
  p->scene.max_distance = 100.0f;
  p->scene.hit_threshold = 0.001f;
  p->hard_max_steps = 1024;
  p->bisect_steps = 8;
  p->min_step = 0.0005f;
  p->near_surface_threshold = 0.02f;
  p->strategy = RKF_STRATEGY_BRUTE;
  p->reserved = 0;
}

}  // extern "C"
