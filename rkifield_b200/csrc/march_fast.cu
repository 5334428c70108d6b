// march_fast.cu — the B200 march: one persistent, work-fetching kernel for
// views (primary rays) and ray batches (closest / any-hit / soft shadow).
//
// Reference algorithm: crates/rkf-render/shaders/ray_march.wgsl:776-858
// (ray_march_brute), :641-773 (ray_march_bvh), :874-985 (ray_march_tiled),
// :941-964 (bisection), :1003-1032
// (normals), :1036-1112 (ray generation and G-buffer), and
// shade_common_shading.wgsl:9-33 (soft_shadow).
//
// Execution model.  Each lane owns one ray at a time.  A warp alternates
//   1. refill: idle lanes take the next work ids from a global counter
//      (one warp-aggregated atomic); ids walk views tile by tile, so a warp's
//      rays stay spatially coherent;
//   2. march: up to K sphere-tracing iterations (K = the compaction interval)
//      in a tight loop, leaving early once no lane is still marching;
//   3. finish: lanes that hit run their bisection (8 samples) and central
//      differences (6 samples) together, one sample per iteration;
//   4. epilogue: finished lanes write their G-buffer entry and go idle.
// So a ray that ends early frees its lane within K iterations instead of
// idling it until the slowest ray of the warp finishes.  The hit material is
// read once, from the position that decided it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "../../include/rkf_cuda_testing.h"
#include "ctx.h"
#include "march.h"
#include "f32x2.cuh"
#include "sampler.cuh"
#include "tiled.h"
#include "tile_order.h"

namespace rkf {

namespace detail {

enum : uint32_t { ST_IDLE = 0, ST_MARCH, ST_BISECT, ST_NORMAL, ST_EPI, ST_SHADOW };

constexpr uint32_t kFull = 0xFFFFFFFFu;

// Per-lane ray state that is read or written only when a ray starts, hits
// or ends.
struct ColdState {
  uint32_t seg, idx, hit_obj, sub;
  float lo, hi, mat_t, gpos, shadow;
  uint32_t tile_base, tile_count;  // tiled strategy: the ray's object list (kNoTiles: every object)
  bool hit, bisected, mat_ok;
  // multi-object empty-space path: bits 0-7, the voxelized objects of the
  // path (KParams::ev) whose EMPTY runs the ray may take (under the tiled
  // strategy, those its object list holds); bits 8-15, the one whose cube
  // the ray is in (its last successful probe).  (Also makes an odd number of
  // words per lane: a warp's accesses hit 32 distinct banks.)
  uint32_t vox_listed;
};
static_assert(sizeof(ColdState) % 8 == 4, "ColdState must span an odd number of 32-bit words");

// Multi-object empty-space path.  Each analytic primitive lies inside a ball
// of radius R around its local origin (sphere r, box |b|, capsule |r|+|h|,
// torus |R|+|r|, cylinder |(r, h)|), and its exact distance is at least |l|-R
// at a local position l.  With c the local origin in world space, sigma a
// lower bound of the smallest singular value of inverse_world's linear part
// and s the object's min_scale, the FP32 value of evaluate_object at a world
// position p is at least (sigma*|p - c| - R - rounding)*s.  The host folds
// the voxelized object's largest EMPTY value and bounds of every rounding
// (the object's own evaluation, the ray's position, this centre's rounding)
// into a radius a + b*P, P = |o| + |d|*|tmax| bounding the magnitude of a
// ray's positions: outside that ball the object's value exceeds every EMPTY
// value, so wherever the voxelized object samples EMPTY, the minimum over
// the scene is that sample, bit for bit.
struct FarBall {
  float c[3];     // world-space centre (half-space: the coefficients G)
  float a, b;     // radius a + b * P (box: margin a + b * P beyond the half extents;
                  // half-space: G.w + H <= a + b * P)
  uint32_t path;  // the object's index in the empty-space path (KParams::ev), or ~0u
  float h[3];     // box: world-space half extents (half-space: h[0] = H)
  uint32_t box;   // 1: an axis-aligned box around c instead of a ball; 2: a half-space
};

// One voxelized object of the multi-object empty-space path.  Wherever the
// ray lies in EMPTY cubes of a set of these objects (each on its own field)
// and outside the balls of every other object (analytic or voxelized), each
// object of the set samples its EMPTY value and every other object a larger
// value, so the scene's minimum is the least EMPTY value of the set.
constexpr uint32_t kMaxEmptyVox = 8;
struct EmptyVox {
  uint32_t obj;       // object index
  uint32_t plain;     // zero translation and unit scale
  float probe_min;    // probe for a cube once a sample was at least this
  float empty_lo;     // lower bound of every EMPTY value (times the scale)
  float empty_lo_t, empty_hi;  // tight bounds of an EMPTY step
};

struct KParams {
  ObjDev objs[kMaxObjectsFast];  // object table in the constant parameter bank
  SceneDev s;
  const Segment* segs;
  uint32_t nseg;
  uint32_t tile_w, tile_h;
  uint32_t interval;
  uint64_t total;          // work ids of this launch: id0 .. id0 + total - 1
  uint64_t id0;
  unsigned long long* counter;
  rkf_march_params p;
  float probe_min;  // empty-space path: probe for a cube once a sample was at least this
  uint32_t budget;     // empty-space path: steps per run before the warp re-converges
  uint32_t plain_obj;  // object 0 has zero translation and unit scale
  uint32_t refill_active;  // leave the march loop once at most this many lanes march
  uint32_t run_probe;      // empty-space path: probe the next cube inside a run
  uint32_t tail_share;     // empty-space path: warp-shared EMPTY runs once at most this many lanes march
  TiledDev td;             // tiled strategy inputs (views of a tiled launch)
  uint32_t tiled;
  float empty_lo;          // empty-space path: lower bound of every EMPTY value
  float empty_lo_t, empty_hi;  // empty-space path: tight bounds of an EMPTY step
  uint32_t settle_links;   // empty-space path: cubes a settling chain may add (0 = off)
  const rkf_bvh_node* bvh; // BVH strategy: the imported tree, root first
  const uint32_t* bvh_next;  // per node: the walk's next node (bits 0-30), descend (bit 31)
  uint32_t use_bvh;
  // multi-object empty-space path: the voxelized objects that take EMPTY
  // runs, and a ball for every object that needs one (bounding the largest
  // EMPTY value of the path)
  EmptyVox ev[kMaxEmptyVox];
  uint32_t n_ev;
  FarBall ball[kMaxObjectsFast];
  uint32_t n_ball;
};
static_assert(sizeof(KParams) <= 32000, "the launch parameters must fit the kernel parameter space");

// The candidate loop of ray_march_bvh (ray_march.wgsl:672-721): a stack walk
// of the tree from the root that skips every node whose AABB lies farther
// from the position than the best distance so far, evaluates the objects of
// the leaves it reaches (object indices beyond the object count are skipped),
// and pushes the left then the right child while fewer than 31 entries are on
// the stack (so the right child is visited first).  On the trees the import
// admits the stack's content at each node is fixed by the tree, so the same
// walk runs from the per-node links bvh.cu derives (next node after the
// subtree, whether to descend), without a stack.  The distance to a box is
// length(clamp(pos, min, max) - pos); its square root is taken only where the
// comparison needs it (an exact zero stays zero, and any length exceeds a
// negative best).
template <int PREC>
__device__ __forceinline__ float eval_bvh(const SceneDev& s, const ObjDev* objs, const rkf_bvh_node* nodes,
                                          const uint32_t* __restrict__ next, uint32_t nobj, float wx, float wy,
                                          float wz, float& best_un, uint32_t& best_i, LaneCache& lc) {
  constexpr uint32_t kEnd = 0x7FFFFFFFu;
  float best = kMaxFloat;
  best_un = kMaxFloat;
  best_i = 0;
  uint32_t i = 0;
  while (i != kEnd) {
    const float4* nd = reinterpret_cast<const float4*>(nodes + i);
    const float4 a = __ldg(nd), b = __ldg(nd + 1);
    const uint32_t link = __ldg(next + i);
    const float ex = __fsub_rn(fminf(fmaxf(wx, a.x), b.x), wx);
    const float ey = __fsub_rn(fminf(fmaxf(wy, a.y), b.y), wy);
    const float ez = __fsub_rn(fminf(fmaxf(wz, a.z), b.z), wz);
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez));
    bool skip;
    if (d2 == 0.0f) skip = 0.0f > best;
    else if (best < 0.0f && d2 == d2) skip = true;
    else skip = __fsqrt_rn(d2) > best;
    if (skip) {
      i = link & kEnd;
      continue;
    }
    const uint32_t left = __float_as_uint(a.w), ro = __float_as_uint(b.w);
    if (left == RKF_BVH_INVALID) {
      if (ro < nobj) {
        float du;
        const float d = eval_obj<PREC>(s, objs[ro], wx, wy, wz, &du, lc);
        if (d < best) {
          best = d;
          best_un = du;
          best_i = ro;
        }
      }
      i = link & kEnd;
    } else {
      i = (link >> 31) ? ro : (link & kEnd);
    }
  }
  return best;
}

// Object set of a launch: several objects, exactly one, or exactly one that
// qualifies for the empty-space path (voxelized, translation-only
// inverse_world, verified exact quotient, fewer than 2^20 voxels per axis).
// OBJ_SINGLE_EMPTY_TILED: the empty-space path of a tiled launch (EMPTY runs
// on the tiled empty-space field, tiled full steps elsewhere).
// OBJ_MULTI_EMPTY: one object that qualifies for the empty-space path plus
// analytic objects that each fit a ball (FarBall) and objects of no type; its
// EMPTY runs and settling chains stay outside every ball.
// OBJ_MULTI_EMPTY_TILED: the same under the tiled strategy (EMPTY runs on
// the tiled empty-space field, for rays whose object list holds the
// voxelized object; tiled full steps elsewhere).
enum : int {
  OBJ_MULTI = 0,
  OBJ_SINGLE = 1,
  OBJ_SINGLE_EMPTY = 2,
  OBJ_SINGLE_EMPTY_TILED = 3,
  OBJ_MULTI_EMPTY = 4,
  OBJ_MULTI_EMPTY_TILED = 5
};

// Interval helpers in directed rounding: each result interval contains the
// exact result for every value of the operand intervals.
__device__ __forceinline__ void iv_mul(float x, float lo, float hi, float& rlo, float& rhi) {  // x * [lo, hi]
  if (x >= 0.0f) {
    rlo = __fmul_rd(x, lo);
    rhi = __fmul_ru(x, hi);
  } else {
    rlo = __fmul_rd(x, hi);
    rhi = __fmul_ru(x, lo);
  }
}
__device__ __forceinline__ void iv_sq(float lo, float hi, float& rlo, float& rhi) {  // [lo, hi]^2
  const float mlo = lo > 0.0f ? lo : (hi < 0.0f ? -hi : 0.0f);
  const float mhi = fmaxf(fabsf(lo), fabsf(hi));
  rlo = __fmul_rd(mlo, mlo);
  rhi = __fmul_ru(mhi, mhi);
}

// Largest t' >= t such that every position of the ray o + d*u, u in [t, t'],
// lies outside every ball (kMaxFloat when no ball lies ahead), skipping the
// balls of the path objects in `skip` (those the run's set samples); -1 when the
// position at t may lie inside one, with *recheck set to the earliest time
// the ray may leave the balls that may hold it (else -1).  Per ball, with
// w = o - c: the line's squared distance to the centre is |w|^2 - (d.w)^2/|d|^2,
// its closest approach is at -(d.w)/|d|^2, and the chord within the ball
// spans sqrt((rho^2 - h^2)/|d|^2) on each side.  Every quantity is an interval
// evaluated in directed rounding, so the entry time used is a lower bound
// and the exit time an upper bound of the exact ones.  A non-finite ray (or
// a zero direction) makes every ball near.  Out of line: the march loop
// calls it about once per ray, and its code would otherwise sit among the
// loop's hot paths (measured 3% faster out of line).
__device__ __noinline__ float far_limit(const FarBall* __restrict__ far, uint32_t n, uint32_t skip, float ox,
                                           float oy, float oz, float dx, float dy, float dz, float tmax, float t,
                                           float& recheck) {
  const float a_lo = __fadd_rd(__fadd_rd(__fmul_rd(dx, dx), __fmul_rd(dy, dy)), __fmul_rd(dz, dz));
  const float a_hi = __fadd_ru(__fadd_ru(__fmul_ru(dx, dx), __fmul_ru(dy, dy)), __fmul_ru(dz, dz));
  // P >= |o| + |d| |tmax| (an L1 norm bounds the L2 norm)
  const float P = __fadd_ru(__fadd_ru(__fadd_ru(fabsf(ox), fabsf(oy)), fabsf(oz)),
                            __fmul_ru(__fsqrt_ru(a_hi), fabsf(tmax)));
  float lim = kMaxFloat;
  bool inside = false;
  recheck = kMaxFloat;
  for (uint32_t j = 0; j < n; ++j) {
    const FarBall& f = far[j];
    if (f.path < 32u && ((skip >> f.path) & 1u)) continue;  // an object of the run's set
    if (f.box == 2) {
      // half-space G.w + H <= m, m = a + b*P (a plane's small values lie in
      // it): along the ray its coordinate G.(o + d u) + H - m is at least
      // s0 + s1 u for u >= 0, both rounded down
      const float m = __fadd_ru(f.a, __fmul_ru(f.b, P));
      const float s0 = __fsub_rd(__fadd_rd(__fadd_rd(__fadd_rd(__fmul_rd(f.c[0], ox), __fmul_rd(f.c[1], oy)),
                                                     __fmul_rd(f.c[2], oz)), f.h[0]), m);
      const float s1 = __fadd_rd(__fadd_rd(__fmul_rd(f.c[0], dx), __fmul_rd(f.c[1], dy)), __fmul_rd(f.c[2], dz));
      const float now = __fadd_rd(s0, __fmul_rd(s1, t));  // t >= 0
      if (s1 >= 0.0f) {
        if (now > 0.0f) continue;  // outside and not approaching: never inside
        inside = true;             // may be inside now
        // s0 <= now <= 0: outside again for u > -s0 / s1
        if (s1 > 0.0f) recheck = fminf(recheck, __fdiv_ru(-s0, s1));
      } else if (s1 < 0.0f && now > 0.0f) {
        // approaching, outside now (s0 > 0): inside no earlier than s0 / -s1
        lim = fminf(lim, fmaxf(t, __fdiv_rd(s0, -s1)));
      } else {  // inside from now on, or NaN
        inside = true;
      }
      continue;
    }
    if (f.box) {
      // slab test of the box [c - h - m, c + h + m], m = a + b*P: the entry
      // time rounded down and the exit time rounded up
      const float m = __fadd_ru(f.a, __fmul_ru(f.b, P));
      const float o3[3] = {ox, oy, oz}, d3[3] = {dx, dy, dz};
      float e = -kMaxFloat, x = kMaxFloat;
      bool miss = false;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float hw = __fadd_ru(f.h[k], m);
        const float lo = __fsub_rd(f.c[k], hw), hi = __fadd_ru(f.c[k], hw);
        if (d3[k] > 0.0f) {
          e = fmaxf(e, __fdiv_rd(__fsub_rd(lo, o3[k]), d3[k]));
          x = fminf(x, __fdiv_ru(__fsub_ru(hi, o3[k]), d3[k]));
        } else if (d3[k] < 0.0f) {
          e = fmaxf(e, __fdiv_rd(__fsub_ru(hi, o3[k]), d3[k]));
          x = fminf(x, __fdiv_ru(__fsub_rd(lo, o3[k]), d3[k]));
        } else if (!(o3[k] >= lo && o3[k] <= hi)) {
          miss = true;  // parallel to this slab and outside it (NaN: not a miss)
        }
      }
      if (miss || e > x) continue;
      if (t < e) {
        lim = fminf(lim, e);
      } else if (!(t > x)) {  // may be inside now (or NaN)
        inside = true;
        recheck = fminf(recheck, x);
      }
      continue;
    }
    const float rho = __fadd_ru(f.a, __fmul_ru(f.b, P));
    const float rho2 = __fmul_ru(rho, rho);
    const float wxl = __fsub_rd(ox, f.c[0]), wxh = __fsub_ru(ox, f.c[0]);
    const float wyl = __fsub_rd(oy, f.c[1]), wyh = __fsub_ru(oy, f.c[1]);
    const float wzl = __fsub_rd(oz, f.c[2]), wzh = __fsub_ru(oz, f.c[2]);
    float sxl, sxh, syl, syh, szl, szh;
    iv_sq(wxl, wxh, sxl, sxh);
    iv_sq(wyl, wyh, syl, syh);
    iv_sq(wzl, wzh, szl, szh);
    const float W_lo = __fadd_rd(__fadd_rd(sxl, syl), szl);
    float pxl, pxh, pyl, pyh, pzl, pzh;  // d.w
    iv_mul(dx, wxl, wxh, pxl, pxh);
    iv_mul(dy, wyl, wyh, pyl, pyh);
    iv_mul(dz, wzl, wzh, pzl, pzh);
    const float b_lo = __fadd_rd(__fadd_rd(pxl, pyl), pzl), b_hi = __fadd_ru(__fadd_ru(pxh, pyh), pzh);
    float b2l, b2h;
    iv_sq(b_lo, b_hi, b2l, b2h);
    const float h2_lo = __fsub_rd(W_lo, __fdiv_ru(b2h, a_lo));
    if (h2_lo > rho2) continue;  // the line never comes within rho (NaN: not skipped)
    const float half = __fsqrt_ru(__fdiv_ru(__fsub_ru(rho2, h2_lo), a_lo));
    const float nb_lo = -b_hi, nb_hi = -b_lo;  // closest approach -(d.w)/|d|^2
    const float tc_lo = __fdiv_rd(nb_lo, nb_lo < 0.0f ? a_lo : a_hi);
    const float tc_hi = __fdiv_ru(nb_hi, nb_hi > 0.0f ? a_lo : a_hi);
    const float e = __fsub_rd(tc_lo, half), x = __fadd_ru(tc_hi, half);
    if (t < e) {
      lim = fminf(lim, e);
    } else if (!(t > x)) {  // may be inside now (or NaN)
      inside = true;
      recheck = fminf(recheck, x);
    }
  }
  if (inside) return -1.0f;
  recheck = -1.0f;
  return lim;
}

// Grid coordinate (position + half grid size, object-local) of the ray at t,
// rounded exactly as eval_obj -> sample_vox round it for a translation-only
// object.
__device__ __forceinline__ float grid_coord(float o, float d, float t, float m, float half) {
  return __fadd_rn(__fadd_rn(__fadd_rn(o, __fmul_rn(d, t)), m), half);
}

// The EMPTY sampling value of sample_vox at a grid coordinate whose trilinear
// cell lies in EMPTY blocks inside the grid and the geometry box (no clamp,
// no outside term), times the object's scale: eval_obj's result there.
__device__ __forceinline__ float empty_value(const ObjDev& o, float gx, float gy, float gz) {
  const float vx = __fsub_rn(exact_div_vs(gx, o.vs, o.rcp_vs), 0.5f);
  const float vy = __fsub_rn(exact_div_vs(gy, o.vs, o.rcp_vs), 0.5f);
  const float vz = __fsub_rn(exact_div_vs(gz, o.vs, o.rcp_vs), 0.5f);
  const float v = mix3_const(o.be, __fsub_rn(vx, floorf(vx)), __fsub_rn(vy, floorf(vy)), __fsub_rn(vz, floorf(vz)));
  return __fmul_rn(v, o.min_scale);
}

// A ray as the EMPTY-cube probes see it: origin and step direction, the
// direction's reciprocals (for the exit times) and the containment margin:
// 0.1 voxel plus 2^-18 of the magnitudes involved, which covers every
// rounding between t and the sampler's grid coordinate and every rounding of
// the cube's faces and exit times computed here.
struct ProbeRay {
  float o[3], d[3], inv[3], margin;
};

__device__ __forceinline__ ProbeRay probe_ray(const ObjDev& ob, float ox, float oy, float oz, float dx, float dy,
                                              float dz) {
  ProbeRay r;
  r.o[0] = ox, r.o[1] = oy, r.o[2] = oz;
  r.d[0] = dx, r.d[1] = dy, r.d[2] = dz;
  float mag = 1.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    r.inv[a] = __frcp_rn(r.d[a]);
    mag += fabsf(r.o[a]) + fabsf(ob.m[12 + a]) + ob.gs[a];
  }
  r.margin = 0.1f * ob.vs + mag * 3.814697265625e-6f;
  return r;
}

// Largest t up to which the ray stays inside a cube of EMPTY blocks (from the
// empty-space distance field), clipped to the grid and the geometry box, and
// shrunk by the ray's margin: for each t' in [t_anchor, result] the trilinear
// corners of the sample at t' lie in the cube, so the sample there is exactly
// empty_value().  The cube is the one around the block of the position at
// t_probe; which block that is only chooses the cube (its EMPTY-ness holds for
// any block), so it is found with plain arithmetic, while the position at
// t_anchor -- rounded exactly as the march rounds it -- must lie in the shrunk
// cube.  Positions are monotone in t along each axis, so the exit faces
// suffice.  -1 when there is no such cube.
__device__ float probe_cube(const ObjDev& o, const uint8_t* __restrict__ field, const ProbeRay& r, float t_anchor,
                            float t_probe) {
  int k[3];
  float p[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    p[a] = __fadd_rn(r.o[a], __fmul_rn(r.d[a], t_anchor));
    const float pp = r.o[a] + r.d[a] * t_probe;
    const float f = floorf((pp + o.m[12 + a] + o.half_gs[a]) * o.rcp_vs - 0.5f);
    if (!(f >= 0.0f && f <= static_cast<float>(o.tv[a] - 1))) return -1.0f;
    k[a] = static_cast<int>(f) >> 6;
  }
  const uint32_t s = __ldg(field + o.top_off + k[0] + k[1] * o.tdim[0] + k[2] * o.tdim[0] * o.tdim[1]);
  if (s == 0) return -1.0f;
  const int rad = static_cast<int>(s) - 1;  // every block within rad is EMPTY
  float t_exit = kMaxFloat;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int lo_v = max(0, (k[a] - rad) * 64), hi_v = min(o.tv[a] - 1, (k[a] + rad) * 64 + 63);
    const float base = -o.half_gs[a] - o.m[12 + a];
    float wlo = (static_cast<float>(lo_v) + 0.5f) * o.vs + base + r.margin;
    float whi = (static_cast<float>(hi_v) + 0.5f) * o.vs + base - r.margin;
    if (o.has_geom) {
      wlo = fmaxf(wlo, o.gmin[a] - o.m[12 + a] + r.margin);
      whi = fminf(whi, o.gmax[a] - o.m[12 + a] - r.margin);
    }
    if (!(p[a] >= wlo && p[a] <= whi)) return -1.0f;
    if (r.d[a] > 0.0f) t_exit = fminf(t_exit, (whi - r.o[a]) * r.inv[a]);
    else if (r.d[a] < 0.0f) t_exit = fminf(t_exit, (wlo - r.o[a]) * r.inv[a]);
  }
  return t_exit;
}

__device__ __forceinline__ float probe_empty(const ObjDev& o, const uint8_t* __restrict__ field, float ox,
                                             float oy, float oz, float dx, float dy, float dz, float t) {
  const ProbeRay r = probe_ray(o, ox, oy, oz, dx, dy, dz);
  return probe_cube(o, field, r, t, t);
}

// Extend an interval [t, cover] of EMPTY-cube positions along the ray through
// at most `links` further cubes, until it reaches `need`.  The next cube is
// the one around the block half a block ahead of the current end (else around
// the end's own block) and must contain the current end, so the union stays
// one interval.  Returns the new end.
__device__ float extend_cover(const ObjDev& o, const uint8_t* __restrict__ field, float ox, float oy, float oz,
                              float dx, float dy, float dz, float cover, float need, uint32_t links) {
  const ProbeRay r = probe_ray(o, ox, oy, oz, dx, dy, dz);
  const float ahead = 32.0f * o.vs;
  for (uint32_t i = 0; i < links && cover < need; ++i) {
    float nx = probe_cube(o, field, r, cover, cover + ahead);
    if (!(nx > cover)) {
      nx = probe_cube(o, field, r, cover, cover);
      if (!(nx > cover)) break;
    }
    cover = nx;
  }
  return cover;
}

__device__ __forceinline__ uint32_t find_segment(const Segment* segs, uint32_t nseg, uint64_t id) {
  uint32_t lo = 0, hi = nseg;  // last segment with first <= id
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (segs[mid].first <= id) lo = mid; else hi = mid;
  }
  return lo;
}

// Minimum over objects [ob, oe) of evaluate_object at world position q.
// SINGLE: the scene is exactly one object (object 0).
template <int PREC, bool SINGLE>
__device__ __forceinline__ float eval_min(const SceneDev& s, const ObjDev* objs, uint32_t ob,
                                          uint32_t oe, float qx, float qy, float qz, float& best_un,
                                          uint32_t& best_i, LaneCache& lc) {
  if (SINGLE) {
    best_i = 0;
    return eval_obj<PREC>(s, objs[0], qx, qy, qz, &best_un, lc);
  }
  float best = kMaxFloat;
  best_un = kMaxFloat;
  best_i = ob;
  for (uint32_t oi = ob; oi < oe; ++oi) {
    float du;
    const float d = eval_obj<PREC>(s, objs[oi], qx, qy, qz, &du, lc);
    if (d < best) {
      best = d;
      best_un = du;
      best_i = oi;
    }
  }
  return best;
}

// Up to n march steps of a ray through EMPTY cubes: each sample is
// empty_value().  The run stops before a step whose sample is below brk or
// whose t is past tmax (the full step decides those), after the step that
// makes max_near samples below near_thr, and where the ray leaves its cube
// (t > box_t).  INRUN: a lane whose cube ends probes the next cube in place
// and runs on (FAR: clipped at far_t, the end of the positions outside every
// ball); stop_full tells whether the next step must be a full one.
// PLAIN: the object's translation is zero and its scale one, where adding the
// translation and multiplying by the scale are exact identities.  CLEAN: every
// EMPTY value is at least brk, near_thr and min_step (the caller checks this
// against a lower bound), so those comparisons are known and skipped.
// Returns the number of steps taken.
template <bool PLAIN, bool CLEAN, bool INRUN, bool FAR>
__device__ __forceinline__ uint32_t empty_run(const ObjDev& o, const uint8_t* __restrict__ field, float ox,
                                              float oy, float oz, float dx, float dy, float dz, float tmax,
                                              uint32_t n, float brk, float near_thr, float min_step,
                                              uint32_t max_near, float far_t, float& t, float& box_t,
                                              float& prev_t, float& prev_dist, uint32_t& near, bool& stop_full) {
  uint32_t c = 0;
  float lim = fminf(box_t, tmax);
  stop_full = false;
#pragma unroll 2
  for (; c < n; ++c) {
    if (t > lim) {
      if (!INRUN || t > tmax) {
        stop_full = t > tmax;
        break;
      }
      box_t = probe_empty(o, field, ox, oy, oz, dx, dy, dz, t);
      if (FAR) box_t = fminf(box_t, far_t);
      lim = fminf(box_t, tmax);
      if (t > lim) {
        stop_full = true;
        break;
      }
    }
    float gx, gy, gz;
    if (PLAIN) {
      gx = __fadd_rn(__fadd_rn(ox, __fmul_rn(dx, t)), o.half_gs[0]);
      gy = __fadd_rn(__fadd_rn(oy, __fmul_rn(dy, t)), o.half_gs[1]);
      gz = __fadd_rn(__fadd_rn(oz, __fmul_rn(dz, t)), o.half_gs[2]);
    } else {
      gx = grid_coord(ox, dx, t, o.m[12], o.half_gs[0]);
      gy = grid_coord(oy, dy, t, o.m[13], o.half_gs[1]);
      gz = grid_coord(oz, dz, t, o.m[14], o.half_gs[2]);
    }
    const float vx = __fsub_rn(exact_div_vs(gx, o.vs, o.rcp_vs), 0.5f);
    const float vy = __fsub_rn(exact_div_vs(gy, o.vs, o.rcp_vs), 0.5f);
    const float vz = __fsub_rn(exact_div_vs(gz, o.vs, o.rcp_vs), 0.5f);
    float d = mix3_const(o.be, __fsub_rn(vx, floorf(vx)), __fsub_rn(vy, floorf(vy)), __fsub_rn(vz, floorf(vz)));
    if (!PLAIN) d = __fmul_rn(d, o.min_scale);
    if (!CLEAN && !(d >= brk)) {  // no step: the full step redoes this sample
      stop_full = true;
      break;
    }
    prev_t = t;
    prev_dist = d;
    if (CLEAN) {
      t = __fadd_rn(t, d);
      continue;
    }
    t = __fadd_rn(t, fmax_(d, min_step));
    if (d < near_thr && ++near >= max_near) {
      stop_full = true;
      return c + 1;
    }
  }
  return c;
}

// The EMPTY value of a plain object (zero translation, unit scale) at the
// ray's position at t: empty_run<PLAIN=true>'s step with the x and y chains
// packed into two-wide FP32 instructions (z stays scalar) -- the same
// operations on the same values, so the same bits.
__device__ __forceinline__ float empty_value_x2(f2 o01, f2 d01, f2 h01, f2 r2, f2 nvs2, f2 half2, float oz, float dz,
                                                float hz, float vs, float rcp, float be, float t) {
  const f2 g01 = f2_add(f2_add(o01, f2_mul(d01, f2_pack(t, t))), h01);
  const f2 q0 = f2_mul(g01, r2);
  const f2 v01 = f2_sub(f2_fma(f2_fma(q0, nvs2, g01), r2, q0), half2);
  const float vz = __fsub_rn(exact_div_vs(__fadd_rn(__fadd_rn(oz, __fmul_rn(dz, t)), hz), vs, rcp), 0.5f);
  float vx, vy;
  f2_unpack(v01, vx, vy);
  float tx, ty;
  f2_unpack(f2_sub(v01, f2_pack(floorf(vx), floorf(vy))), tx, ty);
  return mix3_const(be, tx, ty, __fsub_rn(vz, floorf(vz)));
}

// empty_run<PLAIN=true, CLEAN=true> two steps at a time.  Each step is
// t' = t + E(t), a chain in which every step waits for the last.  E(t)
// equals the brick extent c (the EMPTY constant) exactly for most positions
// (the three nested mix(c, c, f) round back to c for about 93% of
// positions), so the position of the next step is taken to be t + c (the
// rounding the step would make) and both E values are computed
// independently.  The second step is accepted when the first value was
// exactly c -- then its position is the one the serial march reaches, bit
// for bit -- and when it passes the serial loop's checks (budget, cube end,
// tmax); otherwise the first step is taken alone, with its value.  (Four
// steps at a time measured 3-4% slower on the 1080p view: the longer code
// raised instruction-fetch stalls by more than it cut dependency stalls.)
template <bool INRUN, bool FAR>
__device__ __forceinline__ uint32_t empty_run_x2(const ObjDev& o, const uint8_t* __restrict__ field, float ox,
                                                 float oy, float oz, float dx, float dy, float dz, float tmax,
                                                 uint32_t n, float far_t, float& t, float& box_t, float& prev_t,
                                                 float& prev_dist, bool& stop_full) {
  uint32_t c = 0;
  float lim = fminf(box_t, tmax);
  stop_full = false;
  const f2 o01 = f2_pack(ox, oy), d01 = f2_pack(dx, dy), h01 = f2_pack(o.half_gs[0], o.half_gs[1]);
  const f2 r2 = f2_pack(o.rcp_vs, o.rcp_vs), nvs2 = f2_pack(-o.vs, -o.vs), half2 = f2_pack(0.5f, 0.5f);
  const float hz = o.half_gs[2], vs = o.vs, rcp = o.rcp_vs, be = o.be;
  while (c < n) {
    if (t > lim) {
      if (!INRUN || t > tmax) {
        stop_full = t > tmax;
        break;
      }
      box_t = probe_empty(o, field, ox, oy, oz, dx, dy, dz, t);
      if (FAR) box_t = fminf(box_t, far_t);
      lim = fminf(box_t, tmax);
      if (t > lim) {
        stop_full = true;
        break;
      }
    }
    // the position of the next step if this value is c
    const float t1 = __fadd_rn(t, be);
    const float e0 = empty_value_x2(o01, d01, h01, r2, nvs2, half2, oz, dz, hz, vs, rcp, be, t);
    const float e1 = empty_value_x2(o01, d01, h01, r2, nvs2, half2, oz, dz, hz, vs, rcp, be, t1);
    // step 0 passed the checks above; step 1 needs the first value to be c
    // (so that t1 is the serial position) and the serial checks
    float pt = t, pd = e0;
    ++c;
    if (e0 == be && c < n && t1 <= lim) {
      pt = t1;
      pd = e1;
      ++c;
    }
    prev_t = pt;
    prev_dist = pd;
    t = __fadd_rn(pt, pd);
  }
  return c;
}

// empty_run_x2<INRUN=false>'s run taken by a whole warp, for the lanes that
// pass pend, one lane's run after another (the launch's tail: few lanes
// still march and the others have no work left).  Lane j of a round samples
// the j-th step ahead.  Within t's binade [2^e, 2^(e+1)), whose spacing is u,
// every t' is a multiple of u, so fl(t' + c) = t' + r with r = fl(t + c) - t
// (c rounded to a multiple of u) unless c lies exactly halfway between two
// multiples, where the rounding would depend on t' itself.  Away from such a
// tie the serial positions while every value is c are therefore exactly
// t + j*r (j*r and the sum are exact while t + j*r < 2^(e+1)), and lane j
// computes its own without waiting for the others.  A round accepts the
// steps up to the first value that is not c (that step is taken with its
// value), or up to the first position past the binade, the run's end
// (t > lim) or its budget (n steps), and the next position comes from the
// last accepted step as the serial loop makes it.  A tie, or t too small
// for this arithmetic, leaves lane 0 alone: one serial step per round.
// Every lane of the warp must call this.
__device__ __noinline__ void shared_runs(const ObjDev& o, bool pend, float ox, float oy, float oz, float dx,
                                         float dy, float dz, float lim, float tmax, uint32_t n, float& t,
                                         float& prev_t, float& prev_dist, uint32_t& c_out, bool& stop_full) {
  const uint32_t lane = threadIdx.x & 31u;
  const f2 h01 = f2_pack(o.half_gs[0], o.half_gs[1]);
  const f2 r2 = f2_pack(o.rcp_vs, o.rcp_vs), nvs2 = f2_pack(-o.vs, -o.vs), half2 = f2_pack(0.5f, 0.5f);
  const float hz = o.half_gs[2], vs = o.vs, rcp = o.rcp_vs, be = o.be;
  const float fj = static_cast<float>(lane);
  for (uint32_t todo = __ballot_sync(kFull, pend); todo; todo &= todo - 1u) {
    const uint32_t L = __ffs(todo) - 1u;
    const float rox = __shfl_sync(kFull, ox, L), roy = __shfl_sync(kFull, oy, L), roz = __shfl_sync(kFull, oz, L);
    const float rdx = __shfl_sync(kFull, dx, L), rdy = __shfl_sync(kFull, dy, L), rdz = __shfl_sync(kFull, dz, L);
    const float rlim = __shfl_sync(kFull, lim, L), rtmax = __shfl_sync(kFull, tmax, L);
    const uint32_t rn = __shfl_sync(kFull, n, L);
    float rt = __shfl_sync(kFull, t, L);
    const f2 o01 = f2_pack(rox, roy), d01 = f2_pack(rdx, rdy);
    uint32_t c = 0;
    float pt = 0.0f, pd = 0.0f;
    bool sf = false;
    for (;;) {
      const uint32_t bits = __float_as_uint(rt) & 0x7f800000u;  // t >= 0
      const float top = __uint_as_float(bits + 0x00800000u);    // 2^(e+1)
      const float u = __uint_as_float(bits - (23u << 23));      // spacing of [2^e, 2^(e+1))
      const float r = __fsub_rn(__fadd_rn(rt, be), rt);
      const bool wide = rt >= 1.0e-30f && !(fabsf(__fsub_rn(be, r)) == __fmul_rn(0.5f, u));
      const float tj = lane == 0 ? rt : __fadd_rn(rt, __fmul_rn(fj, r));
      const bool ok = (lane == 0 || (wide && tj < top)) && !(tj > rlim) && c + lane < rn;
      const float ej = empty_value_x2(o01, d01, h01, r2, nvs2, half2, roz, rdz, hz, vs, rcp, be, tj);
      const uint32_t m_stop = __ballot_sync(kFull, !ok);
      const uint32_t m_odd = __ballot_sync(kFull, ok && ej != be);
      const uint32_t first_stop = m_stop ? __ffs(m_stop) - 1u : 32u;
      const uint32_t first_odd = m_odd ? __ffs(m_odd) - 1u : 32u;
      const uint32_t steps = first_odd < first_stop ? first_odd + 1u : first_stop;
      if (steps == 0) {  // lane 0 stopped: the run ends here, as the serial loop ends it
        sf = c < rn && rt > rtmax;
        break;
      }
      pt = __shfl_sync(kFull, tj, steps - 1u);
      pd = __shfl_sync(kFull, ej, steps - 1u);
      c += steps;
      rt = __fadd_rn(pt, pd);
    }
    if (lane == L) {
      t = rt;
      c_out = c;
      stop_full = sf;
      if (c) {
        prev_t = pt;
        prev_dist = pd;
      }
    }
  }
}

// Up to n march steps through positions where every object of the set
// (path objects, at least two) samples its EMPTY value and every other
// object lies beyond its ball: each step's value is the least of the set's
// EMPTY values, computed as eval_obj -> sample_vox would round it.  The run
// stops at the end of the nearest cube (box_t, already clipped at the first
// ball ahead), before a step whose value is below brk, and after the step
// that makes max_near values below near_thr; CLEAN: the values clear every
// threshold (a lower bound checked by the caller).  Returns the steps taken.
template <bool CLEAN>
__device__ __noinline__ uint32_t empty_run_set(const ObjDev* objs, const EmptyVox* ev, uint32_t set, uint32_t n_ev,
                                               float ox, float oy, float oz, float dx, float dy, float dz, float tmax,
                                               uint32_t n, float brk, float near_thr, float min_step,
                                               uint32_t max_near, float& t, float box_t, float& prev_t,
                                               float& prev_dist, uint32_t& near, bool& stop_full) {
  uint32_t c = 0;
  const float lim = fminf(box_t, tmax);
  stop_full = false;
  for (; c < n; ++c) {
    if (t > lim) {
      stop_full = t > tmax;
      break;
    }
    float d = kMaxFloat;
    for (uint32_t e = 0; e < n_ev; ++e) {
      if (!((set >> e) & 1u)) continue;
      const ObjDev& o = objs[ev[e].obj];
      const float v = empty_value(o, grid_coord(ox, dx, t, o.m[12], o.half_gs[0]),
                                  grid_coord(oy, dy, t, o.m[13], o.half_gs[1]),
                                  grid_coord(oz, dz, t, o.m[14], o.half_gs[2]));
      if (v < d) d = v;
    }
    if (!CLEAN && !(d >= brk)) {  // no step: the full step redoes this sample
      stop_full = true;
      break;
    }
    prev_t = t;
    prev_dist = d;
    if (CLEAN) {
      t = __fadd_rn(t, d);
      continue;
    }
    t = __fadd_rn(t, fmax_(d, min_step));
    if (d < near_thr && ++near >= max_near) {
      stop_full = true;
      return c + 1;
    }
  }
  return c;
}

constexpr uint32_t kRefillRounds = 8;

// The outputs of a ray that ends at its first check, unhit, with no step
// taken (its tmax is below its starting t): what the epilogue writes for it.
__device__ __noinline__ void write_unmarched(const Segment& sg, uint32_t idx, uint32_t mode,
                                             const rkf_march_params& p) {
  if (mode == RKF_TRACE_SHADOW) {
    sg.t[idx] = 1.0f;  // clampf(1, 0, 1)
    if (sg.flags) sg.flags[idx] = 0;
    return;
  }
  const uint16_t flags = (0u >= p.hard_max_steps || 0u >= p.scene.max_steps) ? RKF_FLAG_STEPS_OUT : 0;
  sg.t[idx] = kMaxFloat;
  if (sg.flags) sg.flags[idx] = flags;
  if (mode == RKF_TRACE_ANY) return;
  if (sg.normal) {
    sg.normal[3 * static_cast<size_t>(idx)] = 0.0f;
    sg.normal[3 * static_cast<size_t>(idx) + 1] = 0.0f;
    sg.normal[3 * static_cast<size_t>(idx) + 2] = 0.0f;
  }
  if (sg.slot) sg.slot[idx] = RKF_EMPTY_SLOT;
  if (sg.material) sg.material[idx] = 0;
  if (sg.position) reinterpret_cast<float4*>(sg.position)[idx] = make_float4(0.f, 0.f, 0.f, kMaxFloat);
  if (sg.packed) sg.packed[idx] = 0u;
  if (sg.motion) reinterpret_cast<float4*>(sg.motion)[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
}

template <int PREC, int OBJ>
__global__ void __launch_bounds__(256, 4) k_march_persistent(const __grid_constant__ KParams kp) {
  constexpr bool MULTI_TILED = OBJ == OBJ_MULTI_EMPTY_TILED;
  constexpr bool MULTI_EMPTY = OBJ == OBJ_MULTI_EMPTY || MULTI_TILED;
  constexpr bool SINGLE = OBJ != OBJ_MULTI && !MULTI_EMPTY;
  constexpr bool EMPTY_PATH = OBJ == OBJ_SINGLE_EMPTY || OBJ == OBJ_SINGLE_EMPTY_TILED || MULTI_EMPTY;
  // tile bookkeeping of tiled launches
  constexpr bool TILES = OBJ != OBJ_SINGLE_EMPTY && OBJ != OBJ_MULTI_EMPTY;
  // warp-shared EMPTY runs in the launch's tail (shared_runs)
  constexpr bool SHARE = OBJ == OBJ_SINGLE_EMPTY;
  // the object table: the launch parameters hold up to kMaxObjectsFast
  // records; a larger scene (the plain multi-object variant only) reads the
  // device copy
  const ObjDev* sh_objs = (OBJ == OBJ_MULTI && kp.s.n_objs > kMaxObjectsFast) ? kp.s.objs : kp.objs;
  const SceneDev& s = kp.s;
  const rkf_march_params& p = kp.p;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nobj = s.n_objs;
  const float hit_thr = p.scene.hit_threshold;

  LaneCache lc;
  uint32_t state = ST_IDLE;
  uint32_t mode = RKF_TRACE_CLOSEST;
  // state a lane touches only when a ray starts, hits or ends lives in shared
  // memory, which keeps the march loop's register footprint small
  __shared__ ColdState cold_all[256];
  ColdState& cs = cold_all[threadIdx.x];
  float ox = 0, oy = 0, oz = 0, rdx = 0, rdy = 0, rdz = 0;
  float t = 0, prev_t = 0, prev_dist = kMaxFloat, tmax = 0;
  float box_t = -1.0f;  // empty-space path: positions up to here sample the EMPTY value
  float far_t = -1.0f;  // multi-object empty-space path: positions up to here lie outside every ball
  float far_recheck = -1.0f;  // multi-object empty-space path: no ball check before this t
  uint32_t near = 0, step = 0;
  bool exhausted = false;

  for (;;) {
    // ---- 1. refill idle lanes ------------------------------------------------
    // A ray that ends before its first sample (tmax below its starting t:
    // the secondary rays of pixels that missed) takes its outputs here and
    // its lane takes the next id at once, for up to kRefillRounds rounds, so
    // that such rays do not leave lanes idle through the march loop.
    for (uint32_t round = 0; round < kRefillRounds; ++round) {
      const bool idle = state == ST_IDLE;
      const uint32_t need = __ballot_sync(kFull, idle);
      bool again = false;  // this lane's id ended at once (or is off the view)
      if (need && !exhausted) {
        const uint32_t leader = __ffs(need) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(kp.counter, static_cast<unsigned long long>(__popc(need)));
        base = __shfl_sync(kFull, base, leader);
        if (base + __popc(need) >= kp.total) exhausted = true;
        if (idle) {
          const uint64_t k = base + __popc(need & ((1u << lane) - 1u));
          if (k < kp.total) {
            const uint64_t id = kp.id0 + k;
            cs.seg = find_segment(kp.segs, kp.nseg, id);
            const Segment& sg = kp.segs[cs.seg];
            const uint64_t local = id - sg.first;
            bool valid = true;
            if (sg.kind == 0) {  // view: tile-ordered pixel ids
              const uint32_t per = kp.tile_w * kp.tile_h;
              uint32_t tile = static_cast<uint32_t>(local / per);
              if (sg.tile_perm) tile = __ldg(sg.tile_perm + tile);  // heaviest-first order
              const uint32_t r = static_cast<uint32_t>(local % per);
              const uint32_t px = (tile % sg.tiles_x) * kp.tile_w + r % kp.tile_w;
              const uint32_t py = (tile / sg.tiles_x) * kp.tile_h + r / kp.tile_w;
              valid = px < sg.w && py < sg.h;
              if (valid) {
                cs.idx = py * sg.w + px;
                // ray generation (ray_march.wgsl:1046-1053)
                const float u = __fdiv_rn(__fadd_rn(__fadd_rn(static_cast<float>(px), 0.5f), sg.jitter[0]),
                                          static_cast<float>(sg.w));
                const float v = __fdiv_rn(__fadd_rn(__fadd_rn(static_cast<float>(py), 0.5f), sg.jitter[1]),
                                          static_cast<float>(sg.h));
                const float nx = __fsub_rn(__fmul_rn(u, 2.0f), 1.0f);
                const float ny = __fsub_rn(1.0f, __fmul_rn(v, 2.0f));
                const float vx = __fadd_rn(__fadd_rn(sg.fwd[0], __fmul_rn(sg.right[0], nx)), __fmul_rn(sg.up[0], ny));
                const float vy = __fadd_rn(__fadd_rn(sg.fwd[1], __fmul_rn(sg.right[1], nx)), __fmul_rn(sg.up[1], ny));
                const float vz = __fadd_rn(__fadd_rn(sg.fwd[2], __fmul_rn(sg.right[2], nx)), __fmul_rn(sg.up[2], ny));
                const float l = len3(vx, vy, vz);
                rdx = __fdiv_rn(vx, l);
                rdy = __fdiv_rn(vy, l);
                rdz = __fdiv_rn(vz, l);
                ox = sg.pos[0];
                oy = sg.pos[1];
                oz = sg.pos[2];
                tmax = p.scene.max_distance;
                mode = RKF_TRACE_CLOSEST;
                if (TILES) {
                  cs.tile_count = kNoTiles;
                  if (kp.tiled) {  // the pixel's tile (ray_march.wgsl:884-893)
                    const uint32_t tl = sg.tile_off + (py / 16) * ((sg.w + 15) / 16) + px / 16;
                    cs.tile_base = tl * kTileObjects;
                    cs.tile_count = __ldg(kp.td.tile_cnt + tl);
                  }
                  if (MULTI_TILED) {
                    uint32_t listed = 0;
                    for (uint32_t e = 0; e < kp.n_ev; ++e) {
                      bool in = cs.tile_count == kNoTiles;
                      for (uint32_t j = 0; !in && j < cs.tile_count; ++j)
                        in = __ldg(kp.td.tile_list + cs.tile_base + j) == kp.ev[e].obj;
                      if (in) listed |= 1u << e;
                    }
                    cs.vox_listed = listed;
                  }
                }
              }
            } else {
              if (TILES) cs.tile_count = kNoTiles;
              if (MULTI_TILED) cs.vox_listed = (1u << kp.n_ev) - 1u;
              cs.idx = static_cast<uint32_t>(local);
              const size_t i3 = 3 * static_cast<size_t>(cs.idx);
              ox = __ldg(sg.origins + i3);
              oy = __ldg(sg.origins + i3 + 1);
              oz = __ldg(sg.origins + i3 + 2);
              rdx = __ldg(sg.dirs + i3);
              rdy = __ldg(sg.dirs + i3 + 1);
              rdz = __ldg(sg.dirs + i3 + 2);
              tmax = __ldg(sg.tmax + cs.idx);
              mode = sg.mode;
            }
            if (valid) {
              near = 0;
              step = 0;
              box_t = -1.0f;
              if (MULTI_EMPTY) {
                far_t = far_recheck = -1.0f;
                if (!MULTI_TILED) cs.vox_listed = (1u << kp.n_ev) - 1u;
              }
              prev_dist = kMaxFloat;
              cs.hit = cs.bisected = cs.mat_ok = false;
              if (mode == RKF_TRACE_SHADOW) {
                t = 0.005f;  // SHADOW_EPSILON (shade_common.wgsl:274)
                cs.shadow = 1.0f;
                state = ST_SHADOW;
              } else {
                t = 0.0f;
                prev_t = 0.0f;
                prev_dist = kMaxFloat;
                // a tile with no objects is sky (ray_march.wgsl:895-897)
                state = (TILES && cs.tile_count == 0) ? ST_EPI : ST_MARCH;
              }
              if (state != ST_EPI && t > tmax) {
                // its first check ends it unhit with no step taken: the
                // epilogue's outputs for that (shadow 1; t max, normal 0,
                // EMPTY slot, material 0, STEPS_OUT only when the near-step
                // limit is 0, the miss position and motion)
                write_unmarched(sg, cs.idx, mode, p);
                state = ST_IDLE;
                again = true;
              }
            } else {
              again = true;
            }
          }
        }
      }
      if (!__any_sync(kFull, again)) break;
    }
    if (__all_sync(kFull, state == ST_IDLE)) {
      if (exhausted) break;
      continue;
    }
    // the march steps along the safe direction (ray_march.wgsl:784); cs.hit
    // positions use the raw direction (:1068)
    const float qdx = fabsf(rdx) < 1e-10f ? 1e-10f : rdx;
    const float qdy = fabsf(rdy) < 1e-10f ? 1e-10f : rdy;
    const float qdz = fabsf(rdz) < 1e-10f ? 1e-10f : rdz;

    // ---- 2. tight march loop -------------------------------------------------
#pragma unroll 1
    for (uint32_t k = 0; k < kp.interval; ++k) {
      bool full = true;  // take a full step (index lookups) this iteration
      // the launch's tail: no work is left to fetch and few lanes march, so
      // the warp takes their plain clean EMPTY runs together (after the
      // per-lane block below, where every lane meets again)
      const bool share = SHARE && exhausted && kp.tail_share && !kp.run_probe &&
                         static_cast<uint32_t>(__popc(__ballot_sync(kFull, state == ST_MARCH || state == ST_SHADOW))) <=
                             kp.tail_share;
      bool pend = false;
      float pend_lim = 0.0f, pend_dx = 0.0f, pend_dy = 0.0f, pend_dz = 0.0f;
      uint32_t pend_n = 0;
      // (a tiled step evaluates the ray's object list only: EMPTY runs need
      // the voxelized object in it)
      if (EMPTY_PATH && (state == ST_MARCH || state == ST_SHADOW) && (!MULTI_EMPTY || (cs.vox_listed & 0xFFu))) {
        // empty-space run: inside a cube of EMPTY blocks every sample is
        // empty_value(), so up to kp.budget steps run without the sampler.
        // Several objects: a probe picks the first voxelized object of the
        // path whose EMPTY cube holds the ray; its constants and balls apply.
        const bool sh = state == ST_SHADOW;
        const float dx = sh ? rdx : qdx, dy = sh ? rdy : qdy, dz = sh ? rdz : qdz;
        const uint32_t max_step = sh ? 256u : p.hard_max_steps;
        const uint32_t max_near = sh ? 32u : p.scene.max_steps;
        // a sample below brk goes to the full step, which decides it
        const float brk = sh ? 0.02f : fmaxf(hit_thr, 0.0f);
        const float near_thr = sh ? -1.0f : p.near_surface_threshold;
        const float min_step = sh ? 0.005f : p.min_step;
        // a ray that may be inside a ball takes full steps until it may have left
        const bool probe = t > box_t && prev_dist >= kp.probe_min && (!MULTI_EMPTY || t > far_recheck);
        if (MULTI_EMPTY && probe) {
          // the set of voxelized objects of the path (that the ray may take
          // runs on) whose EMPTY cubes hold the ray; the run lasts while it is
          // in all of them
          uint32_t set = 0;
          box_t = kMaxFloat;
          for (uint32_t e = 0; e < kp.n_ev; ++e) {
            if (!((cs.vox_listed >> e) & 1u)) continue;
            const float bt = probe_empty(sh_objs[kp.ev[e].obj], s.empty_dist, ox, oy, oz, dx, dy, dz, t);
            if (t <= bt) {
              set |= 1u << e;
              box_t = fminf(box_t, bt);
            }
          }
          if (!set) box_t = -1.0f;
          if (set && set != (cs.vox_listed >> 8)) {
            // other objects in the set: the balls that bound the run are others
            cs.vox_listed = (cs.vox_listed & 0xFFu) | (set << 8);
            far_t = far_recheck = -1.0f;
          }
        }
        const uint32_t set = MULTI_EMPTY ? (cs.vox_listed >> 8) : 1u;
        const bool one = (set & (set - 1u)) == 0u;  // one object's EMPTY value
        const EmptyVox& ev = kp.ev[MULTI_EMPTY ? (__ffs(set | 1u) - 1) : 0];
        const ObjDev& o0 = sh_objs[MULTI_EMPTY ? ev.obj : 0u];
        float e_lo = MULTI_EMPTY ? ev.empty_lo : kp.empty_lo;
        float e_hi = MULTI_EMPTY ? ev.empty_hi : kp.empty_hi;
        float e_lo_t = MULTI_EMPTY ? ev.empty_lo_t : kp.empty_lo_t;
        if (MULTI_EMPTY && !one) {
          for (uint32_t e = 0; e < kp.n_ev; ++e) {
            if (!((set >> e) & 1u)) continue;
            e_lo = fminf(e_lo, kp.ev[e].empty_lo);
            e_lo_t = fminf(e_lo_t, kp.ev[e].empty_lo_t);
            e_hi = fmaxf(e_hi, kp.ev[e].empty_hi);
          }
        }
        const uint32_t plain = MULTI_EMPTY ? (one ? ev.plain : 0u) : kp.plain_obj;
        const bool clean = e_lo >= brk && e_lo >= near_thr && e_lo >= min_step;
        if (probe) {
          if (!MULTI_EMPTY) box_t = probe_empty(o0, s.empty_dist, ox, oy, oz, dx, dy, dz, t);
          const float cube_t = box_t;
          if (MULTI_EMPTY) {
            // only positions outside the balls of every object not in the set
            // sample the set's EMPTY values.  far_t (the first entry into such
            // a ball ahead) stays valid until the ray passes it: balls ahead
            // stay ahead, balls behind stay behind.
            if (t <= box_t && t > far_t)
              far_t = far_limit(kp.ball, kp.n_ball, set, ox, oy, oz, dx, dy, dz, tmax, t, far_recheck);
            box_t = fminf(box_t, far_t);
          }
          if (t <= box_t && clean && one && kp.settle_links && step < max_step && near < max_near) {
            // Settle the ray if every sample it has left is the EMPTY value:
            // then no threshold acts on it, it misses, and its outputs do not
            // depend on its exact t.  t after k more steps lies in
            // [t + k*lo, t + k*hi] widened by one rounding (2^-24) per step;
            // 2^-22 per step (and 4 more) leaves room for this bound's own
            // rounding.  The last sample is the (max_step-step-1)th ahead; the
            // ray runs out of steps if even its largest t stays <= tmax, and
            // ends past tmax (with no step flag) if even its smallest t exceeds
            // tmax.  Either way, when EMPTY cubes cover every position up to
            // that bound (or tmax), the outcome is settled.
            const float k = static_cast<float>(max_step - step - 1);
            const float grow = (k + 4.0f) * 2.384185791015625e-7f;
            const float t_hi = (t + k * e_hi) * (1.0f + grow);
            const float t_lo = (t + k * e_lo_t) * (1.0f - grow);
            const bool out_of_steps = t_hi <= tmax;
            if (out_of_steps || t_lo > tmax) {
              const float need = out_of_steps ? t_hi : tmax;
              if (!MULTI_EMPTY) {
                box_t = extend_cover(o0, s.empty_dist, ox, oy, oz, dx, dy, dz, box_t, need, kp.settle_links);
              } else if (far_t >= need) {
                box_t = fminf(extend_cover(o0, s.empty_dist, ox, oy, oz, dx, dy, dz, cube_t, need, kp.settle_links),
                              far_t);
              }
              if (box_t >= need) {
                if (sh) cs.shadow = clampf(cs.shadow, 0.0f, 1.0f);
                else if (out_of_steps) step = max_step;
                cs.hit = false;
                state = ST_EPI;
              }
            }
          }
        }
        if (state != ST_EPI && t <= box_t) {
          const uint32_t n = step < max_step ? min(kp.budget, max_step - step) : 0u;
          uint32_t c = 0;
          bool stop_full = true;
          if (near < max_near && MULTI_EMPTY && !one) {
            // several objects: the least of their EMPTY values, to the end of
            // the nearest cube
            c = clean ? empty_run_set<true>(sh_objs, kp.ev, set, kp.n_ev, ox, oy, oz, dx, dy, dz, tmax, n, brk,
                                            near_thr, min_step, max_near, t, box_t, prev_t, prev_dist, near, stop_full)
                      : empty_run_set<false>(sh_objs, kp.ev, set, kp.n_ev, ox, oy, oz, dx, dy, dz, tmax, n, brk,
                                             near_thr, min_step, max_near, t, box_t, prev_t, prev_dist, near,
                                             stop_full);
          } else if (near < max_near) {
#define RKF_RUN(P, CL, IN)                                                                                   \
  empty_run<P, CL, IN, MULTI_EMPTY>(o0, s.empty_dist, ox, oy, oz, dx, dy, dz, tmax, n, brk, near_thr, min_step, \
                                    max_near, far_t, t, box_t, prev_t, prev_dist, near, stop_full)
            if (plain && clean && share) {
              // the whole run at once (the budget only paces warps that share
              // nothing); taken with the warp below
              pend = true;
              pend_lim = fminf(box_t, tmax);
              pend_n = step < max_step ? max_step - step : 0u;
              pend_dx = dx;
              pend_dy = dy;
              pend_dz = dz;
            } else if (plain && clean)
              c = kp.run_probe ? empty_run_x2<true, MULTI_EMPTY>(o0, s.empty_dist, ox, oy, oz, dx, dy, dz, tmax, n,
                                                                 far_t, t, box_t, prev_t, prev_dist, stop_full)
                               : empty_run_x2<false, MULTI_EMPTY>(o0, s.empty_dist, ox, oy, oz, dx, dy, dz, tmax, n,
                                                                  far_t, t, box_t, prev_t, prev_dist, stop_full);
            else if (plain)
              c = kp.run_probe ? RKF_RUN(true, false, true) : RKF_RUN(true, false, false);
            else
              c = kp.run_probe ? RKF_RUN(false, false, true) : RKF_RUN(false, false, false);
#undef RKF_RUN
          }
          step += c;
          // a run that used its whole budget, or reached the end of its cube
          // between probes, continues next iteration unless a limit ends the
          // ray; any other stop needs the full step's decision
          full = stop_full || step >= max_step || t > tmax || near >= max_near;
        }
      }
      if (share) {  // warp-uniform: every lane is here
        uint32_t c = 0;
        bool stop_full = false;
        shared_runs(sh_objs[0], pend, ox, oy, oz, pend_dx, pend_dy, pend_dz, pend_lim, tmax, pend_n, t, prev_t,
                    prev_dist, c, stop_full);
        if (pend) {
          const bool sh = state == ST_SHADOW;
          step += c;
          full = stop_full || step >= (sh ? 256u : p.hard_max_steps) || t > tmax ||
                 near >= (sh ? 32u : p.scene.max_steps);
        }
      }
      if (!full) {
      } else if (state == ST_MARCH) {
        if (step >= p.hard_max_steps || t > tmax || near >= p.scene.max_steps) {
          cs.hit = false;
          state = ST_EPI;
        } else {
          float best_un;
          uint32_t best_i;
          const float wx = __fadd_rn(ox, __fmul_rn(qdx, t)), wy = __fadd_rn(oy, __fmul_rn(qdy, t)),
                      wz = __fadd_rn(oz, __fmul_rn(qdz, t));
          float best;
          bool skipped = false;
          if (TILES && kp.tiled && cs.tile_count != kNoTiles) {
            // ray_march_tiled (:899-938): a coarse empty-space skip, else the
            // tile's objects only
            const Segment& sg = kp.segs[cs.seg];
            const float cd = coarse_sample(kp.td, sg.coarse_ocr, __fsub_rn(wx, sg.pos[0]), __fsub_rn(wy, sg.pos[1]),
                                           __fsub_rn(wz, sg.pos[2]));
            best = kMaxFloat;
            best_un = kMaxFloat;
            best_i = 0;
            if (cd > kCoarseNear) {
              prev_dist = kMaxFloat;
              t = __fadd_rn(t, cd);
              step++;
              skipped = true;
            } else {
              for (uint32_t j = 0; j < cs.tile_count; ++j) {
                const uint32_t oi = __ldg(kp.td.tile_list + cs.tile_base + j);
                float du;
                const float d = eval_obj<PREC>(s, sh_objs[oi], wx, wy, wz, &du, lc);
                if (d < best) {
                  best = d;
                  best_un = du;
                  best_i = oi;
                }
              }
            }
          } else if ((!EMPTY_PATH || MULTI_EMPTY) && kp.use_bvh) {
            best = eval_bvh<PREC>(s, sh_objs, kp.bvh, kp.bvh_next, nobj, wx, wy, wz, best_un, best_i, lc);
          } else {
            best = eval_min<PREC, SINGLE>(s, sh_objs, 0, nobj, wx, wy, wz, best_un, best_i, lc);
          }
          if (skipped) {
          } else if (best < 0.0f && prev_dist > hit_thr) {  // overstep (ray_march.wgsl:816)
            cs.hit_obj = best_i;
            cs.hit = true;
            if (mode == RKF_TRACE_ANY) {
              state = ST_EPI;
            } else {
              cs.lo = prev_t;
              cs.hi = t;
              cs.mat_t = t;
              cs.mat_ok = best_un < sh_objs[best_i].vs16;
              cs.sub = 0;
              cs.bisected = true;
              state = ST_BISECT;
            }
          } else if (best < hit_thr) {  // :842
            cs.hit_obj = best_i;
            cs.hit = true;
            if (mode == RKF_TRACE_ANY) {
              state = ST_EPI;
            } else {
              // a direct cs.hit: enter the finish phase with the bisection done
              cs.mat_t = t;
              cs.mat_ok = best_un < sh_objs[best_i].vs16;
              cs.sub = p.bisect_steps;
              state = ST_BISECT;
            }
          } else {
            if (best < p.near_surface_threshold) near++;
            prev_t = t;
            prev_dist = best;
            t = __fadd_rn(t, fmax_(best, p.min_step));
            step++;
          }
        }
      } else if (state == ST_SHADOW) {
        // soft_shadow (shade_common_shading.wgsl:9-33)
        if (step >= 256u || near >= 32u || t > tmax) {
          cs.shadow = clampf(cs.shadow, 0.0f, 1.0f);
          cs.hit = false;
          state = ST_EPI;
        } else {
          float best_un;
          uint32_t best_i;
          const float best = eval_min<PREC, SINGLE>(s, sh_objs, 0, nobj, __fadd_rn(ox, __fmul_rn(rdx, t)),
                                                    __fadd_rn(oy, __fmul_rn(rdy, t)),
                                                    __fadd_rn(oz, __fmul_rn(rdz, t)), best_un, best_i, lc);
          prev_dist = best;
          if (best < 0.005f) {
            cs.shadow = 0.0f;
            cs.hit = true;
            state = ST_EPI;
          } else {
            if (best < 0.02f) {
              cs.shadow = fmin_(cs.shadow, __fdiv_rn(__fmul_rn(16.0f, best), t));
              near++;
            }
            t = __fadd_rn(t, fmax_(best, 0.005f));
            step++;
          }
        }
      }
      // leave to finish and refill once refill_idle lanes are done (or,
      // with no work left to fetch, once none is marching)
      const uint32_t active = __popc(__ballot_sync(kFull, state == ST_MARCH || state == ST_SHADOW));
      if (active <= (exhausted ? 0u : kp.refill_active)) break;
    }

    // ---- 3. finish: bisection and central differences -------------------------
    float g0 = 0, g1 = 0, g2 = 0, lpx = 0, lpy = 0, lpz = 0, eps = 0;
    while (__any_sync(kFull, state == ST_BISECT || state == ST_NORMAL)) {
      if (state == ST_BISECT && cs.sub >= p.bisect_steps) {
        // bisection done (or a direct cs.hit): t = (cs.lo+cs.hi)/2, set up the normal
        if (cs.bisected) t = __fmul_rn(__fadd_rn(cs.lo, cs.hi), 0.5f);
        const ObjDev& o = sh_objs[cs.hit_obj];
        const float hx = __fadd_rn(ox, __fmul_rn(rdx, t));
        const float hy = __fadd_rn(oy, __fmul_rn(rdy, t));
        const float hz = __fadd_rn(oz, __fmul_rn(rdz, t));
        if (o.sdf_type == RKF_SDF_VOXELIZED) {
          to_local_fast(o, hx, hy, hz, lpx, lpy, lpz);
          eps = __fmul_rn(o.vs, 2.0f);
        } else {
          lpx = hx;
          lpy = hy;
          lpz = hz;
          eps = __fmul_rn(hit_thr, 10.0f);
        }
        cs.sub = 0;
        state = ST_NORMAL;
      }
      if (state == ST_BISECT) {
        const float mid = __fmul_rn(__fadd_rn(cs.lo, cs.hi), 0.5f);
        float du;
        const float d = eval_obj<PREC>(s, sh_objs[cs.hit_obj], __fadd_rn(ox, __fmul_rn(qdx, mid)),
                                       __fadd_rn(oy, __fmul_rn(qdy, mid)), __fadd_rn(oz, __fmul_rn(qdz, mid)),
                                       &du, lc);
        if (d < 0.0f) {
          cs.hi = mid;
        } else {
          cs.lo = mid;
          cs.mat_t = mid;
          cs.mat_ok = du < sh_objs[cs.hit_obj].vs16;
        }
        ++cs.sub;
      } else if (state == ST_NORMAL) {
        const ObjDev& o = sh_objs[cs.hit_obj];
        const uint32_t ax = cs.sub >> 1;
        float qx = lpx, qy = lpy, qz = lpz;
        if (ax == 0) qx = (cs.sub & 1) ? __fsub_rn(lpx, eps) : __fadd_rn(lpx, eps);
        if (ax == 1) qy = (cs.sub & 1) ? __fsub_rn(lpy, eps) : __fadd_rn(lpy, eps);
        if (ax == 2) qz = (cs.sub & 1) ? __fsub_rn(lpz, eps) : __fadd_rn(lpz, eps);
        float d;
        if (o.sdf_type == RKF_SDF_VOXELIZED) {
          d = sample_vox<PREC>(s, o, qx, qy, qz, true, lc);
        } else {
          float du;
          d = eval_obj<PREC>(s, o, qx, qy, qz, &du, lc);
        }
        if (cs.sub & 1) {
          const float g = __fsub_rn(cs.gpos, d);
          if (ax == 0) g0 = g;
          else if (ax == 1) g1 = g;
          else g2 = g;
        } else {
          cs.gpos = d;
        }
        if (++cs.sub == 6) state = ST_EPI;
      }
    }

    // ---- 4. epilogue: outputs of finished rays -------------------------------
    if (state == ST_EPI) {
      const Segment& sg = kp.segs[cs.seg];
      if (mode == RKF_TRACE_SHADOW) {
        sg.t[cs.idx] = cs.shadow;
        if (sg.flags) sg.flags[cs.idx] = cs.hit ? RKF_FLAG_HIT : 0;
      } else if (mode == RKF_TRACE_ANY) {
        sg.t[cs.idx] = cs.hit ? t : kMaxFloat;
        if (sg.flags)
          sg.flags[cs.idx] = cs.hit ? RKF_FLAG_HIT
                              : ((step >= p.hard_max_steps || near >= p.scene.max_steps) ? RKF_FLAG_STEPS_OUT : 0);
      } else {
        uint16_t flags = 0;
        float nx = 0, ny = 0, nz = 0;
        uint32_t slot = RKF_EMPTY_SLOT, mat = 0, sec = 0, blend = 0;
        float hx = 0, hy = 0, hz = 0, sdf_hit = 0;
        if (cs.hit) {
          flags |= RKF_FLAG_HIT;
          if (cs.bisected) flags |= RKF_FLAG_BISECTED;
          const ObjDev& o = sh_objs[cs.hit_obj];
          hx = __fadd_rn(ox, __fmul_rn(rdx, t));
          hy = __fadd_rn(oy, __fmul_rn(rdy, t));
          hz = __fadd_rn(oz, __fmul_rn(rdz, t));
          if (o.sdf_type == RKF_SDF_VOXELIZED) {
            // world_grad = transpose(inverse_world) * (g, 0)  (:1014)
            const float wx = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[0], g0), __fmul_rn(o.m[1], g1)),
                                                 __fmul_rn(o.m[2], g2)), __fmul_rn(o.m[3], 0.0f));
            const float wy = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[4], g0), __fmul_rn(o.m[5], g1)),
                                                 __fmul_rn(o.m[6], g2)), __fmul_rn(o.m[7], 0.0f));
            const float wz = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[8], g0), __fmul_rn(o.m[9], g1)),
                                                 __fmul_rn(o.m[10], g2)), __fmul_rn(o.m[11], 0.0f));
            const float l = len3(wx, wy, wz);
            if (l < 1e-10f) {
              ny = 1.0f;
            } else {
              nx = __fdiv_rn(wx, l); ny = __fdiv_rn(wy, l); nz = __fdiv_rn(wz, l);
            }
            uint32_t vi = 0;
            slot = nearest_slot(s, o, lpx, lpy, lpz, vi, lc);
            if (slot < RKF_INTERIOR_SLOT) {
              const size_t v = static_cast<size_t>(slot) * 512 + vi;
              sec = (__ldg(s.mat + v) >> 6) & 0x3Fu;
              blend = __ldg(s.blend + v);
            }
            if (sg.motion) sdf_hit = sample_vox<PREC>(s, o, lpx, lpy, lpz, false, lc);
          } else {
            const float l = len3(g0, g1, g2);
            nx = __fdiv_rn(g0, l); ny = __fdiv_rn(g1, l); nz = __fdiv_rn(g2, l);
          }
          if (cs.mat_ok || o.sdf_type == RKF_SDF_ANALYTICAL)
            mat = material_at(s, o, __fadd_rn(ox, __fmul_rn(qdx, cs.mat_t)), __fadd_rn(oy, __fmul_rn(qdy, cs.mat_t)),
                              __fadd_rn(oz, __fmul_rn(qdz, cs.mat_t)), lc);
        } else if (step >= p.hard_max_steps || near >= p.scene.max_steps) {
          flags |= RKF_FLAG_STEPS_OUT;
        }
        sg.t[cs.idx] = cs.hit ? t : kMaxFloat;
        if (sg.normal) {
          sg.normal[3 * static_cast<size_t>(cs.idx)] = nx;
          sg.normal[3 * static_cast<size_t>(cs.idx) + 1] = ny;
          sg.normal[3 * static_cast<size_t>(cs.idx) + 2] = nz;
        }
        if (sg.slot) sg.slot[cs.idx] = slot;
        if (sg.material) sg.material[cs.idx] = static_cast<uint16_t>(mat);
        if (sg.flags) sg.flags[cs.idx] = flags;
        if (sg.position) {
          const float4 pv = cs.hit ? make_float4(hx, hy, hz, t) : make_float4(0.f, 0.f, 0.f, kMaxFloat);
          reinterpret_cast<float4*>(sg.position)[cs.idx] = pv;
        }
        if (sg.packed)
          sg.packed[cs.idx] = cs.hit ? ((mat & 0x3Fu) | (sec << 6) | (blend << 12) | (sh_objs[cs.hit_obj].object_id << 24))
                               : 0u;
        if (sg.motion) {
          float4 mv = make_float4(0.f, 0.f, 0.f, 0.f);
          if (cs.hit) {
            const float* m = sg.prev_vp;  // ray_march.wgsl:1094-1105
            const float cx = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], hx), __fmul_rn(m[4], hy)),
                                                 __fmul_rn(m[8], hz)), __fmul_rn(m[12], 1.0f));
            const float cy = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[1], hx), __fmul_rn(m[5], hy)),
                                                 __fmul_rn(m[9], hz)), __fmul_rn(m[13], 1.0f));
            const float cw = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[3], hx), __fmul_rn(m[7], hy)),
                                                 __fmul_rn(m[11], hz)), __fmul_rn(m[15], 1.0f));
            float mox = 0.f, moy = 0.f;
            if (cw > 0.0f) {
              const float ndx = __fdiv_rn(cx, cw), ndy = __fdiv_rn(cy, cw);
              const float pu = __fadd_rn(__fmul_rn(ndx, 0.5f), 0.5f);
              const float pv = __fsub_rn(0.5f, __fmul_rn(ndy, 0.5f));
              const uint32_t px = cs.idx % sg.w, py = cs.idx / sg.w;
              const float cu = __fdiv_rn(__fadd_rn(static_cast<float>(px), 0.5f), static_cast<float>(sg.w));
              const float cv = __fdiv_rn(__fadd_rn(static_cast<float>(py), 0.5f), static_cast<float>(sg.h));
              mox = __fsub_rn(cu, pu);
              moy = __fsub_rn(cv, pv);
            }
            mv = make_float4(mox, moy, 1.0f, sdf_hit);
          }
          reinterpret_cast<float4*>(sg.motion)[cs.idx] = mv;
        }
      }
      state = ST_IDLE;
    }
  }
}

// One thread per point: SdfQueryable::evaluate / gradient over the pool.
template <int PREC>
__global__ void k_query_points(SceneDev s, const float* __restrict__ pts, uint32_t n, float* dist,
                               float* grad, uint16_t* material) {
  extern __shared__ ObjDev sh_objs[];
  for (uint32_t i = threadIdx.x; i < s.n_objs; i += blockDim.x) sh_objs[i] = s.objs[i];
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  LaneCache lc;
  const float px = pts[3 * static_cast<size_t>(i)], py = pts[3 * static_cast<size_t>(i) + 1],
              pz = pts[3 * static_cast<size_t>(i) + 2];
  float best_un = kMaxFloat;
  uint32_t bi = 0;
  const float best = eval_min<PREC, false>(s, sh_objs, 0, s.n_objs, px, py, pz, best_un, bi, lc);
  if (dist) dist[i] = best;
  if (material) {
    uint32_t m = 0;
    if (s.n_objs) {
      const ObjDev& o = sh_objs[bi];
      if (o.sdf_type == RKF_SDF_ANALYTICAL || best_un < o.vs16) m = material_at(s, o, px, py, pz, lc);
    }
    material[i] = static_cast<uint16_t>(m);
  }
  if (grad) {
    float nx = 0.0f, ny = 1.0f, nz = 0.0f;
    if (s.n_objs) {
      const ObjDev& o = sh_objs[bi];
      if (o.sdf_type == RKF_SDF_VOXELIZED) {
        float lx, ly, lz;
        to_local_fast(o, px, py, pz, lx, ly, lz);
        const float e = __fmul_rn(o.vs, 2.0f);
        const float g0 = __fsub_rn(sample_vox<PREC>(s, o, __fadd_rn(lx, e), ly, lz, true, lc),
                                   sample_vox<PREC>(s, o, __fsub_rn(lx, e), ly, lz, true, lc));
        const float g1 = __fsub_rn(sample_vox<PREC>(s, o, lx, __fadd_rn(ly, e), lz, true, lc),
                                   sample_vox<PREC>(s, o, lx, __fsub_rn(ly, e), lz, true, lc));
        const float g2 = __fsub_rn(sample_vox<PREC>(s, o, lx, ly, __fadd_rn(lz, e), true, lc),
                                   sample_vox<PREC>(s, o, lx, ly, __fsub_rn(lz, e), true, lc));
        const float wx = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[0], g0), __fmul_rn(o.m[1], g1)),
                                             __fmul_rn(o.m[2], g2)), __fmul_rn(o.m[3], 0.0f));
        const float wy = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[4], g0), __fmul_rn(o.m[5], g1)),
                                             __fmul_rn(o.m[6], g2)), __fmul_rn(o.m[7], 0.0f));
        const float wz = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(o.m[8], g0), __fmul_rn(o.m[9], g1)),
                                             __fmul_rn(o.m[10], g2)), __fmul_rn(o.m[11], 0.0f));
        const float l = len3(wx, wy, wz);
        if (l >= 1e-10f) {
          nx = __fdiv_rn(wx, l); ny = __fdiv_rn(wy, l); nz = __fdiv_rn(wz, l);
        }
      } else {
        // analytic: central differences with eps = 10 * hit_threshold(0.001)
        const float e = __fmul_rn(0.001f, 10.0f);
        float du;
        const float a = __fsub_rn(eval_obj<PREC>(s, o, __fadd_rn(px, e), py, pz, &du, lc),
                                  eval_obj<PREC>(s, o, __fsub_rn(px, e), py, pz, &du, lc));
        const float b = __fsub_rn(eval_obj<PREC>(s, o, px, __fadd_rn(py, e), pz, &du, lc),
                                  eval_obj<PREC>(s, o, px, __fsub_rn(py, e), pz, &du, lc));
        const float c = __fsub_rn(eval_obj<PREC>(s, o, px, py, __fadd_rn(pz, e), &du, lc),
                                  eval_obj<PREC>(s, o, px, py, __fsub_rn(pz, e), &du, lc));
        const float l = len3(a, b, c);
        nx = __fdiv_rn(a, l); ny = __fdiv_rn(b, l); nz = __fdiv_rn(c, l);
      }
    }
    grad[3 * static_cast<size_t>(i)] = nx;
    grad[3 * static_cast<size_t>(i) + 1] = ny;
    grad[3 * static_cast<size_t>(i) + 2] = nz;
  }
}

// One thread per point: sdf_ao (shade_common_shading.wgsl:37-47), four taps
// along the normal at AO_STEP_SIZE * i (0.12 m) through sample_sdf, which for
// points inside the objects' bounds is the minimum of evaluate_object over the
// objects (shade_common.wgsl:521-572); ao = clamp(1 - AO_STRENGTH * sum, 0, 1)
// with AO_STRENGTH 0.7 and tap weights 1, 1/2, 1/4, 1/8.
template <int PREC>
__global__ void k_sdf_ao(SceneDev s, const float* __restrict__ pos, const float* __restrict__ nrm, uint32_t n,
                         float* __restrict__ ao) {
  extern __shared__ ObjDev sh_objs[];
  for (uint32_t i = threadIdx.x; i < s.n_objs; i += blockDim.x) sh_objs[i] = s.objs[i];
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  LaneCache lc;
  const size_t i3 = 3 * static_cast<size_t>(i);
  const float px = pos[i3], py = pos[i3 + 1], pz = pos[i3 + 2];
  const float nx = nrm[i3], ny = nrm[i3 + 1], nz = nrm[i3 + 2];
  float acc = 0.0f, scale = 1.0f;
#pragma unroll 1
  for (uint32_t k = 1; k <= 4; ++k) {
    const float dist = __fmul_rn(0.12f, static_cast<float>(k));
    float du;
    uint32_t bi;
    const float d = eval_min<PREC, false>(s, sh_objs, 0, s.n_objs, __fadd_rn(px, __fmul_rn(nx, dist)),
                                         __fadd_rn(py, __fmul_rn(ny, dist)), __fadd_rn(pz, __fmul_rn(nz, dist)), du,
                                         bi, lc);
    acc = __fadd_rn(acc, __fmul_rn(scale, __fsub_rn(dist, d)));
    scale = __fmul_rn(scale, 0.5f);
  }
  ao[i] = clampf(__fsub_rn(1.0f, __fmul_rn(0.7f, acc)), 0.0f, 1.0f);
}

template <int PREC>
const void* persistent_fn(int obj) {
  if (obj == OBJ_MULTI_EMPTY) return reinterpret_cast<const void*>(&k_march_persistent<PREC, OBJ_MULTI_EMPTY>);
  if (obj == OBJ_MULTI_EMPTY_TILED)
    return reinterpret_cast<const void*>(&k_march_persistent<PREC, OBJ_MULTI_EMPTY_TILED>);
  if (obj == OBJ_SINGLE_EMPTY) return reinterpret_cast<const void*>(&k_march_persistent<PREC, OBJ_SINGLE_EMPTY>);
  if (obj == OBJ_SINGLE_EMPTY_TILED)
    return reinterpret_cast<const void*>(&k_march_persistent<PREC, OBJ_SINGLE_EMPTY_TILED>);
  if (obj == OBJ_SINGLE) return reinterpret_cast<const void*>(&k_march_persistent<PREC, OBJ_SINGLE>);
  return reinterpret_cast<const void*>(&k_march_persistent<PREC, OBJ_MULTI>);
}

}  // namespace detail

namespace {
// A voxelized object the empty-space path can march: translation-only
// inverse_world, verified exact quotient, fewer than 2^20 voxels per axis.
bool empty_object(const Ctx* c, const ObjDev& o) {
  return o.sdf_type == RKF_SDF_VOXELIZED && o.translate_only && o.div_ok && c->empty_dist.p != nullptr &&
         o.tv[0] < (1 << 20) && o.tv[1] < (1 << 20) && o.tv[2] < (1 << 20);
}

// Upper bound of every EMPTY value of a voxelized object: mix(c, c, t) three
// times stays within 12 roundings of c = brick extent * min_scale (relative
// 2^-24 each), far inside 2^-16.
float empty_hi_of(const ObjDev& o) { return o.be * o.min_scale * (1.0f + 1.52587890625e-5f); }

// Radius of the ball around the local origin that holds an analytic
// primitive (analytic_sdf, ray_march.wgsl:182-264): its value is at least
// |l| - R everywhere.  -1 for a plane (unbounded) or non-finite parameters.
double prim_radius(const ObjDev& o) {
  const double a0 = std::fabs(static_cast<double>(o.params[0])), a1 = std::fabs(static_cast<double>(o.params[1])),
               a2 = std::fabs(static_cast<double>(o.params[2]));
  double r = -1.0;
  switch (o.prim_type) {
    case RKF_PRIM_SPHERE: r = a0; break;
    case RKF_PRIM_BOX: r = std::sqrt(a0 * a0 + a1 * a1 + a2 * a2); break;
    case RKF_PRIM_CAPSULE: r = a0 + a1; break;
    case RKF_PRIM_TORUS: r = a0 + a1; break;
    case RKF_PRIM_CYLINDER: r = std::sqrt(a0 * a0 + a1 * a1); break;
    default: return -1.0;
  }
  return std::isfinite(r) ? r : -1.0;
}

double up_float(double v) {  // a float >= v
  const float f = static_cast<float>(v);
  return static_cast<double>(f) >= v ? f : std::nextafter(f, std::numeric_limits<float>::infinity());
}

// The FarBall of an analytic object for EMPTY values up to empty_hi (the
// bound FarBall describes, with every FP32 rounding of evaluate_object held
// to 2^-16 of the magnitudes involved, a wide margin over the few 2^-24
// roundings each step makes).  false when the object has no usable ball.
bool far_ball(const ObjDev& o, float empty_hi, detail::FarBall* out) {
  // A voxelized object's sampler returns the distance to its clamped grid
  // box (a box inside |l| <= |half_gs|) wherever that distance exceeds two
  // brick extents (ray_march.wgsl:371-376), so beyond the ball of radius
  // |half_gs| + max(2 * brick extent, EMPTY value / scale) its value is at
  // least that distance times its scale, above every EMPTY value.  With a
  // translation-only transform the grid box is axis-aligned in world space,
  // and the same holds outside the box widened by that distance (a position
  // beyond it along one axis is that far from the box): the tighter bound.
  const bool vox = o.sdf_type == RKF_SDF_VOXELIZED;
  std::memset(out, 0, sizeof(*out));
  out->path = ~0u;
  if (vox && o.translate_only) {
    const double s = o.min_scale;
    if (!(s > 0.0) || !std::isfinite(s)) return false;
    const double e16 = 0x1p-16, e20 = 0x1p-20;
    const double need = std::max(static_cast<double>(empty_hi) * (1.0 + e16) / s,
                                 static_cast<double>(o.be2) * (1.0 + e16));
    double tn = 0.0, hn = 0.0;
    for (int i = 0; i < 3; ++i) {
      out->c[i] = -o.m[12 + i];  // local = world + m: the local origin (grid centre) in world space
      out->h[i] = static_cast<float>(up_float(static_cast<double>(o.half_gs[i]) * (1.0 + e16)));
      tn += static_cast<double>(o.m[12 + i]) * o.m[12 + i];
      hn += static_cast<double>(o.half_gs[i]) * o.half_gs[i];
    }
    out->a = static_cast<float>(up_float(need + e16 * (std::sqrt(tn) + std::sqrt(hn)) + e20 * std::sqrt(tn)));
    out->b = static_cast<float>(up_float(3.0 * e16 + e20));
    out->box = 1;
    return std::isfinite(out->a) && std::isfinite(out->h[0]) && std::isfinite(out->h[1]) &&
           std::isfinite(out->h[2]) && std::isfinite(out->c[0]) && std::isfinite(out->c[1]) &&
           std::isfinite(out->c[2]);
  }
  const double R = vox ? std::sqrt(static_cast<double>(o.half_gs[0]) * o.half_gs[0] +
                                   static_cast<double>(o.half_gs[1]) * o.half_gs[1] +
                                   static_cast<double>(o.half_gs[2]) * o.half_gs[2])
                       : prim_radius(o);
  const double s = o.min_scale;
  if (R < 0.0 || !std::isfinite(R) || !(s > 0.0) || !std::isfinite(s)) return false;
  double A[3][3], t[3];  // l_i = sum_k A[i][k] p_k + t_i (to_local)
  for (int i = 0; i < 3; ++i) {
    for (int k = 0; k < 3; ++k) A[i][k] = o.m[4 * k + i];
    t[i] = o.m[12 + i];
  }
  const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                     A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                     A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  if (!std::isfinite(det) || det == 0.0) return false;
  double inv[3][3];
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) {
      const int i1 = (k + 1) % 3, i2 = (k + 2) % 3, k1 = (i + 1) % 3, k2 = (i + 2) % 3;
      inv[i][k] = (A[i1][k1] * A[i2][k2] - A[i1][k2] * A[i2][k1]) / det;
    }
  double nf = 0.0, nif = 0.0, tn = 0.0, c[3], cn = 0.0;
  for (int i = 0; i < 3; ++i) {
    c[i] = -(inv[i][0] * t[0] + inv[i][1] * t[1] + inv[i][2] * t[2]);
    cn += c[i] * c[i];
    tn += t[i] * t[i];
    for (int k = 0; k < 3; ++k) {
      nf += A[i][k] * A[i][k];
      nif += inv[i][k] * inv[i][k];
    }
  }
  const double N = std::sqrt(nf), sigma = 1.0 / std::sqrt(nif);  // |A x| >= sigma |x|
  const double e16 = 0x1p-16, e20 = 0x1p-20;
  if (!(sigma > 0.0) || !(N / sigma <= 1024.0)) return false;
  double need = static_cast<double>(empty_hi) * (1.0 + e16) / s;  // local distance beyond R
  if (vox) need = std::max(need, static_cast<double>(o.be2) * (1.0 + e16));
  const double a = (R * (1.0 + e16) + e16 * std::sqrt(tn) + need) / sigma + e20 * std::sqrt(cn);
  const double b = e16 * N / sigma + e20;
  for (int i = 0; i < 3; ++i) out->c[i] = static_cast<float>(c[i]);
  out->a = static_cast<float>(up_float(a));
  out->b = static_cast<float>(up_float(b));
  return std::isfinite(out->c[0]) && std::isfinite(out->c[1]) && std::isfinite(out->c[2]) && std::isfinite(out->a) &&
         std::isfinite(out->b);
}

// The half-space of an analytic plane for EMPTY values up to empty_hi.  The
// plane's value (ray_march.wgsl:206-208, 257-258) is s * n.l with n the
// normalised normal and l = A w + t the local position: exactly G.w + H with
// G = s A^T n, H = s n.t.  The computed value differs from that by at most
// 2^-16 s (|A|_F |w| + |t|) -- about twenty roundings of 2^-24 each over the
// local transform, the normalisation and the dot product -- and the sample
// positions from the line by 2^-16 |w|, so wherever G.w + H exceeds
// empty_hi (1 + 2^-16) + 2^-16 (s |t| + (s |A|_F + |G|) |w|) the plane's value
// exceeds every EMPTY value; |w| <= P along the ray.  Refused for a zero or
// non-finite normal or transform.
bool far_plane(const ObjDev& o, float empty_hi, detail::FarBall* out) {
  std::memset(out, 0, sizeof(*out));
  out->path = ~0u;
  const double s = o.min_scale;
  const double nl = std::sqrt(static_cast<double>(o.params[0]) * o.params[0] +
                              static_cast<double>(o.params[1]) * o.params[1] +
                              static_cast<double>(o.params[2]) * o.params[2]);
  if (!(nl > 0.0) || !std::isfinite(nl) || !(s > 0.0) || !std::isfinite(s)) return false;
  double n[3], G[3] = {0.0, 0.0, 0.0}, H = 0.0, fa = 0.0, tn = 0.0, gn = 0.0;
  for (int i = 0; i < 3; ++i) n[i] = static_cast<double>(o.params[i]) / nl;
  for (int i = 0; i < 3; ++i) {  // l_i = sum_k m[4k + i] w_k + m[12 + i]
    for (int k = 0; k < 3; ++k) {
      const double aik = o.m[4 * k + i];
      G[k] += s * n[i] * aik;
      fa += aik * aik;
    }
    H += s * n[i] * o.m[12 + i];
    tn += static_cast<double>(o.m[12 + i]) * o.m[12 + i];
  }
  for (int k = 0; k < 3; ++k) gn += G[k] * G[k];
  const double e16 = 0x1p-16, e20 = 0x1p-20;
  const double a = static_cast<double>(empty_hi) * (1.0 + e16) + e16 * s * std::sqrt(tn) + e20;
  const double b = e16 * (s * std::sqrt(fa) + std::sqrt(gn)) + e20;
  for (int k = 0; k < 3; ++k) out->c[k] = static_cast<float>(G[k]);
  out->h[0] = static_cast<float>(H);
  out->a = static_cast<float>(up_float(a));
  out->b = static_cast<float>(up_float(b));
  out->box = 2;
  return std::isfinite(out->c[0]) && std::isfinite(out->c[1]) && std::isfinite(out->c[2]) &&
         std::isfinite(out->h[0]) && std::isfinite(out->a) && std::isfinite(out->b);
}

// A scene of several objects the multi-object empty-space path can march:
// one to kMaxEmptyVox voxelized objects that qualify for the empty-space path
// (the first ones by index), each of which takes EMPTY runs on its own field,
// and every object -- analytic, voxelized (on the path or not) or of no type
// -- either bounded by a ball outside which its value exceeds every EMPTY
// value of the path, or (no type, unknown primitives) never below them.
// Fills ev and the balls (with each ball's path index) when given.
bool multi_empty_scene(const Ctx* c, detail::EmptyVox* ev, uint32_t* n_ev, detail::FarBall* balls,
                       uint32_t* n_ball) {
  const uint32_t n = c->obj_count();
  if (n < 2 || n > kMaxObjectsFast) return false;
  uint32_t q[detail::kMaxEmptyVox];
  uint32_t path_of[kMaxObjectsFast];
  uint32_t nq = 0;
  for (uint32_t i = 0; i < n; ++i) {
    path_of[i] = ~0u;
    if (nq < detail::kMaxEmptyVox && empty_object(c, c->objdev_host[i])) {
      path_of[i] = nq;
      q[nq++] = i;
    }
  }
  if (nq == 0) return false;
  float hi = 0.0f;  // the largest EMPTY value of the path
  for (uint32_t j = 0; j < nq; ++j) hi = std::max(hi, empty_hi_of(c->objdev_host[q[j]]));
  uint32_t nb = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const ObjDev& o = c->objdev_host[i];
    if (o.sdf_type == RKF_SDF_NONE) continue;  // no type: kMaxFloat
    if (o.sdf_type == RKF_SDF_ANALYTICAL && o.prim_type > RKF_PRIM_PLANE) {
      // an unknown primitive: kMaxFloat * min_scale
      if (static_cast<double>(kMaxFloat) * o.min_scale * (1.0 - 0x1p-20) >= hi) continue;
      return false;
    }
    detail::FarBall b;
    const bool plane = o.sdf_type == RKF_SDF_ANALYTICAL && o.prim_type == RKF_PRIM_PLANE;
    if (!(plane ? far_plane(o, hi, &b) : far_ball(o, hi, &b))) return false;
    b.path = path_of[i];
    if (balls) balls[nb] = b;
    ++nb;
  }
  for (uint32_t j = 0; ev && j < nq; ++j) {
    const ObjDev& a = c->objdev_host[q[j]];
    detail::EmptyVox e;
    std::memset(&e, 0, sizeof(e));
    e.obj = q[j];
    e.probe_min = 0.99f * a.be * a.min_scale;
    // mix(c, c, t) three times stays within 12 roundings of c (relative
    // 2^-24 each); 0.999 leaves a wide margin, 2^-16 a tight one
    e.empty_lo = 0.999f * a.be * a.min_scale;
    e.empty_lo_t = a.be * a.min_scale * (1.0f - 1.52587890625e-5f);
    e.empty_hi = empty_hi_of(a);
    e.plain = (a.m[12] == 0.0f && a.m[13] == 0.0f && a.m[14] == 0.0f && a.min_scale == 1.0f) ? 1u : 0u;
    ev[j] = e;
  }
  if (n_ev) *n_ev = nq;
  if (n_ball) *n_ball = nb;
  return true;
}

// The BVH walk (eval_bvh) evaluates object vi at every position inside its
// grid (the clamp range every EMPTY cube lies in): some leaf naming vi has
// every node on its path from the root containing that box, and every
// internal node on it descends (the shader's stack had room for its
// children: bit 31 of its walk link).  The walk skips a node only when its
// box distance exceeds the best value so far; inside such nodes that
// distance is 0, and along EMPTY runs outside every ball no value is
// negative, so the leaf is reached and the walk's minimum is the brute one.
bool bvh_reaches(const Ctx* c, uint32_t vi) {
  const std::vector<rkf_bvh_node>& nd = c->bvh_host;
  const std::vector<uint32_t>& link = c->bvh_next_host;
  if (nd.empty() || link.size() != nd.size()) return false;
  const ObjDev& o = c->objdev_host[vi];
  float lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    const float base = -o.half_gs[a] - o.m[12 + a];
    lo[a] = 0.5f * o.vs + base;
    hi[a] = (static_cast<float>(o.tv[a] - 1) + 0.5f) * o.vs + base;
  }
  std::vector<uint32_t> stack{0u};
  while (!stack.empty()) {
    const uint32_t i = stack.back();
    stack.pop_back();
    if (i >= nd.size()) continue;
    const rkf_bvh_node& b = nd[i];
    bool holds = true;
    for (int a = 0; a < 3; ++a) holds = holds && b.aabb_min[a] <= lo[a] && b.aabb_max[a] >= hi[a];
    if (!holds) continue;
    if (b.left == RKF_BVH_INVALID) {
      if (b.right_or_object == vi) return true;
    } else if (link[i] >> 31) {
      stack.push_back(b.left);
      stack.push_back(b.right_or_object);
    }
  }
  return false;
}

// The objects of the multi-object empty-space path of a launch, with their
// balls, into kp.ev: those the BVH walk reaches everywhere in their grids
// when the launch walks the tree.  false when none remains.
bool fill_multi_empty(const Ctx* c, bool walk, detail::KParams& kp) {
  detail::EmptyVox ev[detail::kMaxEmptyVox];
  uint32_t n = 0;
  if (!multi_empty_scene(c, ev, &n, kp.ball, &kp.n_ball)) return false;
  // an object the walk may not reach leaves the path (its ball still bounds
  // the others' runs)
  uint32_t remap[detail::kMaxEmptyVox];
  kp.n_ev = 0;
  kp.probe_min = kMaxFloat;
  for (uint32_t j = 0; j < n; ++j) {
    remap[j] = ~0u;
    if (walk && !bvh_reaches(c, ev[j].obj)) continue;
    remap[j] = kp.n_ev;
    kp.ev[kp.n_ev] = ev[j];
    kp.probe_min = std::min(kp.probe_min, ev[j].probe_min);
    ++kp.n_ev;
  }
  for (uint32_t b = 0; b < kp.n_ball; ++b)
    if (kp.ball[b].path < n) kp.ball[b].path = remap[kp.ball[b].path];
  return kp.n_ev > 0;
}

// Which kernel variant a launch over this context's objects uses.
int object_set(const Ctx* c) {
  if (c->obj_count() != 1)
    return multi_empty_scene(c, nullptr, nullptr, nullptr, nullptr) ? detail::OBJ_MULTI_EMPTY : detail::OBJ_MULTI;
  return empty_object(c, c->objdev_host[0]) ? detail::OBJ_SINGLE_EMPTY : detail::OBJ_SINGLE;
}
}  // namespace

bool empty_order_source(const Ctx* c, const rkf_march_params* p, const rkf_batch_tuning& tu, ObjDev* o) {
  if (tu.no_empty_path || p->strategy == RKF_STRATEGY_TILED || c->obj_count() == 0 ||
      c->obj_count() > kMaxObjectsFast)
    return false;
  const bool use_bvh = p->strategy == RKF_STRATEGY_BVH;
  const int objs = object_set(c);
  if (objs == detail::OBJ_SINGLE_EMPTY) {
    if (use_bvh && !c->bvh_one_leaf0) return false;
    *o = c->objdev_host[0];
    return true;
  }
  if (objs == detail::OBJ_MULTI_EMPTY) {
    // the estimate walks the field of the path's first object
    detail::KParams kp;
    if (!fill_multi_empty(c, use_bvh, kp)) return false;
    *o = c->objdev_host[kp.ev[0].obj];
    return true;
  }
  return false;
}

float order_reach(const ObjDev& o, const rkf_march_params* p) {
  return std::min(p->scene.max_distance, static_cast<float>(p->hard_max_steps) * o.be * o.min_scale);
}

rkf_status launch_persistent(Ctx* c, const std::vector<Segment>& segs_host, uint64_t total,
                             const rkf_march_params* p, const rkf_batch_tuning& tu,
                             cudaStream_t st, DevBuf* seg_buf, unsigned long long* counter, uint64_t id0,
                             bool segs_resident) {
  if (c->obj_count() == 0) return fail(RKF_INVALID_ARG, "march: the scene has no objects");
  const bool tiled = p->strategy == RKF_STRATEGY_TILED;
  const bool use_bvh = p->strategy == RKF_STRATEGY_BVH;
  if (use_bvh && c->bvh_n == 0) return fail(RKF_INVALID_ARG, "march: the BVH strategy needs an imported BVH");
  std::vector<Segment> tiled_segs;
  TiledDev td;
  std::memset(&td, 0, sizeof(td));
  int objs = object_set(c);
  if (tu.no_empty_path) {  // the same outputs through the full sampler only
    if (objs == detail::OBJ_SINGLE_EMPTY) objs = detail::OBJ_SINGLE;
    if (objs == detail::OBJ_MULTI_EMPTY) objs = detail::OBJ_MULTI;
  }
  if (tiled) {
    tiled_segs = segs_host;
    rkf_status s2 = prepare_tiled(c, tiled_segs, st, &td);
    if (s2 != RKF_OK) return s2;
    // the tiled empty-space field of every object of the path
    std::vector<uint32_t> path{0u};
    if (objs == detail::OBJ_MULTI_EMPTY) {
      detail::EmptyVox ev[detail::kMaxEmptyVox];
      uint32_t n = 0;
      multi_empty_scene(c, ev, &n, nullptr, nullptr);
      path.clear();
      for (uint32_t j = 0; j < n; ++j) path.push_back(ev[j].obj);
    }
    if ((objs == detail::OBJ_SINGLE_EMPTY || objs == detail::OBJ_MULTI_EMPTY) &&
        (s2 = prepare_tiled_empty(c, st, path)) != RKF_OK)
      return s2;
  }
  // heaviest-first order of the views' tiles (a whole launch only: a band of
  // a view is ordered by its caller, which plans all bands at once)
  ObjDev order_obj;
  OrderTable order_tbl;
  bool ordered = false;
  std::vector<Segment> ordered_segs;
  if (tu.order_tiles && id0 == 0 && !segs_resident && !tiled && empty_order_source(c, p, tu, &order_obj)) {
    ordered_segs = segs_host;
    rkf_status s2 = tile_order_prepare(c, ordered_segs, tu.tile_w, tu.tile_h, nullptr, 0, &order_tbl, &ordered);
    if (s2 != RKF_OK) return s2;
  }
  const std::vector<Segment>& segs_dev = tiled ? tiled_segs : (ordered ? ordered_segs : segs_host);
  const size_t sb = segs_dev.size() * sizeof(Segment);
  if (!segs_resident || seg_buf->bytes < sb) {
    if (seg_buf->bytes < sb) {
      rkf_status s2 = seg_buf->alloc(sb);
      if (s2 != RKF_OK) return s2;
    }
    // a pageable source: the call returns once the stream has taken the data
    RKF_CUDA_TRY(cudaMemcpyAsync(seg_buf->p, segs_dev.data(), sb, cudaMemcpyHostToDevice, st));
  }
  if (ordered) {
    rkf_status s2 = tile_order_enqueue(c, order_tbl, seg_buf->as<Segment>(), order_obj, c->empty_dist.as<uint8_t>(),
                                       order_reach(order_obj, p), order_obj.be * order_obj.min_scale, st);
    if (s2 != RKF_OK) return s2;
  }
  RKF_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
  detail::KParams kp;
  std::memset(&kp, 0, sizeof(kp));
  // beyond kMaxObjectsFast objects the kernel reads the device table
  std::memcpy(kp.objs, c->objdev_host.data(), sizeof(ObjDev) * std::min<uint32_t>(c->obj_count(), kMaxObjectsFast));
  kp.s = c->scene_dev();
  kp.segs = seg_buf->as<Segment>();
  kp.nseg = static_cast<uint32_t>(segs_host.size());
  kp.tile_w = tu.tile_w ? tu.tile_w : 8;
  kp.tile_h = tu.tile_h ? tu.tile_h : 4;
  kp.interval = tu.compact_interval ? tu.compact_interval : 64;
  kp.total = total;
  kp.id0 = id0;
  kp.counter = counter;
  kp.p = *p;
  kp.p.scene.num_objects = c->obj_count();
  // A BVH of one leaf naming the only, voxelized, object makes every step
  // evaluate exactly what the brute step evaluates (the one box test passes
  // for every finite distance, and where it would not, the object's own
  // distance is not finite either), so that walk is the brute march.
  const bool walk = use_bvh && !(objs == detail::OBJ_SINGLE_EMPTY && c->bvh_one_leaf0);
  int obj = objs;
  if (objs == detail::OBJ_SINGLE_EMPTY && walk) obj = detail::OBJ_SINGLE;
  if (objs == detail::OBJ_SINGLE_EMPTY && tiled) {
    obj = detail::OBJ_SINGLE_EMPTY_TILED;
    kp.s.empty_dist = c->tiled_empty_dist.as<uint8_t>();
  }
  // the multi-object empty-space path marches the brute and tiled
  // strategies, and the BVH strategy for the objects whose grids the tree's
  // walk reaches everywhere
  if (objs == detail::OBJ_MULTI_EMPTY && !fill_multi_empty(c, walk, kp)) obj = detail::OBJ_MULTI;
  if (obj == detail::OBJ_MULTI_EMPTY && tiled) {
    obj = detail::OBJ_MULTI_EMPTY_TILED;
    kp.s.empty_dist = c->tiled_empty_dist.as<uint8_t>();
  }
  const bool multi_empty = obj == detail::OBJ_MULTI_EMPTY || obj == detail::OBJ_MULTI_EMPTY_TILED;
  const bool empty = obj == detail::OBJ_SINGLE_EMPTY || obj == detail::OBJ_SINGLE_EMPTY_TILED || multi_empty;
  kp.td = td;
  kp.tiled = tiled ? 1u : 0u;
  kp.bvh = walk ? c->bvh.as<rkf_bvh_node>() : nullptr;
  kp.bvh_next = walk ? c->bvh_next.as<uint32_t>() : nullptr;
  kp.use_bvh = walk ? 1u : 0u;
  const ObjDev& e0 = kp.objs[0];  // the object of the single-object empty-space path
  if (!multi_empty) kp.probe_min = empty ? 0.99f * e0.be * e0.min_scale : kMaxFloat;
  kp.budget = tu.step_budget ? tu.step_budget : 32;
  kp.refill_active = 32u - std::min<uint32_t>(tu.refill_idle ? tu.refill_idle : 32u, 32u);
  kp.run_probe = tu.probe_in_run ? 1u : 0u;
  kp.tail_share = std::min<uint32_t>(tu.tail_share, 32u);
  // mix(c, c, t) three times stays within 12 roundings of c (relative 2^-24
  // each); 0.999 leaves a wide margin
  kp.empty_lo = empty ? 0.999f * e0.be * e0.min_scale : 0.0f;
  // twelve roundings of 2^-24 stay far inside 2^-16
  kp.empty_lo_t = e0.be * e0.min_scale * (1.0f - 1.52587890625e-5f);
  kp.empty_hi = empty_hi_of(e0);
  kp.settle_links = empty ? 48u : 0u;
  kp.plain_obj = (e0.m[12] == 0.0f && e0.m[13] == 0.0f && e0.m[14] == 0.0f && e0.min_scale == 1.0f) ? 1u : 0u;
  const void* fn = nullptr;
  switch (c->cfg.precision) {
    case RKF_PRECISION_F32:
      fn = detail::persistent_fn<RKF_PRECISION_F32>(obj);
      break;
    case RKF_PRECISION_U8:
      fn = detail::persistent_fn<RKF_PRECISION_U8>(obj);
      break;
    default:
      fn = detail::persistent_fn<RKF_PRECISION_F16>(obj);
  }
  c->last_variant = obj;
  const uint32_t threads = tu.threads_per_block ? tu.threads_per_block : 256;
  if (threads > 256 || threads % 32)
    return fail(RKF_INVALID_ARG, "march: threads_per_block must be a multiple of 32 <= 256");
  const size_t smem = 0;
  uint32_t bps = tu.blocks_per_sm;
  if (bps == 0) {
    int occ = 0;
    RKF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem));
    bps = occ > 0 ? static_cast<uint32_t>(occ) : 1;
  }
  // never launch more lanes than work items
  uint64_t blocks = static_cast<uint64_t>(c->sm_count) * bps;
  const uint64_t need_blocks = (total + threads - 1) / threads;
  if (blocks > need_blocks) blocks = need_blocks ? need_blocks : 1;
  void* args[] = {&kp};
  rkf_status se = c->march_event(st, false);
  if (se != RKF_OK) return se;
  RKF_CUDA_TRY(cudaLaunchKernel(fn, dim3(static_cast<unsigned>(blocks)), dim3(threads), args, smem, st));
  c->counted();
  return c->march_event(st, true);
}

rkf_status check_persistent_scratch(const Ctx* c, const rkf_march_params* p, const rkf_batch_tuning& tu) {
  if (p->strategy != RKF_STRATEGY_BRUTE)
    return fail(RKF_UNSUPPORTED, "march: this launch path runs the brute strategy only");
  if (c->obj_count() == 0) return fail(RKF_INVALID_ARG, "march: the scene has no objects");
  const uint32_t threads = tu.threads_per_block ? tu.threads_per_block : 256;
  if (threads > 256 || threads % 32)
    return fail(RKF_INVALID_ARG, "march: threads_per_block must be a multiple of 32 <= 256");
  return RKF_OK;
}

rkf_status launch_persistent_scratch(Ctx* c, const Segment* segs_host, uint32_t nseg, uint64_t total,
                                     const rkf_march_params* p, const rkf_batch_tuning& tu,
                                     cudaStream_t st, Segment* dev_segs, unsigned long long* dev_counter,
                                     bool segs_uploaded, bool multi_empty) {
  // every refusal comes before anything is enqueued on the stream
  const rkf_status chk = check_persistent_scratch(c, p, tu);
  if (chk != RKF_OK) return chk;
  if (!segs_uploaded)
    RKF_CUDA_TRY(cudaMemcpyAsync(dev_segs, segs_host, sizeof(Segment) * nseg, cudaMemcpyHostToDevice, st));
  RKF_CUDA_TRY(cudaMemsetAsync(dev_counter, 0, sizeof(unsigned long long), st));
  detail::KParams kp;
  std::memset(&kp, 0, sizeof(kp));
  // beyond kMaxObjectsFast objects the kernel reads the device table
  std::memcpy(kp.objs, c->objdev_host.data(), sizeof(ObjDev) * std::min<uint32_t>(c->obj_count(), kMaxObjectsFast));
  kp.s = c->scene_dev();
  kp.segs = dev_segs;
  kp.nseg = nseg;
  kp.tile_w = tu.tile_w ? tu.tile_w : 8;
  kp.tile_h = tu.tile_h ? tu.tile_h : 4;
  kp.interval = tu.compact_interval ? tu.compact_interval : 64;
  kp.total = total;
  kp.counter = dev_counter;
  kp.p = *p;
  kp.p.scene.num_objects = c->obj_count();
  // without multi_empty, several objects march the plain multi-object kernel
  int obj = object_set(c);
  if (obj == detail::OBJ_MULTI_EMPTY && (!multi_empty || !fill_multi_empty(c, false, kp))) obj = detail::OBJ_MULTI;
  const bool memp = obj == detail::OBJ_MULTI_EMPTY;
  const ObjDev& e0 = kp.objs[0];  // the object of the single-object empty-space path
  const bool empty = obj == detail::OBJ_SINGLE_EMPTY || memp;
  if (!memp) kp.probe_min = empty ? 0.99f * e0.be * e0.min_scale : kMaxFloat;
  kp.budget = tu.step_budget ? tu.step_budget : 32;
  kp.refill_active = 32u - std::min<uint32_t>(tu.refill_idle ? tu.refill_idle : 32u, 32u);
  kp.run_probe = tu.probe_in_run ? 1u : 0u;
  kp.tail_share = std::min<uint32_t>(tu.tail_share, 32u);
  // mix(c, c, t) three times stays within 12 roundings of c (relative 2^-24
  // each); 0.999 leaves a wide margin
  kp.empty_lo = empty ? 0.999f * e0.be * e0.min_scale : 0.0f;
  // twelve roundings of 2^-24 stay far inside 2^-16
  kp.empty_lo_t = e0.be * e0.min_scale * (1.0f - 1.52587890625e-5f);
  kp.empty_hi = e0.be * e0.min_scale * (1.0f + 1.52587890625e-5f);
  kp.settle_links = empty ? 48u : 0u;
  kp.plain_obj = (e0.m[12] == 0.0f && e0.m[13] == 0.0f && e0.m[14] == 0.0f && e0.min_scale == 1.0f) ? 1u : 0u;
  const void* fn = nullptr;
  switch (c->cfg.precision) {
    case RKF_PRECISION_F32:
      fn = detail::persistent_fn<RKF_PRECISION_F32>(obj);
      break;
    case RKF_PRECISION_U8:
      fn = detail::persistent_fn<RKF_PRECISION_U8>(obj);
      break;
    default:
      fn = detail::persistent_fn<RKF_PRECISION_F16>(obj);
  }
  c->last_variant = obj;
  const uint32_t threads = tu.threads_per_block ? tu.threads_per_block : 256;  // checked above
  uint32_t bps = tu.blocks_per_sm;
  if (bps == 0) {
    int occ = 0;
    RKF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, 0));
    bps = occ > 0 ? static_cast<uint32_t>(occ) : 1;
  }
  uint64_t blocks = static_cast<uint64_t>(c->sm_count) * bps;
  const uint64_t need_blocks = (total + threads - 1) / threads;
  if (blocks > need_blocks) blocks = need_blocks ? need_blocks : 1;
  void* args[] = {&kp};
  rkf_status se = c->march_event(st, false);
  if (se != RKF_OK) return se;
  RKF_CUDA_TRY(cudaLaunchKernel(fn, dim3(static_cast<unsigned>(blocks)), dim3(threads), args, 0, st));
  c->counted();
  return c->march_event(st, true);
}

rkf_status launch_query(Ctx* c, const float* pts, uint32_t n, float* d, float* g, uint16_t* m,
                        cudaStream_t st) {
  if (n == 0) return RKF_OK;
  const size_t smem = sizeof(ObjDev) * std::max<uint32_t>(1, c->obj_count());
  const unsigned blocks = (n + 127) / 128;
  switch (c->cfg.precision) {
    case RKF_PRECISION_F32:
      detail::k_query_points<RKF_PRECISION_F32><<<blocks, 128, smem, st>>>(c->scene_dev(), pts, n, d, g, m);
      break;
    case RKF_PRECISION_U8:
      detail::k_query_points<RKF_PRECISION_U8><<<blocks, 128, smem, st>>>(c->scene_dev(), pts, n, d, g, m);
      break;
    default:
      detail::k_query_points<RKF_PRECISION_F16><<<blocks, 128, smem, st>>>(c->scene_dev(), pts, n, d, g, m);
  }
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  return RKF_OK;
}

rkf_status launch_ao(Ctx* c, const float* pos, const float* nrm, uint32_t n, float* ao, cudaStream_t st) {
  if (n == 0) return RKF_OK;
  const size_t smem = sizeof(ObjDev) * std::max<uint32_t>(1, c->obj_count());
  const unsigned blocks = (n + 127) / 128;
  switch (c->cfg.precision) {
    case RKF_PRECISION_F32:
      detail::k_sdf_ao<RKF_PRECISION_F32><<<blocks, 128, smem, st>>>(c->scene_dev(), pos, nrm, n, ao);
      break;
    case RKF_PRECISION_U8:
      detail::k_sdf_ao<RKF_PRECISION_U8><<<blocks, 128, smem, st>>>(c->scene_dev(), pos, nrm, n, ao);
      break;
    default:
      detail::k_sdf_ao<RKF_PRECISION_F16><<<blocks, 128, smem, st>>>(c->scene_dev(), pos, nrm, n, ao);
  }
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  return RKF_OK;
}

Segment view_segment(const rkf_camera* cam, uint32_t w, uint32_t h, uint32_t tile_w, uint32_t tile_h,
                     const rkf_gbuffer& out) {
  Segment sg;
  std::memset(&sg, 0, sizeof(sg));
  sg.kind = 0;
  sg.mode = RKF_TRACE_CLOSEST;
  sg.w = w;
  sg.h = h;
  if (!tile_w) tile_w = 8;
  if (!tile_h) tile_h = 4;
  sg.tiles_x = (w + tile_w - 1) / tile_w;
  const uint32_t tiles_y = (h + tile_h - 1) / tile_h;
  sg.n_ids = static_cast<uint64_t>(sg.tiles_x) * tiles_y * tile_w * tile_h;
  for (int a = 0; a < 3; ++a) {
    sg.pos[a] = cam->position[a];
    sg.fwd[a] = cam->forward[a];
    sg.right[a] = cam->right[a];
    sg.up[a] = cam->up[a];
  }
  sg.jitter[0] = cam->jitter[0];
  sg.jitter[1] = cam->jitter[1];
  std::memcpy(sg.prev_vp, cam->prev_vp, sizeof(sg.prev_vp));
  sg.t = out.t;
  sg.normal = out.normal;
  sg.slot = out.slot;
  sg.material = out.material;
  sg.flags = out.flags;
  sg.position = out.position;
  sg.packed = out.packed_material;
  sg.motion = out.motion;
  return sg;
}

Segment ray_segment(const float* o, const float* d, const float* tmax, uint32_t n, uint32_t mode,
                    const rkf_hits& out) {
  Segment sg;
  std::memset(&sg, 0, sizeof(sg));
  sg.kind = 1;
  sg.mode = mode;
  sg.n_ids = n;
  sg.origins = o;
  sg.dirs = d;
  sg.tmax = tmax;
  sg.t = out.t;
  sg.normal = out.normal;
  sg.slot = out.slot;
  sg.material = out.material;
  sg.flags = out.flags;
  return sg;
}

}  // namespace rkf

extern "C" int rkf_testing_last_variant(rkf_ctx* ctx) {
  return ctx ? reinterpret_cast<rkf::Ctx*>(ctx)->last_variant : -1;
}

extern "C" int rkf_testing_far_plane(const rkf_gpu_object* obj, float empty_hi, float out[6]) {
  if (!obj || !out) return 0;
  const rkf::ObjDev od = rkf::make_objdev(*obj, 0, 0);
  if (od.sdf_type != RKF_SDF_ANALYTICAL || od.prim_type != RKF_PRIM_PLANE) return 0;
  rkf::detail::FarBall b;
  if (!rkf::far_plane(od, empty_hi, &b)) return 0;
  out[0] = b.c[0];
  out[1] = b.c[1];
  out[2] = b.c[2];
  out[3] = b.h[0];
  out[4] = b.a;
  out[5] = b.b;
  return 1;
}

extern "C" int rkf_testing_far_ball(const rkf_gpu_object* obj, float empty_hi, float out[5]) {
  if (!obj || !out) return 0;
  const rkf::ObjDev od = rkf::make_objdev(*obj, 0, 0);
  rkf::detail::FarBall b;
  if (!rkf::far_ball(od, empty_hi, &b)) return 0;
  out[0] = b.c[0];
  out[1] = b.c[1];
  out[2] = b.c[2];
  out[3] = b.a;
  out[4] = b.b;
  return 1;
}
