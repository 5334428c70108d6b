// bvh.cu — the BVH of the BVH march strategy: import (GpuScene::upload_bvh,
// gpu_scene.rs:186) and a host-side build with the reference's surface-area
// heuristic (Bvh::build, crates/rkf-core/src/bvh.rs:66-260).
//
// The shader walks the tree once per step with a 32-entry stack
// (ray_march.wgsl:676-721): pop a node, skip it if its box is farther than
// the best distance so far, else evaluate its object (a leaf) or push its left
// then its right child while fewer than 31 entries are on the stack.  On a
// tree whose children follow their parent and whose nodes have one parent
// each -- the only kind the import admits -- that walk visits every node at
// most once, and the stack's content when a node is popped depends on the
// tree alone: the left children of the ancestors whose right subtree holds
// the node.  So the walk is the fixed order "node, right subtree, left
// subtree", with a node's children dropped when 31 or more entries lie
// below it, and the march replays it without a stack: per node the import
// stores the node that follows its subtree in that order (bvh_next, bits
// 0-30; kBvhEnd after the last) and whether the walk descends into it
// (bit 31).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"

namespace rkf {

namespace {

constexpr uint32_t kMaxBvhNodes = 65536;
constexpr uint32_t kBvhEnd = 0x7FFFFFFFu;

struct Box {
  float lo[3], hi[3];
};

// Aabb::expand_aabb (aabb.rs:118-123): componentwise f32::min / f32::max
Box merge(const Box& a, const Box& b) {
  Box r;
  for (int k = 0; k < 3; ++k) {
    r.lo[k] = std::fmin(a.lo[k], b.lo[k]);
    r.hi[k] = std::fmax(a.hi[k], b.hi[k]);
  }
  return r;
}

// Aabb::surface_area (aabb.rs:151-154): 2 (xy + yz + zx) of the side lengths
float area(const Box& b) {
  const float x = b.hi[0] - b.lo[0], y = b.hi[1] - b.lo[1], z = b.hi[2] - b.lo[2];
  const float xy = x * y, yz = y * z, zx = z * x;
  return 2.0f * ((xy + yz) + zx);
}

// Aabb::center (aabb.rs:48-50) along one axis
float centroid(const Box& b, int axis) { return (b.lo[axis] + b.hi[axis]) * 0.5f; }

struct Builder {
  const rkf_bvh_item* items;
  std::vector<Box> box;            // per item
  std::vector<rkf_bvh_node> nodes;

  Box enclosing(const uint32_t* idx, size_t n) const {
    Box e = box[idx[0]];
    for (size_t k = 1; k < n; ++k) e = merge(e, box[idx[k]]);
    return e;
  }

  uint32_t reserve(const Box& e) {
    rkf_bvh_node nd;
    for (int k = 0; k < 3; ++k) {
      nd.aabb_min[k] = e.lo[k];
      nd.aabb_max[k] = e.hi[k];
    }
    nd.left = RKF_BVH_INVALID;
    nd.right_or_object = RKF_BVH_INVALID;
    nodes.push_back(nd);
    return static_cast<uint32_t>(nodes.size() - 1);
  }

  // sort_by on the centroid: a stable sort, so equal keys keep the order of
  // the previous sort
  void sort_axis(uint32_t* idx, size_t n, int axis) const {
    std::stable_sort(idx, idx + n,
                     [&](uint32_t a, uint32_t b) { return centroid(box[a], axis) < centroid(box[b], axis); });
  }

  // build_recursive (bvh.rs:153-250): the node is reserved before its
  // children, so children always follow their parent
  uint32_t build(uint32_t* idx, size_t n) {
    const Box e = enclosing(idx, n);
    if (n == 1) {
      const uint32_t ni = reserve(e);
      nodes[ni].right_or_object = items[idx[0]].object_index;  // GpuBvhNode::from_cpu: a leaf's object
      return ni;
    }
    if (n == 2) {
      const uint32_t ni = reserve(e);
      const uint32_t l = build(idx, 1);
      const uint32_t r = build(idx + 1, 1);
      nodes[ni].left = l;
      nodes[ni].right_or_object = r;
      return ni;
    }
    const float esa = std::fmax(area(e), 1e-10f);
    float best_cost = 3.402823466e+38f;
    int best_axis = 0;
    size_t best_split = n / 2;
    for (int axis = 0; axis < 3; ++axis) {
      sort_axis(idx, n, axis);
      for (size_t split = 1; split < n; ++split) {
        const Box l = enclosing(idx, split), r = enclosing(idx + split, n - split);
        // TRAVERSAL_COST + LEAF_COST * (SA_l * n_l + SA_r * n_r) / SA  (both costs 1)
        const float weighted = area(l) * static_cast<float>(split) + area(r) * static_cast<float>(n - split);
        const float cost = 1.0f + (1.0f * weighted) / esa;
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = axis;
          best_split = split;
        }
      }
    }
    sort_axis(idx, n, best_axis);
    const uint32_t ni = reserve(e);
    const uint32_t l = build(idx, best_split);
    const uint32_t r = build(idx + best_split, n - best_split);
    nodes[ni].left = l;
    nodes[ni].right_or_object = r;
    return ni;
  }
};

// One tree, children after their parent, every node but the root named once.
// The walk's links (see the file comment); nodes must be a valid tree.
std::vector<uint32_t> walk_links(const rkf_bvh_node* nodes, uint32_t n) {
  std::vector<uint32_t> next(n, kBvhEnd), below(n, 0);
  for (uint32_t i = 0; i < n; ++i) {  // parents come before their children
    if (nodes[i].left == RKF_BVH_INVALID) continue;
    const uint32_t l = nodes[i].left, r = nodes[i].right_or_object;
    if (below[i] < 31) next[i] |= 0x80000000u;
    next[r] = l;                      // the right subtree is followed by the left child
    below[r] = below[i] + 1;          // ... which waits on the stack meanwhile
    next[l] = next[i] & ~0x80000000u;  // the left subtree by what follows the parent's
    below[l] = below[i];
  }
  return next;
}

bool valid_tree(const rkf_bvh_node* nodes, uint32_t n) {
  std::vector<uint8_t> named(n, 0);
  for (uint32_t i = 0; i < n; ++i) {
    if (nodes[i].left == RKF_BVH_INVALID) continue;
    const uint32_t l = nodes[i].left, r = nodes[i].right_or_object;
    if (l <= i || r <= i || l >= n || r >= n || l == r) return false;
    if (named[l]++ || named[r]++) return false;
  }
  for (uint32_t i = 1; i < n; ++i)
    if (!named[i]) return false;
  return true;
}

}  // namespace

}  // namespace rkf

using namespace rkf;

extern "C" {

rkf_status rkf_bvh_import(rkf_ctx* ctx, const rkf_bvh_node* nodes, uint32_t n) {
  if (!ctx || (!nodes && n)) return fail(RKF_INVALID_ARG, "rkf_bvh_import: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_bvh_import: the context is serving");
  if (n > kMaxBvhNodes) return fail(RKF_INVALID_ARG, "rkf_bvh_import: more than 65536 nodes");
  if (!valid_tree(nodes, n))
    return fail(RKF_INVALID_ARG,
                "rkf_bvh_import: the nodes are not one tree with each child after its parent");
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  if (n == 0) {
    c->bvh.release();
    c->bvh_next.release();
    c->bvh_n = 0;
    c->bvh_one_leaf0 = false;
    c->bvh_host.clear();
    c->bvh_next_host.clear();
    return RKF_OK;
  }
  const std::vector<uint32_t> next = walk_links(nodes, n);
  DevBuf nb, nn;
  rkf_status st = nb.alloc(static_cast<size_t>(n) * sizeof(rkf_bvh_node));
  if (st == RKF_OK) st = nn.alloc(static_cast<size_t>(n) * 4);
  if (st != RKF_OK) return st;
  RKF_CUDA_TRY(cudaMemcpy(nb.p, nodes, static_cast<size_t>(n) * sizeof(rkf_bvh_node), cudaMemcpyHostToDevice));
  RKF_CUDA_TRY(cudaMemcpy(nn.p, next.data(), static_cast<size_t>(n) * 4, cudaMemcpyHostToDevice));
  std::swap(c->bvh.p, nb.p);
  std::swap(c->bvh.bytes, nb.bytes);
  std::swap(c->bvh_next.p, nn.p);
  std::swap(c->bvh_next.bytes, nn.bytes);
  c->bvh_n = n;
  c->bvh_one_leaf0 = n == 1 && nodes[0].left == RKF_BVH_INVALID && nodes[0].right_or_object == 0;
  c->bvh_host.assign(nodes, nodes + n);
  c->bvh_next_host = next;
  return RKF_OK;
}

rkf_status rkf_bvh_build(const rkf_bvh_item* items, uint32_t n, rkf_bvh_node* out, uint32_t cap,
                         uint32_t* n_out) {
  if ((!items && n) || !n_out || (!out && cap)) return fail(RKF_INVALID_ARG, "rkf_bvh_build: null argument");
  const uint64_t need = n ? 2ull * n - 1 : 0;
  if (need > kMaxBvhNodes) return fail(RKF_INVALID_ARG, "rkf_bvh_build: more than 65536 nodes");
  if (cap < need) return fail(RKF_INVALID_ARG, "rkf_bvh_build: the output holds fewer than 2n-1 nodes");
  Builder b;
  b.items = items;
  b.box.resize(n);
  for (uint32_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      if (std::isnan(items[i].aabb_min[k]) || std::isnan(items[i].aabb_max[k]))
        return fail(RKF_INVALID_ARG, "rkf_bvh_build: NaN in an AABB");
      b.box[i].lo[k] = items[i].aabb_min[k];
      b.box[i].hi[k] = items[i].aabb_max[k];
    }
  if (n) {
    std::vector<uint32_t> idx(n);
    for (uint32_t i = 0; i < n; ++i) idx[i] = i;
    b.nodes.reserve(need);
    b.build(idx.data(), n);
    std::memcpy(out, b.nodes.data(), b.nodes.size() * sizeof(rkf_bvh_node));
  }
  *n_out = static_cast<uint32_t>(b.nodes.size());
  return RKF_OK;
}

}  // extern "C"
