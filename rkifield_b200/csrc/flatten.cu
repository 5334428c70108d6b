// flatten.cu — object records from an object's node tree (host only).
//
// The import side of the march: the runtime turns every scene object into
// GpuObject records each frame by walking the object's node tree depth-first
// (transform_flatten.rs:56-110, flatten_object / flatten_node) and building a
// record per flat node (gpu_object.rs:141-220, GpuObject::from_flat_node).
// The walk composes world = parent world * local, starting from the object's
// scale, rotation and baked position, skips invisible subtrees (the root is
// always kept) and keeps, per node, the inverse of its world matrix and the
// product of the per-axis scales from the object down to it.
//
// The reference composes and inverts in f32 (glam).  Here the matrix products
// and the inverse run in double precision and are rounded to float once, so
// a record's inverse_world is the correctly composed inverse to within one
// rounding per entry; the scale products are f32 products as in the
// reference (the same bits).
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"

using namespace rkf;

namespace {

struct M4 {
  double c[4][4];  // c[col][row]
};

// Transform::to_matrix / Mat4::from_scale_rotation_translation: the rotation
// matrix of the quaternion (x, y, z, w) as given, its columns scaled by s,
// translation t in the last column.
M4 trs(const float q_in[4], const float s[3], const float t[3]) {
  const double x = q_in[0], y = q_in[1], z = q_in[2], w = q_in[3];
  const double r[3][3] = {
      {1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y + w * z), 2.0 * (x * z - w * y)},  // column 0
      {2.0 * (x * y - w * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z + w * x)},  // column 1
      {2.0 * (x * z + w * y), 2.0 * (y * z - w * x), 1.0 - 2.0 * (x * x + y * y)},  // column 2
  };
  M4 m;
  std::memset(&m, 0, sizeof(m));
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row) m.c[col][row] = r[col][row] * static_cast<double>(s[col]);
  for (int row = 0; row < 3; ++row) m.c[3][row] = t[row];
  m.c[3][3] = 1.0;
  return m;
}

M4 mul(const M4& a, const M4& b) {
  M4 m;
  for (int col = 0; col < 4; ++col)
    for (int row = 0; row < 4; ++row) {
      double acc = 0.0;
      for (int k = 0; k < 4; ++k) acc += a.c[k][row] * b.c[col][k];
      m.c[col][row] = acc;
    }
  return m;
}

// Gauss-Jordan elimination with partial pivoting; false when singular.
bool inverse(const M4& m, M4* out) {
  double a[4][8];
  for (int row = 0; row < 4; ++row)
    for (int col = 0; col < 4; ++col) {
      a[row][col] = m.c[col][row];
      a[row][4 + col] = row == col ? 1.0 : 0.0;
    }
  for (int col = 0; col < 4; ++col) {
    int piv = col;
    for (int row = col + 1; row < 4; ++row)
      if (std::fabs(a[row][col]) > std::fabs(a[piv][col])) piv = row;
    if (!(std::fabs(a[piv][col]) > 0.0) || !std::isfinite(a[piv][col])) return false;
    if (piv != col)
      for (int k = 0; k < 8; ++k) std::swap(a[piv][k], a[col][k]);
    const double inv_p = 1.0 / a[col][col];
    for (int k = 0; k < 8; ++k) a[col][k] *= inv_p;
    for (int row = 0; row < 4; ++row) {
      if (row == col || a[row][col] == 0.0) continue;
      const double f = a[row][col];
      for (int k = 0; k < 8; ++k) a[row][k] -= f * a[col][k];
    }
  }
  for (int row = 0; row < 4; ++row)
    for (int col = 0; col < 4; ++col) {
      out->c[col][row] = a[row][4 + col];
      if (!std::isfinite(out->c[col][row])) return false;
    }
  return true;
}

// One entry of the walk's path from the root to the current node.
struct PathEntry {
  uint32_t node;     // input index
  uint32_t flat;     // output index, RKF_NO_PARENT when the node is left out
  uint32_t depth;
  M4 world;
  float scale[3];
};

}  // namespace

extern "C" rkf_status rkf_flatten_object(const rkf_scene_node* nodes, uint32_t n_nodes,
                                         const float object_rotation[4], const float object_scale[3],
                                         const float world_position[3], rkf_flat_node* out, uint32_t* n_out) {
  if (!nodes || !object_rotation || !object_scale || !world_position || !out || !n_out || n_nodes == 0)
    return fail(RKF_INVALID_ARG, "rkf_flatten_object: null argument or no nodes");
  *n_out = 0;
  if (nodes[0].parent != RKF_NO_PARENT)
    return fail(RKF_INVALID_ARG, "rkf_flatten_object: the first node must be the root");
  // flatten_object (transform_flatten.rs:58-76): the object's own transform
  // is the root node's parent world; its scale starts the products
  const M4 object_world = trs(object_rotation, object_scale, world_position);
  std::vector<PathEntry> path;
  uint32_t written = 0;
  for (uint32_t i = 0; i < n_nodes; ++i) {
    const rkf_scene_node& nd = nodes[i];
    const PathEntry* parent = nullptr;
    if (i > 0) {
      if (nd.parent == RKF_NO_PARENT || nd.parent >= i)
        return fail(RKF_INVALID_ARG, "rkf_flatten_object: node " + std::to_string(i) +
                                         " names no earlier parent (one root, pre-order)");
      // pre-order: the parent is on the path from the root to the last node
      while (!path.empty() && path.back().node != nd.parent) path.pop_back();
      if (path.empty())
        return fail(RKF_INVALID_ARG, "rkf_flatten_object: node " + std::to_string(i) +
                                         " is not in depth-first pre-order");
      parent = &path.back();
    }
    PathEntry e;
    e.node = i;
    e.depth = parent ? parent->depth + 1 : 0;
    // flatten_node (:80-110): invisible children are skipped with their
    // subtrees; the root is always flattened
    const bool kept = !parent || (parent->flat != RKF_NO_PARENT && nd.visible != 0);
    e.flat = RKF_NO_PARENT;
    if (kept) {
      const M4& pw = parent ? parent->world : object_world;
      e.world = mul(pw, trs(nd.rotation, nd.scale, nd.position));
      for (int a = 0; a < 3; ++a) e.scale[a] = (parent ? parent->scale[a] : object_scale[a]) * nd.scale[a];
      M4 inv;
      if (!inverse(e.world, &inv))
        return fail(RKF_INVALID_ARG, "rkf_flatten_object: node " + std::to_string(i) + " has a singular world matrix");
      rkf_flat_node& f = out[written];
      for (int col = 0; col < 4; ++col)
        for (int row = 0; row < 4; ++row) f.inverse_world[4 * col + row] = static_cast<float>(inv.c[col][row]);
      for (int a = 0; a < 3; ++a) f.accumulated_scale[a] = e.scale[a];
      f.depth = e.depth;
      f.parent_index = parent ? parent->flat : RKF_NO_PARENT;
      f.node = i;
      e.flat = written++;
    }
    path.push_back(e);
  }
  *n_out = written;
  return RKF_OK;
}

extern "C" rkf_status rkf_gpu_object_from_flat_node(const rkf_flat_node* flat, const rkf_scene_node* source,
                                                    uint32_t object_id, const float aabb_min[4],
                                                    const float aabb_max[4], const float geometry_aabb_min[3],
                                                    const float geometry_aabb_max[3], rkf_gpu_object* out) {
  if (!flat || !source || !aabb_min || !aabb_max || !geometry_aabb_min || !geometry_aabb_max || !out)
    return fail(RKF_INVALID_ARG, "rkf_gpu_object_from_flat_node: null argument");
  if (source->sdf_type > RKF_SDF_VOXELIZED || source->blend_mode > RKF_BLEND_INTERSECT ||
      (source->sdf_type == RKF_SDF_ANALYTICAL && source->primitive_type > RKF_PRIM_PLANE))
    return fail(RKF_INVALID_ARG, "rkf_gpu_object_from_flat_node: bad sdf type, primitive or blend mode");
  rkf_gpu_object o;
  std::memset(&o, 0, sizeof(o));
  std::memcpy(o.inverse_world, flat->inverse_world, sizeof(o.inverse_world));
  std::memcpy(o.aabb_min, aabb_min, sizeof(o.aabb_min));
  std::memcpy(o.aabb_max, aabb_max, sizeof(o.aabb_max));
  o.sdf_type = source->sdf_type;
  if (source->sdf_type == RKF_SDF_ANALYTICAL) {  // (:162-176) and primitive_params (:233-256)
    o.material_id = source->material_id;
    std::memcpy(o.sdf_params, source->params, sizeof(o.sdf_params));
    o.primitive_type = source->primitive_type;
  } else if (source->sdf_type == RKF_SDF_VOXELIZED) {  // (:177-194)
    o.brick_map_offset = source->brick_map_offset;
    std::memcpy(o.brick_map_dims, source->brick_map_dims, sizeof(o.brick_map_dims));
    o.voxel_size = source->voxel_size;
  }
  // blend_mode_encode (:196, :258-266): the radius belongs to the smooth union
  o.blend_mode = source->blend_mode;
  o.blend_radius = source->blend_mode == RKF_BLEND_SMOOTH_UNION ? source->blend_radius : 0.0f;
  std::memcpy(o.accumulated_scale, flat->accumulated_scale, sizeof(o.accumulated_scale));
  o.lod_level = 0;
  o.object_id = object_id;
  std::memcpy(o.geometry_aabb_min, geometry_aabb_min, sizeof(o.geometry_aabb_min));
  std::memcpy(o.geometry_aabb_max, geometry_aabb_max, sizeof(o.geometry_aabb_max));
  *out = o;
  return RKF_OK;
}
