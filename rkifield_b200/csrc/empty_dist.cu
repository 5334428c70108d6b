// empty_dist.cu — the empty-space distance field over each object's top grid.
//
// For every block (8^3 bricks = 64^3 voxels) of an object's top grid the
// field holds 0 when the block is not EMPTY, else the Chebyshev distance, in
// blocks, to the nearest block that is not EMPTY, capped at kEmptyDistCap.
// Cells beyond the grid count as EMPTY.  So every block within distance
// (value - 1) of an EMPTY block is EMPTY too, and a ray position whose
// trilinear cell lies inside that cube samples the EMPTY constant: the march
// uses this to run those steps without touching the index.
//
// The L-infinity distance transform is separable: the distance along x, then
// the min over dy of max(|dy|, d_x), then the same over dz.  Edits only turn
// EMPTY blocks into leaf blocks, so after an edit the field is lowered around
// the touched blocks (a conservative bound that never overstates a distance).
#include <algorithm>

#include "ctx.h"
#include "empty_dist.h"

namespace rkf {

namespace detail {

struct GridDims {
  uint32_t off, nx, ny, nz;
};

// distance along x to the nearest non-EMPTY block of the row
__global__ void k_empty_dist_x(const uint32_t* __restrict__ top, uint8_t* __restrict__ out, GridDims g) {
  const uint64_t n = static_cast<uint64_t>(g.nx) * g.ny * g.nz;
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t x = static_cast<uint32_t>(i % g.nx);
  const uint32_t* row = top + g.off + (i - x);
  uint32_t d = 0;
  if (row[x] == RKF_EMPTY_SLOT) {
    for (d = 1; d < kEmptyDistCap; ++d) {
      if (x >= d && row[x - d] != RKF_EMPTY_SLOT) break;
      if (x + d < g.nx && row[x + d] != RKF_EMPTY_SLOT) break;
    }
  }
  out[i] = static_cast<uint8_t>(d);
}

// out = min over |k| of max(|k|, in at offset k along the axis)
__global__ void k_empty_dist_axis(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, GridDims g,
                                  uint32_t axis) {
  const uint64_t n = static_cast<uint64_t>(g.nx) * g.ny * g.nz;
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t y = static_cast<uint32_t>((i / g.nx) % g.ny);
  const uint32_t z = static_cast<uint32_t>(i / (static_cast<uint64_t>(g.nx) * g.ny));
  const uint32_t pos = axis == 1 ? y : z;
  const uint32_t len = axis == 1 ? g.ny : g.nz;
  const uint64_t stride = axis == 1 ? g.nx : static_cast<uint64_t>(g.nx) * g.ny;
  uint32_t best = in[i];
  for (uint32_t k = 1; k < best; ++k) {
    if (pos >= k) best = min(best, max(k, static_cast<uint32_t>(in[i - k * stride])));
    if (pos + k < len) best = min(best, max(k, static_cast<uint32_t>(in[i + k * stride])));
  }
  out[i] = static_cast<uint8_t>(best);
}

// Lower the field around newly non-EMPTY blocks: field = min(field, distance
// to the nearest of them).  Cells cover the box [lo, hi] of the grid.
__global__ void k_empty_dist_lower(uint8_t* __restrict__ field, GridDims g, const uint32_t* __restrict__ blocks,
                                   uint32_t nb, uint3 lo, uint3 ext) {
  const uint64_t n = static_cast<uint64_t>(ext.x) * ext.y * ext.z;
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t x = lo.x + static_cast<uint32_t>(i % ext.x);
  const uint32_t y = lo.y + static_cast<uint32_t>((i / ext.x) % ext.y);
  const uint32_t z = lo.z + static_cast<uint32_t>(i / (static_cast<uint64_t>(ext.x) * ext.y));
  const uint64_t cell = x + static_cast<uint64_t>(y) * g.nx + static_cast<uint64_t>(z) * g.nx * g.ny;
  uint32_t v = field[cell];
  for (uint32_t b = 0; b < nb && v > 0; ++b) {
    const uint32_t l = blocks[b] - g.off;
    const int bx = static_cast<int>(l % g.nx), by = static_cast<int>((l / g.nx) % g.ny),
              bz = static_cast<int>(l / (g.nx * g.ny));
    const uint32_t d = static_cast<uint32_t>(
        max(abs(bx - static_cast<int>(x)), max(abs(by - static_cast<int>(y)), abs(bz - static_cast<int>(z)))));
    v = min(v, d);
  }
  field[cell] = static_cast<uint8_t>(v);
}

}  // namespace detail

rkf_status build_empty_dist(const ObjDev& o, const uint32_t* top, uint8_t* field, cudaStream_t st) {
  if (o.sdf_type != RKF_SDF_VOXELIZED) return RKF_OK;
  const detail::GridDims g{o.top_off, o.tdim[0], o.tdim[1], o.tdim[2]};
  const uint64_t n = static_cast<uint64_t>(g.nx) * g.ny * g.nz;
  if (n == 0) return RKF_OK;
  DevBuf tmp;
  rkf_status s = tmp.alloc(n);
  if (s != RKF_OK) return s;
  uint8_t* f = field + o.top_off;
  const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
  detail::k_empty_dist_x<<<blocks, 256, 0, st>>>(top, f, g);
  detail::k_empty_dist_axis<<<blocks, 256, 0, st>>>(f, tmp.as<uint8_t>(), g, 1);
  detail::k_empty_dist_axis<<<blocks, 256, 0, st>>>(tmp.as<uint8_t>(), f, g, 2);
  RKF_CUDA_TRY(cudaGetLastError());
  // tmp is freed on return: finish its readers first
  RKF_CUDA_TRY(cudaStreamSynchronize(st));
  return RKF_OK;
}

rkf_status lower_empty_dist(const ObjDev& o, uint8_t* field, const uint32_t* d_blocks,
                            const std::vector<uint32_t>& blocks, cudaStream_t st) {
  if (o.sdf_type != RKF_SDF_VOXELIZED || blocks.empty()) return RKF_OK;
  const detail::GridDims g{o.top_off, o.tdim[0], o.tdim[1], o.tdim[2]};
  int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-1, -1, -1};
  for (uint32_t b : blocks) {
    const uint32_t l = b - g.off;
    const int c[3] = {static_cast<int>(l % g.nx), static_cast<int>((l / g.nx) % g.ny),
                      static_cast<int>(l / (g.nx * g.ny))};
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], c[a]);
      hi[a] = std::max(hi[a], c[a]);
    }
  }
  const int dims[3] = {static_cast<int>(g.nx), static_cast<int>(g.ny), static_cast<int>(g.nz)};
  const int reach = static_cast<int>(kEmptyDistCap) - 1;  // farther cells keep a value <= their distance
  uint3 l3, e3;
  uint32_t* lp = &l3.x;
  uint32_t* ep = &e3.x;
  for (int a = 0; a < 3; ++a) {
    const int a0 = std::max(0, lo[a] - reach), a1 = std::min(dims[a] - 1, hi[a] + reach);
    lp[a] = static_cast<uint32_t>(a0);
    ep[a] = static_cast<uint32_t>(a1 - a0 + 1);
  }
  const uint64_t n = static_cast<uint64_t>(e3.x) * e3.y * e3.z;
  detail::k_empty_dist_lower<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(
      field, g, d_blocks, static_cast<uint32_t>(blocks.size()), l3, e3);
  RKF_CUDA_TRY(cudaGetLastError());
  return RKF_OK;
}

}  // namespace rkf
