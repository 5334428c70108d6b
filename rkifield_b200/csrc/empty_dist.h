// empty_dist.h — empty-space distance field over the top grids (empty_dist.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "device_common.cuh"

namespace rkf {

// Field values are capped here: a block this far from any non-EMPTY block
// only promises an EMPTY cube of radius kEmptyDistCap - 1 blocks.
constexpr uint32_t kEmptyDistCap = 64;

// Compute the field of object o's top grid (top[o.top_off ...]) into
// field[o.top_off ...].  Synchronises st.
rkf_status build_empty_dist(const ObjDev& o, const uint32_t* top, uint8_t* field, cudaStream_t st);

// Lower field[o.top_off ...] around `blocks` (global top indices, also on
// the device at d_blocks), which have just stopped being EMPTY.  Enqueued on
// st; d_blocks must stay valid until st reaches it.
rkf_status lower_empty_dist(const ObjDev& o, uint8_t* field, const uint32_t* d_blocks,
                            const std::vector<uint32_t>& blocks, cudaStream_t st);

}  // namespace rkf
