// edit.h — device CSG edits (edit.cu) and the brick lookup they use.
#pragma once

#include <functional>
#include <vector>

#include "ctx.h"

namespace rkf {

struct EditOutcome {
  uint32_t changed_bricks = 0;
  bool new_epoch = false;         // the edit changed bricks: a new top grid and field exist
  DevBuf new_top;                 // top grid of the new epoch (unless written to top_dst)
  DevBuf new_empty_dist;          // its empty-space distance field (unless field_dst)
  std::vector<uint32_t> retired;  // slots the new epoch no longer references
  std::vector<uint32_t> retired_leaves;  // index leaves the new epoch no longer references
  // optional caller memory for the new epoch (top_len u32 / top_len bytes);
  // when both are set nothing is allocated for it
  uint32_t* top_dst = nullptr;
  uint8_t* field_dst = nullptr;
};

// Device scratch for an edit's temporaries (nullptr: none left).  The memory
// must stay untouched by other work until the edit's stream is synchronised.
using EditScratch = std::function<void*(size_t bytes)>;

// Applies one edit; on success with changed bricks, out->new_top holds the
// new epoch's top grid (the caller publishes it), out->retired the slots and
// out->retired_leaves the leaves to free once no work reads the previous
// epoch.  New leaves reuse freed leaf numbers (Ctx::free_leaves) first.  Synchronises `st`.  With
// scratch, the temporaries come from it instead of device allocations (whose
// release would wait for every stream of the device).
rkf_status apply_edit(Ctx* c, const rkf_edit_op& op, cudaStream_t st, EditOutcome* out,
                      const EditScratch* scratch = nullptr);

// Slots (or sentinels) of n bricks (bxyz: 3 u32 each, device) of object obj
// through the current index, into d_out (device).  Enqueued on st.
rkf_status lookup_bricks(Ctx* c, uint32_t obj, const uint32_t* d_bxyz, uint32_t n, uint32_t* d_out,
                         cudaStream_t st);

}  // namespace rkf
