"""FP64 voxel values for a two-level index (test infrastructure).

The FP64 error reference of the large scene has no flat brick map (it would
take 17.6 GB), so the oracle evaluates FP64 voxel values for bricks listed by
coordinates and slots, read out of the two-level index.  On the small scene
both routes must give the same array, and the index walk must list exactly
the allocated bricks of the flat map."""
import numpy as np

from rkifield_b200 import _abi as abi


def _two_level(flat, dims):
    """A two-level index (top grid of 8^3-brick blocks, 512-entry leaves) of a
    flat brick map, as the device builds it."""
    dx, dy, dz = (int(x) for x in dims)
    tx, ty, tz = (dx + 7) // 8, (dy + 7) // 8, (dz + 7) // 8
    m = flat.reshape(dz, dy, dx)
    top = np.full(tx * ty * tz, abi.EMPTY_SLOT, np.uint32)
    leaves = []
    for kz in range(tz):
        for ky in range(ty):
            for kx in range(tx):
                blk = np.full((8, 8, 8), abi.EMPTY_SLOT, np.uint32)
                sub = m[kz * 8:kz * 8 + 8, ky * 8:ky * 8 + 8, kx * 8:kx * 8 + 8]
                blk[:sub.shape[0], :sub.shape[1], :sub.shape[2]] = sub
                if (blk < abi.INTERIOR_SLOT).any():
                    top[kx + ky * tx + kz * tx * ty] = len(leaves)
                    leaves.append(blk.ravel())
    return top, np.concatenate(leaves), np.array([0, tx, ty, tz], np.uint32)


def test_f64_values_by_brick_list_equal_flat_map(oracle, small_scene):
    v, prims, vp = small_scene["vox"], small_scene["prims"], small_scene["vp"]
    ref = oracle.voxel_values_f64(prims, vp, v.map, v.n_bricks)
    top, leaves, info = _two_level(v.map, v.dims)
    bxyz, slots = oracle.index_bricks(top, leaves, info)
    dx, dy = int(v.dims[0]), int(v.dims[1])
    flat_idx = np.nonzero(v.map < abi.INTERIOR_SLOT)[0]
    assert slots.size == flat_idx.size == v.n_bricks
    f = bxyz[:, 0].astype(np.int64) + bxyz[:, 1] * dx + bxyz[:, 2].astype(np.int64) * dx * dy
    assert (v.map[f] == slots).all(), "the index walk must name each brick's own slot"
    got = oracle.voxel_values_f64_bricks(prims, vp, bxyz, slots, v.n_bricks)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
