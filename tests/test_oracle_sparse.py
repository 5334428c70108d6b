"""The oracle's sparse voxelizer (test infrastructure): it classifies only
the bricks some primitive's candidate test reaches and writes a two-level
index instead of a flat brick map, so the 1.1 M-brick scene can be built on
the host without the 17.6 GB flat map.  On the small scene it must give the
flat voxelizer's slots, words, INTERIOR bricks and marches, bit for bit."""
import numpy as np

from rkifield_b200 import _abi as abi


def test_sparse_voxelizer_equals_flat(oracle, small_scene):
    from rkifield_b200 import scenes
    v = small_scene["vox"]
    sv = oracle.SparseVoxelized(small_scene["prims"], small_scene["vp"])
    assert sv.n_bricks == v.n_bricks and sv.n_interior == v.n_interior
    assert (sv.dims == v.dims).all()
    # every brick of the flat map resolves to the same entry through the index
    dx, dy, dz = (int(x) for x in v.dims)
    f = np.arange(dx * dy * dz, dtype=np.int64)
    bx, by, bz = f % dx, (f // dx) % dy, f // (dx * dy)
    tx, ty = int(sv.tdim[0]), int(sv.tdim[1])
    t = sv.top[bx // 8 + (by // 8) * tx + (bz // 8) * tx * ty]
    leaf = np.where(t < abi.INTERIOR_SLOT, t, 0).astype(np.int64)
    ent = np.where(t < abi.INTERIOR_SLOT,
                   sv.leaves[leaf * 512 + (bx & 7) + (by & 7) * 8 + (bz & 7) * 64], t)
    assert (ent == v.map).all()
    # the planes hold the flat voxelizer's words
    w0 = v.words[0::2]
    assert (sv.dist_f16 == (w0 & 0xFFFF)).all()
    assert (sv.mat == (((w0 >> 16) & 0x3F) | (((w0 >> 22) & 0x3F) << 6))).all()
    assert (sv.blend == (v.words[1::2] >> 24)).all()
    slots = v.map[sv.bxyz[:, 0] + sv.bxyz[:, 1].astype(np.int64) * dx + sv.bxyz[:, 2].astype(np.int64) * dx * dy]
    assert (slots == np.arange(sv.n_bricks)).all()
    # the two scenes march alike
    o = sv.gpu_object()
    ref_o = v.gpu_object()
    assert bytes(o) == bytes(ref_o)
    spec = small_scene["spec"]
    cam = scenes.seeded_camera(spec, 48, 32, seed=11)
    p = scenes.march_params(spec)
    a = oracle.march(sv.scene(), cam, p, 48, 32, threads=4)
    b = oracle.march(oracle.Scene([ref_o], pool_words=v.words, brick_maps=v.map), cam, p, 48, 32, threads=4)
    for k in ("t", "normal", "slot", "material", "flags"):
        assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), k
    assert (a["flags"] & 1).sum() > 50
