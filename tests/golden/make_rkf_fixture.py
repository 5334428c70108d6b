"""Build tests/golden/test_cross_rkf.npz from the reference's scenes/test_cross.rkf.

test_cross.rkf is the reference's own voxelization (voxelize_sdf,
crates/rkf-core/src/voxelize_object.rs:53-182) of five smooth-unioned
spheres, written by crates/rkf-core/examples/gen_test_rkf.rs.  This script
decodes it with rkifield_b200.rkf_asset and stores the finest LOD's brick map
and VoxelSample words, plus the sphere list and parameters the generator
used, so tests can check both voxelizers and the march against reference
output without the reference tree.

Usage: python tests/golden/make_rkf_fixture.py <path to the RKIField checkout>
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from rkifield_b200.rkf_asset import read_rkf  # noqa: E402

# gen_test_rkf.rs:27-38 (centre, radius), voxel size 0.03, smooth k 0.15,
# material 6, AABB = sphere extents + 4 voxels
SPHERES = [((0.0, 0.0, 0.0), 0.35), ((0.55, 0.0, 0.0), 0.25), ((-0.55, 0.0, 0.0), 0.25),
           ((0.0, 0.0, 0.55), 0.25), ((0.0, 0.0, -0.55), 0.25)]


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else "."
    obj = read_rkf(os.path.join(root, "scenes", "test_cross.rkf"))
    lod = obj.lods[-1]
    np.savez_compressed(os.path.join(HERE, "test_cross_rkf.npz"), brick_map=lod.brick_map, words=lod.words,
                        voxel_size=np.float32(lod.voxel_size), dims=np.array(lod.dims, np.uint32),
                        sphere_centres=np.array([s[0] for s in SPHERES], np.float32),
                        sphere_radii=np.array([s[1] for s in SPHERES], np.float32),
                        smooth_k=np.float32(0.15), material=np.uint32(6),
                        aabb_min=np.array(obj.aabb_min, np.float32), aabb_max=np.array(obj.aabb_max, np.float32))
    print("bricks", lod.brick_count, "dims", lod.dims)


if __name__ == "__main__":
    main()
