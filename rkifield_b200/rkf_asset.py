"""Reader for RKIField `.rkf` v2 voxel objects (crates/rkf-core/src/asset_file.rs).

Layout (asset_file.rs:1-28, 76-115): a 128-byte header (magic "RKF2",
version 2, LOD count, material count, AABB, analytic bound, material ids),
then 40-byte LOD entries (voxel size, brick count, brick dims, data offset,
compressed and uncompressed sizes), then per LOD one LZ4 block with the
uncompressed size prepended as a little-endian u32 (lz4_flex
compress_prepend_size, asset_file.rs:458) holding the brick map (u32 per
brick, local slot or EMPTY_SLOT) followed by the bricks (512 VoxelSample of
two u32 each).

The LZ4 block decoder follows the public LZ4 block format: a sequence is a
token byte (high nibble literal length, low nibble match length - 4; 15
means more length bytes follow, each added until one is below 255), the
literals, a 2-byte little-endian match offset, and the match copied from
the output (it may overlap itself); the last sequence has literals only.
"""
from __future__ import annotations

import dataclasses
import struct

import numpy as np

HEADER = struct.Struct("<4sIII3f3fI4f16H36s")
LOD = struct.Struct("<fI3IIQII")
assert HEADER.size == 128 and LOD.size == 40


def lz4_block_decompress(src: bytes, size: int) -> bytes:
    out = bytearray()
    i, n = 0, len(src)
    while i < n:
        token = src[i]
        i += 1
        lit = token >> 4
        if lit == 15:
            while True:
                b = src[i]
                i += 1
                lit += b
                if b != 255:
                    break
        out += src[i:i + lit]
        i += lit
        if i >= n:
            break
        off = src[i] | (src[i + 1] << 8)
        i += 2
        if off == 0 or off > len(out):
            raise ValueError("lz4: bad match offset")
        ml = token & 15
        if ml == 15:
            while True:
                b = src[i]
                i += 1
                ml += b
                if b != 255:
                    break
        ml += 4
        start = len(out) - off
        if off >= ml:
            out += out[start:start + ml]
        else:  # overlapping copy
            for k in range(ml):
                out.append(out[start + k])
    if len(out) != size:
        raise ValueError(f"lz4: decoded {len(out)} bytes, expected {size}")
    return bytes(out)


@dataclasses.dataclass
class RkfLod:
    voxel_size: float
    brick_count: int
    dims: tuple
    brick_map: np.ndarray   # u32, local slot or EMPTY_SLOT, x + y*dx + z*dx*dy
    words: np.ndarray       # u32, 1024 per brick (VoxelSample word0, word1)


@dataclasses.dataclass
class RkfObject:
    aabb_min: tuple
    aabb_max: tuple
    material_ids: list
    lods: list


def read_rkf(path: str) -> RkfObject:
    data = open(path, "rb").read()
    h = HEADER.unpack_from(data, 0)
    magic, version, lod_count, mat_count = h[0], h[1], h[2], h[3]
    if magic != b"RKF2":
        raise ValueError("not an .rkf v2 file")
    if version != 2:
        raise ValueError(f"unsupported .rkf version {version}")
    aabb_min, aabb_max = tuple(h[4:7]), tuple(h[7:10])
    mats = list(h[15:31])[: min(mat_count, 16)]
    lods = []
    for k in range(lod_count):
        vs, bc, dx, dy, dz, _pad, off, csize, usize = LOD.unpack_from(data, HEADER.size + k * LOD.size)
        block = data[off:off + csize]
        (prepended,) = struct.unpack_from("<I", block, 0)
        raw = lz4_block_decompress(block[4:], prepended)
        nmap = dx * dy * dz
        bmap = np.frombuffer(raw, np.uint32, nmap).copy()
        words = np.frombuffer(raw, np.uint32, 1024 * bc, offset=4 * nmap).copy()
        lods.append(RkfLod(vs, bc, (dx, dy, dz), bmap, words))
    return RkfObject(aabb_min, aabb_max, mats, lods)
