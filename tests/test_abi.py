"""The C-ABI library: it loads without a GPU, exports exactly the entry
points include/*.h declares, and its structs have the reference layouts."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

from rkifield_b200 import _abi as abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"^RKF_API\s+[\w\s\*]+?\b(rkf_\w+)\s*\(", src, re.M))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = abi.load_library()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (rkf_\w+)$", out, re.M))
    assert names == exported, (names ^ exported)


def test_ctypes_mirror_covers_header():
    assert declared_functions() == set(abi.SIGNATURES)


def test_reference_struct_sizes():
    # CameraUniforms 144 B (camera.rs:196), SceneUniforms 16 B (gpu_scene.rs:383-410),
    # GpuObject 256 B (gpu_object.rs:279-320)
    assert C.sizeof(abi.rkf_camera) == 144
    assert C.sizeof(abi.rkf_scene_uniforms) == 16
    assert C.sizeof(abi.rkf_gpu_object) == 256
    # GpuObject field offsets (gpu_object.rs:17-38 layout table)
    off = {n: getattr(abi.rkf_gpu_object, n).offset for n, _ in abi.rkf_gpu_object._fields_}
    assert off["aabb_min"] == 64 and off["aabb_max"] == 80
    assert off["brick_map_offset"] == 96 and off["voxel_size"] == 112
    assert off["sdf_type"] == 120 and off["blend_radius"] == 128
    assert off["accumulated_scale"] == 148 and off["object_id"] == 164
    assert off["geometry_aabb_min"] == 172 and off["_padding"] == 196


def test_c_header_layout_matches_ctypes(tmp_path):
    """Compile a C program against include/rkf_cuda.h and compare sizeof."""
    src = tmp_path / "sz.c"
    src.write_text('#include "rkf_cuda.h"\n#include <stdio.h>\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(rkf_camera),'
                   ' sizeof(rkf_scene_uniforms), sizeof(rkf_gpu_object), sizeof(rkf_march_params),'
                   ' sizeof(rkf_config), sizeof(rkf_prim), sizeof(rkf_edit_op), sizeof(rkf_request),'
                   ' sizeof(rkf_batch_tuning), sizeof(rkf_scene_node), sizeof(rkf_flat_node));}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()))
    want = [C.sizeof(t) for t in (abi.rkf_camera, abi.rkf_scene_uniforms, abi.rkf_gpu_object,
                                  abi.rkf_march_params, abi.rkf_config, abi.rkf_prim,
                                  abi.rkf_edit_op, abi.rkf_request, abi.rkf_batch_tuning,
                                  abi.rkf_scene_node, abi.rkf_flat_node)]
    assert got == want


def test_defaults_match_reference():
    lib = abi.load_library()
    p = abi.rkf_march_params()
    lib.rkf_march_params_default(C.byref(p))
    # SceneUniforms::default (gpu_scene.rs:34-43), shader constants (ray_march.wgsl:28-41)
    assert (p.scene.max_steps, p.scene.max_distance) == (128, 100.0)
    assert abs(p.scene.hit_threshold - 0.001) < 1e-9
    assert (p.hard_max_steps, p.bisect_steps) == (1024, 8)
    assert abs(p.min_step - 0.0005) < 1e-9 and abs(p.near_surface_threshold - 0.02) < 1e-9
    q = abi.rkf_march_params()
    abi.march_params_default(q)
    assert bytes(q) == bytes(p)


def test_world_relative_fp64():
    """WorldPosition::relative_to_f64 (world_position.rs:107-120)."""
    lib = abi.load_library()
    a = abi.rkf_world_pos((1000000, -3, 2), (7.5, 0.25, 1.0))
    b = abi.rkf_world_pos((999999, -4, 2), (0.5, 7.75, 0.5))
    d = (C.c_double * 3)()
    f = (C.c_float * 3)()
    lib.rkf_world_relative(C.byref(a), C.byref(b), d, f)
    assert list(d) == [15.0, 0.5, 0.5]
    assert list(f) == [15.0, 0.5, 0.5]


def test_errors_without_device_are_status_codes():
    """Calls fail with a status and a message, never an abort."""
    lib = abi.load_library()
    assert lib.rkf_create(None, None) == abi.RKF_INVALID_ARG
    assert b"null" in lib.rkf_last_error()
    assert lib.rkf_destroy(None) == abi.RKF_INVALID_ARG
