"""The C-ABI library: it loads, exports every symbol the header declares, its structure
layout matches the ctypes mirror, and tt_create validates input without touching a GPU."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.scene import make_params

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "toytrace_gpu.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:tt_status|int32_t|void)\s+(tt_\w+)\s*\(", text, re.M)))


def test_header_symbols_listed():
    assert declared_functions() == sorted(abi.EXPORTED_SYMBOLS)


def test_library_exports_every_symbol(gpu_lib):
    for name in declared_functions():
        assert hasattr(gpu_lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(abi.lib_path())], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (tt_\w+)", out))
    assert set(declared_functions()) <= exported


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text(f'#include "{HEADER}"\n#include <stdio.h>\n#include <stddef.h>\n'
                   "int main(){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n\","
                   "sizeof(tt_material),sizeof(tt_env_light),sizeof(tt_point_light),sizeof(tt_camera),"
                   "sizeof(tt_scene_desc),sizeof(tt_params),sizeof(tt_stats),offsetof(tt_scene_desc,camera),"
                   "offsetof(tt_env_light,tex_rgb),sizeof(tt_medium),offsetof(tt_medium,sigma_t));return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    mine = [C.sizeof(abi.Material), C.sizeof(abi.EnvLight), C.sizeof(abi.PointLight), C.sizeof(abi.Camera),
            C.sizeof(abi.SceneDesc), C.sizeof(abi.Params), C.sizeof(abi.Stats), abi.SceneDesc.camera.offset,
            abi.EnvLight.tex_rgb.offset, C.sizeof(abi.Medium), abi.Medium.sigma_t.offset]
    assert vals == mine


def test_abi_version(gpu_lib):
    assert gpu_lib.tt_abi_version() == 9


def _create(lib, scene, params):
    desc, keep = scene.to_desc()
    h = C.c_void_p()
    st = lib.tt_create(C.byref(desc), C.byref(params), C.byref(h))
    return st, h


def test_create_validates_without_gpu(gpu_lib):
    scene = scenes.cornell_box(8, 8)
    st, h = _create(gpu_lib, scene, make_params())
    assert st == abi.TT_OK and h.value
    # Rendering before the upload is refused with TT_ERR_NOT_READY.
    assert gpu_lib.tt_render_pass(h, 1, 1) == abi.TT_ERR_NOT_READY
    assert "tt_upload_scene" in abi.last_error(gpu_lib, h)
    gpu_lib.tt_destroy(h)
    # Out-of-range material index.
    scene._mats_of_tris[0][:] = 99
    scene._flat = None
    st, h = _create(gpu_lib, scene, make_params())
    assert st == abi.TT_ERR_INVALID and not h.value
    assert "material index" in abi.last_error(gpu_lib, None)
    # Large meshes are checked by several threads; the error names the first bad triangle.
    big = scenes.terrain_spheres(xres=32, yres=18, terrain_n=256, sphere_level=2, num_spheres=2, env_w=16, env_h=8)
    tris = big.arrays()[2]
    assert len(tris) > 100_000
    tris[100_000, 1] = 1 << 30
    tris[70_000, 2] = 1 << 30
    big.arrays()[3][60_000] = 99
    st, h = _create(gpu_lib, big, make_params())
    assert st == abi.TT_ERR_INVALID and "material index out of range in triangle 60000" in abi.last_error(gpu_lib, None)
    big.arrays()[3][60_000] = 0
    st, h = _create(gpu_lib, big, make_params())
    assert st == abi.TT_ERR_INVALID and "vertex index out of range in triangle 70000" in abi.last_error(gpu_lib, None)
    # Bad sample mode.
    st, h = _create(gpu_lib, scenes.cornell_box(8, 8), make_params(pt_sample_mode=7))
    assert st == abi.TT_ERR_INVALID
    # Null arguments.
    assert gpu_lib.tt_create(None, None, None) == abi.TT_ERR_INVALID


def test_stop_flags_are_host_only(gpu_lib):
    st, h = _create(gpu_lib, scenes.cornell_box(8, 8), make_params())
    assert st == abi.TT_OK
    assert gpu_lib.tt_stop_requested(h) == 0
    assert gpu_lib.tt_request_interrupt(h) == abi.TT_OK
    assert gpu_lib.tt_poll_interrupt(h) == 1
    assert gpu_lib.tt_poll_interrupt(h) == 0
    assert gpu_lib.tt_request_stop(h) == abi.TT_OK
    assert gpu_lib.tt_stop_requested(h) == 1
    gpu_lib.tt_destroy(h)
