"""The C-ABI library loads on a CPU-only host and exports every entry point
include/wavefront.h declares (no compute calls without a GPU)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import wfpt
from wfpt import abi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "wavefront.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = wfpt.library()
    names = declared_functions()
    assert len(names) >= 29
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_fast_build_exports_every_declared_symbol():
    """The fast build (when built) carries the same entry points: a stale
    copy would fail every test that loads it."""
    fast = wfpt.native.PACKAGE_DIR / "libwavefront_b200_fast.so"
    if not fast.exists():
        pytest.skip("fast build not built")
    lib = ctypes.CDLL(str(fast))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_declares_every_symbol():
    lib = ctypes.CDLL(str(wfpt.native.LIB_PATH))
    assert sorted(abi.declare(lib)) == declared_functions()


def test_struct_layouts_match_header():
    # Sizes printed by a C compiler for include/wavefront.h on x86-64.
    assert abi.TRIANGLE_DTYPE.itemsize == 80
    assert abi.MATERIAL_DTYPE.itemsize == 124
    assert abi.HIT_DTYPE.itemsize == 68
    assert ctypes.sizeof(abi.SceneDesc) == 184
    assert ctypes.sizeof(abi.RenderConfig) == 136
    assert ctypes.sizeof(abi.Camera) == 56


def test_struct_sizes_compiled_from_header(tmp_path):
    # sizeof of every ctypes mirror against a C compiler reading the header.
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    pairs = {"wf_camera": abi.Camera, "wf_render_config": abi.RenderConfig, "wf_scene_desc": abi.SceneDesc,
             "wf_kernel_profile": abi.KernelProfile, "wf_render_stats": abi.RenderStats,
             "wf_batch_job": abi.BatchJob, "wf_batch_config": abi.BatchConfig, "wf_scene_info": abi.SceneInfo,
             "wf_environment": abi.Environment, "wf_diff_config": abi.DiffConfig,
             "wf_frame_guide": abi.FRAME_GUIDE_DTYPE, "wf_hit": abi.HIT_DTYPE, "wf_ray": abi.RAY_DTYPE,
             "wf_material_textures": abi.MATERIAL_TEXTURES_DTYPE, "wf_tune_space": abi.TuneSpace}
    src = tmp_path / "sizes.c"
    body = "".join(f'    printf("%zu\\n", sizeof({name}));\n' for name in pairs)
    src.write_text('#include <stdio.h>\n#include "wavefront.h"\nint main(void) {\n' + body + "    return 0;\n}\n")
    exe = tmp_path / "sizes"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    for (name, struct), size in zip(pairs.items(), sizes):
        mirrored = struct.itemsize if hasattr(struct, "itemsize") else ctypes.sizeof(struct)
        assert mirrored == size, name


def test_defaults_and_errors_without_gpu():
    lib = wfpt.library()
    assert lib.wf_version().decode().startswith("wavefront-b200")
    cfg = wfpt.render_config(1920, 1080)
    # RenderConfig defaults, include/config.hpp:11-41.
    assert (cfg.max_depth, cfg.rr_start_depth, cfg.photon_count, cfg.photon_max_depth) == (32, 12, 1048576, 8)
    assert abs(cfg.indirect_clamp - 10.0) < 1e-7 and abs(cfg.gather_radius - 0.06) < 1e-7
    assert cfg.rng == abi.RNG_XORSHIFT32 and cfg.mode == abi.MODE_GRAPH
    # Invalid descriptions are rejected on the host before any device work.
    s = wfpt.Scene()
    s.add_material(wfpt.material(abi.MAT_DIFFUSE, (1, 1, 1)))
    sp = np.zeros(1, abi.SPHERE_DTYPE)
    sp[0] = ((0, 0, 0), 1.0, 7, 0)
    s.spheres = sp
    d, keep = s.desc()
    handle = ctypes.c_void_p()
    status = lib.wf_scene_create(ctypes.byref(d), ctypes.byref(handle))
    assert status == 1 and b"material" in lib.wf_last_error()


def test_fnv1a_matches_reference_constants():
    lib = wfpt.library()
    data = np.frombuffer(b"abc", np.uint8)
    # FNV-1a 64 (render_fingerprint.cpp:11-83): offset basis 1469598103934665603, prime 1099511628211.
    h = 1469598103934665603
    for b in b"abc":
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    assert lib.wf_fnv1a64(data.ctypes.data, 3, 0) == h
