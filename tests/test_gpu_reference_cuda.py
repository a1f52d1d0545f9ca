"""The reference's own CUDA renderer on the same GPU.

oracle/_ref/libwfref_cuda.so is the reference's renderer compiled for sm_100a
from its own sources (`make -C oracle cuda`; nvcc's default floating-point
flags, so multiply-adds are contracted there and not here).  Both renderers
run the same seeded scene, camera and absolute sample range through their
task calls: the reference's RenderTaskRenderer::render and this renderer's
wf_render + wf_framebuffer_download.  The two images are the same paths, so
their relative RMSE (root-mean-square difference over the root-mean-square
of the reference image) only reflects contraction and elementary-function
rounding: it must stay below 1 % on the Cornell box (16 spp) and below 2 % on
the reduced large mesh (4 spp; terrain, 50 instances, glass spheres, HDR
environment with a 5e4 sun) with caustics off.  With the reduced large
mesh's 200,000-photon caustics on, each side gathers from its own photon map
(the reference's built by its own kernels with the same grid bounds, cell
lists in atomic order), and the bound is 3 %.

The comparison runs in a child process (oracle/ref_cuda_bench.py), so the
reference's exit-on-error cannot end the test session.  Skipped when the
library has not been built.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "oracle" / "_ref" / "libwfref_cuda.so"

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not LIB.exists(), reason="reference CUDA build absent (make -C oracle cuda)")]


@pytest.mark.parametrize("workload,mode,caustics,tolerance,build", [
    ("cornell", "graph", False, 0.01, "exact"),
    ("cornell", "persistent", False, 0.01, "exact"),
    ("large_mesh_small", "graph", False, 0.02, "exact"),
    ("large_mesh_small", "graph", True, 0.03, "exact"),
    ("cornell", "graph", False, 0.01, "fast"),
    ("large_mesh_small", "graph", True, 0.03, "fast"),
])
def test_image_matches_reference_cuda_renderer(cuda, workload, mode, caustics, tolerance, build):
    """`build` fast: this renderer's fast build (libwavefront_b200_fast.so)."""
    fast = ROOT / "wavefront-path-tracer_b200" / "libwavefront_b200_fast.so"
    if build == "fast" and not fast.exists():
        pytest.skip("fast build absent (make fast)")
    cmd = [sys.executable, str(ROOT / "oracle" / "ref_cuda_bench.py"), "--workload", workload, "--mode", mode,
           "--steps", "1"]
    if not caustics:
        cmd.append("--no-caustics")
    env = dict(os.environ)
    if build == "fast":
        env["WF_BUILD"] = "fast"
    run = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT, env=env)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    line = json.loads(run.stdout.strip().splitlines()[-1])
    ref = line["reference_cuda"][mode]
    assert ref["Mpaths/s"] > 0 and line["b200_renderer"]["Mpaths/s"] > 0
    assert line["caustics"] == int(caustics)
    assert ref["image_relative_rmse"] <= tolerance, line
