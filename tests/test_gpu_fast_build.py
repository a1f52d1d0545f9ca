"""The fast build (libwavefront_b200_fast.so: multiply-adds contracted and
CUDA's own single-precision elementary functions, `make fast`) against the
reference as written -- its renderer compiled for the host with the C
library's math (oracle/_ref/libwfref.so) -- on the same seeded scenes and
sample ranges.  The two differ only in floating-point rounding, so the
images must agree within a relative RMSE: 1 % on the Cornell box (16 spp),
2 % on the reduced large mesh (4 spp, caustics off), 3 % on the reduced
sphere field (16 spp).  The sphere field's glass and fuzzy metal decide
paths by Fresnel and roulette coin flips, so an ulp of difference sends the
odd path elsewhere; each such path is an independent sample, and their
share of the RMSE falls with the sample count (3.4 % measured at 4 spp).
Run in a child process so that this process keeps the default library."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
FAST = ROOT / "wavefront-path-tracer_b200" / "libwavefront_b200_fast.so"

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not FAST.exists(), reason="fast build absent (make fast)")]

CHILD = r'''
import json, sys
sys.path[:0] = [sys.argv[1] + "/wavefront-path-tracer_b200", sys.argv[1] + "/oracle", sys.argv[1] + "/tests"]
import numpy as np
import oracle, wfpt
from wfpt import scenes
from helpers import relative_rmse
cases = {
    "cornell": (scenes.cornell_box(64, 64), 64, 64, dict(max_depth=8, rr_start_depth=3), 16),
    "sphere_field": (scenes.sphere_field(96, 54, frequency=16), 96, 54, dict(max_depth=16), 16),
    "large_mesh": (scenes.large_mesh(96, 54, terrain_quads=64, instance_count=12, instance_frequency=8,
                                     glass_spheres=3, env_size=(256, 128)), 96, 54, dict(max_depth=12), 4),
}
out = {"library": str(wfpt.native.LIB_PATH)}
for name, ((scene, cam), w, h, fields, spp) in cases.items():
    cfg = wfpt.render_config(w, h, **fields)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    got = r.render_task((0, 0, w, h), 500, spp)
    r.close(); dev.close()
    want, _, _ = oracle.RefScene(scene, det=False).render(cam, cfg, sample_start=500, sample_count=spp)
    out[name] = relative_rmse(got, want)
print(json.dumps(out))
'''


def test_fast_build_images_match_the_reference_as_written(cuda):
    env = dict(os.environ, WF_BUILD="fast")
    run = subprocess.run([sys.executable, "-c", CHILD, str(ROOT)], capture_output=True, text=True, timeout=900,
                         cwd=ROOT, env=env)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    r = json.loads(run.stdout.strip().splitlines()[-1])
    assert r["library"].endswith("libwavefront_b200_fast.so")
    assert r["cornell"] <= 0.01, r
    assert r["sphere_field"] <= 0.03 and r["large_mesh"] <= 0.02, r
