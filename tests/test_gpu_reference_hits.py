"""Closest-hit identities against the reference's own CUDA traversal on the
same GPU (oracle/ref_cuda_hits.py, in a child process): the Cornell box's
sample-0 ray batch (65,536 camera rays and their bounce-1 continuations)
and the reduced large mesh's.  The reference's sm_100a build contracts
multiply-adds; the exact build here does not, the fast build does, so a ray
that grazes an edge or meets two surfaces at nearly the same distance may
resolve differently, and a ray that meets a primitive at a distance near
the minimum may take the other root or face.  Bound: at most 1 ray in
10,000 with a different kind, primitive or instance, and at most 1 in
10,000 of the agreeing rays with t apart by more than 1e-4 relative."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "oracle" / "_ref" / "libwfref_cuda.so"
FAST = ROOT / "wavefront-path-tracer_b200" / "libwavefront_b200_fast.so"

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not LIB.exists(), reason="reference CUDA build absent (make -C oracle cuda)")]


@pytest.mark.parametrize("build", ["exact", "fast"])
@pytest.mark.parametrize("workload", ["cornell", "large_mesh_small"])
def test_hit_identities_match_reference_cuda(cuda, workload, build):
    if build == "fast" and not FAST.exists():
        pytest.skip("fast build absent (make -C wavefront-path-tracer_b200 fast)")
    env = dict(os.environ)
    if build == "fast":
        env["WF_BUILD"] = "fast"
    run = subprocess.run([sys.executable, str(ROOT / "oracle" / "ref_cuda_hits.py"), "--workload", workload],
                         capture_output=True, text=True, timeout=900, cwd=ROOT, env=env)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    r = json.loads(run.stdout.strip().splitlines()[-1])
    assert r["build"] == build and r["rays"] > 10_000 and r["hits"] > r["rays"] // 4, r
    differ = r["kind_differs"] + r["primitive_differs"] + r["instance_differs"]
    assert differ <= r["rays"] // 10_000, r
    assert r["t_differs"] <= r["rays"] // 10_000, r
