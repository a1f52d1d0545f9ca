"""ORACLE / TEST INFRASTRUCTURE ONLY: closest hits of this renderer against
the reference's own CUDA traversal on the same GPU.

Loads oracle/_ref/libwfref_cuda.so (the reference built for sm_100a with
nvcc's default floating-point flags, see ref_cuda_harness.cu) and traces one
ray batch with its traceRayExternal (device_traversal.cuh:1196) on the
hit-identity probe copy of the scene, then the same batch with this
renderer's wf_trace_closest (the build WF_BUILD selects).  The batch is the
reference's own ray queues of one sample (the host-compiled reference's
camera rays and their bounce-1 continuations, oracle.RefScene.path_rays).
Prints one JSON line: rays, how many differ in kind / primitive / instance,
and the largest relative difference of t among the rays that agree.

    WF_BUILD=fast python oracle/ref_cuda_hits.py --workload cornell
"""
import argparse
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "wavefront-path-tracer_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
LIB = Path(__file__).resolve().parent / "_ref" / "libwfref_cuda.so"


def reference_hits(scene, rays):
    from wfpt import abi
    lib = C.CDLL(str(LIB))
    P, U32 = C.c_void_p, C.c_uint32
    lib.wfcuda_scene_create_probe.restype = P
    lib.wfcuda_scene_create_probe.argtypes = [P, P, C.c_int]
    lib.wfcuda_scene_destroy.argtypes = [P]
    lib.wfcuda_trace.restype = C.c_int
    lib.wfcuda_trace.argtypes = [P, P, U32, P]
    d, keep = scene.desc()
    env, rgba = scene.environment_struct()
    handle = lib.wfcuda_scene_create_probe(C.addressof(d), C.addressof(env) if env is not None else None, 1)
    del keep, rgba
    if not handle:
        raise SystemExit("reference scene creation failed")
    rays = np.ascontiguousarray(rays, abi.RAY_DTYPE)
    hits = np.zeros(len(rays), abi.HIT_DTYPE)
    rc = lib.wfcuda_trace(handle, rays.ctypes.data, len(rays), hits.ctypes.data)
    lib.wfcuda_scene_destroy(handle)
    if rc != 0:
        raise SystemExit(f"wfcuda_trace failed ({rc})")
    return hits


def compare(workload):
    import bench
    import oracle
    import wfpt
    from wfpt import abi
    scene, cam, width, height, rkw = bench.make_scene(workload)
    cfg = wfpt.render_config(width, height, **{k: v for k, v in rkw.items() if k not in ("caustics", "photon_count")})
    host = oracle.RefScene(scene, det=True)
    rays, counts = host.path_rays(cam, cfg, sample=0, bounces=2)
    host.close()
    want = reference_hits(scene, rays)
    dev = wfpt.DeviceScene(scene)
    got = dev.trace_closest(rays)
    dev.close()
    hit = want["kind"] != abi.HIT_NONE
    same_kind = got["kind"] == want["kind"]
    same_prim = same_kind & ((got["primitive"] == want["primitive"]) | ~hit)
    mesh = want["kind"] == abi.HIT_MESH
    same_inst = ~mesh | (got["instance"] == want["instance"])
    agree = same_prim & same_inst & hit
    rel_t = np.abs(got["t"][agree].astype(np.float64) - want["t"][agree]) / np.abs(want["t"][agree])
    exact_t = int((got["t"][agree].view(np.uint32) == want["t"][agree].view(np.uint32)).sum())
    # e.g. a sphere whose near root lands just below the minimum distance on
    # one side and just above on the other: same primitive, other root
    t_differs = int((rel_t > 1e-4).sum())
    return {"workload": workload, "build": "fast" if "fast" in str(wfpt.native.LIB_PATH) else "exact",
            "rays": int(len(rays)), "per_bounce": [int(c) for c in counts], "hits": int(hit.sum()),
            "kind_differs": int((~same_kind).sum()), "primitive_differs": int((~same_prim).sum()),
            "instance_differs": int((~same_inst).sum()), "t_bit_identical": exact_t, "t_differs": t_differs,
            "t_max_relative_difference": float(rel_t.max()) if rel_t.size else 0.0}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="cornell")
    args = ap.parse_args()
    print(json.dumps(compare(args.workload)), flush=True)


if __name__ == "__main__":
    main()
