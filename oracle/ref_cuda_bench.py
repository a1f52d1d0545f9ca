"""ORACLE / TEST INFRASTRUCTURE ONLY: the reference's CUDA renderer on this GPU.

Loads oracle/_ref/libwfref_cuda.so (the reference's own renderer sources
compiled for sm_100a by `make -C oracle cuda`; see ref_cuda_harness.cu) and
times it beside the B200 renderer on the same seeded scene, camera, depth,
RNG strategy and absolute sample ranges.  Both sides are timed the same way:
the wall time of one whole-frame task, which is the reference's
RenderTaskRenderer::render (clear, sample launches, synchronise, download)
against this renderer's wf_render + wf_framebuffer_download.  Caustics are
off on both sides: the reference builds a photon map only for its Cornell
family of presets, with fixed Cornell grid bounds.

Prints one JSON line: both throughputs in Mpaths/s and the relative RMSE
between the two renderers' images of the last task (the same paths; the two
builds differ only in floating-point contraction and elementary functions).

    python oracle/ref_cuda_bench.py --workload large_mesh --mode graph --steps 5
    python oracle/ref_cuda_bench.py --manifest assets/scenes/sponza.json --spp 4
"""
import argparse
import ctypes as C
import json
import statistics
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "wavefront-path-tracer_b200"))
LIB = Path(__file__).resolve().parent / "_ref" / "libwfref_cuda.so"


def load():
    lib = C.CDLL(str(LIB))
    P, U32 = C.c_void_p, C.c_uint32
    lib.wfcuda_scene_create.restype = P
    lib.wfcuda_scene_create.argtypes = [P, P]
    lib.wfcuda_scene_destroy.argtypes = [P]
    lib.wfcuda_render.restype = C.c_int
    lib.wfcuda_render.argtypes = [P, P, P, C.c_int, U32, U32, U32, P, P]
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="large_mesh")
    ap.add_argument("--mode", choices=("graph", "persistent"), default="graph")
    ap.add_argument("--spp", type=int, default=0, help="samples per task (default: bench.py's samples per step)")
    ap.add_argument("--own-mode", choices=("graph", "persistent", "stream"), default=None,
                    help="schedule of the B200 renderer (default: bench.py's schedule for the workload)")
    ap.add_argument("--steps", type=int, default=5, help="timed tasks (after one warm-up task)")
    ap.add_argument("--sample-start", type=int, default=1000)
    ap.add_argument("--manifest", default=None,
                    help="a scene manifest of the reference's presets, loaded by wfpt.assets, instead of a workload")
    ap.add_argument("--size", default="1280x720", help="image size for --manifest")
    args = ap.parse_args()

    import bench
    import wfpt
    from wfpt import native

    if args.manifest:
        from wfpt import assets
        width, height = (int(x) for x in args.size.split("x"))
        scene, cam = assets.preset_scene(args.manifest, width, height)
        rkw = {}
        args.workload = "preset " + Path(args.manifest).stem
    else:
        scene, cam, width, height, rkw = bench.make_scene(args.workload)
    for k in ("caustics", "photon_count"):
        rkw.pop(k, None)
    args.spp = args.spp or bench.SPP_PER_STEP.get(args.workload, 1)
    own_mode = args.own_mode or bench.DEFAULT_MODE.get(args.workload, "graph")
    cfg = wfpt.render_config(width, height, **rkw)
    own_cfg = wfpt.render_config(width, height, mode=bench.MODES[own_mode], **rkw)
    cam_struct = native.camera_struct(cam)

    # --- the reference's CUDA renderer
    lib = load()
    d, keep = scene.desc()
    env, rgba = scene.environment_struct()
    t0 = time.perf_counter()
    handle = lib.wfcuda_scene_create(C.addressof(d), C.addressof(env) if env is not None else None)
    ref_setup = time.perf_counter() - t0
    if not handle:
        raise SystemExit("reference scene creation failed")
    ref_ms = (C.c_double * args.steps)()
    ref_img = np.zeros((height, width, 3), np.float32)
    rc = lib.wfcuda_render(handle, C.addressof(cam_struct), C.addressof(cfg), int(args.mode == "persistent"),
                           args.sample_start, args.spp, args.steps, ref_img.ctypes.data, ref_ms)
    lib.wfcuda_scene_destroy(handle)
    if rc != 0:
        raise SystemExit(f"reference render failed ({rc})")
    del keep, rgba

    # --- this renderer, same tasks, same timing
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, own_cfg)
    own_ms = []
    own_img = None
    for i in range(args.steps + 1):
        start = args.sample_start + i * args.spp
        t0 = time.perf_counter()
        img = r.render_task((0, 0, width, height), start, args.spp)
        t1 = time.perf_counter()
        if i:
            own_ms.append((t1 - t0) * 1e3)
        own_img = img
    r.close()
    dev.close()

    paths = width * height * args.spp
    ref_t = statistics.median(list(ref_ms))
    own_t = statistics.median(own_ms)
    diff = own_img.astype(np.float64) - ref_img.astype(np.float64)
    rel_rmse = float(np.sqrt(np.mean(diff ** 2)) / max(np.sqrt(np.mean(ref_img.astype(np.float64) ** 2)), 1e-30))
    print(json.dumps({
        "workload": args.workload, "triangles": int(scene.triangle_count()), "width": width, "height": height,
        "spp_per_task": args.spp,
        "max_depth": cfg.max_depth, "caustics": 0, "reference_mode": args.mode, "own_mode": own_mode,
        "reference_cuda": {"Mpaths/s": paths / ref_t / 1e3, "ms_per_task": ref_t,
                           "ms_per_task_all": [round(x, 3) for x in ref_ms], "scene_setup_s": ref_setup},
        "b200_renderer": {"Mpaths/s": paths / own_t / 1e3, "ms_per_task": own_t,
                          "ms_per_task_all": [round(x, 3) for x in own_ms]},
        "speedup": ref_t / own_t,
        "image_relative_rmse": rel_rmse,
        "timing": "wall time per whole-frame task: render + download of the radiance (median)",
    }), flush=True)


if __name__ == "__main__":
    main()
