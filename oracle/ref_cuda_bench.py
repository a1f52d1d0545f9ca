"""ORACLE / TEST INFRASTRUCTURE ONLY: the reference's CUDA renderer on this GPU.

Loads oracle/_ref/libwfref_cuda.so (the reference's own renderer sources
compiled for sm_100a by `make -C oracle cuda`; see ref_cuda_harness.cu) and
times it beside the B200 renderer on the same seeded scene, camera, depth,
RNG strategy and absolute sample ranges.  Both sides are timed the same way:
the wall time of one whole-frame task, which is the reference's
RenderTaskRenderer::render (clear, sample launches, synchronise, download)
against this renderer's wf_render + wf_framebuffer_download.  With caustics
(the large mesh's 2M photons), the reference builds its photon map with its
own kernels (emitPhotons / tracePhotons / buildPhotonGrid), with grid bounds
taken from the stored photons as this renderer takes them
(ref_cuda_harness.cu); its own driver would use fixed Cornell-box bounds.

Prints one JSON line: both throughputs in Mpaths/s and the relative RMSE
between the two renderers' images of the last task (the same paths; the two
builds differ only in floating-point contraction and elementary functions).

    python oracle/ref_cuda_bench.py --workload large_mesh --mode graph,persistent --steps 5
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
    lib.wfcuda_render.argtypes = [P, P, P, C.c_int, U32, U32, U32, P, P, P, P]
    return lib


def rel_rmse(image, reference):
    a = np.asarray(image, np.float64)
    b = np.asarray(reference, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-30))


def compare(workload=None, modes=("graph", "persistent"), steps=5, spp=0, own_mode=None, sample_start=1000,
            manifest=None, size="1280x720", caustics=True, own_fields=None):
    """Times the reference's CUDA renderer (each of `modes`) and this
    renderer on the same whole-frame tasks; returns the result dict."""
    import bench
    import wfpt
    from wfpt import native

    if manifest:
        from wfpt import assets
        width, height = (int(x) for x in size.split("x"))
        scene, cam = assets.preset_scene(manifest, width, height)
        rkw = {}
        workload = "preset " + Path(manifest).stem
    else:
        scene, cam, width, height, rkw = bench.make_scene(workload)
    if not caustics:
        for k in ("caustics", "photon_count"):
            rkw.pop(k, None)
    if rkw.get("caustics"):  # grid bounds derived from the stored photons on both sides
        rkw.setdefault("photon_grid_min", (0, 0, 0))
        rkw.setdefault("photon_grid_max", (0, 0, 0))
    spp = spp or bench.SPP_PER_STEP.get(workload, 1)
    own_mode = own_mode or bench.DEFAULT_MODE.get(workload, "graph")
    cfg = wfpt.render_config(width, height, **rkw)
    own_cfg = wfpt.render_config(width, height, mode=bench.MODES[own_mode], **rkw)
    if own_mode == "graph" and workload in bench.DEFAULT_WAVE:
        own_cfg.samples_per_wave = min(spp, bench.DEFAULT_WAVE[workload])
    for k, v in (own_fields or {}).items():  # e.g. the settings bench.py's autotuner chose
        setattr(own_cfg, k, v)
    cam_struct = native.camera_struct(cam)
    paths = width * height * spp

    # --- the reference's CUDA renderer, one scene for every mode
    lib = load()
    d, keep = scene.desc()
    env, rgba = scene.environment_struct()
    t0 = time.perf_counter()
    handle = lib.wfcuda_scene_create(C.addressof(d), C.addressof(env) if env is not None else None)
    ref_setup = time.perf_counter() - t0
    if not handle:
        raise SystemExit("reference scene creation failed")
    ref = {}
    ref_images = {}
    try:
        for mode in modes:
            ms = (C.c_double * steps)()
            img = np.zeros((height, width, 3), np.float32)
            photon_ms = C.c_double(0.0)
            counts = np.zeros(cfg.max_depth, np.uint32)
            rc = lib.wfcuda_render(handle, C.addressof(cam_struct), C.addressof(cfg), int(mode == "persistent"),
                                   sample_start, spp, steps, img.ctypes.data, ms, C.byref(photon_ms),
                                   counts.ctypes.data if mode == "persistent" else None)
            if rc != 0:
                raise SystemExit(f"reference render failed ({rc}) in {mode} mode")
            t = statistics.median(list(ms))
            ref[mode] = {"Mpaths/s": paths / t / 1e3, "ms_per_task": t, "ms_per_task_all": [round(x, 3) for x in ms],
                         "photon_map_ms": round(photon_ms.value, 2)}
            if mode == "persistent":
                # its --profile-queues record: per-bounce queue sizes of the last sample
                ref[mode]["extension_rays_last_sample"] = int(counts.sum())
            ref_images[mode] = img
    finally:
        lib.wfcuda_scene_destroy(handle)
    del keep, rgba

    # --- this renderer, same tasks, same timing
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, own_cfg)
    own_ms = []
    own_img = None
    r.stats(reset=True)
    for i in range(steps + 1):
        start = sample_start + i * spp
        if i == 1:
            r.stats(reset=True)
        t0 = time.perf_counter()
        img = r.render_task((0, 0, width, height), start, spp)
        t1 = time.perf_counter()
        if i:
            own_ms.append((t1 - t0) * 1e3)
        own_img = img
    stats = r.stats(reset=True)
    r.close()
    dev.close()
    own_t = statistics.median(own_ms)
    rays_per_task = (stats["extension_rays"] + stats["shadow_rays"]) / steps
    for mode in modes:
        ref[mode]["Mrays/s"] = rays_per_task / ref[mode]["ms_per_task"] / 1e3
        ref[mode]["speedup"] = ref[mode]["ms_per_task"] / own_t
        ref[mode]["image_relative_rmse"] = rel_rmse(own_img, ref_images[mode])
    return {
        "workload": workload, "triangles": int(scene.triangle_count()), "width": width, "height": height,
        "spp_per_task": spp, "max_depth": cfg.max_depth,
        "caustics": int(cfg.caustics), "photons": int(cfg.photon_count) if cfg.caustics else 0,
        "own_mode": own_mode, "own_samples_per_wave": max(1, own_cfg.samples_per_wave) if own_mode == "graph" else None,
        "reference_cuda": ref, "reference_scene_setup_s": round(ref_setup, 2),
        "b200_renderer": {"Mpaths/s": paths / own_t / 1e3, "Mrays/s": rays_per_task / own_t / 1e3,
                          "ms_per_task": own_t, "ms_per_task_all": [round(x, 3) for x in own_ms],
                          "extension_rays_per_task": stats["extension_rays"] / steps,
                          "shadow_rays_per_task": stats["shadow_rays"] / steps},
        "timing": "wall time per whole-frame task: render + download of the radiance (median)",
        "rays": "Mrays/s of both renderers count the same rays: this renderer's extension + shadow rays of the "
                "identical paths (the reference's persistent queue counts give its extension rays: "
                "extension_rays_last_sample)",
    }


def batch_sequential(job_count=64, seed=11):
    """The batch workload's jobs (wfpt.scenes.batch_jobs) rendered by the
    reference's CUDA renderer one after another, each as one task of its
    whole sample count through RenderTaskRenderer::render (after one untimed
    warm-up task): the "plain renderer once per job, sequentially" that
    batching replaces.  Scene creation is not timed."""
    import wfpt
    from wfpt import native, scenes
    lib = load()
    specs = scenes.batch_jobs(job_count, seed)
    total_ms, paths, setup_s = 0.0, 0, 0.0
    for j in specs:
        cfg = wfpt.render_config(j["width"], j["height"], max_depth=j["max_depth"])
        cam_struct = native.camera_struct(j["camera"])
        d, keep = j["scene"].desc()
        t0 = time.perf_counter()
        handle = lib.wfcuda_scene_create(C.addressof(d), None)
        setup_s += time.perf_counter() - t0
        del keep
        if not handle:
            raise SystemExit("reference scene creation failed")
        ms = (C.c_double * 1)()
        rc = lib.wfcuda_render(handle, C.addressof(cam_struct), C.addressof(cfg), 0, 0, j["spp"], 1, None, ms,
                               None, None)
        lib.wfcuda_scene_destroy(handle)
        if rc != 0:
            raise SystemExit(f"reference render failed ({rc})")
        total_ms += ms[0]
        paths += j["width"] * j["height"] * j["spp"]
    return {"jobs": len(specs), "seed": seed, "paths": paths, "ms": total_ms, "Mpaths/s": paths / total_ms / 1e3,
            "scene_setup_s": round(setup_s, 2),
            "timing": "sum over jobs of the wall time of one whole-job task: render + download of the radiance"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="large_mesh")
    ap.add_argument("--mode", default="graph,persistent", help="reference schedules, comma-separated")
    ap.add_argument("--spp", type=int, default=0, help="samples per task (default: bench.py's samples per step)")
    ap.add_argument("--own-mode", choices=("graph", "persistent", "stream"), default=None,
                    help="schedule of the B200 renderer (default: bench.py's schedule for the workload)")
    ap.add_argument("--steps", type=int, default=5, help="timed tasks (after one warm-up task)")
    ap.add_argument("--sample-start", type=int, default=1000)
    ap.add_argument("--no-caustics", action="store_true", help="turn the workload's photon caustics off on both sides")
    ap.add_argument("--manifest", default=None,
                    help="a scene manifest of the reference's presets, loaded by wfpt.assets, instead of a workload")
    ap.add_argument("--size", default="1280x720", help="image size for --manifest")
    ap.add_argument("--own-fields", default="{}",
                    help="JSON object of wf_render_config fields for the B200 renderer (e.g. the autotuned settings)")
    ap.add_argument("--batch-jobs", type=int, default=0,
                    help="render the batch workload's jobs one after another with the reference instead")
    args = ap.parse_args()
    if args.batch_jobs:
        print(json.dumps(batch_sequential(args.batch_jobs)), flush=True)
        return
    out = compare(args.workload, tuple(args.mode.split(",")), args.steps, args.spp, args.own_mode, args.sample_start,
                  args.manifest, args.size, caustics=not args.no_caustics, own_fields=json.loads(args.own_fields))
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
