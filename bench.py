#!/usr/bin/env python3
"""Throughput benchmark of the B200 wavefront path tracer.

Workload (default): the large-mesh-with-lights configuration -- 1920x1080,
max depth 12, a 9,999,392-triangle fBm terrain (1% emissive, radiance
log-uniform in [1, 50]), 500 instances of a 200,000-triangle displaced
geodesic sphere, 20 glass spheres, a 2048x1024 HDR sun-and-sky environment
with MIS, and a 2M-photon caustic map.  Synthetic and seeded (no dataset).

One step = `spp` samples per pixel over the full frame (2,073,600 paths
per sample) through the streaming wavefront (one captured graph per step
whose device-side loop regenerates finished paths with their pixel's next
sample; --mode graph replays the reference's per-sample graph instead).  `value` = Mpaths/s over the timed
steps with the scene resident in HBM; `e2e` = the same metric through the
C-ABI task call (RenderTaskRenderer::render semantics: task in from the host,
unnormalized radiance sums back to pinned host memory every step).

--impl reference times the reference's own renderer code (host-compiled from
its sources, oracle/_ref) on the host cores for the same workload.
Multi-GPU (torchrun): every rank renders its own absolute sample range of the
same frame (weak scaling); the framebuffers are summed with one NCCL reduce
after the timed region.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "wavefront-path-tracer_b200"))
sys.path.insert(0, str(ROOT / "oracle"))  # the CPU baseline and the reference arms only

WORKLOADS = {
    # name: (scene kwargs, render kwargs)
    "large_mesh": (dict(width=1920, height=1080), dict(max_depth=12, caustics=1, photon_count=2_000_000)),
    "large_mesh_small": (dict(width=480, height=270, terrain_quads=256, instance_count=50, instance_frequency=30,
                              glass_spheres=6, env_size=(512, 256)),
                         dict(max_depth=12, caustics=1, photon_count=200_000)),
    # profiling-sized variant of large_mesh (about 1 GB on the device, still
    # larger than L2): 2.1M-triangle terrain, the same 500 instances
    "large_mesh_medium": (dict(width=960, height=540, terrain_quads=1024),
                          dict(max_depth=12, caustics=1, photon_count=500_000)),
    "sphere_field": (dict(width=1280, height=720), dict(max_depth=16)),
    "cornell": (dict(width=256, height=256), dict(max_depth=8, rr_start_depth=3)),
}
# Samples per pixel that one step renders (of the configs' 256 / 64 / 16):
# one step traces them as waves of several samples, whose long last bounces
# share one chain of launches.  The medium case stays at one sample per step
# for the ncu captures that index its launches.
SPP_PER_STEP = {"large_mesh": 16, "large_mesh_medium": 1, "large_mesh_small": 4, "sphere_field": 64, "cornell": 16}
# Schedule per workload when not autotuned: the per-wave graph, with this
# many samples per wave (wf_render_config.samples_per_wave).
DEFAULT_MODE = {"large_mesh": "graph", "large_mesh_medium": "graph", "large_mesh_small": "graph",
                "sphere_field": "graph", "cornell": "graph"}
DEFAULT_WAVE = {"large_mesh": 16, "large_mesh_medium": 1, "large_mesh_small": 4, "sphere_field": 64, "cornell": 16}
MODES = {"graph": 0, "persistent": 1, "stream": 2}
HBM_FALLBACK_GBS = 6650.0


def make_scene(name):
    from wfpt import scenes
    kw, rkw = WORKLOADS[name]
    if name.startswith("large_mesh"):
        scene, cam = scenes.large_mesh(**kw)
    elif name == "sphere_field":
        scene, cam = scenes.sphere_field(**kw)
    else:
        scene, cam = scenes.cornell_box(**kw)
    return scene, cam, kw["width"], kw["height"], dict(rkw)


def reference_cuda_comparison(workload, steps=5, own_mode=None, own_fields=None):
    """The reference's own CUDA renderer built for sm_100a
    (oracle/_ref/libwfref_cuda.so), in its graph and persistent schedules,
    and this renderer, timed the same way on the same whole-frame tasks in a
    child process after the timed region (oracle/ref_cuda_bench.py).  Both
    sides render the workload's caustics, each from its own photon map built
    with grid bounds taken from the stored photons.  A baseline beside the
    line, not part of `value`."""
    script = ROOT / "oracle" / "ref_cuda_bench.py"
    if not (ROOT / "oracle" / "_ref" / "libwfref_cuda.so").exists():
        return {"unavailable": "reference CUDA build absent (make -C oracle cuda)"}
    cmd = [sys.executable, str(script), "--workload", workload, "--mode", "graph,persistent", "--steps", str(steps)]
    if own_mode:
        cmd += ["--own-mode", own_mode]
    if own_fields:
        cmd += ["--own-fields", json.dumps(own_fields)]
    run = subprocess.run(cmd, capture_output=True, text=True, timeout=1200, cwd=ROOT)
    if run.returncode != 0:
        return {"failed": (run.stdout + run.stderr)[-400:]}
    return json.loads(run.stdout.strip().splitlines()[-1])


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(profile, kernel):
    """Algorithmic bytes of one kernel's launches in the profiled pass.
    Per ray state: 32 B ray in + 16 B hit/result out.  Traversal: 32 B per
    node visit (one pair of child boxes), 48 B per triangle test, 16 B per
    sphere test, 64 B per instance entry."""
    if kernel == "trace":
        rays, nodes, tris, sph, inst = (profile["extension_rays"], profile["closest_nodes"],
                                        profile["closest_triangles"], profile["closest_spheres"],
                                        profile["closest_instances"])
    else:
        rays, nodes, tris, sph, inst = (profile["shadow_rays"], profile["any_nodes"], profile["any_triangles"],
                                        profile["any_spheres"], profile["any_instances"])
    return 48 * rays + 32 * nodes + 48 * tris + 16 * sph + 64 * inst


def ncu_summary(kernel, workload):
    """The committed ncu summary of `kernel` on `workload` (profiles/), or {}."""
    p = ROOT / "profiles" / f"{kernel}_{workload}.json"
    return json.loads(p.read_text()) if p.exists() else {}


def dram_traffic(kernel, workload, rays_per_launch):
    """DRAM bytes of one launch: the ncu summary's DRAM bytes per ray
    (dram__bytes_read + write of a captured launch over its rays) scaled to
    this launch's rays, or None."""
    per_ray = ncu_summary(kernel, workload).get("dram_bytes_per_ray")
    return per_ray * rays_per_launch if per_ray and rays_per_launch else None


def l2_term(kernel, workload, rays_per_launch, avg_ms):
    """L2 traffic of one launch from the ncu summary's L2 bytes per ray
    (lts__t_bytes of a captured launch over its rays), scaled to this
    launch's rays and divided by its live CUDA-event time."""
    data = ncu_summary(kernel, workload)
    per_ray = data.get("l2_bytes_per_ray")
    if not per_ray or not rays_per_launch:
        return None
    b = per_ray * rays_per_launch
    return {"bytes_per_launch": b, "achieved_gbs": b / (avg_ms / 1e3) / 1e9,
            "ncu_l2_throughput_pct_of_peak": data.get("l2_throughput_pct"),
            "ncu_l2_hit_rate_pct": data.get("l2_hit_rate_pct"), "source": data.get("l2_source")}


def cpu_reference_rate(ref, cam, width, height, render_kwargs, seconds_target=15.0, threads=0):
    """Mpaths/s of the host-compiled reference (an oracle.RefScene) on a band
    of rows at 1 spp, sized to about `seconds_target` seconds."""
    import oracle
    cfg = oracle.reference_config(width, height, **render_kwargs)
    cores = threads or os.cpu_count() or 1
    # One untimed row first: builds the reference's photon map once (it is
    # built in RenderDriver::prepare, outside the trace timing).
    ref.render(cam, cfg, tile=(0, height // 2, width, 1), sample_start=0, sample_count=1, threads=cores)
    band = max(1, height // 64)
    y0 = height // 2 - band // 2
    t0 = time.perf_counter()
    ref.render(cam, cfg, tile=(0, y0, width, band), sample_start=0, sample_count=1, threads=cores)
    dt = time.perf_counter() - t0
    if dt < seconds_target / 4:
        band = min(height, max(band + 1, int(band * seconds_target / max(dt, 1e-3))))
        y0 = max(0, height // 2 - band // 2)
        t0 = time.perf_counter()
        ref.render(cam, cfg, tile=(0, y0, width, band), sample_start=0, sample_count=1, threads=cores)
        dt = time.perf_counter() - t0
    return width * band / dt / 1e6, cores, f"{width}x{band} rows at 1 spp (a band of one sample pass)", dt


def time_frame_guides(dev_scene, cam, width, height, launches=10):
    """wf_frame_guides over the whole frame with a previous camera 1 % of the
    view's width to the side: the denoiser guides of the dataset capture.
    Device time per launch (CUDA events on the launching stream, 3 warm-up
    launches) and the fraction of pixels with a valid history."""
    import ctypes
    import numpy as np
    import torch
    import wfpt
    lib = wfpt.library()
    prev = dict(cam)
    prev["position"] = (np.asarray(cam["position"], np.float32)
                        + 0.01 * np.asarray(cam["right"], np.float32)).tolist()
    c, p = wfpt.camera_struct(cam), wfpt.camera_struct(prev)
    out = torch.empty(width * height * wfpt.abi.FRAME_GUIDE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def call():
        wfpt.check(lib.wf_frame_guides(dev_scene.handle, ctypes.byref(c), ctypes.byref(p), width, height, 0, 0,
                                       width, height, out.data_ptr(), stream.cuda_stream))
    for _ in range(3):
        call()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(launches):
        call()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / launches
    g = out.cpu().numpy().view(wfpt.abi.FRAME_GUIDE_DTYPE)
    # a valid pixel that projects into the previous frame traces a second ray
    second = float((g["valid"] * (np.abs(g["motion"]).sum(axis=1) > 0)).mean())
    return {"ms_per_frame": round(ms, 3), "mpixels_per_s": round(width * height / ms / 1e3, 1),
            "valid_fraction": round(float(g["valid"].mean()), 4),
            "history_valid_fraction": round(float(g["history_valid"].mean()), 4),
            "traversals_per_pixel_at_least": round(1.0 + second, 3), "launches": launches + 3}


def reference_scene(scene):
    import oracle
    return oracle.RefScene(scene)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    scene, cam, width, height, rkw = make_scene(args.workload)
    # photon map is part of the reference render path when caustics are on
    rkw = dict(rkw)
    rkw.setdefault("photon_grid_min", (0, 0, 0))
    rkw.setdefault("photon_grid_max", (0, 0, 0))
    rates = []
    cores = os.cpu_count() or 1
    sample_desc = ""
    ref = reference_scene(scene)
    # every step renders a band of rows sized so the whole run stays near 90 s
    per_step = max(1.0, min(args.cpu_seconds, 90.0 / max(1, args.warmup + args.steps)))
    for step in range(args.warmup + args.steps):
        rate, cores, sample_desc, _ = cpu_reference_rate(ref, cam, width, height, rkw, seconds_target=per_step)
        if step >= args.warmup:
            rates.append(rate)
    value = statistics.median(rates)
    line = {"metric": "Mpaths/s", "value": value, "unit": "Mpaths/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": width * height / (value * 1e6) * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": {"workload": args.workload, "width": width, "height": height,
                       "spp_per_step": args.spp or SPP_PER_STEP.get(args.workload, 1),
                       "max_depth": rkw.get("max_depth"), "rr_start_depth": rkw.get("rr_start_depth", 12),
                       "triangles": int(scene.triangle_count()), "instances": int(len(scene.instances)),
                       "photons": int(rkw.get("photon_count", 0)) if rkw.get("caustics") else 0,
                       "mode": "host-compiled reference (captured-graph chain on host threads)",
                       "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": cores, "kind": "reference",
                             "sample": sample_desc},
            "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_inverse(args):
    """Inverse-rendering step on the subdivided Cornell box (10,240 wall
    triangles, each with RGB albedo and Oren-Nayar roughness, plus boxes and
    the light's emission scale): 512x512, 32 spp, depth 6, L2 image loss.
    One step = forward render + path-replay adjoint.  Reports the adjoint /
    forward time ratio and the peak device memory of the step."""
    import numpy as np
    import torch
    import wfpt
    from wfpt import diff, scenes

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if int(os.environ.get("RANK", "0")) != 0:
        return 0  # one GPU: the parameters are shared by every path
    width = height = 512
    spp, depth = 32, 6
    t0 = time.perf_counter()
    scene, cam, n, _ = scenes.cornell_inverse(width, height, cells=32)
    gt_a, gt_r = scenes.inverse_parameters(scene, n, seed=101)
    a0, r0 = scenes.inverse_parameters(scene, n, seed=202)
    dev = wfpt.DeviceScene(scene)
    cfg = diff.diff_config(width, height, spp, depth, n)
    A = torch.from_numpy(a0).cuda()
    R = torch.from_numpy(r0).cuda()
    target = diff.forward(dev, cam, cfg, torch.from_numpy(gt_a).cuda(), torch.from_numpy(gt_r).cuda(), 1.0)
    setup_s = time.perf_counter() - t0
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    for _ in range(args.warmup):
        img = diff.forward(dev, cam, cfg, A, R, 1.1)
        diff.backward(dev, cam, cfg, A, R, 1.1, 2.0 * (img - target))
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    free0, total = torch.cuda.mem_get_info()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    f_ms = b_ms = 0.0
    for _ in range(args.steps):
        a, b, c = ev(), ev(), ev()
        a.record()
        img = diff.forward(dev, cam, cfg, A, R, 1.1)
        b.record()
        ga, gr, gs = diff.backward(dev, cam, cfg, A, R, 1.1, 2.0 * (img - target))
        c.record()
        torch.cuda.synchronize()
        f_ms += a.elapsed_time(b)
        b_ms += b.elapsed_time(c)
    clock_record = clocks.stop()
    peak_torch = torch.cuda.max_memory_allocated()
    info = dev.info()
    f_ms /= args.steps
    b_ms /= args.steps
    loss = float(((img.double() - target.double()) ** 2).sum())
    paths = width * height * spp
    line = {
        "metric": "adjoint/forward time", "value": b_ms / f_ms, "unit": "ratio", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": f_ms + b_ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (gradients f64)", "data": "synthetic (seeded generator)",
        "config": {"workload": "inverse", "width": width, "height": height, "spp": spp, "max_depth": depth,
                   "triangles": n, "parameters": 4 * n + 1, "wall_triangles": 10240,
                   "l2": "scene, parameters and images stay on the device; no flush"},
        "forward_ms": f_ms, "adjoint_ms": b_ms,
        "forward_mpaths_s": paths / (f_ms / 1e3) / 1e6,
        "peak_device_bytes": {"torch_tensors": int(peak_torch), "scene": int(info.device_bytes),
                              "note": "the adjoint stores no paths: images, parameters and gradients only"},
        "loss": loss,
        "e2e": None, "gpu_launches": 2 * args.steps, "roofline": None, "clocks": clock_record,
        "setup_seconds": setup_s,
    }
    print(json.dumps(line), flush=True)
    dev.close()
    return 0


def run_batch(args):
    """Uneven jobs (64 sphere-field jobs from seed 11: 5k-2M triangles,
    64^2-512^2 pixels, 4/16/64 spp, depth 8) rendered as one batch graph,
    against the same jobs rendered one after another by per-job renderers
    (graph mode, the reference's schedule) on the same GPU.  One step renders
    every job's full sample count once.  Multi-GPU: jobs are assigned to
    ranks longest-first by estimated cost; every rank renders its share."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import wfpt
    from wfpt import scenes, shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    t0 = time.perf_counter()
    specs = scenes.batch_jobs(args.batch_jobs, 11)
    costs = [j["width"] * j["height"] * j["spp"] * math.log2(max(j["triangles"], 2)) for j in specs]
    owner = shard.lpt_assign(costs, world)
    mine = [j for j, r in zip(specs, owner) if r == rank]
    stream = torch.cuda.Stream()
    jobs = []
    for j in mine:
        cfg = wfpt.render_config(j["width"], j["height"], max_depth=j["max_depth"])
        jobs.append(dict(scene=wfpt.DeviceScene(j["scene"]), camera=j["camera"], config=cfg, sample_start=0,
                         sample_count=j["spp"]))
    setup_s = time.perf_counter() - t0
    paths = sum(j["config"].width * j["config"].height * j["sample_count"] for j in jobs)
    total_paths = sum(j["width"] * j["height"] * j["spp"] for j in specs)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(ms):
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return ms

    tune = None
    if not args.autotune:
        batch = wfpt.Batch(jobs, stream=stream.cuda_stream)
    else:
        best, times = wfpt.Batch.autotune(jobs, slot_capacities=(4 << 20, 8 << 20, 16 << 20), block_sizes=(128, 256),
                                          refill_thresholds=(8,), stream=stream.cuda_stream)
        tune = {"candidates_ms": [round(t, 3) for t in times], "slot_capacity": best.slot_capacity,
                "block_size": best.block_size, "refill_threshold": best.refill_threshold}
        batch = wfpt.Batch(jobs, stream=stream.cuda_stream, config=best)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    for _ in range(args.warmup):
        batch.run()
    batch.synchronize()
    batch.stats(reset=True)
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    a, b = ev(), ev()
    a.record(stream)
    for _ in range(args.steps):
        batch.run()
    b.record(stream)
    torch.cuda.synchronize()
    barrier()
    clock_record = clocks.stop()
    batch.synchronize()
    ms = max_over_ranks(a.elapsed_time(b))
    stats = batch.stats(reset=True)
    value = total_paths * args.steps / (ms / 1e3) / 1e6

    # End to end: every step also reads every job framebuffer back to pinned host memory.
    hosts = [torch.empty((j["config"].height, j["config"].width, 3), dtype=torch.float32, pin_memory=True)
             for j in jobs]
    lib = wfpt.library()
    barrier()
    torch.cuda.synchronize()
    a, b = ev(), ev()
    a.record(stream)
    for _ in range(args.steps):
        wfpt.check(lib.wf_batch_reset(batch.handle))
        batch.run()
        for k, h in enumerate(hosts):
            wfpt.check(lib.wf_batch_download(batch.handle, k, h.data_ptr()))
    b.record(stream)
    torch.cuda.synchronize()
    e_ms = max_over_ranks(a.elapsed_time(b))
    e2e = total_paths * args.steps / (e_ms / 1e3) / 1e6

    # Sequential baseline: one per-job renderer each, rendered one after
    # another, each tracing its samples in waves (up to 16 per wave).
    seq_configs = []
    for j in jobs:
        c = wfpt.abi.RenderConfig.from_buffer_copy(bytes(j["config"]))
        c.samples_per_wave = min(j["sample_count"], args.sequential_wave)
        seq_configs.append(c)
    renderers = [wfpt.Renderer(j["scene"], j["camera"], c, stream=stream.cuda_stream)
                 for j, c in zip(jobs, seq_configs)]
    for r, j in zip(renderers, jobs):
        r.render(0, 0, j["config"].width, j["config"].height, 0, j["sample_count"], True)
    torch.cuda.synchronize()
    barrier()
    a, b = ev(), ev()
    a.record(stream)
    for _ in range(args.steps):
        for r, j in zip(renderers, jobs):
            r.render(0, 0, j["config"].width, j["config"].height, 0, j["sample_count"], True)
    b.record(stream)
    torch.cuda.synchronize()
    s_ms = max_over_ranks(a.elapsed_time(b))
    sequential = total_paths * args.steps / (s_ms / 1e3) / 1e6
    # parity spot check: the batch's last run equals the per-job renders
    mismatched = sum(int(not np.array_equal(batch.download(k).view(np.uint32), r.download().view(np.uint32)))
                     for k, r in enumerate(renderers))
    for r in renderers:
        r.close()
    batch.close()
    reference_sequential = None
    if rank == 0 and world == 1 and args.reference_cuda:
        # the reference's CUDA renderer, one job after another (after the timed regions)
        if (ROOT / "oracle" / "_ref" / "libwfref_cuda.so").exists():
            run = subprocess.run([sys.executable, str(ROOT / "oracle" / "ref_cuda_bench.py"), "--batch-jobs",
                                  str(args.batch_jobs)], capture_output=True, text=True, timeout=1800, cwd=ROOT)
            reference_sequential = (json.loads(run.stdout.strip().splitlines()[-1]) if run.returncode == 0
                                    else {"failed": (run.stdout + run.stderr)[-400:]})
        else:
            reference_sequential = {"unavailable": "reference CUDA build absent (make -C oracle cuda)"}
    if rank == 0:
        line = {
            "metric": "Mpaths/s", "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": {"workload": "batch", "jobs": len(specs), "seed": 11, "paths_per_step": total_paths,
                       "pixels": sum(j["width"] * j["height"] for j in specs),
                       "triangles": sum(j["triangles"] for j in specs), "max_depth": 8,
                       "parallelism": f"jobs x{world} (longest first)",
                       "l2": "inputs larger than L2 (64 scenes on the device); no flush"},
            "e2e": {"value": e2e, "unit": "Mpaths/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": sum(h.numel() * 4 for h in hosts)},
            "sequential": {"value": sequential, "unit": "Mpaths/s", "ms_per_step": s_ms / args.steps,
                           "how": "one graph-mode renderer per job, rendered one after another, "
                                  f"in waves of up to {args.sequential_wave} samples"},
            "speedup_vs_sequential": value / sequential,
            "reference_cuda_sequential": reference_sequential,
            "e2e_speedup_vs_reference_sequential": (e2e / reference_sequential["Mpaths/s"]
                                                    if reference_sequential and "Mpaths/s" in reference_sequential
                                                    else None),
            "parity_mismatched_jobs": mismatched,
            "autotune": tune,
            "gpu_launches": int(stats["kernel_launches"]),
            "roofline": None,
            "clocks": clock_record,
            "setup_seconds": setup_s,
        }
        print(json.dumps(line), flush=True)
    for j in jobs:
        j["scene"].close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="large_mesh", choices=sorted(WORKLOADS) + ["batch", "inverse"])
    ap.add_argument("--batch-jobs", type=int, default=64, help="batch workload: number of jobs")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--mode", default=None, choices=sorted(MODES), help="default: per workload")
    ap.add_argument("--spp", type=int, default=0, help="samples per pixel per step (default: per workload)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="scene workloads: skip wf_renderer_autotune and render with the given or default settings "
                         "(batch workload: skip the batch tuner)")
    ap.add_argument("--build", default="exact", choices=["exact", "fast"],
                    help="exact: the bit-exact library (default); fast: multiply-adds contracted and CUDA's own "
                         "elementary functions (make -C wavefront-path-tracer_b200 fast)")
    ap.add_argument("--persistent-kernel", default="auto", choices=["auto", "fused", "staged"],
                    help="persistent mode: the fused per-path kernel, the staged kernel, or by tile size (default)")
    ap.add_argument("--sequential-wave", type=int, default=16,
                    help="batch workload: samples per wave of the per-job sequential baseline")
    ap.add_argument("--samples-per-wave", type=int, default=0,
                    help="graph mode: samples of every pixel traced by one launch of the bounce chain "
                         "(wf_render_config.samples_per_wave; 0 = per workload)")
    ap.add_argument("--regenerate-percent", type=int, default=0,
                    help="streaming mode: share of idle slots (%%) at which waiting slots start their next "
                         "samples together (0 = the renderer's default)")
    ap.add_argument("--concurrent-tiles", type=int, default=0,
                    help="graph mode: 1 = one wavefront, 2 = two on two streams (default)")
    ap.add_argument("--bvh-builder", default="host", choices=["host", "gpu"],
                    help="BVH2 builder of the scene: host binned SAH (default) or GPU PLOC")
    ap.add_argument("--no-reference-cuda", dest="reference_cuda", action="store_false",
                    help="skip timing the reference's own CUDA renderer built for sm_100a (make -C oracle cuda) "
                         "beside this one after the timed region (the `reference_cuda` object of the line)")
    args = ap.parse_args()
    if args.build == "fast":
        os.environ["WF_BUILD"] = "fast"  # read when wfpt loads the library
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "inverse":
        return run_inverse(args)

    import numpy as np
    import torch
    import torch.distributed as dist
    import wfpt

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    t_setup = time.perf_counter()
    scene, cam, width, height, rkw = make_scene(args.workload)
    if rkw.get("caustics"):
        rkw.setdefault("photon_grid_min", (0, 0, 0))  # min == max: grid bounds derived from the photons
        rkw.setdefault("photon_grid_max", (0, 0, 0))
    stream = torch.cuda.Stream()
    scene.bvh_builder = wfpt.abi.BVH_GPU_PLOC if args.bvh_builder == "gpu" else wfpt.abi.BVH_HOST_SAH
    dev_scene = wfpt.DeviceScene(scene)
    scene_info = dev_scene.info()
    mode_given = args.mode is not None
    args.mode = args.mode or DEFAULT_MODE[args.workload]
    stages = {"auto": wfpt.abi.PERSISTENT_AUTO, "fused": wfpt.abi.PERSISTENT_FUSED,
              "staged": wfpt.abi.PERSISTENT_STAGED}[args.persistent_kernel]
    spp = args.spp or SPP_PER_STEP[args.workload]
    wave = args.samples_per_wave or min(spp, DEFAULT_WAVE[args.workload])
    cfg = wfpt.render_config(width, height, mode=MODES[args.mode], concurrent_tiles=args.concurrent_tiles,
                             regenerate_percent=args.regenerate_percent, persistent_stages=stages,
                             samples_per_wave=wave, **rkw)
    tune = None
    if args.autotune:
        # wf_renderer_autotune: one timed frame of `spp` samples per candidate
        # (schedule, CTA size, refill threshold and the schedule's own
        # settings); options given on the command line stay fixed
        modes = (MODES[args.mode],) if mode_given else (MODES["graph"], MODES["stream"])
        waves = (args.samples_per_wave,) if args.samples_per_wave else tuple(sorted({1, max(1, wave // 2), wave}))
        t_tune = time.perf_counter()
        best, table = wfpt.autotune(
            dev_scene, cam, cfg, modes=modes, block_sizes=(128, 256), refill_thresholds=(8, 16),
            concurrent_tiles=(args.concurrent_tiles,) if args.concurrent_tiles else (1, 2),
            regenerate_percents=(args.regenerate_percent,) if args.regenerate_percent else (10, 25),
            samples_per_waves=waves, samples=spp, stream=stream.cuda_stream,
            key=f"{args.workload}/{spp}/{args.build}/{modes}/{waves}")
        cfg = best
        args.mode = {v: k for k, v in MODES.items()}[cfg.mode]
        args.concurrent_tiles = cfg.concurrent_tiles
        tune = {"seconds": round(time.perf_counter() - t_tune, 2), "candidates": len(table),
                "chosen": {"mode": args.mode, "block_size": cfg.block_size, "refill_threshold": cfg.refill_threshold,
                           "concurrent_tiles": cfg.concurrent_tiles, "regenerate_percent": cfg.regenerate_percent,
                           "samples_per_wave": cfg.samples_per_wave},
                "frame_ms": [dict(c, ms=None if ms is None else round(ms, 3)) for c, ms in table]}
    renderer = wfpt.Renderer(dev_scene, cam, cfg, stream=stream.cuda_stream)
    setup_s = time.perf_counter() - t_setup
    scene_bytes = dev_scene.info().device_bytes
    # path state (6 x 16 B), queues, hit records, terms and shadow requests per slot
    slots = width * height * (max(1, cfg.samples_per_wave) if args.mode == "graph" else 1)
    renderer_bytes = slots * (96 + 8 + 20 + 16 * 8 + 16 + 5 * 33) + width * height * 12
    pixels = width * height
    # Each rank owns its own absolute sample range (weak scaling).
    from wfpt import shard
    base = shard.rank_sample_base(rank)

    def barrier():
        if world > 1:
            dist.barrier()

    renderer.set_sample_index(base)
    for _ in range(args.warmup):
        renderer.render_frame(spp)
    renderer.synchronize()
    renderer.stats(reset=True)
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        renderer.render_frame(spp)
    end.record(stream)
    torch.cuda.synchronize()
    barrier()
    clock_record = clocks.stop()
    ms = start.elapsed_time(end)
    stats = renderer.stats(reset=True)
    renderer.synchronize()
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    seconds = ms / 1e3
    value = world * pixels * spp * args.steps / seconds / 1e6
    mrays = (stats["extension_rays"] + stats["shadow_rays"]) / seconds / 1e6

    # End to end through the C-ABI task call with host buffers: every step
    # renders its sample range and copies the frame's sums into pinned host
    # memory; the copy of step i crosses PCIe while step i + 1 renders
    # (wf_framebuffer_download_async), and the timed region ends when the
    # last copy has arrived.
    hosts = [torch.empty((height, width, 3), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    lib = wfpt.library()
    renderer.render_task((0, 0, width, height), base + 999_000, spp)
    wfpt.check(lib.wf_framebuffer_download_async(renderer.handle, 0, 0, width, height, hosts[0].data_ptr()))
    wfpt.check(lib.wf_framebuffer_download_wait(renderer.handle))
    barrier()
    torch.cuda.synchronize()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for i in range(args.steps):
        wfpt.check(lib.wf_render(renderer.handle, 0, 0, width, height, base + 1000 + i * spp, spp, 1))
        wfpt.check(lib.wf_framebuffer_download_async(renderer.handle, 0, 0, width, height,
                                                     hosts[i % 2].data_ptr()))
    wfpt.check(lib.wf_framebuffer_download_wait(renderer.handle))
    e_end.record(stream)
    torch.cuda.synchronize()
    e_ms = e_start.elapsed_time(e_end)
    if world > 1:
        t = torch.tensor([e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e_ms = float(t.item())
    e2e_value = world * pixels * spp * args.steps / (e_ms / 1e3) / 1e6

    # Kernel-level roofline from one profiled pass (event-timed eager launches).
    renderer.profile_sample()  # first use of the per-stage kernels the graph never launches (module loading)
    profile = renderer.profile_sample()
    kernels = {k: v for k, v in profile.items() if isinstance(v, dict) and v["launches"]}
    total_ms = sum(v["ms"] for v in kernels.values())
    if "trace" in kernels or "shadow" in kernels:
        dominant = max(("trace", "shadow"), key=lambda k: kernels.get(k, {"ms": 0})["ms"])
        launches = kernels[dominant]["launches"]
        avg_ms = kernels[dominant]["ms"] / launches
        bytes_per_launch = algorithmic_bytes(profile, dominant) / launches
        peak, peak_kind = measured_peak()
        achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9
        rays_key = "extension_rays" if dominant == "trace" else "shadow_rays"
        roofline = {"bound": "hbm", "kernel": f"k_{dominant}", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_kind,
                    "traffic": dram_traffic(f"k_{dominant}", args.workload, profile[rays_key] / launches),
                    "l2": l2_term(f"k_{dominant}", args.workload, profile[rays_key] / launches, avg_ms),
                    "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_ms": avg_ms,
                    "kernel_share": {k: v["ms"] / total_ms for k, v in kernels.items()}}
    else:
        # the persistent schedule fuses every stage into one kernel that
        # keeps no traversal tallies: no per-kernel roofline
        roofline = {"bound": "hbm", "kernel": "k_persistent", "achieved": None, "peak": measured_peak()[0],
                    "unit": "GB/s", "frac": None, "traffic": None,
                    "note": "fused persistent kernel; traversal tallies are kept only by the wavefront kernels",
                    "kernel_share": {k: v["ms"] / total_ms for k, v in kernels.items()}}

    # Multi-GPU merge: one NCCL reduce of the framebuffers to rank 0.
    if world > 1:
        fb = torch.from_numpy(renderer.download()).cuda()
        shard.reduce_framebuffer(fb, dst=0)
        if rank == 0:
            assert torch.isfinite(fb).all()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            ref = reference_scene(scene)
            rate, cores, sample, _ = cpu_reference_rate(ref, cam, width, height, rkw,
                                                        seconds_target=args.cpu_seconds)
            ref.close()
            cpu = {"value": rate, "unit": "Mpaths/s", "cores": cores, "kind": "reference", "sample": sample}
        except FileNotFoundError as e:
            cpu = {"value": None, "unit": "Mpaths/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    reference_cuda = None
    if rank == 0 and world == 1 and args.reference_cuda:
        own = {k: getattr(cfg, k) for k in ("block_size", "refill_threshold", "concurrent_tiles",
                                            "regenerate_percent", "samples_per_wave", "persistent_stages")}
        reference_cuda = reference_cuda_comparison(args.workload, own_mode=args.mode, own_fields=own)
    guides = time_frame_guides(dev_scene, cam, width, height) if rank == 0 else None

    if rank == 0:
        line = {
            "metric": "Mpaths/s", "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": {"workload": args.workload, "width": width, "height": height, "spp_per_step": spp,
                       "max_depth": cfg.max_depth, "rr_start_depth": cfg.rr_start_depth,
                       "triangles": int(scene.triangle_count()), "instances": int(len(scene.instances)),
                       "photons": int(cfg.photon_count) if cfg.caustics else 0, "mode": args.mode,
                       "regenerate_percent": (cfg.regenerate_percent or None) if args.mode == "stream" else None,
                       "persistent_kernel": args.persistent_kernel if args.mode == "persistent" else None,
                       "samples_per_wave": max(1, cfg.samples_per_wave) if args.mode != "stream" else None,
                       "build": args.build,
                       "wavefronts": 1 if args.mode != "graph" or args.concurrent_tiles == 1 else 2,
                       "block_size": cfg.block_size or 128, "refill_threshold": cfg.refill_threshold or 8,
                       "scene_device_bytes": int(scene_bytes),
                       "bvh_builder": args.bvh_builder, "bvh_build_ms": round(float(scene_info.bvh_build_ms), 1),
                       "gpu_bvh_builds": int(scene_info.gpu_bvh_builds),
                       "l2": ("inputs larger than L2 (scene + path state on the device: "
                              f"{(scene_bytes + renderer_bytes) / 1e6:.0f} MB, no flush)"
                              if scene_bytes + renderer_bytes > 126e6 else
                              "working set fits in the 126 MB L2; no flush between steps"),
                       "parallelism": f"sample-range x{world}"},
            "mrays_per_s": mrays,
            "rays_per_step": (stats["extension_rays"] + stats["shadow_rays"]) / args.steps,
            "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": 24,
                    "d2h_bytes_per_step": pixels * 12},
            "gpu_launches": int(stats["kernel_launches"]),
            "roofline": roofline,
            "profile_pass": {k: (v if not isinstance(v, dict) else v) for k, v in profile.items()},
            "cpu_baseline": cpu,
            "clocks": clock_record,
            "setup_seconds": setup_s,
            "autotune": tune,
        }
        line["frame_guides"] = guides  # measured after the timed region
        if reference_cuda is not None:
            line["reference_cuda"] = reference_cuda
        print(json.dumps(line), flush=True)
    renderer.close()
    dev_scene.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
