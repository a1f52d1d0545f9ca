"""ORACLE / TEST INFRASTRUCTURE ONLY: converged reference images and the
"Mpaths/s at equal image RMSE" comparison.

The converged image of a configuration is rendered by the reference's own
CUDA renderer built for sm_100a (oracle/_ref/libwfref_cuda.so, see
ref_cuda_harness.cu): tasks of at most 64 samples through its
RenderTaskRenderer::render (src/renderer/render_task.cu:26-114), whose FP32
tile sums are accumulated in FP64 on the host (wfcuda_render_sum), over
65,536 samples per pixel by default.  Cases: the Cornell box's whole
256x256 frame, and fixed 32x32 crops of the full-size sphere field and large
mesh (their whole frames at 65,536 spp would take hours).

Against that image, both renderers -- this one through its task call and the
reference's -- render the same crop over the same absolute sample ranges
(disjoint from the oracle's) at 1, 4, 16, ... spp; the script reports each
one's relative RMSE (RMS error over the RMS of the oracle) and the samples
per pixel at which it reaches 1 %, fitted as RMSE = a / sqrt(spp) on the
larger sample counts.  Both trace the same paths, so the two columns agree
to the FP32 rounding of their arithmetic; the time to a given RMSE then
scales with each renderer's Mpaths/s.

    python oracle/converged_oracle.py --case large_mesh --out gpurun_out/converged
"""
import argparse
import ctypes as C
import json
import math
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "wavefront-path-tracer_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

ORACLE_BASE = 1 << 24   # absolute samples [ORACLE_BASE, ORACLE_BASE + spp) make the oracle
ESTIMATE_BASE = 1 << 26  # the estimates' sample ranges start here


def case_setup(case):
    """(scene, camera, render kwargs, width, height, tile) of a case."""
    import bench
    scene, cam, width, height, rkw = bench.make_scene(case)
    if rkw.get("caustics"):
        rkw.setdefault("photon_grid_min", (0, 0, 0))
        rkw.setdefault("photon_grid_max", (0, 0, 0))
    if case == "cornell":
        tile = (0, 0, width, height)
    else:
        tile = (width // 2 - 16, height // 2 - 16, 32, 32)
    return scene, cam, rkw, width, height, tile


class Reference:
    """The reference's CUDA renderer on one scene."""

    def __init__(self, scene):
        import ref_cuda_bench
        self.lib = ref_cuda_bench.load()
        self.lib.wfcuda_render_sum.restype = C.c_int
        self.lib.wfcuda_render_sum.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int] + [C.c_uint32] * 7 + \
            [C.c_void_p]
        d, keep = scene.desc()
        env, rgba = scene.environment_struct()
        self.handle = self.lib.wfcuda_scene_create(C.addressof(d), C.addressof(env) if env is not None else None)
        del keep, rgba
        if not self.handle:
            raise RuntimeError("reference scene creation failed")

    def mean(self, cam, cfg, tile, sample_start, spp, batch=64):
        """FP64 mean radiance of the tile over [sample_start, sample_start + spp)."""
        from wfpt import native
        x, y, w, h = tile
        total = np.zeros((h, w, 3), np.float64)
        cam_struct = native.camera_struct(cam)
        per = min(batch, spp)
        assert spp % per == 0
        rc = self.lib.wfcuda_render_sum(self.handle, C.addressof(cam_struct), C.addressof(cfg), 0, x, y, w, h,
                                        sample_start, per, spp // per, total.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"wfcuda_render_sum failed ({rc})")
        return total / spp

    def close(self):
        if self.handle:
            self.lib.wfcuda_scene_destroy(self.handle)
            self.handle = None


def own_mean(renderer, tile, sample_start, spp, batch=64):
    """FP64 mean of this renderer's FP32 task sums (tasks of <= batch spp)."""
    x, y, w, h = tile
    total = np.zeros((h, w, 3), np.float64)
    done = 0
    while done < spp:
        n = min(batch, spp - done)
        total += renderer.render_task(tile, sample_start + done, n)
        done += n
    return total / spp


def rel_rmse(image, oracle):
    return float(np.sqrt(np.mean((image - oracle) ** 2)) / np.sqrt(np.mean(oracle ** 2)))


def spp_for(rmse_by_spp, target=0.01):
    """Samples per pixel at which RMSE = a / sqrt(spp) reaches `target`, a
    fitted on the largest half of the measured sample counts."""
    pts = sorted(rmse_by_spp.items())
    pts = pts[len(pts) // 2:]
    a = float(np.exp(np.mean([math.log(r) + 0.5 * math.log(s) for s, r in pts])))
    return (a / target) ** 2, a


def run(case, oracle_spp=65536, levels=(1, 4, 16, 64, 256, 1024), out=None, reuse=True):
    import wfpt
    scene, cam, rkw, width, height, tile = case_setup(case)
    x, y, w, h = tile
    fields = dict(rkw)
    if (w, h) != (width, height):
        fields.update(tile_width=w, tile_height=h)  # queues sized for the crop on both sides
    cfg = wfpt.render_config(width, height, **fields)
    ref = Reference(scene)
    path = Path(out) / f"oracle_{case}_{oracle_spp}.npz" if out else None
    t0 = time.perf_counter()
    if path is not None and reuse and path.exists():
        oracle = np.load(path)["mean"]
        oracle_s = None
    else:
        oracle = ref.mean(cam, cfg, tile, ORACLE_BASE, oracle_spp)
        oracle_s = time.perf_counter() - t0
        if path is not None:
            path.parent.mkdir(parents=True, exist_ok=True)
            np.savez_compressed(path, mean=oracle, tile=np.array(tile), spp=oracle_spp, base=ORACLE_BASE)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    table = []
    own_rmse, ref_rmse = {}, {}
    start = ESTIMATE_BASE
    for spp in levels:
        mine = own_mean(r, tile, start, spp)
        theirs = ref.mean(cam, cfg, tile, start, spp)
        own_rmse[spp], ref_rmse[spp] = rel_rmse(mine, oracle), rel_rmse(theirs, oracle)
        table.append({"spp": spp, "sample_start": start, "this_renderer": own_rmse[spp],
                      "reference_cuda": ref_rmse[spp], "between_renderers": rel_rmse(mine, theirs)})
        start += spp
    r.close()
    dev.close()
    ref.close()
    own_spp, own_a = spp_for(own_rmse)
    ref_spp, ref_a = spp_for(ref_rmse)
    return {
        "case": case, "frame": [width, height], "tile": list(tile), "oracle_spp": oracle_spp,
        "oracle_sample_base": ORACLE_BASE, "oracle_seconds": oracle_s,
        "oracle_accumulation": "reference CUDA renderer task sums (<= 64 spp, FP32) accumulated in FP64",
        "caustics": int(cfg.caustics), "max_depth": int(cfg.max_depth),
        "rmse": table,
        "spp_to_1pct": {"this_renderer": own_spp, "reference_cuda": ref_spp},
        "rmse_at_1spp_fit": {"this_renderer": own_a, "reference_cuda": ref_a},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=("cornell", "sphere_field", "large_mesh"), default="cornell")
    ap.add_argument("--oracle-spp", type=int, default=65536)
    ap.add_argument("--levels", default="1,4,16,64,256,1024")
    ap.add_argument("--out", default=None, help="directory for the oracle image (npz), reused when present")
    args = ap.parse_args()
    res = run(args.case, args.oracle_spp, tuple(int(v) for v in args.levels.split(",")), args.out)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
