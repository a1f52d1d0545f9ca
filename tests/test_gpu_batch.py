"""Job batch (wf_batch_*): uneven jobs in one captured graph.

Each job's framebuffer must equal a per-job render of the same sample range
bit for bit (each pixel adds its samples in order after the pass that traced
them), with any slot capacity, including one far below the batch's path
count, so that slots work through many (job, sample, pixel) units one after
another, and with passes that split jobs' sample ranges."""
import numpy as np
import pytest

import wfpt
from wfpt import abi, scenes

pytestmark = pytest.mark.gpu


def _jobs():
    """Six uneven jobs: Cornell, sphere fields of two mesh sizes, a reduced
    large mesh (lights, HDR environment, instances, glass), different
    resolutions, depths, RNG strategies and sample ranges."""
    specs = [
        (scenes.cornell_box(48, 40), (48, 40), dict(max_depth=8, rr_start_depth=3), 11, 5),
        (scenes.sphere_field(64, 36, frequency=12, seed=3), (64, 36), dict(max_depth=6), 0, 3),
        (scenes.sphere_field(24, 16, frequency=40, seed=9), (24, 16), dict(max_depth=16, rng=abi.RNG_PCG32), 1000, 7),
        (scenes.large_mesh(40, 24, terrain_quads=48, instance_count=8, instance_frequency=6, glass_spheres=2,
                           env_size=(128, 64)), (40, 24), dict(max_depth=12), 5, 2),
        (scenes.cornell_box(16, 16), (16, 16), dict(max_depth=4, rr_start_depth=2, indirect_clamp=0.5), 77, 1),
        (scenes.sphere_field(32, 32, frequency=8, seed=21), (32, 32), dict(max_depth=8, rr_start_depth=1), 3, 9),
    ]
    jobs = []
    for (scene, cam), (w, h), fields, start, count in specs:
        jobs.append(dict(scene=wfpt.DeviceScene(scene), camera=cam, config=wfpt.render_config(w, h, **fields),
                         sample_start=start, sample_count=count))
    return jobs


def _per_job(job):
    cfg = job["config"]
    r = wfpt.Renderer(job["scene"], job["camera"], cfg)
    try:
        return r.render_task((0, 0, cfg.width, cfg.height), job["sample_start"], job["sample_count"]), r.stats()
    finally:
        r.close()


@pytest.mark.parametrize("capacity,pass_paths", [(0, 0), (700, 0), (0, 5003), (300, 1024)])
def test_batch_matches_per_job_renders(cuda, capacity, pass_paths):
    jobs = _jobs()
    want = [_per_job(j) for j in jobs]
    batch = wfpt.Batch(jobs, slot_capacity=capacity, pass_paths=pass_paths)
    try:
        for run in range(2):
            batch.reset()
            batch.run()
            batch.synchronize()
            for k, (image, _) in enumerate(want):
                got = batch.download(k)
                diff = np.count_nonzero(got.view(np.uint32) != image.view(np.uint32))
                assert diff == 0, f"job {k} run {run}: {diff} channels differ"
        stats = batch.stats()
        paths = sum(j["config"].width * j["config"].height * j["sample_count"] for j in jobs)
        assert stats["paths"] == 2 * paths
        assert stats["extension_rays"] == 2 * sum(s["extension_rays"] for _, s in want)
        assert stats["shadow_rays"] == 2 * sum(s["shadow_rays"] for _, s in want)
    finally:
        batch.close()
        for j in jobs:
            j["scene"].close()


def test_batch_rejects_caustics_and_autotunes(cuda):
    scene, cam = scenes.cornell_box(32, 32)
    dev = wfpt.DeviceScene(scene)
    try:
        bad = [dict(scene=dev, camera=cam, sample_count=1,
                    config=wfpt.render_config(32, 32, max_depth=4, caustics=1, photon_count=100))]
        with pytest.raises(wfpt.WavefrontError, match="caustics"):
            wfpt.Batch(bad)
        jobs = [dict(scene=dev, camera=cam, sample_count=2, config=wfpt.render_config(32, 32, max_depth=4)),
                dict(scene=dev, camera=cam, sample_count=3, sample_start=9,
                     config=wfpt.render_config(32, 32, max_depth=6))]
        best, times = wfpt.Batch.autotune(jobs, slot_capacities=(256, 512), block_sizes=(64, 128),
                                          refill_thresholds=(8,))
        assert len(times) == 4 and all(t > 0 for t in times)
        assert best.block_size in (64, 128) and best.slot_capacity in (256, 512)
        batch = wfpt.Batch(jobs, config=best)
        batch.run()
        got = batch.download(1)
        batch.close()
        want, _ = _per_job(jobs[1])
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    finally:
        dev.close()


def test_batch_with_textured_job_matches_per_job_renders(cuda):
    """A job whose scene has textured and alpha-textured materials switches
    the batch to the alpha-capable trace and shadow kernels; every job still
    matches its own render bit for bit."""
    tex_scene, tex_cam = scenes.textured_room(48, 40)
    box_scene, box_cam = scenes.cornell_box(32, 32)
    jobs = [dict(scene=wfpt.DeviceScene(tex_scene), camera=tex_cam, sample_start=4, sample_count=3,
                 config=wfpt.render_config(48, 40, max_depth=6, rr_start_depth=3)),
            dict(scene=wfpt.DeviceScene(box_scene), camera=box_cam, sample_start=0, sample_count=2,
                 config=wfpt.render_config(32, 32, max_depth=8, rr_start_depth=3))]
    try:
        want = [_per_job(j)[0] for j in jobs]
        batch = wfpt.Batch(jobs)
        batch.run()
        batch.synchronize()
        for k, image in enumerate(want):
            assert np.array_equal(batch.download(k).view(np.uint32), image.view(np.uint32)), f"job {k}"
        batch.close()
    finally:
        for j in jobs:
            j["scene"].close()
