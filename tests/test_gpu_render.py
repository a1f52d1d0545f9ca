"""Full render parity: the CUDA renderer against the host-compiled reference.

libwfref_det.so is the reference's own renderer code with the renderer's
deterministic elementary functions; the CUDA kernels must reproduce its FP32
framebuffer sums and per-bounce queue counts bit for bit, in graph and in
persistent mode.  Against the reference with the C library's math the
images must agree to a small relative RMSE."""
import os

import numpy as np
import pytest

import oracle
import wfpt
from wfpt import abi, scenes
from helpers import relative_rmse

pytestmark = pytest.mark.gpu


def small_large_mesh(w=96, h=54):
    return scenes.large_mesh(w, h, terrain_quads=64, instance_count=12, instance_frequency=8, glass_spheres=3,
                             env_size=(256, 128))


WORKLOADS = {
    "cornell": (lambda: scenes.cornell_box(64, 64), dict(max_depth=8, rr_start_depth=3), 4),
    "sphere_field": (lambda: scenes.sphere_field(96, 54, frequency=16), dict(max_depth=16), 3),
    "large_mesh": (small_large_mesh, dict(max_depth=12), 2),
}


def render_both(name, mode, **over):
    make, fields, spp = WORKLOADS[name]
    scene, cam = make()
    cfg_fields = dict(fields)
    cfg_fields.update(over)
    w, h = int(round(cam["aspect_ratio"] * 54)) if name != "cornell" else 64, 54 if name != "cornell" else 64
    cfg = wfpt.render_config(w, h, mode=mode, **cfg_fields)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    got = r.render_task((0, 0, w, h), 100, spp)
    counts = r.queue_counts()
    stats = r.stats()
    r.close()
    dev.close()
    ref = oracle.RefScene(scene, det=True)
    want, _, want_counts = ref.render(cam, cfg, sample_start=100, sample_count=spp)
    return got, counts, stats, want, want_counts, (scene, cam, cfg, spp)


@pytest.mark.parametrize("mode", [abi.MODE_GRAPH, abi.MODE_PERSISTENT])
@pytest.mark.parametrize("name", list(WORKLOADS))
def test_framebuffer_bit_exact(cuda, name, mode):
    got, counts, stats, want, want_counts, _ = render_both(name, mode)
    diff = np.nonzero(got.view(np.uint32) != want.view(np.uint32))
    assert diff[0].size == 0, f"{diff[0].size} channels differ; first pixel {diff[0][0], diff[1][0]}: " \
                              f"{got[diff[0][0], diff[1][0]]} vs {want[diff[0][0], diff[1][0]]}"
    assert np.array_equal(counts, want_counts[-1])
    assert got.mean() > 0


@pytest.mark.parametrize("name", list(WORKLOADS))
def test_stream_mode_bit_exact(cuda, name):
    """Streaming mode (slot regeneration inside a graph WHILE loop) gives the
    reference's framebuffer sums bit for bit, and the same ray totals as the
    per-sample graph."""
    got, _, stats, want, want_counts, _ = render_both(name, abi.MODE_STREAM)
    diff = np.nonzero(got.view(np.uint32) != want.view(np.uint32))
    assert diff[0].size == 0, f"{diff[0].size} channels differ"
    assert stats["extension_rays"] == int(want_counts.sum())
    _, _, graph_stats, _, _, _ = render_both(name, abi.MODE_GRAPH)
    for k in ("extension_rays", "shadow_rays", "paths"):
        assert stats[k] == graph_stats[k], k
    assert 0 < stats["kernel_launches"] <= graph_stats["kernel_launches"]


@pytest.mark.parametrize("percent", [1, 25, 100])
@pytest.mark.parametrize("name", ["cornell", "large_mesh"])
def test_stream_regeneration_threshold_keeps_sums(cuda, name, percent):
    """Whatever share of the slots must be idle before waiting slots start
    their next samples together (1 %: almost a sample at a time; 100 %: after
    every bounce), each pixel takes its samples in order, so the sums equal
    the reference's bit for bit."""
    got, _, stats, want, want_counts, _ = render_both(name, abi.MODE_STREAM, regenerate_percent=percent)
    diff = np.nonzero(got.view(np.uint32) != want.view(np.uint32))
    assert diff[0].size == 0, f"{diff[0].size} channels differ"
    assert stats["extension_rays"] == int(want_counts.sum())


def test_stream_mode_tiles_and_long_ranges(cuda):
    """Tile-major frames, split ranges and a 16-sample range in streaming mode
    match the per-sample graph."""
    scene, cam = scenes.cornell_box(64, 64)
    frames = {}
    for mode in (abi.MODE_GRAPH, abi.MODE_STREAM):
        cfg = wfpt.render_config(64, 64, max_depth=8, rr_start_depth=3, tile_width=32, tile_height=32, mode=mode)
        dev = wfpt.DeviceScene(scene)
        r = wfpt.Renderer(dev, cam, cfg)
        r.reset()
        r.render_frame(5)
        assert r.sample_index() == 5
        frame = r.download()
        r.render(0, 32, 32, 32, 7, 2, True)
        r.render(0, 32, 32, 32, 9, 14, False)
        split = r.download(0, 32, 32, 32)
        r.close()
        frames[mode] = (frame, split)
    for a, b in zip(frames[abi.MODE_GRAPH], frames[abi.MODE_STREAM]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("tiles", [None, (32, 24)])
def test_two_wavefronts_match_one(cuda, tiles):
    """Graph mode with the twin wavefront (default) against one wavefront:
    identical sums, queue counts, ray counters and sample indices for frames,
    odd-row tasks and one-row tasks."""
    scene, cam = scenes.cornell_box(64, 48)
    results = []
    for concurrent in (1, 2):
        fields = dict(max_depth=8, rr_start_depth=3, concurrent_tiles=concurrent)
        if tiles:
            fields.update(tile_width=tiles[0], tile_height=tiles[1])
        cfg = wfpt.render_config(64, 48, **fields)
        dev = wfpt.DeviceScene(scene)
        r = wfpt.Renderer(dev, cam, cfg)
        r.set_sample_index(40)
        r.render_frame(3)
        frame = r.download()
        index = r.sample_index()
        counts = r.queue_counts()
        r.render(5, 7, 24, 17, 90, 2, True)
        r.render(0, 3, 20, 1, 200, 3, True)
        task = r.download()
        after = r.sample_index()
        r.render_frame(1)
        stats = r.stats()
        last = r.download()
        r.close()
        dev.close()
        results.append((frame, index, counts, task, after, stats, last))
    one, two = results
    for a, b in ((one[0], two[0]), (one[3], two[3]), (one[6], two[6])):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert one[1] == two[1] == 43 and one[4] == two[4] == 203
    assert np.array_equal(one[2], two[2])
    for k in ("extension_rays", "shadow_rays", "paths"):
        assert one[5][k] == two[5][k], k


def test_ray_counters(cuda):
    got, counts, stats, want, want_counts, (_, _, _, spp) = render_both("cornell", abi.MODE_GRAPH)
    assert stats["extension_rays"] == int(want_counts.sum())
    assert stats["paths"] == 64 * 64 * spp
    assert stats["shadow_rays"] > 0


def test_against_reference_with_c_library_math(cuda):
    """Same seed and spp as the unmodified reference: only the math library
    differs, so the images agree closely (relative RMSE bound 2%)."""
    scene, cam = scenes.cornell_box(64, 64)
    cfg = wfpt.render_config(64, 64, max_depth=8, rr_start_depth=3)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    got = r.render_task((0, 0, 64, 64), 0, 16)
    r.close()
    want, _, _ = oracle.RefScene(scene).render(cam, cfg, sample_count=16)
    assert relative_rmse(got, want) < 0.02


def test_tiles_and_accumulation(cuda):
    scene, cam = scenes.cornell_box(64, 64)
    cfg = wfpt.render_config(64, 64, max_depth=8, rr_start_depth=3, tile_width=32, tile_height=32)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    r.reset()
    r.render_frame(3)
    frame = r.download()
    assert r.sample_index() == 3
    tile = r.render_task((32, 0, 32, 32), 0, 3)
    assert np.array_equal(tile.view(np.uint32), frame[0:32, 32:64].view(np.uint32))
    # accumulate two halves of the range = one range (per-pixel order is the same)
    r.render(0, 32, 32, 32, 0, 2, True)
    r.render(0, 32, 32, 32, 2, 1, False)
    acc = r.download(0, 32, 32, 32)
    assert np.array_equal(acc.view(np.uint32), frame[32:64, 0:32].view(np.uint32))
    with pytest.raises(wfpt.WavefrontError):
        r.render(40, 0, 32, 32, 0, 1)
    r.close()


@pytest.mark.parametrize("wave", [2, 3, 8])
@pytest.mark.parametrize("concurrent,tiles", [(1, None), (2, None), (2, (32, 24))])
def test_sample_waves_match_one_sample_per_launch(cuda, wave, concurrent, tiles):
    """samples_per_wave: several samples of every pixel in one launch of the
    bounce chain give the same sums and sample indices as one sample per
    launch, for sample counts that do not divide into waves, for frames and
    for tile tasks."""
    results = []
    for w in (1, wave):
        fields = dict(max_depth=8, rr_start_depth=3, concurrent_tiles=concurrent, samples_per_wave=w)
        if tiles:
            fields.update(tile_width=tiles[0], tile_height=tiles[1])
        scene, cam = scenes.cornell_box(64, 48)
        cfg = wfpt.render_config(64, 48, **fields)
        dev = wfpt.DeviceScene(scene)
        r = wfpt.Renderer(dev, cam, cfg)
        r.set_sample_index(40)
        r.render_frame(7)
        frame = r.download()
        index = r.sample_index()
        r.render(5, 7, 24, 17, 90, 5, True)
        task = r.download()
        after = r.sample_index()
        stats = r.stats()
        r.close()
        dev.close()
        results.append((frame, index, task, after, stats))
    one, many = results
    for a, b in ((one[0], many[0]), (one[2], many[2])):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert one[1] == many[1] == 47 and one[3] == many[3] == 95
    for k in ("extension_rays", "shadow_rays", "paths"):
        assert one[4][k] == many[4][k], k


@pytest.mark.parametrize("wave", [2, 5])
def test_persistent_sample_waves_match(cuda, wave):
    """Waves in persistent mode (the staged kernel): the same sums and
    sample indices as one sample per cooperative launch."""
    results = []
    for w in (1, wave):
        scene, cam = scenes.cornell_box(64, 48)
        cfg = wfpt.render_config(64, 48, max_depth=8, rr_start_depth=3, mode=abi.MODE_PERSISTENT,
                                 persistent_stages=abi.PERSISTENT_STAGED, samples_per_wave=w)
        dev = wfpt.DeviceScene(scene)
        r = wfpt.Renderer(dev, cam, cfg)
        r.set_sample_index(7)
        r.render_frame(6)
        frame = r.download()
        index = r.sample_index()
        task = r.render_task((3, 5, 30, 20), 50, 7)
        r.close()
        dev.close()
        results.append((frame, index, task))
    one, many = results
    assert np.array_equal(one[0].view(np.uint32), many[0].view(np.uint32))
    assert np.array_equal(one[2].view(np.uint32), many[2].view(np.uint32))
    assert one[1] == many[1] == 13


def test_sample_waves_large_mesh_bit_exact(cuda):
    """A wave of 3 samples on the reduced large mesh (caustics, environment,
    instances) against the host-compiled reference's sums."""
    scene, cam = small_large_mesh()
    w, h = int(round(cam["aspect_ratio"] * 54)), 54
    cfg = wfpt.render_config(w, h, max_depth=12, samples_per_wave=3)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    got = r.render_task((0, 0, w, h), 100, 4)
    r.close()
    dev.close()
    ref = oracle.RefScene(scene, det=True)
    want, _, _ = ref.render(cam, cfg, sample_start=100, sample_count=4)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("concurrent", [1, 2])
def test_async_download_matches_each_step(cuda, concurrent):
    """wf_framebuffer_download_async: each copy holds the framebuffer as it
    stood when the call was made, although later renders (which clear and
    rewrite the tile) were issued before the copies arrived; a third copy
    reuses the first snapshot only after the first copy has left."""
    scene, cam = scenes.cornell_box(64, 48)
    cfg = wfpt.render_config(64, 48, max_depth=8, rr_start_depth=3, concurrent_tiles=concurrent)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    want = []
    for i in range(4):
        r.render(0, 0, 64, 48, 10 + 2 * i, 2, True)
        want.append(r.download())
    got = [np.full((48, 64, 3), np.nan, np.float32) for _ in range(4)]
    for i in range(4):
        r.render(0, 0, 64, 48, 10 + 2 * i, 2, True)
        r.download_async(got[i])
    r.download_wait()
    part = np.full((17, 24, 3), np.nan, np.float32)
    r.download_async(part, 5, 7)
    r.synchronize()
    r.close()
    dev.close()
    for a, b in zip(got, want):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(part.view(np.uint32), want[3][7:24, 5:29].view(np.uint32))


def test_debug_views(cuda):
    scene, cam = scenes.cornell_box(32, 32)
    for debug in (abi.DEBUG_INTERSECTION, abi.DEBUG_SHADING_NORMAL):
        cfg = wfpt.render_config(32, 32, max_depth=4, rr_start_depth=3, debug=debug)
        dev = wfpt.DeviceScene(scene)
        r = wfpt.Renderer(dev, cam, cfg)
        got = r.render_task((0, 0, 32, 32), 0, 1)
        r.close()
        want, _, _ = oracle.RefScene(scene, det=True).render(cam, cfg, sample_count=1)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_checkpoint_roundtrip_and_reference_format(cuda, tmp_path):
    import ctypes
    scene, cam = scenes.cornell_box(32, 24)
    cfg = wfpt.render_config(32, 24, max_depth=6, rr_start_depth=3)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    r.reset()
    r.render_frame(3)
    path = str(tmp_path / "render.checkpoint")
    r.checkpoint_save(path, 0x9B1D4F27A6C35011)
    before = r.download()
    r2 = wfpt.Renderer(dev, cam, cfg)
    assert r2.checkpoint_load(path, 0x9B1D4F27A6C35011) == 3
    assert np.array_equal(r2.download(), before)
    with pytest.raises(wfpt.WavefrontError) as e:
        r2.checkpoint_load(path, 1)
    assert e.value.status == 5
    # The reference's loader reads the file (render_checkpoint.cpp:163-195).
    rgb = np.zeros((24, 32, 3), np.float32)
    sample = ctypes.c_uint32()
    oracle.ref_lib().wfref_checkpoint_roundtrip_read(path.encode(), 32, 24, 0x9B1D4F27A6C35011, rgb.ctypes.data,
                                                     ctypes.addressof(sample))
    assert sample.value == 3 and np.array_equal(rgb, before)
    # ...and the product reads a checkpoint the reference wrote.
    ref_path = str(tmp_path / "ref.checkpoint")
    oracle.ref_lib().wfref_checkpoint_write(ref_path.encode(), 32, 24, 77, before.ctypes.data, 9)
    assert r2.checkpoint_load(ref_path, 77) == 9
    assert np.array_equal(r2.download(), before)
    # Asynchronous writer.
    assert r2.checkpoint_enqueue(str(tmp_path / "async.checkpoint"), 77)
    r2.checkpoint_flush()
    assert os.path.getsize(tmp_path / "async.checkpoint") == 32 + 32 * 24 * 12
    r.close()
    r2.close()


def caustic_scene():
    scene, cam = scenes.cornell_box(64, 64)
    glass = scene.add_material(wfpt.material(abi.MAT_DIELECTRIC, (1, 1, 1), ior=1.5))
    sp = np.zeros(1, abi.SPHERE_DTYPE)
    sp[0] = ((0.0, 0.4, 1.2), 0.6, glass, abi.ACCEL_BVH)
    scene.spheres = sp
    return scene, cam


def test_photon_map_and_caustic_render(cuda):
    scene, cam = caustic_scene()
    cfg = wfpt.render_config(64, 64, max_depth=8, rr_start_depth=3, caustics=1, photon_count=200000)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    stored, emitted = r.photon_stats()
    photons = r.photons()
    ref = oracle.RefScene(scene, det=True)
    rec, flux, ref_stored = ref.photons(cfg)
    assert emitted == 200000 and stored == ref_stored and stored > 1000
    assert np.array_equal(photons.view(np.uint32), rec.view(np.uint32))
    got = r.render_task((0, 0, 64, 64), 0, 2)
    want, _, _ = ref.render(cam, cfg, sample_count=2)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    r.close()
