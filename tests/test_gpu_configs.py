"""Bit-exact parity on the benchmark configurations themselves, at full scene
size (not reduced stand-ins), against the reference's own renderer code
compiled for the host with the renderer's deterministic elementary functions
(oracle/_ref/libwfref_det.so).  Each test mirrors a task of the reference's
RenderTaskRenderer::render (src/renderer/render_task.cu:26-114): the
unnormalized sums of a tile over an absolute sample range.

* Cornell box (256x256, 16 spp, depth 8, Russian roulette from bounce 3,
  sample base 0): the whole frame, per-bounce queue counts, and the hit
  records and primitive / instance identities of the 65,536 camera rays of
  sample 0 plus their bounce-1 continuation rays;
* sphere field (1280x720 camera, the 1,310,720-triangle displaced geodesic
  sphere in three instances, the 22x22 sphere grid): a fixed 32x32 tile,
  2 spp, depth 16, graph and persistent schedules;
* large mesh (1920x1080 camera, 9,999,392-triangle terrain, 500 instances of
  a 200,000-triangle sphere, 2048x1024 environment, 2M photons): the photon
  map record for record, and a fixed 32x32 tile at 1 spp, depth 12, with the
  caustic gather, in graph and persistent schedules.

The inverse-rendering configuration's scene (10,240 wall triangles) is
covered in tests/test_gpu_adjoint_config.py."""
import numpy as np
import pytest

import oracle
import wfpt
from wfpt import abi, scenes

pytestmark = pytest.mark.gpu

needs_oracle = pytest.mark.skipif(not oracle.available(det=True), reason="oracle/_ref/libwfref_det.so not built")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def assert_same(got, want, what):
    diff = np.nonzero(bits(got) != bits(want))
    assert diff[0].size == 0, f"{what}: {diff[0].size} values differ, first at {[d[0] for d in diff]}"


def center_tile(width, height, size=32):
    return (width // 2 - size // 2, height // 2 - size // 2, size, size)


@needs_oracle
def test_cornell_full_frame_and_hit_batch(cuda):
    scene, cam = scenes.cornell_box(256, 256)
    assert scene.triangle_count() == 36
    fields = dict(max_depth=8, rr_start_depth=3)
    ref = oracle.RefScene(scene, det=True)
    want, _, want_counts = ref.render(cam, wfpt.render_config(256, 256, **fields), sample_start=0, sample_count=16)
    dev = wfpt.DeviceScene(scene)
    for mode in (abi.MODE_GRAPH, abi.MODE_PERSISTENT, abi.MODE_STREAM):
        cfg = wfpt.render_config(256, 256, mode=mode, **fields)
        r = wfpt.Renderer(dev, cam, cfg)
        got = r.render_task((0, 0, 256, 256), 0, 16)
        counts = r.queue_counts()
        r.close()
        assert_same(got, want, f"Cornell framebuffer (mode {mode})")
        if mode != abi.MODE_STREAM:  # the streaming loop keeps no per-sample bounce record
            assert np.array_equal(counts, want_counts[-1]), (mode, counts, want_counts[-1])
    # the hit-ID batch: sample 0's camera rays and their bounce-1 continuations
    cfg = wfpt.render_config(256, 256, **fields)
    rays, per_bounce = ref.path_rays(cam, cfg, sample=0, bounces=2)
    assert per_bounce[0] == 65536 and per_bounce[1] == want_counts[0][1]
    got = dev.trace_closest(rays)
    expect = ref.trace(rays)
    probe = oracle.RefScene(scene, det=True, probe=True).trace(rays)
    for f in ("t", "position", "geometric_normal", "normal", "material", "light_index"):
        assert_same(got[f], expect[f], f"hit {f}")
    assert np.array_equal(got["kind"], probe["kind"])
    hit = got["kind"] != abi.HIT_NONE
    assert hit.mean() > 0.9
    assert np.array_equal(got["primitive"][hit], probe["primitive"][hit])
    mesh = got["kind"] == abi.HIT_MESH
    assert np.array_equal(got["instance"][mesh], probe["instance"][mesh])
    dev.close()


def render_tile(scene, cam, width, height, fields, tile, sample_start, spp, modes):
    dev = wfpt.DeviceScene(scene)
    out = {}
    photons = None
    for mode in modes:
        cfg = wfpt.render_config(width, height, mode=mode, **fields)
        r = wfpt.Renderer(dev, cam, cfg)
        if fields.get("caustics") and photons is None:
            photons = (r.photon_stats(), r.photons())
        out[mode] = (r.render_task(tile, sample_start, spp), r.queue_counts())
        r.close()
    dev.close()
    return out, photons


@needs_oracle
def test_sphere_field_full_scene_tile(cuda):
    scene, cam = scenes.sphere_field(1280, 720)
    assert scene.triangle_count() == 1_310_720
    fields = dict(max_depth=16)
    tile = center_tile(1280, 720)
    got, _ = render_tile(scene, cam, 1280, 720, fields, tile, 1 << 20, 2, (abi.MODE_GRAPH, abi.MODE_PERSISTENT))
    ref = oracle.RefScene(scene, det=True)
    want, _, want_counts = ref.render(cam, wfpt.render_config(1280, 720, **fields), tile=tile,
                                      sample_start=1 << 20, sample_count=2)
    assert want.mean() > 0
    for mode, (image, counts) in got.items():
        assert_same(image, want, f"sphere-field tile (mode {mode})")
        assert np.array_equal(counts, want_counts[-1]), (mode, counts, want_counts[-1])


@needs_oracle
def test_large_mesh_full_scene_tile_and_photon_map(cuda):
    scene, cam = scenes.large_mesh(1920, 1080)
    assert scene.triangle_count() == 10_199_392 and len(scene.instances) == 501
    fields = dict(max_depth=12, caustics=1, photon_count=2_000_000, photon_grid_min=(0, 0, 0),
                  photon_grid_max=(0, 0, 0))
    tile = center_tile(1920, 1080)
    got, (stats, photons) = render_tile(scene, cam, 1920, 1080, fields, tile, 2 << 20, 1,
                                        (abi.MODE_GRAPH, abi.MODE_PERSISTENT))
    ref = oracle.RefScene(scene, det=True)
    cfg = wfpt.render_config(1920, 1080, **fields)
    rec, _, ref_stored = ref.photons(cfg)
    stored, emitted = stats
    assert emitted == 2_000_000 and stored == ref_stored and stored > 10_000
    assert_same(photons, rec, "photon records")
    want, _, want_counts = ref.render(cam, cfg, tile=tile, sample_start=2 << 20, sample_count=1)
    assert want.mean() > 0
    for mode, (image, counts) in got.items():
        assert_same(image, want, f"large-mesh tile (mode {mode})")
        assert np.array_equal(counts, want_counts[-1]), (mode, counts, want_counts[-1])
