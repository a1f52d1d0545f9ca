"""Loaded asset presets rendered on the GPU against the reference end to end:
the reference's own loaders and preset assembly build the HostScene
(oracle.RefHostScene), its uploadScene and renderer run in libwfref_det.so;
the product's loaders (wfpt.assets) build the scene description that
wf_scene_create uploads and wf_render renders.  Framebuffer sums and queue
counts must be identical bit for bit, and so must the denoiser guides."""
from pathlib import Path

import numpy as np
import pytest

import oracle
import wfpt
from wfpt import abi, assets

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "assets"
KIND = {"sponza": "gltf", "deer": "obj", "demo": "demo", "rtweek": "rtweek"}
W, H = 64, 48


@pytest.fixture(scope="module", autouse=True)
def _need_oracle():
    if not oracle.available(det=True):
        pytest.skip("oracle/_ref/libwfref_det.so not built")


def _reference(config):
    kind = KIND.get(config.preset, "cornell")
    return oracle.RefHostScene(kind, config.object_file,
                               scale=config.gltf_scale if kind == "gltf" else config.object_scale,
                               translation=config.object_translation, object_source=config.object_source,
                               neutral_room=config.neutral_room, remove_backdrop=config.remove_backdrop,
                               dielectric=config.dielectric, material_override=config.material_override,
                               light_profile=config.light_profile, add_top_light=config.add_sponza_top_light)


@pytest.mark.parametrize("manifest", sorted(p.name for p in GOLDEN.glob("fixture_*.json")))
@pytest.mark.parametrize("mode", [abi.MODE_GRAPH, abi.MODE_PERSISTENT])
def test_loaded_preset_renders_match_the_reference(manifest, mode):
    config = assets.load_manifest(GOLDEN / manifest)
    scene, cam = assets.preset_scene(config, W, H)
    cfg = wfpt.render_config(W, H, max_depth=6, rr_start_depth=3, mode=mode)
    dev = wfpt.DeviceScene(scene)
    try:
        r = wfpt.Renderer(dev, cam, cfg)
        try:
            got = r.render_task((0, 0, W, H), 5, 3)
            counts = r.queue_counts()
        finally:
            r.close()
        guides = dev.frame_guides(cam, W, H)
    finally:
        dev.close()
    host = _reference(config)
    ref = host.render_scene(disable_normal_maps=not config.use_normal_maps,
                            normal_map_minimum_cosine=config.normal_map_minimum_cosine)
    try:
        want, _, ref_counts = ref.render(cam, cfg, sample_start=5, sample_count=3,
                                         persistent=mode == abi.MODE_PERSISTENT)
        want_guides = ref.frame_guides(cam, W, H)
    finally:
        ref.close()
        host.close()
    assert got.mean() > 0, "empty render"
    bad = np.argwhere(got.view(np.uint32) != want.view(np.uint32))
    assert len(bad) == 0, f"{len(bad)} framebuffer words differ, first {tuple(bad[0])}"
    assert np.array_equal(counts, ref_counts[-1])
    assert np.array_equal(guides.view(np.uint8), want_guides.view(np.uint8))
