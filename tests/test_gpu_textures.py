"""Textured materials against the host-compiled reference.

The reference's own texture code (getTriangleUv, getTextureUv /
sampleTexture, getMaterialAlbedo / Opacity / Emission / Metallic /
Roughness / Normal, getSpecGlossSurface, getGltfPbrSurface,
getMaterialThickness and the tangent frames of intersectTriangleHit and
intersectMeshInstance) runs in libwfref_det.so, with tex2D as the host
replay's bilinear fetch and the renderer's deterministic elementary
functions.  The CUDA renderer must give the same framebuffer sums and queue
counts bit for bit on a scene that uses every binding: albedo with a
transform, normal maps (vertex and face tangents, both coordinate sets,
instance transforms), metallic-roughness, glTF PBR clearcoat with its own
normal map, specular-glossiness on coordinate set 1 with a rotation, an
emissive texture, an alpha-masked card and a thickness texture.
"""
import numpy as np
import pytest

import oracle
import wfpt
from wfpt import abi, scenes

pytestmark = pytest.mark.gpu

W = H = 64


def _render(scene, cam, mode, debug=0, samples=(11, 3)):
    cfg = wfpt.render_config(W, H, max_depth=6, rr_start_depth=3, mode=mode, debug=debug)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    try:
        img = r.render_task((0, 0, W, H), *samples)
        counts = r.queue_counts()
    finally:
        r.close()
        dev.close()
    ref = oracle.RefScene(scene, det=True)
    want, _, ref_counts = ref.render(cam, cfg, sample_start=samples[0], sample_count=samples[1],
                                     persistent=mode == abi.MODE_PERSISTENT)
    ref.close()
    return img, counts, want, ref_counts


def _assert_same(img, counts, want, ref_counts, check_counts=True):
    assert want.mean() > 0.0
    diff = np.count_nonzero(img.view(np.uint32) != want.view(np.uint32))
    assert diff == 0, f"{diff} channels differ"
    if check_counts:
        assert np.array_equal(counts, ref_counts[-1])


@pytest.mark.parametrize("mode", [abi.MODE_GRAPH, abi.MODE_PERSISTENT, abi.MODE_STREAM])
def test_textured_room_bit_exact(cuda, mode):
    """Streaming mode regenerates paths inside one launch and keeps no
    per-bounce queue counts; its sums are compared."""
    scene, cam = scenes.textured_room(W, H)
    _assert_same(*_render(scene, cam, mode), check_counts=mode != abi.MODE_STREAM)


@pytest.mark.parametrize("setting", ["no_normal_maps", "minimum_cosine"])
def test_normal_map_settings_bit_exact(cuda, setting):
    scene, cam = scenes.textured_room(W, H)
    if setting == "no_normal_maps":
        scene.disable_normal_maps = True
    else:
        scene.normal_map_minimum_cosine = 0.97
    _assert_same(*_render(scene, cam, abi.MODE_GRAPH))


def test_shading_normal_debug_view_bit_exact(cuda):
    scene, cam = scenes.textured_room(W, H)
    img, _, want, _ = _render(scene, cam, abi.MODE_GRAPH, debug=abi.DEBUG_SHADING_NORMAL, samples=(0, 1))
    assert np.array_equal(img.view(np.uint32), want.view(np.uint32))


def test_textures_change_the_image(cuda):
    scene, cam = scenes.textured_room(W, H)
    img, _, _, _ = _render(scene, cam, abi.MODE_GRAPH, samples=(0, 1))
    scene.material_textures = None
    plain, _, _, _ = _render(scene, cam, abi.MODE_GRAPH, samples=(0, 1))
    assert np.mean(img != plain) > 0.5
