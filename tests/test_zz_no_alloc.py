"""wf_render_tile_static: the render entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc while they render (a host
running inside another framework's memory pool, or one whose device-memory
budget is fixed at start-up).  Its working memory is a fixed array inside
the library, shared by every call, so two calls in a row check that each
call starts from clean counters.  The framebuffers it fills must match the
persistent-mode renderer (wf_render) bit for bit, the same bar as the other
render parity tests.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import wfpt
from wfpt import abi, scenes

pytestmark = pytest.mark.gpu


def _reference_tile(dev, cam, cfg, tile, sample_start, sample_count):
    r = wfpt.Renderer(dev, cam, cfg)
    try:
        x, y, w, h = tile
        r.render(x, y, w, h, sample_start, sample_count, True)
        return r.download(x, y, w, h)
    finally:
        r.close()


def _static_tile(torch, dev, cam, cfg, tile, sample_start, sample_count):
    lib = wfpt.library()
    fb = torch.zeros((cfg.height, cfg.width, 3), dtype=torch.float32, device="cuda")
    camera = wfpt.camera_struct(cam)
    x, y, w, h = tile
    stream = torch.cuda.current_stream().cuda_stream
    wfpt.check(lib.wf_render_tile_static(dev.handle, C.byref(camera), C.byref(cfg), x, y, w, h, sample_start,
                                         sample_count, C.c_void_p(fb.data_ptr()), C.c_void_p(stream)))
    out = fb.cpu().numpy()
    outside = np.ones(out.shape[:2], bool)
    outside[y:y + h, x:x + w] = False
    assert not out[outside].any(), "pixels outside the tile were written"
    return out[y:y + h, x:x + w]


def test_static_entry_matches_persistent_renderer_twice(cuda):
    scene, cam = scenes.cornell_box(64, 48)
    cfg = wfpt.render_config(64, 48, max_depth=8, rr_start_depth=3, mode=abi.MODE_PERSISTENT)
    dev = wfpt.DeviceScene(scene)
    try:
        for tile, start, count in (((0, 0, 64, 48), 100, 3), ((16, 8, 40, 32), 7, 2)):
            want = _reference_tile(dev, cam, cfg, tile, start, count)
            got = _static_tile(cuda, dev, cam, cfg, tile, start, count)
            assert got.mean() > 0
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    finally:
        dev.close()


def test_static_entry_rejects_oversized_tiles_and_caustics(cuda):
    scene, cam = scenes.cornell_box(320, 240)
    dev = wfpt.DeviceScene(scene)
    try:
        cfg = wfpt.render_config(320, 240, max_depth=4, rr_start_depth=3)
        with pytest.raises(wfpt.WavefrontError, match="at most 65536 pixels"):
            _static_tile(cuda, dev, cam, cfg, (0, 0, 320, 240), 0, 1)
        cfg = wfpt.render_config(320, 240, max_depth=4, rr_start_depth=3, caustics=1, photon_count=1000)
        with pytest.raises(wfpt.WavefrontError, match="caustics"):
            _static_tile(cuda, dev, cam, cfg, (0, 0, 64, 64), 0, 1)
        # a rejected call leaves the entry point usable
        cfg = wfpt.render_config(320, 240, max_depth=4, rr_start_depth=3, mode=abi.MODE_PERSISTENT)
        want = _reference_tile(dev, cam, cfg, (100, 100, 32, 32), 5, 1)
        got = _static_tile(cuda, dev, cam, cfg, (100, 100, 32, 32), 5, 1)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    finally:
        dev.close()


@pytest.mark.parametrize("alpha", [True, False], ids=["alpha-textured", "textured-opaque"])
def test_static_entry_textured_kernel_variants(cuda, alpha):
    """The two other persistent-kernel variants the entry point picks per
    scene: with the texture alpha test (an alpha-masked, albedo-textured
    card) and with textures but no alpha test (the same room with alpha
    masking turned off).  Two calls in a row, each against wf_render."""
    scene, cam = scenes.textured_room(64, 64)
    if not alpha:
        scene.materials["alpha_masked"] = 0
    cfg = wfpt.render_config(64, 64, max_depth=6, rr_start_depth=3, mode=abi.MODE_PERSISTENT)
    dev = wfpt.DeviceScene(scene)
    try:
        for tile, start, count in (((0, 0, 64, 64), 40, 2), ((8, 16, 48, 40), 3, 1)):
            want = _reference_tile(dev, cam, cfg, tile, start, count)
            got = _static_tile(cuda, dev, cam, cfg, tile, start, count)
            assert got.mean() > 0
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    finally:
        dev.close()
