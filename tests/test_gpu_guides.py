"""Denoiser guide buffers (wf_frame_guides) against the reference's own
generateFrameGuides (include/renderer/device_frame_guides.cuh:6-41), which
runs in libwfref_det.so as host code with the renderer's deterministic
elementary functions.  Every field of every pixel must match bit for bit:
albedo through the material's textures and sRGB curve, the normal map in the
hit's tangent frame, the geometric normal, the forward depth, and, with a
previous camera, the reprojected motion and the visibility check behind
history_valid."""
import numpy as np
import pytest

import oracle
import wfpt
from wfpt import scenes

pytestmark = pytest.mark.gpu


def _moved(cam, offset, yaw=0.0):
    prev = {k: np.array(v, np.float32) if isinstance(v, (list, tuple, np.ndarray)) else v for k, v in cam.items()}
    prev["position"] = np.asarray(cam["position"], np.float32) + np.asarray(offset, np.float32)
    if yaw:
        c, s = np.cos(yaw), np.sin(yaw)
        rot = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]], np.float32)
        for k in ("forward", "right", "up"):
            prev[k] = (rot @ np.asarray(cam[k], np.float32)).astype(np.float32)
    return prev


def _check(scene, cam, width, height, tile=None, previous=None):
    dev = wfpt.DeviceScene(scene)
    try:
        got = dev.frame_guides(cam, width, height, tile=tile, previous=previous)
    finally:
        dev.close()
    ref = oracle.RefScene(scene, det=True)
    want = ref.frame_guides(cam, width, height, tile=tile, previous=previous)
    ref.close()
    assert got.shape == want.shape
    for field in want.dtype.names:
        a, b = got[field], want[field]
        bad = np.argwhere(a.view(np.uint32) != b.view(np.uint32))
        assert len(bad) == 0, f"{field}: {len(bad)} words differ, first at {bad[0]}: {a[tuple(bad[0][:2])]} vs {b[tuple(bad[0][:2])]}"
    return got


@pytest.fixture(scope="module", autouse=True)
def _need_oracle():
    if not oracle.available(det=True):
        pytest.skip("oracle/_ref/libwfref_det.so not built")


def test_cornell_guides_without_previous_camera():
    scene, cam = scenes.cornell_box(96, 64)
    g = _check(scene, cam, 96, 64)
    assert (g["valid"] == 1).all()
    assert not g["motion"].any() and not g["history_valid"].any()


def test_cornell_guides_with_camera_motion():
    scene, cam = scenes.cornell_box(96, 64)
    g = _check(scene, cam, 96, 64, previous=_moved(cam, (0.08, -0.03, 0.05), yaw=0.04))
    assert 0.5 < g["history_valid"].mean() < 1.0  # some pixels leave the previous frustum


def test_guides_reproject_onto_themselves():
    # projectFramePoint inverts Camera::generateRay at pixel centres
    # (tests/frame_export_tests.cpp:54-66): with the previous camera equal to
    # the current one every motion vector is within 1e-5 pixels of zero.
    scene, cam = scenes.cornell_box(64, 64)
    g = _check(scene, cam, 64, 64, previous=cam)
    assert np.abs(g["motion"]).max() < 1e-5
    assert (g["history_valid"] == 1).all()


def test_textured_room_guides():
    # albedo textures with transforms on both UV sets, normal maps through
    # instance transforms, alpha-masked cards in the primary and history rays
    scene, cam = scenes.textured_room(96, 72)
    g = _check(scene, cam, 96, 72, previous=_moved(cam, (0.1, 0.05, -0.05)))
    assert g["albedo"].std() > 0.05


def test_tile_guides_equal_the_frame_block():
    scene, cam = scenes.cornell_box(80, 60)
    prev = _moved(cam, (-0.05, 0.0, 0.02))
    dev = wfpt.DeviceScene(scene)
    try:
        full = dev.frame_guides(cam, 80, 60, previous=prev)
        tile = dev.frame_guides(cam, 80, 60, tile=(17, 9, 31, 23), previous=prev)
    finally:
        dev.close()
    assert np.array_equal(tile.view(np.uint8), full[9:32, 17:48].copy().view(np.uint8))


def test_guides_of_a_large_mesh_tile():
    scene, cam = scenes.large_mesh(128, 96, terrain_quads=192, instance_count=30, instance_frequency=40,
                                   glass_spheres=4, env_size=(64, 32))
    _check(scene, cam, 128, 96, tile=(32, 16, 64, 48), previous=_moved(cam, (0.2, 0.0, 0.1)))


def test_guides_reject_tiles_outside_the_image():
    scene, cam = scenes.cornell_box(32, 32)
    dev = wfpt.DeviceScene(scene)
    try:
        with pytest.raises(wfpt.WavefrontError):
            dev.frame_guides(cam, 32, 32, tile=(16, 0, 32, 32))
    finally:
        dev.close()


def test_captured_frame_export(tmp_path):
    # One frame of the dataset capture through wf_render and wf_frame_guides,
    # published as frame.exr + manifest.json and read back channel by channel.
    from wfpt import frame_export as fe
    scene, cam = scenes.cornell_box(48, 32)
    prev = _moved(cam, (0.04, 0.0, 0.0))
    cfg = wfpt.render_config(48, 32, max_depth=6, rr_start_depth=3)
    dev = wfpt.DeviceScene(scene)
    try:
        radiance, reference, guides = fe.capture_frame(dev, cam, cfg, 8, 2, 4, previous=prev)
    finally:
        dev.close()
    ref = oracle.RefScene(scene, det=True)
    sums, _, _ = ref.render(cam, cfg, sample_start=8, sample_count=2)
    want_guides = ref.frame_guides(cam, 48, 32, previous=prev)
    ref.close()
    assert np.array_equal(radiance.view(np.uint32), (sums * (np.float32(1) / np.float32(2))).view(np.uint32))
    assert np.array_equal(guides.view(np.uint8), want_guides.view(np.uint8))
    metadata = {"sequence_id": "cornell", "frame_index": 1, "previous_frame_index": 0,
                "camera": fe.frame_camera_metadata(cam), "previous_camera": fe.frame_camera_metadata(prev)}
    fe.write_captured_frame(tmp_path / "frame_000001", 48, 32, 2, 4, radiance, reference, guides, metadata)
    _, _, ch = fe.read_exr(tmp_path / "frame_000001" / "frame.exr")
    assert np.array_equal(ch["radiance.B"][1], radiance[:, :, 2])
    assert np.array_equal(ch["reference.R"][1], reference[:, :, 0])
    assert np.array_equal(ch["motion.X"][1], guides["motion"][:, :, 0])
    assert np.array_equal(ch["history_valid.Y"][1], guides["history_valid"])
