"""Frame and sample-layer export (wfpt.frame_export), the checks of the
reference's tests/frame_export_tests.cpp: float32 HDR radiance and uint32
sample counts survive the round trip with the image layout intact, the
manifest carries the version and the image digest, existing captures are
never overwritten, and non-finite or overlapping inputs publish nothing.
The EXR encoder is also read back by OpenCV's OpenEXR decoder when that is
available."""
import hashlib
import json
import os

import numpy as np
import pytest

from wfpt import abi
from wfpt import frame_export as fe


def _fixture():
    # tests/frame_export_tests.cpp:20-38: 3 x 2 pixels, an asymmetric last pixel
    radiance = np.tile(np.float32([0.125, 4.0, 32.0]), (6, 1))
    radiance[-1] = [1.0, 2.0, 3.0]
    reference = np.tile(np.float32([0.25, 5.0, 33.0]), (6, 1))
    guides = np.zeros(6, abi.FRAME_GUIDE_DTYPE)
    guides["albedo"] = [0.2, 0.5, 0.8]
    guides["normal"] = guides["geometric_normal"] = [0.0, 0.0, -1.0]
    guides["depth"] = 2.0
    guides["valid"] = 1.0
    return radiance, reference, guides


def _camera():
    return {"position": [0, 0, 0], "forward": [0, 0, 1], "right": [-1, 0, 0], "up": [0, 1, 0],
            "vertical_fov": np.float32(3.14159265359 / 2), "aspect_ratio": 1.5}


def _metadata():
    return {"sequence_id": "fixture", "frame_index": 0, "previous_frame_index": None, "scene": "fixture",
            "camera": fe.frame_camera_metadata(_camera()), "previous_camera": None, "render_fingerprint": "fixture",
            "render": {"rng": "pcg32", "rng_key": "pixel_sample_v1", "sample_start": 0, "samples": 4,
                       "reference_sample_start": 4, "reference_samples": 16,
                       "reference_estimator": "matched_renderer_settings"}}


def test_captured_frame_round_trip(tmp_path):
    out = tmp_path / "frame"
    radiance, reference, guides = _fixture()
    fe.write_captured_frame(out, 3, 2, 4, 16, radiance, reference, guides, _metadata())
    manifest = json.loads((out / "manifest.json").read_text())
    assert manifest["version"] == 1 and manifest["schema"] == "cuda-wavefront-frame"
    assert manifest["image"] == "frame.exr" and manifest["conventions"] == fe.frame_conventions()
    assert manifest["image_sha256"] == hashlib.sha256((out / "frame.exr").read_bytes()).hexdigest()
    w, h, ch = fe.read_exr(out / "frame.exr")
    assert (w, h) == (3, 2)
    assert ch["radiance.G"][0] == fe.EXR_FLOAT and ch["sample_count.N"][0] == fe.EXR_UINT
    green = ch["radiance.G"][1].reshape(-1)
    assert green[0] == 4.0 and green[5] == 2.0
    assert (ch["sample_count.N"][1] == 4).all() and (ch["reference_count.N"][1] == 16).all()
    assert set(ch) == {f"{p}.{c}" for p in ("radiance", "reference", "albedo") for c in "RGB"} | {
        f"{p}.{c}" for p in ("normal", "geometric_normal") for c in "XYZ"} | {
        "depth.Z", "motion.X", "motion.Y", "guide_valid.Y", "history_valid.Y", "sample_count.N", "reference_count.N"}
    assert (ch["normal.Z"][1] == -1).all() and (ch["albedo.B"][1] == np.float32(0.8)).all()
    assert not (tmp_path / "frame.partial").exists()


def test_existing_capture_is_never_overwritten(tmp_path):
    out = tmp_path / "frame"
    radiance, reference, guides = _fixture()
    fe.write_captured_frame(out, 3, 2, 4, 16, radiance, reference, guides, _metadata())
    before = (out / "frame.exr").read_bytes()
    with pytest.raises(FileExistsError):
        fe.write_captured_frame(out, 3, 2, 4, 16, radiance, reference, guides, _metadata())
    assert (out / "frame.exr").read_bytes() == before


@pytest.mark.parametrize("spoil", ["nan_radiance", "inf_reference", "negative_depth", "history_without_valid",
                                   "flag_half", "count"])
def test_invalid_capture_publishes_nothing(tmp_path, spoil):
    radiance, reference, guides = _fixture()
    if spoil == "nan_radiance":
        radiance[0, 0] = np.nan
    elif spoil == "inf_reference":
        reference[3, 2] = np.inf
    elif spoil == "negative_depth":
        guides["depth"][1] = -1.0
    elif spoil == "history_without_valid":
        guides["valid"][2] = 0.0
        guides["history_valid"][2] = 1.0
    elif spoil == "flag_half":
        guides["valid"][0] = 0.5
    else:
        radiance = radiance[:5]
    bad = tmp_path / "frame-invalid"
    with pytest.raises(ValueError):
        fe.write_captured_frame(bad, 3, 2, 4, 16, radiance, reference, guides, _metadata())
    assert not bad.exists() and not (tmp_path / "frame-invalid.partial").exists()


def _layers():
    a = np.tile(np.float32([0.25, 2.0, 64.0]), (6, 1))
    b = np.tile(np.float32([0.5, 4.0, 128.0]), (6, 1))
    b[-1] = [1.0, 3.0, 200.0]
    return [(1, 4100, a), (2, 4101, b)]


def test_sample_layers_round_trip(tmp_path):
    out = tmp_path / "sample-layers"
    fe.write_captured_sample_layers(out, 3, 2, _layers(), _metadata())
    manifest = json.loads((out / "manifest.json").read_text())
    assert manifest["schema"] == "cuda-wavefront-sample-layers" and len(manifest["image_sha256"]) == 64
    assert manifest["layers"][1]["sample_start"] == 4101
    assert manifest["layers"][0]["channels"] == ["spp_1.R", "spp_1.G", "spp_1.B"]
    assert "reference_samples" not in manifest["render"] and "samples" not in manifest["render"]
    _, _, ch = fe.read_exr(out / "layers.exr")
    assert "reference.R" not in ch
    blue = ch["spp_2.B"][1].reshape(-1)
    assert blue[0] == 128.0 and blue[-1] == 200.0
    with pytest.raises(FileExistsError):
        fe.write_captured_sample_layers(out, 3, 2, _layers(), _metadata())


@pytest.mark.parametrize("spoil", ["overlap", "duplicate_spp", "nan", "negative", "not_power_of_two", "too_many"])
def test_invalid_sample_layers_publish_nothing(tmp_path, spoil):
    layers = _layers()
    if spoil == "overlap":
        layers[1] = (2, 4100, layers[1][2])
    elif spoil == "duplicate_spp":
        layers[1] = (1, 5000, layers[1][2])
    elif spoil == "nan":
        layers[0][2][0, 0] = np.nan
    elif spoil == "negative":
        layers[0][2][0, 1] = -1.0
    elif spoil == "not_power_of_two":
        layers[1] = (3, 4101, layers[1][2])
    else:
        layers[1] = (64, 4101, layers[1][2])
    bad = tmp_path / "bad-layers"
    with pytest.raises(ValueError):
        fe.write_captured_sample_layers(bad, 3, 2, layers, _metadata())
    assert not bad.exists()


@pytest.mark.parametrize("compression", [fe.NO_COMPRESSION, fe.ZIPS_COMPRESSION, fe.ZIP_COMPRESSION])
@pytest.mark.parametrize("size", [(3, 2), (37, 23), (64, 41)])
def test_exr_encoder_round_trip(tmp_path, compression, size):
    w, h = size
    rng = np.random.default_rng(w * 100 + h)
    planes = {"a.R": (fe.EXR_FLOAT, (rng.standard_normal((h, w)) * 10).astype(np.float32)),
              "b.N": (fe.EXR_UINT, rng.integers(0, 2**32, (h, w), dtype=np.uint64).astype(np.uint32)),
              "c.Z": (fe.EXR_FLOAT, np.full((h, w), 2.5, np.float32))}
    fe.write_exr(tmp_path / "t.exr", w, h, planes, compression)
    ww, hh, ch = fe.read_exr(tmp_path / "t.exr")
    assert (ww, hh) == (w, h)
    for name, (kind, values) in planes.items():
        assert ch[name][0] == kind and np.array_equal(ch[name][1], values)


def test_exr_encoder_against_openexr_decoder(tmp_path):
    # An independent OpenEXR implementation (the one bundled with OpenCV)
    # must decode the encoder's files to the same float32 values.
    os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")
    cv2 = pytest.importorskip("cv2")
    if "OpenEXR" not in cv2.getBuildInformation():
        pytest.skip("OpenCV without OpenEXR")
    rng = np.random.default_rng(5)
    for compression in (fe.NO_COMPRESSION, fe.ZIPS_COMPRESSION, fe.ZIP_COMPRESSION):
        img = (rng.standard_normal((41, 37, 3)) * 10).astype(np.float32)
        img[::3] = np.round(img[::3])
        path = tmp_path / f"rgb{compression}.exr"
        fe.write_exr(path, 37, 41, {c: (fe.EXR_FLOAT, img[:, :, i]) for i, c in enumerate("RGB")}, compression)
        got = cv2.imread(str(path), cv2.IMREAD_UNCHANGED)
        assert got is not None and np.array_equal(got[:, :, ::-1], img)
