"""Frame and sample-layer export for denoiser datasets.

The counterpart of the reference's src/renderer/frame_export.cpp (interface
include/renderer/frame_export.hpp:9-36): a captured frame (mean radiance, a
higher-sample reference, and the per-pixel guides of wf_frame_guides) or a
set of independent sample layers is written as one OpenEXR image plus a
manifest.json, published together by renaming a staging directory.  The
same checks reject bad captures before anything is published: sizes and
counts, non-finite values, guide flags outside {0, 1}, a history flag
without a valid guide, duplicate or overlapping sample layers, and an
output directory that already exists.

The reference writes through OpenEXR's Imf::OutputFile with a default
Header, i.e. a single-part scanline image with ZIP compression (16-line
blocks).  write_exr() produces that file layout directly from the published
OpenEXR file format: magic and version, the required header attributes, the
chunk offset table, and per chunk the rows of every channel in name order,
byte-interleaved, delta-predicted and deflated (stored raw when deflating
does not shrink it).  FLOAT channels are IEEE float32 and UINT channels
uint32, both little-endian, as in the reference's frame.
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import shutil
import struct
import zlib
from pathlib import Path

import numpy as np

from . import abi

EXR_UINT, EXR_HALF, EXR_FLOAT = 0, 1, 2
NO_COMPRESSION, ZIPS_COMPRESSION, ZIP_COMPRESSION = 0, 2, 3
_LINES_PER_CHUNK = {NO_COMPRESSION: 1, ZIPS_COMPRESSION: 1, ZIP_COMPRESSION: 16}
_TYPES = {EXR_UINT: np.dtype("<u4"), EXR_HALF: np.dtype("<f2"), EXR_FLOAT: np.dtype("<f4")}


# ------------------------------------------------------------------ OpenEXR
def _attribute(name: str, kind: str, value: bytes) -> bytes:
    return name.encode() + b"\0" + kind.encode() + b"\0" + struct.pack("<i", len(value)) + value


def _zip_block(raw: bytes) -> bytes:
    """OpenEXR ZIP/ZIPS chunk: even bytes then odd bytes, each byte stored as
    its difference from the previous one plus 128, deflated; the raw bytes
    when that is not smaller."""
    a = np.frombuffer(raw, np.uint8)
    t = np.concatenate([a[0::2], a[1::2]])
    p = t.copy()
    if len(t) > 1:
        p[1:] = (t[1:].astype(np.int16) - t[:-1].astype(np.int16) + 128).astype(np.uint8)
    packed = zlib.compress(p.tobytes())
    return packed if len(packed) < len(raw) else raw


def write_exr(path, width: int, height: int, channels: dict, compression: int = ZIP_COMPRESSION) -> None:
    """Single-part scanline OpenEXR image.  channels maps a name to
    (pixel_type, array of height*width values, row-major from the top)."""
    if compression not in _LINES_PER_CHUNK:
        raise ValueError(f"unsupported compression {compression}")
    if width <= 0 or height <= 0 or width > 2**31 - 1 or height > 2**31 - 1:
        raise ValueError("invalid image size")
    names = sorted(channels)  # OpenEXR keeps channels in name order
    planes = []
    chlist = b""
    for name in names:
        kind, values = channels[name]
        plane = np.ascontiguousarray(values, _TYPES[kind]).reshape(height, width)
        planes.append(plane)
        chlist += name.encode() + b"\0" + struct.pack("<iB3xii", kind, 0, 1, 1)
    chlist += b"\0"
    box = struct.pack("<iiii", 0, 0, width - 1, height - 1)
    header = (b"\x76\x2f\x31\x01" + struct.pack("<I", 2)
              + _attribute("channels", "chlist", chlist)
              + _attribute("compression", "compression", bytes([compression]))
              + _attribute("dataWindow", "box2i", box)
              + _attribute("displayWindow", "box2i", box)
              + _attribute("lineOrder", "lineOrder", b"\0")
              + _attribute("pixelAspectRatio", "float", struct.pack("<f", 1.0))
              + _attribute("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
              + _attribute("screenWindowWidth", "float", struct.pack("<f", 1.0))
              + b"\0")
    lines = _LINES_PER_CHUNK[compression]
    chunks = []
    for y0 in range(0, height, lines):
        y1 = min(height, y0 + lines)
        raw = b"".join(plane[y].tobytes() for y in range(y0, y1) for plane in planes)
        data = raw if compression == NO_COMPRESSION else _zip_block(raw)
        chunks.append(struct.pack("<ii", y0, len(data)) + data)
    offsets = []
    position = len(header) + 8 * len(chunks)
    for c in chunks:
        offsets.append(position)
        position += len(c)
    with open(path, "wb") as f:
        f.write(header)
        f.write(struct.pack(f"<{len(offsets)}Q", *offsets))
        for c in chunks:
            f.write(c)


def read_exr(path) -> tuple[int, int, dict]:
    """Reads what write_exr writes (NO, ZIPS and ZIP compression):
    (width, height, {name: (pixel_type, (height, width) array)})."""
    data = Path(path).read_bytes()
    if data[:4] != b"\x76\x2f\x31\x01":
        raise ValueError("not an OpenEXR file")
    pos = 8
    attrs = {}
    while data[pos] != 0:
        end = data.index(b"\0", pos)
        name = data[pos:end].decode()
        tend = data.index(b"\0", end + 1)
        size = struct.unpack_from("<i", data, tend + 1)[0]
        attrs[name] = data[tend + 5:tend + 5 + size]
        pos = tend + 5 + size
    pos += 1
    chans = []
    c = attrs["channels"]
    i = 0
    while c[i] != 0:
        end = c.index(b"\0", i)
        kind = struct.unpack_from("<i", c, end + 1)[0]
        chans.append((c[i:end].decode(), kind))
        i = end + 17
    compression = attrs["compression"][0]
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"])
    width, height = x1 - x0 + 1, y1 - y0 + 1
    lines = _LINES_PER_CHUNK[compression]
    count = math.ceil(height / lines)
    offsets = struct.unpack_from(f"<{count}Q", data, pos)
    out = {name: np.zeros((height, width), _TYPES[kind]) for name, kind in chans}
    for off in offsets:
        y, size = struct.unpack_from("<ii", data, off)
        block = data[off + 8:off + 8 + size]
        rows = min(lines, height - (y - y0))
        expected = rows * width * sum(_TYPES[k].itemsize for _, k in chans)
        if compression != NO_COMPRESSION and size < expected:
            p = np.frombuffer(zlib.decompress(block), np.uint8)
            t = (np.cumsum(np.concatenate([[int(p[0])], p[1:].astype(np.int64) - 128])) & 0xFF).astype(np.uint8)
            half = (len(t) + 1) // 2
            raw = np.empty_like(t)
            raw[0::2] = t[:half]
            raw[1::2] = t[half:]
            block = raw.tobytes()
        at = 0
        for r in range(rows):
            for name, kind in chans:
                n = width * _TYPES[kind].itemsize
                out[name][y - y0 + r] = np.frombuffer(block[at:at + n], _TYPES[kind])
                at += n
    return width, height, {name: (kind, out[name]) for name, kind in chans}


# ----------------------------------------------------------------- manifests
def frame_camera_metadata(camera) -> dict:
    """frameCameraMetadata (frame_export.cpp:111-117)."""
    vec = lambda v: [float(x) for x in v]  # noqa: E731
    return {"position": vec(camera["position"]), "forward": vec(camera["forward"]), "right": vec(camera["right"]),
            "up": vec(camera["up"]), "vertical_fov_radians": float(camera["vertical_fov"]),
            "aspect_ratio": float(camera["aspect_ratio"])}


def frame_conventions() -> dict:
    """frameConventions (frame_export.cpp:119-128)."""
    return {"radiance": "linear_scene_referred_rgb", "radiance_normalization": "mean", "exposure": 1.0,
            "image_origin": "top_left", "normal_space": "world", "depth": "camera_forward_distance",
            "motion": "previous_pixel_minus_current_pixel", "motion_units": "pixels",
            "pixel_coordinates": "integer_centers", "guides": "unjittered_pixel_centers",
            "radiance_sampling": "independent_uniform_subpixel_jitter", "scene_motion": "static",
            "history_valid": "previous_frustum_and_visibility"}


def _rgb(values, count, what):
    a = np.asarray(values, np.float32)
    if a.size != 3 * count:
        raise ValueError(f"{what}: expected {count} RGB pixels")
    return a.reshape(count, 3)


def _publish(directory: Path, image_name: str, write_image, manifest: dict) -> None:
    directory = Path(directory)
    staging = Path(str(directory) + ".partial")
    if directory.exists() or staging.exists():
        raise FileExistsError(f"output or staging directory already exists: {directory}")
    if str(directory.parent):
        directory.parent.mkdir(parents=True, exist_ok=True)
    staging.mkdir()
    try:
        write_image(staging / image_name)
        manifest["image"] = image_name
        manifest["image_sha256"] = hashlib.sha256((staging / image_name).read_bytes()).hexdigest()
        manifest["conventions"] = frame_conventions()
        with open(staging / "manifest.json", "w") as f:
            f.write(json.dumps(manifest, indent=2) + "\n")
        os.rename(staging, directory)
    except BaseException:
        shutil.rmtree(staging, ignore_errors=True)
        raise


def write_captured_frame(directory, width: int, height: int, samples: int, reference_samples: int, radiance,
                         reference, guides, metadata: dict) -> None:
    """writeCapturedFrame (frame_export.cpp:130-161): frame.exr with
    radiance.{R,G,B}, reference.{R,G,B}, the guide channels and the sample
    counts, and manifest.json (schema cuda-wavefront-frame, version 1)."""
    count = int(width) * int(height)
    if (width <= 0 or height <= 0 or width > 2**31 - 1 or height > 2**31 - 1 or samples <= 0
            or reference_samples <= 0):
        raise ValueError("invalid capture dimensions or sample counts")
    radiance = _rgb(radiance, count, "radiance")
    reference = _rgb(reference, count, "reference")
    g = np.asarray(guides)
    if g.dtype != abi.FRAME_GUIDE_DTYPE:
        g = np.ascontiguousarray(g).view(abi.FRAME_GUIDE_DTYPE)
    g = g.reshape(-1)
    if g.size != count:
        raise ValueError(f"guides: expected {count} records")
    finite = (np.isfinite(radiance).all() and np.isfinite(reference).all() and np.isfinite(g["albedo"]).all()
              and np.isfinite(g["normal"]).all() and np.isfinite(g["geometric_normal"]).all()
              and np.isfinite(g["depth"]).all() and np.isfinite(g["motion"]).all())
    flags = (np.isin(g["valid"], (0.0, 1.0)).all() and np.isin(g["history_valid"], (0.0, 1.0)).all()
             and not (g["history_valid"] > g["valid"]).any())
    if not finite or not flags or (g["depth"] < 0).any():
        raise ValueError("invalid or non-finite capture pixel")
    if not isinstance(metadata, dict):
        raise TypeError("capture metadata must be an object")
    F, U = EXR_FLOAT, EXR_UINT
    channels = {}
    for prefix, rgb in (("radiance", radiance), ("reference", reference)):
        for i, c in enumerate("RGB"):
            channels[f"{prefix}.{c}"] = (F, rgb[:, i])
    for i, c in enumerate("RGB"):
        channels[f"albedo.{c}"] = (F, g["albedo"][:, i])
    for i, c in enumerate("XYZ"):
        channels[f"normal.{c}"] = (F, g["normal"][:, i])
        channels[f"geometric_normal.{c}"] = (F, g["geometric_normal"][:, i])
    channels["depth.Z"] = (F, g["depth"])
    channels["motion.X"] = (F, g["motion"][:, 0])
    channels["motion.Y"] = (F, g["motion"][:, 1])
    channels["guide_valid.Y"] = (F, g["valid"])
    channels["history_valid.Y"] = (F, g["history_valid"])
    channels["sample_count.N"] = (U, np.full(count, samples, np.uint32))
    channels["reference_count.N"] = (U, np.full(count, reference_samples, np.uint32))
    manifest = dict(metadata)
    manifest.update({"schema": "cuda-wavefront-frame", "version": 1, "width": int(width), "height": int(height)})
    _publish(directory, "frame.exr", lambda p: write_exr(p, width, height, channels), manifest)


def write_captured_sample_layers(directory, width: int, height: int, layers, metadata: dict) -> None:
    """writeCapturedSampleLayers (frame_export.cpp:163-232): layers is a list
    of (samples, sample_start, radiance) with power-of-two sample counts of
    at most 32 and disjoint sample ranges; layers.exr holds spp_<n>.{R,G,B}
    per layer and the manifest describes each layer's provenance."""
    if (width <= 0 or height <= 0 or width > 2**31 - 1 or height > 2**31 - 1 or not layers
            or not isinstance(metadata, dict)):
        raise ValueError("invalid sample-layer dimensions or metadata")
    count = int(width) * int(height)
    descriptions = []
    planes = []
    for i, (samples, start, radiance) in enumerate(layers):
        rgb = np.asarray(radiance, np.float32)
        if (not samples or samples > 32 or samples & (samples - 1) or rgb.size != 3 * count
                or start + samples > 0xFFFFFFFF):
            raise ValueError("invalid sample-layer count, range or buffer")
        rgb = rgb.reshape(count, 3)
        if not np.isfinite(rgb).all() or (rgb < 0).any():
            raise ValueError("sample layers must be finite nonnegative RGB")
        for other_samples, other_start, _ in layers[:i]:
            if samples == other_samples or (start < other_start + other_samples and other_start < start + samples):
                raise ValueError("duplicate SPP or overlapping independent sample layers")
        prefix = f"spp_{samples}"
        descriptions.append({"samples": int(samples), "sample_start": int(start),
                             "channels": [f"{prefix}.R", f"{prefix}.G", f"{prefix}.B"]})
        planes.append(rgb)
    channels = {}
    for d, rgb in zip(descriptions, planes):
        for c, name in enumerate(d["channels"]):
            channels[name] = (EXR_FLOAT, rgb[:, c])
    manifest = json.loads(json.dumps(metadata))
    manifest.update({"schema": "cuda-wavefront-sample-layers", "version": 1, "width": int(width),
                     "height": int(height), "layers": descriptions})
    render = manifest.get("render")
    if isinstance(render, dict):
        for key in ("sample_start", "samples", "reference_sample_start", "reference_samples"):
            render.pop(key, None)
    _publish(directory, "layers.exr", lambda p: write_exr(p, width, height, channels), manifest)


def capture_frame(device_scene, camera, config, sample_start: int, samples: int, reference_samples: int,
                  previous=None):
    """One frame of the reference's dataset capture (tools/dataset_capture.cu:
    262-275): the mean radiance of samples [sample_start, +samples), the
    reference of the next reference_samples, and the guides with the previous
    frame's camera.  Returns (radiance, reference, guides) as (h, w, 3),
    (h, w, 3) and (h, w) FRAME_GUIDE_DTYPE arrays."""
    from .native import Renderer
    width, height = config.width, config.height
    renderer = Renderer(device_scene, camera, config)
    # Vec3 / float is a multiply by the float reciprocal (core/vec3.cuh:43-46)
    try:
        radiance = renderer.render_task((0, 0, width, height), sample_start, samples) * (
            np.float32(1) / np.float32(samples))
        reference = renderer.render_task((0, 0, width, height), sample_start + samples, reference_samples) * (
            np.float32(1) / np.float32(reference_samples))
    finally:
        renderer.close()
    guides = device_scene.frame_guides(camera, width, height, previous=previous)
    return radiance, reference, guides
