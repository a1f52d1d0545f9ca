"""Asset loaders and presets (wfpt.assets) against the reference's own
loaders and preset assembly (obj_loader.cpp, gltf_loader.cpp with
tinyobjloader / tinygltf / stb_image, and scene_host.cpp), which run in
oracle/_ref/libwfref_det.so.  Geometry, per-triangle attributes and tangent
frames, materials and texture bindings, instances, spheres and punctual
lights must be identical bit for bit.  Texels must be identical for PNG and
PPM images; JPEG texels (the reference's own assets) may differ by a few
levels, because the two JPEG decoders round their inverse DCTs differently.

The fixtures under tests/golden/assets are made by
tests/golden/make_asset_fixtures.py.  The reference's own asset presets are
compared too when its asset tree is present."""
import json
import os
from pathlib import Path

import numpy as np
import pytest

import oracle
from wfpt import abi, assets

GOLDEN = Path(__file__).resolve().parent / "golden" / "assets"
# The reference's asset presets: $WF_REFERENCE, or a checkout named
# "reference" beside this repository; the preset comparisons skip without it.
REFERENCE_ROOT = (Path(os.environ["WF_REFERENCE"]) if os.environ.get("WF_REFERENCE")
                  else Path(__file__).resolve().parents[2] / "reference")
REFERENCE_SCENES = REFERENCE_ROOT / "assets" / "scenes"
KIND = {"sponza": "gltf", "deer": "obj", "demo": "demo", "rtweek": "rtweek"}

needs_oracle = pytest.mark.skipif(not oracle.available(det=True), reason="oracle/_ref/libwfref_det.so not built")


def reference_scene(config):
    kind = KIND.get(config.preset, "cornell")
    return oracle.RefHostScene(kind, config.object_file,
                               scale=config.gltf_scale if kind == "gltf" else config.object_scale,
                               translation=config.object_translation, object_source=config.object_source,
                               neutral_room=config.neutral_room, remove_backdrop=config.remove_backdrop,
                               dielectric=config.dielectric, material_override=config.material_override,
                               light_profile=config.light_profile, add_top_light=config.add_sponza_top_light)


def same_bits(name, a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, f"{name}: shape {a.shape} != {b.shape}"
    if a.dtype.names:
        for f in a.dtype.names:
            same_bits(f"{name}.{f}", a[f], b[f])
        return
    ua = a.view(np.uint32) if a.dtype == np.float32 else a
    ub = b.view(np.uint32) if b.dtype == np.float32 else b
    bad = np.argwhere(ua != ub)
    assert len(bad) == 0, f"{name}: {len(bad)} values differ, first at {tuple(bad[0])}: {a[tuple(bad[0])]} vs {b[tuple(bad[0])]}"


def compare(scene, ref, jpeg_tolerance=0):
    same_bits("static_triangles", scene.static_triangles, ref["static_triangles"])
    assert len(scene.meshes) == len(ref["meshes"])
    for i, (m, r) in enumerate(zip(scene.meshes, ref["meshes"])):
        same_bits(f"mesh[{i}]", m, r)
        attrs = scene.mesh_attributes[i] if i < len(scene.mesh_attributes) else None
        if attrs is None:  # no attributes: the reference's value-initialised fields
            attrs = np.zeros(len(m), abi.TRIANGLE_ATTRIBUTES_DTYPE)
        same_bits(f"mesh_attributes[{i}]", attrs, ref["mesh_attributes"][i])
    same_bits("triangles", scene.triangles, ref["triangles"])
    for name in ("instances", "materials", "spheres", "punctual"):
        same_bits(name, getattr(scene, name), ref[name])
    textures = scene.material_textures
    if textures is None:  # untextured: every binding empty
        textures = assets._no_textures(len(scene.materials))
    same_bits("material_textures", textures, ref["material_textures"])
    assert len(scene.textures) == len(ref["textures"])
    for i, (t, r) in enumerate(zip(scene.textures, ref["textures"])):
        assert t.shape == r.shape, f"texture {i}"
        diff = np.abs(t.astype(np.int16) - r.astype(np.int16))
        assert diff.max() <= jpeg_tolerance, f"texture {i}: texels differ by up to {diff.max()}"
    assert scene.black_background == ref["black_background"]


def light_counts(scene, host):
    """Triangle lights the reference registers for the product's scene
    description and for its own assembly (both uploaded by its uploadScene)."""
    mine = oracle.RefScene(scene, det=True)
    theirs = host.render_scene()
    try:
        return mine.light_count(), theirs.light_count()
    finally:
        mine.close()
        theirs.close()


@needs_oracle
@pytest.mark.parametrize("manifest", sorted(p.name for p in GOLDEN.glob("fixture_*.json")))
def test_fixture_presets_match_the_reference(manifest):
    config = assets.load_manifest(GOLDEN / manifest)
    scene, _ = assets.preset_scene(config, 64, 64)
    ref = reference_scene(config)
    try:
        compare(scene, ref.arrays())
        mine, theirs = light_counts(scene, ref)
        assert mine == theirs
    finally:
        ref.close()


@needs_oracle
@pytest.mark.skipif(not REFERENCE_SCENES.exists(), reason="the reference's asset tree is not present")
@pytest.mark.parametrize("preset", ["cornell", "crystal", "deer", "hurricane", "sponza"])
def test_reference_asset_presets_match_the_reference(preset):
    config = assets.load_manifest(REFERENCE_SCENES / f"{preset}.json")
    scene, _ = assets.preset_scene(config, 64, 64)
    ref = reference_scene(config)
    try:
        compare(scene, ref.arrays(), jpeg_tolerance=4)
    finally:
        ref.close()


def test_fixture_features_are_exercised():
    # the fixtures cover what the loaders branch on
    loaded = assets.load_gltf_scene(GOLDEN / "nodes.gltf")
    assert len(loaded.meshes) == 6 and len(loaded.instances) == 7
    assert sorted(loaded.punctual["type"].tolist()) == [abi.LIGHT_POINT, abi.LIGHT_SPOT, abi.LIGHT_DIRECTIONAL]
    m = loaded.materials
    assert m["type"].tolist() == [abi.MAT_DIFFUSE, abi.MAT_DIFFUSE, abi.MAT_DIFFUSE, abi.MAT_DIELECTRIC,
                                  abi.MAT_SPECGLOSS, abi.MAT_EMISSIVE]
    t = loaded.material_textures
    assert t[1]["albedo"]["has_transform"] == 1 and t[1]["metallic_roughness"]["texcoord"] == 1
    assert t[4]["specular_glossiness"]["texcoord"] == 1 and t[1]["clearcoat_normal"]["texture"] == 1
    attrs = np.concatenate(loaded.mesh_attributes)
    assert attrs["has_vertex_tangents"].any() and attrs["has_texcoords1"].any() and (attrs["tangent"] != 0).any()
    obj = assets.load_obj_scene(GOLDEN / "mixed.obj")
    assert len(obj.meshes) == 3 and len(obj.textures) == 1  # untitled shape, two objects; one shared texture
    mats = np.concatenate([x["material"] for x in obj.meshes])
    assert 0 in mats and 2 in mats  # no usemtl / unknown name -> 0; the emissive entry
    assert obj.materials[2]["type"] == abi.MAT_EMISSIVE


def test_loader_rejections(tmp_path):
    (tmp_path / "quad.obj").write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")
    with pytest.raises(ValueError, match="triangulated"):
        assets.load_obj_scene(tmp_path / "quad.obj")
    (tmp_path / "empty.obj").write_text("v 0 0 0\n")
    with pytest.raises(ValueError, match="no triangles"):
        assets.load_obj_scene(tmp_path / "empty.obj")
    import json
    doc = json.loads((GOLDEN / "nodes.gltf").read_text())
    (tmp_path / "nodes.bin").write_bytes((GOLDEN / "nodes.bin").read_bytes())
    for name in ("checker.png", "normal.png", "metal_rough.png", "pixel.ppm"):
        (tmp_path / name).write_bytes((GOLDEN / name).read_bytes())
    bad = json.loads(json.dumps(doc))
    bad["materials"][3]["extensions"]["KHR_materials_pbrSpecularGlossiness"]["glossinessFactor"] = 1.5
    (tmp_path / "bad_sg.gltf").write_text(json.dumps(bad))
    with pytest.raises(ValueError, match="specular-glossiness"):
        assets.load_gltf_scene(tmp_path / "bad_sg.gltf")
    bad = json.loads(json.dumps(doc))
    bad["materials"][0]["extensions"]["KHR_materials_clearcoat"]["clearcoatFactor"] = 2.0
    (tmp_path / "bad_coat.gltf").write_text(json.dumps(bad))
    with pytest.raises(ValueError, match="clearcoat"):
        assets.load_gltf_scene(tmp_path / "bad_coat.gltf")
    bad = json.loads(json.dumps(doc))
    bad["extensions"]["KHR_lights_punctual"]["lights"][1]["spot"]["outerConeAngle"] = 0.1
    (tmp_path / "bad_spot.gltf").write_text(json.dumps(bad))
    with pytest.raises(ValueError, match="cone"):
        assets.load_gltf_scene(tmp_path / "bad_spot.gltf")
    bad = json.loads(json.dumps(doc))
    bad["images"][2] = {"uri": "data:image/png;base64,AAAA"}
    (tmp_path / "data_uri.gltf").write_text(json.dumps(bad))
    with pytest.raises(ValueError, match="image"):
        assets.load_gltf_scene(tmp_path / "data_uri.gltf")


def test_preset_cameras_match_the_reference_formulas():
    # createCornellCamera / createDemoCamera (src/scene/camera.cu:3-28)
    cam = assets.camera("cornell", 200, 100)
    assert np.allclose(cam["forward"], np.array([0, -0.4, -7.1]) / np.linalg.norm([0, -0.4, -7.1]), atol=1e-6)
    assert cam["aspect_ratio"] == np.float32(2.0)
    demo = assets.camera("demo", 64, 64)
    assert abs(np.dot(demo["right"], demo["forward"])) < 1e-6 and demo["up"][1] > 0.9


def _write_hdr(path, rgbe, rle=True, header=b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n"):
    """A Radiance .hdr file from (h, w, 4) RGBE bytes: run-length encoded
    scanlines (runs of repeated bytes and literals, per channel) or flat."""
    h, w, _ = rgbe.shape
    out = bytearray(header + b"\n" + f"-Y {h} +X {w}\n".encode())
    if not rle:
        out += rgbe.astype(np.uint8).tobytes()
    else:
        for y in range(h):
            out += bytes([2, 2, w >> 8, w & 255])
            for ch in range(4):
                row = rgbe[y, :, ch].astype(np.uint8)
                x = 0
                while x < w:
                    run = 1
                    while x + run < w and run < 127 and row[x + run] == row[x]:
                        run += 1
                    if run >= 3:
                        out += bytes([128 + run, int(row[x])])
                        x += run
                        continue
                    lit = 1
                    while x + lit < w and lit < 128 and not (x + lit + 2 < w and row[x + lit] == row[x + lit + 1]
                                                             == row[x + lit + 2]):
                        lit += 1
                    out += bytes([lit]) + row[x:x + lit].tobytes()
                    x += lit
    path.write_bytes(bytes(out))


@needs_oracle
@pytest.mark.parametrize("rle,width", [(True, 64), (False, 64), (True, 8), (False, 5)])
def test_hdr_environment_matches_reference_loader(tmp_path, rle, width):
    """wfpt.assets.load_environment_map against the reference's
    loadEnvironmentMap (stb_image) on run-length-encoded and flat files:
    texels bit for bit, including zero-exponent texels and runs."""
    rng = np.random.default_rng(width + rle)
    h = 7
    rgbe = rng.integers(0, 256, (h, width, 4)).astype(np.uint8)
    rgbe[..., 3] = rng.integers(100, 160, (h, width))
    rgbe[0, : width // 2] = (10, 20, 30, 130)   # a run in every channel
    rgbe[1, 0] = (200, 100, 50, 0)              # exponent 0: black
    path = tmp_path / "env.hdr"
    _write_hdr(path, rgbe, rle=rle)
    got = assets.load_environment_map(path)
    want = oracle.load_environment(path)
    assert got.shape == (h, width, 4) and want is not None
    same_bits("environment texels", got, want)
    assert got[1, 0, :3].sum() == 0 and (got[..., 3] == 1).all()


@needs_oracle
def test_hdr_environment_rejections(tmp_path):
    bad = tmp_path / "bad.hdr"
    _write_hdr(bad, np.zeros((2, 8, 4), np.uint8), header=b"#?RADIANCE\nFORMAT=32-bit_rle_xyze\n")
    with pytest.raises(ValueError):
        assets.load_environment_map(bad)
    assert oracle.load_environment(bad) is None
    notes = tmp_path / "notes.hdr"
    notes.write_bytes(b"not an image\n")
    with pytest.raises(ValueError):
        assets.load_environment_map(notes)
    assert oracle.load_environment(notes) is None


def test_manifest_environment_becomes_the_scene_environment(tmp_path):
    """A manifest's environment block (scene_manifest.cpp:146-168): the file,
    resolved beside the manifest, its intensity and rotation."""
    rgbe = np.full((4, 8, 4), (128, 128, 128, 129), np.uint8)
    _write_hdr(tmp_path / "sky.hdr", rgbe)
    manifest = tmp_path / "scene.json"
    manifest.write_text(json.dumps({"name": "demo-sky", "preset": "demo",
                                    "environment": {"file": "sky.hdr", "intensity": 2.5, "rotation_degrees": 30}}))
    scene, cam = assets.preset_scene(manifest, 64, 48)
    env = scene.environment
    assert env["rgba"].shape == (4, 8, 4) and env["intensity"] == 2.5 and env["rotation"] == 30
    assert np.allclose(env["rgba"][..., :3], 128 * 2.0 ** (129 - 136))
