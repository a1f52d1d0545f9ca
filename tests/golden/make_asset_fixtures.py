"""Writes the loader fixtures under tests/golden/assets/ (run from anywhere;
the output is committed).  Small assets of this project's own making that
exercise every path of the OBJ and glTF loaders the reference's assets leave
out: objects and groups (and an empty group), faces with and without normals
and texture coordinates, negative indices, unknown materials, emissive and
refractive MTL entries, a PNG and a PPM texture; glTF node hierarchies with
TRS and matrix transforms, interleaved and strided vertex data, 8-, 16- and
32-bit indices, vertex tangents, two UV sets, skipped primitives, every
material extension the loader reads with KHR_texture_transform, point, spot
and directional lights, external, data-URI and buffer-view images, and a
binary .glb; plus scene manifests that assemble them as presets."""
import io
import json
import math
import struct
from pathlib import Path

import numpy as np
from PIL import Image

OUT = Path(__file__).resolve().parent / "assets"


def png_bytes(rgba):
    buf = io.BytesIO()
    Image.fromarray(np.asarray(rgba, np.uint8)).save(buf, format="PNG")
    return buf.getvalue()


def textures():
    y, x = np.mgrid[0:16, 0:16]
    checker = np.zeros((16, 16, 4), np.uint8)
    on = ((x // 4 + y // 4) % 2) == 0
    checker[..., 0] = np.where(on, 230, 40)
    checker[..., 1] = np.where(on, 200, 60 + 8 * x)
    checker[..., 2] = np.where(on, 90, 30 + 8 * y)
    checker[..., 3] = np.where((x - 8) ** 2 + (y - 8) ** 2 < 20, 40, 255)
    normal = np.zeros((8, 8, 4), np.uint8)
    normal[..., 0] = 128 + 40 * np.sin(np.arange(8) * 0.9)[None, :]
    normal[..., 1] = 128 + 30 * np.cos(np.arange(8) * 0.7)[:, None]
    normal[..., 2] = 230
    normal[..., 3] = 255
    mr = np.zeros((4, 4, 4), np.uint8)
    mr[..., 1] = np.arange(16).reshape(4, 4) * 15
    mr[..., 2] = 255 - np.arange(16).reshape(4, 4) * 12
    mr[..., 3] = 255
    return checker, normal, mr


def write_obj():
    checker, _, _ = textures()
    (OUT / "checker.png").write_bytes(png_bytes(checker))
    (OUT / "mixed.mtl").write_text(
        "# materials for mixed.obj\n"
        "newmtl painted\nKd 0.8 0.7 0.6\nNi 1.33\nmap_Kd checker.png\n\n"
        "newmtl glow\nKd 1 1 1\nKe 4.0 3.5 2.0\n\n"
        "newmtl plain\nKa 0.1 0.1 0.1\n\n"
        "newmtl painted_again\nKd 0.2 0.3 0.9\nmap_Kd checker.png\n")
    lines = ["# mixed.obj: faces before any object, two objects, an empty group", "mtllib mixed.mtl"]
    rng = np.random.default_rng(7)
    verts = []
    for i in range(12):
        a = 2 * math.pi * i / 12
        verts.append((math.cos(a) * 0.8, 0.1 * (i % 3), math.sin(a) * 0.8))
    verts += [(0.0, 0.6, 0.0), (0.0, -0.4, 0.0)]
    verts += [tuple(rng.uniform(-1, 1, 3).round(6)) for _ in range(6)]
    for v in verts:
        lines.append("v %.6f %.6f %.6f" % v)
    for i in range(12):
        lines.append("vt %.5f %.5f" % (i / 12, (i % 3) / 2))
    lines.append("vt 0.5 1.0")
    for n in [(0, 1, 0), (0, -1, 0), (0.6, 0.8, 0.0)]:
        lines.append("vn %.6f %.6f %.6f" % n)
    # untitled shape: no material, position-only faces (generated normals)
    lines += ["f 1 2 13", "f 2 3 13"]
    lines += ["o cap_top", "usemtl painted"]
    for i in range(2, 8):
        lines.append(f"f {i + 1}/{i + 1}/1 {(i + 1) % 12 + 1}/{(i + 1) % 12 + 1}/1 13/13/1")
    lines += ["usemtl glow", "f 9//2 10//2 14//2", "f 10//2 11//2 14//2"]
    lines += ["g empty_group", "g cap_bottom", "usemtl plain"]
    lines += ["f -8/3 -7/4 -6/5", "f 11/11 12/12 14/1"]
    lines += ["usemtl does_not_exist", "f 15 16 17", "usemtl painted_again", "f 18/1/3 19/2/3 20/3/3",
              "f 15//3 17//3 19//3"]
    (OUT / "mixed.obj").write_text("\n".join(lines) + "\n")


class Buffer:
    def __init__(self):
        self.data = bytearray()
        self.views = []
        self.accessors = []

    def align(self, n=4):
        while len(self.data) % n:
            self.data.append(0)

    def view(self, payload, stride=None):
        self.align()
        v = {"buffer": 0, "byteOffset": len(self.data), "byteLength": len(payload)}
        if stride:
            v["byteStride"] = stride
        self.data += payload
        self.views.append(v)
        return len(self.views) - 1

    def accessor(self, view, component, count, kind, offset=0):
        a = {"bufferView": view, "componentType": component, "count": count, "type": kind}
        if offset:
            a["byteOffset"] = offset
        self.accessors.append(a)
        return len(self.accessors) - 1


def grid_primitive(buf, n, z_wave, index_type, interleave=False, tangents=False, uv1=False, material=None):
    """An (n+1)^2 vertex grid in the XY plane with a height wave in z."""
    ys, xs = np.mgrid[0:n + 1, 0:n + 1]
    pos = np.stack([xs / n - 0.5, ys / n - 0.5, z_wave * np.sin(xs * 1.3) * np.cos(ys * 0.7)], -1)
    pos = pos.reshape(-1, 3).astype(np.float32)
    nrm = np.tile(np.float32([0, 0, 1]), (len(pos), 1))
    uv = np.stack([xs / n * 1.5, ys / n * 0.75], -1).reshape(-1, 2).astype(np.float32)
    quads = [(y * (n + 1) + x, y * (n + 1) + x + 1, (y + 1) * (n + 1) + x + 1, (y + 1) * (n + 1) + x)
             for y in range(n) for x in range(n)]
    idx = np.array([t for a, b, c, d in quads for t in ((a, b, c), (a, c, d))]).reshape(-1)
    attrs = {}
    if interleave:
        inter = np.concatenate([pos, nrm, uv], axis=1).astype(np.float32)
        v = buf.view(inter.tobytes(), stride=32)
        attrs["POSITION"] = buf.accessor(v, 5126, len(pos), "VEC3", 0)
        attrs["NORMAL"] = buf.accessor(v, 5126, len(pos), "VEC3", 12)
        attrs["TEXCOORD_0"] = buf.accessor(v, 5126, len(pos), "VEC2", 24)
    else:
        attrs["POSITION"] = buf.accessor(buf.view(pos.tobytes()), 5126, len(pos), "VEC3")
        attrs["NORMAL"] = buf.accessor(buf.view(nrm.tobytes()), 5126, len(pos), "VEC3")
        attrs["TEXCOORD_0"] = buf.accessor(buf.view(uv.tobytes()), 5126, len(pos), "VEC2")
    if tangents:
        tg = np.tile(np.float32([1, 0, 0, -1]), (len(pos), 1))
        tg[::3, 3] = 1.0
        attrs["TANGENT"] = buf.accessor(buf.view(tg.tobytes()), 5126, len(pos), "VEC4")
    if uv1:
        uv_b = (uv[:, ::-1] * np.float32(0.5) + np.float32(0.25)).astype(np.float32)
        attrs["TEXCOORD_1"] = buf.accessor(buf.view(uv_b.tobytes()), 5126, len(pos), "VEC2")
    dtype, comp = {"u8": (np.uint8, 5121), "u16": (np.uint16, 5123), "u32": (np.uint32, 5125)}[index_type]
    prim = {"attributes": attrs, "indices": buf.accessor(buf.view(idx.astype(dtype).tobytes()), comp, len(idx),
                                                         "SCALAR")}
    if material is not None:
        prim["material"] = material
    return prim


def quaternion(axis, angle):
    axis = np.asarray(axis, float) / np.linalg.norm(axis)
    s = math.sin(angle / 2)
    return [axis[0] * s, axis[1] * s, axis[2] * s, math.cos(angle / 2)]


def write_gltf():
    checker, normal, mr = textures()
    (OUT / "normal.png").write_bytes(png_bytes(normal))
    # a 2x2 binary PPM
    (OUT / "pixel.ppm").write_bytes(b"P6\n2 2\n255\n" + bytes([200, 120, 40, 10, 220, 90, 60, 60, 240, 255, 255, 255]))
    buf = Buffer()
    tx = {"KHR_texture_transform": {"offset": [0.1, -0.2], "scale": [2.0, 0.5], "rotation": 0.4}}
    prims = [
        grid_primitive(buf, 4, 0.05, "u16", tangents=True, uv1=True, material=0),
        grid_primitive(buf, 3, 0.10, "u8", interleave=True, material=1),
        grid_primitive(buf, 5, 0.02, "u32", uv1=True, material=2),
        grid_primitive(buf, 2, 0.00, "u16", material=3),
        grid_primitive(buf, 2, 0.03, "u16", tangents=True, material=4),
        grid_primitive(buf, 2, 0.00, "u16"),
    ]
    lines = dict(prims[3])
    lines["mode"] = 1  # LINES: skipped
    no_indices = {"attributes": dict(prims[3]["attributes"])}  # no indices: skipped
    meshes = [{"primitives": [prims[0], lines]}, {"primitives": [prims[1], prims[2]]},
              {"primitives": [no_indices, prims[3]]}, {"primitives": [prims[4]]}, {"primitives": [prims[5]]}]
    materials = [
        {"name": "pbr_textured", "pbrMetallicRoughness": {
            "baseColorFactor": [0.9, 0.8, 0.7, 1.0], "metallicFactor": 0.3, "roughnessFactor": 0.6,
            "baseColorTexture": {"index": 0, "extensions": tx},
            "metallicRoughnessTexture": {"index": 2, "texCoord": 1}},
         "normalTexture": {"index": 1, "scale": 0.7},
         "extensions": {"KHR_materials_specular": {"specularFactor": 0.5, "specularColorFactor": [1.0, 0.9, 0.8],
                                                   "specularTexture": {"index": 2}},
                        "KHR_materials_clearcoat": {"clearcoatFactor": 0.6, "clearcoatRoughnessFactor": 0.25,
                                                    "clearcoatTexture": {"index": 2},
                                                    "clearcoatNormalTexture": {"index": 1, "scale": 0.4}}}},
        {"name": "masked", "alphaMode": "MASK", "alphaCutoff": 0.35,
         "pbrMetallicRoughness": {"baseColorFactor": [1.0, 1.0, 1.0, 0.8], "baseColorTexture": {"index": 0}}},
        {"name": "glass", "extensions": {
            "KHR_materials_transmission": {"transmissionFactor": 1.0}, "KHR_materials_ior": {"ior": 1.45},
            "KHR_materials_volume": {"thicknessFactor": 0.3, "attenuationDistance": 0.9,
                                     "attenuationColor": [0.8, 0.9, 1.0], "thicknessTexture": {"index": 2}}}},
        {"name": "specgloss", "pbrMetallicRoughness": {"baseColorFactor": [1, 0, 0, 1]},
         "extensions": {"KHR_materials_pbrSpecularGlossiness": {
             "diffuseFactor": [0.5, 0.4, 0.3, 0.9], "specularFactor": [0.04, 0.08, 0.12], "glossinessFactor": 0.75,
             "diffuseTexture": {"index": 3},
             "specularGlossinessTexture": {"index": 0, "extensions": {
                 "KHR_texture_transform": {"offset": [0.1, 0.2], "texCoord": 1}}}}}},
        {"name": "emissive", "emissiveFactor": [2.0, 1.5, 0.5], "emissiveTexture": {"index": 3},
         "pbrMetallicRoughness": {"baseColorFactor": [0.2, 0.2, 0.2, 1.0]}},
    ]
    (OUT / "metal_rough.png").write_bytes(png_bytes(mr))
    images = [{"uri": "checker.png"}, {"uri": "normal.png"}, {"uri": "metal_rough.png"}, {"uri": "pixel.ppm"}]
    textures_ = [{"source": 0}, {"source": 1}, {"source": 2}, {"source": 3}, {"source": -1}]
    lights = [{"type": "point", "color": [1.0, 0.5, 0.25], "intensity": 8.0, "range": 10.0},
              {"type": "spot", "intensity": 20.0, "spot": {"innerConeAngle": 0.2, "outerConeAngle": 0.6}},
              {"type": "directional", "color": [0.9, 0.9, 1.0], "intensity": 2.5}]
    nodes = [
        {"name": "root", "translation": [0.2, -0.3, 0.1], "rotation": quaternion([0.3, 1.0, 0.2], 0.7),
         "scale": [1.2, 0.9, 1.1], "children": [1, 2, 5]},
        {"name": "floor", "mesh": 0, "rotation": quaternion([1, 0, 0], -math.pi / 2)},
        {"name": "arm", "matrix": [0.8, 0.1, 0.0, 0.0, -0.1, 0.8, 0.05, 0.0, 0.0, -0.05, 0.8, 0.0,
                                   0.5, 0.6, -0.4, 1.0], "children": [3, 4]},
        {"name": "hand", "mesh": 1, "translation": [0.0, 0.3, 0.2]},
        {"name": "lamp", "translation": [0.0, 2.0, 0.0], "rotation": quaternion([1, 0, 0], -1.2),
         "extensions": {"KHR_lights_punctual": {"light": 1}}},
        {"name": "shelf", "mesh": 2, "translation": [-0.6, 0.2, 0.3], "scale": [0.5, 0.5, 0.5],
         "children": [6]},
        {"name": "card", "mesh": 3, "translation": [0.0, 0.0, 0.4]},
        {"name": "sun", "rotation": quaternion([1, 0.2, 0], -0.9),
         "extensions": {"KHR_lights_punctual": {"light": 2}}},
        {"name": "bulb", "translation": [0.3, 2.5, -0.2], "extensions": {"KHR_lights_punctual": {"light": 0}}},
        {"name": "panel", "mesh": 3, "translation": [0.8, 0.9, -0.7], "rotation": quaternion([0, 1, 0], 0.5)},
        {"name": "unused", "mesh": 4},
        {"name": "untextured", "mesh": 4, "translation": [-0.9, 0.5, 0.6]},
    ]
    doc = {"asset": {"version": "2.0", "generator": "make_asset_fixtures.py"},
           "extensionsUsed": ["KHR_materials_pbrSpecularGlossiness", "KHR_lights_punctual", "KHR_texture_transform",
                              "KHR_materials_specular", "KHR_materials_clearcoat", "KHR_materials_transmission",
                              "KHR_materials_ior", "KHR_materials_volume"],
           "extensions": {"KHR_lights_punctual": {"lights": lights}},
           "scene": 1, "scenes": [{"nodes": [10]}, {"nodes": [0, 7, 8, 9, 11]}],
           "nodes": nodes, "meshes": meshes, "materials": materials, "textures": textures_, "images": images,
           "buffers": [{"uri": "nodes.bin", "byteLength": len(buf.data)}],
           "bufferViews": buf.views, "accessors": buf.accessors}
    (OUT / "nodes.bin").write_bytes(bytes(buf.data))
    (OUT / "nodes.gltf").write_text(json.dumps(doc, indent=1) + "\n")

    # binary container with an image in a buffer view
    g = Buffer()
    prim = grid_primitive(g, 3, 0.08, "u16", tangents=True, material=0)
    image_view = g.view(png_bytes(checker))
    g.align()
    doc = {"asset": {"version": "2.0"}, "scenes": [{"nodes": [0]}],
           "nodes": [{"mesh": 0, "scale": [2.0, 2.0, 2.0], "translation": [0.0, 0.5, 0.0]}],
           "meshes": [{"primitives": [prim]}],
           "materials": [{"pbrMetallicRoughness": {"baseColorTexture": {"index": 0}, "roughnessFactor": 0.4},
                          "normalTexture": {"index": 0}}],
           "textures": [{"source": 0}], "images": [{"bufferView": image_view, "mimeType": "image/png"}],
           "buffers": [{"byteLength": len(g.data)}], "bufferViews": g.views, "accessors": g.accessors}
    js = json.dumps(doc).encode()
    js += b" " * (-len(js) % 4)
    binary = bytes(g.data) + b"\0" * (-len(g.data) % 4)
    glb = struct.pack("<4sII", b"glTF", 2, 12 + 8 + len(js) + 8 + len(binary))
    glb += struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(binary), 0x004E4942) + binary
    (OUT / "embedded.glb").write_bytes(glb)


def write_manifests():
    manifests = {
        "fixture_sponza.json": {"name": "fixture_sponza", "preset": "sponza",
                                "object": {"source": "gltf", "file": "nodes.gltf"}, "gltf_scale": 2.0,
                                "lighting": {"add_sponza_top_light": True}},
        "fixture_cornell.json": {"name": "fixture_cornell", "preset": "cornell",
                                 "object": {"source": "gltf", "file": "nodes.gltf", "scale": 0.9,
                                            "translation": [0.1, -0.5, -0.3]},
                                 "room": {"remove_backdrop": True}, "lighting": {"profile": "standard"}},
        "fixture_glb.json": {"name": "fixture_glb", "preset": "hurricane",
                             "object": {"source": "glb", "file": "embedded.glb", "scale": 1.5,
                                        "translation": [0.0, -0.8, 0.0]},
                             "room": {"neutral": True},
                             "normal_maps": {"enabled": True, "minimum_cosine": 0.2}},
        "fixture_crystal.json": {"name": "fixture_crystal", "preset": "crystal",
                                 "object": {"source": "obj", "file": "mixed.obj", "scale": 0.9,
                                            "translation": [0.0, -0.4, 0.0], "dielectric": True},
                                 "room": {"neutral": True}, "lighting": {"profile": "crystal"}},
        "fixture_demo.json": {"name": "fixture_demo", "preset": "demo"},
        "fixture_rtweek.json": {"name": "fixture_rtweek", "preset": "rtweek",
                                "object": {"source": "obj", "file": "mixed.obj"},
                                "normal_maps": {"enabled": False}},
        "fixture_prism.json": {"name": "fixture_prism", "preset": "prism",
                               "object": {"source": "procedural_prism", "file": "__caustic_prism__", "scale": 1.0,
                                          "translation": [0.0, 0.0, 0.0], "dielectric": True},
                               "lighting": {"profile": "prism"}},
        "fixture_deer.json": {"name": "fixture_deer", "preset": "deer",
                              "object": {"source": "obj", "file": "mixed.obj", "scale": 1.5,
                                         "translation": [0.1, 0.2, 0.0]},
                              "acceleration": "tlas_blas_bvh2"},
    }
    for name, doc in manifests.items():
        (OUT / name).write_text(json.dumps(doc, indent=2) + "\n")


if __name__ == "__main__":
    OUT.mkdir(parents=True, exist_ok=True)
    write_obj()
    write_gltf()
    write_manifests()
    print("wrote", sorted(p.name for p in OUT.iterdir()))
