"""Asset loaders and the reference's asset-based scene presets.

Builds the scene description (wfpt.Scene) that the reference builds as a
HostScene from its assets:

* load_obj_scene / load_obj_mesh: Wavefront OBJ + MTL (loadObjScene /
  loadObjMesh, src/scene/obj_loader.cpp:54-212): one mesh per OBJ object or
  group, materials from Kd / Ke / Ni / map_Kd behind a default material 0,
  area-weighted generated vertex normals where the file has none, texture
  coordinates;
* load_gltf_scene: glTF 2.0, .gltf or .glb (loadGltfScene,
  src/scene/gltf_loader.cpp:293-503): one mesh per triangle primitive,
  instances from the node hierarchy (double-precision matrices), metallic-
  roughness and specular-glossiness materials with the KHR extensions the
  reference reads (transmission, volume, ior, specular, clearcoat,
  texture_transform), per-triangle tangent frames from the UVs, vertex
  tangents, both UV sets, and KHR_lights_punctual lights;
* preset_scene: a scene manifest (assets/scenes/<preset>.json, parsed as
  loadSceneManifest does, src/scene/scene_manifest.cpp) assembled as
  assembleGltfScene / assembleCornellScene / assembleObjScene
  (src/scene/scene_host.cpp:242-421) with the preset's camera
  (src/scene/camera.cu:3-28).

Every float is computed in float32 with the reference's operation order
(vector helpers of include/core/vec3.cuh: dot left to right, normalize as a
multiply by the reciprocal length, division by a scalar as a multiply by its
reciprocal), and node matrices in double, so geometry, frames and materials
equal the reference's bit for bit.  Images are decoded with Pillow; the
reference uses stb_image.  PNG and PPM texels agree exactly; JPEG decoders
may differ by a few levels in a few texels (different inverse DCT and chroma
upsampling).
"""
from __future__ import annotations

import base64
import json
import math
import os
import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import abi
from .native import Scene, material

F32 = np.float32


# ------------------------------------------------------------ float32 vectors
def _dot(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _normalize(v):
    inv = F32(1.0) / np.sqrt(_dot(v, v))
    return v * inv[..., None]


def _f3(x):
    return np.asarray(x, np.float64).astype(F32)


def load_image_rgba8(path=None, data=None):
    """(height, width, 4) uint8 RGBA texels, top row first (stbi_load with
    STBI_rgb_alpha)."""
    from PIL import Image
    import io
    image = Image.open(io.BytesIO(data) if data is not None else path)
    image.load()
    if image.mode not in ("RGBA",):
        image = image.convert("RGBA")
    return np.ascontiguousarray(np.asarray(image, np.uint8))


# ----------------------------------------------------------------------- OBJ
@dataclass
class LoadedScene:
    """The loaders' output (ObjScene / GltfScene): per-mesh triangles with
    attributes, materials with their texture records, RGBA8 textures,
    instances and punctual lights."""
    meshes: list = field(default_factory=list)          # TRIANGLE_DTYPE arrays
    mesh_attributes: list = field(default_factory=list)  # TRIANGLE_ATTRIBUTES_DTYPE arrays
    materials: np.ndarray = None                        # MATERIAL_DTYPE
    material_textures: np.ndarray = None                # MATERIAL_TEXTURES_DTYPE
    textures: list = field(default_factory=list)        # uint8 (h, w, 4)
    instances: np.ndarray = None                        # INSTANCE_DTYPE
    punctual: np.ndarray = None                         # PUNCTUAL_DTYPE


def _no_textures(count):
    t = np.zeros(count, abi.MATERIAL_TEXTURES_DTYPE)
    t["normal_scale"] = 1.0
    t["clearcoat_normal_scale"] = 1.0
    for slot in abi.TEXTURE_SLOTS:
        t[slot]["texture"] = abi.NO_TEXTURE
        t[slot]["scale"] = 1.0
    return t


def _parse_mtl(path, names, records, textures_by_name):
    """newmtl / Kd / Ke / Ni / map_Kd of one MTL file (the fields
    makeMaterial reads, obj_loader.cpp:14-25)."""
    current = None
    for raw in Path(path).read_text(errors="replace").splitlines():
        line = raw.strip()
        if not line or line.startswith("#"):
            continue
        key, _, rest = line.partition(" ")
        rest = rest.strip()
        if key == "newmtl":
            current = {"name": rest, "Kd": (0.0, 0.0, 0.0), "Ke": (0.0, 0.0, 0.0), "Ni": 1.0, "map_Kd": ""}
            names.append(rest)
            records.append(current)
        elif current is None:
            continue
        elif key in ("Kd", "Ke"):
            v = [float(x) for x in rest.split()[:3]]
            current[key] = tuple(v + [v[-1]] * (3 - len(v))) if v else (0.0, 0.0, 0.0)
        elif key == "Ni":
            current["Ni"] = float(rest.split()[0])
        elif key == "map_Kd":
            current["map_Kd"] = rest.split()[-1] if rest else ""


def _obj_index(token, count):
    i = int(token)
    return i - 1 if i > 0 else count + i


def load_obj_scene(path) -> LoadedScene:
    """loadObjScene (obj_loader.cpp:54-199): a mesh per object/group, the
    default material 0 (albedo (0.65, 0.3, 0.18)) and one material per MTL
    entry, the diffuse textures they name."""
    path = Path(path)
    directory = path.parent
    positions, normals, texcoords = [], [], []
    material_names, material_records = [], []
    shapes = []  # per shape: list of faces (list of (v, vt, vn)), material ids
    faces, face_materials = [], []
    current_material = -1

    def close_shape():
        nonlocal faces, face_materials
        if faces:
            shapes.append((faces, face_materials))
        faces, face_materials = [], []

    for raw in path.read_text(errors="replace").splitlines():
        line = raw.strip()
        if not line or line.startswith("#"):
            continue
        key, _, rest = line.partition(" ")
        if key == "v":
            positions.append([float(x) for x in rest.split()[:3]])
        elif key == "vn":
            normals.append([float(x) for x in rest.split()[:3]])
        elif key == "vt":
            t = [float(x) for x in rest.split()[:2]]
            texcoords.append(t + [0.0] * (2 - len(t)))
        elif key == "f":
            corners = []
            for token in rest.split():
                parts = token.split("/")
                v = _obj_index(parts[0], len(positions))
                vt = _obj_index(parts[1], len(texcoords)) if len(parts) > 1 and parts[1] else -1
                vn = _obj_index(parts[2], len(normals)) if len(parts) > 2 and parts[2] else -1
                corners.append((v, vt, vn))
            if len(corners) != 3:
                raise ValueError("OBJ loader expected triangulated faces")
            faces.append(corners)
            face_materials.append(current_material)
        elif key in ("o", "g"):
            close_shape()
        elif key == "usemtl":
            name = rest.strip()
            current_material = material_names.index(name) if name in material_names else -1
        elif key == "mtllib":
            for name in rest.split():
                if (directory / name).exists():
                    _parse_mtl(directory / name, material_names, material_records, None)
    close_shape()

    out = LoadedScene()
    mats = [material(abi.MAT_DIFFUSE, (0.65, 0.3, 0.18), (0.0, 0.0, 0.0), 0.0, 1.0)]
    for rec in material_records:
        emissive = any(x != 0.0 for x in rec["Ke"])
        mats.append(material(abi.MAT_EMISSIVE if emissive else abi.MAT_DIFFUSE, _f3(rec["Kd"]), _f3(rec["Ke"]), 0.0,
                             float(F32(rec["Ni"])) if F32(rec["Ni"]) > 0 else 1.0))
    out.materials = np.array(mats, abi.MATERIAL_DTYPE)
    out.material_textures = _no_textures(len(mats))
    texture_index = {}
    for i, rec in enumerate(material_records):
        name = rec["map_Kd"]
        if not name:
            continue
        if name not in texture_index:
            texture_index[name] = len(out.textures)
            out.textures.append(load_image_rgba8(directory / name))
        out.material_textures[i + 1]["albedo"]["texture"] = texture_index[name]

    P = np.asarray(positions, np.float64).astype(F32).reshape(-1, 3)
    N = np.asarray(normals, np.float64).astype(F32).reshape(-1, 3)
    T = np.asarray(texcoords, np.float64).astype(F32).reshape(-1, 2)

    # generated normals: every triangle's unnormalised face normal added to
    # its three vertices in file order, then normalised (obj_loader.cpp:120-147)
    all_v = np.array([[c[0] for c in f] for s in shapes for f in s[0]], np.int64).reshape(-1, 3)
    generated = np.zeros_like(P)
    if len(all_v):
        v0, v1, v2 = P[all_v[:, 0]], P[all_v[:, 1]], P[all_v[:, 2]]
        face_normal = _cross(v1 - v0, v2 - v0)
        np.add.at(generated, all_v.reshape(-1), np.repeat(face_normal, 3, axis=0))
        ls = _dot(generated, generated)
        nz = ls > 0
        generated[nz] = generated[nz] * (F32(1.0) / np.sqrt(ls[nz]))[:, None]

    for shape_faces, shape_materials in shapes:
        idx = np.array(shape_faces, np.int64).reshape(-1, 3, 3)
        n = len(idx)
        tri = np.zeros(n, abi.TRIANGLE_DTYPE)
        attrs = np.zeros(n, abi.TRIANGLE_ATTRIBUTES_DTYPE)
        vi, ti, ni = idx[:, :, 0], idx[:, :, 1], idx[:, :, 2]
        for k in range(3):
            tri[f"v{k}"] = P[vi[:, k]]
        has_n = (ni >= 0).all(axis=1)
        has_t = (ti >= 0).all(axis=1)
        for k in range(3):
            tri[f"n{k}"] = np.where(has_n[:, None], N[np.where(has_n, ni[:, k], 0)] if len(N) else 0,
                                    generated[vi[:, k]])
        tri["has_vertex_normals"] = 1
        mids = np.asarray(shape_materials, np.int64)
        tri["material"] = np.where(mids >= 0, mids + 1, 0).astype(np.uint32)
        attrs["has_texcoords"] = has_t
        if len(T):
            for k in range(3):
                uv = T[np.where(has_t, ti[:, k], 0)]
                attrs["uv"][:, k] = np.where(has_t[:, None], uv, 0)
        out.meshes.append(tri)
        out.mesh_attributes.append(attrs)
    if not out.meshes:
        raise ValueError(f"OBJ contains no triangles: {path}")
    return out


def load_obj_mesh(path) -> LoadedScene:
    """loadObjMesh (obj_loader.cpp:201-212): every shape in one mesh."""
    s = load_obj_scene(path)
    s.meshes = [np.concatenate(s.meshes)]
    s.mesh_attributes = [np.concatenate(s.mesh_attributes)]
    return s


# ---------------------------------------------------------------------- glTF
_COMPONENT_BYTES = {5120: 1, 5121: 1, 5122: 2, 5123: 2, 5125: 4, 5126: 4}
_TYPE_COUNT = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT2": 4, "MAT3": 9, "MAT4": 16}


class _Gltf:
    def __init__(self, path):
        path = Path(path)
        self.directory = path.parent
        data = path.read_bytes()
        binary = None
        if path.suffix.lower() == ".glb":
            magic, version, length = struct.unpack_from("<4sII", data, 0)
            if magic != b"glTF" or version != 2:
                raise ValueError(f"not a glTF 2 binary: {path}")
            pos = 12
            doc = None
            while pos < min(length, len(data)):
                chunk_length, chunk_type = struct.unpack_from("<II", data, pos)
                chunk = data[pos + 8:pos + 8 + chunk_length]
                if chunk_type == 0x4E4F534A:
                    doc = json.loads(chunk.decode("utf-8"))
                elif chunk_type == 0x004E4942 and binary is None:
                    binary = chunk
                pos += 8 + chunk_length
            self.doc = doc
        else:
            self.doc = json.loads(data.decode("utf-8"))
        self.buffers = []
        for i, b in enumerate(self.doc.get("buffers", [])):
            uri = b.get("uri")
            if uri is None:
                self.buffers.append(binary if binary is not None else b"")
            elif uri.startswith("data:"):
                self.buffers.append(base64.b64decode(uri.split(",", 1)[1]))
            else:
                self.buffers.append((self.directory / uri).read_bytes())

    def get(self, key):
        return self.doc.get(key, [])

    def accessor_bytes(self, index):
        """(bytes, offset, stride) of an accessor (getAccessorData /
        Accessor::ByteStride: the view's stride, else the element size)."""
        a = self.doc["accessors"][index]
        view = self.doc["bufferViews"][a["bufferView"]]
        element = _COMPONENT_BYTES[a["componentType"]] * _TYPE_COUNT[a["type"]]
        stride = view.get("byteStride", 0) or element
        return self.buffers[view["buffer"]], view.get("byteOffset", 0) + a.get("byteOffset", 0), stride, a

    def read_floats(self, index, rows, width):
        buf, off, stride, _ = self.accessor_bytes(index)
        rows = np.asarray(rows, np.int64)
        base = np.frombuffer(buf, np.uint8)
        byte_index = off + rows[:, None] * stride + np.arange(width * 4)[None, :]
        return base[byte_index].copy().view("<f4").reshape(len(rows), width)

    def read_indices(self, index):
        buf, off, stride, a = self.accessor_bytes(index)
        size = _COMPONENT_BYTES[a["componentType"]]
        kind = {1: "<u1", 2: "<u2", 4: "<u4"}[size if a["componentType"] in (5121, 5123, 5125) else 4]
        n = a["count"]
        base = np.frombuffer(buf, np.uint8)
        byte_index = off + np.arange(n, dtype=np.int64)[:, None] * stride + np.arange(np.dtype(kind).itemsize)[None, :]
        return base[byte_index].copy().view(kind).reshape(n).astype(np.int64)


def _binding(info, gltf, record):
    """getTextureBinding / getExtensionTexture (gltf_loader.cpp:59-119)."""
    if not isinstance(info, dict) or "index" not in info:
        return
    textures = gltf.get("textures")
    index = int(info["index"])
    if index < 0 or index >= len(textures) or textures[index].get("source", -1) < 0:
        return
    record["texture"] = textures[index]["source"]
    record["texcoord"] = int(info.get("texCoord", 0))
    transform = info.get("extensions", {}).get("KHR_texture_transform")
    if isinstance(transform, dict):
        def vec2(value, default):
            return (F32(value[0]), F32(value[1])) if isinstance(value, list) and len(value) == 2 else default
        record["offset"] = vec2(transform.get("offset"), tuple(record["offset"]))
        record["scale"] = vec2(transform.get("scale"), tuple(record["scale"]))
        if "rotation" in transform:
            record["rotation"] = F32(transform["rotation"])
        if "texCoord" in transform:
            record["texcoord"] = int(transform["texCoord"])
        record["has_transform"] = 1


def _gltf_materials(gltf):
    """The material loop of loadGltfScene (gltf_loader.cpp:328-425)."""
    sources = gltf.get("materials")
    mats = np.zeros(len(sources) + 1, abi.MATERIAL_DTYPE)
    mats[0] = material(abi.MAT_DIFFUSE, (0.7, 0.7, 0.7), (0.0, 0.0, 0.0), 0.0, 1.0)
    tex = _no_textures(len(sources) + 1)
    for i, src in enumerate(sources):
        ext = src.get("extensions", {})

        def number(name, prop, default):
            e = ext.get(name)
            return F32(e[prop]) if isinstance(e, dict) and prop in e else F32(default)

        def color(name, prop, default):
            e = ext.get(name)
            if not isinstance(e, dict) or prop not in e or not isinstance(e[prop], list) or len(e[prop]) != 3:
                return _f3(default)
            return _f3(e[prop])

        pbr = src.get("pbrMetallicRoughness", {})
        factor = pbr.get("baseColorFactor", [1.0, 1.0, 1.0, 1.0])
        m = material(abi.MAT_DIFFUSE)
        t = tex[i + 1]
        m["albedo"] = _f3(factor[:3])
        m["emission"] = _f3(src.get("emissiveFactor", [0.0, 0.0, 0.0]))
        transmission = number("KHR_materials_transmission", "transmissionFactor", 0.0)
        emission = m["emission"].astype(F32)
        if _dot(emission, emission) > 0:
            m["type"] = abi.MAT_EMISSIVE
        elif transmission > 0:
            m["type"] = abi.MAT_DIELECTRIC
        m["roughness"] = F32(pbr.get("roughnessFactor", 1.0))
        m["metallic"] = F32(pbr.get("metallicFactor", 1.0))
        t["normal_scale"] = F32(src.get("normalTexture", {}).get("scale", 1.0))
        m["alpha_cutoff"] = F32(src.get("alphaCutoff", 0.5))
        m["alpha_masked"] = 1 if src.get("alphaMode", "OPAQUE") == "MASK" else 0
        m["ior"] = number("KHR_materials_ior", "ior", 1.5)
        m["attenuation_color"] = color("KHR_materials_volume", "attenuationColor", (1.0, 1.0, 1.0))
        m["attenuation_distance"] = number("KHR_materials_volume", "attenuationDistance", 0.0)
        m["volume_density"] = number("KHR_materials_volume", "thicknessFactor", 1.0)
        _binding(ext.get("KHR_materials_volume", {}).get("thicknessTexture"), gltf, t["thickness"])
        _binding(pbr.get("baseColorTexture"), gltf, t["albedo"])
        _binding(pbr.get("metallicRoughnessTexture"), gltf, t["metallic_roughness"])
        _binding(src.get("emissiveTexture"), gltf, t["emissive"])
        _binding(src.get("normalTexture"), gltf, t["normal"])
        m["opacity"] = F32(factor[3])
        m["gltf_pbr"] = 1 if m["type"] == abi.MAT_DIFFUSE else 0
        m["specular_weight"] = number("KHR_materials_specular", "specularFactor", 1.0)
        m["specular_color"] = color("KHR_materials_specular", "specularColorFactor", (1.0, 1.0, 1.0))
        spec = ext.get("KHR_materials_specular", {})
        _binding(spec.get("specularTexture"), gltf, t["specular_weight"])
        _binding(spec.get("specularColorTexture"), gltf, t["specular_color"])
        m["clearcoat"] = number("KHR_materials_clearcoat", "clearcoatFactor", 0.0)
        m["clearcoat_roughness"] = number("KHR_materials_clearcoat", "clearcoatRoughnessFactor", 0.0)
        coat = ext.get("KHR_materials_clearcoat", {})
        _binding(coat.get("clearcoatTexture"), gltf, t["clearcoat"])
        _binding(coat.get("clearcoatRoughnessTexture"), gltf, t["clearcoat_roughness"])
        _binding(coat.get("clearcoatNormalTexture"), gltf, t["clearcoat_normal"])
        if isinstance(coat, dict) and isinstance(coat.get("clearcoatNormalTexture"), dict) \
                and "scale" in coat["clearcoatNormalTexture"]:
            t["clearcoat_normal_scale"] = F32(coat["clearcoatNormalTexture"]["scale"])

        def unit(x):
            return math.isfinite(x) and 0.0 <= x <= 1.0
        sc = m["specular_color"]
        if (not unit(m["specular_weight"]) or not unit(m["clearcoat"]) or not unit(m["clearcoat_roughness"])
                or not all(math.isfinite(x) and x >= 0 for x in sc)
                or not math.isfinite(t["clearcoat_normal_scale"])):
            raise ValueError("Invalid glTF specular/clearcoat factors")
        sg_name = "KHR_materials_pbrSpecularGlossiness"
        if sg_name in ext:
            sg = ext[sg_name]
            m["gltf_pbr"] = 0
            m["specgloss_workflow"] = 1
            m["albedo"] = 1.0
            m["opacity"] = 1.0
            if "diffuseFactor" in sg:
                d = sg["diffuseFactor"]
                if not isinstance(d, list) or len(d) != 4:
                    raise ValueError("Invalid glTF specular-glossiness diffuseFactor")
                m["albedo"] = _f3(d[:3])
                m["opacity"] = F32(d[3])
            m["specular"] = color(sg_name, "specularFactor", (1.0, 1.0, 1.0))
            m["glossiness"] = number(sg_name, "glossinessFactor", 1.0)
            t["albedo"] = _no_textures(1)[0]["albedo"]
            _binding(sg.get("diffuseTexture"), gltf, t["albedo"])
            _binding(sg.get("specularGlossinessTexture"), gltf, t["specular_glossiness"])
            values = list(m["albedo"]) + [m["opacity"]] + list(m["specular"]) + [m["glossiness"]]
            if not all(unit(x) for x in values):
                raise ValueError("Invalid glTF specular-glossiness factors")
            if m["type"] == abi.MAT_DIFFUSE:
                m["type"] = abi.MAT_SPECGLOSS
        mats[i + 1] = m
    return mats, tex


def _node_matrix(node):
    """getNodeMatrix (gltf_loader.cpp:134-155), column-major, in double."""
    if len(node.get("matrix", [])) == 16:
        return [float(x) for x in node["matrix"]]
    r = node.get("rotation", [])
    x, y, z, w = (r if len(r) == 4 else [0.0, 0.0, 0.0, 1.0])
    s = node.get("scale", [])
    sx, sy, sz = (s if len(s) == 3 else [1.0, 1.0, 1.0])
    t = node.get("translation", [])
    tx, ty, tz = (t if len(t) == 3 else [0.0, 0.0, 0.0])
    x, y, z, w, sx, sy, sz, tx, ty, tz = (float(v) for v in (x, y, z, w, sx, sy, sz, tx, ty, tz))
    return [sx * (1.0 - 2.0 * y * y - 2.0 * z * z), sx * (2.0 * x * y + 2.0 * w * z), sx * (2.0 * x * z - 2.0 * w * y),
            0.0,
            sy * (2.0 * x * y - 2.0 * w * z), sy * (1.0 - 2.0 * x * x - 2.0 * z * z), sy * (2.0 * y * z + 2.0 * w * x),
            0.0,
            sz * (2.0 * x * z + 2.0 * w * y), sz * (2.0 * y * z - 2.0 * w * x), sz * (1.0 - 2.0 * x * x - 2.0 * y * y),
            0.0,
            tx, ty, tz, 1.0]


def _multiply(a, b):
    """multiply (gltf_loader.cpp:124-132): each element summed from 0 in
    i order."""
    out = [0.0] * 16
    for column in range(4):
        for row in range(4):
            acc = 0.0
            for i in range(4):
                acc += a[i * 4 + row] * b[column * 4 + i]
            out[column * 4 + row] = acc
    return out


def _instance_from_matrix(mesh, m):
    """makeTransform (gltf_loader.cpp:157-167): the basis in float, the
    inverse rows as cross products divided by the float determinant."""
    x = _f3(m[0:3])
    y = _f3(m[4:7])
    z = _f3(m[8:11])
    yz, zx, xy = _cross(y, z), _cross(z, x), _cross(x, y)
    det = _dot(x, yz)
    inv = F32(1.0) / det
    row0, row1, row2 = yz * inv, zx * inv, xy * inv
    r = np.zeros(1, abi.INSTANCE_DTYPE)
    r["mesh"] = mesh
    r["material_override"] = abi.NO_MATERIAL
    r["accel"] = abi.ACCEL_BVH
    r["local_to_world"] = np.stack([x, y, z])
    r["world_to_local"] = np.stack([[row0[0], row1[0], row2[0]], [row0[1], row1[1], row2[1]],
                                    [row0[2], row1[2], row2[2]]])
    r["translation"] = _f3(m[12:15])
    return r


def _tangent_space(tri, attrs, second):
    """calculateTangentSpace (gltf_loader.cpp:205-232), vectorised."""
    have = attrs["has_texcoords1" if second else "has_texcoords"] != 0
    uv = attrs["uv1" if second else "uv"]
    uv0, uv1, uv2 = uv[:, 0], uv[:, 1], uv[:, 2]
    e1 = tri["v1"] - tri["v0"]
    e2 = tri["v2"] - tri["v0"]
    det = (uv1[:, 0] - uv0[:, 0]) * (uv2[:, 1] - uv0[:, 1]) - (uv1[:, 1] - uv0[:, 1]) * (uv2[:, 0] - uv0[:, 0])
    ok = have & ~(np.abs(det) < F32(0.000001))
    if not ok.any():
        return
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        inv = F32(1.0) / det
        tangent = (e1 * (uv2[:, 1] - uv0[:, 1])[:, None] - e2 * (uv1[:, 1] - uv0[:, 1])[:, None]) * inv[:, None]
        bitangent = (e2 * (uv1[:, 0] - uv0[:, 0])[:, None] - e1 * (uv2[:, 0] - uv0[:, 0])[:, None]) * inv[:, None]
        tangent = _normalize(tangent)
        bitangent = _normalize(bitangent)
    names = ("tangent1", "bitangent1") if second else ("tangent", "bitangent")
    attrs[names[0]][ok] = tangent[ok]
    attrs[names[1]][ok] = bitangent[ok]


def _light(gltf, index, world):
    """The KHR_lights_punctual part of addNodeInstances (gltf_loader.cpp:237-276)."""
    lights = gltf.doc.get("extensions", {}).get("KHR_lights_punctual", {}).get("lights", [])
    if index >= len(lights):
        raise ValueError("glTF node references an invalid punctual light")
    src = lights[index]
    kind = {"point": abi.LIGHT_POINT, "spot": abi.LIGHT_SPOT, "directional": abi.LIGHT_DIRECTIONAL}.get(src.get("type"))
    if kind is None:
        raise ValueError("Unknown glTF punctual light type")
    light = np.zeros(1, abi.PUNCTUAL_DTYPE)[0]
    light["type"] = kind
    light["position"] = _f3(world[12:15])
    direction = _f3([-world[8], -world[9], -world[10]])
    if not _dot(direction, direction) > 0:
        raise ValueError("Degenerate glTF light transform")
    light["direction"] = _normalize(direction)
    color = _f3(src["color"]) if src.get("color") else _f3([1.0, 1.0, 1.0])
    intensity = float(src.get("intensity", 1.0))
    rng = float(src.get("range", 0.0))
    spot = src.get("spot", {})
    inner, outer = float(spot.get("innerConeAngle", 0.0)), float(spot.get("outerConeAngle", math.pi / 4))
    if not math.isfinite(intensity) or intensity < 0 or not math.isfinite(rng) or rng < 0:
        raise ValueError("Invalid glTF light intensity or range")
    if not np.isfinite(color).all() or (color < 0).any():
        raise ValueError("Invalid glTF light color")
    if kind == abi.LIGHT_SPOT and (not math.isfinite(inner) or not math.isfinite(outer) or inner < 0
                                   or outer <= inner or outer > 1.5707963267948966):
        raise ValueError("Invalid glTF spotlight cone angles")
    light["intensity"] = color * F32(intensity)
    light["range"] = F32(rng)
    light["inner_cone_cos"] = np.cos(F32(inner))
    light["outer_cone_cos"] = np.cos(F32(outer))
    return light


def load_gltf_scene(path) -> LoadedScene:
    """loadGltfScene (gltf_loader.cpp:293-503)."""
    gltf = _Gltf(path)
    out = LoadedScene()
    out.materials, out.material_textures = _gltf_materials(gltf)
    for image in gltf.get("images"):
        if image.get("uri"):
            uri = image["uri"]
            if uri.startswith("data:"):
                # the reference's loader fails on data-URI images ("Failed to
                # load glTF image") and exits
                raise ValueError(f"Failed to load glTF image: {image.get('name', '')}")
            # the URI is used as written (tinygltf does not percent-decode it)
            out.textures.append(load_image_rgba8(gltf.directory / uri))
        elif image.get("bufferView", -1) >= 0:
            view = gltf.doc["bufferViews"][image["bufferView"]]
            buf = gltf.buffers[view["buffer"]]
            start = view.get("byteOffset", 0)
            out.textures.append(load_image_rgba8(data=buf[start:start + view["byteLength"]]))
        else:
            raise ValueError(f"Failed to load glTF image: {image.get('name', '')}")

    mesh_assets = []
    for mesh in gltf.get("meshes"):
        assets = []
        for prim in mesh.get("primitives", []):
            attributes = prim.get("attributes", {})
            if prim.get("mode", 4) != 4 or "POSITION" not in attributes or prim.get("indices", -1) < 0:
                continue
            idx = gltf.read_indices(prim["indices"])
            count = (len(idx) // 3) * 3
            if count == 0:
                continue
            corners = idx[:count].reshape(-1, 3)
            n = len(corners)
            flat = corners.reshape(-1)
            tri = np.zeros(n, abi.TRIANGLE_DTYPE)
            attrs = np.zeros(n, abi.TRIANGLE_ATTRIBUTES_DTYPE)
            p = gltf.read_floats(attributes["POSITION"], flat, 3).reshape(n, 3, 3)
            tri["v0"], tri["v1"], tri["v2"] = p[:, 0], p[:, 1], p[:, 2]
            m = prim.get("material", -1)
            tri["material"] = m + 1 if m >= 0 else 0
            if "NORMAL" in attributes:
                nrm = gltf.read_floats(attributes["NORMAL"], flat, 3).reshape(n, 3, 3)
                tri["n0"], tri["n1"], tri["n2"] = nrm[:, 0], nrm[:, 1], nrm[:, 2]
                tri["has_vertex_normals"] = 1
            if "TANGENT" in attributes:
                tg = gltf.read_floats(attributes["TANGENT"], flat, 4).reshape(n, 3, 4)
                attrs["vertex_tangent"] = tg[:, :, :3]
                attrs["vertex_tangent_sign"] = tg[:, :, 3]
                attrs["has_vertex_tangents"] = 1
            for name, field_name, flag in (("TEXCOORD_0", "uv", "has_texcoords"), ("TEXCOORD_1", "uv1", "has_texcoords1")):
                if name in attributes:
                    uv = gltf.read_floats(attributes[name], flat, 2).reshape(n, 3, 2)
                    uv[:, :, 1] = F32(1.0) - uv[:, :, 1]
                    attrs[field_name] = uv
                    attrs[flag] = 1
            _tangent_space(tri, attrs, False)
            _tangent_space(tri, attrs, True)
            assets.append(len(out.meshes))
            out.meshes.append(tri)
            out.mesh_attributes.append(attrs)
        mesh_assets.append(assets)

    instances, lights = [], []
    nodes = gltf.get("nodes")

    def visit(index, parent):
        node = nodes[index]
        world = _multiply(parent, _node_matrix(node))
        light = node.get("extensions", {}).get("KHR_lights_punctual", {}).get("light", -1)
        if light >= 0:
            lights.append(_light(gltf, light, world))
        if node.get("mesh", -1) >= 0:
            for mesh_index in mesh_assets[node["mesh"]]:
                instances.append(_instance_from_matrix(mesh_index, world))
        for child in node.get("children", []):
            visit(child, world)

    identity = [1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0]
    scenes = gltf.get("scenes")
    scene_index = gltf.doc.get("scene", 0)
    if 0 <= scene_index < len(scenes):
        for node_index in scenes[scene_index].get("nodes", []):
            visit(node_index, identity)
    out.instances = np.concatenate(instances) if instances else np.zeros(0, abi.INSTANCE_DTYPE)
    out.punctual = np.array(lights, abi.PUNCTUAL_DTYPE) if lights else np.zeros(0, abi.PUNCTUAL_DTYPE)
    return out


# ------------------------------------------------------------------ presets
def _quad(v0, eu, ev, mat):
    """addQuad (scene_host.cpp:21-24) of the corner, corner+u, corner+u+v,
    corner+v in float."""
    v0 = _f3(v0)
    eu = _f3(eu)
    ev = _f3(ev)
    a, b, d = v0, v0 + eu, v0 + ev
    c = (v0 + eu) + ev
    t = np.zeros(2, abi.TRIANGLE_DTYPE)
    t["v0"] = [a, a]
    t["v1"] = [b, c]
    t["v2"] = [c, d]
    t["material"] = mat
    return t


def _quad_points(p0, p1, p2, p3, mat):
    t = np.zeros(2, abi.TRIANGLE_DTYPE)
    t["v0"] = [_f3(p0), _f3(p0)]
    t["v1"] = [_f3(p1), _f3(p2)]
    t["v2"] = [_f3(p2), _f3(p3)]
    t["material"] = mat
    return t


def _scaled_instance(mesh, translation, scale):
    """makeScaledTransform (include/scene/scene.cuh:57-63)."""
    s = F32(scale)
    inv = F32(1.0) / s
    r = np.zeros(1, abi.INSTANCE_DTYPE)
    r["mesh"] = mesh
    r["material_override"] = abi.NO_MATERIAL
    r["accel"] = abi.ACCEL_BVH
    r["local_to_world"] = np.diag([s, s, s]).astype(F32)
    r["world_to_local"] = np.diag([inv, inv, inv]).astype(F32)
    r["translation"] = _f3(translation)
    return r


def _rotate_vector(v, axis, angle):
    """rotateVector (include/scene/scene.cuh:65-70) with the float sine and
    cosine of the float angle (correctly rounded)."""
    unit = _normalize(_f3(axis))
    c = F32(math.cos(float(angle)))
    s = F32(math.sin(float(angle)))
    v = _f3(v)
    return (v * c + _cross(unit, v) * s) + unit * (_dot(unit, v) * (F32(1.0) - c))


def _rotate_instance(r, axis, degrees):
    """rotateTransform (include/scene/scene.cuh:76-95)."""
    angle = F32(degrees) * (F32(3.14159265359) / F32(180.0))
    old = r["world_to_local"][0].copy()
    r["local_to_world"][0] = np.stack([_rotate_vector(r["local_to_world"][0][k], axis, angle) for k in range(3)])
    inverse = [_rotate_vector(e, axis, -angle) for e in np.eye(3, dtype=F32)]
    # transformBasis: bx * v.x + by * v.y + bz * v.z
    r["world_to_local"][0] = np.stack([(old[0] * inv[0] + old[1] * inv[1]) + old[2] * inv[2] for inv in inverse])


def _caustic_prism():
    """makeCausticPrism (scene_host.cpp:26-43)."""
    h = F32(1.25)
    a0, b0, c0 = (-h, -0.82, -0.68), (-h, -0.82, 0.68), (-h, 0.38, 0.0)
    a1, b1, c1 = (h, -0.82, -0.68), (h, -0.82, 0.68), (h, 0.38, 0.0)
    faces = [(a0, a1, b1), (a0, b1, b0), (b0, b1, c1), (b0, c1, c0), (c0, c1, a1), (c0, a1, a0), (a0, c0, b0),
             (a1, b1, c1)]
    t = np.zeros(len(faces), abi.TRIANGLE_DTYPE)
    for i, (p, q, r) in enumerate(faces):
        t[i]["v0"], t[i]["v1"], t[i]["v2"] = _f3(p), _f3(q), _f3(r)
    return t


def _scale_instances(instances, scale, translation=None):
    """The instance scaling of assembleGltfScene / assembleCornellScene
    (scene_host.cpp:310-318, 366-374)."""
    s = F32(scale)
    inv = F32(1.0) / s
    instances["local_to_world"] = instances["local_to_world"] * s
    instances["world_to_local"] = instances["world_to_local"] * inv
    instances["translation"] = instances["translation"] * s
    if translation is not None:
        instances["translation"] = instances["translation"] + _f3(translation)


def camera(kind, width, height):
    """createDemoCamera / createCornellCamera / createRtWeekCamera
    (src/scene/camera.cu:3-42) in float."""
    if kind == "cornell":
        position, target, fov_deg = _f3([0.0, 1.2, 6.5]), _f3([0.0, 0.8, -0.6]), F32(42.0)
        world_up = _f3([0.0, 1.0, 0.0])
    elif kind == "rtweek":  # createRtWeekCamera, camera.cu:30-42
        position, target, fov_deg = _f3([13.0, 2.0, 3.0]), _f3([0.0, 0.8, 0.0]), F32(32.0)
        world_up = None
    else:
        position, target, fov_deg = _f3([-10.0, 0.35, 0.8]), _f3([6.0, 3.2, 2.4]), F32(45.0)
        world_up = None
    forward = _normalize(target - position)
    if world_up is None:
        world_up = _f3([0.0, 0.0, 1.0]) if abs(forward[1]) > F32(0.999) else _f3([0.0, 1.0, 0.0])
    right = _normalize(_cross(forward, world_up))
    up = _cross(right, forward)
    fov = fov_deg * F32(3.14159265359) / F32(180.0)
    return {"position": position, "forward": forward, "right": right, "up": up, "vertical_fov": fov,
            "aspect_ratio": F32(width) / F32(height)}


@dataclass
class PresetConfig:
    """SceneConfig fields a manifest sets (include/config.hpp:40-57 defaults)."""
    name: str = "sponza"
    preset: str = "sponza"
    object_file: str = ""
    object_source: str = "obj"
    gltf_scale: float = 1.0
    object_scale: float = 0.1
    object_translation: tuple = (0.181, -0.906, -0.2)
    dielectric: bool = False
    material_override: int = -1
    neutral_room: bool = False
    remove_backdrop: bool = False
    light_profile: str = "standard"
    add_sponza_top_light: bool = True
    ignore_sponza_light_occlusion: bool = False
    use_normal_maps: bool = True
    normal_map_minimum_cosine: float = 0.0
    acceleration: str = "tlas_blas_bvh2"
    environment_file: str = ""
    environment_intensity: float = 1.0
    environment_rotation_degrees: float = 0.0


def load_manifest(path) -> PresetConfig:
    """loadSceneManifest (src/scene/scene_manifest.cpp:77-224): asset paths
    relative to the manifest."""
    path = Path(path)
    root = json.loads(path.read_text())
    if not isinstance(root, dict) or not isinstance(root.get("preset"), str):
        raise ValueError("scene manifest requires a string 'preset' field")
    c = PresetConfig(preset=root["preset"], name=root.get("name", root["preset"]))

    def resolve(name):
        if not name or name.startswith("__") or os.path.isabs(name):
            return name
        return os.path.normpath(str(path.parent / name))
    obj = root.get("object")
    if obj is not None:
        c.object_source = obj.get("source", "obj")
        if c.object_source == "glb":
            c.object_source = "gltf"
        if c.object_source not in ("obj", "gltf", "procedural_prism"):
            raise ValueError(f"scene manifest contains an unknown object source: {c.object_source}")
        if "file" in obj:
            c.object_file = resolve(obj["file"])
        c.object_scale = float(F32(obj.get("scale", c.object_scale)))
        if "translation" in obj:
            c.object_translation = tuple(float(F32(x)) for x in obj["translation"])
        c.dielectric = bool(obj.get("dielectric", c.dielectric))
        c.material_override = int(obj.get("material_override", c.material_override))
    c.gltf_scale = float(F32(root.get("gltf_scale", c.gltf_scale)))
    env = root.get("environment")
    if env is not None:
        c.environment_file = resolve(env["file"])
        c.environment_intensity = float(env.get("intensity", 1.0))
        c.environment_rotation_degrees = float(env.get("rotation_degrees", 0.0))
    room = root.get("room", {})
    c.neutral_room = bool(room.get("neutral", c.neutral_room))
    c.remove_backdrop = bool(room.get("remove_backdrop", c.remove_backdrop))
    lighting = root.get("lighting", {})
    c.light_profile = lighting.get("profile", "standard")
    c.add_sponza_top_light = bool(lighting.get("add_sponza_top_light", c.add_sponza_top_light))
    c.ignore_sponza_light_occlusion = bool(lighting.get("ignore_sponza_light_occlusion",
                                                        c.ignore_sponza_light_occlusion))
    maps = root.get("normal_maps", {})
    c.use_normal_maps = bool(maps.get("enabled", c.use_normal_maps))
    c.normal_map_minimum_cosine = float(F32(maps.get("minimum_cosine", c.normal_map_minimum_cosine)))
    c.acceleration = root.get("acceleration", c.acceleration)
    return c


def _from_loaded(scene, loaded, material_offset=0, override=-1):
    for tri in loaded.meshes:
        tri = tri.copy()
        tri["material"] = np.uint32(override) if override >= 0 else tri["material"] + material_offset
        scene.meshes.append(tri)
    scene.mesh_attributes = [a.copy() if a is not None else None for a in loaded.mesh_attributes]


def gltf_scene(path, scale=1.0, add_top_light=True):
    """assembleGltfScene (scene_host.cpp:351-391)."""
    loaded = load_gltf_scene(path)
    if not loaded.meshes or not len(loaded.instances):
        raise ValueError("glTF scene contains no renderable mesh instances")
    s = Scene()
    _from_loaded(s, loaded)
    s.instances = loaded.instances.copy()
    _scale_instances(s.instances, scale)
    s.materials = loaded.materials.copy()
    s.material_textures = loaded.material_textures.copy()
    s.textures = loaded.textures
    s.punctual = loaded.punctual.copy()
    if len(s.punctual):
        s.punctual["position"] = s.punctual["position"] * F32(scale)
    if add_top_light:
        light = s.add_material(material(abi.MAT_EMISSIVE, (1.0, 1.0, 1.0), (80.0, 80.0, 80.0)))
        s.material_textures = np.concatenate([s.material_textures, _no_textures(1)])
        s.static_triangles = _quad((-4.0, 9.2, -4.0), (8.0, 0.0, 0.0), (0.0, 0.0, 8.0), light)
    return s


def cornell_scene(config: PresetConfig):
    """assembleCornellScene (scene_host.cpp:242-349) for OBJ and glTF objects."""
    s = Scene()
    offset = 5
    profile = config.light_profile
    if config.object_source == "gltf":
        loaded = load_gltf_scene(config.object_file)
        instances = loaded.instances.copy()
        if config.remove_backdrop:
            instances = instances[instances["mesh"] != 0]
        _scale_instances(instances, config.object_scale, config.object_translation)
        punctual = loaded.punctual.copy()
        if len(punctual):
            punctual["position"] = punctual["position"] * F32(config.object_scale) + _f3(config.object_translation)
    else:
        if config.object_source == "obj":
            loaded = load_obj_scene(config.object_file)
        else:
            loaded = LoadedScene(meshes=[_caustic_prism()], mesh_attributes=[None],
                                 materials=np.array([material(abi.MAT_DIELECTRIC, (0.98, 0.99, 1.0), ior=1.52,
                                                              dispersion=0.035)], abi.MATERIAL_DTYPE),
                                 material_textures=_no_textures(1))
        instances = []
        for i in range(len(loaded.meshes)):
            r = _scaled_instance(i, config.object_translation, config.object_scale)
            if profile == "prism":
                _rotate_instance(r, (0.0, 1.0, 0.0), -20.0)
            instances.append(r)
        instances = np.concatenate(instances)
        punctual = np.zeros(0, abi.PUNCTUAL_DTYPE)
    object_materials = loaded.materials.copy()
    object_textures = loaded.material_textures.copy()
    # the procedural prism's own material is not an imported one: the
    # dielectric conversion of imported materials leaves it alone
    if config.dielectric and config.object_source != "procedural_prism":
        object_materials["type"] = abi.MAT_DIELECTRIC
        object_materials["albedo"] = 1.0
        object_materials["emission"] = 0.0
        object_materials["roughness"] = 0.0
        object_materials["ior"] = F32(1.52)
        object_materials["dispersion"] = F32(0.02)
        object_textures["albedo"]["texture"] = abi.NO_TEXTURE
    _from_loaded(s, loaded, offset, config.material_override)
    s.instances = instances
    s.punctual = punctual
    s.textures = loaded.textures
    w, fy, cy, bz, fz = 2.5, -1.0, 3.0, -2.5, 2.5
    walls = [
        _quad_points((-w, fy, fz), (w, fy, fz), (w, fy, bz), (-w, fy, bz), 0),
        _quad_points((-w, cy, bz), (w, cy, bz), (w, cy, fz), (-w, cy, fz), 0),
        _quad_points((-w, fy, bz), (w, fy, bz), (w, cy, bz), (-w, cy, bz), 0),
        _quad_points((-w, fy, fz), (-w, fy, bz), (-w, cy, bz), (-w, cy, fz), 1),
        _quad_points((w, fy, bz), (w, fy, fz), (w, cy, fz), (w, cy, bz), 2),
    ]
    crystal, prism = config.dielectric, profile == "prism"
    corner = (-0.5, 2.35, -1.6) if crystal else ((-0.9, 2.35, -1.6) if prism else (-0.75, 2.95, -0.75))
    eu = (1.0, 0.0, 0.0) if crystal else ((1.8, 0.0, 0.0) if prism else (1.5, 0.0, 0.0))
    ev = (0.0, 0.25, 0.42) if crystal else ((0.0, 0.45, 0.75) if prism else (0.0, 0.0, 1.5))
    walls.append(_quad(corner, eu, ev, 4))
    s.static_triangles = np.concatenate(walls)
    emission = 32.0 if crystal else (10.0 if prism else 16.0)
    room = [material(abi.MAT_DIFFUSE, (0.73, 0.73, 0.73)),
            material(abi.MAT_DIFFUSE, (0.68, 0.68, 0.68) if config.neutral_room else (0.65, 0.05, 0.05)),
            material(abi.MAT_DIFFUSE, (0.58, 0.58, 0.58) if config.neutral_room else (0.12, 0.45, 0.15)),
            material(abi.MAT_DIFFUSE, (0.72, 0.72, 0.72)),
            material(abi.MAT_EMISSIVE, (1.0, 1.0, 1.0), (emission, emission, emission))]
    s.materials = np.concatenate([np.array(room, abi.MATERIAL_DTYPE), object_materials])
    s.material_textures = np.concatenate([_no_textures(offset), object_textures])
    s.black_background = True
    return s


def obj_scene(config: PresetConfig):
    """assembleObjScene (scene_host.cpp:393-421), TLAS/BLAS acceleration."""
    loaded = load_obj_mesh(config.object_file)
    s = Scene()
    s.spheres = np.array([((0.0, -100.5, 0.0), 100.0, 0, abi.ACCEL_DIRECT)], abi.SPHERE_DTYPE)
    s.materials = np.concatenate([np.array([material(abi.MAT_DIFFUSE, (0.75, 0.75, 0.75))], abi.MATERIAL_DTYPE),
                                  loaded.materials])
    s.material_textures = np.concatenate([_no_textures(1), loaded.material_textures])
    s.textures = loaded.textures
    _from_loaded(s, loaded, 1)
    if config.acceleration != "tlas_blas_bvh2":
        raise NotImplementedError("OBJ presets with acceleration other than tlas_blas_bvh2")
    s.instances = _scaled_instance(0, config.object_translation, config.object_scale)
    # assembleObjScene registers no triangle lights: emissive OBJ materials
    # are only seen by paths that hit them
    s.register_triangle_lights = False
    return s


def demo_scene():
    """assembleDemoScene (scene_host.cpp:116-163): a cube, a pyramid, a glass
    sphere and a ground sphere under the sky."""
    s = Scene()
    s.spheres = np.array([((0.0, -100.5, 0.0), 100.0, 3, abi.ACCEL_DIRECT), ((1.35, 0.08, 0.0), 0.5, 2, abi.ACCEL_BVH)],
                         abi.SPHERE_DTYPE)
    c = [(-1.85, -0.42, -0.5), (-0.85, -0.42, -0.5), (-0.85, 0.58, -0.5), (-1.85, 0.58, -0.5),
         (-1.85, -0.42, 0.5), (-0.85, -0.42, 0.5), (-0.85, 0.58, 0.5), (-1.85, 0.58, 0.5)]
    cube = [(4, 5, 6), (4, 6, 7), (0, 2, 1), (0, 3, 2), (0, 4, 7), (0, 7, 3), (1, 2, 6), (1, 6, 5), (3, 7, 6),
            (3, 6, 2), (0, 1, 5), (0, 5, 4)]
    p = [(-0.183, -0.42, -0.683), (0.683, -0.42, -0.183), (0.183, -0.42, 0.683), (-0.683, -0.42, 0.183),
         (0.0, 0.73, 0.0)]
    pyramid = [(0, 1, 4), (1, 2, 4), (2, 3, 4), (3, 0, 4), (0, 2, 1), (0, 3, 2)]
    tris = [(c[a], c[b], c[d], 0) for a, b, d in cube] + [(p[a], p[b], p[d], 1) for a, b, d in pyramid]
    t = np.zeros(len(tris), abi.TRIANGLE_DTYPE)
    for i, (v0, v1, v2, m) in enumerate(tris):
        t[i]["v0"], t[i]["v1"], t[i]["v2"], t[i]["material"] = _f3(v0), _f3(v1), _f3(v2), m
    s.triangles = t
    s.materials = np.array([material(abi.MAT_DIFFUSE, (0.7, 0.2, 0.15)),
                            material(abi.MAT_METAL, (0.85, 0.65, 0.25), roughness=0.08),
                            material(abi.MAT_DIELECTRIC, (1.0, 1.0, 1.0), ior=1.5),
                            material(abi.MAT_DIFFUSE, (0.75, 0.75, 0.75))], abi.MATERIAL_DTYPE)
    return s


def rtweek_scene(obj_path):
    """assembleRtWeekScene (scene_host.cpp:165-240): the seeded small-sphere
    field of Ray Tracing in One Weekend and three instances of an OBJ mesh
    with material overrides, under the sky, with no area lights."""
    from .scenes import SceneRng
    loaded = load_obj_mesh(obj_path)
    s = Scene()
    D, M, G = abi.MAT_DIFFUSE, abi.MAT_METAL, abi.MAT_DIELECTRIC
    s.materials = np.array([material(D, (0.50, 0.50, 0.50)), material(D, (0.72, 0.20, 0.12)),
                            material(D, (0.16, 0.35, 0.72)), material(D, (0.22, 0.62, 0.28)),
                            material(M, (0.82, 0.84, 0.88), roughness=0.08),
                            material(M, (0.88, 0.60, 0.20), roughness=0.05),
                            material(G, (1.0, 1.0, 1.0), ior=1.5), material(D, (0.80, 0.30, 0.30)),
                            material(M, (0.80, 0.82, 0.90), roughness=0.05), material(G, (1.0, 1.0, 1.0), ior=1.5)],
                           abi.MATERIAL_DTYPE)
    spheres = [((0.0, -1000.0, 0.0), 1000.0, 0, abi.ACCEL_DIRECT)]
    rng = SceneRng(0x4D595DF4)
    for x in range(-11, 11):
        for z in range(-11, 11):
            choose = F32(rng.next())
            # Vec3(x + random(), 0.2f, z + random()): the reference's compiler
            # evaluates the constructor's arguments right to left, so z's
            # draw comes first
            cz = F32(z) + F32(rng.next())
            cx = F32(x) + F32(rng.next())
            if choose < F32(0.70):
                color = F32(rng.next())
                mat = 1 if color < F32(0.34) else (2 if color < F32(0.67) else 3)
            elif choose < F32(0.85):
                mat = 4 if F32(rng.next()) < F32(0.5) else 5
            else:
                mat = 6
            spheres.append(((cx, F32(0.2), cz), 0.20, mat, abi.ACCEL_BVH))
    s.spheres = np.array(spheres, abi.SPHERE_DTYPE)
    mesh = loaded.meshes[0].copy()
    mesh["material"] = 0
    s.meshes = [mesh]
    s.mesh_attributes = [loaded.mesh_attributes[0].copy()]  # the OBJ's textures are not kept
    instances = []
    for offset, mat in zip([(-4.0, -0.043, 1.0), (4.0, -0.043, 1.0), (0.0, -0.043, 1.0)], (7, 8, 9)):
        r = _scaled_instance(0, offset, 0.0035)
        r["material_override"] = mat
        instances.append(r)
    s.instances = np.concatenate(instances)
    return s


def load_environment_map(path):
    """loadEnvironmentMap (src/scene/environment.cpp:66-82): a Radiance .hdr
    file as float RGBA texels (alpha 1), row 0 at the top, shape (h, w, 4).
    The reference decodes it with stb_image's stbi_loadf; this is the same
    decoding written from the file format: a text header that must start
    with "#?RADIANCE" or "#?RGBE" and declare FORMAT=32-bit_rle_rgbe, the
    resolution line "-Y height +X width", then scanlines that are either
    flat RGBE or, for widths 8..32767, run-length encoded per channel
    (2, 2, width >> 8, width & 255, then each channel as runs: a count above
    128 repeats the next byte count - 128 times, otherwise count literal
    bytes).  A texel is (r, g, b) * 2^(e - 136) in float32, or 0 when e is 0."""
    data = Path(path).read_bytes()
    pos = 0

    def line():
        nonlocal pos
        end = data.find(b"\n", pos)
        if end < 0:
            raise ValueError(f"Could not decode HDR environment: {path}")
        text = data[pos:end].decode("latin-1")
        pos = end + 1
        return text

    magic = line()
    if magic not in ("#?RADIANCE", "#?RGBE"):
        raise ValueError(f"Environment must be a readable Radiance .hdr file: {path}")
    valid = False
    while True:
        text = line()
        if text == "":
            break
        if text == "FORMAT=32-bit_rle_rgbe":
            valid = True
    parts = line().split()
    if not valid or len(parts) != 4 or parts[0] != "-Y" or parts[2] != "+X":
        raise ValueError(f"Could not decode HDR environment: {path}")
    height, width = int(parts[1]), int(parts[3])
    if width <= 0 or height <= 0:
        raise ValueError(f"Could not decode HDR environment: {path}")
    rgbe = np.zeros((height, width, 4), np.uint8)
    buf = np.frombuffer(data, np.uint8)
    flat = width < 8 or width >= 32768
    if not flat and pos + 4 <= len(buf):
        c1, c2, c3 = int(buf[pos]), int(buf[pos + 1]), int(buf[pos + 2])
        flat = c1 != 2 or c2 != 2 or (c3 & 0x80) != 0
    if flat:  # the rest of the file is plain RGBE quadruples
        need = width * height * 4
        if pos + need > len(buf):
            raise ValueError(f"Could not decode HDR environment: {path}")
        rgbe[:] = buf[pos:pos + need].reshape(height, width, 4)
    else:
        for y in range(height):
            if pos + 4 > len(buf) or buf[pos] != 2 or buf[pos + 1] != 2 or \
                    (int(buf[pos + 2]) << 8 | int(buf[pos + 3])) != width:
                raise ValueError(f"Could not decode HDR environment: {path}")
            pos += 4
            for ch in range(4):
                x = 0
                row = rgbe[y, :, ch]
                while x < width:
                    count = int(buf[pos])
                    pos += 1
                    if count > 128:
                        count -= 128
                        if x + count > width:
                            raise ValueError(f"Could not decode HDR environment: {path}")
                        row[x:x + count] = buf[pos]
                        pos += 1
                    else:
                        if count == 0 or x + count > width:
                            raise ValueError(f"Could not decode HDR environment: {path}")
                        row[x:x + count] = buf[pos:pos + count]
                        pos += count
                    x += count
    e = rgbe[..., 3].astype(np.int32)
    scale = np.where(e != 0, np.ldexp(np.float32(1.0), e - 136).astype(np.float32), np.float32(0.0))
    out = np.ones((height, width, 4), np.float32)
    out[..., :3] = rgbe[..., :3].astype(np.float32) * scale[..., None]
    out[..., :3][e == 0] = 0.0
    return out


def preset_scene(manifest, width, height):
    """The preset a manifest names, as RenderDriver builds it
    (createSceneFromConfig + applySceneConfig, src/scene/scene_factory.cpp:
    22-104, and createSceneCamera): (Scene, camera)."""
    c = load_manifest(manifest) if not isinstance(manifest, PresetConfig) else manifest
    if c.preset == "sponza":
        s = gltf_scene(c.object_file or c.name, c.gltf_scale, c.add_sponza_top_light)
        s.ignore_direct_light_occlusion = c.ignore_sponza_light_occlusion
        cam = camera("demo", width, height)
    elif c.preset in ("cornell", "hurricane", "crystal", "prism"):
        s = cornell_scene(c)
        cam = camera("cornell", width, height)
    elif c.preset == "deer":
        s = obj_scene(c)
        cam = camera("demo", width, height)
    elif c.preset == "demo":
        s = demo_scene()
        cam = camera("demo", width, height)
    elif c.preset == "rtweek":
        s = rtweek_scene(c.object_file)
        cam = camera("rtweek", width, height)
    else:
        raise NotImplementedError(f"preset {c.preset} has no asset path")
    s.disable_normal_maps = not c.use_normal_maps
    s.normal_map_minimum_cosine = c.normal_map_minimum_cosine
    if c.environment_file:  # scene_factory.cpp:102-104
        s.environment = dict(rgba=load_environment_map(c.environment_file), intensity=c.environment_intensity,
                             rotation=c.environment_rotation_degrees)
    return s, cam
