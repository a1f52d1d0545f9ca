"""Shared test helpers: scenes, ray batches, comparisons."""
import math

import numpy as np

from wfpt import abi, scenes
from wfpt.native import Scene, material


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def acceleration_rays(seed=12345, count=2048):
    """The ray set of the reference's scene_acceleration_tests
    (tests/scene_acceleration_tests.cu:188-204): 8 fixed rays plus `count`
    random rays with origins U(-4, 4)^3 and normalized U(-1, 1)^3 directions
    (numpy's Mersenne Twister stands in for std::mt19937)."""
    fixed = [((0, 0, 0), (0, 0, 1)), ((1, 0, 0), (0, 0, 1)), ((0, 0, 3), (1, 0, 0)), ((0, 0, 0), (0, -1, 0)),
             ((0, 0, 0), (0, 0, -1)), ((-3, 0, 0), (0, 0, 1)), ((3, 0, 0), (0, 0, 1)), ((0, 0, 8), (0, 0, -1))]
    rng = np.random.RandomState(seed)
    o = rng.uniform(-4, 4, (count, 3)).astype(np.float32)
    d = rng.uniform(-1, 1, (count, 3)).astype(np.float32)
    d = normalize_f32(d)
    rays = np.zeros(len(fixed) + count, abi.RAY_DTYPE)
    rays["origin"][:8] = [f[0] for f in fixed]
    rays["direction"][:8] = [f[1] for f in fixed]
    rays["origin"][8:] = o
    rays["direction"][8:] = d
    return rays


def normalize_f32(v):
    """normalize() of include/core/vec3.cuh:91-94 in float32."""
    v = np.asarray(v, np.float32)
    d = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]
    inv = np.float32(1.0) / np.sqrt(d.astype(np.float32))
    return v * inv[:, None]


def camera_rays(cam, width, height, jitter_seed=0):
    """Pixel-centre primary rays of a camera (inputs, not a parity subject)."""
    ys, xs = np.mgrid[0:height, 0:width]
    rng = np.random.RandomState(jitter_seed)
    u = ((xs + rng.uniform(0, 1, xs.shape)) / width).astype(np.float32).ravel()
    v = ((ys + rng.uniform(0, 1, ys.shape)) / height).astype(np.float32).ravel()
    th = np.float32(math.tan(float(cam["vertical_fov"]) * 0.5))
    x = (np.float32(2) * u - np.float32(1)) * cam["aspect_ratio"] * th
    y = (np.float32(1) - np.float32(2) * v) * th
    d = cam["forward"][None, :] + cam["right"][None, :] * x[:, None] + cam["up"][None, :] * y[:, None]
    rays = np.zeros(len(u), abi.RAY_DTYPE)
    rays["origin"] = cam["position"]
    rays["direction"] = normalize_f32(d)
    return rays


def triangle_at(z, mat):
    """triangleAt of scene_acceleration_tests.cu:237-251 (positions only)."""
    t = np.zeros(1, abi.TRIANGLE_DTYPE)
    t["v0"], t["v1"], t["v2"] = (-2, -1, z), (2, -1, z), (0, 2, z)
    t["material"] = mat
    return t


def acceleration_cases():
    """The scene cases of scene_acceleration_tests.cu:265-354 that use no
    textures (the alpha-masked material is modelled by its untextured
    opacity; the reference's 1x1 alpha-0 texture gives the same rejection)."""
    def base():
        s = Scene()
        for _ in range(4):
            s.add_material(material(abi.MAT_DIFFUSE, (0.5, 0.5, 0.5)))
        s.materials[3]["alpha_masked"] = 1
        s.materials[3]["opacity"] = 0.0
        s.black_background = True
        return s

    def spheres_of(s, rows):
        sp = np.zeros(len(rows), abi.SPHERE_DTYPE)
        for i, r in enumerate(rows):
            sp[i] = r
        s.spheres = sp

    cases = {}
    cases["empty scene"] = base()
    s = base()
    spheres_of(s, [((0, 0, 3), 1, 0, 0), ((-3, 0, 3), 0.5, 1, 1), ((0, -21, 0), 20, 2, 1)])
    cases["sphere partitions"] = s
    a = base(); a.spheres = s.spheres.copy(); a.spheres["accel"] = 1
    cases["all direct spheres"] = a
    b = base(); b.spheres = s.spheres.copy(); b.spheres["accel"] = 0
    cases["all accelerated spheres"] = b
    c = base(); c.spheres = np.concatenate([s.spheres, np.array([((0, 0, 3), 1, 1, 1)], abi.SPHERE_DTYPE)])
    cases["coincident spheres across partitions"] = c
    f = base()
    rows = [((0, -21, 0), 20, 2, 1)]
    for x in range(12):
        for z in range(12):
            for layer in range(2):
                rows.append(((-3.3 + 0.6 * x, -0.3 + 0.6 * layer, 1.0 + 0.6 * z), 0.15, (x + z + layer) % 3, 0))
    spheres_of(f, rows)
    cases["large sphere hierarchy"] = f
    m = base(); m.spheres = c.spheres.copy()
    mesh = m.add_mesh(np.concatenate([triangle_at(1, 3), triangle_at(5, 2)]))
    m.instances = np.concatenate([scenes.instance(mesh), scenes.instance(mesh, (4, 0, 1), 0.5, 0.0, 1, abi.ACCEL_DIRECT)])
    m.static_triangles = triangle_at(0.5, 3)
    cases["mixed geometry and shared mesh"] = m
    m2 = base(); m2.spheres = m.spheres.copy(); m2.meshes = list(m.meshes); m2.instances = m.instances.copy()
    m2.static_triangles = m.static_triangles.copy(); m2.triangles = triangle_at(7, 2)
    cases["mesh TLAS with additional flat triangles"] = m2
    dm = base(); dm.meshes = list(m.meshes)
    dm.instances = scenes.instance(0, (0, 0, 0), 1.0, 0.0, 1, abi.ACCEL_DIRECT)
    cases["direct mesh without BLAS or TLAS"] = dm
    am = base(); am.meshes = list(m.meshes); am.instances = scenes.instance(0, (0, 0, 0), 1.0, 0.0, 1, abi.ACCEL_BVH)
    cases["accelerated mesh without spheres"] = am
    em = base(); em.meshes = [np.zeros(0, abi.TRIANGLE_DTYPE)]; em.instances = scenes.instance(0)
    cases["empty accelerated mesh"] = em
    ed = base(); ed.meshes = [np.zeros(0, abi.TRIANGLE_DTYPE)]; ed.instances = scenes.instance(0, accel=abi.ACCEL_DIRECT)
    cases["empty direct mesh"] = ed
    ra = base(); spheres_of(ra, [((0, 0, 3), 1, 0, 0)]); ra.meshes = [triangle_at(5, 2)]
    ra.instances = scenes.instance(0, accel=abi.ACCEL_DIRECT)
    cases["sphere replaces direct mesh attributes"] = ra
    dt = base(); dt.spheres = c.spheres.copy(); dt.triangles = np.concatenate([triangle_at(1, 3), triangle_at(5, 2)])
    cases["sphere TLAS with triangle BVH"] = dt
    return cases


def hit_diff(a, b, fields=("t", "position", "geometric_normal", "normal", "material", "light_index")):
    """Indices where two HIT_DTYPE arrays differ in the given fields (bitwise)."""
    bad = np.zeros(len(a), bool)
    for f in fields:
        x, y = a[f], b[f]
        if x.dtype == np.float32:
            x, y = x.view(np.uint32), y.view(np.uint32)
        bad |= (x != y).reshape(len(a), -1).any(1)
    return np.nonzero(bad)[0]


def relative_rmse(image, reference):
    image = np.asarray(image, np.float64)
    reference = np.asarray(reference, np.float64)
    return float(np.sqrt(np.mean((image - reference) ** 2)) / max(1e-12, np.sqrt(np.mean(reference ** 2))))
