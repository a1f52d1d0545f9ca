"""Synthetic scene generators for the benchmark and parity workloads.

No public dataset is involved: every scene is generated from a seed.  Scene
randomness uses the reference's scene LCG, state * 1664525 + 1013904223 with
(state >> 8) / 2^24 (src/scene/scene_host.cpp:55-58), so a scene is fully
determined by its seed.

Workloads (sizes as stated in the task's configuration list):
  * cornell_box            256x256 Cornell box, 36 triangles, one emissive quad.
  * sphere_field           22x22 jittered spheres + ground sphere + 3 instances
                           of a displaced geodesic sphere (frequency 256 =
                           1,310,720 triangles), sky gradient.
  * large_mesh             2236x2236-quad fBm terrain (9,999,392 triangles,
                           1% emissive), 500 instances of a 200,000-triangle
                           displaced geodesic sphere, 20 glass spheres, HDR
                           environment with a 0.5 degree sun.
All sizes are parameters so tests can run reduced versions.
"""
import math

import numpy as np

from . import abi
from .native import Scene, material

# ------------------------------------------------------------------- RNG


class SceneRng:
    """The reference's scene LCG (scene_host.cpp:55-58), vectorised."""

    A = 1664525
    C = 1013904223

    def __init__(self, seed):
        self.state = np.uint32(seed)

    def next(self):
        self.state = np.uint32((int(self.state) * self.A + self.C) & 0xFFFFFFFF)
        return float(np.float32(int(self.state) >> 8) * np.float32(1.0 / 16777216.0))

    def stream(self, n):
        """n successive draws (same values as n calls of next())."""
        out = np.empty(n, np.float32)
        lanes = min(n, 4096) if n > 0 else 0
        if n == 0:
            return out
        # First `lanes` states sequentially, then leapfrog by `lanes` steps.
        states = np.empty(lanes, np.uint64)
        s = int(self.state)
        for i in range(lanes):
            s = (s * self.A + self.C) & 0xFFFFFFFF
            states[i] = s
        a_k, c_k = 1, 0
        for _ in range(lanes):
            a_k, c_k = (a_k * self.A) & 0xFFFFFFFF, (c_k * self.A + self.C) & 0xFFFFFFFF
        rows = (n + lanes - 1) // lanes
        block = np.empty((rows, lanes), np.uint64)
        cur = states.copy()
        for r in range(rows):
            block[r] = cur
            cur = (cur * np.uint64(a_k) + np.uint64(c_k)) & np.uint64(0xFFFFFFFF)
        flat = block.reshape(-1)[:n]
        self.state = np.uint32(int(flat[-1]))
        out[:] = (flat >> np.uint64(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)
        return out


# ------------------------------------------------------------ geometry


def triangles(v0, v1, v2, mat):
    t = np.zeros(len(v0), abi.TRIANGLE_DTYPE)
    t["v0"], t["v1"], t["v2"] = v0, v1, v2
    t["material"] = mat
    return t


def quad(v0, v1, v2, v3, mat):
    """addQuad (scene_host.cpp:21-24): (v0, v1, v2) and (v0, v2, v3)."""
    a = np.array([v0, v0], np.float32)
    b = np.array([v1, v2], np.float32)
    c = np.array([v2, v3], np.float32)
    return triangles(a, b, c, mat)


def box(center, size, yaw_deg, mat):
    """Axis-aligned box rotated about +Y: 12 outward-wound triangles."""
    cx, cy, cz = center
    sx, sy, sz = size
    corners = np.array([[x, y, z] for z in (-0.5, 0.5) for y in (-0.5, 0.5) for x in (-0.5, 0.5)], np.float64)
    corners *= np.array([sx, sy, sz])
    a = math.radians(yaw_deg)
    rot = np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])
    p = corners @ rot.T + np.array([cx, cy, cz])
    faces = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    out = [quad(p[f[0]], p[f[1]], p[f[2]], p[f[3]], mat) for f in faces]
    return np.concatenate(out)


def transform(translation=(0, 0, 0), scale=1.0, yaw_deg=0.0):
    """(local_to_world, world_to_local) basis vectors of S * R_y."""
    a = math.radians(yaw_deg)
    rot = np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])
    l2w = rot * scale
    w2l = np.linalg.inv(l2w)
    # Basis vectors: localToWorldX is the image of local +X = column 0.
    return l2w.T.astype(np.float32), w2l.T.astype(np.float32), np.array(translation, np.float32)


def instance(mesh, translation=(0, 0, 0), scale=1.0, yaw_deg=0.0, override=abi.NO_MATERIAL,
             accel=abi.ACCEL_BVH):
    r = np.zeros(1, abi.INSTANCE_DTYPE)
    l2w, w2l, t = transform(translation, scale, yaw_deg)
    r["mesh"] = mesh
    r["material_override"] = override
    r["accel"] = accel
    r["local_to_world"] = l2w
    r["world_to_local"] = w2l
    r["translation"] = t
    return r


def _hash3(ix, iy, iz, seed):
    h = (ix.astype(np.uint32) * np.uint32(73856093)) ^ (iy.astype(np.uint32) * np.uint32(19349663)) \
        ^ (iz.astype(np.uint32) * np.uint32(83492791)) ^ np.uint32(seed * 2654435761 & 0xFFFFFFFF)
    h ^= h >> np.uint32(13)
    h *= np.uint32(0x5BD1E995)
    h ^= h >> np.uint32(15)
    return (h & np.uint32(0xFFFFFF)).astype(np.float64) / float(0xFFFFFF) * 2.0 - 1.0


def value_noise(p, seed, octaves=3, frequency=2.0):
    """Seeded fractal value noise in [-1, 1] (trilinear lattice, smoothstep)."""
    total = np.zeros(len(p))
    amp, norm = 1.0, 0.0
    with np.errstate(over="ignore"):
        for o in range(octaves):
            q = p * frequency * (2 ** o)
            i = np.floor(q).astype(np.int64)
            f = q - i
            f = f * f * (3 - 2 * f)
            acc = np.zeros(len(p))
            for dz in (0, 1):
                for dy in (0, 1):
                    for dx in (0, 1):
                        w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * \
                            (f[:, 2] if dz else 1 - f[:, 2])
                        acc += w * _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed + o)
            total += amp * acc
            norm += amp
            amp *= 0.5
    return total / norm


def geodesic_sphere(frequency, mat=0, displacement=0.0, seed=0, octaves=3):
    """Icosahedron with every face split into frequency^2 triangles
    (20 * frequency^2 total), vertices on the unit sphere, radially displaced
    by seeded value noise."""
    t = (1 + 5 ** 0.5) / 2
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    f = frequency
    ii, jj = np.meshgrid(np.arange(f + 1), np.arange(f + 1), indexing="ij")
    mask = ii + jj <= f
    ii, jj = ii[mask], jj[mask]
    index = -np.ones((f + 1, f + 1), np.int64)
    index[ii, jj] = np.arange(len(ii))
    ui, uj = np.meshgrid(np.arange(f), np.arange(f), indexing="ij")
    up = ui + uj <= f - 1
    a_up = index[ui[up], uj[up]], index[ui[up] + 1, uj[up]], index[ui[up], uj[up] + 1]
    dn = ui + uj <= f - 2
    a_dn = index[ui[dn] + 1, uj[dn]], index[ui[dn] + 1, uj[dn] + 1], index[ui[dn], uj[dn] + 1]
    tri_idx = np.concatenate([np.stack(a_up, 1), np.stack(a_dn, 1)])
    out = []
    for (a, b, c) in faces:
        pts = v[a] + (v[b] - v[a]) * (ii[:, None] / f) + (v[c] - v[a]) * (jj[:, None] / f)
        pts /= np.linalg.norm(pts, axis=1, keepdims=True)
        if displacement:
            pts *= (1.0 + displacement * value_noise(pts, seed, octaves))[:, None]
        out.append(pts[tri_idx])
    tri = np.concatenate(out)
    return triangles(tri[:, 0].astype(np.float32), tri[:, 1].astype(np.float32), tri[:, 2].astype(np.float32), mat)


def look_at_camera(position, target, vertical_fov_deg, width, height):
    """Camera as the reference's presets build it (src/scene/camera.cu:3-42)."""
    p = np.array(position, np.float32)
    fwd = np.array(target, np.float32) - p
    fwd = fwd * np.float32(1.0 / math.sqrt(float(np.dot(fwd, fwd))))
    up0 = np.array([0, 0, 1], np.float32) if abs(fwd[1]) > 0.999 else np.array([0, 1, 0], np.float32)
    right = np.cross(fwd, up0).astype(np.float32)
    right = right * np.float32(1.0 / math.sqrt(float(np.dot(right, right))))
    up = np.cross(right, fwd).astype(np.float32)
    return {"position": p, "forward": fwd, "right": right, "up": up,
            "vertical_fov": np.float32(vertical_fov_deg * 3.14159265359 / 180.0),
            "aspect_ratio": np.float32(width / height)}


# --------------------------------------------------------------- scenes


def cornell_box(width=256, height=256):
    """Plain Cornell box: 5 walls (10 triangles), a 2-triangle ceiling light of
    radiance 15 and two boxes rotated +-18 degrees (24 triangles), all 36 in one
    mesh with one identity instance (TLAS/BLAS path).  Room, palette and light
    placement follow assembleCornellScene (scene_host.cpp:325-341)."""
    s = Scene()
    white = s.add_material(material(abi.MAT_DIFFUSE, (0.73, 0.73, 0.73)))
    red = s.add_material(material(abi.MAT_DIFFUSE, (0.65, 0.05, 0.05)))
    green = s.add_material(material(abi.MAT_DIFFUSE, (0.12, 0.45, 0.15)))
    box_white = s.add_material(material(abi.MAT_DIFFUSE, (0.72, 0.72, 0.72)))
    light = s.add_material(material(abi.MAT_EMISSIVE, (1.0, 1.0, 1.0), (15.0, 15.0, 15.0)))
    w, fy, cy, bz, fz = 2.5, -1.0, 3.0, -2.5, 2.5
    tris = [
        quad((-w, fy, fz), (w, fy, fz), (w, fy, bz), (-w, fy, bz), white),
        quad((-w, cy, bz), (w, cy, bz), (w, cy, fz), (-w, cy, fz), white),
        quad((-w, fy, bz), (w, fy, bz), (w, cy, bz), (-w, cy, bz), white),
        quad((-w, fy, fz), (-w, fy, bz), (-w, cy, bz), (-w, cy, fz), red),
        quad((w, fy, bz), (w, fy, fz), (w, cy, fz), (w, cy, bz), green),
    ]
    corner, eu, ev = np.array([-0.75, 2.95, -0.75]), np.array([1.5, 0, 0]), np.array([0, 0, 1.5])
    tris.append(quad(corner, corner + eu, corner + eu + ev, corner + ev, light))
    tris.append(box((0.85, -0.4, 0.55), (1.2, 1.2, 1.2), -18.0, box_white))
    tris.append(box((-0.8, 0.2, -0.65), (1.2, 2.4, 1.2), 18.0, box_white))
    mesh = s.add_mesh(np.concatenate(tris))
    s.instances = instance(mesh)
    s.black_background = True
    cam = look_at_camera((0.0, 1.2, 6.5), (0.0, 0.8, -0.6), 42.0, width, height)
    return s, cam


def sphere_field(width=1280, height=720, frequency=256, grid=22, seed=7):
    """22x22 radius-0.2 spheres jittered +-0.45 (80% Lambertian albedo u*u,
    15% metal albedo U(0.5,1) fuzz U(0,0.5), 5% glass ior 1.5), a radius-1000
    ground sphere tested directly, three instances (glass, metal, diffuse) of
    one displaced geodesic sphere BLAS, sky gradient."""
    s = Scene()
    rng = SceneRng(seed)
    ground = s.add_material(material(abi.MAT_DIFFUSE, (0.5, 0.5, 0.5)))
    glass = s.add_material(material(abi.MAT_DIELECTRIC, (1.0, 1.0, 1.0), ior=1.5))
    metal = s.add_material(material(abi.MAT_METAL, (0.8, 0.82, 0.9), roughness=0.05))
    diffuse = s.add_material(material(abi.MAT_DIFFUSE, (0.8, 0.3, 0.3)))
    spheres = [((0.0, -1000.0, 0.0), 1000.0, ground, abi.ACCEL_DIRECT)]
    mats = []
    half = grid // 2
    for a in range(-half, grid - half):
        for b in range(-half, grid - half):
            choose = rng.next()
            cx = a + (rng.next() - 0.5) * 0.9
            cz = b + (rng.next() - 0.5) * 0.9
            if choose < 0.80:
                m = material(abi.MAT_DIFFUSE, (rng.next() * rng.next(), rng.next() * rng.next(), rng.next() * rng.next()))
            elif choose < 0.95:
                alb = (0.5 + 0.5 * rng.next(), 0.5 + 0.5 * rng.next(), 0.5 + 0.5 * rng.next())
                m = material(abi.MAT_METAL, alb, roughness=0.5 * rng.next())
            else:
                m = material(abi.MAT_DIELECTRIC, (1.0, 1.0, 1.0), ior=1.5)
            mats.append(m)
            spheres.append(((cx, 0.2, cz), 0.2, len(s.materials) + len(mats) - 1, abi.ACCEL_BVH))
    s.materials = np.concatenate([s.materials, np.array(mats, abi.MATERIAL_DTYPE)])
    sp = np.zeros(len(spheres), abi.SPHERE_DTYPE)
    for i, (c, r, m, acc) in enumerate(spheres):
        sp[i] = (c, r, m, acc)
    s.spheres = sp
    mesh = s.add_mesh(geodesic_sphere(frequency, ground, displacement=0.08, seed=seed))
    s.instances = np.concatenate([
        instance(mesh, (-4.0, 1.0, 0.0), 1.0, 0.0, glass),
        instance(mesh, (4.0, 1.0, 0.0), 1.0, 30.0, metal),
        instance(mesh, (0.0, 1.0, 0.0), 1.0, 60.0, diffuse),
    ])
    s.black_background = False
    cam = look_at_camera((13.0, 2.0, 3.0), (0.0, 0.8, 0.0), 32.0, width, height)
    return s, cam


def sun_sky_environment(width=2048, height=1024, sun_radius_deg=0.5, sun_intensity=5.0e4,
                        sun_elevation_deg=35.0, sun_azimuth_deg=120.0):
    """Synthetic HDR equirect map: a sky gradient plus a 0.5 degree sun disk.
    Row 0 = +Y; columns follow environmentUv (environment.cuh:26-33)."""
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = v * math.pi
    phi = (u - 0.5) * 2 * math.pi
    st, ct = np.sin(theta)[:, None], np.cos(theta)[:, None]
    d = np.stack([st * np.cos(phi)[None, :], np.broadcast_to(ct, (height, width)), st * np.sin(phi)[None, :]], -1)
    up = np.clip(d[..., 1], -1, 1)
    sky = np.stack([0.45 + 0.25 * (1 - up), 0.6 + 0.2 * (1 - up), 1.0 + 0.0 * up], -1) * np.clip(up + 0.3, 0.05, 1.3)[..., None]
    el, az = math.radians(sun_elevation_deg), math.radians(sun_azimuth_deg)
    sun = np.array([math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az)])
    cosang = d @ sun
    disk = cosang > math.cos(math.radians(sun_radius_deg))
    rgba = np.zeros((height, width, 4), np.float32)
    rgba[..., :3] = sky
    rgba[disk, :3] = sun_intensity
    rgba[..., 3] = 1.0
    return {"rgba": rgba, "intensity": 1.0, "rotation": 0.0}


def heightfield(n, extent, amplitude, seed):
    """fBm terrain over an n x n quad grid: 2 n^2 triangles."""
    xs = np.linspace(-extent, extent, n + 1)
    gx, gz = np.meshgrid(xs, xs, indexing="xy")
    p = np.stack([gx.ravel() / extent, np.zeros(gx.size), gz.ravel() / extent], 1)
    h = amplitude * value_noise(p, seed, octaves=5, frequency=3.0)
    pts = np.stack([gx.ravel(), h, gz.ravel()], 1).astype(np.float32).reshape(n + 1, n + 1, 3)
    a = pts[:-1, :-1].reshape(-1, 3)
    b = pts[:-1, 1:].reshape(-1, 3)
    c = pts[1:, 1:].reshape(-1, 3)
    d = pts[1:, :-1].reshape(-1, 3)
    v0 = np.concatenate([a, a])
    v1 = np.concatenate([d, c])
    v2 = np.concatenate([c, b])
    return v0, v1, v2, pts


def large_mesh(width=1920, height=1080, terrain_quads=2236, instance_count=500, instance_frequency=100,
               emissive_fraction=0.01, glass_spheres=20, env_size=(2048, 1024), seed=3):
    """Large mesh with lights: fBm terrain, emissive terrain triangles
    (radiance log-uniform in [1, 50], quantized to 64 materials), instanced
    displaced geodesic spheres (scale U(0.5, 3), random yaw), glass spheres for
    caustics, HDR sun-and-sky environment."""
    s = Scene()
    rng = np.random.default_rng(seed)
    extent = 60.0
    terrain_mat = s.add_material(material(abi.MAT_DIFFUSE, (0.45, 0.42, 0.38)))
    rock_mats = [s.add_material(material(abi.MAT_DIFFUSE, (0.3 + 0.5 * rng.random(), 0.3 + 0.4 * rng.random(),
                                                             0.25 + 0.3 * rng.random()))) for _ in range(4)]
    rock_mats.append(s.add_material(material(abi.MAT_METAL, (0.9, 0.85, 0.7), roughness=0.2)))
    glass = s.add_material(material(abi.MAT_DIELECTRIC, (1.0, 1.0, 1.0), ior=1.5))
    levels = np.exp(np.linspace(math.log(1.0), math.log(50.0), 64))
    emissive = [s.add_material(material(abi.MAT_EMISSIVE, (1, 1, 1), (float(l), float(l * 0.85), float(l * 0.6))))
                for l in levels]
    v0, v1, v2, pts = heightfield(terrain_quads, extent, 4.0, seed)
    terrain = triangles(v0, v1, v2, terrain_mat)
    n = len(terrain)
    k = int(round(n * emissive_fraction))
    pick = rng.choice(n, size=k, replace=False)
    terrain["material"][pick] = np.array(emissive, np.uint32)[rng.integers(0, 64, size=k)]
    tmesh = s.add_mesh(terrain)
    rock = s.add_mesh(geodesic_sphere(instance_frequency, terrain_mat, displacement=0.15, seed=seed + 1))
    inst = [instance(tmesh)]
    grid_res = terrain_quads + 1

    def ground_height(x, z):
        i = np.clip(np.round((x + extent) / (2 * extent) * terrain_quads).astype(int), 0, grid_res - 1)
        j = np.clip(np.round((z + extent) / (2 * extent) * terrain_quads).astype(int), 0, grid_res - 1)
        return pts[j, i, 1]

    xs = rng.uniform(-extent * 0.8, extent * 0.8, instance_count)
    zs = rng.uniform(-extent * 0.8, extent * 0.8, instance_count)
    scales = rng.uniform(0.5, 3.0, instance_count)
    yaws = rng.uniform(0.0, 360.0, instance_count)
    hs = ground_height(xs, zs)
    for i in range(instance_count):
        inst.append(instance(rock, (xs[i], hs[i] + 0.6 * scales[i], zs[i]), scales[i], yaws[i],
                             rock_mats[i % len(rock_mats)]))
    s.instances = np.concatenate(inst)
    sp = np.zeros(glass_spheres, abi.SPHERE_DTYPE)
    gx = rng.uniform(-12, 12, glass_spheres)
    gz = rng.uniform(-12, 12, glass_spheres)
    gr = rng.uniform(0.6, 1.6, glass_spheres)
    gh = ground_height(gx, gz)
    for i in range(glass_spheres):
        sp[i] = ((gx[i], gh[i] + gr[i] + 0.2, gz[i]), gr[i], glass, abi.ACCEL_BVH)
    s.spheres = sp
    s.environment = sun_sky_environment(*env_size)
    s.black_background = False
    cam = look_at_camera((0.0, 14.0, 38.0), (0.0, 0.0, 0.0), 50.0, width, height)
    return s, cam


def batch_jobs(count=64, seed=11, min_triangles=5_000, max_triangles=2_000_000, sizes=(64, 128, 256, 512),
               spps=(4, 16, 64), max_depth=8):
    """Uneven render jobs for the batch workload: `count` sphere-field jobs
    drawn from `seed`, each with its own scene seed and a displaced geodesic
    mesh of log-uniform size in [min_triangles, max_triangles] (20 f^2
    triangles for frequency f), a square resolution drawn from `sizes`, a
    sample count drawn from `spps`, and depth `max_depth`.
    Returns dicts: scene, camera, width, height, spp, max_depth, triangles."""
    rng = SceneRng(seed)
    lo, hi = math.log(min_triangles), math.log(max_triangles)
    jobs = []
    for _ in range(count):
        triangles = math.exp(lo + (hi - lo) * rng.next())
        frequency = max(16, int(round(math.sqrt(triangles / 20.0))))
        size = sizes[min(int(rng.next() * len(sizes)), len(sizes) - 1)]
        spp = spps[min(int(rng.next() * len(spps)), len(spps) - 1)]
        scene_seed = 1 + int(rng.next() * 1_000_000)
        scene, cam = sphere_field(size, size, frequency=frequency, seed=scene_seed)
        jobs.append(dict(scene=scene, camera=cam, width=size, height=size, spp=spp, max_depth=max_depth,
                         triangles=scene.triangle_count()))
    return jobs


def _grid_quad(p0, eu, ev, n, mat):
    """Quad p0 + [0,1]^2 (eu, ev) split into n x n cells of two triangles each
    (same diagonal and winding as quad())."""
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    i, j = i.ravel()[:, None], j.ravel()[:, None]
    p0, eu, ev = (np.asarray(a, np.float64) for a in (p0, eu, ev))
    a = p0 + eu * (i / n) + ev * (j / n)
    b = p0 + eu * ((i + 1) / n) + ev * (j / n)
    c = p0 + eu * ((i + 1) / n) + ev * ((j + 1) / n)
    d = p0 + eu * (i / n) + ev * ((j + 1) / n)
    v0 = np.concatenate([a, a], axis=1).reshape(-1, 3)
    v1 = np.concatenate([b, c], axis=1).reshape(-1, 3)
    v2 = np.concatenate([c, d], axis=1).reshape(-1, 3)
    return triangles(v0.astype(np.float32), v1.astype(np.float32), v2.astype(np.float32), mat)


def cornell_inverse(width=512, height=512, cells=32):
    """Cornell box for inverse rendering: each of the 5 walls split into
    cells x cells quads (2 * cells^2 triangles; 10,240 walls triangles for
    cells = 32), the two rotated boxes (24 triangles) and the 2-triangle
    ceiling light (radiance 15), in one mesh.  The mesh index of a triangle is
    its parameter index for wf_diff_*: walls first, then boxes, then the
    light.  Returns (scene, camera, parameter_count, light_triangles)."""
    s = Scene()
    grey = s.add_material(material(abi.MAT_DIFFUSE, (0.5, 0.5, 0.5)))
    light = s.add_material(material(abi.MAT_EMISSIVE, (1.0, 1.0, 1.0), (15.0, 15.0, 15.0)))
    w, fy, cy, bz, fz = 2.5, -1.0, 3.0, -2.5, 2.5
    walls = [  # (origin, edge u, edge v) with the windings of cornell_box
        ((-w, fy, fz), (2 * w, 0, 0), (0, 0, bz - fz)),
        ((-w, cy, bz), (2 * w, 0, 0), (0, 0, fz - bz)),
        ((-w, fy, bz), (2 * w, 0, 0), (0, cy - fy, 0)),
        ((-w, fy, fz), (0, 0, bz - fz), (0, cy - fy, 0)),
        ((w, fy, bz), (0, 0, fz - bz), (0, cy - fy, 0)),
    ]
    tris = [_grid_quad(p, u, v, cells, grey) for p, u, v in walls]
    tris.append(box((0.85, -0.4, 0.55), (1.2, 1.2, 1.2), -18.0, grey))
    tris.append(box((-0.8, 0.2, -0.65), (1.2, 2.4, 1.2), 18.0, grey))
    corner, eu, ev = np.array([-0.75, 2.95, -0.75]), np.array([1.5, 0, 0]), np.array([0, 0, 1.5])
    tris.append(quad(corner, corner + eu, corner + eu + ev, corner + ev, light))
    mesh = np.concatenate(tris)
    s.add_mesh(mesh)
    s.instances = instance(0)
    s.black_background = True
    cam = look_at_camera((0.0, 1.2, 6.5), (0.0, 0.8, -0.6), 42.0, width, height)
    return s, cam, len(mesh), 2


def inverse_parameters(scene, parameter_count, seed, albedo_range=(0.15, 0.85), roughness_range=(0.0, 0.8)):
    """Smooth seeded parameter fields over a mesh's triangle centroids:
    RGB albedo and Oren-Nayar roughness (radians) per triangle."""
    mesh = scene.meshes[0]
    centroid = (mesh["v0"].astype(np.float64) + mesh["v1"] + mesh["v2"]) / 3.0
    lo, hi = albedo_range
    albedo = np.stack([lo + (hi - lo) * 0.5 * (1.0 + value_noise(centroid, seed + c, frequency=0.6))
                       for c in range(3)], axis=1)
    rlo, rhi = roughness_range
    rough = rlo + (rhi - rlo) * 0.5 * (1.0 + value_noise(centroid, seed + 17, frequency=0.6))
    return albedo[:parameter_count].astype(np.float32), rough[:parameter_count].astype(np.float32)


# ------------------------------------------------------ textured materials
def texture_binding(texture=abi.NO_TEXTURE, texcoord=0, offset=(0.0, 0.0), scale=(1.0, 1.0), rotation=None):
    """One wf_texture_binding; `rotation` (or a non-unit scale/offset) sets
    the KHR_texture_transform."""
    b = np.zeros((), abi.TEXTURE_BINDING_DTYPE)
    b["texture"], b["texcoord"] = texture, texcoord
    b["offset"], b["scale"] = offset, scale
    b["rotation"] = rotation or 0.0
    b["has_transform"] = int(rotation is not None or tuple(scale) != (1.0, 1.0) or tuple(offset) != (0.0, 0.0))
    return b


def material_textures(**slots):
    """One wf_material_textures record: unbound slots get WF_NO_TEXTURE,
    normal scales default to 1."""
    r = np.zeros(1, abi.MATERIAL_TEXTURES_DTYPE)
    r["normal_scale"] = slots.pop("normal_scale", 1.0)
    r["clearcoat_normal_scale"] = slots.pop("clearcoat_normal_scale", 1.0)
    for k in abi.TEXTURE_SLOTS:
        r[k] = slots.pop(k, texture_binding())
    assert not slots, f"unknown slots {sorted(slots)}"
    return r


def _uv_grid(p0, eu, ev, n, mat, uv_scale=1.0, vertex_tangents=True, sign=1.0):
    """A grid quad (as _grid_quad) with texture coordinates: set 0 runs along
    (eu, ev) over [0, uv_scale]^2, set 1 along (ev, eu) over [0, 1]^2; face
    tangents follow eu / ev (set 0) and ev / eu (set 1); vertex tangents
    (every other cell) carry `sign`."""
    tris = _grid_quad(p0, eu, ev, n, mat)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    i, j = i.ravel().astype(np.float64), j.ravel().astype(np.float64)
    a = np.stack([i / n, j / n], 1)
    b = np.stack([(i + 1) / n, j / n], 1)
    c = np.stack([(i + 1) / n, (j + 1) / n], 1)
    d = np.stack([i / n, (j + 1) / n], 1)
    uv = np.stack([np.stack([a, b, c], 1), np.stack([a, c, d], 1)], 1).reshape(-1, 3, 2)
    attrs = np.zeros(len(tris), abi.TRIANGLE_ATTRIBUTES_DTYPE)
    attrs["uv"] = uv * uv_scale
    attrs["uv1"] = uv[:, :, ::-1]
    tu = np.asarray(eu, np.float64) / np.linalg.norm(eu)
    tv = np.asarray(ev, np.float64) / np.linalg.norm(ev)
    attrs["tangent"], attrs["bitangent"] = tu, tv
    attrs["tangent1"], attrs["bitangent1"] = tv, tu
    attrs["has_texcoords"] = 1
    attrs["has_texcoords1"] = 1
    if vertex_tangents:
        every_other = (np.arange(len(tris)) // 2) % 2 == 0
        attrs["vertex_tangent"][every_other] = tu
        attrs["vertex_tangent_sign"][every_other] = sign
        attrs["has_vertex_tangents"][every_other] = 1
    return tris, attrs


def _procedural_textures(seed=5):
    """RGBA8 textures (uint8[h, w, 4]): checker, bump normal map, metallic-
    roughness, emissive pattern, alpha card with round holes, specular-
    glossiness, clearcoat factors."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:64, 0:64] / 64.0
    checker = (((x * 8).astype(int) + (y * 8).astype(int)) % 2).astype(np.float64)
    albedo = np.stack([0.2 + 0.7 * checker, 0.25 + 0.5 * (1 - checker), 0.3 + 0.4 * x, np.ones_like(x)], -1)
    hx = np.cos(x * 2 * np.pi * 4) * 0.6
    hy = np.sin(y * 2 * np.pi * 3) * 0.6
    nrm = np.stack([hx, hy, np.ones_like(x)], -1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    normal = np.concatenate([nrm * 0.5 + 0.5, np.ones_like(x)[..., None]], -1)
    mr = np.stack([np.zeros_like(x), 0.1 + 0.8 * y, ((x * 6).astype(int) % 2).astype(np.float64), np.ones_like(x)], -1)
    emissive = np.stack([0.5 + 0.5 * np.sin(x * 20), 0.5 + 0.5 * np.cos(y * 17), 0.8 * x * y, np.ones_like(x)], -1)
    holes = ((np.mod(x * 5, 1.0) - 0.5) ** 2 + (np.mod(y * 5, 1.0) - 0.5) ** 2) < 0.09
    card = np.stack([0.3 + 0.5 * y, 0.6 * np.ones_like(x), 0.2 + 0.3 * x, np.where(holes, 0.1, 1.0)], -1)
    specgloss = np.stack([0.4 + 0.5 * x, 0.4 + 0.5 * y, 0.5 * np.ones_like(x), 0.2 + 0.75 * checker], -1)
    coat = np.stack([0.3 + 0.7 * checker, 0.1 + 0.8 * x, np.zeros_like(x), np.ones_like(x)], -1)
    noise = rng.uniform(0, 1, (64, 64, 4)) * 0.02
    to8 = lambda t: np.clip(np.round((t + noise) * 255.0), 0, 255).astype(np.uint8)
    return [to8(t) for t in (albedo, normal, mr, emissive, card, specgloss, coat)]


def textured_room(width=96, height=96):
    """A room whose surfaces use every texture path of the shading code:
    checker albedo with a transform and a normal map (floor), glTF PBR with
    metallic-roughness, clearcoat and clearcoat normal textures (back wall),
    specular-glossiness on coordinate set 1 with a rotated transform (left
    wall), an emissive-textured light panel, an alpha-masked card with holes,
    two instances of a normal-mapped metal panel (tangents through instance
    transforms), and a glass block with a thickness texture."""
    s = Scene()
    ALB, NRM, MR, EMI, CARD, SG, COAT = range(7)
    s.textures = _procedural_textures()
    tex = []
    white = s.add_material(material(abi.MAT_DIFFUSE, (0.9, 0.9, 0.9)))
    tex.append(material_textures(albedo=texture_binding(ALB, 0, (0.1, 0.2), (3.0, 3.0), 0.3),
                                 normal=texture_binding(NRM, 0, scale=(2.0, 2.0)), normal_scale=0.8))
    pbr = s.add_material(material(abi.MAT_DIFFUSE, (0.95, 0.9, 0.85), roughness=1.0, metallic=1.0, gltf_pbr=1,
                                  clearcoat=0.8, clearcoat_roughness=0.6, ior=1.5))
    tex.append(material_textures(albedo=texture_binding(ALB), metallic_roughness=texture_binding(MR),
                                 clearcoat=texture_binding(COAT), clearcoat_roughness=texture_binding(COAT),
                                 clearcoat_normal=texture_binding(NRM, 1), clearcoat_normal_scale=0.5))
    sg = s.add_material(material(abi.MAT_SPECGLOSS, (0.8, 0.8, 0.8), specgloss_workflow=1, glossiness=0.9,
                                 specular=(0.9, 0.9, 0.9)))
    tex.append(material_textures(albedo=texture_binding(ALB, 1),
                                 specular_glossiness=texture_binding(SG, 1, (0.05, 0.0), (1.5, 1.5), -0.7)))
    plain = s.add_material(material(abi.MAT_DIFFUSE, (0.12, 0.45, 0.15)))
    tex.append(material_textures())
    light = s.add_material(material(abi.MAT_EMISSIVE, (1.0, 1.0, 1.0), (12.0, 12.0, 12.0)))
    tex.append(material_textures(emissive=texture_binding(EMI)))
    card = s.add_material(material(abi.MAT_DIFFUSE, (1.0, 1.0, 1.0), alpha_masked=1, alpha_cutoff=0.5))
    tex.append(material_textures(albedo=texture_binding(CARD)))
    panel = s.add_material(material(abi.MAT_METAL, (0.9, 0.85, 0.7), roughness=0.4, metallic=1.0))
    tex.append(material_textures(metallic_roughness=texture_binding(MR), normal=texture_binding(NRM, 0, rotation=1.1)))
    glass = s.add_material(material(abi.MAT_DIELECTRIC, (1.0, 1.0, 1.0), ior=1.5, attenuation_color=(0.6, 0.8, 0.9),
                                    attenuation_distance=0.8, volume_density=1.5))
    tex.append(material_textures(thickness=texture_binding(MR)))
    s.material_textures = np.concatenate(tex)

    w, fy, cy, bz, fz = 2.5, -1.0, 3.0, -2.5, 2.5
    parts = [
        _uv_grid((-w, fy, fz), (2 * w, 0, 0), (0, 0, bz - fz), 6, white, uv_scale=2.0, sign=-1.0),
        _uv_grid((-w, fy, bz), (2 * w, 0, 0), (0, cy - fy, 0), 6, pbr),
        _uv_grid((-w, fy, fz), (0, 0, bz - fz), (0, cy - fy, 0), 6, sg),
        _uv_grid((w, fy, bz), (0, 0, fz - bz), (0, cy - fy, 0), 2, plain, vertex_tangents=False),
        _uv_grid((-w, cy, bz), (2 * w, 0, 0), (0, 0, fz - bz), 2, white),
        _uv_grid((-0.8, 2.95, -0.8), (1.6, 0, 0), (0, 0, 1.6), 2, light),
        _uv_grid((-1.8, -0.9, -0.2), (1.6, 0, 0.3), (0, 2.2, 0), 3, card),
        _uv_grid((0.6, -0.99, -0.2), (0.9, 0, 0), (0, 0, 0.9), 1, glass),
    ]
    room = np.concatenate([p[0] for p in parts])
    room_attrs = np.concatenate([p[1] for p in parts])
    panel_tris, panel_attrs = _uv_grid((-0.5, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), 3, panel, sign=-1.0)
    m_room = s.add_mesh(room)
    m_panel = s.add_mesh(panel_tris)
    s.mesh_attributes = [room_attrs, panel_attrs]
    s.instances = np.concatenate([instance(m_room), instance(m_panel, (1.2, 0.2, -1.6), 1.2, 35.0),
                                  instance(m_panel, (-0.2, 1.4, -2.0), 0.8, -20.0)])
    s.spheres = np.array([((0.9, -0.6, 0.9), 0.4, glass, abi.ACCEL_BVH)], abi.SPHERE_DTYPE)
    s.black_background = True
    cam = look_at_camera((0.0, 1.0, 6.2), (0.0, 0.8, -0.6), 45.0, width, height)
    return s, cam
