"""ORACLE / TEST INFRASTRUCTURE ONLY.

Loads the host-compiled reference (oracle/_ref/libwfref.so, built by
oracle/Makefile from the reference's own sources) and its deterministic-math
twin (libwfref_det.so: identical code, elementary functions from wf_math.h).
Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this
module; the product never does.
"""
import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
_libs = {}


def available(det=False):
    return (REF_DIR / ("libwfref_det.so" if det else "libwfref.so")).exists()


def ref_lib(det=False):
    """det=False: the reference as written (C-library math); det=True: the
    reference with the renderer's deterministic elementary functions."""
    key = bool(det)
    if key not in _libs:
        path = REF_DIR / ("libwfref_det.so" if det else "libwfref.so")
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle)")
        lib = C.CDLL(str(path))
        P, U32, I = C.c_void_p, C.c_uint32, C.c_int
        lib.wfref_scene_create.restype = P
        lib.wfref_scene_create.argtypes = [P, P, I]
        lib.wfref_scene_destroy.argtypes = [P]
        lib.wfref_scene_light_count.restype = U32
        lib.wfref_scene_light_count.argtypes = [P]
        lib.wfref_scene_lights.argtypes = [P, P, P]
        lib.wfref_environment_distribution.restype = I
        lib.wfref_environment_distribution.argtypes = [P, U32, U32, P, P, P]
        lib.wfref_trace.argtypes = [P, P, U32, P, I]
        lib.wfref_occluded.argtypes = [P, P, P, U32, P, I]
        lib.wfref_photons.restype = I
        lib.wfref_photons.argtypes = [P, P, P, P, P, I]
        lib.wfref_load_environment.restype = I
        lib.wfref_load_environment.argtypes = [C.c_char_p, P, P, P]
        lib.wfref_path_rays.restype = U32
        lib.wfref_path_rays.argtypes = [P, P, P, U32, U32, U32, U32, U32, U32, P, U32, P, I]
        lib.wfref_render.restype = I
        lib.wfref_render.argtypes = [P, P, P, U32, U32, U32, U32, U32, U32, P, P, P, I, I]
        lib.wfref_frame_guides.restype = I
        lib.wfref_frame_guides.argtypes = [P, P, P, U32, U32, U32, U32, U32, U32, P, I]
        lib.wfref_host_preset.restype = P
        lib.wfref_host_preset.argtypes = [I, C.c_char_p, C.c_float, P, I, I, I, I, I, I, I, I]
        lib.wfref_host_scene_destroy.argtypes = [P]
        lib.wfref_host_scene_counts.argtypes = [P, P]
        lib.wfref_host_scene_triangle_count.restype = C.c_uint64
        lib.wfref_host_scene_triangle_count.argtypes = [P, I, U32]
        lib.wfref_host_scene_triangles.argtypes = [P, I, U32, P, P]
        lib.wfref_host_scene_materials.argtypes = [P, P, P]
        lib.wfref_host_scene_instances.argtypes = [P, P]
        lib.wfref_host_scene_spheres.argtypes = [P, P]
        lib.wfref_host_scene_punctual.argtypes = [P, P]
        lib.wfref_host_scene_texture.argtypes = [P, U32, P, P]
        lib.wfref_scene_from_host.restype = P
        lib.wfref_scene_from_host.argtypes = [P, I, C.c_float]
        lib.wfref_dist_tasks.restype = C.c_uint64
        lib.wfref_dist_tasks.argtypes = [U32, U32, U32, U32, U32, U32, C.c_uint64, P, C.c_uint64]
        lib.wfref_dist_task_key.restype = C.c_uint64
        lib.wfref_dist_task_key.argtypes = [C.c_uint64, U32, U32, U32]
        lib.wfref_dist_checkpoint_write.restype = I
        lib.wfref_dist_checkpoint_write.argtypes = [C.c_char_p, C.c_uint64, P, C.c_uint64, P, P, P, C.c_uint64,
                                                    C.c_char_p, C.c_uint64]
        lib.wfref_dist_checkpoint_read.restype = I
        lib.wfref_dist_checkpoint_read.argtypes = [C.c_char_p, P, P, P, P, C.c_char_p, C.c_uint64]
        lib.wfref_dielectric_reflectance.restype = C.c_float
        lib.wfref_dielectric_reflectance.argtypes = [C.c_float, C.c_float]
        lib.wfref_checkpoint_roundtrip_read.restype = I
        lib.wfref_checkpoint_roundtrip_read.argtypes = [C.c_char_p, U32, U32, C.c_uint64, P, P]
        lib.wfref_checkpoint_write.restype = I
        lib.wfref_checkpoint_write.argtypes = [C.c_char_p, U32, U32, C.c_uint64, P, U32]
        _libs[key] = lib
    return _libs[key]


def reference_config(width, height, **fields):
    """A wf_render_config holding the reference's RenderConfig defaults
    (include/config.hpp:11-41) at the given size, made without loading the
    B200 library: the CPU reference arm of bench.py runs only the
    reference's code.  tests/test_oracle_pins.py checks it field by field
    against wf_render_config_default."""
    from wfpt import abi
    cfg = abi.RenderConfig()
    cfg.width, cfg.height = width, height
    cfg.max_depth, cfg.rr_start_depth = 32, 12
    cfg.mode, cfg.rng = abi.MODE_GRAPH, abi.RNG_XORSHIFT32
    cfg.indirect_clamp = 10.0
    cfg.caustic_gather = 1
    cfg.photon_count, cfg.photon_max_depth = 1048576, 8
    cfg.gather_radius = 0.06
    cfg.photon_grid_min[:] = [-2.5, -1.0, -2.5]
    cfg.photon_grid_max[:] = [2.5, 3.0, 2.5]
    cfg.photon_grid_resolution = 64
    cfg.photon_seed = 0x13579BDF
    cfg.profile_queues = 1
    for k, v in fields.items():
        if k in ("photon_grid_min", "photon_grid_max"):
            getattr(cfg, k)[:] = [float(x) for x in v]
        else:
            setattr(cfg, k, v)
    return cfg


class RefScene:
    """The reference's uploadScene() of a wfpt.Scene, in host memory."""

    def __init__(self, scene, det=False, probe=False):
        from wfpt import abi  # noqa: F401  (layouts shared with the C ABI)
        self.lib = ref_lib(det)
        d, keep = scene.desc()
        env, rgba = scene.environment_struct()
        self.handle = self.lib.wfref_scene_create(C.addressof(d), C.addressof(env) if env is not None else None,
                                                  int(probe))
        del keep, rgba
        if not self.handle:
            raise RuntimeError("reference scene creation failed")
        self.probe = probe

    def close(self):
        if self.handle:
            self.lib.wfref_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def light_count(self):
        return self.lib.wfref_scene_light_count(self.handle)

    def lights(self):
        n = self.light_count()
        rec = np.zeros((n, 16), np.float32)
        alias = np.zeros(n, np.uint32)
        if n:
            self.lib.wfref_scene_lights(self.handle, rec.ctypes.data, alias.ctypes.data)
        return rec, alias

    def trace(self, rays, threads=0):
        from wfpt import abi
        rays = np.ascontiguousarray(rays, abi.RAY_DTYPE)
        hits = np.zeros(len(rays), abi.HIT_DTYPE)
        self.lib.wfref_trace(self.handle, rays.ctypes.data, len(rays), hits.ctypes.data, threads)
        return hits

    def path_rays(self, camera, config, tile=None, sample=0, bounces=2, threads=0):
        """The reference's ray queues of one sample of a tile: the camera
        rays, then the continuation rays of each following bounce, in queue
        order.  Returns (rays as RAY_DTYPE, per-bounce counts)."""
        from wfpt import abi
        from wfpt.native import camera_struct
        x, y, w, h = tile if tile is not None else (0, 0, config.width, config.height)
        cam = camera_struct(camera)
        cap = w * h * bounces
        rays = np.zeros(cap, abi.RAY_DTYPE)
        counts = np.zeros(bounces, np.uint32)
        n = self.lib.wfref_path_rays(self.handle, C.addressof(cam), C.addressof(config), x, y, w, h, sample,
                                     bounces, rays.ctypes.data, cap, counts.ctypes.data, threads)
        if n == 0xFFFFFFFF:
            raise RuntimeError("wfref_path_rays failed")
        return rays[:n], counts

    def occluded(self, rays, max_distance, threads=0):
        from wfpt import abi
        rays = np.ascontiguousarray(rays, abi.RAY_DTYPE)
        md = np.ascontiguousarray(max_distance, np.float32)
        out = np.zeros(len(rays), np.uint8)
        self.lib.wfref_occluded(self.handle, rays.ctypes.data, md.ctypes.data, len(rays), out.ctypes.data, threads)
        return out

    def photons(self, config, threads=0):
        n = config.photon_count
        rec = np.zeros((n, 8), np.float32)
        flux = np.zeros((n, 3), np.float32)
        stored = C.c_uint32()
        self.lib.wfref_photons(self.handle, C.addressof(config), rec.ctypes.data, flux.ctypes.data,
                               C.addressof(stored), threads)
        return rec, flux, stored.value

    def frame_guides(self, camera, width, height, tile=None, previous=None, threads=0):
        """The reference's generateFrameGuides over a tile: (h, w) FRAME_GUIDE_DTYPE records."""
        from wfpt import abi
        from wfpt.native import camera_struct
        cam = camera_struct(camera)
        prev = camera_struct(previous) if previous is not None else None
        x, y, w, h = tile if tile is not None else (0, 0, width, height)
        out = np.zeros((h, w), abi.FRAME_GUIDE_DTYPE)
        rc = self.lib.wfref_frame_guides(self.handle, C.addressof(cam), C.addressof(prev) if prev else None,
                                         width, height, x, y, w, h, out.ctypes.data, threads)
        if rc != 0:
            raise RuntimeError("reference frame guides failed")
        return out

    def render(self, camera, config, tile=None, sample_start=0, sample_count=1, threads=0, persistent=False,
               fp64=False):
        """Reference captured-graph (or persistent) render of a tile: FP32 sums,
        optional FP64 sums, per-sample per-bounce queue counts."""
        from wfpt.native import camera_struct
        cam = camera_struct(camera)
        x, y, w, h = tile if tile is not None else (0, 0, config.width, config.height)
        fb32 = np.zeros((h, w, 3), np.float32)
        fb64 = np.zeros((h, w, 3), np.float64) if fp64 else None
        counts = np.zeros((sample_count, config.max_depth), np.uint32)
        rc = self.lib.wfref_render(self.handle, C.addressof(cam), C.addressof(config), x, y, w, h, sample_start,
                                   sample_count, fb32.ctypes.data, fb64.ctypes.data if fp64 else None,
                                   counts.ctypes.data, threads, int(persistent))
        if rc != 0:
            raise RuntimeError("reference render failed")
        return fb32, fb64, counts


def load_environment(path, det=False):
    """The reference's loadEnvironmentMap (stb_image's stbi_loadf) on a
    Radiance .hdr file: float32 (h, w, 4) texels, or None when it throws."""
    import os
    lib = ref_lib(det)
    w, h = C.c_uint32(), C.c_uint32()
    if lib.wfref_load_environment(os.fsencode(path), C.byref(w), C.byref(h), None) != 0:
        return None
    out = np.zeros((h.value, w.value, 4), np.float32)
    lib.wfref_load_environment(os.fsencode(path), C.byref(w), C.byref(h), out.ctypes.data)
    return out


def environment_distribution(rgba, det=False):
    """buildEnvironmentDistribution of the reference (environment.cpp:10-64)."""
    rgba = np.ascontiguousarray(rgba, np.float32)
    h, w = rgba.shape[:2]
    p = np.zeros(w * h, np.float32)
    ap = np.zeros(w * h, np.float32)
    al = np.zeros(w * h, np.uint32)
    rc = ref_lib(det).wfref_environment_distribution(rgba.ctypes.data, w, h, p.ctypes.data, ap.ctypes.data,
                                                     al.ctypes.data)
    if rc != 0:
        raise ValueError("environment rejected")
    return p, ap, al


# ---------------------------------------------------------------------------
# The oracle's own CPU restatement (pt_oracle.cpp), pinned against the
# host-compiled reference above.
PORT_DIR = HERE / "_build"
_port_libs = {}


def port_available(det=False):
    return (PORT_DIR / ("liboracle_det.so" if det else "liboracle.so")).exists()


def port_lib(det=False):
    key = bool(det)
    if key not in _port_libs:
        path = PORT_DIR / ("liboracle_det.so" if det else "liboracle.so")
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle port)")
        lib = C.CDLL(str(path))
        P, U32, I = C.c_void_p, C.c_uint32, C.c_int
        lib.oracle_scene_create.restype = P
        lib.oracle_scene_create.argtypes = [P, P]
        lib.oracle_scene_destroy.argtypes = [P]
        lib.oracle_light_count.restype = U32
        lib.oracle_light_count.argtypes = [P]
        lib.oracle_trace.argtypes = [P, P, U32, P]
        lib.oracle_occluded.argtypes = [P, P, P, U32, P]
        lib.oracle_photons.restype = U32
        lib.oracle_photons.argtypes = [P, P, P]
        lib.oracle_render.restype = I
        lib.oracle_render.argtypes = [P, P, P, U32, U32, U32, U32, U32, U32, P, P, I]
        lib.oracle_diff.restype = I
        lib.oracle_diff.argtypes = [P, P, P, P, P, C.c_double, P, P, P, P, P, I]
        _port_libs[key] = lib
    return _port_libs[key]


class PortScene:
    """The CPU restatement's scene (det selects wf_math.h elementary functions)."""

    def __init__(self, scene, det=False):
        self.lib = port_lib(det)
        d, keep = scene.desc()
        env, rgba = scene.environment_struct()
        self.handle = self.lib.oracle_scene_create(C.addressof(d), C.addressof(env) if env is not None else None)
        del keep, rgba
        if not self.handle:
            raise RuntimeError("oracle scene creation failed")

    def close(self):
        if self.handle:
            self.lib.oracle_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def light_count(self):
        return self.lib.oracle_light_count(self.handle)

    def trace(self, rays):
        from wfpt import abi
        rays = np.ascontiguousarray(rays, abi.RAY_DTYPE)
        hits = np.zeros(len(rays), abi.HIT_DTYPE)
        self.lib.oracle_trace(self.handle, rays.ctypes.data, len(rays), hits.ctypes.data)
        return hits

    def occluded(self, rays, max_distance):
        from wfpt import abi
        rays = np.ascontiguousarray(rays, abi.RAY_DTYPE)
        md = np.ascontiguousarray(max_distance, np.float32)
        out = np.zeros(len(rays), np.uint8)
        self.lib.oracle_occluded(self.handle, rays.ctypes.data, md.ctypes.data, len(rays), out.ctypes.data)
        return out

    def photons(self, config):
        rec = np.zeros((config.photon_count, 8), np.float32)
        stored = self.lib.oracle_photons(self.handle, C.addressof(config), rec.ctypes.data)
        return rec, stored

    def diff(self, camera, config, albedo, roughness, emission_scale, d_image=None, threads=0):
        """FP64 forward (and, with d_image, adjoint) of the differentiable
        renderer over config's crop: (image (h, w, 3) float64, d_albedo,
        d_roughness, d_emission_scale)."""
        from wfpt.native import camera_struct
        cam = camera_struct(camera)
        cw = config.crop_width or config.width
        ch = config.crop_height or config.height
        albedo = np.ascontiguousarray(albedo, np.float32)
        roughness = np.ascontiguousarray(roughness, np.float32)
        image = np.zeros((ch, cw, 3), np.float64)
        n = config.parameter_count
        ga, gr, gs = np.zeros((n, 3)), np.zeros(n), np.zeros(1)
        dimg = None if d_image is None else np.ascontiguousarray(d_image, np.float32)
        rc = self.lib.oracle_diff(self.handle, C.addressof(cam), C.addressof(config), albedo.ctypes.data,
                                  roughness.ctypes.data, float(emission_scale),
                                  dimg.ctypes.data if dimg is not None else None, image.ctypes.data,
                                  ga.ctypes.data, gr.ctypes.data, gs.ctypes.data, threads)
        if rc != 0:
            raise RuntimeError("a hit triangle's parameter index is not below parameter_count")
        return image, ga, gr, float(gs[0])

    def render(self, camera, config, tile=None, sample_start=0, sample_count=1, threads=0):
        from wfpt.native import camera_struct
        cam = camera_struct(camera)
        x, y, w, h = tile if tile is not None else (0, 0, config.width, config.height)
        fb = np.zeros((h, w, 3), np.float32)
        counts = np.zeros((sample_count, config.max_depth), np.uint32)
        rc = self.lib.oracle_render(self.handle, C.addressof(cam), C.addressof(config), x, y, w, h, sample_start,
                                    sample_count, fb.ctypes.data, counts.ctypes.data, threads)
        if rc != 0:
            raise RuntimeError("oracle render failed")
        return fb, counts


PRESET_KINDS = {"gltf": 0, "cornell": 1, "obj": 2, "demo": 3, "rtweek": 4}
OBJECT_SOURCES = {"obj": 0, "gltf": 1, "procedural_prism": 2}
LIGHT_PROFILES = {"standard": 0, "prism": 1, "crystal": 2}


class RefHostScene:
    """A HostScene built by the reference's own loaders and preset assembly
    (ref_assets.cpp), exported in the wfpt array layouts."""

    def __init__(self, kind, filename, scale=1.0, translation=(0.0, 0.0, 0.0), object_source="obj",
                 neutral_room=False, remove_backdrop=False, dielectric=False, material_override=-1,
                 light_profile="standard", add_top_light=True, det=True):
        self.lib = ref_lib(det)
        t = np.asarray(translation, np.float32)
        self.handle = self.lib.wfref_host_preset(PRESET_KINDS[kind], str(filename or "").encode(), float(scale),
                                                 t.ctypes.data, OBJECT_SOURCES[object_source], int(neutral_room),
                                                 int(remove_backdrop), int(dielectric), int(material_override),
                                                 LIGHT_PROFILES[light_profile], int(add_top_light), 0)
        if not self.handle:
            raise RuntimeError("the reference's preset assembly failed")

    def close(self):
        if self.handle:
            self.lib.wfref_host_scene_destroy(self.handle)
            self.handle = None

    def arrays(self, texels=True):
        """dict: spheres, triangles, static_triangles, meshes, mesh_attributes,
        instances, materials, material_textures, textures, punctual,
        light_count, black_background."""
        from wfpt import abi
        counts = np.zeros(10, np.uint64)
        self.lib.wfref_host_scene_counts(self.handle, counts.ctypes.data)
        n_sph, n_tri, n_static, n_mesh, n_inst, n_mat, n_tex, n_punct, n_lights, black = (int(x) for x in counts)

        def tris(which, mesh=0):
            n = int(self.lib.wfref_host_scene_triangle_count(self.handle, which, mesh))
            t = np.zeros(n, abi.TRIANGLE_DTYPE)
            a = np.zeros(n, abi.TRIANGLE_ATTRIBUTES_DTYPE)
            self.lib.wfref_host_scene_triangles(self.handle, which, mesh, t.ctypes.data, a.ctypes.data)
            return t, a
        out = {"light_count": n_lights, "black_background": bool(black)}
        out["triangles"], out["triangle_attributes"] = tris(0)
        out["static_triangles"], out["static_triangle_attributes"] = tris(1)
        meshes = [tris(2, m) for m in range(n_mesh)]
        out["meshes"] = [m[0] for m in meshes]
        out["mesh_attributes"] = [m[1] for m in meshes]
        out["materials"] = np.zeros(n_mat, abi.MATERIAL_DTYPE)
        out["material_textures"] = np.zeros(n_mat, abi.MATERIAL_TEXTURES_DTYPE)
        self.lib.wfref_host_scene_materials(self.handle, out["materials"].ctypes.data,
                                            out["material_textures"].ctypes.data)
        out["instances"] = np.zeros(n_inst, abi.INSTANCE_DTYPE)
        self.lib.wfref_host_scene_instances(self.handle, out["instances"].ctypes.data)
        out["spheres"] = np.zeros(n_sph, abi.SPHERE_DTYPE)
        self.lib.wfref_host_scene_spheres(self.handle, out["spheres"].ctypes.data)
        out["punctual"] = np.zeros(n_punct, abi.PUNCTUAL_DTYPE)
        self.lib.wfref_host_scene_punctual(self.handle, out["punctual"].ctypes.data)
        textures = []
        for i in range(n_tex):
            size = np.zeros(2, np.uint32)
            self.lib.wfref_host_scene_texture(self.handle, i, size.ctypes.data, None)
            rgba = np.zeros((int(size[1]), int(size[0]), 4), np.uint8)
            if texels:
                self.lib.wfref_host_scene_texture(self.handle, i, size.ctypes.data, rgba.ctypes.data)
            textures.append(rgba)
        out["textures"] = textures
        return out

    def render_scene(self, disable_normal_maps=False, normal_map_minimum_cosine=0.0):
        """A RefScene rendering this HostScene (BVH2s from the same builder as
        scenes from a description)."""
        r = RefScene.__new__(RefScene)
        r.lib = self.lib
        r.handle = self.lib.wfref_scene_from_host(self.handle, int(disable_normal_maps),
                                                  float(normal_map_minimum_cosine))
        if not r.handle:
            raise RuntimeError("wfref_scene_from_host failed")
        return r


def dist_tasks(width, height, tile_width, tile_height, spp, spp_per_task, fingerprint=0):
    """The reference's createRenderTasks as (n, 7) uint32 rows: tile, sample
    start, sample count, x, y, width, height."""
    lib = ref_lib(True)
    n = lib.wfref_dist_tasks(width, height, tile_width, tile_height, spp, spp_per_task, fingerprint, None, 0)
    out = np.zeros((n, 7), np.uint32)
    lib.wfref_dist_tasks(width, height, tile_width, tile_height, spp, spp_per_task, fingerprint, out.ctypes.data, n)
    return out


def dist_task_key(fingerprint, tile, sample_start, sample_count):
    return int(ref_lib(True).wfref_dist_task_key(fingerprint, tile, sample_start, sample_count))


def dist_checkpoint_write(path, fingerprint, job, sequence, radiance, counts, completed):
    """writeDistributedCheckpoint; job = (width, height, tile width, tile
    height, spp, spp per task).  Raises with the reference's message."""
    job = np.asarray(job, np.uint32)
    radiance = np.ascontiguousarray(radiance, np.float32)
    counts = np.ascontiguousarray(counts, np.uint32)
    completed = np.ascontiguousarray(completed, np.uint8)
    error = C.create_string_buffer(256)
    if ref_lib(True).wfref_dist_checkpoint_write(str(path).encode(), fingerprint, job.ctypes.data, sequence,
                                                 radiance.ctypes.data, counts.ctypes.data, completed.ctypes.data,
                                                 len(completed), error, 256):
        raise ValueError(error.value.decode())


def dist_checkpoint_read(path):
    """readDistributedCheckpoint: (header (9 uint64), radiance, counts,
    completed); raises with the reference's message."""
    lib = ref_lib(True)
    header = np.zeros(9, np.uint64)
    error = C.create_string_buffer(256)
    if lib.wfref_dist_checkpoint_read(str(path).encode(), header.ctypes.data, None, None, None, error, 256):
        raise ValueError(error.value.decode())
    pixels = int(header[1]) * int(header[2])
    radiance = np.zeros((pixels, 3), np.float32)
    counts = np.zeros(pixels, np.uint32)
    completed = np.zeros(int(header[8]), np.uint8)
    lib.wfref_dist_checkpoint_read(str(path).encode(), header.ctypes.data, radiance.ctypes.data, counts.ctypes.data,
                                   completed.ctypes.data, error, 256)
    return header, radiance, counts, completed
