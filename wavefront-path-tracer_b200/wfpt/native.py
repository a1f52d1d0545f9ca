"""Host-side mirror of the reference's render interface over the C ABI.

`Scene` plays the role of the reference's HostScene (include/scene/scene_host.hpp),
`DeviceScene` of DeviceScene/uploadScene (src/scene/scene.cu:336-389),
`Renderer` of RenderDriver + RenderTaskRenderer (render_driver.cuh,
render_task.cuh).  All compute runs in libwavefront_b200.so; this module only
marshals arrays.  There is no fallback: a missing library is an error.
"""
import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import abi

PACKAGE_DIR = Path(__file__).resolve().parents[1]
# WF_BUILD=fast selects the fast build (multiply-adds contracted, CUDA's own
# elementary functions: images within an RMSE of the reference instead of bit
# for bit); the default is the bit-exact build.
LIB_PATH = PACKAGE_DIR / ("libwavefront_b200_fast.so" if os.environ.get("WF_BUILD") == "fast"
                          else "libwavefront_b200.so")
_lib = None


class WavefrontError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def library():
    """Loads libwavefront_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PACKAGE_DIR}` "
                               "or __graft_entry__.build()")
        lib = C.CDLL(str(LIB_PATH))
        abi.declare(lib)
        _lib = lib
    return _lib


def check(status):
    if status != abi.WF_OK:
        msg = library().wf_last_error()
        raise WavefrontError(status, msg.decode() if msg else "")


def material(kind, albedo=(0.0, 0.0, 0.0), emission=(0.0, 0.0, 0.0), roughness=0.0, ior=1.0, **extra):
    """One wf_material record with the reference's member defaults
    (include/scene/material.cuh:30-70; roughness 0 and ior 1 as makeMaterial
    sets them, src/scene/scene_host.cpp:44-52)."""
    m = np.zeros(1, abi.MATERIAL_DTYPE)
    m["type"] = kind
    m["attenuation_color"] = 1.0
    m["volume_density"] = 1.0
    m["opacity"] = 1.0
    m["alpha_cutoff"] = 0.5
    m["specular"] = 1.0
    m["glossiness"] = 1.0
    m["specular_weight"] = 1.0
    m["specular_color"] = 1.0
    m["albedo"] = albedo
    m["emission"] = emission
    m["roughness"] = roughness
    m["ior"] = ior
    for k, v in extra.items():
        m[k] = v
    return m[0]


class Scene:
    """HostScene equivalent: numpy arrays in wf_* layouts."""

    def __init__(self):
        self.spheres = np.zeros(0, abi.SPHERE_DTYPE)
        self.triangles = np.zeros(0, abi.TRIANGLE_DTYPE)
        self.static_triangles = np.zeros(0, abi.TRIANGLE_DTYPE)
        self.meshes = []
        self.instances = np.zeros(0, abi.INSTANCE_DTYPE)
        self.materials = np.zeros(0, abi.MATERIAL_DTYPE)
        self.punctual = np.zeros(0, abi.PUNCTUAL_DTYPE)
        self.environment = None  # dict(rgba=float32[h, w, 4], intensity=, rotation=)
        self.black_background = False
        self.ignore_direct_light_occlusion = False
        self.register_triangle_lights = True
        self.build_threads = 0
        self.bvh_builder = abi.BVH_HOST_SAH  # or abi.BVH_GPU_PLOC
        # textured materials (all optional): RGBA8 textures (uint8[h, w, 4]),
        # one MATERIAL_TEXTURES_DTYPE record per material, and per-triangle
        # TRIANGLE_ATTRIBUTES_DTYPE arrays parallel to triangles,
        # static_triangles and each mesh (mesh_attributes[i] or None)
        self.textures = []
        self.material_textures = None
        self.triangle_attributes = None
        self.static_triangle_attributes = None
        self.mesh_attributes = []
        self.disable_normal_maps = False
        self.normal_map_minimum_cosine = 0.0

    def add_material(self, record):
        self.materials = np.concatenate([self.materials, np.array([record], abi.MATERIAL_DTYPE)])
        return len(self.materials) - 1

    def add_mesh(self, triangles):
        self.meshes.append(np.ascontiguousarray(triangles, abi.TRIANGLE_DTYPE))
        return len(self.meshes) - 1

    def triangle_count(self):
        return len(self.triangles) + len(self.static_triangles) + sum(len(m) for m in self.meshes)

    def desc(self):
        """(SceneDesc, keepalive list) for the C ABI."""
        keep = []

        def arr(a, dtype):
            a = np.ascontiguousarray(a, dtype)
            keep.append(a)
            return a

        meshes = np.zeros(len(self.meshes), abi.MESH_DTYPE)
        for i, m in enumerate(self.meshes):
            m = arr(m, abi.TRIANGLE_DTYPE)
            meshes[i]["triangles"] = m.ctypes.data if len(m) else 0
            meshes[i]["triangle_count"] = len(m)
            attrs = self.mesh_attributes[i] if i < len(self.mesh_attributes) else None
            if attrs is not None:
                a = arr(attrs, abi.TRIANGLE_ATTRIBUTES_DTYPE)
                assert len(a) == len(m), "one attribute record per mesh triangle"
                meshes[i]["attributes"] = a.ctypes.data
        keep.append(meshes)
        d = abi.SceneDesc()
        for name, src, dtype in [("spheres", self.spheres, abi.SPHERE_DTYPE),
                                 ("triangles", self.triangles, abi.TRIANGLE_DTYPE),
                                 ("static_triangles", self.static_triangles, abi.TRIANGLE_DTYPE),
                                 ("instances", self.instances, abi.INSTANCE_DTYPE),
                                 ("materials", self.materials, abi.MATERIAL_DTYPE),
                                 ("punctual_lights", self.punctual, abi.PUNCTUAL_DTYPE)]:
            a = arr(src, dtype)
            setattr(d, name, abi.ptr(a))
            count_name = "punctual_light_count" if name == "punctual_lights" else name[:-1] + "_count"
            setattr(d, count_name, len(a))
        d.meshes = abi.ptr(meshes)
        d.mesh_count = len(meshes)
        d.black_background = int(self.black_background)
        d.ignore_direct_light_occlusion = int(self.ignore_direct_light_occlusion)
        d.register_triangle_lights = int(self.register_triangle_lights)
        d.build_threads = self.build_threads
        d.bvh_builder = self.bvh_builder
        if self.textures:
            tex = np.zeros(len(self.textures), abi.TEXTURE_DTYPE)
            for i, t in enumerate(self.textures):
                t = arr(t, np.uint8)
                assert t.ndim == 3 and t.shape[2] == 4, "textures are uint8[h, w, 4]"
                tex[i] = (t.shape[1], t.shape[0], t.ctypes.data)
            keep.append(tex)
            d.textures = abi.ptr(tex)
            d.texture_count = len(tex)
        if self.material_textures is not None:
            mt = arr(self.material_textures, abi.MATERIAL_TEXTURES_DTYPE)
            assert len(mt) == len(self.materials), "one texture record per material"
            d.material_textures = abi.ptr(mt)
        for name, attrs, tris in [("triangle_attributes", self.triangle_attributes, self.triangles),
                                  ("static_triangle_attributes", self.static_triangle_attributes,
                                   self.static_triangles)]:
            if attrs is not None:
                a = arr(attrs, abi.TRIANGLE_ATTRIBUTES_DTYPE)
                assert len(a) == len(tris), f"one {name} record per triangle"
                setattr(d, name, abi.ptr(a))
        d.disable_normal_maps = int(self.disable_normal_maps)
        d.normal_map_minimum_cosine = float(self.normal_map_minimum_cosine)
        return d, keep

    def environment_struct(self):
        if self.environment is None:
            return None, None
        rgba = np.ascontiguousarray(self.environment["rgba"], np.float32)
        e = abi.Environment(rgba.shape[1], rgba.shape[0], rgba.ctypes.data,
                            float(self.environment.get("intensity", 1.0)),
                            float(self.environment.get("rotation", 0.0)))
        return e, rgba


class DeviceScene:
    """A scene uploaded to the current CUDA device (wf_scene_create)."""

    def __init__(self, scene):
        lib = library()
        d, keep = scene.desc()
        handle = C.c_void_p()
        check(lib.wf_scene_create(C.byref(d), C.byref(handle)))
        self.handle = handle
        env, rgba = scene.environment_struct()
        if env is not None:
            check(lib.wf_scene_set_environment(self.handle, C.byref(env)))
        del keep, rgba

    def info(self):
        info = abi.SceneInfo()
        check(library().wf_scene_get_info(self.handle, C.byref(info)))
        return info

    def set_albedos(self, materials, rgb):
        """wf_scene_set_albedos: new RGB albedos (len(materials), 3) for the
        listed materials, in place on the device."""
        ids = np.ascontiguousarray(materials, np.uint32).reshape(-1)
        values = np.ascontiguousarray(rgb, np.float32).reshape(len(ids), 3)
        check(library().wf_scene_set_albedos(self.handle, ids.ctypes.data, values.ctypes.data, len(ids)))

    def set_environment(self, environment):
        lib = library()
        if environment is None:
            check(lib.wf_scene_set_environment(self.handle, None))
            return
        rgba = np.ascontiguousarray(environment["rgba"], np.float32)
        e = abi.Environment(rgba.shape[1], rgba.shape[0], rgba.ctypes.data,
                            float(environment.get("intensity", 1.0)), float(environment.get("rotation", 0.0)))
        check(lib.wf_scene_set_environment(self.handle, C.byref(e)))

    def close(self):
        if self.handle:
            library().wf_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def trace_closest(self, rays):
        """Closest hits of a numpy RAY_DTYPE batch (device round trip via torch)."""
        import torch
        rays = np.ascontiguousarray(rays, abi.RAY_DTYPE)
        n = len(rays)
        d_rays = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
        d_hits = torch.empty(n * abi.HIT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        check(library().wf_trace_closest(self.handle, d_rays.data_ptr(), n, d_hits.data_ptr(), stream))
        torch.cuda.synchronize()
        return d_hits.cpu().numpy().view(abi.HIT_DTYPE)

    def frame_guides(self, camera, width, height, tile=None, previous=None):
        """wf_frame_guides: the denoiser guides of a tile of a width x height
        image as (h, w) FRAME_GUIDE_DTYPE records; previous is the previous
        frame's camera (None: no motion or history)."""
        import torch
        x, y, w, h = tile if tile is not None else (0, 0, width, height)
        out = torch.empty(w * h * abi.FRAME_GUIDE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        cam = camera_struct(camera)
        prev = camera_struct(previous) if previous is not None else None
        stream = torch.cuda.current_stream().cuda_stream
        check(library().wf_frame_guides(self.handle, C.byref(cam), C.byref(prev) if prev is not None else None,
                                        width, height, x, y, w, h, out.data_ptr(), stream))
        torch.cuda.synchronize()
        return out.cpu().numpy().view(abi.FRAME_GUIDE_DTYPE).reshape(h, w)

    def trace_any(self, rays, max_distance):
        import torch
        rays = np.ascontiguousarray(rays, abi.RAY_DTYPE)
        n = len(rays)
        d_rays = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
        d_max = torch.from_numpy(np.ascontiguousarray(max_distance, np.float32)).cuda()
        d_out = torch.empty(n, dtype=torch.uint8, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        check(library().wf_trace_any(self.handle, d_rays.data_ptr(), d_max.data_ptr(), n, d_out.data_ptr(), stream))
        torch.cuda.synchronize()
        return d_out.cpu().numpy()


BVH_NODE_DTYPE = np.dtype([("lo", np.float32, 3), ("hi", np.float32, 3), ("left", np.uint32), ("right", np.uint32)])


def build_bvh(boxes, builder=abi.BVH_HOST_SAH):
    """wf_bvh_build: one binary BVH2 over boxes (n, 6) = lo xyz, hi xyz.
    Returns (nodes as BVH_NODE_DTYPE, milliseconds); the root is nodes[-1]."""
    boxes = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
    n = len(boxes)
    nodes = np.zeros(max(2 * n - 1, 0), BVH_NODE_DTYPE)
    ms = C.c_double(0.0)
    check(library().wf_bvh_build(builder, boxes.ctypes.data, n, nodes.ctypes.data, C.byref(ms)))
    return nodes, ms.value


def camera_struct(cam):
    c = abi.Camera()
    for k in ("position", "forward", "right", "up"):
        getattr(c, k)[:] = [float(x) for x in cam[k]]
    c.vertical_fov = float(cam["vertical_fov"])
    c.aspect_ratio = float(cam["aspect_ratio"])
    return c


def render_config(width, height, **fields):
    """wf_render_config with the reference's defaults (config.hpp:11-41)."""
    cfg = abi.RenderConfig()
    library().wf_render_config_default(C.byref(cfg), width, height)
    for k, v in fields.items():
        if k in ("photon_grid_min", "photon_grid_max"):
            getattr(cfg, k)[:] = [float(x) for x in v]
        else:
            setattr(cfg, k, v)
    return cfg


class Renderer:
    """RenderDriver / RenderTaskRenderer equivalent (wf_renderer_*)."""

    def __init__(self, device_scene, camera, config, stream=None):
        self.scene = device_scene
        self.config = config
        self.width, self.height = config.width, config.height
        handle = C.c_void_p()
        cam = camera_struct(camera)
        check(library().wf_renderer_create(device_scene.handle, C.byref(cam), C.byref(config), stream,
                                           C.byref(handle)))
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            library().wf_renderer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, x, y, w, h, sample_start, sample_count, clear_tile=True):
        check(library().wf_render(self.handle, x, y, w, h, sample_start, sample_count, int(clear_tile)))

    def render_task(self, tile, sample_start, sample_count):
        """RenderTaskRenderer::render: unnormalized tile sums over the sample range."""
        x, y, w, h = tile
        self.render(x, y, w, h, sample_start, sample_count, True)
        return self.download(x, y, w, h)

    def render_frame(self, sample_count):
        check(library().wf_render_frame(self.handle, sample_count))

    def synchronize(self):
        check(library().wf_synchronize(self.handle))

    def set_watchdog(self, barrier_cycles=0, loop_iterations=0):
        """wf_renderer_set_watchdog: bounds of the device-side waits (0 = default)."""
        check(library().wf_renderer_set_watchdog(self.handle, int(barrier_cycles), int(loop_iterations)))

    def reset(self):
        check(library().wf_framebuffer_reset(self.handle))

    def download(self, x=0, y=0, w=None, h=None):
        w = self.width if w is None else w
        h = self.height if h is None else h
        out = np.empty((h, w, 3), np.float32)
        check(library().wf_framebuffer_download(self.handle, x, y, w, h, out.ctypes.data))
        return out

    def download_async(self, out, x=0, y=0):
        """wf_framebuffer_download_async into `out`, a C-contiguous
        (h, w, 3) float32 host array (numpy, or a torch CPU tensor, pinned
        for the copy to overlap later renders); returns at once.  `out` holds
        the tile once download_wait() has returned."""
        h, w = int(out.shape[0]), int(out.shape[1])
        ptr = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
        check(library().wf_framebuffer_download_async(self.handle, x, y, w, h, ptr))

    def download_wait(self):
        check(library().wf_framebuffer_download_wait(self.handle))

    def sample_index(self):
        v = C.c_uint32()
        check(library().wf_get_sample_index(self.handle, C.byref(v)))
        return v.value

    def set_sample_index(self, value):
        check(library().wf_set_sample_index(self.handle, value))

    def queue_counts(self):
        out = np.zeros(self.config.max_depth, np.uint32)
        check(library().wf_queue_counts(self.handle, out.ctypes.data, len(out)))
        return out

    def stats(self, reset=False):
        s = abi.RenderStats()
        check(library().wf_render_stats_get(self.handle, C.byref(s), int(reset)))
        return {"extension_rays": s.extension_rays, "shadow_rays": s.shadow_rays, "paths": s.paths,
                "kernel_launches": s.kernel_launches}

    def profile_sample(self):
        """wf_profile_sample: per-kernel event times and traversal tallies of
        one extra sample pass (accumulates into the framebuffer)."""
        p = abi.KernelProfile()
        check(library().wf_profile_sample(self.handle, C.byref(p)))
        out = {name: {"launches": p.launches[i], "ms": p.milliseconds[i]} for i, name in enumerate(abi.KERNEL_NAMES)}
        for f, _ in abi.KernelProfile._fields_[2:12]:
            out[f] = getattr(p, f)
        depth = min(self.config.max_depth, abi.PROFILE_BOUNCES)
        out["bounces"] = [{"extension_rays": p.bounce_extension_rays[b], "shadow_rays": p.bounce_shadow_rays[b],
                           **{k: p.bounce_milliseconds[i][b] for i, k in enumerate(("trace_ms", "shade_ms",
                                                                                     "shadow_ms", "finalize_ms",
                                                                                     "gather_ms"))}}
                          for b in range(depth)]
        return out

    def photon_stats(self):
        stored, emitted = C.c_uint32(), C.c_uint32()
        check(library().wf_photon_stats(self.handle, C.byref(stored), C.byref(emitted)))
        return stored.value, emitted.value

    def photons(self):
        _, emitted = self.photon_stats()
        out = np.zeros((emitted, 8), np.float32)
        check(library().wf_photons_download(self.handle, out.ctypes.data, emitted))
        return out

    def checkpoint_save(self, path, fingerprint):
        check(library().wf_checkpoint_save(self.handle, os.fsencode(path), fingerprint))

    def checkpoint_enqueue(self, path, fingerprint):
        q = C.c_uint32()
        check(library().wf_checkpoint_enqueue(self.handle, os.fsencode(path), fingerprint, C.byref(q)))
        return bool(q.value)

    def checkpoint_flush(self):
        check(library().wf_checkpoint_flush(self.handle))

    def checkpoint_load(self, path, fingerprint):
        s = C.c_uint32()
        check(library().wf_checkpoint_load(self.handle, os.fsencode(path), fingerprint, C.byref(s)))
        return s.value


_TUNED = {}


def autotune(device_scene, camera, config, modes=(abi.MODE_GRAPH, abi.MODE_STREAM), block_sizes=(128,),
             refill_thresholds=(4, 8, 16), concurrent_tiles=(1, 2), regenerate_percents=(10, 25),
             chunks=(), persistent_stages=(abi.PERSISTENT_FUSED, abi.PERSISTENT_STAGED), tile_sizes=(), samples=1,
             samples_per_waves=(), stream=None, key=None, cache_path=None):
    """wf_renderer_autotune: times one frame per candidate setting and
    returns (best RenderConfig, [(candidate settings, ms), ...]).

    The choice is cached for the process under `key` (default: the scene
    handle, camera, base config and candidate lists) and, with `cache_path`,
    in that JSON file, so a later call with the same key returns the stored
    settings without rendering (the table is then empty)."""
    import json
    fields = ("mode", "block_size", "refill_threshold", "tile_width", "tile_height", "concurrent_tiles",
              "regenerate_percent", "chunk", "persistent_stages", "samples_per_wave")
    if key is None:
        key = repr((device_scene.handle.value, sorted((k, tuple(v) if hasattr(v, "__len__") else v)
                                                      for k, v in camera.items()),
                    bytes(config), modes, block_sizes, refill_thresholds, concurrent_tiles, regenerate_percents,
                    chunks, persistent_stages, tile_sizes, samples, samples_per_waves))
    stored = _TUNED.get(key)
    if stored is None and cache_path is not None and os.path.exists(cache_path):
        with open(cache_path) as f:
            stored = json.load(f).get(key)
    if stored is not None:
        best = abi.RenderConfig.from_buffer_copy(bytes(config))
        for k in fields:
            setattr(best, k, stored.get(k, getattr(config, k)))
        return best, []

    def arr(v):
        a = (C.c_uint32 * max(1, len(v)))(*v)
        return a, len(v)
    lists = {}
    space = abi.TuneSpace()
    for name, vals in (("modes", modes), ("block_sizes", block_sizes), ("refill_thresholds", refill_thresholds),
                       ("concurrent_tiles", concurrent_tiles), ("regenerate_percents", regenerate_percents),
                       ("chunks", chunks), ("persistent_stages", persistent_stages), ("tile_sizes", tile_sizes),
                       ("samples_per_waves", samples_per_waves)):
        a, n = arr(list(vals))
        lists[name] = a
        setattr(space, name, C.cast(a, C.c_void_p))
        count_field = {"modes": "mode_count", "block_sizes": "block_size_count",
                       "refill_thresholds": "refill_threshold_count", "concurrent_tiles": "concurrent_tiles_count",
                       "regenerate_percents": "regenerate_percent_count", "chunks": "chunk_count",
                       "persistent_stages": "persistent_stage_count", "tile_sizes": "tile_size_count",
                       "samples_per_waves": "samples_per_wave_count"}[name]
        setattr(space, count_field, n)
    space.samples = samples
    capacity = 4096
    times = (C.c_float * capacity)()
    evaluated = C.c_uint32()
    best = abi.RenderConfig()
    cam = camera_struct(camera)
    check(library().wf_renderer_autotune(device_scene.handle, C.byref(cam), C.byref(config), C.byref(space), stream,
                                         C.byref(best), times, capacity, C.byref(evaluated)))
    # candidate settings in the tuner's loop order
    table = []
    base_tile = config.tile_width if config.tile_width == config.tile_height else 0
    for mode in (modes or (config.mode,)):
        if mode == abi.MODE_GRAPH:
            own = [{"concurrent_tiles": v, "samples_per_wave": w}
                   for v in (concurrent_tiles or (config.concurrent_tiles,))
                   for w in (samples_per_waves or (config.samples_per_wave,))]
        elif mode == abi.MODE_STREAM:
            own = [{"regenerate_percent": v} for v in (regenerate_percents or (config.regenerate_percent,))]
        else:
            own = []
            for k in (persistent_stages or (config.persistent_stages,)):
                if k == abi.PERSISTENT_STAGED:
                    own.append({"persistent_stages": k})
                else:
                    own += [{"persistent_stages": k, "chunk": ch} for ch in (chunks or (config.chunk,))]
        for b in (block_sizes or (config.block_size,)):
            for rf in (refill_thresholds or (config.refill_threshold,)):
                for t in (tile_sizes or (base_tile,)):
                    for o in own:
                        table.append(dict({"mode": mode, "block_size": b, "refill_threshold": rf, "tile": t}, **o))
    # a candidate skipped for lack of device memory has no time (None)
    table = [(cand, times[i] if times[i] != float("inf") else None) for i, cand in enumerate(table[:evaluated.value])]
    chosen = {k: getattr(best, k) for k in fields}
    _TUNED[key] = chosen
    if cache_path is not None:
        data = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                data = json.load(f)
        data[key] = chosen
        with open(cache_path, "w") as f:
            json.dump(data, f)
    return best, table


class Batch:
    """Many render jobs in one captured graph (wf_batch_*).  `jobs` is a list
    of dicts: scene (DeviceScene), camera (camera dict), config
    (render_config), sample_start, sample_count."""

    def __init__(self, jobs, slot_capacity=0, block_size=0, refill_threshold=0, longest_first=True, stream=None,
                 config=None, pass_paths=0):
        arr = (abi.BatchJob * len(jobs))()
        self.jobs = list(jobs)
        for i, j in enumerate(jobs):
            arr[i].scene = j["scene"].handle
            arr[i].camera = camera_struct(j["camera"])
            arr[i].config = j["config"]
            arr[i].sample_start = j.get("sample_start", 0)
            arr[i].sample_count = j["sample_count"]
        self._arr = arr
        if config is None:
            config = abi.BatchConfig()
            library().wf_batch_config_default(C.byref(config))
            config.slot_capacity = slot_capacity
            config.block_size = block_size
            config.refill_threshold = refill_threshold
            config.longest_first = int(longest_first)
            config.pass_paths = pass_paths
        self.config = config
        handle = C.c_void_p()
        check(library().wf_batch_create(arr, len(jobs), C.byref(config), stream, C.byref(handle)))
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            library().wf_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self):
        check(library().wf_batch_run(self.handle))

    def synchronize(self):
        check(library().wf_batch_synchronize(self.handle))

    def reset(self):
        check(library().wf_batch_reset(self.handle))

    def download(self, job):
        cfg = self.jobs[job]["config"]
        out = np.empty((cfg.height, cfg.width, 3), np.float32)
        check(library().wf_batch_download(self.handle, job, out.ctypes.data))
        return out

    def stats(self, reset=False):
        s = abi.RenderStats()
        check(library().wf_batch_stats(self.handle, C.byref(s), int(reset)))
        return {"extension_rays": s.extension_rays, "shadow_rays": s.shadow_rays, "paths": s.paths,
                "kernel_launches": s.kernel_launches}

    @staticmethod
    def autotune(jobs, slot_capacities=(0,), block_sizes=(128,), refill_thresholds=(8,), stream=None):
        """wf_batch_autotune: times one run per candidate, returns (best
        BatchConfig, list of candidate times in ms)."""
        arr = (abi.BatchJob * len(jobs))()
        for i, j in enumerate(jobs):
            arr[i].scene = j["scene"].handle
            arr[i].camera = camera_struct(j["camera"])
            arr[i].config = j["config"]
            arr[i].sample_start = j.get("sample_start", 0)
            arr[i].sample_count = j["sample_count"]

        def zlist(v):
            a = (C.c_uint32 * (len(v) + 1))(*v, 0)
            return a
        caps, blocks, refills = zlist(slot_capacities), zlist(block_sizes), zlist(refill_thresholds)
        n = max(1, len(slot_capacities)) * len(block_sizes) * len(refill_thresholds)
        times = (C.c_float * n)()
        best = abi.BatchConfig()
        check(library().wf_batch_autotune(arr, len(jobs), caps, blocks, refills, stream, C.byref(best), times, n))
        return best, list(times)
