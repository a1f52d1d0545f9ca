"""ctypes/numpy mirror of include/wavefront.h.

Every struct here has the exact layout of its C counterpart; numpy dtypes are
used for the arrays (triangles, spheres, instances, rays, hits) so large
scenes are built without Python loops.
"""
import ctypes as C

import numpy as np

WF_OK = 0
(WF_ERR_INVALID_ARG, WF_ERR_OOM, WF_ERR_CUDA, WF_ERR_TIMEOUT, WF_ERR_FINGERPRINT, WF_ERR_CAPACITY, WF_ERR_IO,
 WF_ERR_FORMAT, WF_ERR_UNSUPPORTED, WF_ERR_STATE) = range(1, 11)
STATUS_NAMES = {
    0: "WF_OK", 1: "WF_ERR_INVALID_ARG", 2: "WF_ERR_OOM", 3: "WF_ERR_CUDA", 4: "WF_ERR_TIMEOUT",
    5: "WF_ERR_FINGERPRINT", 6: "WF_ERR_CAPACITY", 7: "WF_ERR_IO", 8: "WF_ERR_FORMAT",
    9: "WF_ERR_UNSUPPORTED", 10: "WF_ERR_STATE",
}

MAT_DIFFUSE, MAT_METAL, MAT_DIELECTRIC, MAT_EMISSIVE, MAT_SPECGLOSS = 0, 1, 2, 3, 4
ACCEL_BVH, ACCEL_DIRECT = 0, 1
LIGHT_POINT, LIGHT_SPOT, LIGHT_DIRECTIONAL = 0, 1, 2
NO_MATERIAL = 0xFFFFFFFF
MODE_GRAPH, MODE_PERSISTENT, MODE_STREAM = 0, 1, 2
PERSISTENT_AUTO, PERSISTENT_FUSED, PERSISTENT_STAGED = 0, 1, 2
RNG_XORSHIFT32, RNG_PCG32 = 0, 1
DEBUG_NONE, DEBUG_INTERSECTION, DEBUG_SHADING_NORMAL = 0, 1, 2
HIT_NONE, HIT_MESH, HIT_STATIC_TRIANGLE, HIT_TRIANGLE, HIT_SPHERE = 0, 1, 2, 3, 4

TRIANGLE_DTYPE = np.dtype([
    ("v0", "<f4", (3,)), ("v1", "<f4", (3,)), ("v2", "<f4", (3,)),
    ("n0", "<f4", (3,)), ("n1", "<f4", (3,)), ("n2", "<f4", (3,)),
    ("material", "<u4"), ("has_vertex_normals", "<u4"),
])
SPHERE_DTYPE = np.dtype([("center", "<f4", (3,)), ("radius", "<f4"), ("material", "<u4"), ("accel", "<u4")])
MESH_DTYPE = np.dtype([("triangles", "<u8"), ("triangle_count", "<u4"), ("pad", "<u4"), ("attributes", "<u8")])
# Texture coordinates and tangent frames of a triangle (wf_triangle_attributes).
TRIANGLE_ATTRIBUTES_DTYPE = np.dtype([
    ("uv", "<f4", (3, 2)), ("uv1", "<f4", (3, 2)),
    ("tangent", "<f4", (3,)), ("bitangent", "<f4", (3,)), ("tangent1", "<f4", (3,)), ("bitangent1", "<f4", (3,)),
    ("vertex_tangent", "<f4", (3, 3)), ("vertex_tangent_sign", "<f4", (3,)),
    ("has_vertex_tangents", "<u4"), ("has_texcoords", "<u4"), ("has_texcoords1", "<u4"),
])
NO_TEXTURE = 0xFFFFFFFF
TEXTURE_DTYPE = np.dtype([("width", "<u4"), ("height", "<u4"), ("rgba", "<u8")])
TEXTURE_BINDING_DTYPE = np.dtype([
    ("texture", "<u4"), ("texcoord", "<u4"), ("offset", "<f4", (2,)), ("scale", "<f4", (2,)),
    ("rotation", "<f4"), ("has_transform", "<u4"),
])
TEXTURE_SLOTS = ("albedo", "metallic_roughness", "emissive", "normal", "thickness", "specular_glossiness",
                 "specular_weight", "specular_color", "clearcoat", "clearcoat_roughness", "clearcoat_normal")
MATERIAL_TEXTURES_DTYPE = np.dtype([("normal_scale", "<f4"), ("clearcoat_normal_scale", "<f4")] +
                                   [(k, TEXTURE_BINDING_DTYPE) for k in TEXTURE_SLOTS])
INSTANCE_DTYPE = np.dtype([
    ("mesh", "<u4"), ("material_override", "<u4"), ("accel", "<u4"),
    ("local_to_world", "<f4", (3, 3)), ("world_to_local", "<f4", (3, 3)), ("translation", "<f4", (3,)),
])
MATERIAL_DTYPE = np.dtype([
    ("type", "<u4"), ("albedo", "<f4", (3,)), ("emission", "<f4", (3,)),
    ("roughness", "<f4"), ("ior", "<f4"), ("dispersion", "<f4"), ("metallic", "<f4"),
    ("attenuation_color", "<f4", (3,)), ("attenuation_distance", "<f4"), ("volume_density", "<f4"),
    ("opacity", "<f4"), ("alpha_cutoff", "<f4"), ("alpha_masked", "<u4"),
    ("specgloss_workflow", "<u4"), ("gltf_pbr", "<u4"),
    ("specular", "<f4", (3,)), ("glossiness", "<f4"), ("specular_weight", "<f4"),
    ("specular_color", "<f4", (3,)), ("clearcoat", "<f4"), ("clearcoat_roughness", "<f4"),
])
PUNCTUAL_DTYPE = np.dtype([
    ("type", "<u4"), ("position", "<f4", (3,)), ("direction", "<f4", (3,)), ("intensity", "<f4", (3,)),
    ("range", "<f4"), ("inner_cone_cos", "<f4"), ("outer_cone_cos", "<f4"),
])
RAY_DTYPE = np.dtype([("origin", "<f4", (3,)), ("direction", "<f4", (3,))])
HIT_DTYPE = np.dtype([
    ("t", "<f4"), ("position", "<f4", (3,)), ("geometric_normal", "<f4", (3,)), ("normal", "<f4", (3,)),
    ("material", "<u4"), ("light_index", "<u4"), ("kind", "<u4"), ("instance", "<u4"), ("primitive", "<u4"),
    ("u", "<f4"), ("v", "<f4"),
])
# wf_frame_guide (FrameGuide, include/renderer/frame_guides.cuh:9-17)
FRAME_GUIDE_DTYPE = np.dtype([
    ("albedo", "<f4", (3,)), ("normal", "<f4", (3,)), ("geometric_normal", "<f4", (3,)), ("depth", "<f4"),
    ("motion", "<f4", (2,)), ("valid", "<f4"), ("history_valid", "<f4"),
])

assert TRIANGLE_DTYPE.itemsize == 80 and SPHERE_DTYPE.itemsize == 24 and INSTANCE_DTYPE.itemsize == 96
assert MESH_DTYPE.itemsize == 24 and TRIANGLE_ATTRIBUTES_DTYPE.itemsize == 156 and TEXTURE_DTYPE.itemsize == 16
assert TEXTURE_BINDING_DTYPE.itemsize == 32 and MATERIAL_TEXTURES_DTYPE.itemsize == 360
assert MATERIAL_DTYPE.itemsize == 124 and PUNCTUAL_DTYPE.itemsize == 52
assert RAY_DTYPE.itemsize == 24 and HIT_DTYPE.itemsize == 68 and FRAME_GUIDE_DTYPE.itemsize == 56


BVH_HOST_SAH = 0
BVH_GPU_PLOC = 1


class SceneDesc(C.Structure):
    _fields_ = [
        ("spheres", C.c_void_p), ("sphere_count", C.c_uint32),
        ("triangles", C.c_void_p), ("triangle_count", C.c_uint32),
        ("static_triangles", C.c_void_p), ("static_triangle_count", C.c_uint32),
        ("meshes", C.c_void_p), ("mesh_count", C.c_uint32),
        ("instances", C.c_void_p), ("instance_count", C.c_uint32),
        ("materials", C.c_void_p), ("material_count", C.c_uint32),
        ("punctual_lights", C.c_void_p), ("punctual_light_count", C.c_uint32),
        ("black_background", C.c_uint32),
        ("ignore_direct_light_occlusion", C.c_uint32),
        ("register_triangle_lights", C.c_uint32),
        ("build_threads", C.c_uint32),
        ("bvh_builder", C.c_uint32), ("reserved", C.c_uint32),
        ("textures", C.c_void_p), ("texture_count", C.c_uint32), ("disable_normal_maps", C.c_uint32),
        ("material_textures", C.c_void_p), ("triangle_attributes", C.c_void_p),
        ("static_triangle_attributes", C.c_void_p), ("normal_map_minimum_cosine", C.c_float),
        ("reserved2", C.c_uint32),
    ]


class Environment(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("rgba", C.c_void_p),
                ("intensity", C.c_float), ("rotation_degrees", C.c_float)]


class SceneInfo(C.Structure):
    _fields_ = [("light_count", C.c_uint32), ("tlas_leaf_count", C.c_uint32), ("blas_count", C.c_uint32),
                ("material_count", C.c_uint32), ("device_bytes", C.c_uint64), ("build_seconds", C.c_double),
                ("gpu_bvh_builds", C.c_uint32), ("bvh_build_ms", C.c_float)]


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("forward", C.c_float * 3), ("right", C.c_float * 3),
                ("up", C.c_float * 3), ("vertical_fov", C.c_float), ("aspect_ratio", C.c_float)]


class RenderConfig(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("max_depth", C.c_uint32), ("rr_start_depth", C.c_uint32),
        ("mode", C.c_uint32), ("rng", C.c_uint32),
        ("indirect_clamp", C.c_float),
        ("tile_width", C.c_uint32), ("tile_height", C.c_uint32),
        ("block_size", C.c_uint32), ("persistent_blocks", C.c_uint32), ("chunk", C.c_uint32),
        ("debug", C.c_uint32),
        ("caustics", C.c_uint32), ("caustic_gather", C.c_uint32),
        ("photon_count", C.c_uint32), ("photon_max_depth", C.c_uint32),
        ("gather_radius", C.c_float),
        ("photon_grid_min", C.c_float * 3), ("photon_grid_max", C.c_float * 3),
        ("photon_grid_resolution", C.c_uint32), ("photon_seed", C.c_uint32), ("spectral", C.c_uint32),
        ("profile_queues", C.c_uint32), ("refill_threshold", C.c_uint32), ("concurrent_tiles", C.c_uint32),
        ("shadow_queue_capacity", C.c_uint32), ("regenerate_percent", C.c_uint32),
        ("persistent_stages", C.c_uint32),
        ("samples_per_wave", C.c_uint32),
    ]


class TuneSpace(C.Structure):
    _fields_ = [("modes", C.c_void_p), ("mode_count", C.c_uint32),
                ("block_sizes", C.c_void_p), ("block_size_count", C.c_uint32),
                ("refill_thresholds", C.c_void_p), ("refill_threshold_count", C.c_uint32),
                ("concurrent_tiles", C.c_void_p), ("concurrent_tiles_count", C.c_uint32),
                ("regenerate_percents", C.c_void_p), ("regenerate_percent_count", C.c_uint32),
                ("chunks", C.c_void_p), ("chunk_count", C.c_uint32),
                ("persistent_stages", C.c_void_p), ("persistent_stage_count", C.c_uint32),
                ("tile_sizes", C.c_void_p), ("tile_size_count", C.c_uint32),
                ("samples", C.c_uint32),
                ("samples_per_waves", C.c_void_p), ("samples_per_wave_count", C.c_uint32)]


class BatchJob(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", Camera), ("config", RenderConfig),
                ("sample_start", C.c_uint32), ("sample_count", C.c_uint32)]


class BatchConfig(C.Structure):
    _fields_ = [("slot_capacity", C.c_uint32), ("block_size", C.c_uint32), ("refill_threshold", C.c_uint32),
                ("longest_first", C.c_uint32), ("pass_paths", C.c_uint32)]


class DiffConfig(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("crop_x", C.c_uint32), ("crop_y", C.c_uint32),
                ("crop_width", C.c_uint32), ("crop_height", C.c_uint32), ("spp", C.c_uint32),
                ("sample_start", C.c_uint32), ("max_depth", C.c_uint32), ("rng", C.c_uint32),
                ("parameter_count", C.c_uint32)]


PROFILE_BOUNCES = 32
KERNEL_NAMES = ["raygen", "trace", "shade", "shadow", "finalize", "persistent", "gather"]


class KernelProfile(C.Structure):
    _fields_ = [("launches", C.c_uint32 * 7), ("milliseconds", C.c_float * 7),
                ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("closest_nodes", C.c_uint64), ("closest_triangles", C.c_uint64),
                ("closest_spheres", C.c_uint64), ("closest_instances", C.c_uint64),
                ("any_nodes", C.c_uint64), ("any_triangles", C.c_uint64),
                ("any_spheres", C.c_uint64), ("any_instances", C.c_uint64),
                ("bounce_milliseconds", (C.c_float * PROFILE_BOUNCES) * 5),
                ("bounce_extension_rays", C.c_uint32 * PROFILE_BOUNCES),
                ("bounce_shadow_rays", C.c_uint32 * PROFILE_BOUNCES)]


class RenderStats(C.Structure):
    _fields_ = [("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("paths", C.c_uint64),
                ("kernel_launches", C.c_uint64)]


def declare(lib):
    """Declares the signatures of every entry point of include/wavefront.h."""
    P, U32, U64, F = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float
    S = C.c_int32
    sigs = {
        "wf_last_error": (C.c_char_p, []),
        "wf_version": (C.c_char_p, []),
        "wf_material_default": (None, [P, U32]),
        "wf_scene_create": (S, [C.POINTER(SceneDesc), C.POINTER(P)]),
        "wf_scene_set_environment": (S, [P, C.POINTER(Environment)]),
        "wf_scene_set_albedos": (S, [P, P, P, U32]),
        "wf_scene_destroy": (S, [P]),
        "wf_scene_get_info": (S, [P, C.POINTER(SceneInfo)]),
        "wf_bvh_build": (S, [U32, P, U32, P, P]),
        "wf_trace_closest": (S, [P, P, U32, P, P]),
        "wf_frame_guides": (S, [P, P, P, U32, U32, U32, U32, U32, U32, P, P]),
        "wf_trace_any": (S, [P, P, P, U32, P, P]),
        "wf_render_config_default": (None, [C.POINTER(RenderConfig), U32, U32]),
        "wf_renderer_create": (S, [P, C.POINTER(Camera), C.POINTER(RenderConfig), P, C.POINTER(P)]),
        "wf_renderer_destroy": (S, [P]),
        "wf_render": (S, [P, U32, U32, U32, U32, U32, U32, U32]),
        "wf_render_frame": (S, [P, U32]),
        "wf_diff_forward": (S, [P, C.POINTER(Camera), C.POINTER(DiffConfig), P, P, F, P, P]),
        "wf_diff_backward": (S, [P, C.POINTER(Camera), C.POINTER(DiffConfig), P, P, F, P, P, P, P, P]),
        "wf_render_albedo_gradient": (S, [P, U32, U32, U32, U32, U32, U32, P, U32, P, P, P]),
        "wf_renderer_autotune": (S, [P, C.POINTER(Camera), C.POINTER(RenderConfig), C.POINTER(TuneSpace), P,
                                     C.POINTER(RenderConfig), P, U32, C.POINTER(U32)]),
        "wf_batch_config_default": (None, [C.POINTER(BatchConfig)]),
        "wf_batch_create": (S, [C.POINTER(BatchJob), U32, C.POINTER(BatchConfig), P, C.POINTER(P)]),
        "wf_batch_run": (S, [P]),
        "wf_batch_synchronize": (S, [P]),
        "wf_batch_reset": (S, [P]),
        "wf_batch_download": (S, [P, U32, P]),
        "wf_batch_framebuffer_device": (S, [P, U32, C.POINTER(P)]),
        "wf_batch_stats": (S, [P, C.POINTER(RenderStats), U32]),
        "wf_batch_destroy": (S, [P]),
        "wf_batch_autotune": (S, [C.POINTER(BatchJob), U32, P, P, P, P, C.POINTER(BatchConfig), P, U32]),
        "wf_render_tile_static": (S, [P, C.POINTER(Camera), C.POINTER(RenderConfig), U32, U32, U32, U32, U32, U32, P,
                                      P]),
        "wf_framebuffer_reset": (S, [P]),
        "wf_set_sample_index": (S, [P, U32]),
        "wf_get_sample_index": (S, [P, C.POINTER(U32)]),
        "wf_framebuffer_download": (S, [P, U32, U32, U32, U32, P]),
        "wf_framebuffer_download_async": (S, [P, U32, U32, U32, U32, P]),
        "wf_framebuffer_download_wait": (S, [P]),
        "wf_framebuffer_device": (S, [P, C.POINTER(P)]),
        "wf_synchronize": (S, [P]),
        "wf_renderer_set_watchdog": (S, [P, U64, U32]),
        "wf_test_fail_allocation": (None, [C.c_int64]),
        "wf_queue_counts": (S, [P, P, U32]),
        "wf_render_stats_get": (S, [P, C.POINTER(RenderStats), U32]),
        "wf_profile_sample": (S, [P, C.POINTER(KernelProfile)]),
        "wf_photon_stats": (S, [P, C.POINTER(U32), C.POINTER(U32)]),
        "wf_photons_download": (S, [P, P, U32]),
        "wf_checkpoint_save": (S, [P, C.c_char_p, U64]),
        "wf_checkpoint_enqueue": (S, [P, C.c_char_p, U64, C.POINTER(U32)]),
        "wf_checkpoint_flush": (S, [P]),
        "wf_checkpoint_load": (S, [P, C.c_char_p, U64, C.POINTER(U32)]),
        "wf_fnv1a64": (U64, [P, C.c_size_t, U64]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return list(sigs)


def ptr(array):
    """Address of a numpy array's data (None for empty arrays)."""
    if array is None or array.size == 0:
        return None
    return array.ctypes.data
