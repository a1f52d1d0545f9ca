"""Differentiable rendering over the C ABI (wf_diff_forward / wf_diff_backward).

`render(scene, camera, config, albedo, roughness, emission_scale)` is a
torch.autograd.Function: its forward is the path tracer of wf_diff_forward
and its backward is the path-replay adjoint of wf_diff_backward, which
re-traces every path from its RNG key instead of storing it.  Parameters are
CUDA float32 tensors: albedo (N, 3), roughness (N,) in radians, emission
scale (1,).  The image is (height, width, 3).

`albedo_gradient(renderer, materials, adjoint, ...)` differentiates the
production renderer instead (wf_render_albedo_gradient): the gradient of
sum(adjoint * image) with respect to the albedo of diffuse materials of the
renderer's scene, replaying its own shading.
"""
import ctypes as C

import torch

from . import abi
from .native import camera_struct, check, library


def diff_config(width, height, spp, max_depth, parameter_count, sample_start=0, rng=abi.RNG_XORSHIFT32,
                crop=None):
    cfg = abi.DiffConfig()
    cfg.width, cfg.height, cfg.spp, cfg.max_depth = width, height, spp, max_depth
    cfg.parameter_count, cfg.sample_start, cfg.rng = parameter_count, sample_start, rng
    if crop is not None:
        cfg.crop_x, cfg.crop_y, cfg.crop_width, cfg.crop_height = crop
    return cfg


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def forward(scene, camera, config, albedo, roughness, emission_scale):
    image = torch.zeros((config.height, config.width, 3), dtype=torch.float32, device=albedo.device)
    cam = camera_struct(camera)
    check(library().wf_diff_forward(scene.handle, C.byref(cam), C.byref(config), C.c_void_p(albedo.data_ptr()),
                                    C.c_void_p(roughness.data_ptr()), float(emission_scale), C.c_void_p(image.data_ptr()),
                                    _stream()))
    return image


def backward(scene, camera, config, albedo, roughness, emission_scale, d_image):
    """Returns float64 gradients (d_albedo (N, 3), d_roughness (N,), d_emission_scale (1,))."""
    d_image = d_image.contiguous().float()
    ga = torch.zeros(albedo.shape, dtype=torch.float64, device=albedo.device)
    gr = torch.zeros(roughness.shape, dtype=torch.float64, device=albedo.device)
    gs = torch.zeros(1, dtype=torch.float64, device=albedo.device)
    cam = camera_struct(camera)
    check(library().wf_diff_backward(scene.handle, C.byref(cam), C.byref(config), C.c_void_p(albedo.data_ptr()),
                                     C.c_void_p(roughness.data_ptr()), float(emission_scale),
                                     C.c_void_p(d_image.data_ptr()), C.c_void_p(ga.data_ptr()),
                                     C.c_void_p(gr.data_ptr()), C.c_void_p(gs.data_ptr()), _stream()))
    return ga, gr, gs


class DiffRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, albedo, roughness, emission_scale, scene, camera, config):
        albedo = albedo.contiguous()
        roughness = roughness.contiguous()
        scale = float(emission_scale.reshape(-1)[0])
        ctx.save_for_backward(albedo, roughness)
        ctx.scene, ctx.camera, ctx.config, ctx.scale = scene, camera, config, scale
        return forward(scene, camera, config, albedo, roughness, scale)

    @staticmethod
    def backward(ctx, grad_image):
        albedo, roughness = ctx.saved_tensors
        ga, gr, gs = backward(ctx.scene, ctx.camera, ctx.config, albedo, roughness, ctx.scale, grad_image)
        return ga.to(albedo.dtype), gr.to(roughness.dtype), gs.float(), None, None, None


def render(scene, camera, config, albedo, roughness, emission_scale):
    return DiffRender.apply(albedo, roughness, emission_scale, scene, camera, config)


def albedo_gradient(renderer, materials, adjoint, tile=None, sample_start=0, sample_count=1, image=False):
    """wf_render_albedo_gradient: gradients of the production renderer's image.

    Returns the float64 (len(materials), 3) derivative of
    sum(adjoint * image) with respect to the RGB albedo of each listed
    diffuse material, where image is the sum of samples
    [sample_start, sample_start + sample_count) that `renderer` (a
    wfpt.Renderer) renders over `tile` (x, y, w, h; default the whole
    image); Russian roulette's weights are held constant.  `adjoint` is a
    (height, width, 3) CUDA float32 tensor.  With image=True also returns
    the replayed (height, width, 3) image (only the tile is written), equal
    bit for bit to what renderer.render_task returns for the same tile and
    samples."""
    x, y, w, h = tile if tile is not None else (0, 0, renderer.width, renderer.height)
    adjoint = adjoint.contiguous().float()
    if tuple(adjoint.shape) != (renderer.height, renderer.width, 3):
        raise ValueError("adjoint must be (height, width, 3)")
    ids = (C.c_uint32 * len(materials))(*[int(m) for m in materials])
    grad = torch.zeros((len(materials), 3), dtype=torch.float64, device=adjoint.device)
    out = torch.zeros_like(adjoint) if image else None
    torch.cuda.current_stream().synchronize()  # the call runs on the renderer's stream
    check(library().wf_render_albedo_gradient(renderer.handle, x, y, w, h, sample_start, sample_count, ids,
                                              len(materials), C.c_void_p(adjoint.data_ptr()),
                                              C.c_void_p(out.data_ptr()) if image else None,
                                              C.c_void_p(grad.data_ptr())))
    return (grad, out) if image else grad
