"""Albedo gradients of the production renderer (wf_render_albedo_gradient).

* The replay's image is bit for bit the framebuffer wf_render leaves for the
  same tile and samples (graph mode with and without sample waves and with
  two wavefronts, the persistent and streaming modes; Russian roulette on;
  the three scenes below), so the gradient belongs to the image the
  renderer actually makes.
* With Russian roulette off the gradient is the exact derivative of the
  image: it matches central finite differences of wf_render (eps = 1e-3 on
  one albedo channel at a time, fresh scene per evaluation) on the Cornell
  box, the sphere field (glass, metal and sky on the paths) and a small
  large-mesh scene (instanced rocks, emissive terrain triangles, glass
  spheres, HDR sun-and-sky environment), within 1e-3 of each entry plus
  1e-4 of the largest; on the sphere field also with 8 materials at once.
* With Russian roulette on (weights held constant) it estimates the same
  gradient: 256 samples per pixel agree with the roulette-free gradient
  within 2 % of the gradient's norm.
* Inverse rendering with it: Adam recovers the Cornell walls' albedos from
  a target image rendered with the same samples.
* wf_scene_set_albedos: renderers see the new albedos, bit for bit those of
  a scene built with them.
* The argument checks of the entry point.
"""
import numpy as np
import pytest

import wfpt
from wfpt import abi, diff, scenes

pytestmark = pytest.mark.gpu


def _cornell():
    scene, cam = scenes.cornell_box(64, 64)
    return scene, cam, [0, 1, 2, 3]


def _sphere_field(spheres=2):
    scene, cam = scenes.sphere_field(96, 54, frequency=16)
    mats = scene.materials
    picked = [k for k in range(4, len(mats))
              if mats[k]["type"] == abi.MAT_DIFFUSE and mats[k]["albedo"].min() > 0.1][:spheres]
    return scene, cam, [0, 3] + picked


def _large_mesh():
    scene, cam = scenes.large_mesh(96, 54, terrain_quads=64, instance_count=12, instance_frequency=8,
                                   glass_spheres=3, env_size=(256, 128))
    return scene, cam, [0, 1, 2, 3]


SCENES = {"cornell": (_cornell, 64, 64), "sphere_field": (_sphere_field, 96, 54), "large_mesh": (_large_mesh, 96, 54),
          "sphere_field_8": (lambda: _sphere_field(6), 96, 54)}  # the most parameters a call takes


def _adjoint(torch, w, h, seed):
    rng = np.random.default_rng(seed)
    return torch.from_numpy(rng.uniform(0.5, 1.5, (h, w, 3)).astype(np.float32)).cuda()


def _render(scene, cam, cfg, tile, start, count):
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    try:
        return r.render_task(tile, start, count)
    finally:
        r.close()
        dev.close()


@pytest.mark.parametrize("case", [
    ("cornell", dict(mode=abi.MODE_GRAPH, max_depth=8, rr_start_depth=3), (0, 0, 64, 64), 100, 4),
    ("cornell", dict(mode=abi.MODE_GRAPH, max_depth=8, rr_start_depth=3, samples_per_wave=4), (5, 9, 40, 33), 7, 8),
    ("cornell", dict(mode=abi.MODE_PERSISTENT, max_depth=8, rr_start_depth=3), (0, 0, 64, 64), 0, 3),
    ("cornell", dict(mode=abi.MODE_STREAM, max_depth=8, rr_start_depth=3), (0, 0, 64, 64), 5, 6),
    ("sphere_field", dict(mode=abi.MODE_GRAPH, max_depth=16), (0, 0, 96, 54), 100, 3),
    ("sphere_field", dict(mode=abi.MODE_GRAPH, max_depth=16, samples_per_wave=2), (17, 3, 64, 40), 11, 4),
    ("sphere_field", dict(mode=abi.MODE_GRAPH, max_depth=16, samples_per_wave=2, concurrent_tiles=2), (0, 0, 96, 54),
     3, 4),
    ("large_mesh", dict(mode=abi.MODE_GRAPH, max_depth=12), (0, 0, 96, 54), 100, 2),
], ids=["cornell-graph", "cornell-wave-tile", "cornell-persistent", "cornell-stream", "sphere-graph",
        "sphere-wave-tile", "sphere-two-wavefronts", "large-mesh-graph"])
def test_replay_image_bit_exact(cuda, case):
    torch = cuda
    name, fields, tile, start, count = case
    make, w, h = SCENES[name]
    scene, cam, params = make()
    cfg = wfpt.render_config(w, h, indirect_clamp=0.0, **fields)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    try:
        _, image = diff.albedo_gradient(r, params, _adjoint(torch, w, h, 1), tile, start, count, image=True)
        want = r.render_task(tile, start, count)
    finally:
        r.close()
        dev.close()
    x, y, tw, th = tile
    got = image.cpu().numpy()[y:y + th, x:x + tw]
    bad = np.nonzero(got.view(np.uint32) != want.view(np.uint32))
    assert bad[0].size == 0, f"{bad[0].size} channels differ; first {got[bad[0][0], bad[1][0]]} vs " \
                             f"{want[bad[0][0], bad[1][0]]}"
    assert want.mean() > 0


def _finite_differences(scene, cam, cfg, params, adjoint, spp, eps):
    w, h = cfg.width, cfg.height
    out = np.zeros((len(params), 3))
    for i, m in enumerate(params):
        for c in range(3):
            losses = []
            for sign in (1.0, -1.0):
                albedo = scene.materials["albedo"]  # a view
                saved = float(albedo[m, c])
                albedo[m, c] = saved + sign * eps
                try:
                    img = _render(scene, cam, cfg, (0, 0, w, h), 0, spp)
                finally:
                    albedo[m, c] = saved
                losses.append(float((adjoint.astype(np.float64) * img.astype(np.float64)).sum()))
            out[i, c] = (losses[0] - losses[1]) / (2.0 * eps)
    return out


@pytest.mark.parametrize("name,depth,spp", [("cornell", 8, 8), ("sphere_field", 12, 4), ("large_mesh", 12, 2),
                                            ("sphere_field_8", 12, 4)])
def test_gradient_matches_central_differences(cuda, name, depth, spp):
    torch = cuda
    make, w, h = SCENES[name]
    scene, cam, params = make()
    cfg = wfpt.render_config(w, h, mode=abi.MODE_GRAPH, max_depth=depth, rr_start_depth=depth, indirect_clamp=0.0)
    adjoint = _adjoint(torch, w, h, 2)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    try:
        grad = diff.albedo_gradient(r, params, adjoint, None, 0, spp).cpu().numpy()
    finally:
        r.close()
        dev.close()
    fd = _finite_differences(scene, cam, cfg, params, adjoint.cpu().numpy(), spp, 1e-3)
    assert np.abs(fd).max() > 0
    tol = 1e-3 * np.abs(fd) + 1e-4 * np.abs(fd).max()
    assert np.all(np.abs(grad - fd) <= tol), f"replay\n{grad}\nfinite differences\n{fd}"


def test_russian_roulette_gradient_is_unbiased(cuda):
    torch = cuda
    scene, cam, params = _cornell()
    adjoint = _adjoint(torch, 64, 64, 3)
    grads = []
    for rr in (3, 8):
        cfg = wfpt.render_config(64, 64, mode=abi.MODE_GRAPH, max_depth=8, rr_start_depth=rr, indirect_clamp=0.0)
        dev = wfpt.DeviceScene(scene)
        r = wfpt.Renderer(dev, cam, cfg)
        try:
            grads.append(diff.albedo_gradient(r, params, adjoint, None, 0, 256).cpu().numpy())
        finally:
            r.close()
            dev.close()
    with_rr, exact = grads
    assert np.linalg.norm(with_rr - exact) <= 0.02 * np.linalg.norm(exact), f"{with_rr}\n{exact}"


def test_inverse_rendering_recovers_wall_albedos(cuda):
    torch = cuda
    scene, cam, _ = _cornell()
    walls = [0, 1, 2]
    truth = scene.materials["albedo"][walls].copy()
    cfg = wfpt.render_config(64, 64, mode=abi.MODE_GRAPH, max_depth=6, rr_start_depth=6, indirect_clamp=0.0)
    spp = 8
    target = torch.from_numpy(_render(scene, cam, cfg, (0, 0, 64, 64), 0, spp)).cuda()
    x = torch.full((3, 3), 0.4, dtype=torch.float64, requires_grad=True)
    # a short second-moment memory: the early gradients are far larger
    opt = torch.optim.Adam([x], lr=0.03, betas=(0.9, 0.9))
    schedule = torch.optim.lr_scheduler.ExponentialLR(opt, 0.97)
    losses = []
    for _ in range(120):
        scene.materials["albedo"][walls] = x.detach().clamp(0.02, 0.98).cpu().numpy()
        dev = wfpt.DeviceScene(scene)
        r = wfpt.Renderer(dev, cam, cfg)
        try:
            image = torch.from_numpy(r.render_task((0, 0, 64, 64), 0, spp)).cuda()
            losses.append(float(((image - target) ** 2).sum()))
            x.grad = diff.albedo_gradient(r, walls, 2.0 * (image - target), None, 0, spp).cpu()
        finally:
            r.close()
            dev.close()
        opt.step()
        schedule.step()
    scene.materials["albedo"][walls] = truth
    err = np.abs(x.detach().numpy() - truth).max()
    assert losses[-1] < 1e-4 * losses[0], losses[::10]
    assert err < 0.01, (x.detach().numpy(), truth)


def test_set_albedos_matches_a_fresh_scene(cuda):
    """wf_scene_set_albedos: a renderer made before the update renders, and
    replays, exactly what a scene built with the new albedos renders."""
    torch = cuda
    scene, cam, _ = _cornell()
    cfg = wfpt.render_config(64, 64, mode=abi.MODE_GRAPH, max_depth=8, rr_start_depth=3, indirect_clamp=0.0)
    new = np.array([[0.3, 0.6, 0.2], [0.9, 0.1, 0.4]], np.float32)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    try:
        before = r.render_task((0, 0, 64, 64), 0, 4)
        dev.set_albedos([0, 2], new)
        got = r.render_task((0, 0, 64, 64), 0, 4)
        _, replay = diff.albedo_gradient(r, [0, 2], _adjoint(torch, 64, 64, 5), None, 0, 4, image=True)
        for bad in (([99], new[:1]), ([0], np.array([[np.nan, 0.5, 0.5]], np.float32))):
            with pytest.raises(wfpt.WavefrontError) as e:
                dev.set_albedos(*bad)
            assert e.value.status == abi.WF_ERR_INVALID_ARG
    finally:
        r.close()
        dev.close()
    scene.materials["albedo"][[0, 2]] = new
    want = _render(scene, cam, cfg, (0, 0, 64, 64), 0, 4)
    assert not np.array_equal(before, want)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.array_equal(replay.cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_argument_checks(cuda):
    torch = cuda
    scene, cam, params = _cornell()
    adjoint = _adjoint(torch, 64, 64, 4)
    dev = wfpt.DeviceScene(scene)
    try:
        cfg = wfpt.render_config(64, 64, max_depth=8, indirect_clamp=0.0)
        r = wfpt.Renderer(dev, cam, cfg)
        try:
            bad = [
                (dict(materials=[4]), abi.WF_ERR_UNSUPPORTED),         # the emissive light
                (dict(materials=[99]), abi.WF_ERR_INVALID_ARG),
                (dict(materials=[0, 0]), abi.WF_ERR_INVALID_ARG),
                (dict(materials=list(range(9))), abi.WF_ERR_INVALID_ARG),
                (dict(materials=[0], tile=(60, 0, 8, 8)), abi.WF_ERR_INVALID_ARG),
                (dict(materials=[0], sample_count=0), abi.WF_ERR_INVALID_ARG),
            ]
            for kw, status in bad:
                args = dict(tile=None, sample_start=0, sample_count=1)
                args.update(kw)
                with pytest.raises(wfpt.WavefrontError) as e:
                    diff.albedo_gradient(r, args.pop("materials"), adjoint, **args)
                assert e.value.status == status, kw
            assert diff.albedo_gradient(r, [0], adjoint).abs().sum() > 0  # still usable
        finally:
            r.close()
        for fields in (dict(indirect_clamp=10.0), dict(indirect_clamp=0.0, debug=1)):
            r = wfpt.Renderer(dev, cam, wfpt.render_config(64, 64, max_depth=8, **fields))
            try:
                with pytest.raises(wfpt.WavefrontError) as e:
                    diff.albedo_gradient(r, [0], adjoint)
                assert e.value.status == abi.WF_ERR_UNSUPPORTED
            finally:
                r.close()
    finally:
        dev.close()
