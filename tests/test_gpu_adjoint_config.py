"""The path-replay adjoint on the inverse-rendering configuration's own scene:
the Cornell box whose five walls are subdivided into 10,240 triangles, each
with its own RGB albedo and Oren-Nayar roughness, at 512x512 and depth 6.

The configuration renders 32 spp; these checks use fewer samples, which
changes only how many paths each check replays, not the scene, the image size
or the depth:
* the FP64 host adjoint on a 32x32 crop at 4 spp: the GPU crop image within
  1e-4 and the gradient vector within 1e-3 (relative L2);
* central finite differences (eps = 1e-3) of the GPU forward over the whole
  512x512 image at 2 spp, on 256 random parameters with a visible gradient:
  each within 2 %."""
import numpy as np
import pytest

import oracle
import wfpt
from wfpt import diff, scenes

pytestmark = pytest.mark.gpu

W = H = 512
DEPTH = 6


@pytest.fixture(scope="module")
def setup(cuda):
    torch = cuda
    scene, cam, n, _ = scenes.cornell_inverse(W, H, cells=32)
    gt_a, gt_r = scenes.inverse_parameters(scene, n, seed=101)
    a0, r0 = scenes.inverse_parameters(scene, n, seed=202)
    dev = wfpt.DeviceScene(scene)
    yield dict(torch=torch, scene=scene, cam=cam, n=n, dev=dev, gt=(gt_a, gt_r), init=(a0, r0))
    dev.close()


def _t(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def test_scene_is_the_configuration(setup):
    scene, n = setup["scene"], setup["n"]
    # 5 walls x 32 x 32 cells x 2 triangles, plus the light and the two boxes
    assert n >= 10_240 and n == scene.triangle_count()


@pytest.mark.skipif(not oracle.port_available(det=True), reason="oracle/_build/liboracle_det.so not built")
def test_crop_matches_fp64_host_adjoint(setup):
    torch, cam, n = setup["torch"], setup["cam"], setup["n"]
    a, r = setup["init"]
    ga_t, gr_t = setup["gt"]
    crop = (240, 300, 32, 32)  # a crop on the back wall and floor
    full = diff.diff_config(W, H, 4, DEPTH, n)
    target = diff.forward(setup["dev"], cam, full, _t(torch, ga_t), _t(torch, gr_t), 1.0)
    cfg = diff.diff_config(W, H, 4, DEPTH, n, crop=crop)
    img = diff.forward(setup["dev"], cam, cfg, _t(torch, a), _t(torch, r), 0.9)
    d_image = 2.0 * (img - target)
    d_image[img == 0] = 0.0  # outside the crop
    ga, gr, gs = diff.backward(setup["dev"], cam, cfg, _t(torch, a), _t(torch, r), 0.9, d_image)
    port = oracle.PortScene(setup["scene"], det=True)
    host, ha, hr, hs = port.diff(cam, cfg, a, r, 0.9, d_image=d_image.cpu().numpy())
    x, y, w, h = crop
    gpu_crop = img.cpu().numpy()[y:y + h, x:x + w]
    assert host.mean() > 0
    assert np.abs(gpu_crop - host).max() <= 1e-4 * max(1.0, np.abs(host).max())
    g = np.concatenate([ga.cpu().numpy().ravel(), gr.cpu().numpy(), gs.cpu().numpy()])
    hv = np.concatenate([ha.ravel(), hr, [hs]])
    assert np.count_nonzero(hv) > 100 and np.linalg.norm(hv) > 0
    assert np.linalg.norm(g - hv) <= 1e-3 * np.linalg.norm(hv)


def test_central_differences_on_256_parameters(setup):
    torch, cam, n = setup["torch"], setup["cam"], setup["n"]
    a, r = setup["init"]
    ga_t, gr_t = setup["gt"]
    cfg = diff.diff_config(W, H, 2, DEPTH, n, sample_start=3)
    target = diff.forward(setup["dev"], cam, cfg, _t(torch, ga_t), _t(torch, gr_t), 1.0).double()
    A, R = _t(torch, a), _t(torch, r)

    def loss(av, rv, s):
        img = diff.forward(setup["dev"], cam, cfg, av, rv, s).double()
        return float(((img - target) ** 2).sum())

    img = diff.forward(setup["dev"], cam, cfg, A, R, 1.0)
    ga, gr, gs = diff.backward(setup["dev"], cam, cfg, A, R, 1.0, 2.0 * (img.double() - target).float())
    ga, gr, gs = ga.cpu().numpy(), gr.cpu().numpy(), float(gs.cpu().numpy()[0])
    scale = max(np.abs(ga).max(), np.abs(gr).max())
    live_a = np.flatnonzero(np.abs(ga).ravel() > 1e-3 * scale)
    live_r = np.flatnonzero(np.abs(gr) > 1e-3 * scale)
    rng = np.random.default_rng(17)
    pick_a = rng.choice(live_a, size=min(200, len(live_a)), replace=False)
    pick_r = rng.choice(live_r, size=min(255 - len(pick_a), len(live_r)), replace=False)
    eps = 1e-3
    checked = bad = 0
    worst = []
    for j in pick_a:
        k, c = divmod(int(j), 3)
        ap, am = A.clone(), A.clone()
        ap[k, c] += eps
        am[k, c] -= eps
        fd = (loss(ap, R, 1.0) - loss(am, R, 1.0)) / (2 * eps)
        g = ga[k, c]
        checked += 1
        err = abs(fd - g) / max(abs(fd), abs(g))
        bad += err > 0.02
        worst.append(err)
    for k in pick_r:
        rp, rm = R.clone(), R.clone()
        rp[k] += eps
        rm[k] -= eps
        fd = (loss(A, rp, 1.0) - loss(A, rm, 1.0)) / (2 * eps)
        checked += 1
        err = abs(fd - gr[k]) / max(abs(fd), abs(gr[k]))
        bad += err > 0.02
        worst.append(err)
    fd = (loss(A, R, 1.0 + eps) - loss(A, R, 1.0 - eps)) / (2 * eps)
    checked += 1
    bad += abs(fd - gs) > 0.02 * max(abs(fd), abs(gs))
    assert checked == 256
    assert bad == 0, f"{bad} of {checked} parameters differ from central differences by more than 2% " \
                     f"(worst {max(worst):.4f})"
