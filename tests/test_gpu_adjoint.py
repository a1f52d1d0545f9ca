"""Path-replay adjoint (wf_diff_forward / wf_diff_backward).

Checks, on the subdivided Cornell box with per-triangle Oren-Nayar albedo
and roughness:
* the GPU image against the FP64 host restatement (same paths, double
  radiometry), relative error below 1e-4;
* the GPU gradients of an L2 image loss against the FP64 host adjoint on a
  crop: relative L2 error of the gradient vector below 1e-3;
* central finite differences (eps = 1e-3) of the GPU forward on 256 random
  parameters: within 2 % (relative to the larger of the two values, for
  parameters whose gradient is not negligible);
* the torch.autograd.Function binding, and that gradient steps lower the loss.
"""
import numpy as np
import pytest

import oracle
import wfpt
from wfpt import diff, scenes

pytestmark = pytest.mark.gpu

W = H = 48


@pytest.fixture(scope="module")
def setup(cuda):
    torch = cuda
    scene, cam, n, _ = scenes.cornell_inverse(W, H, cells=16)
    gt_a, gt_r = scenes.inverse_parameters(scene, n, seed=101)
    a0, r0 = scenes.inverse_parameters(scene, n, seed=202)
    dev = wfpt.DeviceScene(scene)
    yield dict(torch=torch, scene=scene, cam=cam, n=n, dev=dev, gt=(gt_a, gt_r), init=(a0, r0))
    dev.close()


def _t(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def test_forward_matches_fp64_host(setup):
    torch, cam, n = setup["torch"], setup["cam"], setup["n"]
    a, r = setup["init"]
    cfg = diff.diff_config(W, H, 4, 5, n, sample_start=7, crop=(8, 12, 24, 20))
    img = diff.forward(setup["dev"], cam, cfg, _t(torch, a), _t(torch, r), 1.3).cpu().numpy()
    host, _, _, _ = oracle.PortScene(setup["scene"], det=True).diff(cam, cfg, a, r, 1.3)
    crop = img[12:32, 8:32]
    assert host.mean() > 0
    assert np.abs(crop - host).max() <= 1e-4 * max(1.0, np.abs(host).max())
    outside = np.ones((H, W), bool)
    outside[12:32, 8:32] = False
    assert not img[outside].any()


def test_gradients_match_fp64_host_adjoint(setup):
    torch, cam, n = setup["torch"], setup["cam"], setup["n"]
    a, r = setup["init"]
    ga_t, gr_t = setup["gt"]
    full = diff.diff_config(W, H, 4, 5, n)
    target = diff.forward(setup["dev"], cam, full, _t(torch, ga_t), _t(torch, gr_t), 1.0)
    cfg = diff.diff_config(W, H, 4, 5, n, crop=(10, 6, 32, 32))
    img = diff.forward(setup["dev"], cam, cfg, _t(torch, a), _t(torch, r), 0.9)
    d_image = 2.0 * (img - target)
    d_image[img == 0] = 0.0  # outside the crop
    ga, gr, gs = diff.backward(setup["dev"], cam, cfg, _t(torch, a), _t(torch, r), 0.9, d_image)
    _, ha, hr, hs = oracle.PortScene(setup["scene"], det=True).diff(cam, cfg, a, r, 0.9,
                                                                   d_image=d_image.cpu().numpy())
    g = np.concatenate([ga.cpu().numpy().ravel(), gr.cpu().numpy(), gs.cpu().numpy()])
    h = np.concatenate([ha.ravel(), hr, [hs]])
    assert np.linalg.norm(h) > 0
    assert np.linalg.norm(g - h) <= 1e-3 * np.linalg.norm(h)


def test_gradients_match_central_differences(setup):
    torch, cam, n = setup["torch"], setup["cam"], setup["n"]
    a, r = setup["init"]
    ga_t, gr_t = setup["gt"]
    cfg = diff.diff_config(W, H, 2, 4, n, sample_start=3)
    target = diff.forward(setup["dev"], cam, cfg, _t(torch, ga_t), _t(torch, gr_t), 1.0).double()
    A, R = _t(torch, a), _t(torch, r)

    def loss(av, rv, s):
        img = diff.forward(setup["dev"], cam, cfg, av, rv, s).double()
        return float(((img - target) ** 2).sum())

    img = diff.forward(setup["dev"], cam, cfg, A, R, 1.0)
    ga, gr, gs = diff.backward(setup["dev"], cam, cfg, A, R, 1.0, 2.0 * (img.double() - target).float())
    ga, gr, gs = ga.cpu().numpy(), gr.cpu().numpy(), float(gs.cpu().numpy()[0])
    # parameters that the camera sees through at least one path: nonzero gradient
    live_a = np.flatnonzero(np.abs(ga).ravel() > 1e-3)
    live_r = np.flatnonzero(np.abs(gr) > 1e-3)
    rng = np.random.default_rng(5)
    pick_a = rng.choice(live_a, size=min(200, len(live_a)), replace=False)
    pick_r = rng.choice(live_r, size=min(55, len(live_r)), replace=False)
    eps = 1e-3
    checked = bad = 0
    for j in pick_a:
        k, c = divmod(int(j), 3)
        ap, am = A.clone(), A.clone()
        ap[k, c] += eps
        am[k, c] -= eps
        fd = (loss(ap, R, 1.0) - loss(am, R, 1.0)) / (2 * eps)
        g = ga[k, c]
        checked += 1
        bad += abs(fd - g) > 0.02 * max(abs(fd), abs(g))
    for k in pick_r:
        rp, rm = R.clone(), R.clone()
        rp[k] += eps
        rm[k] -= eps
        fd = (loss(A, rp, 1.0) - loss(A, rm, 1.0)) / (2 * eps)
        checked += 1
        bad += abs(fd - gr[k]) > 0.02 * max(abs(fd), abs(gr[k]))
    fd = (loss(A, R, 1.0 + eps) - loss(A, R, 1.0 - eps)) / (2 * eps)
    checked += 1
    bad += abs(fd - gs) > 0.02 * max(abs(fd), abs(gs))
    assert checked == 256
    assert bad == 0, f"{bad} of {checked} parameters differ from central differences by more than 2%"


def test_autograd_binding_and_descent(setup):
    torch, cam, n = setup["torch"], setup["cam"], setup["n"]
    a, r = setup["init"]
    ga_t, gr_t = setup["gt"]
    cfg = diff.diff_config(W, H, 4, 5, n, sample_start=11)
    target = diff.forward(setup["dev"], cam, cfg, _t(torch, ga_t), _t(torch, gr_t), 1.0)
    A = _t(torch, a).requires_grad_(True)
    R = _t(torch, r).requires_grad_(True)
    S = torch.tensor([1.2], device="cuda", requires_grad=True)
    img = diff.render(setup["dev"], cam, cfg, A, R, S)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    ga, gr, gs = diff.backward(setup["dev"], cam, cfg, A.detach(), R.detach(), 1.2, 2.0 * (img.detach() - target))
    assert torch.allclose(A.grad, ga.float(), rtol=1e-6, atol=1e-9)
    assert torch.allclose(R.grad, gr.float(), rtol=1e-6, atol=1e-9)
    assert abs(float(S.grad) - float(gs)) <= 1e-6 * abs(float(gs))
    losses = [float(loss.detach())]
    opt = torch.optim.Adam([A, R, S], lr=0.03)
    for _ in range(15):
        opt.zero_grad()
        l = ((diff.render(setup["dev"], cam, cfg, A, R, S) - target) ** 2).sum()
        l.backward()
        opt.step()
        with torch.no_grad():
            A.clamp_(0.01, 1.0)
            R.clamp_(0.0, 1.5)
        losses.append(float(l.detach()))
    assert losses[-1] < 0.7 * losses[0]
