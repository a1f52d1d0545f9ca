"""Failure paths of the render loop, made to happen without faulting the GPU.

The reference exits the process on any CUDA error or failed check
(render_driver.cu:18-27, scene.cu:21-26).  This library returns a status
instead and stays usable, which these tests check for each failure it can
meet:

* a device-side wait that runs out: the persistent kernel's grid barrier and
  the streaming schedule's device loop, each given a tiny bound through
  wf_renderer_set_watchdog, so the wait gives up on its own (no spin is made
  endless and no kernel is broken on purpose);
* a queue that overflows: a shadow-ray queue smaller than one bounce needs;
* a device allocation that fails: injected on the host (wf_test_fail_allocation)
  at every allocation of scene and renderer creation in turn.

After each failure the same renderer (or a new one) must render the oracle's
framebuffer bit for bit."""
import ctypes

import numpy as np
import pytest

import oracle
import wfpt
from wfpt import abi, scenes

pytestmark = pytest.mark.gpu

W = H = 64
SPP = 2


def cornell():
    return scenes.cornell_box(W, H)


def expected_image(scene, cam, cfg, start):
    if not oracle.available(det=True):
        pytest.skip("oracle/_ref/libwfref_det.so not built")
    ref = oracle.RefScene(scene, det=True)
    want, _, _ = ref.render(cam, cfg, sample_start=start, sample_count=SPP)
    ref.close()
    return want


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


@pytest.mark.parametrize("mode", [abi.MODE_PERSISTENT, abi.MODE_STREAM])
def test_wait_that_runs_out_reports_timeout_and_recovers(cuda, mode):
    scene, cam = cornell()
    cfg = wfpt.render_config(W, H, max_depth=8, rr_start_depth=3, mode=mode)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    if mode == abi.MODE_PERSISTENT:
        r.set_watchdog(barrier_cycles=1)      # the first barrier wait gives up at once
    else:
        r.set_watchdog(loop_iterations=1)     # one pass of the device loop, paths still live
    r.render(0, 0, W, H, 10, SPP, True)
    with pytest.raises(wfpt.WavefrontError) as err:
        r.synchronize()
    assert err.value.status == abi.WF_ERR_TIMEOUT
    r.synchronize()                           # reported once, then cleared
    r.set_watchdog(0, 0)
    got = r.render_task((0, 0, W, H), 10, SPP)
    r.close()
    dev.close()
    assert same(got, expected_image(scene, cam, cfg, 10))


def test_shadow_queue_overflow_reports_capacity(cuda):
    scene, cam = cornell()
    small = wfpt.render_config(W, H, max_depth=8, rr_start_depth=3, shadow_queue_capacity=64)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, small)
    r.render(0, 0, W, H, 10, SPP, True)
    with pytest.raises(wfpt.WavefrontError) as err:
        r.synchronize()
    assert err.value.status == abi.WF_ERR_CAPACITY
    r.synchronize()
    # writes stayed inside the queue: the framebuffer is finite and the
    # renderer keeps working (each render reports the overflow again)
    r.render(0, 0, W, H, 10, SPP, True)
    with pytest.raises(wfpt.WavefrontError):
        r.download()
    r.close()
    cfg = wfpt.render_config(W, H, max_depth=8, rr_start_depth=3)
    r = wfpt.Renderer(dev, cam, cfg)
    got = r.render_task((0, 0, W, H), 10, SPP)
    r.close()
    dev.close()
    assert same(got, expected_image(scene, cam, cfg, 10))


def free_bytes(torch):
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_injected_allocation_failures_free_everything(cuda):
    """Every allocation of scene creation and of a graph renderer with its
    twin wavefront and a photon map fails once in turn: each failed call
    returns WF_ERR_OOM and frees what it had allocated."""
    torch = cuda
    lib = wfpt.library()
    scene, cam = scenes.large_mesh(160, 90, terrain_quads=32, instance_count=4, instance_frequency=6,
                                   glass_spheres=2, env_size=(64, 32))
    cfg = wfpt.render_config(512, 512, max_depth=6, caustics=1, photon_count=20000,
                             photon_grid_min=(0, 0, 0), photon_grid_max=(0, 0, 0))
    d, keep = scene.desc()
    before = free_bytes(torch)
    scene_failures = renderer_failures = 0
    try:
        for k in range(10000):
            lib.wf_test_fail_allocation(k)
            handle = ctypes.c_void_p()
            status = lib.wf_scene_create(ctypes.byref(d), ctypes.byref(handle))
            lib.wf_test_fail_allocation(-1)
            if status == abi.WF_OK:
                lib.wf_scene_destroy(handle)
                break
            assert status == abi.WF_ERR_OOM, lib.wf_last_error()
            assert not handle.value
            scene_failures += 1
        dev = wfpt.DeviceScene(scene)
        c = wfpt.camera_struct(cam)
        for k in range(10000):
            lib.wf_test_fail_allocation(k)
            handle = ctypes.c_void_p()
            status = lib.wf_renderer_create(dev.handle, ctypes.byref(c), ctypes.byref(cfg), None,
                                            ctypes.byref(handle))
            lib.wf_test_fail_allocation(-1)
            if status == abi.WF_OK:
                lib.wf_renderer_destroy(handle)
                break
            assert status == abi.WF_ERR_OOM, lib.wf_last_error()
            renderer_failures += 1
        dev.close()
    finally:
        lib.wf_test_fail_allocation(-1)
    del keep
    after = free_bytes(torch)
    assert scene_failures >= 8 and renderer_failures >= 20, (scene_failures, renderer_failures)
    # a 512x512 renderer holds ~100 MB; leaking from dozens of failed
    # creations would show far above this tolerance
    assert before - after < 16 << 20, (before - after) / 2**20
    # and a renderer made after all that renders correctly
    scene, cam = cornell()
    cfg = wfpt.render_config(W, H, max_depth=8, rr_start_depth=3)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    got = r.render_task((0, 0, W, H), 3, SPP)
    r.close()
    dev.close()
    assert same(got, expected_image(scene, cam, cfg, 3))
