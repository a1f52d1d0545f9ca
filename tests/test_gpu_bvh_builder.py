"""GPU BVH2 builder (PLOC, wf_bvh_gpu.cu) against the host binned-SAH builder.

* Structure: every box in exactly one leaf, children inside parents, the
  root last, depth within the 60-level stack bound; the same tree on every
  build (deterministic sort, tie-breaks and node numbering).
* Quality: SAH cost within 10 % of the host builder's on random and
  clustered boxes.
* Scenes built with either builder give the same closest hits for a ray
  batch and the same rendered sums bit for bit: closest hits are a minimum
  over exact per-triangle tests, independent of the tree except at exact-t
  ties, which these scenes do not produce.
"""
import numpy as np
import pytest

import wfpt
from wfpt import abi, native, scenes
from bvh_check import check_tree, sah_cost

pytestmark = pytest.mark.gpu


def _random(n, seed):
    rng = np.random.default_rng(seed)
    lo = rng.uniform(-100, 100, (n, 3)).astype(np.float32)
    return np.concatenate([lo, lo + rng.uniform(0.01, 1.0, (n, 3)).astype(np.float32)], axis=1)


def _clustered(n, seed):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-100, 100, (64, 3))
    lo = (centres[rng.integers(0, 64, n)] + rng.normal(0, 2.0, (n, 3))).astype(np.float32)
    return np.concatenate([lo, lo + rng.uniform(0.01, 0.5, (n, 3)).astype(np.float32)], axis=1)


@pytest.mark.parametrize("n", [1, 2, 3, 33, 4097, 100_000])
def test_gpu_builder_structure_and_determinism(cuda, n):
    boxes = _random(n, seed=n)
    nodes, _ = native.build_bvh(boxes, abi.BVH_GPU_PLOC)
    check_tree(nodes, boxes)
    again, _ = native.build_bvh(boxes, abi.BVH_GPU_PLOC)
    assert nodes.tobytes() == again.tobytes()


@pytest.mark.parametrize("make", [_random, _clustered])
def test_gpu_builder_sah_close_to_host(cuda, make):
    boxes = make(200_000, seed=3)
    gpu, _ = native.build_bvh(boxes, abi.BVH_GPU_PLOC)
    host, _ = native.build_bvh(boxes, abi.BVH_HOST_SAH)
    check_tree(gpu, boxes)
    assert sah_cost(gpu) <= 1.10 * sah_cost(host), (sah_cost(gpu), sah_cost(host))


def test_gpu_builder_identical_and_flat_boxes(cuda):
    same = np.tile(np.array([[0, 0, 0, 1, 1, 1]], np.float32), (50_000, 1))
    nodes, _ = native.build_bvh(same, abi.BVH_GPU_PLOC)
    assert check_tree(nodes, same) <= 17  # pairs halve every round: a balanced tree
    flat = _random(20_000, seed=9)
    flat[:, 1] = 0.0
    flat[:, 4] = 0.0  # zero-height boxes: zero-area merges everywhere
    nodes, _ = native.build_bvh(flat, abi.BVH_GPU_PLOC)
    check_tree(nodes, flat)


@pytest.mark.parametrize("which", ["large_mesh_small", "sphere_field"])
def test_scene_hits_and_images_independent_of_builder(cuda, which):
    if which == "large_mesh_small":
        scene, cam = scenes.large_mesh(96, 54, terrain_quads=192, instance_count=30, instance_frequency=40,
                                       glass_spheres=4, env_size=(256, 128))
        w, h, depth = 96, 54, 8
    else:
        scene, cam = scenes.sphere_field(64, 36, frequency=40, seed=3)
        w, h, depth = 64, 36, 8
    results = {}
    for builder in (abi.BVH_HOST_SAH, abi.BVH_GPU_PLOC):
        scene.bvh_builder = builder
        dev = wfpt.DeviceScene(scene)
        info = dev.info()
        if builder == abi.BVH_GPU_PLOC:
            assert info.gpu_bvh_builds >= 1
        else:
            assert info.gpu_bvh_builds == 0
        rng = np.random.default_rng(17)
        rays = np.zeros(65536, abi.RAY_DTYPE)
        rays["origin"] = np.asarray(cam["position"], np.float32) + rng.normal(0, 0.05, (65536, 3)).astype(np.float32)
        d = rng.normal(0, 1, (65536, 3)).astype(np.float32)
        rays["direction"] = d / np.linalg.norm(d, axis=1, keepdims=True)
        hits = dev.trace_closest(rays)
        r = wfpt.Renderer(dev, cam, wfpt.render_config(w, h, max_depth=depth))
        image = r.render_task((0, 0, w, h), 5, 2)
        r.close()
        dev.close()
        results[builder] = (hits, image)
    (h0, i0), (h1, i1) = results[abi.BVH_HOST_SAH], results[abi.BVH_GPU_PLOC]
    for field in ("t", "primitive", "instance", "kind"):
        assert np.array_equal(h0[field], h1[field]), field
    assert np.array_equal(i0.view(np.uint32), i1.view(np.uint32))
