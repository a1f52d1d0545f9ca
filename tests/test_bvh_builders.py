"""The host BVH2 builder through wf_bvh_build (no GPU needed): structure,
depth bound, determinism, argument errors."""
import numpy as np
import pytest

import wfpt
from wfpt import abi, native
from bvh_check import check_tree, sah_cost


def _boxes(n, seed, spread=100.0, size=1.0):
    rng = np.random.default_rng(seed)
    lo = rng.uniform(-spread, spread, (n, 3)).astype(np.float32)
    return np.concatenate([lo, lo + rng.uniform(0.01, size, (n, 3)).astype(np.float32)], axis=1)


@pytest.mark.parametrize("n", [0, 1, 2, 3, 17, 5000])
def test_host_builder_structure(n):
    boxes = _boxes(n, seed=n)
    nodes, ms = native.build_bvh(boxes, abi.BVH_HOST_SAH)
    check_tree(nodes, boxes)
    again, _ = native.build_bvh(boxes, abi.BVH_HOST_SAH)
    assert nodes.tobytes() == again.tobytes()
    if n > 1:
        assert sah_cost(nodes) > 1.0 and ms >= 0.0


def test_identical_boxes_stay_within_the_depth_bound():
    boxes = np.tile(np.array([[0, 0, 0, 1, 1, 1]], np.float32), (20000, 1))
    nodes, _ = native.build_bvh(boxes, abi.BVH_HOST_SAH)
    assert check_tree(nodes, boxes) <= 60


def test_bvh_build_rejects_bad_arguments():
    with pytest.raises(wfpt.WavefrontError, match="unknown BVH builder"):
        native.build_bvh(_boxes(4, 0), 7)
