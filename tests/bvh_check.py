"""Structural checks of a binary BVH2 in the builders' output format
(wfpt.native.BVH_NODE_DTYPE: 2n-1 nodes, leaves left == 0xffffffff and
right == box index, the root last), and its SAH cost."""
import numpy as np

INVALID = 0xFFFFFFFF


def check_tree(nodes, boxes, max_depth=60):
    """Asserts the tree is a valid BVH2 over `boxes`; returns its depth."""
    boxes = np.asarray(boxes, np.float32).reshape(-1, 6)
    n = len(boxes)
    assert len(nodes) == max(2 * n - 1, 0)
    if n == 0:
        return 0
    leaf = nodes["left"] == INVALID
    assert leaf.sum() == n
    prims = nodes["right"][leaf].astype(np.int64)
    assert np.array_equal(np.sort(prims), np.arange(n)), "every box in exactly one leaf"
    assert np.array_equal(nodes["lo"][leaf], boxes[prims, :3]) and np.array_equal(nodes["hi"][leaf], boxes[prims, 3:])
    internal = np.flatnonzero(~leaf)
    children = np.concatenate([nodes["left"][internal], nodes["right"][internal]]).astype(np.int64)
    assert children.size == 0 or children.max() < len(nodes)
    refs = np.bincount(children, minlength=len(nodes))
    root = len(nodes) - 1
    assert refs[root] == 0 and np.all(np.delete(refs, root) == 1), "a tree with the root last"
    for side in ("left", "right"):
        c = nodes[side][internal].astype(np.int64)
        assert np.all(nodes["lo"][internal] <= nodes["lo"][c]) and np.all(nodes["hi"][internal] >= nodes["hi"][c])
    depth, level = 0, np.array([root])
    while True:
        level = level[nodes["left"][level] != INVALID]
        if level.size == 0:
            break
        level = np.concatenate([nodes["left"][level], nodes["right"][level]]).astype(np.int64)
        depth += 1
        assert depth <= max_depth, f"deeper than {max_depth}"
    return depth


def sah_cost(nodes):
    """Sum over all nodes of surface area / root surface area (unit costs)."""
    d = nodes["hi"].astype(np.float64) - nodes["lo"].astype(np.float64)
    area = d[:, 0] * d[:, 1] + d[:, 1] * d[:, 2] + d[:, 2] * d[:, 0]
    return float(area.sum() / max(area[-1], 1e-30))
