"""The block-per-region overlap kernel's stack bound, checked on the host.

overlap_heavy_kernel (spatial_query_b200/csrc/traverse.cuh) walks one region
with 128 threads over one shared stack: each step takes the top min(sp, 128)
entries (thread t takes entry sp - take + t), and pushes, in thread order,
each taken interior node's overlapping children (child_a, then child_b),
the children of the tree::Node arrays (accel/tree.rs:21-49). The kernel's
stack is sized 256 x (depth + 1) entries and states that it never holds
more than 128 x (depth + 2); a push past its size is refused and the call
returns SQ_ERR_CAPACITY. This test replays exactly that step rule on host
trees (the library's own tree::build) for regions that cover the whole
scene -- every node visited, the worst case -- and for random regions, and
checks the largest stack against the stated bound."""
import numpy as np
import pytest

import spatial_query_b200 as sq
from spatial_query_b200 import scenes

THREADS = 128


def tree_depth(t: sq.HostBvh) -> int:
    """Nodes on the longest root-to-leaf path (the upload's depth)."""
    n = t.node_count
    depth = np.ones(n, np.int64)
    for i in range(n - 1, -1, -1):
        if t.prim_count[i] == 0:
            depth[i] = 1 + max(depth[t.child_a[i]], depth[t.child_b[i]])
    return int(depth[0])


def max_stack(t: sq.HostBvh, lo: np.ndarray, hi: np.ndarray) -> int:
    d = t.dim
    b = t.bounds.reshape(-1, 2 * d)

    def overlaps(nodes):
        return np.all(b[nodes, :d] <= hi, axis=1) & np.all(lo <= b[nodes, d:], axis=1)

    stack = np.array([0], np.int64) if overlaps(np.array([0]))[0] else np.zeros(0, np.int64)
    most = stack.size
    while stack.size:
        take = min(stack.size, THREADS)
        taken, stack = stack[stack.size - take:], stack[: stack.size - take]
        inner = taken[t.prim_count[taken] == 0]
        if inner.size:
            kids = np.stack([t.child_a[inner], t.child_b[inner]], axis=1).astype(np.int64).reshape(-1)
            stack = np.concatenate([stack, kids[overlaps(kids)]])
        most = max(most, stack.size)
    return most


def scenes_under_test():
    s = scenes.boxes_scene(seed=40, n_boxes=120_000, n_rays=1, dim=3)
    yield "boxes3d", sq.HostBvh.build(sq.Geometry("boxes", 3, s["prims"]))
    s = scenes.boxes_scene(seed=41, n_boxes=60_000, n_rays=1, dim=6)
    yield "boxes6d", sq.HostBvh.build(sq.Geometry("boxes", 6, s["prims"]))
    s = scenes.terrain_scene(seed=42, nx=256, ny=128, n_coherent=1, n_incoherent=1)
    yield "terrain", sq.HostBvh.build(sq.Geometry("tris", 3, s["prims"]))


@pytest.mark.parametrize("name,tree", list(scenes_under_test()))
def test_block_walk_stack_stays_within_bound(name, tree):
    d = tree.dim
    depth = tree_depth(tree)
    bound = THREADS * (depth + 2)
    size = 256 * (depth + 1)
    root = tree.bounds.reshape(-1, 2 * d)[0]
    # the whole scene: every node is visited
    most = max_stack(tree, root[:d] - 1.0, root[d:] + 1.0)
    assert most <= bound <= size, f"{name}: whole-scene walk held {most} entries, bound {bound}, size {size}"
    assert most > THREADS, f"{name}: the whole-scene walk should fill more than one step"
    rng = np.random.default_rng(7)
    ext = root[d:] - root[:d]
    for _ in range(12):
        c = root[:d] + rng.uniform(0.0, 1.0, d) * ext
        h = rng.uniform(0.05, 0.5, d) * ext
        most = max_stack(tree, (c - h).astype(np.float32), (c + h).astype(np.float32))
        assert most <= bound, f"{name}: region walk held {most} entries, bound {bound}"
