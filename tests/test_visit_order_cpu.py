"""The tie rule of the batched tracer, restated on the CPU.

The GPU tracer visits BVH children in its own order and settles exactly
equal hit distances with `ref_before` (tracer.cuh): of two accepted leaves,
the one the reference meets first is the one on the side its lowest common
ancestor descends into first, i.e. the child with the smaller entry span.x
(the left child only when its entry is strictly smaller, Arbor.cu:224-225).
This test walks the reference's depth-first visiting order over the accepted
boxes of the oracle's BVH for a set of rays (float32 slab tests with the
reference's operation order, no pruning) and checks that the lowest-common-
ancestor rule reproduces that order for every pair of visited leaves.
"""
import numpy as np
import pytest

CAPACITY = 32768
NODE_COUNT = 65536


def spans(nodes, ro, inv):
    """span.x, span.y and acceptance (count > 0, span.y >= max(1e-4, span.x))
    of every node for one ray, in float32 as the reference computes them."""
    n = nodes.reshape(NODE_COUNT, 8)
    lo, hi = n[:, 0:3], n[:, 4:7]
    a = (lo - ro) * inv
    b = (hi - ro) * inv
    mn, mx = np.minimum(a, b), np.maximum(a, b)
    sx = np.maximum(mn[:, 0], np.maximum(mn[:, 1], mn[:, 2]))
    sy = np.minimum(mx[:, 0], np.minimum(mx[:, 1], mx[:, 2]))
    ok = (n[:, 3] > 0) & (sy >= np.maximum(np.float32(1e-4), sx))
    return sx, sy, ok


def reference_leaf_order(sx, ok):
    """Accepted leaves in the reference's depth-first visiting order."""
    order, stack = [], [1] if ok[1] else []
    while stack:
        node = stack.pop()
        if node >= CAPACITY:
            order.append(node - CAPACITY)
            continue
        l, r = 2 * node, 2 * node + 1
        if ok[l] and ok[r]:
            first, second = (l, r) if sx[l] < sx[r] else (r, l)
            stack.append(second)
            stack.append(first)
        elif ok[l]:
            stack.append(l)
        elif ok[r]:
            stack.append(r)
    return order


def ref_before(sx, a, b):
    """tracer.cuh's rule: leaf slot a before leaf slot b."""
    na, nb = a + CAPACITY, b + CAPACITY
    while (na >> 1) != (nb >> 1):
        na >>= 1
        nb >>= 1
    left = na & ~1
    return (na == left) == bool(sx[left] < sx[left + 1])


def inv_safe(d):
    return np.where(np.abs(d) < np.float32(1e-8), np.where(d < 0, np.float32(-1e8), np.float32(1e8)), np.float32(1) / d).astype(np.float32)


@pytest.mark.parametrize("seed", [1, 7])
def test_lowest_common_ancestor_rule_reproduces_the_visiting_order(scenes, seed):
    nodes = scenes(seed)["Nodes"]
    rng = np.random.default_rng(seed)
    checked = 0
    for _ in range(24):
        # rays from around the tree toward its crown, and from inside it (as
        # shadow rays start)
        if rng.random() < 0.5:
            ang = rng.random() * 2 * np.pi
            ro = np.array([6 * np.cos(ang), 1.72, 6 * np.sin(ang)], np.float32)
        else:
            ro = np.array([rng.uniform(-2, 2), rng.uniform(3, 8), rng.uniform(-2, 2)], np.float32)
        target = np.array([rng.uniform(-1.5, 1.5), rng.uniform(2, 9), rng.uniform(-1.5, 1.5)], np.float32)
        rd = target - ro
        rd = (rd / np.float32(np.sqrt(np.float32(rd @ rd)))).astype(np.float32)
        sx, sy, ok = spans(nodes, ro, inv_safe(rd))
        order = reference_leaf_order(sx, ok)
        if len(order) < 2:
            continue
        pos = {leaf: i for i, leaf in enumerate(order)}
        pairs = rng.integers(0, len(order), size=(min(400, len(order) * 4), 2))
        for i, j in pairs:
            if i == j:
                continue
            a, b = order[i], order[j]
            assert ref_before(sx, a, b) == (pos[a] < pos[b]), (seed, a, b)
            checked += 1
    assert checked > 1000
