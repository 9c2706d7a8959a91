"""The BVH builders: the host binned-SAH builder and the GPU build that uses the
same split rule (cg_bvh_build).  The GPU build must produce the host's nodes
bit for bit and, per leaf, the same primitives (only their order inside a leaf
may differ: the host partition is not stable)."""
import numpy as np
import pytest

from crystalgraphics_b200 import _abi
from crystalgraphics_b200 import backend as B


def _boxes(n, seed, size=0.01, spread=1.0):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 3)).astype(np.float32)
    h = rng.uniform(0.2, 1.0, (n, 3)).astype(np.float32) * size
    return np.concatenate([c - h, c + h], axis=1).astype(np.float32)


def _leaves(nodes):
    """(first, count) of every leaf child, in node order."""
    out = []
    links = nodes[:, 12:14].view(np.int32)
    cnts = nodes[:, 14:16]
    for i in range(nodes.shape[0]):
        for c in range(2):
            l = int(links[i, c])
            if l < 0 and cnts[i, c] > 0:
                v = ~l & 0xFFFFFFFF
                out.append((v >> 3, v & 7))
    return out


def test_host_build_is_a_tree_over_all_primitives():
    boxes = _boxes(3000, 1)
    nodes, order = B.bvh_build(boxes, _abi.CG_BVH_BUILD_HOST)
    assert sorted(order.tolist()) == list(range(3000))
    leaves = _leaves(nodes)
    assert sum(c for _, c in leaves) == 3000
    assert all(1 <= c <= 4 for _, c in leaves)
    # leaf ranges tile the permutation
    spans = sorted(leaves)
    pos = 0
    for f, c in spans:
        assert f == pos
        pos += c
    assert pos == 3000


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed,size", [(20000, 2, 0.01), (70000, 3, 0.003), (5000, 4, 0.2),
                                         (17, 5, 0.1)])
def test_device_build_matches_host_build(n, seed, size):
    boxes = _boxes(n, seed, size)
    hn, ho = B.bvh_build(boxes, _abi.CG_BVH_BUILD_HOST)
    dn, do = B.bvh_build(boxes, _abi.CG_BVH_BUILD_DEVICE)
    assert hn.shape == dn.shape
    assert np.array_equal(hn, dn)
    for first, count in _leaves(hn):
        assert sorted(ho[first:first + count]) == sorted(do[first:first + count])


@pytest.mark.gpu
def test_device_build_of_clustered_and_coincident_boxes():
    """Clusters of identical boxes (centroids that coincide) exercise the
    halve-by-position fallback, which may order primitives differently; the
    tree shape (node count, leaf sizes) still agrees."""
    base = _boxes(4000, 6, 0.01)
    boxes = np.repeat(base, 9, axis=0)  # 9 copies of each box
    hn, ho = B.bvh_build(boxes, _abi.CG_BVH_BUILD_HOST)
    dn, do = B.bvh_build(boxes, _abi.CG_BVH_BUILD_DEVICE)
    assert hn.shape == dn.shape
    assert sorted(c for _, c in _leaves(hn)) == sorted(c for _, c in _leaves(dn))
    assert sorted(do.tolist()) == list(range(boxes.shape[0]))
    # every inner node box is the same (the node's primitive set is the same)
    assert np.array_equal(hn[:, :12], dn[:, :12])
