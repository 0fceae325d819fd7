"""Host partition of a batch of problems (ki_partition_batch): every
problem's tree inside the forest equals the partition that problem gets on
its own (ki_partition, the reference's QuadTree::initialize_tree), with its
dofs shifted by the dofs of the problems before it."""
import numpy as np

import ki_geometry as G
import kinterp


def _by_tree(part, n_trees):
    out = [[] for _ in range(n_trees)]
    for l in range(part.levels()):
        for i in range(part.nodes(l)):
            b = part.node(l, i)
            out[b["tree"]].append(b)
    return out


def test_forest_trees_match_single_partitions():
    probs = G.random_star_cases(count=6, seed=9, nmin=300, nmax=3000)
    bp = kinterp.BatchPartition(probs)
    trees = _by_tree(bp, len(probs))
    off = 0
    for p, pr in enumerate(probs):
        single = kinterp.Partition(pr.points, pr.sol_dim, pr.max_leaf_dofs)
        boxes = [single.node(l, i) for l in range(single.levels()) for i in range(single.nodes(l))]
        assert len(boxes) == len(trees[p])
        for a, b in zip(boxes, trees[p]):
            assert a["level"] == b["level"] and a["is_leaf"] == b["is_leaf"]
            assert np.array_equal(a["original"] + off, b["original"])
            assert np.array_equal(a["active"] + off, b["active"])
            assert abs(a["side"] - b["side"]) == 0.0
        off += pr.n_dofs
        single.close()
    bp.close()


def test_forest_rejects_bad_sizes():
    import ctypes as C
    lib = kinterp.load()
    h = C.c_void_p()
    n = np.array([10, 0], dtype=np.int32)
    pts = np.zeros(20)
    rc = lib.ki_partition_batch(2, n.ctypes.data_as(C.POINTER(C.c_int)),
                                pts.ctypes.data_as(C.POINTER(C.c_double)), 1, 64, C.byref(h))
    assert rc != 0
