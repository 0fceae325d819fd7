"""The product's host quadtree (libkinterp.so, ki_partition; no GPU needed)
against the reference partition: same boxes, corners, parents, leaf flags,
level order and per-box dofs (quadtree.cpp:27-285)."""
import numpy as np
import pytest

import helpers as H
import ki_geometry as G
import kinterp
import kioracle as K

CASES = {name: (pr, tol, leaf) for name, pr, tol, leaf in H.golden_cases()}


@pytest.mark.parametrize("name", sorted(CASES))
def test_partition_matches_reference_fixture(name):
    pr, tol, leaf = CASES[name]
    gold = H.load_golden(name)
    p = kinterp.Partition(pr.points, pr.sol_dim, leaf)
    assert H.compare_partition(H.flatten(p), gold) == 0


@pytest.mark.parametrize("make", [G.star_case, G.stokes_holes_case, G.fourier_star_case])
def test_partition_full_size_matches_oracle(make):
    H.ensure_oracle()
    pr = make()
    p = kinterp.Partition(pr.points, pr.sol_dim, pr.max_leaf_dofs)
    o = K.PortSolver(pr, id_tol=0.5)  # partition only matters here
    assert p.levels() == o.levels()
    for l in range(p.levels()):
        assert p.nodes(l) == o.nodes(l)
        for i in range(p.nodes(l)):
            a, b = p.node(l, i), o.node(l, i)
            assert np.array_equal(a["original"], b["original"])
            assert a["corner"] == b["corner"] and a["side"] == b["side"]
            assert a["parent"] == b["parent"] and a["is_leaf"] == b["is_leaf"]


def test_partition_edge_cases():
    # a single point: one leaf; points on the split lines go to the upper/right child
    p = kinterp.Partition(np.array([0.3, 0.7]), 1, 32)
    assert p.levels() == 1 and p.node(0, 0)["is_leaf"]
    pts = np.array([[x, y] for x in np.linspace(0, 1, 9) for y in np.linspace(0, 1, 9)]).ravel()
    q = kinterp.Partition(pts, 1, 4)
    o = K.PortSolver(G.Problem("grid", 0, pts, np.tile([1.0, 0.0], 81), np.ones(81),
                               np.full(81, 0.01), np.zeros((0, 4)), np.zeros(81),
                               np.zeros(2), np.zeros(1), 4, 0.5), id_tol=0.5, max_leaf_dofs=4)
    assert q.levels() == o.levels()
    for l in range(q.levels()):
        for i in range(q.nodes(l)):
            assert np.array_equal(q.node(l, i)["original"], o.node(l, i)["original"])
    with pytest.raises(kinterp.KiError):
        kinterp.Partition(np.zeros(0), 1, 32)
    with pytest.raises(kinterp.KiError):
        kinterp.Partition(np.array([0.0, 0.0]), 3, 32)
