"""Boundary update on the CPU: the partition half of QuadTree::perturb
(quadtree.cpp:359-560) in the library (ki_partition_update, host code)
against the reference's own perturb, compiled from its sources
(oracle/_ref/libkiref.so), over frame sequences that move, add and delete
nodes (leaves split by node_subdivide, subtrees merged by consolidate_node).
Bar: every box identical (corners, side, parent, leaf flag, dof list)."""
import numpy as np
import pytest

import helpers as H
import ki_geometry as G
import kinterp
import kioracle as K

needs_ref = pytest.mark.skipif(not K.ref_available(),
                               reason="reference library not built (make -C oracle ref)")

FRAMES = {
    "move": [dict(center=2.0, amp=0.05, width=0.12, extra=0)],
    "add": [dict(center=2.0, amp=0.05, width=0.12, extra=60),
            dict(center=4.0, amp=0.1, width=0.05, extra=200)],
    "delete": [dict(center=3.5, amp=0.02, width=0.2, extra=-150),
               dict(center=1.0, amp=0.0, width=0.15, extra=-120)],
    "back_and_forth": [dict(center=2.0, amp=0.05, width=0.12, extra=60),
                       dict(center=2.0, amp=0.0, width=0.12, extra=0),
                       dict(center=5.0, amp=-0.04, width=0.1, extra=-40)],
}


def _same(a, b):
    return (np.array_equal(a["original"], b["original"]) and a["corner"] == b["corner"]
            and a["side"] == b["side"] and a["parent"] == b["parent"]
            and a["is_leaf"] == b["is_leaf"])


@needs_ref
@pytest.mark.parametrize("leaf", [32, 64])
@pytest.mark.parametrize("name", sorted(FRAMES))
def test_partition_update_matches_reference(name, leaf):
    n = 2048
    base = G.star_case(n=n, n_targets=16)
    ref = K.RefSolver(base, id_tol=1e-6, max_leaf_dofs=leaf)
    part = kinterp.Partition(base.points, 1, leaf)
    for fr in FRAMES[name]:
        new = G.bumped_star_case(n=n, n_targets=16, **fr)
        ref.update(new)
        part.update(new.points)
        assert ref.levels() == part.levels()
        br, bp = H.flatten(ref), H.flatten(part)
        assert len(br) == len(bp)
        assert sum(not _same(x, y) for x, y in zip(br, bp)) == 0


@needs_ref
def test_partition_update_stokes_dofs():
    """Two dofs per point: the renumbering keeps each point's pair."""
    base = G.star_case(n=1024, n_targets=16)
    ref_pr = G.Problem("s", G.STOKES, base.points, base.normals, base.curvatures, base.weights,
                       np.zeros((0, 4)), np.zeros(2048), base.targets, np.zeros(0), 32, 1e-6)
    new = G.bumped_star_case(n=1024, extra=50, n_targets=16)
    new_pr = G.Problem("s2", G.STOKES, new.points, new.normals, new.curvatures, new.weights,
                       np.zeros((0, 4)), np.zeros(2 * new.n_points), base.targets, np.zeros(0),
                       32, 1e-6)
    ref = K.RefSolver(ref_pr, id_tol=1e-6, max_leaf_dofs=64)
    ref.update(new_pr)
    part = kinterp.Partition(base.points, 2, 64)
    part.update(new.points)
    br, bp = H.flatten(ref), H.flatten(part)
    assert len(br) == len(bp)
    assert sum(not _same(x, y) for x, y in zip(br, bp)) == 0


def test_partition_update_rejects_bad_handles():
    base = G.star_case(n=512, n_targets=16)
    part = kinterp.Partition(base.points, 1, 32)
    with pytest.raises(kinterp.KiError):
        part.update(np.zeros(0))
