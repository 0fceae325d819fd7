"""GPU boundary update and tree copy (ki_update / ki_copy): QuadTree::perturb
+ skeletonize and QuadTree::copy_into + skeletonize (quadtree.cpp:359-641).

Bars: after a sequence of boundary frames, the partition, the compressed
flags, the ranks and the skeleton sets identical to the reference's own
update (the committed fixture, and the reference library when it is built),
the solution within 1e-10 relative of the reference's; an updated
factorization within 20 id_tol of a fresh one on the same boundary (the
reference's Ex3UpdateLosesNoAcc bar, kern_interp_test.cpp:491-530); a copy
solving to within 1e-15 of its source (TreeCopyGivesSameAnswer,
kern_interp_test.cpp:533-567) and independent of it afterwards."""
import os
import sys

import numpy as np
import pytest

import helpers as H
import ki_geometry as G
import kinterp
import kioracle as K

pytestmark = pytest.mark.gpu

sys.path.insert(0, H.GOLDEN)
import make_golden  # noqa: E402

needs_ref = pytest.mark.skipif(not K.ref_available(),
                               reason="reference library not built (make -C oracle ref)")

FRAMES = {
    "add": [dict(center=2.0, amp=0.05, width=0.12, extra=60),
            dict(center=4.0, amp=0.1, width=0.05, extra=200)],
    "delete": [dict(center=3.5, amp=0.02, width=0.2, extra=-150),
               dict(center=1.0, amp=0.0, width=0.15, extra=-120)],
    "back_and_forth": [dict(center=2.0, amp=0.05, width=0.12, extra=60),
                       dict(center=2.0, amp=0.0, width=0.12, extra=0),
                       dict(center=5.0, amp=-0.04, width=0.1, extra=-40)],
}


def test_update_matches_reference_fixture():
    for name, base, frames, tol, leaf in make_golden.update_cases():
        gold = H.load_golden(name)
        s = kinterp.Solver(base, id_tol=tol, max_leaf_dofs=leaf)
        kept = [s.update(fr) for fr in frames]
        assert min(kept) > 0
        pr = frames[-1]
        boxes = H.flatten(s)
        assert H.compare_partition(boxes, gold) == 0
        assert H.compare_skeletons(boxes, gold) == (0, 0, 0)
        assert np.array_equal(np.sort(s.allskel()), np.sort(gold["allskel"]))
        mu, alpha = s.solve(pr.f)
        assert H.rel(mu, gold["mu"]) < 1e-10
        assert H.rel(s.eval_targets(pr.targets, mu, alpha), gold["targets_out"]) < 1e-10


@needs_ref
@pytest.mark.parametrize("name", sorted(FRAMES))
def test_update_matches_reference(name):
    base = G.star_case(n=2048, n_targets=16)
    ref = K.RefSolver(base, id_tol=1e-10, max_leaf_dofs=64)
    s = kinterp.Solver(base, id_tol=1e-10, max_leaf_dofs=64)
    for fr in FRAMES[name]:
        new = G.bumped_star_case(n=2048, n_targets=16, **fr)
        ref.update(new)
        s.update(new)
        d = H.compare_solvers(s, ref)
        assert d["partition"] == 0 and d["rank"] == 0 and d["skel"] == 0, d
        assert H.rel(s.solve(new.f)[0], ref.solve(new.f)[0]) < 1e-10


def _moved_hole(pr, h, dx, dy):
    """pr with hole h (its nodes and centre) shifted by (dx, dy) and the
    Stokeslet data recomputed."""
    pts, holes = pr.points.copy(), pr.holes.copy()
    counts = holes[:, 3].astype(int)
    start = pr.n_points - counts.sum() + counts[:h].sum()
    sl = slice(2 * start, 2 * (start + counts[h]))
    pts[sl][0::2] += dx
    pts[sl][1::2] += dy
    holes[h, 0] += dx
    holes[h, 1] += dy
    f = G.stokeslet_velocity(pts, pr.extra["sources"], pr.extra["forces"])
    return G.Problem(pr.name + "_moved", pr.pde, pts, pr.normals, pr.curvatures, pr.weights,
                     holes, f, pr.targets, pr.exact, pr.leaf_points, pr.id_tol, pr.extra)


def _frames_stokes():
    pr = G.stokes_holes_case(n_total=4096, n_targets=16)
    out, cur = [], pr
    for k in range(3):
        cur = _moved_hole(cur, k, 0.004 * (k + 1), -0.003)
        out.append(cur)
    return pr, out


@pytest.mark.parametrize("kind", ["laplace", "stokes_holes"])
def test_update_loses_no_accuracy(kind):
    tol = 1e-6
    if kind == "laplace":
        base = G.star_case(n=4096, n_targets=16)
        frames = [G.bumped_star_case(n=4096, n_targets=16, center=0.7 + 0.6 * k, amp=0.04,
                                     width=0.1, extra=(-1) ** k * 30) for k in range(4)]
    else:
        base, frames = _frames_stokes()
    s = kinterp.Solver(base, id_tol=tol)
    for fr in frames:
        kept = s.update(fr)
        assert kept > 0
        fresh = kinterp.Solver(fr, id_tol=tol)
        mu_u, al_u = s.solve(fr.f)
        mu_f, al_f = fresh.solve(fr.f)
        u = np.concatenate([mu_u, al_u])
        f = np.concatenate([mu_f, al_f])
        assert np.linalg.norm(u - f) / np.linalg.norm(f) <= 20 * tol
        fresh.close()


def test_update_keeps_most_boxes_for_a_local_change():
    base = G.star_case(n=16384, n_targets=16)
    s = kinterp.Solver(base, id_tol=1e-10)
    n_comp = sum(b["compressed"] for b in H.flatten(s))
    kept = s.update(G.bumped_star_case(n=16384, n_targets=16, center=2.0, amp=0.02,
                                       width=0.03, extra=10))
    assert kept > 0.7 * n_comp


def test_copy_gives_same_answer_and_is_independent():
    pr = G.stokes_holes_case(n_total=4096, n_targets=16)
    s = kinterp.Solver(pr, id_tol=1e-6)
    mu, alpha = s.solve(pr.f)
    c = s.copy()
    mu_c, alpha_c = c.solve(pr.f)
    assert np.linalg.norm(mu_c - mu) <= 1e-15
    assert np.linalg.norm(alpha_c - alpha) <= 1e-15
    # updating the copy leaves the source as it was
    moved = _moved_hole(pr, 0, 0.005, 0.0)
    c.update(moved)
    mu2, alpha2 = s.solve(pr.f)
    assert np.array_equal(mu2, mu) and np.array_equal(alpha2, alpha)
    c.close()
    mu3, _ = s.solve(pr.f)
    assert np.array_equal(mu3, mu)


def test_copy_of_an_updated_handle():
    base = G.star_case(n=2048, n_targets=16)
    s = kinterp.Solver(base, id_tol=1e-10)
    new = G.bumped_star_case(n=2048, n_targets=16, extra=60)
    s.update(new)
    c = s.copy()
    assert H.compare_solvers(s, c)["rank"] == 0
    assert np.linalg.norm(c.solve(new.f)[0] - s.solve(new.f)[0]) <= 1e-15


def test_many_updates_keep_pinned_staging_bounded():
    """A shape-optimisation loop calls ki_update many times: the pinned
    staging a handle uses must not grow with the number of updates (each
    update stages only its own refactorization)."""
    base = G.star_case(n=8192, n_targets=16)
    s = kinterp.Solver(base, id_tol=1e-8)
    held = []
    for k in range(16):
        fr = G.bumped_star_case(n=8192, n_targets=16, center=0.5 + 0.3 * k, amp=0.03,
                                width=0.1, extra=(-1) ** k * 20)
        s.update(fr)
        s.solve_refined(fr.f, rel_tol=1e-12)
        held.append(s.stats()["staging_bytes"])
    assert max(held) <= 1.5 * min(held), held
    s.close()
