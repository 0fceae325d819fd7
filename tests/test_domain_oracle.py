"""Domain tests and grids of boundary_integral_solve (linear_solve.cpp:142-193):
the CPU restatement (oracle/domain.py) against the reference's own
CubicBoundary / Circle / Annulus / Donut::is_in_domain and
get_domain_points, compiled from its sources (oracle/_ref/libkiref.so), and
the library's ki_domain_points (host code, no GPU) against both."""
import numpy as np
import pytest

import domain as D
import ki_geometry as G
import kinterp
import kioracle

needs_ref = pytest.mark.skipif(not kioracle.ref_available(),
                               reason="reference library not built (make -C oracle ref)")


def _grid(n, lo, hi):
    return D.domain_points(n, lo, hi, lo, hi)


def _edge_targets(points, rng):
    """Points on nodes, just inside / outside the 1e-2 node distance, and at
    node heights (the crossing test's boundary cases)."""
    p = points.reshape(-1, 2)
    k = rng.choice(p.shape[0], 64, replace=False)
    ang = rng.uniform(0, 2 * np.pi, 64)
    out = [p[k]]
    for r in (0.0099999, 0.0100001, 0.02):
        out.append(p[k] + r * np.stack([np.cos(ang), np.sin(ang)], 1))
    same_y = p[k].copy()
    same_y[:, 0] -= rng.uniform(0.05, 0.3, 64)
    out.append(same_y)
    return np.concatenate(out).reshape(-1)


CASES = {
    "star": lambda: G.star_case(n=2048),
    "stokes_holes": lambda: G.stokes_holes_case(n_total=4096, n_holes=8),
    "ellipse": lambda: G.ellipse_case(n=1024),
}


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
def test_nodes_test_matches_reference(name):
    pr = CASES[name]()
    rng = np.random.default_rng(11)
    tg = np.concatenate([_grid(60, -1.45, 1.45), _edge_targets(pr.points, rng)])
    got = D.in_domain_nodes(pr.points, pr.holes, tg)
    ref = D.ref_in_domain("nodes", pr.points, pr.holes, tg)
    assert np.array_equal(got, ref)
    assert 0 < got.sum() < got.size


@needs_ref
@pytest.mark.parametrize("kind", ["circle", "annulus", "donut"])
def test_reference_shape_tests_match_reference(kind):
    pts, nrm, kap, w, holes = G.reference_shape(kind, 1000)
    rng = np.random.default_rng(12)
    tg = np.concatenate([_grid(64, -0.6, 1.6), _edge_targets(pts, rng)])
    cx, cy, R = (0.5, 0.5, 0.25) if kind == "circle" else (0.5, 0.5, 1.0)
    got = D.in_domain_disk(cx, cy, R, holes, tg)
    assert np.array_equal(got, D.ref_in_domain(kind, pts, holes, tg))
    # the node-curve test on the same shapes
    got_n = D.in_domain_nodes(pts, holes, tg)
    assert np.array_equal(got_n, D.ref_in_domain("nodes", pts, holes, tg))


@needs_ref
@pytest.mark.parametrize("args", [(20, 0.0, 1.0, 0.0, 1.0), (37, -1.2, 1.3, -0.7, 2.1),
                                  (2, -1.0, 1.0, -1.0, 1.0)])
def test_domain_points_match_reference(args):
    ref = D.ref_domain_points(*args)
    assert np.array_equal(D.domain_points(*args), ref)
    assert np.array_equal(kinterp.domain_points(*args), ref)
