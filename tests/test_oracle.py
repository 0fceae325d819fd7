"""The oracle (CPU restatement, oracle/ki_oracle.cpp) pinned against the
reference: golden fixtures made by the reference build, the reference test
suite's own acceptance criteria (kern_interp_test.cpp:26-95), and -- when
oracle/_ref is built in this checkout -- the live reference."""
import numpy as np
import pytest

import helpers as H
import ki_geometry as G
import kioracle as K

CASES = {name: (pr, tol, leaf) for name, pr, tol, leaf in H.golden_cases()}
WORKLOADS = ["ellipse_laplace_1024", "star_laplace_2048", "disk_holes_stokes_2048",
             "fourier_star_laplace_1024"]
SHAPES = [n for n in CASES if n not in WORKLOADS]


@pytest.fixture(scope="module", autouse=True)
def _oracle_built():
    H.ensure_oracle()


@pytest.mark.parametrize("name", sorted(CASES))
def test_geometry_matches_fixture(name):
    pr, tol, leaf = CASES[name]
    import make_golden
    assert make_golden.geometry_hash(pr) == str(H.load_golden(name)["geometry_sha256"])


@pytest.mark.parametrize("name", WORKLOADS)
def test_port_reproduces_reference_fixture(name):
    pr, tol, leaf = CASES[name]
    gold = H.load_golden(name)
    s = K.PortSolver(pr, id_tol=tol, max_leaf_dofs=leaf)
    boxes = H.flatten(s)
    assert H.compare_partition(boxes, gold) == 0
    rank_bad, skel_bad, red_bad = H.compare_skeletons(boxes, gold)
    assert (rank_bad, skel_bad, red_bad) == (0, 0, 0)
    assert np.array_equal(s.allskel(), gold["allskel"])
    mu, alpha = s.solve(pr.f)
    assert H.rel(mu, gold["mu"]) < 1e-10
    if len(alpha):
        assert np.abs(alpha - gold["alpha"]).max() < 1e-10 * max(1.0, np.abs(mu).max())
    out = s.eval_targets(pr.targets, mu, alpha)
    assert H.rel(out, gold["targets_out"]) < 1e-10


@pytest.mark.parametrize("name", SHAPES)
def test_port_reference_shapes(name):
    """Symmetric test shapes: exact column-norm ties let LAPACK and the
    restatement pick different (equally valid) skeletons, and a different
    pick can move a later |R_ii| across the rank threshold; the partition is
    compared exactly, ranks to within one in a few boxes, and the solution by
    the reference test's own criterion, ||K mu - f|| / ||f|| <= 10 id_tol
    (kern_interp_test.cpp:79,92)."""
    pr, tol, leaf = CASES[name]
    gold = H.load_golden(name)
    s = K.PortSolver(pr, id_tol=tol, max_leaf_dofs=leaf)
    boxes = H.flatten(s)
    assert H.compare_partition(boxes, gold) == 0
    so = gold["skel_off"]
    diffs = [abs(len(b["skel"]) - (so[q + 1] - so[q])) for q, b in enumerate(boxes)]
    assert max(diffs) <= 1 and sum(d > 0 for d in diffs) <= max(2, len(boxes) // 20)
    mu, alpha = s.solve(pr.f)
    x = np.concatenate([mu, alpha])
    y = np.zeros_like(x)
    import ctypes as C
    s.lib.kiora_apply_dense(C.c_void_p(s.h), x.ctypes.data_as(C.POINTER(C.c_double)),
                            y.ctypes.data_as(C.POINTER(C.c_double)))
    f = np.concatenate([pr.f, np.zeros(len(alpha))])
    assert np.linalg.norm(y - f) / np.linalg.norm(pr.f) <= 10 * tol
    # and the two valid solutions agree to the compression tolerance
    assert H.rel(mu, gold["mu"]) < 1e3 * tol


def test_analytic_ellipse():
    """Interior Dirichlet data from exterior charges, checked at interior
    targets (the reference's analytic-agreement tests, kern_interp_test.cpp:392-488)."""
    pr = G.ellipse_case()
    s = K.PortSolver(pr)
    mu, alpha = s.solve(pr.f)
    u = s.eval_targets(pr.targets, mu, alpha)
    assert H.rel(u, pr.exact) < 1e-11


@pytest.mark.skipif(not K.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("make", [G.star_case, G.stokes_holes_case])
def test_port_matches_live_reference_full_size(make):
    """The restatement against the reference build on the two full-size
    workloads (16,384-dof star; 65,536-dof Stokes disk with 8 holes)."""
    pr = make()
    a = K.RefSolver(pr, threads=4)
    b = K.PortSolver(pr, threads=4)
    d = H.compare_solvers(a, b)
    assert d["partition"] == 0 and d["rank"] == 0 and d["skel"] == 0, d
    ma, aa = a.solve(pr.f)
    mb, ab = b.solve(pr.f)
    assert H.rel(mb, ma) < 1e-10
    if len(aa):
        assert np.abs(ab - aa).max() < 1e-10 * max(1.0, np.abs(ma).max())


SYMMETRIC_SHAPES = [n for n in CASES if n.split("_")[0] in ("circle", "annulus", "donut")]


@pytest.mark.parametrize("name", SYMMETRIC_SHAPES)
def test_symmetric_shape_ties_are_blas_defined(name):
    """On the reference's rotation/mirror-symmetric test shapes columns tie
    exactly in norm, and which tied column dgeqp3 takes first is decided by
    the last bits of the BLAS's norms and reflector products.  The
    restatement runs the reference's own steps (dgeqp3's dlaqp2 pivoting,
    the same rank rule) with plain-loop BLAS; against the fixtures made by
    the reference build (OpenBLAS) it shows the same kind of differences the
    GPU tests allow on these shapes: identical partition, ranks off by at
    most one in a few boxes, skeleton sets that differ where ties were
    broken the other way."""
    pr, tol, leaf = CASES[name]
    gold = H.load_golden(name)
    s = K.PortSolver(pr, id_tol=tol, max_leaf_dofs=leaf)
    boxes = H.flatten(s)
    assert H.compare_partition(boxes, gold) == 0
    so = gold["skel_off"]
    diffs = [abs(len(b["skel"]) - (so[q + 1] - so[q])) for q, b in enumerate(boxes)]
    assert max(diffs) <= 1 and sum(d > 0 for d in diffs) <= max(2, len(boxes) // 20)


def test_planted_error_is_caught():
    """A mistake planted in the oracle's input (a perturbed weight) must be
    visible to the fixture comparison: guards against a vacuous check."""
    name = "ellipse_laplace_1024"
    pr, tol, leaf = CASES[name]
    gold = H.load_golden(name)
    bad = G.Problem(pr.name, pr.pde, pr.points, pr.normals, pr.curvatures,
                    pr.weights * (1 + 1e-6), pr.holes, pr.f, pr.targets, pr.exact,
                    pr.leaf_points, pr.id_tol)
    s = K.PortSolver(bad, id_tol=tol, max_leaf_dofs=leaf)
    mu, _ = s.solve(bad.f)
    assert H.rel(mu, gold["mu"]) > 1e-10


def test_restatement_breaks_some_ties_differently():
    """The evidence behind the bar above: with the same algorithm and plain
    loops in place of OpenBLAS, the restatement's skeleton sets differ from
    the reference build's on some boxes of the symmetric shapes (54 of 2,141
    boxes when written), while matching them exactly on the four asymmetric
    workload fixtures."""
    skel_bad = 0
    for name in SYMMETRIC_SHAPES:
        pr, tol, leaf = CASES[name]
        s = K.PortSolver(pr, id_tol=tol, max_leaf_dofs=leaf)
        skel_bad += H.compare_skeletons(H.flatten(s), H.load_golden(name))[1]
    assert skel_bad > 0
    for name in ("ellipse_laplace_1024", "star_laplace_2048", "disk_holes_stokes_2048",
                 "fourier_star_laplace_1024"):
        pr, tol, leaf = CASES[name]
        s = K.PortSolver(pr, id_tol=tol, max_leaf_dofs=leaf)
        assert H.compare_skeletons(H.flatten(s), H.load_golden(name)) == (0, 0, 0)
