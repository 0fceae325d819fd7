"""The dense FP64 gradient oracle (oracle/adjoint_dense.py), pinned on the
CPU: its matrix equals the oracle restatement's kernel entries
(Kernel::operator(), kernel.cpp:99-111), and its gradient equals central
finite differences of the same dense objective."""
import numpy as np

import adjoint_dense as AD
import helpers as H
import ki_geometry as G
import kioracle as K


def _case(n=256, seed=5):
    pr = G.fourier_star_case(n=n, seed=seed, n_targets=16)
    return pr, pr.extra["coef"], pr.extra["u_star"]


def test_geometry_matches_problem_builder():
    pr, coef, _ = _case()
    x, y, nx, ny, k, w = AD.star_geometry(coef, pr.n_points)
    assert np.allclose(np.stack([x, y], 1).reshape(-1), pr.points, rtol=0, atol=1e-14)
    assert np.allclose(np.stack([nx, ny], 1).reshape(-1), pr.normals, rtol=0, atol=1e-14)
    assert np.allclose(k, pr.curvatures, rtol=1e-13, atol=1e-13)
    assert np.allclose(w, pr.weights, rtol=1e-14, atol=0)


def test_dense_matrix_matches_oracle_entries():
    H.ensure_oracle()
    pr, coef, _ = _case()
    A = AD.laplace_matrix(*AD.star_geometry(coef, pr.n_points))
    o = K.PortSolver(pr, id_tol=1e-6)
    idx = np.arange(pr.n_points, dtype=np.int32)
    B = o.kernel_block(idx, idx)
    o.close()
    assert np.abs(A - B).max() <= 1e-14 * np.abs(B).max()


def test_dense_gradient_matches_finite_differences():
    pr, coef, u_star = _case()
    out = AD.dense_gradient(coef, pr.n_points, pr.f, pr.targets, u_star)
    h = 1e-6
    for q in (0, 3, 17, 31):
        cp, cm = coef.copy(), coef.copy()
        cp[q] += h
        cm[q] -= h
        fd = (AD.objective(cp, pr.n_points, pr.f, pr.targets, u_star) -
              AD.objective(cm, pr.n_points, pr.f, pr.targets, u_star)) / (2 * h)
        assert abs(fd - out["dJdc"][q]) <= 1e-6 * max(1.0, np.abs(out["dJdc"]).max()), q
    # dJ/df against finite differences in two data entries
    for j in (0, 101):
        fp, fm = pr.f.copy(), pr.f.copy()
        fp[j] += h
        fm[j] -= h
        fd = (AD.objective(coef, pr.n_points, fp, pr.targets, u_star) -
              AD.objective(coef, pr.n_points, fm, pr.targets, u_star)) / (2 * h)
        assert abs(fd - out["dJdf"][j]) <= 1e-6 * max(1.0, np.abs(out["dJdf"]).max())
