"""GPU adjoint: the transposed solve and the backward pass of the target
potential (ki_adjoint_forward / ki_adjoint_backward through the
torch.autograd wrapper), against the dense FP64 gradient oracle and central
finite differences (h = 1e-6) of the GPU objective.

Bars: A^T x = b to 1e-9 relative (factorization at id_tol 1e-10); gradient
with respect to the 32 Fourier shape coefficients and to the boundary data
within 1e-7 relative of the dense FP64 gradient; finite differences within
1e-4 relative (their own truncation and the 1e-10 solve accuracy / h)."""
import numpy as np
import pytest

import adjoint_dense as AD
import helpers as H
import ki_geometry as G
import kinterp

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


@pytest.mark.parametrize("pr", [G.ellipse_case(n=1024), G.fourier_star_case(n=2048)],
                         ids=["ellipse1024", "fourier2048"])
def test_transpose_solve(pr):
    import torch
    s = kinterp.Solver(pr, id_tol=1e-10)
    b = np.random.default_rng(5).standard_normal(s.n_dofs)
    bd = _dev(b)
    x = torch.empty_like(bd)
    s.solve_transpose_device(bd.data_ptr(), x.data_ptr())
    torch.cuda.synchronize()
    idx = np.arange(s.n_dofs, dtype=np.int32)
    A = s.kernel_block(idx, idx)
    xh = x.cpu().numpy()
    assert np.linalg.norm(A.T @ xh - b) / np.linalg.norm(b) < 1e-9


def _autograd_grad(pr, coef, u_star):
    import torch
    import ki_autograd as KA
    c = torch.tensor(coef, dtype=torch.float64, device="cuda", requires_grad=True)
    f = torch.tensor(pr.f, dtype=torch.float64, device="cuda", requires_grad=True)
    pts, nrm, kap, w = KA.fourier_star_geometry(c, pr.n_points)
    tg = torch.tensor(pr.targets, dtype=torch.float64, device="cuda")
    u = KA.target_potential(pts, nrm, kap, w, f, tg, pr.leaf_points, 1e-10)
    us = torch.tensor(u_star, dtype=torch.float64, device="cuda")
    J = ((u - us) ** 2).sum()
    J.backward()
    return float(J), c.grad.cpu().numpy(), f.grad.cpu().numpy()


def test_adjoint_matches_dense_gradient():
    pr = G.fourier_star_case(n=2048)
    coef, u_star = pr.extra["coef"], pr.extra["u_star"]
    J, gc, gf = _autograd_grad(pr, coef, u_star)
    ref = AD.dense_gradient(coef, pr.n_points, pr.f, pr.targets, u_star)
    assert abs(J - ref["J"]) <= 1e-9 * abs(ref["J"])
    assert np.linalg.norm(gc - ref["dJdc"]) <= 1e-7 * np.linalg.norm(ref["dJdc"])
    assert np.linalg.norm(gf - ref["dJdf"]) <= 1e-7 * np.linalg.norm(ref["dJdf"])


def _gpu_objective(pr, coef, u_star):
    import torch
    import ki_autograd as KA
    c = torch.tensor(coef, dtype=torch.float64, device="cuda")
    pts, nrm, kap, w = KA.fourier_star_geometry(c, pr.n_points)
    f = torch.tensor(pr.f, dtype=torch.float64, device="cuda")
    tg = torch.tensor(pr.targets, dtype=torch.float64, device="cuda")
    u = KA.target_potential(pts, nrm, kap, w, f, tg, pr.leaf_points, 1e-10)
    return float(((u.cpu().numpy() - u_star) ** 2).sum())


@pytest.mark.parametrize("n", [2048, 8192])
def test_adjoint_matches_finite_differences(n):
    pr = G.fourier_star_case(n=n)
    coef, u_star = pr.extra["coef"], pr.extra["u_star"]
    _, gc, gf = _autograd_grad(pr, coef, u_star)
    h = 1e-6
    scale = np.abs(gc).max()
    for q in (0, 7, 16, 31):
        cp, cm = coef.copy(), coef.copy()
        cp[q] += h
        cm[q] -= h
        fd = (_gpu_objective(pr, cp, u_star) - _gpu_objective(pr, cm, u_star)) / (2 * h)
        assert abs(fd - gc[q]) <= 1e-4 * scale, (q, fd, gc[q])


@pytest.mark.parametrize("data", ["fixed", "trace"])
def test_shape_optimization_decreases_objective(data):
    """Adjoint-driven shape optimisation (the finite-difference stencil of
    the reference's shape experiment replaced by the adjoint): starting from
    the unit circle, the objective falls toward a target shape's potentials,
    both for boundary data fixed per node and for data that is a function of
    the moving boundary points."""
    import torch
    import ki_autograd as KA
    import ki_shape_opt as SO
    target = G.fourier_star_case(n=2048, seed=7)
    n = target.n_points
    c_t = torch.tensor(target.extra["coef"], dtype=torch.float64, device="cuda")
    pts, nrm, kap, w = KA.fourier_star_geometry(c_t, n)
    tg = torch.tensor(target.targets, dtype=torch.float64, device="cuda")
    f = SO.trace_data if data == "trace" else target.f
    f_t = f(pts) if callable(f) else torch.tensor(f, dtype=torch.float64, device="cuda")
    u_star = KA.target_potential(pts, nrm, kap, w, f_t, tg).detach().cpu().numpy()
    coef0 = np.zeros_like(target.extra["coef"])
    coef, hist = SO.optimize(coef0, n, target.targets, u_star, f, steps=10, lr=2e-3)
    J = [h[0] for h in hist]
    assert J[0] > 0 and J[-1] < 0.7 * J[0], J
