"""Shape optimisation by the adjoint: gradient descent on the Fourier shape
coefficients of a star-shaped boundary to match target potentials.

The reference's shape experiment (experiment_three.cpp:22-56, 152-209)
estimates the objective's gradient with a four-point finite-difference
stencil, one full factor and solve per stencil point.  Here the gradient of

    J(c) = sum_t (u(x_t; c) - u*_t)^2,   u = K_t A(c)^{-1} f(c)

comes from one forward solve and one backward pass of the factorization
(ki_adjoint_forward / ki_adjoint_backward through ki_autograd), including
the dependence of the boundary data f on the boundary points when f is
given as a differentiable function of them.
"""
from __future__ import annotations

import torch

import ki_autograd as KA


def optimize(coef0, n, targets, u_star, data, steps=20, lr=1e-2, leaf_points=64,
             id_tol=1e-10, optimizer="adam", device="cuda"):
    """Runs `steps` optimizer steps from coef0 (2 K Fourier coefficients,
    r(t) = 1 + sum_k c_k cos kt + s_k sin kt, n nodes).  `data` is either
    the boundary data per node (n values, fixed while the shape moves) or a
    torch function of the interleaved boundary points (its dependence on the
    shape is then differentiated too).  Returns the final coefficients
    (numpy) and the history of (J, |grad J|) before each step."""
    c = torch.tensor(coef0, dtype=torch.float64, device=device, requires_grad=True)
    tg = torch.as_tensor(targets, dtype=torch.float64, device=device)
    us = torch.as_tensor(u_star, dtype=torch.float64, device=device)
    opt = (torch.optim.Adam([c], lr=lr) if optimizer == "adam"
           else torch.optim.SGD([c], lr=lr))
    fixed = (None if callable(data) else
             torch.as_tensor(data, dtype=torch.float64, device=device))
    history = []
    for _ in range(steps):
        opt.zero_grad()
        pts, nrm, kap, w = KA.fourier_star_geometry(c, n)
        f = data(pts) if callable(data) else fixed
        u = KA.target_potential(pts, nrm, kap, w, f, tg, leaf_points, id_tol)
        J = ((u - us) ** 2).sum()
        J.backward()
        history.append((float(J.detach()), float(c.grad.norm())))
        opt.step()
    return c.detach().cpu().numpy(), history


def trace_data(points):
    """f = x^2 - x y / 2 on the boundary: the trace of a non-harmonic
    function, so the interior potential depends on the shape."""
    p = points.reshape(-1, 2)
    return p[:, 0] * p[:, 0] - 0.5 * p[:, 0] * p[:, 1]
