"""torch.autograd wrapper of the differentiable target potential.

    u = TargetPotential.apply(points, normals, curvatures, weights, f, targets)

solves the Laplace double-layer boundary integral equation A(geometry) mu = f
with the B200 recursive-skeletonization factorization and returns the
potential u = K_t mu at the targets (the schur_solve target map of
linear_solve.cpp:126-140).  The backward pass calls ki_adjoint_backward: one
transposed solve with the same factorization plus the derivative-of-kernel
contractions, giving gradients with respect to f and to every node's
position, normal, weight and curvature.  Gradients with respect to shape
parameters follow by ordinary autograd through the geometry, e.g.
`fourier_star_geometry` below.
"""
from __future__ import annotations

import math
import types

import numpy as np
import torch

import kinterp

LAPLACE = 0


def fourier_star_geometry(coef: torch.Tensor, n: int):
    """Differentiable nodes of r(t) = 1 + sum_k c_k cos kt + s_k sin kt,
    t_j = 2 pi j / n: interleaved points and outward normals, curvatures,
    trapezoid weights |x'(t_j)| 2 pi / n (the same curve as
    ki_geometry.fourier_star_geometry)."""
    kmax = coef.shape[0] // 2
    dt = dict(dtype=coef.dtype, device=coef.device)
    t = 2.0 * math.pi * torch.arange(n, **dt) / n
    k = torch.arange(1, kmax + 1, **dt)[:, None]
    cc, ss = coef[:kmax, None], coef[kmax:, None]
    ck, sk = torch.cos(k * t), torch.sin(k * t)
    r = 1.0 + (cc * ck + ss * sk).sum(0)
    dr = (k * (-cc * sk + ss * ck)).sum(0)
    ddr = (-(k * k) * (cc * ck + ss * sk)).sum(0)
    c, s = torch.cos(t), torch.sin(t)
    x, y = r * c, r * s
    xp, yp = dr * c - r * s, dr * s + r * c
    xpp = ddr * c - 2.0 * dr * s - r * c
    ypp = ddr * s + 2.0 * dr * c - r * s
    speed = torch.sqrt(xp * xp + yp * yp)
    kappa = (xp * ypp - yp * xpp) / speed ** 3
    points = torch.stack([x, y], 1).reshape(-1)
    normals = torch.stack([yp / speed, -xp / speed], 1).reshape(-1)
    weights = speed * (2.0 * math.pi / n)
    return points, normals, kappa, weights


def _problem(points, normals, curvatures, weights, leaf_points, id_tol):
    n = weights.shape[0]
    return types.SimpleNamespace(
        pde=LAPLACE, points=points, normals=normals, curvatures=curvatures, weights=weights,
        holes=np.zeros((0, 4)), n_points=n, max_leaf_dofs=leaf_points, id_tol=id_tol)


class TargetPotential(torch.autograd.Function):
    """u = K_t A^-1 f; inputs float64 tensors (points 2n, normals 2n,
    curvatures n, weights n, f n, targets 2 nt); u and the gradients live on
    the current CUDA device."""

    @staticmethod
    def forward(ctx, points, normals, curvatures, weights, f, targets, leaf_points=64,
                id_tol=1e-10):
        dev = torch.device("cuda", torch.cuda.current_device())
        cur = torch.cuda.current_stream(dev)
        # the library runs on its own side stream, ordered after the caller's
        # current stream and joined back into it before returning
        side = torch.cuda.Stream(dev)
        host = [a.detach().to("cpu", torch.float64).contiguous().numpy()
                for a in (points, normals, curvatures, weights)]
        f_d = f.detach().to(dev, torch.float64).contiguous()
        tg = targets.detach().to(dev, torch.float64).contiguous()
        nt = tg.numel() // 2
        mu = torch.empty_like(f_d)
        u = torch.empty(nt, dtype=torch.float64, device=dev)
        side.wait_stream(cur)
        s = kinterp.Solver(_problem(*host, leaf_points, id_tol), stream=side.cuda_stream)
        s.adjoint_forward(f_d.data_ptr(), nt, tg.data_ptr(), mu.data_ptr(), u.data_ptr())
        for t in (f_d, tg, mu, u):
            t.record_stream(side)
        cur.wait_stream(side)
        ctx.solver = s
        ctx.side = side
        ctx.nt = nt
        ctx.src_devices = [a.device for a in (points, normals, curvatures, weights, f)]
        ctx.save_for_backward(tg, mu)
        return u

    @staticmethod
    def backward(ctx, grad_u):
        tg, mu = ctx.saved_tensors
        s, side = ctx.solver, ctx.side
        cur = torch.cuda.current_stream(mu.device)
        n = mu.numel()
        gu = grad_u.detach().to(mu.device, torch.float64).contiguous()
        gf = torch.empty_like(mu)
        gp = torch.empty(2 * n, dtype=torch.float64, device=mu.device)
        gn = torch.empty_like(gp)
        gw = torch.empty_like(mu)
        gk = torch.empty_like(mu)
        side.wait_stream(cur)
        s.adjoint_backward(ctx.nt, tg.data_ptr(), mu.data_ptr(), gu.data_ptr(), gf.data_ptr(),
                           gp.data_ptr(), gn.data_ptr(), gw.data_ptr(), gk.data_ptr())
        for t in (gu, gf, gp, gn, gw, gk, tg, mu):
            t.record_stream(side)
        cur.wait_stream(side)
        d = ctx.src_devices
        return (gp.to(d[0]), gn.to(d[1]), gk.to(d[2]), gw.to(d[3]), gf.to(d[4]),
                None, None, None)


def target_potential(points, normals, curvatures, weights, f, targets, leaf_points=64,
                     id_tol=1e-10):
    return TargetPotential.apply(points, normals, curvatures, weights, f, targets, leaf_points,
                                 id_tol)
