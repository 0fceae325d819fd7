"""Dense FP64 reference gradient of the target-potential objective.

TEST INFRASTRUCTURE ONLY: the checker for the GPU adjoint, never the product.

Objective (Laplace double layer, simply connected star curve):
    A(c) mu = f,  u = K_t(c) mu,  J = sum_t (u_t - u*_t)^2
with the node geometry (positions, normals, curvatures, trapezoid weights)
of r(t) = 1 + sum_k c_k cos kt + s_k sin kt.  Entries restate the reference
Laplace kernel (kernel.cpp:11-36): off the diagonal
    A_ij = -(w_j / 2 pi) (r . n_j) / |r|^2,  r = x_i - x_j,
on it 1/2 + kappa_i w_i / (4 pi); the target matrix is the same formula
with the target point as x_i (kernel.cpp:337-357).  The operator matrix can
also be taken from the oracle's Kernel::operator() restatement (kioracle
kernel_block) to tie the two together.

Gradient: lam = A^-T K_t^T g_u, g_u = 2 (u - u*); dJ/df = lam;
dJ/d(geometry) = g_u^T dK_t mu - lam^T dA mu, formed densely; dJ/dc by the
chain rule with the geometry Jacobian taken by complex-step differentiation
(exact to rounding, the curve formulas being analytic in c).
"""
from __future__ import annotations

import numpy as np


def star_geometry(coef, n):
    """Nodes of the Fourier star (works for complex coef: complex step)."""
    coef = np.asarray(coef)
    kmax = coef.size // 2
    t = 2.0 * np.pi * np.arange(n) / n
    k = np.arange(1, kmax + 1)[:, None]
    cc, ss = coef[:kmax, None], coef[kmax:, None]
    ck, sk = np.cos(k * t), np.sin(k * t)
    r = 1.0 + (cc * ck + ss * sk).sum(0)
    dr = (k * (-cc * sk + ss * ck)).sum(0)
    ddr = (-(k * k) * (cc * ck + ss * sk)).sum(0)
    c, s = np.cos(t), np.sin(t)
    x, y = r * c, r * s
    xp, yp = dr * c - r * s, dr * s + r * c
    xpp = ddr * c - 2.0 * dr * s - r * c
    ypp = ddr * s + 2.0 * dr * c - r * s
    speed = np.sqrt(xp * xp + yp * yp)
    kappa = (xp * ypp - yp * xpp) / speed ** 3
    return x, y, yp / speed, -xp / speed, kappa, speed * (2.0 * np.pi / n)


def geometry_jacobian(coef, n, h=1e-30):
    """d(x, y, nx, ny, kappa, w)/dc: array (len(coef), 6, n), complex step."""
    coef = np.asarray(coef, dtype=np.float64)
    out = np.empty((coef.size, 6, n))
    for q in range(coef.size):
        cz = coef.astype(np.complex128)
        cz[q] += 1j * h
        g = star_geometry(cz, n)
        for a in range(6):
            out[q, a] = np.imag(g[a]) / h
    return out


def laplace_matrix(x, y, nx, ny, kappa, w):
    rx = x[:, None] - x[None, :]
    ry = y[:, None] - y[None, :]
    rho = rx * rx + ry * ry
    np.fill_diagonal(rho, 1.0)
    A = -(w[None, :] / (2 * np.pi)) * (rx * nx[None, :] + ry * ny[None, :]) / rho
    np.fill_diagonal(A, 0.5 + kappa * w / (4 * np.pi))
    return A


def target_matrix(tx, ty, x, y, nx, ny, w):
    rx = tx[:, None] - x[None, :]
    ry = ty[:, None] - y[None, :]
    rho = rx * rx + ry * ry
    return -(w[None, :] / (2 * np.pi)) * (rx * nx[None, :] + ry * ny[None, :]) / rho


def _source_grads(px, py, lam, x, y, nx, ny, w, mu, skip_diag):
    """mu_j sum_i lam_i dK(p_i, j)/d(x_j, y_j, nx_j, ny_j, w_j)."""
    rx = px[:, None] - x[None, :]
    ry = py[:, None] - y[None, :]
    rho = rx * rx + ry * ry
    if skip_diag:
        np.fill_diagonal(rho, np.inf)
    inv = 1.0 / rho
    rn = rx * nx[None, :] + ry * ny[None, :]
    c = -w / (2 * np.pi)
    L = lam[:, None]
    # dK/dx_j = -c [n_j / rho - 2 (r.n) r / rho^2]
    gx = -c * ((L * (nx[None, :] * inv - 2 * rn * rx * inv * inv)).sum(0))
    gy = -c * ((L * (ny[None, :] * inv - 2 * rn * ry * inv * inv)).sum(0))
    gnx = c * (L * rx * inv).sum(0)
    gny = c * (L * ry * inv).sum(0)
    gw = -(L * rn * inv).sum(0) / (2 * np.pi)
    return mu * gx, mu * gy, mu * gnx, mu * gny, mu * gw


def dense_gradient(coef, n, f, targets, u_star, A=None):
    """Returns J, dJ/dcoef, dJ/df (and u, mu) by dense FP64 algebra."""
    x, y, nx, ny, kappa, w = star_geometry(np.asarray(coef, dtype=np.float64), n)
    if A is None:
        A = laplace_matrix(x, y, nx, ny, kappa, w)
    tg = np.asarray(targets, dtype=np.float64).reshape(-1, 2)
    Kt = target_matrix(tg[:, 0], tg[:, 1], x, y, nx, ny, w)
    mu = np.linalg.solve(A, f)
    u = Kt @ mu
    gu = 2.0 * (u - u_star)
    J = float(((u - u_star) ** 2).sum())
    lam = np.linalg.solve(A.T, Kt.T @ gu)
    # target term (targets fixed)
    t_src = _source_grads(tg[:, 0], tg[:, 1], gu, x, y, nx, ny, w, mu, False)
    # operator term: node j as source, node i as target, diagonal
    o_src = _source_grads(x, y, lam, x, y, nx, ny, w, mu, True)
    rx = x[:, None] - x[None, :]
    ry = y[:, None] - y[None, :]
    rho = rx * rx + ry * ry
    np.fill_diagonal(rho, np.inf)
    inv = 1.0 / rho
    c = -w / (2 * np.pi)
    ax, ay = c * nx, c * ny  # per source
    rn = rx * ax[None, :] + ry * ay[None, :]
    M = mu[None, :]
    o_tgt_x = lam * (M * (ax[None, :] * inv - 2 * rn * rx * inv * inv)).sum(1)
    o_tgt_y = lam * (M * (ay[None, :] * inv - 2 * rn * ry * inv * inv)).sum(1)
    lm = lam * mu
    g = np.zeros((6, n))
    g[0] = t_src[0] - o_src[0] - o_tgt_x
    g[1] = t_src[1] - o_src[1] - o_tgt_y
    g[2] = t_src[2] - o_src[2]
    g[3] = t_src[3] - o_src[3]
    g[4] = -lm * w / (4 * np.pi)                      # kappa
    g[5] = t_src[4] - o_src[4] - lm * kappa / (4 * np.pi)  # w
    jac = geometry_jacobian(coef, n)  # (ncoef, 6, n) in (x, y, nx, ny, kappa, w)
    dJdc = np.einsum("qan,an->q", jac, g)
    return {"J": J, "dJdc": dJdc, "dJdf": lam, "u": u, "mu": mu, "node_grad": g}


def objective(coef, n, f, targets, u_star):
    x, y, nx, ny, kappa, w = star_geometry(np.asarray(coef, dtype=np.float64), n)
    A = laplace_matrix(x, y, nx, ny, kappa, w)
    tg = np.asarray(targets, dtype=np.float64).reshape(-1, 2)
    Kt = target_matrix(tg[:, 0], tg[:, 1], x, y, nx, ny, w)
    u = Kt @ np.linalg.solve(A, f)
    return float(((u - u_star) ** 2).sum())
