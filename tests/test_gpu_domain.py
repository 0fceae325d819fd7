"""GPU domain evaluation (ki_eval_domain / ki_domain_mask_device): the
solution on grids of domain points as boundary_integral_solve computes it
(linear_solve.cpp:142-180).

Bars: the domain test bit-exact against the CPU restatement of
Boundary::is_in_domain (itself pinned to the reference's compiled functions
on the CPU); the values within 1e-12 relative of the exact-entry target
evaluation (which matches the oracle) and of the oracle's dense evaluation,
exactly zero outside; and the reference's five analytic agreement tests
(kern_interp_test.cpp:397-488: grid of 20^2 points over the boundary's
coordinate range, id_tol 1e-13, error <= 10 x 1e-13) through
boundary_integral_solve."""
import numpy as np
import pytest

import domain as D
import helpers as H
import ki_geometry as G
import kinterp
import kioracle as K

pytestmark = pytest.mark.gpu


def _ref_shape_problem(kind, pde, n, leaf=32, tol=1e-13):
    pts, nrm, kap, w, holes = G.reference_shape(kind, n)
    if pde == G.STOKES:
        f = G.tangent_vec(nrm)
    elif pde == G.LAPLACE_NEUMANN:
        # Donut DEFAULT data (donut.cpp:52-58): 1 on the outer curve, -1/r on the hole
        f = np.ones(pts.size // 2)
        f[n:] = -1.0 / holes[0, 2]
    else:
        f = G.single_electron(pts)
    return G.Problem("%s_%d_%d" % (kind, pde, n), pde, pts, nrm, kap, w, holes, f,
                     np.zeros(0), np.zeros(0), leaf // (2 if pde == G.STOKES else 1), tol)


DISKS = {"circle": (0.5, 0.5, 0.25), "annulus": (0.5, 0.5, 1.0), "donut": (0.5, 0.5, 1.0)}


def _cases():
    return {
        "star16k_nodes": (lambda: G.star_case(n=16384), (100, -1.35, 1.35), "nodes", None),
        "stokes_holes16k_nodes": (lambda: G.stokes_holes_case(n_total=16384),
                                  (64, -1.05, 1.05), "nodes", None),
        "ellipse_few_targets": (lambda: G.ellipse_case(n=1024), (4, -0.7, 0.7), "nodes", None),
        "annulus_stokes_disk": (lambda: _ref_shape_problem("annulus", G.STOKES, 1024, 64, 1e-10),
                                (40, -0.6, 1.6), "disk", DISKS["annulus"]),
        "donut_neumann_disk": (lambda: _ref_shape_problem("donut", G.LAPLACE_NEUMANN, 1024, 64,
                                                          1e-10),
                               (40, -0.6, 1.6), "disk", DISKS["donut"]),
        "circle_laplace_nodes": (lambda: _ref_shape_problem("circle", G.LAPLACE, 1024, 64, 1e-10),
                                 (30, 0.2, 0.8), "nodes", None),
    }


CASES = _cases()


def _mask_oracle(pr, tg, domain, disk):
    if domain == "nodes":
        return D.in_domain_nodes(pr.points, pr.holes, tg)
    return D.in_domain_disk(disk[0], disk[1], disk[2], pr.holes, tg)


@pytest.mark.parametrize("name", sorted(CASES))
def test_domain_mask_bit_exact(name):
    import torch
    make, grid, domain, disk = CASES[name]
    pr = make()
    tg = D.domain_points(*grid[:1], grid[1], grid[2], grid[1], grid[2])
    # add points on and around nodes (the 1e-2 distance and the crossing
    # test's equal-height cases)
    p = pr.points.reshape(-1, 2)
    k = np.arange(0, p.shape[0], max(1, p.shape[0] // 50))
    extra = [p[k], p[k] + 0.0099999, p[k] - 0.0100001, p[k] * np.array([0.9, 1.0])]
    tg = np.concatenate([tg] + [e.reshape(-1) for e in extra])
    s = kinterp.Solver(pr)
    d_tg = torch.tensor(tg, device="cuda", dtype=torch.float64)
    m = torch.empty(tg.size // 2, device="cuda", dtype=torch.uint8)
    s.domain_mask_device(tg.size // 2, d_tg.data_ptr(), m.data_ptr(), domain, disk)
    torch.cuda.synchronize()
    assert np.array_equal(m.cpu().numpy(), _mask_oracle(pr, tg, domain, disk))


@pytest.mark.parametrize("name", sorted(CASES))
def test_domain_eval_matches_exact_entries(name):
    make, grid, domain, disk = CASES[name]
    pr = make()
    tg = D.domain_points(grid[0], grid[1], grid[2], grid[1], grid[2])
    s = kinterp.Solver(pr)
    mu, alpha = s.solve(pr.f)
    al = alpha if s.n_border else None
    out = s.eval_domain(tg, mu, al, domain, disk)
    exact = s.eval_targets(tg, mu, al)
    inside = np.repeat(_mask_oracle(pr, tg, domain, disk).astype(bool), pr.sol_dim)
    assert inside.any()
    assert np.all(out[~inside] == 0.0)
    assert np.abs(out[inside] - exact[inside]).max() <= 1e-12 * np.abs(exact[inside]).max()
    # no test: every point evaluated
    out_all = s.eval_domain(tg, mu, al, "all")
    far = np.repeat(D.in_domain_nodes(pr.points, pr.holes, tg).astype(bool) |
                    ~_near_any(pr, tg), pr.sol_dim)
    assert np.abs(out_all[far] - exact[far]).max() <= 1e-12 * np.abs(exact[far]).max()


def _near_any(pr, tg):
    """Points within 1e-6 of a node (the fast evaluation skips an exactly
    coincident node; its neighbourhood is ill-conditioned for both)."""
    p = pr.points.reshape(-1, 2)
    t = tg.reshape(-1, 2)
    out = np.zeros(t.shape[0], dtype=bool)
    for b in range(0, t.shape[0], 512):
        d = np.hypot(t[b:b + 512, None, 0] - p[None, :, 0], t[b:b + 512, None, 1] - p[None, :, 1])
        out[b:b + 512] = (d < 1e-6).any(1)
    return out


@pytest.mark.parametrize("kind,pde", [("circle", G.LAPLACE), ("annulus", G.STOKES),
                                      ("donut", G.LAPLACE_NEUMANN)])
def test_domain_eval_matches_oracle(kind, pde):
    H.ensure_oracle()
    pr = _ref_shape_problem(kind, pde, 1024, 64, 1e-10)
    lo, hi = pr.points.min(), pr.points.max()
    tg = D.domain_points(24, lo, hi, lo, hi)
    s = kinterp.Solver(pr)
    mu, alpha = s.solve(pr.f)
    al = alpha if s.n_border else None
    out = s.eval_domain(tg, mu, al, "disk", DISKS[kind])
    o = K.PortSolver(pr, id_tol=1e-10)
    ref = o.eval_targets(tg, mu, al)
    ref[~np.repeat(D.in_domain_disk(*DISKS[kind], pr.holes, tg).astype(bool), pr.sol_dim)] = 0.0
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()


# ---------------------------------------------------------------- the
# reference's analytic agreement tests (kern_interp_test.cpp:296-488)


def _laplace_error(sol, tg, inside):
    t = tg.reshape(-1, 2)[inside]
    pot = np.log(np.sqrt((t[:, 0] + 3) ** 2 + (t[:, 1] + 2) ** 2)) / (2 * np.pi)
    return np.sqrt(((pot - sol[inside]) ** 2).sum()) / np.sqrt((pot ** 2).sum())


def _neumann_error(sol, tg, inside):
    t = tg.reshape(-1, 2)[inside]
    truth = np.log(np.sqrt((t[:, 0] - 0.5) ** 2 + (t[:, 1] - 0.5) ** 2))
    res = sol[inside] - sol[inside].mean()
    truth = truth - truth.mean()
    return np.sqrt(((res - truth) ** 2).sum()) / np.sqrt((truth ** 2).sum())


def _stokes_error(sol, tg, inside, n_holes):
    t = tg.reshape(-1, 2)[inside]
    r = t - 0.5
    rn = np.hypot(r[:, 0], r[:, 1])
    truth = np.stack([-r[:, 1], r[:, 0]], 1)
    tn = np.hypot(truth[:, 0], truth[:, 1])
    if n_holes == 0:
        truth = truth * (rn / tn * 4.0)[:, None]
    else:
        truth = truth * ((-1.0 / rn + 2 * rn) / tn)[:, None]
    u = sol.reshape(-1, 2)[inside]
    return np.sqrt(((u - truth) ** 2).sum()) / np.sqrt((truth ** 2).sum())


@pytest.mark.parametrize("kind,pde", [("circle", G.LAPLACE), ("annulus", G.LAPLACE),
                                      ("donut", G.LAPLACE_NEUMANN), ("circle", G.STOKES),
                                      ("donut", G.STOKES)])
def test_reference_analytic_agreement(kind, pde):
    pr = _ref_shape_problem(kind, pde, 4096)
    lo, hi = pr.points.min(), pr.points.max()   # quadtree.min / max (quadtree.cpp:80-86)
    tg = kinterp.domain_points(20, lo, hi, lo, hi)
    sol = kinterp.boundary_integral_solve(pr, tg, id_tol=1e-13, max_leaf_dofs=32,
                                          domain="disk", disk=DISKS[kind])
    inside = D.in_domain_disk(*DISKS[kind], pr.holes, tg).astype(bool)
    assert np.all(sol.reshape(-1, pr.sol_dim)[~inside] == 0.0)
    if pde == G.STOKES:
        err = _stokes_error(sol, tg, inside, pr.holes.shape[0])
    elif pde == G.LAPLACE_NEUMANN:
        err = _neumann_error(sol, tg, inside)
    else:
        err = _laplace_error(sol, tg, inside)
    assert err <= 10 * 1e-13, err
