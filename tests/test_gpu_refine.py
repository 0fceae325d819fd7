"""GPU refinement path: the fast FP64 operator product, the preconditioner
with a border right-hand side, and GMRES refinement of a loose
factorization to FP64 accuracy, against the FP64 oracle and dense solves.

Bars: the fast product equals the entry-exact product to 1e-13 relative
(FP64 rounding of a reassociated sum); the refined solution of a factorization
at id_tol 1e-6 has true relative residual <= 1e-12 and is within 1e-10
relative of the FP64 oracle's solution at id_tol 1e-10."""
import numpy as np
import pytest

import helpers as H
import ki_geometry as G
import kinterp
import kioracle as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _oracle_built():
    H.ensure_oracle()


def _problems():
    return {
        "ellipse_laplace_1024": G.ellipse_case(),
        "stokes_holes_4096": G.stokes_holes_case(n_total=4096),
        "fourier_star_laplace_2048": G.fourier_star_case(n=2048),
    }


def _dev(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


@pytest.mark.parametrize("name", list(_problems()))
def test_fast_matvec_matches_entry_exact_product(name):
    import torch
    pr = _problems()[name]
    s = kinterp.Solver(pr, id_tol=1e-6)
    rng = np.random.default_rng(7)
    x = _dev(rng.standard_normal(s.n_dofs + s.n_border))
    y0 = torch.empty_like(x)
    y1 = torch.empty_like(x)
    s.apply_device(x.data_ptr(), y0.data_ptr())
    s.matvec_device(x.data_ptr(), y1.data_ptr())
    torch.cuda.synchronize()
    a, b = y0.cpu().numpy(), y1.cpu().numpy()
    assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-13


@pytest.mark.parametrize("name", list(_problems()) + ["star_laplace_16384", "stokes_holes_65536"])
def test_correction_product_error(name):
    """The FP32 far-field / FP64 near-field product of a correction: within
    2e-6 of the FP64 product relative to |y|, for any scaling of the
    density (the FP32 stage sees d * dscale), on vectors of magnitude 1e-9
    like the late corrections of a refinement."""
    import torch
    pr = {"star_laplace_16384": lambda: G.star_case(),
          "stokes_holes_65536": lambda: G.stokes_holes_case()}.get(name, lambda: _problems()[name])()
    s = kinterp.Solver(pr, id_tol=1e-6, mode=1)
    rng = np.random.default_rng(11)
    x = _dev(1e-9 * rng.standard_normal(s.n_dofs + s.n_border))
    y0 = torch.empty_like(x)
    y1 = torch.empty_like(x)
    s.matvec_device(x.data_ptr(), y0.data_ptr())
    errs = []
    for scale in (1e9, 1e7):
        s.matvec_correction_device(x.data_ptr(), y1.data_ptr(), scale)
        torch.cuda.synchronize()
        a, b = y0.cpu().numpy(), y1.cpu().numpy()
        errs.append(np.linalg.norm(a - b) / np.linalg.norm(a))
    assert max(errs) < 2e-6, errs
    s.close()


def test_fast_matvec_laplace_neumann():
    import torch
    pr = G.ellipse_case(n=1024)
    pr.pde = G.LAPLACE_NEUMANN
    s = kinterp.Solver(pr, id_tol=1e-6)
    x = _dev(np.random.default_rng(3).standard_normal(s.n_dofs))
    y0 = torch.empty_like(x)
    y1 = torch.empty_like(x)
    s.apply_device(x.data_ptr(), y0.data_ptr())
    s.matvec_device(x.data_ptr(), y1.data_ptr())
    torch.cuda.synchronize()
    a, b = y0.cpu().numpy(), y1.cpu().numpy()
    assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-13


def test_preconditioner_border_rhs():
    """The bordered solve with a nonzero border right-hand side g inverts the
    bordered operator: A M^-1 [f; g] = [f; g] to the factorization's accuracy."""
    import torch
    pr = G.stokes_holes_case(n_total=4096)
    s = kinterp.Solver(pr, id_tol=1e-10)
    rng = np.random.default_rng(11)
    N, nb = s.n_dofs, s.n_border
    f = rng.standard_normal(N)
    g = rng.standard_normal(nb)
    fd, gd = _dev(f), _dev(g)
    x = torch.zeros(N + nb, dtype=torch.float64, device="cuda")
    s.solve_bordered_device(fd.data_ptr(), gd.data_ptr(), x.data_ptr(), x.data_ptr() + 8 * N)
    y = torch.empty_like(x)
    s.apply_device(x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    r = y.cpu().numpy() - np.concatenate([f, g])
    assert np.linalg.norm(r) / np.linalg.norm(np.concatenate([f, g])) < 1e-8


@pytest.mark.parametrize("mode", [0, 1], ids=["reference_ids", "sketched_ids"])
@pytest.mark.parametrize("name", list(_problems()))
def test_refined_loose_factor_reaches_fp64(name, mode):
    """The FP64 oracle at id_tol 1e-10 carries its own ~1e-10 error (it is a
    1e-10 factorization); the converged reference here is the same oracle
    at id_tol 1e-13.  The refined GPU solution must be within 1e-10 of it,
    and no farther from the 1e-10 oracle than that oracle's own error allows."""
    pr = _problems()[name]
    s = kinterp.Solver(pr, id_tol=1e-6, mode=mode)
    mu, alpha, it, rr = s.solve_refined(pr.f, rel_tol=1e-12, max_iters=30)
    assert rr <= 1e-12, (it, rr)
    assert it <= 10
    o = K.PortSolver(pr, threads=8)
    mo, ao = o.solve(pr.f)
    o.close()
    o = K.PortSolver(pr, id_tol=1e-13, threads=8)
    mt, at = o.solve(pr.f)
    o.close()
    assert H.rel(mu, mt) < 1e-10
    if len(alpha):
        assert np.abs(alpha - at).max() < 1e-10 * max(1.0, np.abs(mt).max())
    own = H.rel(mo, mt)
    assert H.rel(mu, mo) < max(1e-10, 2.0 * own)


@pytest.mark.parametrize("name,tol", [("star_laplace_16384", 3e-7),
                                      ("stokes_holes_65536", 3e-8),
                                      ("stokes_holes_4096", 1e-6)])
def test_refined_true_residual(name, tol):
    """The refinement updates small residuals with the correction product:
    the residual it reports must agree with the true FP64 residual
    ||[f; 0] - A [mu; alpha]|| / ||f|| of the solution it returns, which must
    meet the 1e-12 bar."""
    import torch
    pr = {"star_laplace_16384": lambda: G.star_case(),
          "stokes_holes_65536": lambda: G.stokes_holes_case()}.get(name, lambda: _problems()[name])()
    s = kinterp.Solver(pr, id_tol=tol, mode=1)
    mu, alpha, it, rr = s.solve_refined(pr.f, rel_tol=1e-12, max_iters=30)
    assert rr <= 1e-12, (it, rr)
    x = _dev(np.concatenate([mu, alpha]))
    y = torch.empty_like(x)
    s.matvec_device(x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    b = np.concatenate([pr.f, np.zeros(len(alpha))])
    true = np.linalg.norm(b - y.cpu().numpy()) / np.linalg.norm(pr.f)
    assert true <= 1.5e-12, (true, rr, it)
    assert abs(true - rr) <= 0.5e-12 + 0.5 * rr, (true, rr)
    s.close()


def test_refined_matches_dense_solve():
    """Small Laplace problem: dense FP64 matrix from the exact entries,
    numpy solve; the refined GPU solution agrees to 1e-12."""
    pr = G.ellipse_case(n=1024)
    s = kinterp.Solver(pr, id_tol=1e-6)
    idx = np.arange(s.n_dofs, dtype=np.int32)
    A = s.kernel_block(idx, idx)
    mu_dense = np.linalg.solve(A, pr.f)
    mu, _, it, rr = s.solve_refined(pr.f, rel_tol=1e-13, max_iters=30)
    assert H.rel(mu, mu_dense) < 1e-12


@pytest.mark.parametrize("tol", [1e-2, 1e-3])
def test_refine_from_very_loose_factorization(tol):
    """A factorization too loose for stationary refinement to converge fast
    hands over to GMRES, which still reaches the FP64 residual."""
    pr = G.star_case(n=4096)
    s = kinterp.Solver(pr, id_tol=tol)
    mu, _, it, rr = s.solve_refined(pr.f, rel_tol=1e-12, max_iters=60)
    assert rr <= 1e-12, (it, rr)
    o = K.PortSolver(pr, id_tol=1e-13, threads=8)
    mt, _ = o.solve(pr.f)
    o.close()
    assert H.rel(mu, mt) < 1e-10


def test_sketched_ids_in_clusters_reach_fp64():
    """Preconditioner mode on a problem whose top-level boxes need
    multi-CTA clusters for their sketches (wide boxes at levels 1-2)."""
    pr = G.stokes_holes_case(n_total=16384)
    s = kinterp.Solver(pr, id_tol=1e-6, mode=1)
    mu, alpha, it, rr = s.solve_refined(pr.f, rel_tol=1e-12, max_iters=30)
    assert rr <= 1e-12, (it, rr)
    assert it <= 10
    o = K.PortSolver(pr, id_tol=1e-13, threads=8)
    mt, at = o.solve(pr.f)
    o.close()
    assert H.rel(mu, mt) < 1e-10


def test_tune_id_tol_returns_the_fastest_converging_candidate():
    """The autotuner times factor + refinement per candidate tolerance and
    returns the fastest one among those whose refinement reaches the target."""
    pr = _problems()["stokes_holes_4096"]
    tol, table = kinterp.tune_id_tol(pr, candidates=(1e-5, 1e-8), reps=1)
    assert [row[0] for row in table] == [1e-5, 1e-8]
    assert all(row[3] <= 1e-12 and row[2] >= 1 for row in table)
    assert tol == min(table, key=lambda row: row[1])[0]
