"""Failure detection on a B200, without a GPU fault: the top-level
cooperative LU's bounded waits (200 ms, %globaltimer) end a factorization
with KI_ERR_NUMERIC instead of hanging, both when its abort word is raised
before it starts and when one thread block withholds its flag so that the
others' waits run out; the device stays usable and the next factorization
is exact.  Coincident boundary nodes make two columns of the operator equal
(the reference's entry formula takes r = 0 as the diagonal), an exactly
singular system no pivot reveals in floating point: the factorization
refuses them with KI_ERR_NUMERIC instead of returning meaningless factors.  The reference exits or asserts in these
cases (skel_factorization.cpp:151-154)."""
import ctypes as C
import time

import numpy as np
import pytest

import helpers as H
import ki_geometry as G
import kinterp
import kioracle as K

pytestmark = pytest.mark.gpu

KI_ERR_NUMERIC = 3


def _expect_numeric_failure(pr, **kw):
    with pytest.raises(kinterp.KiError) as ei:
        kinterp.Solver(pr, **kw)
    assert "(%d)" % KI_ERR_NUMERIC in str(ei.value), str(ei.value)
    return str(ei.value)


@pytest.mark.parametrize("mode", [1, 2], ids=["abort_raised", "flag_withheld"])
def test_cooperative_lu_bounded_wait_fails_cleanly(mode):
    lib = kinterp.load()
    pr = G.star_case(n=4096, n_targets=16)
    assert lib.ki_test_inject_fault(mode) == 0
    t0 = time.time()
    msg = _expect_numeric_failure(pr)
    assert "bounded wait" in msg
    assert time.time() - t0 < 30.0
    # the hook is one-shot and the context is intact: a clean factorization
    s = kinterp.Solver(pr)
    mu, _ = s.solve(pr.f)
    o = K.PortSolver(pr)
    mo, _ = o.solve(pr.f)
    o.close()
    assert H.rel(mu, mo) < 1e-10
    s.close()


def test_coincident_nodes_fail_with_numeric_error():
    pr = G.star_case(n=2048, n_targets=16)
    pts = pr.points.copy()
    pts[2 * 700:2 * 701] = pts[2 * 701:2 * 702]  # node 700 on top of node 701
    bad = G.Problem(pr.name + "_dup", pr.pde, pts, pr.normals, pr.curvatures, pr.weights,
                    pr.holes, pr.f, pr.targets, pr.exact, pr.leaf_points, pr.id_tol, pr.extra)
    msg = _expect_numeric_failure(bad)
    assert "coincident" in msg
    # and the device is still usable
    s = kinterp.Solver(pr)
    mu, _ = s.solve(pr.f)
    assert np.all(np.isfinite(mu))
    s.close()
