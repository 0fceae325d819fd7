"""Failure paths of the C ABI that need no GPU: non-finite boundary data is
refused with KI_ERR_ARG before any device work (the reference would carry
NaN through its factorization), and the test hook of the cooperative LU
accepts only its documented values."""
import ctypes as C

import numpy as np
import pytest

import ki_geometry as G
import kinterp

KI_ERR_ARG = 1


def _factor_rc(pr, points=None, normals=None, weights=None):
    lib = kinterp.load()
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    pts = f64(pr.points if points is None else points)
    nrm = f64(pr.normals if normals is None else normals)
    kap = f64(pr.curvatures)
    w = f64(pr.weights if weights is None else weights)
    d = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    h = C.c_void_p()
    rc = lib.ki_factor(pr.pde, pr.n_points, d(pts), d(nrm), d(kap), d(w), 0, None,
                       pr.max_leaf_dofs, 1e-10, None, C.byref(h))
    return rc, lib.ki_last_error()


@pytest.mark.parametrize("field,value", [("points", np.nan), ("normals", np.inf),
                                         ("weights", -np.inf)])
def test_non_finite_geometry_is_refused(field, value):
    pr = G.ellipse_case(n=1024)
    arr = getattr(pr, field).copy()
    arr[137] = value
    rc, msg = _factor_rc(pr, **{field: arr})
    assert rc == KI_ERR_ARG
    assert b"non-finite" in msg


def test_fault_injection_hook_values():
    lib = kinterp.load()
    assert lib.ki_test_inject_fault(7) == KI_ERR_ARG
    assert lib.ki_test_inject_fault(-1) == KI_ERR_ARG
    for v in (1, 2, 0):
        assert lib.ki_test_inject_fault(v) == 0
