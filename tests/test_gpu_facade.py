"""The C++ drop-in API on a B200: the repository's caller
(tests/cxx/facade_caller.cpp: backward errors of Laplace, Laplace-Neumann
and Stokes factorizations against the dense operator, analytic agreement,
copy_into and perturb + skeletonize) and the reference's own test file
compiled unmodified against include/kern_interp (oracle/_ref/
facade_ref_tests, built where the reference sources are present).  Bars are
the reference's: backward error <= 10 id_tol, analytic <= 10 x 1e-13,
update within 20 id_tol of a fresh factorization, copy within 1e-15."""
import os
import subprocess

import pytest

import facade_build as FB

pytestmark = pytest.mark.gpu


def test_caller_on_gpu():
    exe = FB.build_caller()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failed checks" in r.stdout


def test_reference_test_file_on_the_drop_in():
    exe = FB.build_reference_tests()
    if exe is None or not os.path.exists(exe):
        pytest.skip("reference test binary not built (needs the reference sources)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "0 failed checks" in r.stdout
    assert r.stdout.count("[ RUN ]") >= 25
