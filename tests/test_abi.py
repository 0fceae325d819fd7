"""The C ABI library loads and exports every entry point include/kinterp.h
declares; argument errors come back as codes, never as aborts (no GPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import kinterp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "kinterp.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ki_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = kinterp.load()
    names = declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_version_and_error_string():
    lib = kinterp.load()
    assert lib.ki_version() >= 100
    assert isinstance(lib.ki_last_error(), bytes)


def test_argument_errors_return_codes():
    lib = kinterp.load()
    h = C.c_void_p()
    one = np.ones(4)
    dp = C.POINTER(C.c_double)
    d = one.ctypes.data_as(dp)
    assert lib.ki_factor(7, 2, d, d, d, d, 0, None, 32, 1e-6, None, C.byref(h)) == 1
    assert lib.ki_factor(0, 0, d, d, d, d, 0, None, 32, 1e-6, None, C.byref(h)) == 1
    assert lib.ki_factor(0, 2, d, d, d, d, 0, None, 32, -1.0, None, C.byref(h)) == 1
    assert lib.ki_solve(None, d, d, None) == 1
    assert lib.ki_num_levels(None) < 0


def test_partition_handle_rejects_solves():
    p = kinterp.Partition(np.array([0.1, 0.2, 0.3, 0.4]), 1, 32)
    lib = kinterp.load()
    x = np.zeros(4)
    rc = lib.ki_solve(p.h, x.ctypes.data_as(C.POINTER(C.c_double)),
                      x.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert rc == 4


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") is None and
                    os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_factor_without_device_fails_cleanly():
    lib = kinterp.load()
    h = C.c_void_p()
    pts = np.array([0.0, 0.0, 1.0, 0.0, 0.0, 1.0, 1.0, 1.0])
    d = pts.ctypes.data_as(C.POINTER(C.c_double))
    w = np.ones(4)
    dw = w.ctypes.data_as(C.POINTER(C.c_double))
    rc = lib.ki_factor(0, 4, d, d, dw, dw, 0, None, 32, 1e-6, None, C.byref(h))
    assert rc == 2 and b"CUDA" in lib.ki_last_error() or b"device" in lib.ki_last_error()
