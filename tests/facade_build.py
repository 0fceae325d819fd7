"""Builds the C++ callers of the drop-in API (test infrastructure): the
repository's own caller tests/cxx/facade_caller.cpp, and, where the
reference sources are present, the reference's own test file compiled
unmodified against include/kern_interp (make -C oracle facade)."""
from __future__ import annotations

import os
import shutil
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "kern-interp-old_b200")
INCLUDE = os.path.join(ROOT, "include")
CALLER_SRC = os.path.join(ROOT, "tests", "cxx", "facade_caller.cpp")
CALLER_BIN = os.path.join(PKG, "_build", "facade_caller")
REF_TESTS_BIN = os.path.join(ROOT, "oracle", "_ref", "facade_ref_tests")
REF_DIR = os.environ.get("KI_REFERENCE_DIR", "/root/reference")


def facade_lib():
    import build as kbuild
    kbuild.build()
    return kbuild.FACADE_LIB


def build_caller():
    facade_lib()
    os.makedirs(os.path.dirname(CALLER_BIN), exist_ok=True)
    cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-I" + INCLUDE, "-o", CALLER_BIN, CALLER_SRC,
           "-L" + PKG, "-l:libkern_interp.so", "-Wl,-rpath," + PKG]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("facade caller build failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return CALLER_BIN


def build_reference_tests():
    """The reference's kern_interp_test.cpp (and its spline boundaries)
    against the drop-in headers; None when the reference is absent."""
    if not os.path.isdir(os.path.join(REF_DIR, "kern_interp")):
        return REF_TESTS_BIN if os.path.exists(REF_TESTS_BIN) else None
    facade_lib()
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "facade", "KI_REFERENCE_DIR=" + REF_DIR],
                   check=True, capture_output=True)
    return REF_TESTS_BIN
