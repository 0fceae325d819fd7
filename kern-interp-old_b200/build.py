"""Builds libkinterp.so (the B200 solver: CUDA kernels + host C++ + C ABI).

    python kern-interp-old_b200/build.py [--force]

Every translation unit is compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); objects go to _build/ next to this
file and the shared library is written in place so it travels with the tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkinterp.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
         "-I" + CSRC, "-I" + INCLUDE]


def nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def ccbin():
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith(".cu") or f.endswith(".cpp"):
            out.append(os.path.join(CSRC, f))
    return out


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
          if f.endswith(".h") or f.endswith(".cuh")]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _compile(src, force):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj, None
    lang = [] if src.endswith(".cu") else ["-x", "cu"]
    cmd = [nvcc()] + ccbin() + ARCH + FLAGS + lang + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr)
    return obj, None


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if (force or not os.path.exists(LIB) or
            os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)):
        cmd = [nvcc()] + ccbin() + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    build_facade(force)
    if verbose:
        print("built", LIB, "and", FACADE_LIB)
    return LIB


FACADE = os.path.join(HERE, "facade")
FACADE_LIB = os.path.join(HERE, "libkern_interp.so")


def build_facade(force=False):
    """libkern_interp.so: the C++ drop-in API (include/kern_interp/*.h),
    host code over the C ABI of libkinterp.so (found next to it at run
    time through its rpath)."""
    srcs = sorted(os.path.join(FACADE, f) for f in os.listdir(FACADE) if f.endswith(".cpp"))
    hdrs = []
    for d, _, fs in os.walk(os.path.join(INCLUDE, "kern_interp")):
        hdrs += [os.path.join(d, f) for f in fs if f.endswith(".h")]
    hdrs.append(os.path.join(INCLUDE, "kinterp.h"))
    newest = max(os.path.getmtime(x) for x in srcs + hdrs + [LIB])
    if not force and os.path.exists(FACADE_LIB) and os.path.getmtime(FACADE_LIB) >= newest:
        return FACADE_LIB
    cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-I" + INCLUDE, "-o", FACADE_LIB] + srcs + \
          ["-L" + HERE, "-l:libkinterp.so", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("facade build failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return FACADE_LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
