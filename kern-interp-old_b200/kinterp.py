"""Python binding of the B200 solver's C ABI (include/kinterp.h).

The product is libkinterp.so next to this file (built by build.py).  This
module only marshals arrays through ctypes; every computation happens in the
library's CUDA kernels.  If the library is missing or cannot be loaded,
``load()`` raises -- there is no CPU fallback.

``Solver`` mirrors the reference pipeline (jpryan1/kern-interp-old):
constructing it runs QuadTree::initialize_tree + SkelFactorization::
skeletonize (quadtree.h:85-86, skel_factorization.h:40), ``solve`` is
linear_solve (linear_solve.h:27-29), ``eval_targets`` is schur_solve's target
evaluation (linear_solve.cpp:126-140) and ``kernel_block`` is
Kernel::operator() (kernel.cpp:99-111).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkinterp.so")

LAPLACE, LAPLACE_NEUMANN, STOKES = 0, 1, 2
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


class KiError(RuntimeError):
    pass


def load():
    """Loads libkinterp.so (raises if it is missing: no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise KiError("libkinterp.so not built: run kern-interp-old_b200/build.py")
    lib = C.CDLL(LIB_PATH)
    lib.ki_last_error.restype = C.c_char_p
    lib.ki_kernel_launches.restype = C.c_longlong
    fac_args = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_int, _dp, C.c_int, C.c_double,
                C.c_void_p, C.POINTER(C.c_void_p)]
    for name in ("ki_factor", "ki_factor_timed"):
        getattr(lib, name).argtypes = fac_args
        getattr(lib, name).restype = C.c_int
    lib.ki_partition.argtypes = [C.c_int, _dp, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    lib.ki_destroy.argtypes = [C.c_void_p]
    lib.ki_destroy.restype = None
    for name in ("ki_num_dofs", "ki_num_border", "ki_num_levels"):
        getattr(lib, name).argtypes = [C.c_void_p]
    lib.ki_num_boxes.argtypes = [C.c_void_p, C.c_int]
    lib.ki_solve.argtypes = [C.c_void_p, _dp, _dp, _dp]
    lib.ki_solve_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ki_apply_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ki_eval_targets.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]
    lib.ki_kernel_block.argtypes = [C.c_void_p, C.c_int, _ip, C.c_int, _ip, _dp]
    lib.ki_box_info.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _dp]
    lib.ki_box_lists.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip, _ip, _ip]
    lib.ki_allskel.argtypes = [C.c_void_p, _ip]
    lib.ki_stats.argtypes = [C.c_void_p, _dp, C.c_int]
    lib.ki_launch_log.argtypes = [C.c_void_p, _dp, C.c_int]
    _lib = lib
    return lib


def kernel_launches():
    """Kernels launched by the library so far in this process."""
    return int(load().ki_kernel_launches())


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _i(a):
    return None if a is None else a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _check(rc, what):
    if rc != 0:
        raise KiError("%s failed (%d): %s" % (what, rc, load().ki_last_error().decode()))


class _Tree:
    """Introspection shared by Solver and Partition."""

    def levels(self):
        return self.lib.ki_num_levels(self.h)

    def nodes(self, level):
        return self.lib.ki_num_boxes(self.h, level)

    def node(self, level, idx):
        info = np.zeros(8, dtype=np.int32)
        geom = np.zeros(3)
        _check(self.lib.ki_box_info(self.h, level, idx, _i(info), _d(geom)), "ki_box_info")
        lists = [np.zeros(int(n), dtype=np.int32) for n in info[2:6]]
        _check(self.lib.ki_box_lists(self.h, level, idx, *[_i(x) for x in lists]),
               "ki_box_lists")
        return {"is_leaf": bool(info[0]), "compressed": bool(info[1]),
                "parent": int(info[6]), "level": int(info[7]),
                "corner": (geom[0], geom[1]), "side": geom[2],
                "original": lists[0], "active": lists[1], "skel": lists[2],
                "redundant": lists[3]}

    def all_nodes(self):
        return [[self.node(l, i) for i in range(self.nodes(l))]
                for l in range(self.levels())]

    def close(self):
        if getattr(self, "h", None):
            self.lib.ki_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Partition(_Tree):
    """Quadtree only (host side, no GPU): QuadTree::initialize_tree."""

    def __init__(self, points, sol_dim, max_leaf_dofs):
        self.lib = load()
        pts = _f64(points)
        h = C.c_void_p()
        _check(self.lib.ki_partition(pts.size // 2, _d(pts), sol_dim, max_leaf_dofs,
                                     C.byref(h)), "ki_partition")
        self.h = h


class Solver(_Tree):
    """A factorization on the GPU (QuadTree + SkelFactorization)."""

    def __init__(self, problem, id_tol=None, max_leaf_dofs=None, stream=None, timed=False):
        self.lib = load()
        pr = problem
        self.problem = pr
        self._keep = [_f64(pr.points), _f64(pr.normals), _f64(pr.curvatures),
                      _f64(pr.weights), _f64(pr.holes).reshape(-1)]
        pts, nrm, kap, w, holes = self._keep
        tol = pr.id_tol if id_tol is None else id_tol
        leaf = pr.max_leaf_dofs if max_leaf_dofs is None else max_leaf_dofs
        h = C.c_void_p()
        fn = self.lib.ki_factor_timed if timed else self.lib.ki_factor
        _check(fn(pr.pde, pr.n_points, _d(pts), _d(nrm), _d(kap), _d(w),
                  pr.holes.shape[0], _d(holes) if holes.size else None, leaf, tol,
                  C.c_void_p(stream) if stream else None, C.byref(h)), "ki_factor")
        self.h = h
        self.n_dofs = self.lib.ki_num_dofs(h)
        self.n_border = self.lib.ki_num_border(h)

    def solve(self, f):
        f = _f64(f)
        mu = np.zeros(self.n_dofs)
        alpha = np.zeros(max(1, self.n_border))
        _check(self.lib.ki_solve(self.h, _d(f), _d(mu), _d(alpha) if self.n_border else None),
               "ki_solve")
        return mu, alpha[:self.n_border].copy()

    def solve_device(self, f_ptr, mu_ptr, alpha_ptr=None):
        _check(self.lib.ki_solve_device(self.h, C.c_void_p(f_ptr), C.c_void_p(mu_ptr),
                                        C.c_void_p(alpha_ptr) if alpha_ptr else None),
               "ki_solve_device")

    def apply_device(self, x_ptr, y_ptr):
        _check(self.lib.ki_apply_device(self.h, C.c_void_p(x_ptr), C.c_void_p(y_ptr)),
               "ki_apply_device")

    def eval_targets(self, targets, mu, alpha=None):
        targets = _f64(targets)
        nt = targets.size // 2
        out = np.zeros(nt * self.problem.sol_dim)
        al = _f64(alpha) if alpha is not None and len(alpha) else None
        _check(self.lib.ki_eval_targets(self.h, nt, _d(targets), _d(_f64(mu)), _d(al),
                                        _d(out)), "ki_eval_targets")
        return out

    def kernel_block(self, tgt, src):
        tgt = np.ascontiguousarray(tgt, dtype=np.int32)
        src = np.ascontiguousarray(src, dtype=np.int32)
        out = np.zeros(tgt.size * src.size)
        _check(self.lib.ki_kernel_block(self.h, tgt.size, _i(tgt), src.size, _i(src),
                                        _d(out)), "ki_kernel_block")
        return out.reshape(src.size, tgt.size).T

    def allskel(self):
        n = self.lib.ki_allskel(self.h, None)
        out = np.zeros(n, dtype=np.int32)
        self.lib.ki_allskel(self.h, _i(out))
        return out

    def stats(self):
        out = np.zeros(13)
        self.lib.ki_stats(self.h, _d(out), 13)
        return {"factor_ms": float(out[0]), "id_ms": float(out[1]),
                "id_launches": int(out[2]), "id_flops": float(out[3]),
                "id_bytes": float(out[4]), "decouple_ms": float(out[5]),
                "top_ms": float(out[6]), "wait_ms": float(out[7]),
                "host_prep_ms": float(out[8]), "host_post_ms": float(out[9]),
                "upload_ms": float(out[10]), "host_top_ms": float(out[11]),
                "id_fold_flops": float(out[12])}

    def launch_log(self):
        n = self.lib.ki_launch_log(self.h, None, 0)
        out = np.zeros(7 * max(n, 1))
        self.lib.ki_launch_log(self.h, _d(out), n)
        return out[:7 * n].reshape(n, 7)
