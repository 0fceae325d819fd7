"""ctypes bindings for the CPU checkers (test infrastructure only).

``RefSolver`` drives the reference solver compiled from its own sources
(oracle/_ref/libkiref.so, built by ``make -C oracle ref``).  ``PortSolver``
drives the CPU restatement in oracle/ki_oracle.cpp (oracle/libkioracle.so).
Only tests/, ``__graft_entry__.smoke`` and bench.py's CPU arms use these; the
product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libkiref.so")
PORT_SO = os.path.join(HERE, "libkioracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _i(a):
    return None if a is None else a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _Common:
    """Shared query surface of both CPU solvers."""

    def __init__(self, lib, prefix, problem, id_tol, max_leaf_dofs, threads):
        self.lib, self.p = lib, prefix
        self.problem = problem
        pr = problem
        self._keep = [_f64(pr.points), _f64(pr.normals), _f64(pr.curvatures),
                      _f64(pr.weights), _f64(pr.holes).reshape(-1)]
        pts, nrm, kap, w, holes = self._keep
        tf = C.c_double(0.0)
        fn = getattr(lib, prefix + "create")
        fn.restype = C.c_void_p
        fn.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_int, _dp,
                       C.c_int, C.c_double, C.c_int, _dp]
        self.h = fn(pr.pde, pr.n_points, _d(pts), _d(nrm), _d(kap), _d(w),
                    pr.holes.shape[0], _d(holes) if holes.size else None,
                    max_leaf_dofs, id_tol, threads, C.byref(tf))
        if not self.h:
            raise RuntimeError(prefix + "create failed")
        self.t_factor = tf.value
        self.n_dofs = pr.n_dofs

    def close(self):
        if self.h:
            getattr(self.lib, self.p + "destroy")(C.c_void_p(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, f):
        f = _f64(f)
        mu = np.zeros(self.n_dofs)
        alpha = np.zeros(max(1, 3 * self.problem.holes.shape[0]))
        ts = C.c_double(0.0)
        fn = getattr(self.lib, self.p + "solve")
        fn.restype = C.c_int
        fn.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        na = fn(C.c_void_p(self.h), _d(f), _d(mu), _d(alpha), C.byref(ts))
        self.t_solve = ts.value
        return mu, alpha[:na].copy()

    def levels(self):
        fn = getattr(self.lib, self.p + "num_levels")
        fn.restype = C.c_int
        return fn(C.c_void_p(self.h))

    def nodes(self, level):
        fn = getattr(self.lib, self.p + "num_nodes")
        fn.restype = C.c_int
        return fn(C.c_void_p(self.h), level)

    def node(self, level, idx):
        info = np.zeros(8, dtype=np.int32)
        geom = np.zeros(3)
        getattr(self.lib, self.p + "node_info")(
            C.c_void_p(self.h), level, idx, _i(info), _d(geom))
        lists = [np.zeros(int(n), dtype=np.int32) for n in info[2:6]]
        getattr(self.lib, self.p + "node_lists")(
            C.c_void_p(self.h), level, idx, *[_i(x) for x in lists])
        return {"is_leaf": bool(info[0]), "compressed": bool(info[1]),
                "parent": int(info[6]), "level": int(info[7]),
                "corner": (geom[0], geom[1]), "side": geom[2],
                "original": lists[0], "active": lists[1], "skel": lists[2],
                "redundant": lists[3]}

    def all_nodes(self):
        return [[self.node(l, i) for i in range(self.nodes(l))]
                for l in range(self.levels())]

    def allskel(self):
        fn = getattr(self.lib, self.p + "allskel")
        fn.restype = C.c_int
        n = fn(C.c_void_p(self.h), None)
        out = np.zeros(n, dtype=np.int32)
        fn(C.c_void_p(self.h), _i(out))
        return out

    def kernel_block(self, tgt, src):
        tgt = np.ascontiguousarray(tgt, dtype=np.int32)
        src = np.ascontiguousarray(src, dtype=np.int32)
        out = np.zeros(tgt.size * src.size)
        getattr(self.lib, self.p + "kernel_block")(
            C.c_void_p(self.h), tgt.size, _i(tgt), src.size, _i(src), _d(out))
        return out.reshape(src.size, tgt.size).T

    def eval_targets(self, targets, mu, alpha=None):
        targets = _f64(targets)
        nt = targets.size // 2
        out = np.zeros(nt * self.problem.sol_dim)
        getattr(self.lib, self.p + "eval_targets")(
            C.c_void_p(self.h), nt, _d(targets), _d(_f64(mu)),
            _d(_f64(alpha)) if alpha is not None and len(alpha) else None,
            _d(out))
        return out

    def border(self):
        fn = getattr(self.lib, self.p + "border")
        fn.restype = C.c_int
        cols = fn(C.c_void_p(self.h), None, None)
        if cols == 0:
            return None, None
        U = np.zeros(self.n_dofs * cols)
        Psi = np.zeros(self.n_dofs * cols)
        fn(C.c_void_p(self.h), _d(U), _d(Psi))
        return (U.reshape(cols, self.n_dofs).T.copy(),
                Psi.reshape(self.n_dofs, cols).T.copy())


_ref_lib = None
_port_lib = None


def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    """The reference library (loaded once)."""
    global _ref_lib
    if _ref_lib is None:
        _ref_lib = C.CDLL(REF_SO)
    return _ref_lib


class RefSolver(_Common):
    """The reference solver (oracle/_ref/libkiref.so)."""

    def __init__(self, problem, id_tol=None, max_leaf_dofs=None, threads=1):
        global _ref_lib
        if _ref_lib is None:
            _ref_lib = C.CDLL(REF_SO)
        super().__init__(_ref_lib, "kiref_", problem,
                         problem.id_tol if id_tol is None else id_tol,
                         problem.max_leaf_dofs if max_leaf_dofs is None
                         else max_leaf_dofs, threads)


def _ref_update(self, problem):
    """kiref_update: QuadTree::perturb + skeletonize on the reference."""
    pr = problem
    self.problem = pr
    self._keep = [_f64(pr.points), _f64(pr.normals), _f64(pr.curvatures),
                  _f64(pr.weights), _f64(pr.holes).reshape(-1)]
    pts, nrm, kap, w, holes = self._keep
    tf = C.c_double(0.0)
    fn = self.lib.kiref_update
    fn.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp]
    fn(C.c_void_p(self.h), pr.n_points, _d(pts), _d(nrm), _d(kap), _d(w), pr.holes.shape[0],
       _d(holes) if holes.size else None, C.byref(tf))
    self.t_factor = tf.value
    self.n_dofs = pr.n_dofs


def _ref_copy(self):
    """kiref_copy: QuadTree::copy_into + skeletonize on the reference."""
    fn = self.lib.kiref_copy
    fn.restype = C.c_void_p
    fn.argtypes = [C.c_void_p]
    c = RefSolver.__new__(RefSolver)
    c.lib, c.p, c.problem, c._keep = self.lib, self.p, self.problem, list(self._keep)
    c.h = fn(C.c_void_p(self.h))
    c.t_factor = 0.0
    c.n_dofs = self.n_dofs
    return c


RefSolver.update = _ref_update
RefSolver.copy = _ref_copy


class PortSolver(_Common):
    """The CPU restatement (oracle/libkioracle.so)."""

    def __init__(self, problem, id_tol=None, max_leaf_dofs=None, threads=1):
        global _port_lib
        if _port_lib is None:
            _port_lib = C.CDLL(PORT_SO)
        super().__init__(_port_lib, "kiora_", problem,
                         problem.id_tol if id_tol is None else id_tol,
                         problem.max_leaf_dofs if max_leaf_dofs is None
                         else max_leaf_dofs, threads)
