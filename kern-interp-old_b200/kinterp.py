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
    lib.ki_partition_batch.argtypes = [C.c_int, _ip, _dp, C.c_int, C.c_int,
                                       C.POINTER(C.c_void_p)]
    lib.ki_factor_batch.argtypes = [C.c_int, C.c_int, _ip, _dp, _dp, _dp, _dp, C.c_int,
                                    C.c_double, C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]
    lib.ki_factor_ex.argtypes = fac_args[:10] + [C.c_int, C.c_int] + fac_args[10:]
    lib.ki_num_problems.argtypes = [C.c_void_p]
    lib.ki_box_tree.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.ki_destroy.argtypes = [C.c_void_p]
    lib.ki_destroy.restype = None
    for name in ("ki_num_dofs", "ki_num_border", "ki_num_levels"):
        getattr(lib, name).argtypes = [C.c_void_p]
    lib.ki_num_boxes.argtypes = [C.c_void_p, C.c_int]
    lib.ki_solve.argtypes = [C.c_void_p, _dp, _dp, _dp]
    lib.ki_solve_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ki_apply_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ki_solve_bordered_device.argtypes = [C.c_void_p] + [C.c_void_p] * 4
    lib.ki_solve_transpose_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ki_eval_targets_device.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 4
    lib.ki_adjoint_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_void_p]
    lib.ki_adjoint_backward.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 8
    lib.ki_matvec_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ki_matvec_correction_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]
    lib.ki_solve_refined.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_double, C.c_int, _ip, _dp]
    lib.ki_solve_refined_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_double, C.c_int, _ip, _dp]
    lib.ki_eval_targets.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]
    lib.ki_partition_update.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.ki_update.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, C.c_int, _dp, _ip]
    lib.ki_copy.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]
    lib.ki_eval_domain.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, C.c_int, _dp, _dp]
    lib.ki_eval_domain_device.argtypes = ([C.c_void_p, C.c_int] + [C.c_void_p] * 3 +
                                          [C.c_int, _dp, C.c_void_p])
    lib.ki_domain_mask_device.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, _dp,
                                          C.c_void_p]
    lib.ki_domain_points.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                     _dp]
    lib.ki_kernel_block.argtypes = [C.c_void_p, C.c_int, _ip, C.c_int, _ip, _dp]
    lib.ki_box_info.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _dp]
    lib.ki_box_lists.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip, _ip, _ip]
    lib.ki_allskel.argtypes = [C.c_void_p, _ip]
    lib.ki_box_neighbors.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip]
    lib.ki_stats.argtypes = [C.c_void_p, _dp, C.c_int]
    lib.ki_launch_log.argtypes = [C.c_void_p, _dp, C.c_int]
    lib.ki_timeline.argtypes = [C.c_void_p, _dp, C.c_int]
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


DOMAIN_KINDS = {"all": 0, "nodes": 1, "disk": 2}


def _domain(kind, disk):
    k = DOMAIN_KINDS[kind]
    dk = None
    if k == 2:
        if disk is None:
            raise ValueError("the disk test needs disk=(cx, cy, R)")
        dk = np.ascontiguousarray(disk, dtype=np.float64)
    return k, dk


def domain_points(domain_size, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0):
    """get_domain_points (linear_solve.cpp:183-193): a domain_size^2 grid,
    x in the outer loop, interleaved xy."""
    out = np.zeros(2 * domain_size * domain_size)
    _check(load().ki_domain_points(domain_size, x_min, x_max, y_min, y_max, _d(out)),
           "ki_domain_points")
    return out


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
                "redundant": lists[3], "tree": int(self.lib.ki_box_tree(self.h, level, idx))}

    def neighbors(self, level, idx):
        """(level, index) of each neighbour of box idx of `level`, in the
        reference's neighbour-list order."""
        n = self.lib.ki_box_neighbors(self.h, level, idx, None, None)
        if n < 0:
            _check(-n, "ki_box_neighbors")
        lv = np.zeros(max(n, 1), dtype=np.int32)
        ix = np.zeros(max(n, 1), dtype=np.int32)
        self.lib.ki_box_neighbors(self.h, level, idx, _i(lv), _i(ix))
        return list(zip(lv[:n].tolist(), ix[:n].tolist()))

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

    def update(self, points):
        """The partition half of QuadTree::perturb (ki_partition_update)."""
        pts = _f64(points)
        _check(self.lib.ki_partition_update(self.h, pts.size // 2, _d(pts)),
               "ki_partition_update")


class Solver(_Tree):
    """A factorization on the GPU (QuadTree + SkelFactorization)."""

    def __init__(self, problem, id_tol=None, max_leaf_dofs=None, stream=None, timed=False,
                 mode=0):
        """mode 0 (KI_MODE_REFERENCE): the reference's factorization; mode 1
        (KI_MODE_PRECONDITIONER): for use with solve_refined."""
        self.lib = load()
        pr = problem
        self.problem = pr
        self._keep = [_f64(pr.points), _f64(pr.normals), _f64(pr.curvatures),
                      _f64(pr.weights), _f64(pr.holes).reshape(-1)]
        pts, nrm, kap, w, holes = self._keep
        tol = pr.id_tol if id_tol is None else id_tol
        leaf = pr.max_leaf_dofs if max_leaf_dofs is None else max_leaf_dofs
        h = C.c_void_p()
        _check(self.lib.ki_factor_ex(pr.pde, pr.n_points, _d(pts), _d(nrm), _d(kap), _d(w),
                                     pr.holes.shape[0], _d(holes) if holes.size else None, leaf,
                                     tol, mode, 1 if timed else 0,
                                     C.c_void_p(stream) if stream else None, C.byref(h)),
               "ki_factor")
        self.h = h
        self.n_dofs = self.lib.ki_num_dofs(h)
        self.n_border = self.lib.ki_num_border(h)

    def update(self, problem):
        """QuadTree::perturb + skeletonize (ki_update): follow the boundary to
        `problem`'s geometry, keeping the factors of untouched boxes.
        Returns the number of boxes kept."""
        pr = problem
        self.problem = pr
        self._keep = [_f64(pr.points), _f64(pr.normals), _f64(pr.curvatures),
                      _f64(pr.weights), _f64(pr.holes).reshape(-1)]
        pts, nrm, kap, w, holes = self._keep
        kept = np.zeros(1, dtype=np.int32)
        _check(self.lib.ki_update(self.h, pr.n_points, _d(pts), _d(nrm), _d(kap), _d(w),
                                  pr.holes.shape[0], _d(holes) if holes.size else None,
                                  _i(kept)), "ki_update")
        self.n_dofs = self.lib.ki_num_dofs(self.h)
        self.n_border = self.lib.ki_num_border(self.h)
        return int(kept[0])

    def copy(self, stream=None):
        """QuadTree::copy_into + skeletonize (ki_copy): an independent handle."""
        h = C.c_void_p()
        _check(self.lib.ki_copy(self.h, C.c_void_p(stream) if stream else None, C.byref(h)),
               "ki_copy")
        c = Solver.__new__(Solver)
        c.lib, c.problem, c._keep, c.h = self.lib, self.problem, list(self._keep), h
        c.n_dofs, c.n_border = self.n_dofs, self.n_border
        return c

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

    def solve_bordered_device(self, f_ptr, g_ptr, mu_ptr, alpha_ptr):
        _check(self.lib.ki_solve_bordered_device(self.h, C.c_void_p(f_ptr),
                                                 C.c_void_p(g_ptr) if g_ptr else None,
                                                 C.c_void_p(mu_ptr),
                                                 C.c_void_p(alpha_ptr) if alpha_ptr else None),
               "ki_solve_bordered_device")

    def solve_transpose_device(self, b_ptr, x_ptr):
        _check(self.lib.ki_solve_transpose_device(self.h, C.c_void_p(b_ptr), C.c_void_p(x_ptr)),
               "ki_solve_transpose_device")

    def eval_targets_device(self, n_targets, tg_ptr, mu_ptr, alpha_ptr, out_ptr):
        _check(self.lib.ki_eval_targets_device(self.h, n_targets, C.c_void_p(tg_ptr),
                                               C.c_void_p(mu_ptr),
                                               C.c_void_p(alpha_ptr) if alpha_ptr else None,
                                               C.c_void_p(out_ptr)), "ki_eval_targets_device")

    def adjoint_forward(self, f_ptr, n_targets, tg_ptr, mu_ptr, u_ptr):
        _check(self.lib.ki_adjoint_forward(self.h, C.c_void_p(f_ptr), n_targets,
                                           C.c_void_p(tg_ptr), C.c_void_p(mu_ptr),
                                           C.c_void_p(u_ptr)), "ki_adjoint_forward")

    def adjoint_backward(self, n_targets, tg_ptr, mu_ptr, gu_ptr, gf_ptr, gp_ptr, gn_ptr, gw_ptr,
                         gk_ptr):
        _check(self.lib.ki_adjoint_backward(self.h, n_targets, C.c_void_p(tg_ptr),
                                            C.c_void_p(mu_ptr), C.c_void_p(gu_ptr),
                                            C.c_void_p(gf_ptr), C.c_void_p(gp_ptr),
                                            C.c_void_p(gn_ptr), C.c_void_p(gw_ptr),
                                            C.c_void_p(gk_ptr)), "ki_adjoint_backward")

    def matvec_device(self, x_ptr, y_ptr):
        _check(self.lib.ki_matvec_device(self.h, C.c_void_p(x_ptr), C.c_void_p(y_ptr)),
               "ki_matvec_device")

    def matvec_correction_device(self, x_ptr, y_ptr, dscale=1.0):
        _check(self.lib.ki_matvec_correction_device(self.h, C.c_void_p(x_ptr), C.c_void_p(y_ptr),
                                                    dscale), "ki_matvec_correction_device")

    def solve_refined(self, f, rel_tol=1e-12, max_iters=20):
        """FP64 GMRES refinement preconditioned by this factorization.
        Returns (mu, alpha, iterations, final true relative residual)."""
        f = _f64(f)
        mu = np.zeros(self.n_dofs)
        alpha = np.zeros(max(1, self.n_border))
        it = np.zeros(1, dtype=np.int32)
        rr = np.zeros(1)
        _check(self.lib.ki_solve_refined(self.h, _d(f), _d(mu),
                                         _d(alpha) if self.n_border else None, rel_tol,
                                         max_iters, _i(it), _d(rr)), "ki_solve_refined")
        return mu, alpha[:self.n_border].copy(), int(it[0]), float(rr[0])

    def solve_refined_device(self, f_ptr, mu_ptr, alpha_ptr=None, rel_tol=1e-12, max_iters=20):
        it = np.zeros(1, dtype=np.int32)
        rr = np.zeros(1)
        _check(self.lib.ki_solve_refined_device(self.h, C.c_void_p(f_ptr), C.c_void_p(mu_ptr),
                                                C.c_void_p(alpha_ptr) if alpha_ptr else None,
                                                rel_tol, max_iters, _i(it), _d(rr)),
               "ki_solve_refined_device")
        return int(it[0]), float(rr[0])

    def eval_targets(self, targets, mu, alpha=None):
        targets = _f64(targets)
        nt = targets.size // 2
        out = np.zeros(nt * self.problem.sol_dim)
        al = _f64(alpha) if alpha is not None and len(alpha) else None
        _check(self.lib.ki_eval_targets(self.h, nt, _d(targets), _d(_f64(mu)), _d(al),
                                        _d(out)), "ki_eval_targets")
        return out

    def eval_domain(self, targets, mu, alpha=None, domain="nodes", disk=None):
        """boundary_integral_solve's evaluation (linear_solve.cpp:142-180):
        the solution at the points, zero outside the domain.  domain:
        "nodes" (CubicBoundary::is_in_domain on the node curves), "disk"
        (Circle / Annulus / Donut::is_in_domain with disk = (cx, cy, R)) or
        "all" (no test)."""
        k, dk = _domain(domain, disk)
        targets = _f64(targets)
        nt = targets.size // 2
        out = np.zeros(nt * self.problem.sol_dim)
        al = _f64(alpha) if alpha is not None and len(alpha) else None
        _check(self.lib.ki_eval_domain(self.h, nt, _d(targets), _d(_f64(mu)), _d(al), k, _d(dk),
                                       _d(out)), "ki_eval_domain")
        return out

    def eval_domain_device(self, n_targets, tg_ptr, mu_ptr, alpha_ptr, out_ptr, domain="nodes",
                           disk=None):
        k, dk = _domain(domain, disk)
        _check(self.lib.ki_eval_domain_device(self.h, n_targets, C.c_void_p(tg_ptr),
                                              C.c_void_p(mu_ptr),
                                              C.c_void_p(alpha_ptr) if alpha_ptr else None, k,
                                              _d(dk), C.c_void_p(out_ptr)),
               "ki_eval_domain_device")

    def domain_mask_device(self, n_targets, tg_ptr, mask_ptr, domain="nodes", disk=None):
        k, dk = _domain(domain, disk)
        _check(self.lib.ki_domain_mask_device(self.h, n_targets, C.c_void_p(tg_ptr), k, _d(dk),
                                              C.c_void_p(mask_ptr)), "ki_domain_mask_device")

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
        out = np.zeros(17)
        self.lib.ki_stats(self.h, _d(out), 17)
        return {"factor_ms": float(out[0]), "id_ms": float(out[1]),
                "id_launches": int(out[2]), "id_flops": float(out[3]),
                "id_bytes": float(out[4]), "decouple_ms": float(out[5]),
                "top_ms": float(out[6]), "wait_ms": float(out[7]),
                "host_prep_ms": float(out[8]), "host_post_ms": float(out[9]),
                "upload_ms": float(out[10]), "host_top_ms": float(out[11]),
                "id_onchip_flops": float(out[12]), "staging_bytes": float(out[13]),
                "dec_flops": float(out[14]), "top_flops": float(out[15]),
                "solve_bytes": float(out[16])}

    def timeline(self):
        n = self.lib.ki_timeline(self.h, None, 0)
        out = np.zeros(4 * max(n, 1))
        self.lib.ki_timeline(self.h, _d(out), n)
        return out[:4 * n].reshape(n, 4)

    def launch_log(self):
        n = self.lib.ki_launch_log(self.h, None, 0)
        out = np.zeros(7 * max(n, 1))
        self.lib.ki_launch_log(self.h, _d(out), n)
        return out[:7 * n].reshape(n, 7)


def _concat(problems):
    n = np.array([p.n_points for p in problems], dtype=np.int32)
    cat = lambda name: np.ascontiguousarray(np.concatenate([getattr(p, name) for p in problems]),
                                            dtype=np.float64)
    return n, cat("points"), cat("normals"), cat("curvatures"), cat("weights")


class BatchPartition(_Tree):
    """The host partition of many problems (one quadtree each)."""

    def __init__(self, problems, max_leaf_dofs=None):
        self.lib = load()
        pr0 = problems[0]
        leaf = pr0.max_leaf_dofs if max_leaf_dofs is None else max_leaf_dofs
        self._n, pts, _, _, _ = _concat(problems)
        self._keep = [pts]
        h = C.c_void_p()
        _check(self.lib.ki_partition_batch(len(problems), _i(self._n), _d(pts), pr0.sol_dim, leaf,
                                           C.byref(h)), "ki_partition_batch")
        self.h = h


class BatchSolver(_Tree):
    """Many independent problems factored together (ki_factor_batch): dofs
    of problem p follow those of problems 0..p-1."""

    def __init__(self, problems, id_tol=None, max_leaf_dofs=None, stream=None, mode=0):
        self.lib = load()
        pr0 = problems[0]
        self.problems = problems
        self._n, pts, nrm, kap, w = _concat(problems)
        self._keep = [pts, nrm, kap, w]
        tol = pr0.id_tol if id_tol is None else id_tol
        leaf = pr0.max_leaf_dofs if max_leaf_dofs is None else max_leaf_dofs
        h = C.c_void_p()
        _check(self.lib.ki_factor_batch(pr0.pde, len(problems), _i(self._n), _d(pts), _d(nrm),
                                        _d(kap), _d(w), leaf, tol, mode,
                                        C.c_void_p(stream) if stream else None, C.byref(h)),
               "ki_factor_batch")
        self.h = h
        self.n_dofs = self.lib.ki_num_dofs(h)
        sd = pr0.sol_dim
        self.offsets = np.concatenate([[0], np.cumsum(self._n * sd)]).astype(np.int64)

    def split(self, x):
        return [x[self.offsets[p]:self.offsets[p + 1]] for p in range(len(self.problems))]

    def solve(self, f=None):
        f = _f64(np.concatenate([p.f for p in self.problems]) if f is None else f)
        mu = np.zeros(self.n_dofs)
        _check(self.lib.ki_solve(self.h, _d(f), _d(mu), None), "ki_solve")
        return mu

    def solve_device(self, f_ptr, mu_ptr):
        _check(self.lib.ki_solve_device(self.h, C.c_void_p(f_ptr), C.c_void_p(mu_ptr), None),
               "ki_solve_device")

    def solve_refined(self, f=None, rel_tol=1e-12, max_iters=20):
        f = _f64(np.concatenate([p.f for p in self.problems]) if f is None else f)
        mu = np.zeros(self.n_dofs)
        it = np.zeros(1, dtype=np.int32)
        rr = np.zeros(1)
        _check(self.lib.ki_solve_refined(self.h, _d(f), _d(mu), None, rel_tol, max_iters,
                                         _i(it), _d(rr)), "ki_solve_refined")
        return mu, int(it[0]), float(rr[0])

    def solve_refined_device(self, f_ptr, mu_ptr, rel_tol=1e-12, max_iters=20):
        it = np.zeros(1, dtype=np.int32)
        rr = np.zeros(1)
        _check(self.lib.ki_solve_refined_device(self.h, C.c_void_p(f_ptr), C.c_void_p(mu_ptr),
                                                None, rel_tol, max_iters, _i(it), _d(rr)),
               "ki_solve_refined_device")
        return int(it[0]), float(rr[0])

    def apply_device(self, x_ptr, y_ptr):
        _check(self.lib.ki_apply_device(self.h, C.c_void_p(x_ptr), C.c_void_p(y_ptr)),
               "ki_apply_device")

    def stats(self):
        return Solver.stats(self)


def tune_id_tol(problem, candidates=(1e-6, 3e-7, 1e-7, 3e-8, 1e-8), rel_tol=1e-12,
                max_iters=20, reps=3, stream=None):
    """Autotuner for the mixed method: the preconditioner's ID tolerance
    trades factorization time (tighter: higher ranks) against refinement
    steps (looser: more of them).  Times factor + refinement for each
    candidate (host wall clock around the public calls, which synchronise:
    the best of `reps` after one untimed run) and returns (best_tol, table),
    table = [(tol, seconds, iterations, residual)].  Candidates whose
    refinement does not reach rel_tol are skipped."""
    import time
    table = []
    for tol in candidates:
        best, it, rr = None, None, None
        for rep in range(reps + 1):
            t0 = time.perf_counter()
            s = Solver(problem, id_tol=tol, stream=stream, mode=1)
            _, _, it, rr = s.solve_refined(problem.f, rel_tol=rel_tol, max_iters=max_iters)
            dt = time.perf_counter() - t0
            s.close()
            if rep > 0 and (best is None or dt < best):
                best = dt
        if rr <= rel_tol:
            table.append((tol, best, it, rr))
    if not table:
        raise KiError("tune_id_tol: no candidate tolerance reached the refinement target")
    return min(table, key=lambda row: row[1])[0], table


def boundary_integral_solve(problem, domain_pts, id_tol=None, max_leaf_dofs=None,
                            domain="nodes", disk=None):
    """boundary_integral_solve (linear_solve.cpp:142-180): factor the
    problem's boundary operator, solve for mu (and alpha with holes) with the
    problem's boundary data, and return the solution at domain_pts
    (interleaved xy), zero outside the domain (see Solver.eval_domain)."""
    s = Solver(problem, id_tol=id_tol, max_leaf_dofs=max_leaf_dofs)
    try:
        mu, alpha = s.solve(problem.f)
        return s.eval_domain(domain_pts, mu, alpha if s.n_border else None, domain, disk)
    finally:
        s.close()
