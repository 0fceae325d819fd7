"""The interpolative decomposition entry point that allocates no device
memory (ki_id_noalloc).

It exists for callers that cannot call cudaMalloc: their device memory is
owned by another allocator (a framework's caching allocator, or a pool
reserved up front) and a raw cudaMalloc/cudaFree would bypass it and
synchronise the device.  The box's working matrix then lives in the
library's static 8 MiB device array.  These checks compare it with the
existing entry point, ki_factor (whose per-box skeletons come back through
ki_box_lists and whose kernel entries come back through ki_kernel_block),
on two calls in a row, and check that calls too large for the static array
are refused with an error instead of being launched.  The file is named so
that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import ki_geometry as G
import kinterp

pytestmark = pytest.mark.gpu


def _nodes(pr):
    rec = np.zeros((pr.n_points, 8))
    rec[:, 0], rec[:, 1] = pr.points[0::2], pr.points[1::2]
    rec[:, 2], rec[:, 3] = pr.normals[0::2], pr.normals[1::2]
    rec[:, 4], rec[:, 5] = pr.weights, pr.curvatures
    return rec.ravel()


def _call(lib, pr, d_nodes, act, rows, tol, torch, circle=None):
    d_act = torch.tensor(act, dtype=torch.int32, device="cuda")
    d_rows = torch.tensor(rows, dtype=torch.int32, device="cuda")
    n = len(act)
    d_rank = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    d_perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_T = torch.zeros(n * n // 4 + 1, dtype=torch.float64, device="cuda")
    cx, cy, rad = circle if circle is not None else (0.0, 0.0, 0.0)
    torch.cuda.synchronize()
    rc = lib.ki_id_noalloc(pr.pde, C.c_void_p(d_nodes.data_ptr()), pr.n_points,
                           C.c_void_p(d_act.data_ptr()), n, C.c_void_p(d_rows.data_ptr()),
                           len(rows), 1 if circle is not None else 0, C.c_double(cx),
                           C.c_double(cy), C.c_double(rad),
                           C.c_double(tol), C.c_void_p(d_rank.data_ptr()),
                           C.c_void_p(d_perm.data_ptr()), C.c_void_p(d_T.data_ptr()), None)
    assert rc == 0, lib.ki_last_error()
    torch.cuda.synchronize()
    k = int(d_rank.item())
    return k, d_perm.cpu().numpy(), d_T.cpu().numpy()


def test_noalloc_id_matches_factor_on_two_calls():
    import torch
    lib = kinterp.load()
    lib.ki_id_noalloc.restype = C.c_int
    pr = G.star_case(n=4096, n_targets=16)
    s = kinterp.Solver(pr)  # the existing entry point
    d_nodes = torch.tensor(_nodes(pr), device="cuda", dtype=torch.float64)
    level1 = [s.node(1, i) for i in range(s.nodes(1))]
    calls = 0
    for idx, box in enumerate(level1):
        if not box["compressed"]:
            continue
        # level-1 ID rows: every other level-1 box's active dofs, both ways
        # (kernel.cpp:164-179)
        act = box["active"]
        rows = np.concatenate([o["active"] for j, o in enumerate(level1) if j != idx])
        k, perm, Tflat = _call(lib, pr, d_nodes, act, rows, pr.id_tol, torch)
        assert k == len(box["skel"])
        assert np.array_equal(act[perm[:k]], box["skel"])
        assert np.array_equal(np.sort(act[perm[k:]]), np.sort(box["redundant"]))
        # T against the ID matrix built from the existing entry point's kernel
        # blocks: A[:, redundant] = A[:, skeleton] T up to the ID tolerance
        A = np.vstack([s.kernel_block(rows, act), s.kernel_block(act, rows).T])
        T = Tflat[:k * (len(act) - k)].reshape(len(act) - k, k).T
        resid = A[:, perm[k:]] - A[:, perm[:k]] @ T
        assert np.linalg.norm(resid) <= 1e3 * pr.id_tol * np.linalg.norm(A)
        calls += 1
        if calls == 2:
            break
    assert calls == 2


def _proxy_rows(s, pr, level, idx, box):
    """The ID rows ki_factor uses for a box of level >= 3 (kernel.cpp:209-218):
    the dofs of its neighbours at this level or coarser (a leaf's original
    dofs, otherwise its active dofs) whose node lies inside the proxy circle
    of radius 1.5 side about the box centre, in neighbour-list order; and the
    circle (centre x, centre y, radius)."""
    side = box["side"]
    cx, cy = box["corner"][0] + side / 2.0, box["corner"][1] + side / 2.0
    R = 1.5 * side
    rows = []
    for ol, oi in s.neighbors(level, idx):
        if ol > level:
            continue
        o = s.node(ol, oi)
        for dof in (o["original"] if o["is_leaf"] else o["active"]):
            pt = dof // pr.sol_dim
            dx, dy = cx - pr.points[2 * pt], cy - pr.points[2 * pt + 1]
            if np.sqrt(dx * dx + dy * dy) < R:
                rows.append(dof)
    return np.array(rows, dtype=np.int32), (cx, cy, R)


@pytest.mark.parametrize("kind", ["laplace", "stokes"])
def test_noalloc_id_with_proxy_rows_matches_factor(kind):
    """Boxes of level >= 3 take the proxy-circle rows (256 for Laplace, 512
    for Stokes) besides their near rows: two such calls in a row must give
    ki_factor's rank and skeleton for the box, and a T that reproduces the
    redundant columns of the near-row block."""
    import torch
    lib = kinterp.load()
    lib.ki_id_noalloc.restype = C.c_int
    if kind == "laplace":
        pr = G.star_case(n=4096, n_targets=16)
    else:
        pr = G.stokes_holes_case(n_total=4096, n_targets=16)
    s = kinterp.Solver(pr)
    d_nodes = torch.tensor(_nodes(pr), device="cuda", dtype=torch.float64)
    calls = 0
    for level in range(3, s.levels()):
        for idx in range(s.nodes(level)):
            box = s.node(level, idx)
            if not box["compressed"] or len(box["active"]) < 24:
                continue
            act = box["active"]
            rows, circle = _proxy_rows(s, pr, level, idx, box)
            if len(rows) == 0:
                continue
            k, perm, Tflat = _call(lib, pr, d_nodes, act, rows, pr.id_tol, torch, circle)
            assert k == len(box["skel"]), (level, idx)
            assert np.array_equal(np.sort(act[perm[:k]]), np.sort(box["skel"])), (level, idx)
            assert np.array_equal(np.sort(act[perm[k:]]), np.sort(box["redundant"]))
            A = np.vstack([s.kernel_block(rows, act), s.kernel_block(act, rows).T])
            T = Tflat[:k * (len(act) - k)].reshape(len(act) - k, k).T
            resid = A[:, perm[k:]] - A[:, perm[:k]] @ T
            assert np.linalg.norm(resid) <= 1e3 * pr.id_tol * np.linalg.norm(A)
            calls += 1
            if calls == 2:
                return
    assert calls == 2


def test_noalloc_rejects_oversized_matrix():
    import torch
    lib = kinterp.load()
    lib.ki_last_error.restype = C.c_char_p
    pr = G.ellipse_case(n=1024)
    d_nodes = torch.tensor(_nodes(pr), device="cuda", dtype=torch.float64)
    act = torch.arange(1000, dtype=torch.int32, device="cuda")
    out = torch.zeros(1000 * 250 + 1, dtype=torch.float64, device="cuda")
    ints = torch.zeros(1001, dtype=torch.int32, device="cuda")
    rc = lib.ki_id_noalloc(pr.pde, C.c_void_p(d_nodes.data_ptr()), pr.n_points,
                           C.c_void_p(act.data_ptr()), 1000, C.c_void_p(act.data_ptr()), 1000,
                           0, C.c_double(0), C.c_double(0), C.c_double(0), C.c_double(1e-10),
                           C.c_void_p(ints.data_ptr()), C.c_void_p(ints.data_ptr() + 4),
                           C.c_void_p(out.data_ptr()), None)
    assert rc == 1
    assert b"8 MiB" in lib.ki_last_error()
