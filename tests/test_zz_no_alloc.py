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


def _call(lib, pr, d_nodes, act, rows, tol, torch):
    d_act = torch.tensor(act, dtype=torch.int32, device="cuda")
    d_rows = torch.tensor(rows, dtype=torch.int32, device="cuda")
    n = len(act)
    d_rank = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    d_perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_T = torch.zeros(n * n // 4 + 1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.ki_id_noalloc(pr.pde, C.c_void_p(d_nodes.data_ptr()), pr.n_points,
                           C.c_void_p(d_act.data_ptr()), n, C.c_void_p(d_rows.data_ptr()),
                           len(rows), 0, C.c_double(0.0), C.c_double(0.0), C.c_double(0.0),
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
