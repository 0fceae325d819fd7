"""CPU restatement of the reference's domain tests and grid (test
infrastructure only; the product never imports this module).

* ``in_domain_nodes``: CubicBoundary::is_in_domain
  (kern_interp/boundaries/cubic_boundary.cpp:182-230) on node curves, outer
  nodes first, then each hole's nodes.
* ``in_domain_disk``: Circle / Annulus / Donut::is_in_domain
  (circle.cpp:34-42, annulus.cpp:66-79, donut.cpp:67-80) for a disk
  (cx, cy, R) with holes.
* ``domain_points``: get_domain_points (linear_solve.cpp:183-193).
* ``ref_in_domain`` / ``ref_domain_points``: the same functions of the
  reference compiled from its own sources (oracle/_ref/libkiref.so), used to
  pin the restatement.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

EPS = 1e-2  # cubic_boundary.cpp:185, circle.cpp:37, annulus.cpp:69


def _near(tx, ty, px, py):
    """sqrt((t - p)_x^2 + (t - p)_y^2) < eps for every (target, node) pair of
    the given blocks, rounded as the reference's doubles."""
    dx = tx[:, None] - px[None, :]
    dy = ty[:, None] - py[None, :]
    return (np.sqrt(dx * dx + dy * dy) < EPS).any(axis=1)


def _crossings(tx, ty, px, py, pyn):
    """Signed crossing count of cubic_boundary.cpp:193-199: for node i right
    of the point (x_i > x), +1 when y_i < y < y_next, -1 when y_i > y > y_next."""
    right = px[None, :] > tx[:, None]
    up = (py[None, :] < ty[:, None]) & (pyn[None, :] > ty[:, None])
    down = (py[None, :] > ty[:, None]) & (pyn[None, :] < ty[:, None])
    return (right & up).sum(1) - (right & down).sum(1)


def _c_mod2(w):
    """C's w % 2 (sign of the dividend)."""
    return np.fmod(w, 2)


def in_domain_nodes(points, holes, targets, block=2048):
    """CubicBoundary::is_in_domain for every target; returns uint8 1 inside."""
    p = np.asarray(points, dtype=np.float64).reshape(-1, 2)
    t = np.asarray(targets, dtype=np.float64).reshape(-1, 2)
    holes = np.asarray(holes, dtype=np.float64).reshape(-1, 4)
    n = p.shape[0]
    counts = [int(h[3]) for h in holes]
    outer = n - sum(counts)
    curves = [(0, outer, True)]
    start = outer
    for c in counts:
        curves.append((start, start + c, False))
        start += c
    out = np.ones(t.shape[0], dtype=np.uint8)
    for b0 in range(0, t.shape[0], block):
        tx, ty = t[b0:b0 + block, 0], t[b0:b0 + block, 1]
        bad = np.zeros(tx.size, dtype=bool)
        for c0, c1, is_outer in curves:
            px, py = p[c0:c1, 0], p[c0:c1, 1]
            pyn = np.roll(py, -1)
            bad |= _near(tx, ty, px, py)
            w = _c_mod2(_crossings(tx, ty, px, py, pyn))
            bad |= (w == 0) if is_outer else (w == 1)
        out[b0:b0 + block][bad] = 0
    return out


def in_domain_disk(cx, cy, R, holes, targets):
    """Circle / Annulus / Donut::is_in_domain; returns uint8 1 inside."""
    t = np.asarray(targets, dtype=np.float64).reshape(-1, 2)
    holes = np.asarray(holes, dtype=np.float64).reshape(-1, 4)
    x, y = t[:, 0] - cx, t[:, 1] - cy
    bad = np.sqrt(x * x + y * y) + EPS > R
    for h in holes:
        rx, ry = t[:, 0] - h[0], t[:, 1] - h[1]
        bad |= np.sqrt(rx * rx + ry * ry) - EPS < h[2]
    return (~bad).astype(np.uint8)


def domain_points(domain_size, x_min, x_max, y_min, y_max):
    """get_domain_points: x in the outer loop, interleaved xy."""
    i = np.arange(domain_size, dtype=np.float64)
    xs = x_min + (i / (domain_size - 1)) * (x_max - x_min)
    ys = y_min + (i / (domain_size - 1)) * (y_max - y_min)
    out = np.empty((domain_size, domain_size, 2))
    out[:, :, 0] = xs[:, None]
    out[:, :, 1] = ys[None, :]
    return out.reshape(-1)


REF_KINDS = {"nodes": 0, "circle": 1, "annulus": 2, "donut": 3}


def ref_in_domain(kind, points, holes, targets):
    """The reference's own is_in_domain (kind: nodes, circle, annulus, donut)."""
    import kioracle
    lib = kioracle.ref_lib()
    p = np.ascontiguousarray(points, dtype=np.float64)
    h = np.ascontiguousarray(holes, dtype=np.float64).reshape(-1)
    t = np.ascontiguousarray(targets, dtype=np.float64)
    out = np.zeros(t.size // 2, dtype=np.uint8)
    dp = C.POINTER(C.c_double)
    lib.kiref_in_domain(REF_KINDS[kind], p.size // 2, p.ctypes.data_as(dp), h.size // 4,
                        h.ctypes.data_as(dp) if h.size else None, t.size // 2,
                        t.ctypes.data_as(dp), out.ctypes.data_as(C.POINTER(C.c_ubyte)))
    return out


def ref_domain_points(domain_size, x_min, x_max, y_min, y_max):
    import kioracle
    lib = kioracle.ref_lib()
    out = np.zeros(2 * domain_size * domain_size)
    lib.kiref_domain_points(domain_size, C.c_double(x_min), C.c_double(x_max),
                            C.c_double(y_min), C.c_double(y_max),
                            out.ctypes.data_as(C.POINTER(C.c_double)))
    return out
