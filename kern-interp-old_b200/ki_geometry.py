"""Boundary geometries and boundary data for the solver's workloads.

Every boundary is returned as the arrays the reference's ``Boundary`` class
carries (kern_interp/boundaries/boundary.h:35-51): ``points`` and ``normals``
interleaved xy (2N), ``curvatures`` (N), ``weights`` (N), plus ``holes`` as
rows (cx, cy, radius, num_nodes).  Conventions follow the reference shapes:
the outer curve runs counter-clockwise with the outward normal and positive
curvature on convex parts (circle.cpp:13-23); hole nodes carry the normal
pointing into the hole and curvature -1/r (annulus.cpp:37-51).  Quadrature is
the trapezoid rule in the curve parameter, weight = |gamma'(theta)| 2 pi / N.

Workloads (all seeded with numpy's PCG64 ``default_rng``):
  * ``ellipse_case``      -- Laplace, ellipse (1.0, 0.6), N=1024, 4 sources at
                             radius 2.5, 100 interior targets.
  * ``star_case``         -- Laplace, r = 1 + 0.3 cos 5t, N=16384, 8 sources at
                             radius 2.0, 256 interior targets.
  * ``stokes_holes_case`` -- Stokes, unit disk with 8 circular holes of radius
                             0.05-0.15, 32768 nodes split by perimeter, 6
                             exterior Stokeslets.
  * ``random_star_cases`` -- 256 random stars, N log-uniform in [512, 8192].
  * ``fourier_star_case`` -- star with 32 Fourier shape coefficients, N=8192,
                             64 targets.
The reference's own test shapes (circle, annulus, donut, cubic-spline
starfish) are restated in ``reference_shape`` for the parity fixtures.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

LAPLACE, LAPLACE_NEUMANN, STOKES = 0, 1, 2


@dataclass
class Problem:
    """One boundary integral problem: geometry, data and evaluation targets."""

    name: str
    pde: int
    points: np.ndarray
    normals: np.ndarray
    curvatures: np.ndarray
    weights: np.ndarray
    holes: np.ndarray  # (n_holes, 4): cx, cy, radius, num_nodes
    f: np.ndarray  # boundary data, N (Laplace) or 2N (Stokes) entries
    targets: np.ndarray  # (n_targets * 2,) interleaved xy, inside the domain
    exact: np.ndarray  # exact solution at the targets (analytic check)
    leaf_points: int = 64
    id_tol: float = 1e-10
    extra: dict = field(default_factory=dict)

    @property
    def n_points(self) -> int:
        return self.weights.shape[0]

    @property
    def sol_dim(self) -> int:
        return 2 if self.pde == STOKES else 1

    @property
    def n_dofs(self) -> int:
        return self.n_points * self.sol_dim

    @property
    def max_leaf_dofs(self) -> int:
        return self.leaf_points * self.sol_dim


# --------------------------------------------------------------------------
# curve samplers


def _radial_curve(r, dr, ddr, n, center=(0.0, 0.0)):
    """Samples a star-shaped curve x = c + r(t)(cos t, sin t) at t = 2 pi j/n."""
    t = 2.0 * np.pi * np.arange(n) / n
    rt, drt, ddrt = r(t), dr(t), ddr(t)
    c, s = np.cos(t), np.sin(t)
    x = center[0] + rt * c
    y = center[1] + rt * s
    xp = drt * c - rt * s
    yp = drt * s + rt * c
    xpp = ddrt * c - 2.0 * drt * s - rt * c
    ypp = ddrt * s + 2.0 * drt * c - rt * s
    speed = np.sqrt(xp * xp + yp * yp)
    kappa = (xp * ypp - yp * xpp) / speed**3
    nx, ny = yp / speed, -xp / speed
    w = speed * (2.0 * np.pi / n)
    return x, y, nx, ny, kappa, w


def _pack(parts):
    xs, ys, nxs, nys, ks, ws = (np.concatenate(a) for a in zip(*parts))
    pts = np.empty(2 * xs.size)
    pts[0::2], pts[1::2] = xs, ys
    nrm = np.empty(2 * xs.size)
    nrm[0::2], nrm[1::2] = nxs, nys
    return pts, nrm, ks, ws


def _circle(cx, cy, rad, n, inward=False):
    t = 2.0 * np.pi * np.arange(n) / n
    c, s = np.cos(t), np.sin(t)
    sign = -1.0 if inward else 1.0
    return (cx + rad * c, cy + rad * s, sign * c, sign * s,
            np.full(n, sign / rad), np.full(n, 2.0 * np.pi * rad / n))


# --------------------------------------------------------------------------
# boundary data and exact solutions


def laplace_sources(rng, k, radius):
    ang = rng.uniform(0.0, 2.0 * np.pi, k)
    src = np.stack([radius * np.cos(ang), radius * np.sin(ang)], axis=1)
    q = rng.standard_normal(k)
    return src, q


def laplace_potential(xy, src, q):
    """u(x) = sum_s q_s log|x - y_s| / (2 pi) (same form as boundary.cpp:49-54)."""
    xy = xy.reshape(-1, 2)
    d = xy[:, None, :] - src[None, :, :]
    return (np.log(np.sqrt((d * d).sum(-1))) * q[None, :]).sum(1) / (2 * np.pi)


def stokeslet_velocity(xy, src, force):
    """u(x) = sum_s G(x - y_s) F_s, G = (-log r I + r r^T / r^2) / (4 pi),
    the Stokeslet of linear_solve.cpp:41-51."""
    xy = xy.reshape(-1, 2)
    out = np.zeros_like(xy)
    for (sx, sy), (fx, fy) in zip(src, force):
        rx, ry = xy[:, 0] - sx, xy[:, 1] - sy
        r2 = rx * rx + ry * ry
        lg = -0.5 * np.log(r2)
        out[:, 0] += (lg * fx + (rx * rx * fx + rx * ry * fy) / r2) / (4 * np.pi)
        out[:, 1] += (lg * fy + (rx * ry * fx + ry * ry * fy) / r2) / (4 * np.pi)
    return out.reshape(-1)


def _targets_in(rng, n, inside, box):
    out = []
    while len(out) < n:
        p = rng.uniform(box[0], box[1], size=(4 * n, 2))
        keep = p[inside(p)]
        out.extend(keep.tolist())
    return np.asarray(out[:n]).reshape(-1)


# --------------------------------------------------------------------------
# workloads


def ellipse_case(n=1024, seed=1, a=1.0, b=0.6, leaf_points=64, id_tol=1e-10):
    rng = np.random.default_rng(seed)
    t = 2.0 * np.pi * np.arange(n) / n
    c, s = np.cos(t), np.sin(t)
    xp, yp = -a * s, b * c
    speed = np.sqrt(xp * xp + yp * yp)
    parts = [(a * c, b * s, yp / speed, -xp / speed, a * b / speed**3,
              speed * 2.0 * np.pi / n)]
    pts, nrm, kap, w = _pack(parts)
    src, q = laplace_sources(rng, 4, 2.5)
    f = laplace_potential(pts, src, q)
    tg = _targets_in(rng, 100,
                     lambda p: (p[:, 0] / (0.8 * a))**2 + (p[:, 1] / (0.8 * b))**2 < 1,
                     (-a, a))
    return Problem("ellipse_laplace_n%d" % n, LAPLACE, pts, nrm, kap, w,
                   np.zeros((0, 4)), f, tg, laplace_potential(tg, src, q),
                   leaf_points, id_tol, {"sources": src, "strengths": q})


def _star_r(amp, k):
    return (lambda t: 1.0 + amp * np.cos(k * t),
            lambda t: -amp * k * np.sin(k * t),
            lambda t: -amp * k * k * np.cos(k * t))


def star_case(n=16384, seed=2, leaf_points=64, id_tol=1e-10, n_targets=256):
    rng = np.random.default_rng(seed)
    r, dr, ddr = _star_r(0.3, 5)
    pts, nrm, kap, w = _pack([_radial_curve(r, dr, ddr, n)])
    src, q = laplace_sources(rng, 8, 2.0)
    f = laplace_potential(pts, src, q)

    def inside(p):
        rad = np.hypot(p[:, 0], p[:, 1])
        return rad < 0.8 * r(np.arctan2(p[:, 1], p[:, 0]))

    tg = _targets_in(rng, n_targets, inside, (-1.3, 1.3))
    return Problem("star_laplace_n%d" % n, LAPLACE, pts, nrm, kap, w,
                   np.zeros((0, 4)), f, tg, laplace_potential(tg, src, q),
                   leaf_points, id_tol, {"sources": src, "strengths": q})


def bumped_star_case(n=2048, center=2.0, amp=0.05, width=0.12, extra=0, seed=2,
                     leaf_points=64, id_tol=1e-10, n_targets=64):
    """star_case's boundary with the nodes of one arc (|t - center| < 3 width)
    replaced: r gets a Gaussian bump amp exp(-((t - center) / width)^2) there,
    and the arc holds `extra` more (or fewer) nodes, evenly spaced in t
    between the arc's first and last parameter.  Every node outside the arc
    is bit-identical to star_case(n)'s, so a boundary update matches it.
    Boundary data and targets are star_case(n)'s sources and targets."""
    base = star_case(n=n, seed=seed, leaf_points=leaf_points, id_tol=id_tol,
                     n_targets=n_targets)
    r0, dr0, ddr0 = _star_r(0.3, 5)
    t = 2.0 * np.pi * np.arange(n) / n
    arc = np.nonzero(np.abs(t - center) < 3.0 * width)[0]
    a0, a1 = int(arc[0]), int(arc[-1])
    m = arc.size + extra
    tn = np.linspace(t[a0], t[a1], m)

    def bump(tt):
        u = (tt - center) / width
        g = amp * np.exp(-u * u)
        return g, g * (-2.0 * u / width), g * (4.0 * u * u - 2.0) / (width * width)

    b0, b1, b2 = bump(tn)
    rt, drt, ddrt = r0(tn) + b0, dr0(tn) + b1, ddr0(tn) + b2
    c, s_ = np.cos(tn), np.sin(tn)
    xp = drt * c - rt * s_
    yp = drt * s_ + rt * c
    xpp = ddrt * c - 2.0 * drt * s_ - rt * c
    ypp = ddrt * s_ + 2.0 * drt * c - rt * s_
    speed = np.sqrt(xp * xp + yp * yp)
    new = (rt * c, rt * s_, yp / speed, -xp / speed, (xp * ypp - yp * xpp) / speed**3,
           speed * ((t[a1] - t[a0]) / (m - 1)))
    old = (base.points[0::2], base.points[1::2], base.normals[0::2], base.normals[1::2],
           base.curvatures, base.weights)
    parts = [tuple(np.concatenate([o[:a0], nw, o[a1 + 1:]]) for o, nw in zip(old, new))]
    pts, nrm, kap, w = _pack(parts)
    src, q = base.extra["sources"], base.extra["strengths"]
    return Problem("bumped_star_n%d_e%d" % (n, extra), LAPLACE, pts, nrm, kap, w,
                   np.zeros((0, 4)), laplace_potential(pts, src, q), base.targets,
                   laplace_potential(base.targets, src, q), leaf_points, id_tol,
                   {"sources": src, "strengths": q, "arc": (a0, a1)})


def _place_holes(rng, k, rmin, rmax, outer=1.0, gap=0.05):
    holes = []
    while len(holes) < k:
        rad = rng.uniform(rmin, rmax)
        lim = outer - rad - gap
        c = rng.uniform(-lim, lim, 2)
        if np.hypot(*c) > lim:
            continue
        if all(np.hypot(c[0] - h[0], c[1] - h[1]) > rad + h[2] + gap
               for h in holes):
            holes.append((c[0], c[1], rad))
    return holes


def stokes_holes_case(n_total=32768, seed=3, n_holes=8, leaf_points=64,
                      id_tol=1e-10, n_targets=256):
    rng = np.random.default_rng(seed)
    holes = _place_holes(rng, n_holes, 0.05, 0.15)
    perim = np.array([1.0] + [h[2] for h in holes])
    counts = np.floor(n_total * perim / perim.sum()).astype(int)
    counts[0] += n_total - counts.sum()
    parts = [_circle(0.0, 0.0, 1.0, counts[0])]
    hole_rows = []
    for (cx, cy, rad), cnt in zip(holes, counts[1:]):
        parts.append(_circle(cx, cy, rad, cnt, inward=True))
        hole_rows.append((cx, cy, rad, cnt))
    pts, nrm, kap, w = _pack(parts)
    ang = rng.uniform(0.0, 2.0 * np.pi, 6)
    src = np.stack([2.0 * np.cos(ang), 2.0 * np.sin(ang)], axis=1)
    force = rng.standard_normal((6, 2))
    f = stokeslet_velocity(pts, src, force)
    hr = np.asarray(hole_rows)

    def inside(p):
        ok = np.hypot(p[:, 0], p[:, 1]) < 0.9
        for cx, cy, rad, _ in hole_rows:
            ok &= np.hypot(p[:, 0] - cx, p[:, 1] - cy) > rad + 0.05
        return ok

    tg = _targets_in(rng, n_targets, inside, (-1.0, 1.0))
    return Problem("disk8holes_stokes_n%d" % n_total, STOKES, pts, nrm, kap, w,
                   hr, f, tg, stokeslet_velocity(tg, src, force), leaf_points,
                   id_tol, {"sources": src, "forces": force})


def random_star(rng, n, leaf_points=64, id_tol=1e-10, name="rstar"):
    a = rng.uniform(0.0, 0.05, 5)
    ph = rng.uniform(0.0, 2.0 * np.pi, 5)
    ks = np.arange(2, 7)

    def r(t):
        return 1.0 + (a[:, None] * np.cos(ks[:, None] * t + ph[:, None])).sum(0)

    def dr(t):
        return (-a[:, None] * ks[:, None] *
                np.sin(ks[:, None] * t + ph[:, None])).sum(0)

    def ddr(t):
        return (-a[:, None] * ks[:, None]**2 *
                np.cos(ks[:, None] * t + ph[:, None])).sum(0)

    pts, nrm, kap, w = _pack([_radial_curve(r, dr, ddr, n)])
    src, q = laplace_sources(rng, 4, 2.0)
    f = laplace_potential(pts, src, q)

    def inside(p):
        return np.hypot(p[:, 0], p[:, 1]) < 0.8 * r(np.arctan2(p[:, 1], p[:, 0]))

    tg = _targets_in(rng, 16, inside, (-1.3, 1.3))
    return Problem(name, LAPLACE, pts, nrm, kap, w, np.zeros((0, 4)), f, tg,
                   laplace_potential(tg, src, q), leaf_points, id_tol,
                   {"a": a, "phi": ph})


def random_star_cases(count=256, seed=4, nmin=512, nmax=8192, leaf_points=64,
                      id_tol=1e-10):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(nmin), math.log(nmax), count))
    sizes = np.round(sizes).astype(int)
    return [random_star(rng, int(n), leaf_points, id_tol, "rstar%d_n%d" % (i, n))
            for i, n in enumerate(sizes)]


def fourier_radius(coef):
    """r(t) = 1 + sum_k c_k cos(k t) + s_k sin(k t), k = 1..len(coef)/2."""
    coef = np.asarray(coef, dtype=np.float64)
    kmax = coef.size // 2
    ks = np.arange(1, kmax + 1)
    cc, ss = coef[:kmax], coef[kmax:]

    def r(t):
        return 1.0 + (cc[:, None] * np.cos(ks[:, None] * t) +
                      ss[:, None] * np.sin(ks[:, None] * t)).sum(0)

    def dr(t):
        return (ks[:, None] * (-cc[:, None] * np.sin(ks[:, None] * t) +
                               ss[:, None] * np.cos(ks[:, None] * t))).sum(0)

    def ddr(t):
        return (-(ks[:, None]**2) * (cc[:, None] * np.cos(ks[:, None] * t) +
                                      ss[:, None] * np.sin(ks[:, None] * t))).sum(0)

    return r, dr, ddr


def fourier_star_geometry(coef, n):
    r, dr, ddr = fourier_radius(coef)
    return _pack([_radial_curve(r, dr, ddr, n)])


def fourier_star_case(n=8192, seed=5, n_coef=32, leaf_points=64, id_tol=1e-10,
                      n_targets=64):
    rng = np.random.default_rng(seed)
    coef = rng.uniform(-0.03, 0.03, n_coef)
    pts, nrm, kap, w = fourier_star_geometry(coef, n)
    src, q = laplace_sources(rng, 4, 2.0)
    f = laplace_potential(pts, src, q)
    ang = rng.uniform(0.0, 2.0 * np.pi, n_targets)
    rad = 0.6 * np.sqrt(rng.uniform(0.0, 1.0, n_targets))
    tg = np.stack([rad * np.cos(ang), rad * np.sin(ang)], axis=1).reshape(-1)
    u_star = laplace_potential(tg, src, q) + 0.01 * rng.standard_normal(n_targets)
    return Problem("fourier_star_n%d" % n, LAPLACE, pts, nrm, kap, w,
                   np.zeros((0, 4)), f, tg, laplace_potential(tg, src, q),
                   leaf_points, id_tol,
                   {"coef": coef, "u_star": u_star, "sources": src,
                    "strengths": q})


# --------------------------------------------------------------------------
# the reference test-suite shapes (kern_interp/boundaries), for parity fixtures


def reference_shape(kind, n):
    """Restates the reference test shapes: 'circle' (circle.cpp:8-32),
    'annulus' (annulus.cpp:8-63), 'donut' (donut.cpp:8-64).  Returns
    (points, normals, curvatures, weights, holes)."""
    if kind == "circle":
        t = np.arange(n) * 2.0 * np.pi / n
        parts = [(0.5 + 0.25 * np.cos(t), 0.5 + 0.25 * np.sin(t), np.cos(t),
                  np.sin(t), np.full(n, 4.0), np.full(n, np.pi / (n * 2)))]
        holes = np.zeros((0, 4))
    elif kind in ("annulus", "donut"):
        hole_list = ([(0.9, 0.5, 0.2), (0.1, 0.5, 0.2)] if kind == "annulus"
                     else [(0.5, 0.5, 0.5)])
        hn = n // 5
        t = np.arange(n) * 2.0 * np.pi / n
        parts = [(0.5 + np.cos(t), 0.5 + np.sin(t), np.cos(t), np.sin(t),
                  np.full(n, 1.0), np.full(n, 2 * np.pi / n))]
        for cx, cy, rad in hole_list:
            th = np.arange(hn) * 2.0 * np.pi / hn
            parts.append((cx + rad * np.cos(th), cy + rad * np.sin(th),
                          -np.cos(th), -np.sin(th), np.full(hn, -1.0 / rad),
                          np.full(hn, (2 * rad * np.pi) / hn)))
        holes = np.array([(cx, cy, rad, hn) for cx, cy, rad in hole_list])
    else:
        raise ValueError(kind)
    pts, nrm, kap, w = _pack(parts)
    return pts, nrm, kap, w, holes


def single_electron(points):
    """Laplace data of a unit charge at (-3, -2) (boundary.cpp:49-54)."""
    p = points.reshape(-1, 2)
    return np.log(np.sqrt((p[:, 0] + 3)**2 + (p[:, 1] + 2)**2)) / (2 * np.pi)


def tangent_vec(normals):
    """Stokes data t = (-n_y, n_x) (boundary.cpp:70-73)."""
    nrm = normals.reshape(-1, 2)
    out = np.empty_like(nrm)
    out[:, 0], out[:, 1] = -nrm[:, 1], nrm[:, 0]
    return out.reshape(-1)
