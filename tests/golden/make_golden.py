"""Generates the golden fixtures in tests/golden/ by running the REFERENCE
solver (compiled from its own sources into oracle/_ref/libkiref.so by
``make -C oracle ref``) on seeded geometries.

    python tests/golden/make_golden.py           # every fixture
    python tests/golden/make_golden.py update    # the boundary-update ones only

Each fixture stores, for one problem: the solver settings, the quadtree
partition (per level and box: corner, side, parent, leaf flag, original dofs),
the skeletonization (per box: compressed flag, skeleton dofs in pivot order,
redundant dofs as a set), the top-level skeleton, the solution mu (and alpha
with holes) for the problem's boundary data, and the potential at its
targets.  The geometry itself is regenerated from ki_geometry with the same
seeds; its SHA-256 is stored to catch drift.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "kern-interp-old_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ki_geometry as G  # noqa: E402


def cases():
    """(name, problem, id_tol, max_leaf_dofs) of every fixture."""
    out = [("ellipse_laplace_1024", G.ellipse_case(), 1e-10, 64),
           ("star_laplace_2048", G.star_case(n=2048, n_targets=64), 1e-10, 64),
           ("disk_holes_stokes_2048", G.stokes_holes_case(n_total=2048, n_targets=32),
            1e-10, 128),
           ("fourier_star_laplace_1024", G.fourier_star_case(n=1024), 1e-10, 64)]
    for kind in ("circle", "annulus", "donut"):
        for pde in (G.LAPLACE, G.STOKES):
            pts, nrm, kap, w, holes = G.reference_shape(kind, 1024)
            f = G.single_electron(pts) if pde == G.LAPLACE else G.tangent_vec(nrm)
            tg = np.array([0.5, 0.52, 0.47, 0.55])
            pr = G.Problem("%s_%s_1024" % (kind, "laplace" if pde == 0 else "stokes"), pde,
                           pts, nrm, kap, w, holes, f, tg, np.zeros(0), 16, 1e-6)
            out.append((pr.name, pr, 1e-6, 32))
        # the reference's Laplace-Neumann tests use all-ones data
        # (kern_interp_test.cpp:109-206, boundary.cpp:56-58); holes get no
        # border for this kernel (kern_interp_test.cpp:39-40)
        pts, nrm, kap, w, holes = G.reference_shape(kind, 1024)
        pr = G.Problem("%s_neumann_1024" % kind, G.LAPLACE_NEUMANN, pts, nrm, kap, w, holes,
                       np.ones(pts.size // 2), np.array([0.5, 0.52, 0.47, 0.55]), np.zeros(0),
                       16, 1e-6)
        out.append((pr.name, pr, 1e-6, 32))
    return out


def update_cases():
    """(name, base problem, boundary frames, id_tol, max_leaf_dofs) of the
    boundary-update fixtures: the reference factors the base boundary, then
    follows it through the frames (QuadTree::perturb + skeletonize each);
    the fixture holds the state after the last frame."""
    base = G.star_case(n=2048, n_targets=64)
    frames = [G.bumped_star_case(n=2048, center=2.0, amp=0.05, width=0.12, extra=60),
              G.bumped_star_case(n=2048, center=3.5, amp=0.03, width=0.2, extra=-150)]
    return [("star_update_2048", base, frames, 1e-10, 64)]


def geometry_hash(pr):
    h = hashlib.sha256()
    for a in (pr.points, pr.normals, pr.curvatures, pr.weights, pr.holes, pr.f, pr.targets):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def dump(solver, pr, tol, leaf):
    rec = {"pde": pr.pde, "id_tol": tol, "max_leaf_dofs": leaf,
           "geometry_sha256": geometry_hash(pr)}
    corner, side, parent, leafv, level, comp = [], [], [], [], [], []
    orig, orig_off, skel, skel_off, red, red_off = [], [0], [], [0], [], [0]
    for l in range(solver.levels()):
        for i in range(solver.nodes(l)):
            nd = solver.node(l, i)
            corner.append(nd["corner"])
            side.append(nd["side"])
            parent.append(nd["parent"])
            leafv.append(nd["is_leaf"])
            level.append(l)
            comp.append(nd["compressed"])
            orig.extend(nd["original"])
            orig_off.append(len(orig))
            skel.extend(nd["skel"])
            skel_off.append(len(skel))
            red.extend(np.sort(nd["redundant"]))
            red_off.append(len(red))
    rec.update(corner=np.array(corner), side=np.array(side), parent=np.array(parent),
               is_leaf=np.array(leafv), level=np.array(level), compressed=np.array(comp),
               original=np.array(orig, dtype=np.int32), original_off=np.array(orig_off),
               skel=np.array(skel, dtype=np.int32), skel_off=np.array(skel_off),
               redundant_sorted=np.array(red, dtype=np.int32), redundant_off=np.array(red_off),
               allskel=solver.allskel())
    mu, alpha = solver.solve(pr.f)
    rec["mu"] = mu
    rec["alpha"] = alpha
    rec["targets_out"] = solver.eval_targets(pr.targets, mu, alpha)
    return rec


def main():
    import kioracle as K
    if not K.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    for name, base, frames, tol, leaf in update_cases():
        s = K.RefSolver(base, id_tol=tol, max_leaf_dofs=leaf, threads=1)
        for fr in frames:
            s.update(fr)
        rec = dump(s, frames[-1], tol, leaf)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **rec)
        print("wrote %s (%d bytes)" % (path, os.path.getsize(path)))
    if len(sys.argv) > 1 and sys.argv[1] == "update":
        return
    for name, pr, tol, leaf in cases():
        s = K.RefSolver(pr, id_tol=tol, max_leaf_dofs=leaf, threads=1)
        rec = dump(s, pr, tol, leaf)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **rec)
        print("wrote %s (%d bytes)" % (path, os.path.getsize(path)))


if __name__ == "__main__":
    main()
