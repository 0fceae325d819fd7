"""Shared helpers of the test suite: golden fixtures and structural
comparisons between two solvers (or a solver and a fixture)."""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)


def golden_cases():
    import make_golden
    return make_golden.cases()


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def ensure_oracle():
    """Builds oracle/libkioracle.so (the CPU restatement) if missing."""
    so = os.path.join(ROOT, "oracle", "libkioracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                       capture_output=True)
    return so


def flatten(solver):
    """Per-box records of a solver, in level order."""
    out = []
    for l in range(solver.levels()):
        for i in range(solver.nodes(l)):
            out.append(solver.node(l, i))
    return out


def compare_partition(boxes, gold):
    """Number of boxes whose geometry, parent, leaf flag or dofs differ."""
    bad = 0
    if len(boxes) != len(gold["side"]):
        return max(len(boxes), len(gold["side"]))
    off = gold["original_off"]
    for q, b in enumerate(boxes):
        same = (tuple(b["corner"]) == tuple(gold["corner"][q]) and b["side"] == gold["side"][q]
                and b["parent"] == gold["parent"][q] and b["is_leaf"] == bool(gold["is_leaf"][q])
                and np.array_equal(b["original"], gold["original"][off[q]:off[q + 1]]))
        bad += not same
    return bad


def compare_skeletons(boxes, gold, order=None):
    """(rank mismatches, skeleton-set mismatches, redundant-set mismatches).

    Skeletons are compared as sets: columns whose partial norms tie exactly
    (mirror-symmetric node pairs) may be pivoted in either order by LAPACK and
    by this implementation, which permutes the skeleton without changing it.
    When `order` is a list, boxes whose skeleton order differs are appended."""
    rank_bad = skel_bad = red_bad = 0
    so, ro = gold["skel_off"], gold["redundant_off"]
    for q, b in enumerate(boxes):
        gs = gold["skel"][so[q]:so[q + 1]]
        gr = gold["redundant_sorted"][ro[q]:ro[q + 1]]
        if b["compressed"] != bool(gold["compressed"][q]) or len(b["skel"]) != len(gs):
            rank_bad += 1
            continue
        if not np.array_equal(np.sort(b["skel"]), np.sort(gs)):
            skel_bad += 1
        elif order is not None and not np.array_equal(b["skel"], gs):
            order.append(q)
        if not np.array_equal(np.sort(b["redundant"]), gr):
            red_bad += 1
    return rank_bad, skel_bad, red_bad


def compare_solvers(a, b):
    """Structural differences between two live solvers (same problem)."""
    ba, bb = flatten(a), flatten(b)
    if len(ba) != len(bb):
        return {"boxes": (len(ba), len(bb))}
    part = rank = skel = red = 0
    for x, y in zip(ba, bb):
        if not (np.array_equal(x["original"], y["original"]) and x["corner"] == y["corner"]):
            part += 1
        if x["compressed"] != y["compressed"] or len(x["skel"]) != len(y["skel"]):
            rank += 1
        elif not np.array_equal(np.sort(x["skel"]), np.sort(y["skel"])):
            skel += 1
        elif not np.array_equal(np.sort(x["redundant"]), np.sort(y["redundant"])):
            red += 1
    return {"partition": part, "rank": rank, "skel": skel, "redundant": red,
            "boxes": len(ba)}


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
