"""The C++ drop-in API (include/kern_interp/*.h, libkern_interp.so) on the
CPU: a caller written against the reference's API compiles and links, the
reference's own test file compiles unmodified against the drop-in headers
(where the reference sources are present), the library exports the
reference's entry points, and calls that need no GPU (the partition and
the dense helpers) work."""
import ctypes as C
import os
import subprocess

import pytest

import facade_build as FB

ROOT = FB.ROOT


def test_caller_compiles_and_links():
    assert os.path.exists(FB.build_caller())


def test_reference_test_file_compiles_against_the_drop_in():
    out = FB.build_reference_tests()
    if out is None:
        pytest.skip("reference sources not present")
    assert os.path.exists(out)


def test_library_exports_reference_entry_points():
    lib = FB.facade_lib()
    syms = subprocess.run(["nm", "-DC", "--defined-only", lib], capture_output=True,
                          text=True, check=True).stdout
    for name in ("kern_interp::SkelFactorization::skeletonize(kern_interp::Kernel const&, "
                 "kern_interp::QuadTree*)",
                 "kern_interp::SkelFactorization::solve(",
                 "kern_interp::SkelFactorization::multiply_connected_solve(",
                 "kern_interp::QuadTree::initialize_tree(kern_interp::Boundary*, int, int)",
                 "kern_interp::QuadTree::perturb(",
                 "kern_interp::QuadTree::copy_into(",
                 "kern_interp::linear_solve(",
                 "kern_interp::schur_solve(",
                 "kern_interp::boundary_integral_solve(",
                 "kern_interp::initialize_U_mat(",
                 "kern_interp::initialize_Psi_mat(",
                 "kern_interp::get_domain_points(",
                 "kern_interp::Kernel::operator()(",
                 "kern_interp::Kernel::forward() const",
                 "kern_interp::ki_Mat::id(",
                 "kern_interp::ki_Mat::LU_factorize(",
                 "kern_interp::ki_Mat::operator*(kern_interp::ki_Mat const&) const",
                 "kern_interp::Circle::initialize(",
                 "kern_interp::Annulus::is_in_domain(",
                 "kern_interp::Donut::initialize("):
        assert name in syms, name


def test_host_side_calls_without_gpu(tmp_path):
    """QuadTree::initialize_tree is host work: it runs without a GPU and its
    mirrored levels match the C-ABI partition of the same points."""
    src = tmp_path / "tree.cpp"
    src.write_text(r'''
#include <cstdio>
#include "kern_interp/boundaries/circle.h"
#include "kern_interp/quadtree/quadtree.h"
#include "kern_interp/ki_mat.h"
using namespace kern_interp;
int main() {
  Circle c;
  c.initialize(1024, SINGLE_ELECTRON);
  QuadTree t;
  t.initialize_tree(&c, 1, 2);
  int boxes = 0, leaf_dofs = 0, bad = 0;
  for (auto* l : t.levels)
    for (auto* n : l->nodes) {
      boxes++;
      if (n->is_leaf) leaf_dofs += n->dof_lists.original_box.size();
      for (int q = 0; q < 4; q++)
        if (!n->is_leaf && (!n->children[q] || n->children[q]->parent != n)) bad++;
    }
  ki_Mat a(3, 3), lu;
  for (int i = 0; i < 3; i++) a.set(i, i, 2.0 + i);
  a.set(0, 2, 1.0);
  std::vector<lapack_int> piv;
  a.LU_factorize(&lu, &piv);
  std::printf("%d %d %d %d %.17g %.17g\n", (int)t.levels.size(), boxes, leaf_dofs, bad,
              t.min, t.max);
  return 0;
}
''')
    lib = FB.facade_lib()
    exe = tmp_path / "tree"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), "-o",
                    str(exe), str(src), "-L" + FB.PKG, "-l:libkern_interp.so",
                    "-Wl,-rpath," + FB.PKG], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    levels, boxes, leaf_dofs, bad = map(int, out[:4])
    assert leaf_dofs == 1024 and bad == 0
    import numpy as np
    import kinterp
    import ki_geometry as G
    ang = 2 * np.pi * np.arange(1024) / 1024
    pts = np.empty(2048)
    pts[0::2], pts[1::2] = 0.5 + 0.25 * np.cos(ang), 0.5 + 0.25 * np.sin(ang)
    p = kinterp.Partition(pts, 1, 32)
    assert p.levels() == levels
    assert sum(p.nodes(l) for l in range(p.levels())) == boxes
    assert float(out[4]) == pts.min() and float(out[5]) == pts.max()
