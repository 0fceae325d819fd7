// A caller written against the reference's C++ API (kern_interp/*.h), built
// against the drop-in headers in include/kern_interp and linked with
// libkern_interp.so.  Each check prints one line; the exit status is the
// number of failed checks.  Test infrastructure only.
#include <cmath>
#include <cstdio>
#include <memory>
#include <vector>

#include "kern_interp/boundaries/annulus.h"
#include "kern_interp/boundaries/circle.h"
#include "kern_interp/boundaries/donut.h"
#include "kern_interp/ki_mat.h"
#include "kern_interp/kernel/kernel.h"
#include "kern_interp/linear_solve.h"
#include "kern_interp/quadtree/quadtree.h"
#include "kern_interp/skel_factorization/skel_factorization.h"

using namespace kern_interp;

static int failures = 0;

static void expect_le(const char* what, double v, double bound) {
  const bool ok = v <= bound;
  std::printf("%-44s %.3e <= %.3e %s\n", what, v, bound, ok ? "ok" : "FAIL");
  if (!ok) failures++;
}

// ||A [mu; alpha] - [f; 0]|| / ||f|| with A formed densely by Kernel::operator()
static double backward_error(const Kernel& kernel, Boundary* b, double tol, bool holes) {
  QuadTree tree;
  tree.initialize_tree(b, kernel.solution_dimension, kernel.domain_dimension);
  SkelFactorization skel(tol, 4);
  const int n = kernel.solution_dimension * static_cast<int>(b->weights.size());
  std::vector<int> all(n);
  for (int i = 0; i < n; i++) all[i] = i;
  ki_Mat A = kernel(all, all);
  if (!holes) {
    skel.skeletonize(kernel, &tree);
    ki_Mat mu;
    linear_solve(skel, tree, b->boundary_values, &mu);
    return (A * mu - b->boundary_values).vec_two_norm() / b->boundary_values.vec_two_norm();
  }
  tree.U = initialize_U_mat(kernel.pde, b->holes, b->points);
  tree.Psi = initialize_Psi_mat(kernel.pde, b->holes, *b);
  skel.skeletonize(kernel, &tree);
  ki_Mat mu, alpha;
  linear_solve(skel, tree, b->boundary_values, &mu, &alpha);
  ki_Mat r1 = A * mu + tree.U * alpha - b->boundary_values;
  ki_Mat r2 = tree.Psi * mu - alpha;
  return std::sqrt(std::pow(r1.vec_two_norm(), 2) + std::pow(r2.vec_two_norm(), 2)) /
         b->boundary_values.vec_two_norm();
}

int main() {
  const double tol = 1e-6;
  {
    Circle c;
    c.initialize(1024, SINGLE_ELECTRON);
    Kernel k(1, 2, Kernel::LAPLACE, &c, std::vector<double>());
    expect_le("Laplace circle backward error", backward_error(k, &c, tol, false), 10 * tol);
  }
  {
    Circle c;
    c.initialize(1024, ALL_ONES);
    Kernel k(1, 2, Kernel::LAPLACE_NEUMANN, &c, std::vector<double>());
    expect_le("Laplace-Neumann circle backward error", backward_error(k, &c, tol, false),
              10 * tol);
  }
  {
    Annulus a;
    a.initialize(1024, TANGENT_VEC);
    Kernel k(2, 2, Kernel::STOKES, &a, std::vector<double>());
    expect_le("Stokes annulus backward error", backward_error(k, &a, tol, true), 10 * tol);
  }
  {
    Annulus a;
    a.initialize(1024, SINGLE_ELECTRON);
    Kernel k(1, 2, Kernel::LAPLACE, &a, std::vector<double>());
    expect_le("Laplace annulus backward error", backward_error(k, &a, tol, true), 10 * tol);
  }
  {
    // domain solution against the potential of the charge at (-3, -2)
    Circle c;
    c.initialize(4096, SINGLE_ELECTRON);
    QuadTree tree;
    tree.initialize_tree(&c, 1, 2);
    std::vector<double> pts;
    get_domain_points(20, &pts, tree.min, tree.max, tree.min, tree.max);
    Kernel k(1, 2, Kernel::LAPLACE, &c, pts);
    ki_Mat sol = boundary_integral_solve(k, c, &tree, 1e-13, 4, pts);
    double num = 0, den = 0;
    for (size_t i = 0; i < pts.size(); i += 2) {
      if (!c.is_in_domain(Vec2(pts[i], pts[i + 1]))) continue;
      const double u = std::log(std::sqrt(std::pow(pts[i] + 3, 2) + std::pow(pts[i + 1] + 2, 2))) /
                       (2 * M_PI);
      num += std::pow(u - sol.get(static_cast<int>(i / 2), 0), 2);
      den += u * u;
    }
    expect_le("Laplace circle analytic agreement", std::sqrt(num / den), 1e-12);
    // a copy of the factored tree solves to the same values
    QuadTree copy;
    tree.copy_into(&copy);
    ki_Mat again = boundary_integral_solve(k, c, &copy, 1e-13, 4, pts);
    expect_le("copy_into gives the same answer", (again - sol).vec_two_norm(), 1e-15);
  }
  {
    // perturb + skeletonize (refactors only what moved) against a fresh tree
    Donut d;
    d.initialize(2048, TANGENT_VEC);
    QuadTree tree;
    tree.initialize_tree(&d, 2, 2);
    std::vector<double> pts;
    get_domain_points(12, &pts, tree.min, tree.max, tree.min, tree.max);
    Kernel k(2, 2, Kernel::STOKES, &d, pts);
    ki_Mat first = boundary_integral_solve(k, d, &tree, tol, 4, pts);
    Donut moved = d;
    for (size_t i = 0; i < moved.points.size(); i += 2)
      if (moved.points[i] > 1.2) moved.points[i] += 1e-3;  // one arc of the outer curve
    moved.apply_boundary_condition(0, static_cast<int>(moved.weights.size()), TANGENT_VEC);
    tree.perturb(moved);
    k.update_boundary(&moved);
    ki_Mat upd = boundary_integral_solve(k, moved, &tree, tol, 4, pts);
    QuadTree fresh;
    fresh.initialize_tree(&moved, 2, 2);
    ki_Mat ref = boundary_integral_solve(k, moved, &fresh, tol, 4, pts);
    expect_le("perturb + skeletonize vs fresh", (upd - ref).vec_two_norm() / ref.vec_two_norm(),
              20 * tol);
    expect_le("the update changed the solution", 1e-12, (upd - first).vec_two_norm());
  }
  {
    // dense helpers: LU solves and the interpolative decomposition
    const int n = 40;
    ki_Mat X(n, n), K(n, 3);
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) X.set(i, j, (i == j ? 4.0 : 0.0) + std::sin(1.0 + i * 7 + j * 3));
    for (int j = 0; j < 3; j++)
      for (int i = 0; i < n; i++) K.set(i, j, std::cos(0.5 * i + j));
    ki_Mat U, L;
    X.left_multiply_inverse(K, &U);
    X.right_multiply_inverse(K.transpose(), &L);
    expect_le("left_multiply_inverse", (X * U - K).frob_norm() / K.frob_norm(), 1e-13);
    expect_le("right_multiply_inverse", (L * X - K.transpose()).frob_norm() / K.frob_norm(),
              1e-13);
    // rank 8: a product of 60 x 8 and 8 x 30 factors with pseudo-random
    // entries in [-1, 1)
    unsigned long long seed = 12345;
    auto rnd = [&seed]() {
      seed = seed * 6364136223846793005ull + 1442695040888963407ull;
      return static_cast<double>(seed >> 11) / 9007199254740992.0 * 2.0 - 1.0;
    };
    ki_Mat F(60, 8), Gm(8, 30);
    for (int j = 0; j < 8; j++)
      for (int i = 0; i < 60; i++) F.set(i, j, rnd());
    for (int j = 0; j < 30; j++)
      for (int i = 0; i < 8; i++) Gm.set(i, j, rnd());
    ki_Mat A = F * Gm;
    std::vector<int> p;
    ki_Mat Z;
    const int k = A.id(&p, &Z, 1e-10);
    std::vector<int> sk(p.begin(), p.begin() + k), rd(p.begin() + k, p.end());
    expect_le("id rank", std::fabs(k - 8.0), 0.0);
    expect_le("id reconstruction", (A(0, 60, rd) - A(0, 60, sk) * Z).frob_norm() / A.frob_norm(),
              1e-9);
  }
  std::printf("facade caller: %d failed checks\n", failures);
  return failures;
}
