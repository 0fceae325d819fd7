// C-ABI driver around the UNMODIFIED reference solver (compiled from its own
// sources by oracle/Makefile into oracle/_ref/libkiref.so).  It feeds the
// reference the same geometry arrays the product gets, runs the reference's
// own QuadTree::initialize_tree (quadtree.cpp:72-114),
// SkelFactorization::skeletonize (skel_factorization.cpp:94-243) and
// linear_solve (linear_solve.cpp:113-123), and exposes the partition, the
// per-box skeleton sets and the solution for parity checks.
// Test infrastructure and CPU baseline only; never part of the product.
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

#include "kern_interp/boundaries/annulus.h"
#include "kern_interp/boundaries/boundary.h"
#include "kern_interp/boundaries/circle.h"
#include "kern_interp/boundaries/donut.h"
#include "kern_interp/kernel/kernel.h"
#include "kern_interp/linear_solve.h"
#include "kern_interp/quadtree/quadtree.h"
#include "kern_interp/skel_factorization/skel_factorization.h"

extern int kiref_max_leaf_dofs;

namespace {
using namespace kern_interp;

// A Boundary whose arrays are given by the caller (boundary.h:35-51).
class ArrayBoundary : public Boundary {
 public:
  void initialize(int, BoundaryCondition) override {}
  bool is_in_domain(const Vec2&) const override { return true; }
  std::unique_ptr<Boundary> clone() const override {
    return std::make_unique<ArrayBoundary>(*this);
  }
};

// A CubicBoundary whose node arrays are given by the caller, so the
// reference's own CubicBoundary::is_in_domain (cubic_boundary.cpp:182-230)
// runs on them.
class ArrayCubic : public CubicBoundary {
 public:
  void initialize(int, BoundaryCondition) override {}
  void get_spline_points(std::vector<double>*, std::vector<double>*) override {}
  std::unique_ptr<Boundary> clone() const override {
    return std::make_unique<ArrayCubic>(*this);
  }
};

struct Handle {
  ArrayBoundary boundary;
  Kernel kernel;
  QuadTree tree;
  SkelFactorization fact;
  int sol_dim = 1;
  bool holes = false;
};

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}

Kernel::Pde to_pde(int pde) {
  return pde == 2 ? Kernel::Pde::STOKES
                  : (pde == 1 ? Kernel::Pde::LAPLACE_NEUMANN
                              : Kernel::Pde::LAPLACE);
}
}  // namespace

extern "C" {

// pde: 0 Laplace, 1 Laplace-Neumann, 2 Stokes.  holes: 4 doubles per hole
// (cx, cy, radius, num_nodes).  Returns an opaque handle, factor time in
// *t_factor (seconds, steady_clock around skeletonize only).
void* kiref_create(int pde, int n_points, const double* points,
                   const double* normals, const double* curvatures,
                   const double* weights, int n_holes, const double* holes,
                   int max_leaf_dofs, double id_tol, int threads,
                   double* t_factor) {
  kiref_max_leaf_dofs = max_leaf_dofs;
  Handle* h = new Handle();
  h->sol_dim = pde == 2 ? 2 : 1;
  Boundary& b = h->boundary;
  b.points.assign(points, points + 2 * n_points);
  b.normals.assign(normals, normals + 2 * n_points);
  b.curvatures.assign(curvatures, curvatures + n_points);
  b.weights.assign(weights, weights + n_points);
  for (int i = 0; i < n_holes; i++) {
    Hole hole;
    hole.center = Vec2(holes[4 * i], holes[4 * i + 1]);
    hole.radius = holes[4 * i + 2];
    hole.num_nodes = static_cast<int>(holes[4 * i + 3]);
    b.holes.push_back(hole);
  }
  h->kernel = Kernel(h->sol_dim, 2, to_pde(pde), &b, std::vector<double>());
  h->tree.initialize_tree(&b, h->sol_dim, 2);
  h->fact = SkelFactorization(id_tol, threads);
  h->holes = n_holes > 0 && pde != 1;
  if (h->holes) {
    h->tree.U = initialize_U_mat(h->kernel.pde, b.holes, b.points);
    h->tree.Psi = initialize_Psi_mat(h->kernel.pde, b.holes, b);
  }
  double t0 = now_s();
  h->fact.skeletonize(h->kernel, &h->tree);
  if (t_factor) *t_factor = now_s() - t0;
  return h;
}

void kiref_destroy(void* hp) { delete static_cast<Handle*>(hp); }

// Solves with the reference factorization; alpha may be null when the domain
// has no holes.  Returns the solve time (seconds) in *t_solve.
int kiref_solve(void* hp, const double* f, double* mu, double* alpha,
                double* t_solve) {
  Handle* h = static_cast<Handle*>(hp);
  int n = static_cast<int>(h->boundary.weights.size()) * h->sol_dim;
  ki_Mat fm(n, 1);
  std::memcpy(fm.mat, f, sizeof(double) * n);
  ki_Mat m, a;
  double t0 = now_s();
  if (h->holes) {
    linear_solve(h->fact, h->tree, fm, &m, &a);
  } else {
    linear_solve(h->fact, h->tree, fm, &m);
  }
  if (t_solve) *t_solve = now_s() - t0;
  std::memcpy(mu, m.mat, sizeof(double) * n);
  if (h->holes && alpha) {
    std::memcpy(alpha, a.mat, sizeof(double) * a.height());
  }
  return h->holes ? a.height() : 0;
}

int kiref_num_levels(void* hp) {
  return static_cast<int>(static_cast<Handle*>(hp)->tree.levels.size());
}

int kiref_num_nodes(void* hp, int level) {
  return static_cast<int>(
      static_cast<Handle*>(hp)->tree.levels[level]->nodes.size());
}

// info[0..7] = is_leaf, compressed, |original|, |active|, |skel|,
// |redundant|, index of parent within its level (-1 for the root), level.
// geom[0..2] = corner x, corner y, side length.
void kiref_node_info(void* hp, int level, int idx, int* info, double* geom) {
  Handle* h = static_cast<Handle*>(hp);
  QuadTreeNode* n = h->tree.levels[level]->nodes[idx];
  info[0] = n->is_leaf;
  info[1] = n->compressed;
  info[2] = static_cast<int>(n->dof_lists.original_box.size());
  info[3] = static_cast<int>(n->dof_lists.active_box.size());
  info[4] = static_cast<int>(n->dof_lists.skel.size());
  info[5] = static_cast<int>(n->dof_lists.redundant.size());
  info[6] = -1;
  if (n->parent) {
    auto& pl = h->tree.levels[level - 1]->nodes;
    for (size_t i = 0; i < pl.size(); i++) {
      if (pl[i] == n->parent) info[6] = static_cast<int>(i);
    }
  }
  info[7] = n->level;
  geom[0] = n->corners[0];
  geom[1] = n->corners[1];
  geom[2] = n->side_length;
}

// Copies the node's index lists; each buffer must hold the size reported by
// kiref_node_info.  Any pointer may be null.
void kiref_node_lists(void* hp, int level, int idx, int* original,
                      int* active, int* skel, int* redundant) {
  Handle* h = static_cast<Handle*>(hp);
  QuadTreeNode* n = h->tree.levels[level]->nodes[idx];
  auto cp = [](const std::vector<int>& v, int* out) {
    if (out && !v.empty()) std::memcpy(out, v.data(), sizeof(int) * v.size());
  };
  cp(n->dof_lists.original_box, original);
  cp(n->dof_lists.active_box, active);
  cp(n->dof_lists.skel, skel);
  cp(n->dof_lists.redundant, redundant);
}

// Dense kernel block K(tgt, src) through Kernel::operator() (kernel.cpp:99-111),
// column-major |tgt| x |src|.
void kiref_kernel_block(void* hp, int nt, const int* tgt, int ns,
                        const int* src, double* out) {
  Handle* h = static_cast<Handle*>(hp);
  std::vector<int> t(tgt, tgt + nt), s(src, src + ns);
  ki_Mat m = h->kernel(t, s);
  std::memcpy(out, m.mat, sizeof(double) * nt * ns);
}

// Target evaluation as schur_solve does it (linear_solve.cpp:126-140):
// K_domain * mu (+ U_forward * alpha with holes).  targets: 2*nt doubles.
void kiref_eval_targets(void* hp, int nt, const double* targets,
                        const double* mu, const double* alpha, double* out) {
  Handle* h = static_cast<Handle*>(hp);
  std::vector<double> dp(targets, targets + 2 * nt);
  Kernel k(h->sol_dim, 2, h->kernel.pde, &h->boundary, dp);
  ki_Mat kd = k.forward();
  int n = static_cast<int>(h->boundary.weights.size()) * h->sol_dim;
  ki_Mat m(n, 1);
  std::memcpy(m.mat, mu, sizeof(double) * n);
  ki_Mat sol = kd * m;
  if (h->holes && alpha) {
    ki_Mat uf = initialize_U_mat(h->kernel.pde, h->boundary.holes, dp);
    ki_Mat a(uf.width(), 1);
    std::memcpy(a.mat, alpha, sizeof(double) * uf.width());
    sol += uf * a;
  }
  std::memcpy(out, sol.mat, sizeof(double) * sol.height());
}

// Border matrices of the multiply-connected system (linear_solve.cpp:18-110):
// U is (dofs x cols), Psi is (cols x dofs), both column-major.  Returns cols.
int kiref_border(void* hp, double* U, double* Psi) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h->holes) return 0;
  if (U) std::memcpy(U, h->tree.U.mat,
                     sizeof(double) * h->tree.U.height() * h->tree.U.width());
  if (Psi) std::memcpy(Psi, h->tree.Psi.mat, sizeof(double) *
                       h->tree.Psi.height() * h->tree.Psi.width());
  return h->tree.U.width();
}

int kiref_allskel(void* hp, int* out) {
  Handle* h = static_cast<Handle*>(hp);
  auto& v = h->tree.root->dof_lists.active_box;
  if (out && !v.empty()) std::memcpy(out, v.data(), sizeof(int) * v.size());
  return static_cast<int>(v.size());
}

// Boundary::is_in_domain of the reference's classes for nt points
// (interleaved xy): kind 0 CubicBoundary on the given nodes (outer nodes
// first, then the holes' nodes), 1 Circle, 2 Annulus, 3 Donut (their
// analytic tests with the given holes).  out[t] = 1 inside, 0 outside.
void kiref_in_domain(int kind, int n_points, const double* points, int n_holes,
                     const double* holes, int nt, const double* targets,
                     unsigned char* out) {
  std::unique_ptr<Boundary> b;
  if (kind == 1) b.reset(new Circle());
  else if (kind == 2) b.reset(new Annulus());
  else if (kind == 3) b.reset(new Donut());
  else b.reset(new ArrayCubic());
  b->points.assign(points, points + 2 * n_points);
  int outer = n_points;
  for (int i = 0; i < n_holes; i++) {
    Hole hole;
    hole.center = Vec2(holes[4 * i], holes[4 * i + 1]);
    hole.radius = holes[4 * i + 2];
    hole.num_nodes = static_cast<int>(holes[4 * i + 3]);
    outer -= hole.num_nodes;
    b->holes.push_back(hole);
  }
  b->num_outer_nodes = outer;
  for (int t = 0; t < nt; t++)
    out[t] = b->is_in_domain(Vec2(targets[2 * t], targets[2 * t + 1])) ? 1 : 0;
}

// get_domain_points (linear_solve.cpp:183-193) into points (2 size^2).
void kiref_domain_points(int domain_size, double x_min, double x_max, double y_min,
                         double y_max, double* points) {
  std::vector<double> v;
  get_domain_points(domain_size, &v, x_min, x_max, y_min, y_max);
  if (!v.empty()) std::memcpy(points, v.data(), sizeof(double) * v.size());
}

// QuadTree::perturb (quadtree.cpp:359-560) to new node arrays, then the
// reference's own update of the kernel, the hole border and skeletonize, as
// the boundary-update test runs them (kern_interp_test.cpp:509-517).
// Factor time in *t_factor (seconds, skeletonize only).
void kiref_update(void* hp, int n_points, const double* points, const double* normals,
                  const double* curvatures, const double* weights, int n_holes,
                  const double* holes, double* t_factor) {
  Handle* h = static_cast<Handle*>(hp);
  Boundary& b = h->boundary;
  b.points.assign(points, points + 2 * n_points);
  b.normals.assign(normals, normals + 2 * n_points);
  b.curvatures.assign(curvatures, curvatures + n_points);
  b.weights.assign(weights, weights + n_points);
  b.holes.clear();
  for (int i = 0; i < n_holes; i++) {
    Hole hole;
    hole.center = Vec2(holes[4 * i], holes[4 * i + 1]);
    hole.radius = holes[4 * i + 2];
    hole.num_nodes = static_cast<int>(holes[4 * i + 3]);
    b.holes.push_back(hole);
  }
  h->tree.perturb(b);
  h->kernel.update_boundary(&b);
  if (h->holes) {
    h->tree.U = initialize_U_mat(h->kernel.pde, b.holes, b.points);
    h->tree.Psi = initialize_Psi_mat(h->kernel.pde, b.holes, b);
  }
  double t0 = now_s();
  h->fact.skeletonize(h->kernel, &h->tree);
  if (t_factor) *t_factor = now_s() - t0;
}

// QuadTree::copy_into (quadtree.cpp:584-641) into a new handle, which is
// then skeletonized again (kern_interp_test.cpp:555-563).
void* kiref_copy(void* hp) {
  Handle* h = static_cast<Handle*>(hp);
  Handle* c = new Handle();
  c->sol_dim = h->sol_dim;
  c->holes = h->holes;
  c->boundary = h->boundary;
  c->kernel = h->kernel;
  c->kernel.update_boundary(&c->boundary);
  c->fact = h->fact;
  h->tree.copy_into(&c->tree);
  c->fact.skeletonize(c->kernel, &c->tree);
  return c;
}
}
