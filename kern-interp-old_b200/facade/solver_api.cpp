// Kernel, QuadTree, SkelFactorization and the solve entry points of the C++
// drop-in API, forwarding to the library's C ABI (include/kinterp.h): the
// partition, the factorization and the solves run in libkinterp.so, the
// factors stay on the GPU inside the QuadTree that owns them.  Reference
// interfaces: kern_interp/kernel/kernel.h:15-86, quadtree/quadtree.h:74-102,
// skel_factorization/skel_factorization.h:19-62, linear_solve.h:15-35.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <utility>

#include "kern_interp/linear_solve.h"
#include "kinterp.h"

namespace kern_interp {

namespace {

// The reference asserts or exits on failure; the drop-in prints the
// library's message and aborts.
void check(int rc, const char* what) {
  if (rc == KI_OK) return;
  std::fprintf(stderr, "kern_interp: %s failed (%d): %s\n", what, rc, ki_last_error());
  std::abort();
}

ki_solver_t as_handle(void* p) { return static_cast<ki_solver_t>(p); }

std::vector<double> holes_array(const std::vector<Hole>& holes) {
  // the C ABI's {cx, cy, r, node count} per hole (the count only serves the
  // node-curve domain test, which this API replaces by Boundary::is_in_domain)
  std::vector<double> out;
  for (const Hole& h : holes) {
    out.push_back(h.center.a[0]);
    out.push_back(h.center.a[1]);
    out.push_back(h.radius);
    out.push_back(0.0);
  }
  return out;
}

}  // namespace

// ---------------------------------------------------------------- Kernel
void* Kernel::geometry() const {
  if (!geometry_) {
    ki_solver_t h = nullptr;
    const int n = static_cast<int>(boundary_weights.size());
    check(ki_geometry(static_cast<int>(pde), n, boundary_points.data(), boundary_normals.data(),
                      boundary_curvatures.data(), boundary_weights.data(), nullptr, &h),
          "Kernel geometry");
    geometry_ = std::shared_ptr<void>(h, [](void* p) { ki_destroy(static_cast<ki_solver_t>(p)); });
  }
  return geometry_.get();
}

ki_Mat Kernel::operator()(const std::vector<int>& tgt_inds, const std::vector<int>& src_inds,
                          bool forward) const {
  const int nt = static_cast<int>(tgt_inds.size()), ns = static_cast<int>(src_inds.size());
  ki_Mat ret(nt, ns);
  if (nt == 0 || ns == 0) return ret;
  if (forward) {
    check(ki_forward_block(as_handle(geometry()), static_cast<int>(domain_points.size() / 2),
                           domain_points.data(), nt, tgt_inds.data(), ns, src_inds.data(),
                           ret.mat),
          "Kernel::operator() (forward)");
  } else {
    check(ki_kernel_block(as_handle(geometry()), nt, tgt_inds.data(), ns, src_inds.data(),
                          ret.mat),
          "Kernel::operator()");
  }
  return ret;
}

ki_Mat Kernel::laplace_get(const std::vector<int>& tgt_inds, const std::vector<int>& src_inds,
                           bool forward) const {
  return (*this)(tgt_inds, src_inds, forward);
}

ki_Mat Kernel::stokes_get(const std::vector<int>& tgt_inds, const std::vector<int>& src_inds,
                          bool forward) const {
  return (*this)(tgt_inds, src_inds, forward);
}

ki_Mat Kernel::forward() const {
  const int sd = solution_dimension == 1 ? 1 : 2;
  std::vector<int> tgt(sd * (domain_points.size() / 2)), src(sd * (boundary_points.size() / 2));
  for (size_t i = 0; i < tgt.size(); i++) tgt[i] = static_cast<int>(i);
  for (size_t j = 0; j < src.size(); j++) src[j] = static_cast<int>(j);
  return (*this)(tgt, src, true);
}

void Kernel::update_boundary(Boundary* boundary) {
  boundary_points = boundary->points;
  boundary_normals = boundary->normals;
  boundary_weights = boundary->weights;
  boundary_curvatures = boundary->curvatures;
  geometry_.reset();
}

// ---------------------------------------------------------------- QuadTree
struct QuadTree::State {
  ki_solver_t h = nullptr;  // partition-only handle, or the factorization
  bool factored = false;
  bool perturbed = false;   // perturb() since the last skeletonize
  std::vector<Hole> holes;  // of the boundary given to initialize_tree / perturb
  ~State() {
    if (h) ki_destroy(h);
  }
  void replace(ki_solver_t nh, bool f) {
    if (h) ki_destroy(h);
    h = nh;
    factored = f;
  }
};

QuadTree::QuadTree() : solution_dimension(1), domain_dimension(2), min(0), max(0) {}

QuadTree::~QuadTree() { clear_levels(); }

QuadTree::QuadTree(QuadTree&& o) noexcept { *this = std::move(o); }

QuadTree& QuadTree::operator=(QuadTree&& o) noexcept {
  if (this == &o) return *this;
  clear_levels();
  solution_dimension = o.solution_dimension;
  domain_dimension = o.domain_dimension;
  no_proxy_level = o.no_proxy_level;
  min = o.min;
  max = o.max;
  boundary_points = std::move(o.boundary_points);
  root = o.root;
  allskel_mat = std::move(o.allskel_mat);
  allskel_mat_lu = std::move(o.allskel_mat_lu);
  U = std::move(o.U);
  Psi = std::move(o.Psi);
  S_LU = std::move(o.S_LU);
  allskel_mat_piv = std::move(o.allskel_mat_piv);
  S_piv = std::move(o.S_piv);
  levels = std::move(o.levels);
  max_leaf_dofs = o.max_leaf_dofs;
  st_ = std::move(o.st_);
  o.root = nullptr;
  o.levels.clear();
  return *this;
}

void QuadTree::clear_levels() {
  for (QuadTreeLevel* l : levels) delete l;
  levels.clear();
  root = nullptr;
}

void* QuadTree::factorization() const { return st_ && st_->factored ? st_->h : nullptr; }

void QuadTree::initialize_tree(Boundary* boundary, int solution_dimension_,
                               int domain_dimension_) {
  if (boundary->points.empty()) {
    std::fprintf(stderr, "kern_interp: number of boundary_points to init tree cannot be 0.\n");
    std::abort();
  }
  boundary_points = boundary->points;
  solution_dimension = solution_dimension_;
  domain_dimension = domain_dimension_;
  min = max = boundary_points[0];
  for (double v : boundary_points) {
    min = std::min(min, v);
    max = std::max(max, v);
  }
  if (!st_) st_.reset(new State());
  st_->holes = boundary->holes;
  st_->perturbed = false;
  ki_solver_t h = nullptr;
  check(ki_partition(static_cast<int>(boundary_points.size() / 2), boundary_points.data(),
                     solution_dimension, max_leaf_dofs, &h),
        "QuadTree::initialize_tree");
  st_->replace(h, false);
  mirror();
}

void QuadTree::mirror() {
  clear_levels();
  ki_solver_t h = st_->h;
  const int L = ki_num_levels(h);
  std::vector<std::vector<QuadTreeNode*>> by_level(L);
  for (int l = 0; l < L; l++) {
    QuadTreeLevel* lv = new QuadTreeLevel();
    levels.push_back(lv);
    const int nb = ki_num_boxes(h, l);
    for (int i = 0; i < nb; i++) {
      int info[8];
      double geom[3];
      check(ki_box_info(h, l, i, info, geom), "ki_box_info");
      QuadTreeNode* nd = new QuadTreeNode();
      nd->level = l;
      nd->is_leaf = info[0] != 0;
      nd->compressed = info[1] != 0;
      nd->side_length = geom[2];
      const double x0 = geom[0], y0 = geom[1], s = geom[2];
      const double c[8] = {x0, y0, x0, y0 + s, x0 + s, y0 + s, x0 + s, y0};
      std::memcpy(nd->corners, c, sizeof(c));
      InteractionLists& d = nd->dof_lists;
      d.original_box.resize(info[2]);
      d.active_box.resize(info[3]);
      d.skel.resize(info[4]);
      d.redundant.resize(info[5]);
      check(ki_box_lists(h, l, i, d.original_box.data(), d.active_box.data(), d.skel.data(),
                         d.redundant.data()),
            "ki_box_lists");
      nd->dofs_below = info[2];
      d.skelnear = d.skel;
      nd->parent = info[6] >= 0 ? by_level[l - 1][info[6]] : nullptr;
      lv->nodes.push_back(nd);
      by_level[l].push_back(nd);
    }
  }
  // children in {BL, TL, TR, BR} order: from each child's corner
  for (int l = 1; l < L; l++)
    for (QuadTreeNode* nd : by_level[l]) {
      QuadTreeNode* p = nd->parent;
      if (!p) continue;
      const double half = p->side_length / 2;
      const bool right = nd->corners[0] >= p->corners[0] + 0.5 * half;
      const bool top = nd->corners[1] >= p->corners[1] + 0.5 * half;
      const int q = !right ? (top ? 1 : 0) : (top ? 2 : 3);
      p->children[q] = nd;
      p->is_leaf = false;
    }
  for (int l = 0; l < L; l++) {
    const int nb = static_cast<int>(by_level[l].size());
    for (int i = 0; i < nb; i++) {
      const int cnt = ki_box_neighbors(h, l, i, nullptr, nullptr);
      if (cnt <= 0) continue;
      std::vector<int> nl(cnt), ni(cnt);
      ki_box_neighbors(h, l, i, nl.data(), ni.data());
      for (int q = 0; q < cnt; q++) by_level[l][i]->neighbors.push_back(by_level[nl[q]][ni[q]]);
    }
  }
  root = L > 0 && !by_level[0].empty() ? by_level[0][0] : nullptr;
}

void QuadTree::perturb(const Boundary& new_boundary) {
  boundary_points = new_boundary.points;
  st_->holes = new_boundary.holes;
  if (st_->factored) {
    // applied by the next skeletonize (ki_update: the partition's perturb
    // and the refactorization of what it touched)
    st_->perturbed = true;
    return;
  }
  check(ki_partition_update(st_->h, static_cast<int>(boundary_points.size() / 2),
                            boundary_points.data()),
        "QuadTree::perturb");
  mirror();
}

void QuadTree::copy_into(QuadTree* new_tree) const {
  QuadTree fresh;
  fresh.solution_dimension = solution_dimension;
  fresh.domain_dimension = domain_dimension;
  fresh.no_proxy_level = no_proxy_level;
  fresh.min = min;
  fresh.max = max;
  fresh.boundary_points = boundary_points;
  fresh.U = U;
  fresh.Psi = Psi;
  fresh.max_leaf_dofs = max_leaf_dofs;
  fresh.st_.reset(new State());
  fresh.st_->holes = st_ ? st_->holes : std::vector<Hole>();
  ki_solver_t h = nullptr;
  if (st_ && st_->factored && !st_->perturbed) {
    check(ki_copy(st_->h, nullptr, &h), "QuadTree::copy_into");
    fresh.st_->replace(h, true);
  } else {
    check(ki_partition(static_cast<int>(boundary_points.size() / 2), boundary_points.data(),
                       solution_dimension, max_leaf_dofs, &h),
          "QuadTree::copy_into");
    fresh.st_->replace(h, false);
  }
  fresh.mirror();
  *new_tree = std::move(fresh);
}

void QuadTree::reset() {
  clear_levels();
  st_.reset();
}

void QuadTree::reset(Boundary* boundary_) {
  clear_levels();
  initialize_tree(boundary_, solution_dimension, domain_dimension);
}

// ------------------------------------------------------ SkelFactorization
SkelFactorization::SkelFactorization(double id_tol_, int fact_threads_)
    : id_tol(id_tol_), fact_threads(fact_threads_) {
  if (!(id_tol > 0)) {
    std::fprintf(stderr, "kern_interp: id_tol must be greater than 0\n");
    std::abort();
  }
}

void SkelFactorization::skeletonize(const Kernel& K, QuadTree* tree) {
  if (!tree->st_) {
    std::fprintf(stderr, "kern_interp: skeletonize before QuadTree::initialize_tree\n");
    std::abort();
  }
  QuadTree::State& st = *tree->st_;
  const int n = static_cast<int>(K.boundary_weights.size());
  // a nonzero U width selects the multiply-connected factorization
  // (skel_factorization.cpp:130), as in the reference
  const bool border = tree->U.width() > 0 && K.pde != Kernel::LAPLACE_NEUMANN;
  const std::vector<double> holes = border ? holes_array(st.holes) : std::vector<double>();
  const int nh = static_cast<int>(holes.size() / 4);
  if (st.factored && !st.perturbed) {
    // every box is compressed already: the reference's skeletonize skips
    // compressed boxes and redoes only the top level, which is the same
    return;
  }
  if (st.factored && st.perturbed) {
    int kept = 0;
    check(ki_update(st.h, n, K.boundary_points.data(), K.boundary_normals.data(),
                    K.boundary_curvatures.data(), K.boundary_weights.data(), nh,
                    nh ? holes.data() : nullptr, &kept),
          "SkelFactorization::skeletonize (update)");
  } else {
    ki_solver_t h = nullptr;
    check(ki_factor(static_cast<int>(K.pde), n, K.boundary_points.data(),
                    K.boundary_normals.data(), K.boundary_curvatures.data(),
                    K.boundary_weights.data(), nh, nh ? holes.data() : nullptr,
                    tree->max_leaf_dofs, id_tol, nullptr, &h),
          "SkelFactorization::skeletonize");
    st.replace(h, true);
  }
  st.perturbed = false;
  tree->boundary_points = K.boundary_points;
  tree->mirror();
}

void SkelFactorization::solve(const QuadTree& quadtree, ki_Mat* x, const ki_Mat& b) const {
  ki_solver_t h = as_handle(quadtree.factorization());
  if (!h) {
    std::fprintf(stderr, "kern_interp: solve before skeletonize\n");
    std::abort();
  }
  if (x->height() != b.height() || x->width() != 1) *x = ki_Mat(b.height(), 1);
  const int nb = ki_num_border(h);
  ki_Mat alpha(std::max(nb, 1), 1);
  check(ki_solve(h, b.mat, x->mat, nb > 0 ? alpha.mat : nullptr), "SkelFactorization::solve");
}

void SkelFactorization::multiply_connected_solve(const QuadTree& quadtree, ki_Mat* x,
                                                 ki_Mat* alpha, const ki_Mat& b) const {
  ki_solver_t h = as_handle(quadtree.factorization());
  if (!h) {
    std::fprintf(stderr, "kern_interp: solve before skeletonize\n");
    std::abort();
  }
  if (x->height() != b.height() || x->width() != 1) *x = ki_Mat(b.height(), 1);
  const int nb = ki_num_border(h);
  if (alpha->height() != nb || alpha->width() != 1) *alpha = ki_Mat(nb, 1);
  ki_Mat scratch(1, 1);
  check(ki_solve(h, b.mat, x->mat, nb > 0 ? alpha->mat : scratch.mat),
        "SkelFactorization::multiply_connected_solve");
}

// ------------------------------------------------------------ linear_solve
ki_Mat initialize_U_mat(const Kernel::Pde pde, const std::vector<Hole>& holes,
                        const std::vector<double>& tgt_points) {
  if (holes.empty() || pde == Kernel::LAPLACE_NEUMANN) return ki_Mat(0, 0);
  const int np = static_cast<int>(tgt_points.size() / 2);
  const int nh = static_cast<int>(holes.size());
  if (pde == Kernel::LAPLACE) {
    ki_Mat U(np, nh);
    for (int i = 0; i < np; i++)
      for (int h = 0; h < nh; h++)
        U.set(i, h, std::log((Vec2(tgt_points[2 * i], tgt_points[2 * i + 1]) -
                              holes[h].center).norm()));
    return U;
  }
  // Stokeslet columns (x and y forces) and the rotlet, per hole
  ki_Mat U(2 * np, 3 * nh);
  const double scale = 1.0 / (4 * M_PI);
  for (int i = 0; i < np; i++)
    for (int h = 0; h < nh; h++) {
      const Vec2 r = Vec2(tgt_points[2 * i], tgt_points[2 * i + 1]) - holes[h].center;
      const double rn = r.norm(), inv2 = 1.0 / std::pow(rn, 2), lg = std::log(1 / rn);
      U.set(2 * i, 3 * h, scale * (lg + inv2 * r.a[0] * r.a[0]));
      U.set(2 * i + 1, 3 * h, scale * (inv2 * r.a[1] * r.a[0]));
      U.set(2 * i, 3 * h + 1, scale * (inv2 * r.a[0] * r.a[1]));
      U.set(2 * i + 1, 3 * h + 1, scale * (lg + inv2 * r.a[1] * r.a[1]));
      U.set(2 * i, 3 * h + 2, r.a[1] * (scale / std::pow(rn, 2)));
      U.set(2 * i + 1, 3 * h + 2, -r.a[0] * (scale / std::pow(rn, 2)));
    }
  return U;
}

ki_Mat initialize_Psi_mat(const Kernel::Pde pde, const std::vector<Hole>& holes,
                          const Boundary& boundary) {
  if (holes.empty() || pde == Kernel::LAPLACE_NEUMANN) return ki_Mat(0, 0);
  const int np = static_cast<int>(boundary.points.size() / 2);
  const int nh = static_cast<int>(holes.size());
  const bool stokes = pde == Kernel::STOKES;
  ki_Mat Psi(stokes ? 3 * nh : nh, stokes ? 2 * np : np);
  for (int i = 0; i < np; i++) {
    const Vec2 x(boundary.points[2 * i], boundary.points[2 * i + 1]);
    const double w = boundary.weights[i];
    for (int h = 0; h < nh; h++) {
      if (!((x - holes[h].center).norm() < holes[h].radius + 1e-8)) continue;
      if (!stokes) {
        Psi.set(h, i, w);
      } else {
        Psi.set(3 * h, 2 * i, w);
        Psi.set(3 * h + 1, 2 * i + 1, w);
        Psi.set(3 * h + 2, 2 * i, w * x.a[1]);
        Psi.set(3 * h + 2, 2 * i + 1, -w * x.a[0]);
      }
      break;
    }
  }
  return Psi;
}

void get_domain_points(int domain_size, std::vector<double>* points, double x_min,
                       double x_max, double y_min, double y_max) {
  if (domain_size <= 0) return;
  std::vector<double> out(2 * static_cast<size_t>(domain_size) * domain_size);
  check(ki_domain_points(domain_size, x_min, x_max, y_min, y_max, out.data()),
        "get_domain_points");
  points->insert(points->end(), out.begin(), out.end());
}

void linear_solve(const SkelFactorization& skel_factorization, const QuadTree& quadtree,
                  const ki_Mat& f, ki_Mat* mu, ki_Mat* alpha) {
  *mu = ki_Mat(f.height(), 1);
  if (alpha == nullptr) {
    skel_factorization.solve(quadtree, mu, f);
  } else {
    *alpha = ki_Mat(quadtree.U.width(), 1);
    skel_factorization.multiply_connected_solve(quadtree, mu, alpha, f);
  }
}

void schur_solve(const SkelFactorization& skel_factorization, const QuadTree& quadtree,
                 const ki_Mat& U, const ki_Mat&, const ki_Mat& f, const ki_Mat& K_domain,
                 const ki_Mat& U_forward, ki_Mat* solution) {
  ki_Mat mu;
  if (U.width() == 0) {
    linear_solve(skel_factorization, quadtree, f, &mu);
    *solution = K_domain * mu;
  } else {
    ki_Mat alpha;
    linear_solve(skel_factorization, quadtree, f, &mu, &alpha);
    *solution = (K_domain * mu) + (U_forward * alpha);
  }
}

ki_Mat boundary_integral_solve(const Kernel& kernel, const Boundary& boundary,
                               QuadTree* quadtree, double id_tol, int fact_threads,
                               const std::vector<double>& domain_points) {
  SkelFactorization skel(id_tol, fact_threads);
  quadtree->U = initialize_U_mat(kernel.pde, boundary.holes, boundary.points);
  quadtree->Psi = initialize_Psi_mat(kernel.pde, boundary.holes, boundary);
  skel.skeletonize(kernel, quadtree);
  ki_Mat mu, alpha;
  const bool border = quadtree->U.width() > 0;
  linear_solve(skel, *quadtree, boundary.boundary_values, &mu, border ? &alpha : nullptr);
  // the domain sums on the GPU (no |targets| x N matrix), then the
  // boundary's own domain test on the host
  const int nt = static_cast<int>(domain_points.size() / 2);
  const int sd = kernel.solution_dimension == 2 ? 2 : 1;
  ki_Mat sol(nt * sd, 1);
  if (nt > 0)
    check(ki_eval_domain(as_handle(quadtree->factorization()), nt, domain_points.data(), mu.mat,
                         border ? alpha.mat : nullptr, KI_DOMAIN_ALL, nullptr, sol.mat),
          "boundary_integral_solve");
  for (int i = 0; i < nt; i++) {
    if (boundary.is_in_domain(Vec2(domain_points[2 * i], domain_points[2 * i + 1]))) continue;
    for (int c = 0; c < sd; c++) sol.set(sd * i + c, 0, 0.0);
  }
  return sol;
}

}  // namespace kern_interp
