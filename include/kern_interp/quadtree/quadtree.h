// C++ drop-in API of the B200 solver: kern_interp::QuadTree.
//
// Same types and public members as the reference's kern_interp/quadtree/
// quadtree.h:14-102.  initialize_tree builds the adaptive partition (the
// library's host quadtree: same split rule, child order and neighbour
// lists as the reference) and mirrors it into `levels` / `root`; after
// SkelFactorization::skeletonize the mirrored boxes carry their skeleton and
// redundant dofs.  The factorization itself (every box's T, L, U, X_rr^-1
// and the top-level LU) stays in GPU memory, owned by the tree: the ki_Mat
// factor members of QuadTreeNode and the top-level matrices stay empty.
// perturb() and copy_into() keep the reference's meaning: the next
// skeletonize refactors only what perturb touched (ki_update), and a copy
// owns an independent copy of the factors (ki_copy).
#ifndef KERN_INTERP_QUADTREE_QUADTREE_H_
#define KERN_INTERP_QUADTREE_QUADTREE_H_

#include <cassert>
#include <memory>
#include <vector>

#include "kern_interp/boundaries/boundary.h"
#include "kern_interp/ki_mat.h"

#ifndef MAX_LEAF_DOFS
#define MAX_LEAF_DOFS 32
#endif

namespace kern_interp {

struct InteractionLists {
  std::vector<int> original_box, active_box, redundant, skel, near, skelnear, permutation;

  void set_rs_ranges(const std::vector<int>& prm, int sk, int rd) {
    assert(static_cast<int>(prm.size()) == sk + rd);
    for (int i = 0; i < sk + rd; i++) {
      (i < sk ? skel : redundant).push_back(active_box[prm[i]]);
      permutation.push_back(prm[i]);
    }
  }
  void set_skelnear_range() { skelnear.assign(skel.begin(), skel.end()); }
};

struct QuadTreeNode {
  int level, dofs_below;
  bool is_leaf, X_rr_is_LU_factored = false, compressed = false;
  double side_length;
  QuadTreeNode* parent;
  QuadTreeNode* children[4];
  std::vector<QuadTreeNode*> neighbors;
  InteractionLists dof_lists;
  // factors: kept on the GPU (empty here)
  ki_Mat T, L, U, X_rr, schur_update, X_rr_lu;
  std::vector<lapack_int> X_rr_piv;
  // {BL, TL, TR, BR}
  double corners[8];
  QuadTreeNode() {
    is_leaf = true;
    for (int i = 0; i < 4; i++) children[i] = nullptr;
  }
};

struct QuadTreeLevel {
  std::vector<QuadTreeNode*> nodes;
  ~QuadTreeLevel() {
    for (QuadTreeNode* node : nodes) delete node;
  }
};

class QuadTree {
 public:
  int solution_dimension, domain_dimension;
  int no_proxy_level = 0;
  double min, max;
  std::vector<double> boundary_points;
  QuadTreeNode* root = nullptr;
  // U and Psi as set by the caller (initialize_U_mat / initialize_Psi_mat):
  // a nonzero U width selects the multiply-connected factorization, whose
  // border the GPU forms from the boundary's holes with the same formulas
  ki_Mat allskel_mat, allskel_mat_lu, U, Psi, S_LU;
  std::vector<lapack_int> allskel_mat_piv, S_piv;
  std::vector<QuadTreeLevel*> levels;
  // Leaf size in dofs (the reference's compile-time MAX_LEAF_DOFS); set it
  // before initialize_tree to partition with another leaf size.
  int max_leaf_dofs = MAX_LEAF_DOFS;

  QuadTree();
  ~QuadTree();
  QuadTree(const QuadTree&) = delete;
  QuadTree& operator=(const QuadTree&) = delete;
  QuadTree(QuadTree&& o) noexcept;
  QuadTree& operator=(QuadTree&& o) noexcept;

  void initialize_tree(Boundary* boundary, int solution_dimension_, int domain_dimension_);
  void copy_into(QuadTree* new_tree) const;
  void perturb(const Boundary& new_boundary);
  void reset();
  void reset(Boundary* boundary_);

  // The GPU factorization this tree holds (a ki_solver_t from
  // include/kinterp.h; null before the first skeletonize).
  void* factorization() const;

 private:
  friend class SkelFactorization;
  struct State;
  std::unique_ptr<State> st_;
  void mirror();  // levels / root from the library's host tree
  void clear_levels();
};

}  // namespace kern_interp

#endif  // KERN_INTERP_QUADTREE_QUADTREE_H_
