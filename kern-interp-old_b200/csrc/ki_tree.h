// Host-side adaptive quadtree for the B200 solver.
//
// Builds the same partition, level order and neighbour lists as the
// reference QuadTree (kern_interp/quadtree/quadtree.cpp:27-285) and keeps the
// per-box dof bookkeeping of remove_inactive_dofs_at_level/_box
// (quadtree.cpp:656-720) as flat arrays that the level scheduler turns into
// device work descriptors.  Boxes are numbered in creation order; `levels`
// lists them in the reference's level order, which fixes the order of the
// top-level skeleton and therefore the row/column order of its matrix.
#ifndef KI_TREE_H_
#define KI_TREE_H_

#include <vector>

namespace kib {

struct Box {
  int tree = 0;  // which problem of a forest the box belongs to
  int level = 0;
  int parent = -1;
  int child[4] = {-1, -1, -1, -1};  // order {BL, TL, TR, BR}
  bool leaf = true;
  bool compressed = false;
  double corner[8] = {0};  // BL, TL, TR, BR corners, xy interleaved
  double side = 0;
  std::vector<int> nbr;       // neighbour boxes, reference order
  std::vector<int> original;  // dofs of the points in the box
  std::vector<int> active;    // dofs not yet eliminated below this box
  std::vector<int> skel, redundant;
  std::vector<int> perm;      // ID pivots (local active indices)
  int rank = 0;
  bool dead = false;  // removed from the levels by a consolidation (perturb)
};

class QuadTreeHost {
 public:
  // points: interleaved xy of n points; sol_dim dofs per point.
  void build(const double* points, int n, int sol_dim, int max_leaf_dofs);
  // A forest of independent problems: problem p owns points
  // [starts[p], starts[p + 1]) and gets its own root (its own bounding
  // square, quadtree.cpp:83-105); level l lists every tree's level-l boxes,
  // tree by tree.  Boxes of different trees are never neighbours.
  void build_forest(const double* points, int n, int sol_dim, int max_leaf_dofs,
                    const std::vector<int>& starts);
  std::vector<int> roots;  // root box of each tree

  int sol_dim() const { return sol_dim_; }
  double min() const { return min_; }
  double max() const { return max_; }
  const double* points() const { return pts_; }

  std::vector<Box> boxes;
  std::vector<std::vector<int>> levels;

  // Fills the `original` lists of split boxes, which the build leaves empty
  // (only leaves' lists are used by the factorization).  Idempotent.
  void materialize_originals();

  // QuadTree::perturb (quadtree.cpp:359-560): the tree of old_points
  // (n_old points) follows the boundary to new_points (n_new).  Points are
  // matched by exact coordinates; matched dofs are renumbered in every
  // list, unmatched new points are added to their leaves, unmatched old
  // points are deleted.  The leaf of every added or deleted point, its
  // neighbours, its ancestors and their neighbours lose their compression
  // (mark_neighbors_and_parents, :288-313); over-full leaves are split
  // (node_subdivide) and the highest box below max_leaf dofs on a deleted
  // point's path is merged into one leaf (consolidate_node, :316-356); the
  // neighbour lists are rebuilt.  Boxes still `compressed` afterwards keep
  // their factors.  new_points must stay valid during the call.  One tree.
  void perturb(const double* old_points, int n_old, const double* new_points, int n_new);

  // active(b) for every not-yet-compressed box of `level`, then near(b) for
  // every box of the level (quadtree.cpp:664-691).
  void refresh_level(int level, std::vector<std::vector<int>>* near);
  void refresh_box(int b);

 private:
  int pick_child(const Box& b, double x, double y) const;
  void build_partition(int p0, int p1, int tree_id, double lo, double hi);
  void descendant_neighbors(int big, int small, std::vector<int>* found) const;
  void neighbor_lists();
  void subdivide(int id);    // node_subdivide (quadtree.cpp:203-285)
  void consolidate(int id);  // consolidate_node (quadtree.cpp:316-356)
  void mark_up(int id);      // mark_neighbors_and_parents (quadtree.cpp:288-313)
  void unmark(int id);

  int sol_dim_ = 1;
  int max_leaf_ = 32;
  bool orig_pending_ = false;  // split boxes' original lists not made yet
  double min_ = 0, max_ = 0;
  const double* pts_ = nullptr;  // caller's points, valid during the build
  void build_one(int p0, int p1, int tree_id);  // one tree into boxes/levels
};

}  // namespace kib

#endif  // KI_TREE_H_
