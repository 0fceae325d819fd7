// Host quadtree: same partition rules as the reference
// (kern_interp/quadtree/quadtree.cpp), written over an index-addressed box
// array instead of pointer-linked nodes.
#include "ki_tree.h"

#include "ki_pool.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace kib {

int QuadTreeHost::pick_child(const Box& b, double x, double y) const {
  // Split point and child choice of quadtree.cpp:171-185.
  double mx = ((b.corner[6] - b.corner[0]) / 2.0) + b.corner[0];
  double my = ((b.corner[3] - b.corner[1]) / 2.0) + b.corner[1];
  if (x < mx) return y < my ? 0 : 1;
  return y < my ? 3 : 2;
}

void QuadTreeHost::subdivide(int id) {
  // quadtree.cpp:203-285: four children appended to the next level in
  // {BL, TL, TR, BR} order, the parent's dofs handed down point by point,
  // then any over-full child split depth first.
  boxes[id].leaf = false;
  double c[8];
  std::memcpy(c, boxes[id].corner, sizeof(c));
  const double mx = ((c[6] - c[0]) / 2.0) + c[0];
  const double my = ((c[3] - c[1]) / 2.0) + c[1];
  const int lvl = boxes[id].level + 1;
  const double half = boxes[id].side / 2.0;
  if (static_cast<int>(levels.size()) < lvl + 1) levels.emplace_back();
  int kid[4];
  for (int q = 0; q < 4; q++) {
    Box ch;
    std::memcpy(ch.corner, c, sizeof(c));
    ch.tree = boxes[id].tree;
    ch.level = lvl;
    ch.side = half;
    ch.parent = id;
    kid[q] = static_cast<int>(boxes.size());
    boxes.push_back(ch);
    levels[lvl].push_back(kid[q]);
  }
  // Corner edits per child: {index, value} pairs.
  const int edit_idx[4][4] = {{3, 4, 5, 6}, {1, 4, 6, 7}, {0, 1, 2, 7}, {0, 2, 3, 5}};
  const double edit_val[4][4] = {{my, mx, my, mx}, {my, mx, mx, my},
                                 {mx, my, mx, my}, {mx, mx, my, my}};
  for (int q = 0; q < 4; q++)
    for (int e = 0; e < 4; e++) boxes[kid[q]].corner[edit_idx[q][e]] = edit_val[q][e];
  for (int q = 0; q < 4; q++) boxes[id].child[q] = kid[q];
  const std::vector<int>& dofs = boxes[id].original;
  for (int q = 0; q < 4; q++) boxes[kid[q]].original.reserve(dofs.size() / 2);
  for (size_t t = 0; t < dofs.size(); t += sol_dim_) {
    const int d = dofs[t];
    const int p = d / sol_dim_;
    const int q = pick_child(boxes[id], pts_[2 * p], pts_[2 * p + 1]);
    for (int s = 0; s < sol_dim_; s++) boxes[kid[q]].original.push_back(d + s);
  }
  for (int q = 0; q < 4; q++)
    if (static_cast<int>(boxes[kid[q]].original.size()) > max_leaf_) subdivide(kid[q]);
}

void QuadTreeHost::insert(int id, double x, double y, int pt) {
  // quadtree.cpp:164-197: the point's dofs join every box on its path; the
  // leaf it reaches splits once it holds more than max_leaf dofs.  Here
  // only the leaf's list grows; the lists of boxes that were already split
  // are completed once at the end (fill_internal_lists), which gives the
  // same lists because points arrive in index order.
  for (;;) {
    Box& b = boxes[id];
    const int ch = b.child[pick_child(b, x, y)];
    if (ch >= 0) {
      id = ch;
      continue;
    }
    for (int s = 0; s < sol_dim_; s++) b.original.push_back(sol_dim_ * pt + s);
    if (b.leaf && static_cast<int>(b.original.size()) > max_leaf_) subdivide(id);
    return;
  }
}

void QuadTreeHost::fill_internal_lists() {
  // Every internal box holds the dofs of all points in it in insertion
  // (= index) order: the merge of its children's sorted lists, built from
  // the deepest level up.
  std::vector<int> tmp;
  for (int l = static_cast<int>(levels.size()) - 1; l >= 0; l--) {
    for (int id : levels[l]) {
      Box& b = boxes[id];
      if (b.leaf) continue;
      const std::vector<int>& c0 = boxes[b.child[0]].original;
      const std::vector<int>& c1 = boxes[b.child[1]].original;
      const std::vector<int>& c2 = boxes[b.child[2]].original;
      const std::vector<int>& c3 = boxes[b.child[3]].original;
      tmp.resize(c0.size() + c1.size());
      std::merge(c0.begin(), c0.end(), c1.begin(), c1.end(), tmp.begin());
      std::vector<int> t2(c2.size() + c3.size());
      std::merge(c2.begin(), c2.end(), c3.begin(), c3.end(), t2.begin());
      b.original.resize(tmp.size() + t2.size());
      std::merge(tmp.begin(), tmp.end(), t2.begin(), t2.end(), b.original.begin());
    }
  }
}

void QuadTreeHost::descendant_neighbors(int big, int small) {
  // quadtree.cpp:119-161, including its "y < top && y < bottom" side test.
  const double top = boxes[big].corner[3], bottom = boxes[big].corner[1];
  const double left = boxes[big].corner[0], right = boxes[big].corner[4];
  for (int q = 0; q < 8; q += 2) {
    const double x = boxes[small].corner[q], y = boxes[small].corner[q + 1];
    const bool horiz = x > left && x < right &&
                       (std::fabs(y - top) < 1e-14 || std::fabs(y - bottom) < 1e-14);
    const bool vert = y < top && y < bottom &&
                      (std::fabs(x - left) < 1e-14 || std::fabs(x - right) < 1e-14);
    if (horiz || vert) {
      boxes[big].nbr.push_back(small);
      boxes[small].nbr.push_back(big);
      break;
    }
  }
  for (int q = 0; q < 4; q++)
    if (boxes[small].child[q] >= 0) descendant_neighbors(big, boxes[small].child[q]);
}

void QuadTreeHost::neighbor_lists() {
  // quadtree.cpp:27-69: siblings, same-level cousins whose lower-left corners
  // lie within side*sqrt(2), then (for leaves) adjacent finer boxes.
  for (size_t l = 0; l < levels.size(); l++) {
    for (int a : levels[l]) {
      const int par = boxes[a].parent;
      if (par >= 0) {
        for (int q = 0; q < 4; q++)
          if (boxes[par].child[q] != a) boxes[a].nbr.push_back(boxes[par].child[q]);
        const std::vector<int>& pn = boxes[par].nbr;  // not modified below
        for (int o : pn) {
          for (int q = 0; q < 4; q++) {
            const int cz = boxes[o].child[q];
            if (cz < 0 || boxes[cz].level != boxes[a].level) continue;
            const double dist =
                std::sqrt(std::pow(boxes[a].corner[0] - boxes[cz].corner[0], 2) +
                          std::pow(boxes[a].corner[1] - boxes[cz].corner[1], 2));
            if (dist < boxes[a].side * std::sqrt(2) + 1e-5) boxes[a].nbr.push_back(cz);
          }
        }
      }
      if (boxes[a].leaf) {
        for (size_t t = 0; t < boxes[a].nbr.size(); t++) {
          const int o = boxes[a].nbr[t];
          if (boxes[o].level != boxes[a].level) continue;
          for (int q = 0; q < 4; q++)
            if (boxes[o].child[q] >= 0) descendant_neighbors(a, boxes[o].child[q]);
        }
      }
    }
  }
}

void QuadTreeHost::build(const double* points, int n, int sol_dim,
                         int max_leaf_dofs) {
  build_forest(points, n, sol_dim, max_leaf_dofs, {0, n});
}

void QuadTreeHost::build_one(int p0, int p1, int tree_id) {
  // quadtree.cpp:72-114: root square [min - 0.01, max + 0.01]^2 over all
  // of the tree's coordinates, its points inserted in order, then the
  // neighbour lists.
  double lo_v = pts_[2 * static_cast<size_t>(p0)], hi_v = lo_v;
  for (size_t i = 2 * static_cast<size_t>(p0); i < 2 * static_cast<size_t>(p1); i++) {
    if (pts_[i] < lo_v) lo_v = pts_[i];
    if (pts_[i] > hi_v) hi_v = pts_[i];
  }
  min_ = lo_v;
  max_ = hi_v;
  const double lo = lo_v - 0.01, hi = hi_v + 0.01;
  boxes.clear();
  levels.clear();
  boxes.reserve(4 * (static_cast<size_t>(p1 - p0) * sol_dim_ / std::max(1, max_leaf_)) + 16);
  Box root;
  root.tree = tree_id;
  const double c[8] = {lo, lo, lo, hi, hi, hi, hi, lo};
  std::memcpy(root.corner, c, sizeof(c));
  root.side = hi - lo;
  boxes.push_back(root);
  levels.push_back({0});
  for (int q = p0; q < p1; q++) insert(0, pts_[2 * q], pts_[2 * q + 1], q);
  fill_internal_lists();
  neighbor_lists();
}

void QuadTreeHost::build_forest(const double* points, int n, int sol_dim, int max_leaf_dofs,
                                const std::vector<int>& starts) {
  pts_ = points;
  sol_dim_ = sol_dim;
  max_leaf_ = max_leaf_dofs;
  const int P = static_cast<int>(starts.size()) - 1;
  roots.clear();
  if (P == 1) {
    build_one(starts[0], starts[1], 0);
    roots.push_back(0);
    pts_ = nullptr;
    return;
  }
  // trees are independent: build them in parallel, then lay them end to
  // end (tree p's boxes after tree p - 1's, level lists concatenated in
  // tree order), shifting box ids
  std::vector<QuadTreeHost> part(P);
  parallel_for(P, 1, [&](int a, int e) {
    for (int p = a; p < e; p++) {
      part[p].pts_ = points;
      part[p].sol_dim_ = sol_dim;
      part[p].max_leaf_ = max_leaf_dofs;
      part[p].build_one(starts[p], starts[p + 1], p);
    }
  }, 2);
  std::vector<int> off(P + 1, 0);
  size_t depth = 0;
  for (int p = 0; p < P; p++) {
    off[p + 1] = off[p] + static_cast<int>(part[p].boxes.size());
    depth = std::max(depth, part[p].levels.size());
  }
  boxes.clear();
  boxes.resize(off[P]);
  levels.assign(depth, {});
  parallel_for(P, 1, [&](int a, int e) {
    for (int p = a; p < e; p++) {
      const int o = off[p];
      for (size_t i = 0; i < part[p].boxes.size(); i++) {
        Box& b = boxes[o + i];
        b = std::move(part[p].boxes[i]);
        if (b.parent >= 0) b.parent += o;
        for (int& c : b.child)
          if (c >= 0) c += o;
        for (int& x : b.nbr) x += o;
      }
    }
  }, 2);
  for (size_t l = 0; l < depth; l++)
    for (int p = 0; p < P; p++)
      if (l < part[p].levels.size())
        for (int id : part[p].levels[l]) levels[l].push_back(id + off[p]);
  for (int p = 0; p < P; p++) roots.push_back(off[p]);
  min_ = part[0].min_;
  max_ = part[0].max_;
  pts_ = nullptr;
}

void QuadTreeHost::refresh_box(int id) {
  // quadtree.cpp:694-720.
  Box& b = boxes[id];
  b.skel.clear();
  b.redundant.clear();
  b.active.clear();
  if (b.leaf) {
    b.active = b.original;
    return;
  }
  for (int q = 0; q < 4; q++) {
    const Box& ch = boxes[b.child[q]];
    const std::vector<int>& src = ch.compressed ? ch.skel : ch.active;
    b.active.insert(b.active.end(), src.begin(), src.end());
  }
}

void QuadTreeHost::refresh_level(int level, std::vector<std::vector<int>>* near) {
  // quadtree.cpp:664-691.
  for (int id : levels[level])
    if (!boxes[id].compressed) refresh_box(id);
  if (!near) return;
  for (int id : levels[level]) {
    std::vector<int>& nr = (*near)[id];
    nr.clear();
    for (int o : boxes[id].nbr) {
      if (boxes[o].level > boxes[id].level) continue;
      const std::vector<int>& src = boxes[o].leaf ? boxes[o].original : boxes[o].active;
      nr.insert(nr.end(), src.begin(), src.end());
    }
  }
}

}  // namespace kib
