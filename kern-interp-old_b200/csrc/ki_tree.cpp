// Host quadtree: same partition rules as the reference
// (kern_interp/quadtree/quadtree.cpp), written over an index-addressed box
// array instead of pointer-linked nodes.
#include "ki_tree.h"

#include "ki_pool.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <utility>

namespace kib {

int QuadTreeHost::pick_child(const Box& b, double x, double y) const {
  // Split point and child choice of quadtree.cpp:171-185.
  double mx = ((b.corner[6] - b.corner[0]) / 2.0) + b.corner[0];
  double my = ((b.corner[3] - b.corner[1]) / 2.0) + b.corner[1];
  if (x < mx) return y < my ? 0 : 1;
  return y < my ? 3 : 2;
}

// Children's corners: {index, value} edits of the parent's corners per child
// {BL, TL, TR, BR} (quadtree.cpp:203-285).
namespace {
const int kEditIdx[4][4] = {{3, 4, 5, 6}, {1, 4, 6, 7}, {0, 1, 2, 7}, {0, 2, 3, 5}};
}  // namespace

void QuadTreeHost::build_partition(int p0, int p1, int tree_id, double lo, double hi) {
  // The reference inserts points one at a time (quadtree.cpp:164-197) and
  // splits a leaf as soon as it holds more than max_leaf dofs
  // (node_subdivide, :203-285), over-full children at once, depth first.
  // The resulting tree does not depend on the order: a box is split exactly
  // when all its points together exceed max_leaf, so it is built here top
  // down, every level's boxes partitioned in parallel.  What the insertion
  // order does decide is the order in which boxes were created (their ids
  // and the level lists): a box splits when its (cap+1)-th point, in index
  // order, arrives (cap = max_leaf / sol_dim points), or when its parent
  // creates it already over-full; splits at the same moment happen depth
  // first.  Sorting the splits by (that point index, depth-first position)
  // and numbering the children in that order reproduces the reference ids.
  //
  // Boxes hold contiguous ranges of one point permutation, the coordinates
  // permuted along with the indices; splitting a box stably partitions its
  // range into its children's ranges (counting sort by child), so every
  // range is in point-index order until its own box splits.  Leaves take
  // their lists from their ranges; the lists of split boxes are merged from
  // their children's only when asked for (materialize_originals).
  struct Tmp {
    int parent = -1, level = 0, child[4] = {-1, -1, -1, -1};
    int begin = 0, count = 0;
    long long moment = -1;  // a split box's (cap+1)-th point, in index order
    double corner[8];
  };
  std::vector<Tmp> tb(1);
  const double c0[8] = {lo, lo, lo, hi, hi, hi, hi, lo};
  std::memcpy(tb[0].corner, c0, sizeof(c0));
  const int np = p1 - p0;
  tb[0].count = np;
  // work arrays kept per thread between builds (no zero fill, no fresh
  // pages: a build is otherwise dominated by first-touch page faults)
  struct Work {
    std::vector<int> perm, tmpi;
    std::vector<double> pxy, tmpxy;
    std::vector<unsigned char> quad;
  };
  thread_local Work wk;
  auto grow = [](auto& v, size_t n) {
    if (v.size() < n) v.resize(n);
  };
  grow(wk.perm, np);
  grow(wk.tmpi, np);
  grow(wk.pxy, 2 * static_cast<size_t>(np));
  grow(wk.tmpxy, 2 * static_cast<size_t>(np));
  grow(wk.quad, np);
  std::vector<int>& perm = wk.perm;
  std::vector<int>& tmpi = wk.tmpi;
  std::vector<double>& pxy = wk.pxy;
  std::vector<double>& tmpxy = wk.tmpxy;
  std::vector<unsigned char>& quad = wk.quad;
  for (int q = 0; q < np; q++) {
    perm[q] = p0 + q;
    pxy[2 * q] = pts_[2 * static_cast<size_t>(p0 + q)];
    pxy[2 * q + 1] = pts_[2 * static_cast<size_t>(p0 + q) + 1];
  }
  const int cap = max_leaf_ / sol_dim_;  // split when a box holds more points
  // Box P's range into its four children ch[0..3] (ranges, corners, level;
  // the caller links them): classify the points by child, then a stable
  // scatter from a copy of the range.  A big box (the first levels) is cut
  // into chunks classified and scattered in parallel at per-chunk offsets
  // (chunks in order, sequential inside: still stable).
  auto split_one = [&](Tmp& P, Tmp* ch, bool inner_parallel) {
    const int b0 = P.begin, cnt_all = P.count;
    int* rp = perm.data() + b0;
    double* rxy = pxy.data() + 2 * static_cast<size_t>(b0);
    P.moment = rp[cap];  // the range is still in index order
    const double mx = ((P.corner[6] - P.corner[0]) / 2.0) + P.corner[0];
    const double my = ((P.corner[3] - P.corner[1]) / 2.0) + P.corner[1];
    const int kChunk = 4096;
    const int nch = inner_parallel ? (cnt_all + kChunk - 1) / kChunk : 1;
    const int csz = inner_parallel ? kChunk : cnt_all;
    std::array<int, 4> ccnt1{0, 0, 0, 0}, cpos1{};
    std::vector<std::array<int, 4>> ccntv, cposv;
    if (nch > 1) {
      ccntv.assign(nch, std::array<int, 4>{0, 0, 0, 0});
      cposv.resize(nch);
    }
    std::array<int, 4>* ccnt = nch > 1 ? ccntv.data() : &ccnt1;
    std::array<int, 4>* cpos = nch > 1 ? cposv.data() : &cpos1;
    auto classify = [&](int c0, int c1) {
      for (int c = c0; c < c1; c++) {
        const int i0 = c * csz, i1 = std::min(cnt_all, i0 + csz);
        for (int i = i0; i < i1; i++) {
          const double x = rxy[2 * i], y = rxy[2 * i + 1];
          const int q = x < mx ? (y < my ? 0 : 1) : (y < my ? 3 : 2);  // quadtree.cpp:171-185
          quad[b0 + i] = static_cast<unsigned char>(q);
          ccnt[c][q]++;
        }
        std::memcpy(tmpi.data() + b0 + i0, rp + i0, sizeof(int) * (i1 - i0));
        std::memcpy(tmpxy.data() + 2 * static_cast<size_t>(b0 + i0), rxy + 2 * i0,
                    2 * sizeof(double) * (i1 - i0));
      }
    };
    if (nch > 1) parallel_for(nch, 1, classify, 2); else classify(0, 1);
    int cnt[4] = {0, 0, 0, 0};
    for (int c = 0; c < nch; c++)
      for (int q = 0; q < 4; q++) cnt[q] += ccnt[c][q];
    int pos[4];
    pos[0] = 0;
    for (int q = 1; q < 4; q++) pos[q] = pos[q - 1] + cnt[q - 1];
    {
      // each chunk's first destination per child
      int run[4] = {pos[0], pos[1], pos[2], pos[3]};
      for (int c = 0; c < nch; c++)
        for (int q = 0; q < 4; q++) {
          cpos[c][q] = run[q];
          run[q] += ccnt[c][q];
        }
    }
    const double ev[4][4] = {{my, mx, my, mx}, {my, mx, mx, my},
                             {mx, my, mx, my}, {mx, mx, my, my}};
    for (int q = 0; q < 4; q++) {
      Tmp& C = ch[q];
      C.level = P.level + 1;
      C.begin = b0 + pos[q];
      C.count = cnt[q];
      std::memcpy(C.corner, P.corner, sizeof(C.corner));
      for (int e2 = 0; e2 < 4; e2++) C.corner[kEditIdx[q][e2]] = ev[q][e2];
    }
    const int* oi = tmpi.data() + b0;
    const double* oxy = tmpxy.data() + 2 * static_cast<size_t>(b0);
    auto scatter = [&](int c0, int c1) {
      for (int c = c0; c < c1; c++) {
        int at[4] = {cpos[c][0], cpos[c][1], cpos[c][2], cpos[c][3]};
        const int i0 = c * csz, i1 = std::min(cnt_all, i0 + csz);
        for (int i = i0; i < i1; i++) {
          const int d = at[quad[b0 + i]]++;
          rp[d] = oi[i];
          rxy[2 * d] = oxy[2 * i];
          rxy[2 * d + 1] = oxy[2 * i + 1];
        }
      }
    };
    if (nch > 1) parallel_for(nch, 1, scatter, 2); else scatter(0, 1);
  };
  // The first levels level by level (a few big boxes: each split in
  // parallel chunks, or side by side), until the frontier holds enough
  // boxes to keep every thread busy; then each frontier box's subtree by
  // one thread, breadth first into its own list, appended after the
  // others (parents keep smaller indices than their children, all that the
  // numbering below relies on).
  const int seeds = 4 * pool_threads();
  std::vector<int> frontier{0};
  while (!frontier.empty() && static_cast<int>(frontier.size()) < seeds) {
    std::vector<int> split;
    for (int id : frontier)
      if (tb[id].count > cap) split.push_back(id);
    if (split.empty()) {
      frontier.clear();
      break;
    }
    const int base = static_cast<int>(tb.size());
    tb.resize(base + 4 * split.size());
    auto link = [&](int s) {
      for (int q = 0; q < 4; q++) {
        tb[base + 4 * s + q].parent = split[s];
        tb[split[s]].child[q] = base + 4 * s + q;
      }
    };
    std::vector<int> small_ones;
    for (int s = 0; s < static_cast<int>(split.size()); s++) {
      if (tb[split[s]].count >= 16384) {
        split_one(tb[split[s]], &tb[base + 4 * s], true);
        link(s);
      } else {
        small_ones.push_back(s);
      }
    }
    // every box is real work: spread even a handful of them
    parallel_for(static_cast<int>(small_ones.size()), 1, [&](int a, int e) {
      for (int q = a; q < e; q++) {
        split_one(tb[split[small_ones[q]]], &tb[base + 4 * small_ones[q]], false);
        link(small_ones[q]);
      }
    }, 2);
    frontier.clear();
    for (size_t i = base; i < tb.size(); i++) frontier.push_back(static_cast<int>(i));
  }
  if (!frontier.empty()) {
    const int nf = static_cast<int>(frontier.size());
    std::vector<std::vector<Tmp>> sub(nf);
    parallel_for(nf, 1, [&](int a, int e) {
      for (int f = a; f < e; f++) {
        std::vector<Tmp>& loc = sub[f];
        loc.push_back(tb[frontier[f]]);  // [0]: the seed
        for (size_t q = 0; q < loc.size(); q++) {
          if (loc[q].count <= cap) continue;
          const size_t base = loc.size();
          loc.resize(base + 4);
          split_one(loc[q], &loc[base], false);
          for (int c = 0; c < 4; c++) {
            loc[base + c].parent = static_cast<int>(q);
            loc[q].child[c] = static_cast<int>(base + c);
          }
        }
      }
    }, 2);
    // seed f keeps its index; its local box j >= 1 becomes off[f] + j - 1
    std::vector<int> off(nf + 1);
    off[0] = static_cast<int>(tb.size());
    for (int f = 0; f < nf; f++) off[f + 1] = off[f] + static_cast<int>(sub[f].size()) - 1;
    tb.resize(off[nf]);
    parallel_for(nf, 4, [&](int a, int e) {
      for (int f = a; f < e; f++) {
        const std::vector<Tmp>& loc = sub[f];
        auto gid = [&](int j) { return j == 0 ? frontier[f] : off[f] + j - 1; };
        for (size_t j = 0; j < loc.size(); j++) {
          Tmp& t = tb[gid(static_cast<int>(j))];
          const int parent = t.parent;
          t = loc[j];
          t.parent = j == 0 ? parent : gid(loc[j].parent);
          for (int q = 0; q < 4; q++)
            if (loc[j].child[q] >= 0) t.child[q] = gid(loc[j].child[q]);
        }
      }
    });
  }
  // split moments: s(B) = max(index of B's (cap+1)-th point, s(parent));
  // depth-first positions from an explicit pre-order walk
  const int nt = static_cast<int>(tb.size());
  std::vector<long long> when(nt, -1);
  std::vector<int> pre(nt, 0);
  {
    std::vector<int> stack{0};
    int counter = 0;
    while (!stack.empty()) {
      const int id = stack.back();
      stack.pop_back();
      pre[id] = counter++;
      for (int q = 3; q >= 0; q--)
        if (tb[id].child[q] >= 0) stack.push_back(tb[id].child[q]);
    }
  }
  std::vector<int> splits;
  for (int id = 0; id < nt; id++) {
    if (tb[id].child[0] < 0) continue;
    long long t = tb[id].moment;
    if (tb[id].parent >= 0) t = std::max(t, when[tb[id].parent]);
    when[id] = t;
    splits.push_back(id);
  }
  std::sort(splits.begin(), splits.end(), [&](int a, int b) {
    return when[a] != when[b] ? when[a] < when[b] : pre[a] < pre[b];
  });
  // number the boxes in creation order and lay them out
  std::vector<int> idmap(nt, -1);
  idmap[0] = 0;
  int next = 1;
  for (int id : splits)
    for (int q = 0; q < 4; q++) idmap[tb[id].child[q]] = next++;
  // (a reused tree keeps its boxes' list capacities: every field is reset
  // below, the lists cleared rather than freed)
  boxes.resize(nt);
  std::vector<int> order(nt);
  for (int id = 0; id < nt; id++) order[idmap[id]] = id;
  int depth = 0;
  for (int id = 0; id < nt; id++) depth = std::max(depth, tb[id].level);
  levels.assign(depth + 1, {});
  for (int i = 0; i < nt; i++) levels[tb[order[i]].level].push_back(i);
  const double side0 = hi - lo;
  parallel_for(nt, 64, [&](int a, int e) {
    for (int id = a; id < e; id++) {
      const Tmp& t = tb[id];
      Box& b = boxes[idmap[id]];
      b.nbr.clear();
      b.original.clear();
      b.active.clear();
      b.skel.clear();
      b.redundant.clear();
      b.perm.clear();
      b.compressed = false;
      b.rank = 0;
      b.dead = false;
      b.tree = tree_id;
      b.level = t.level;
      b.parent = t.parent >= 0 ? idmap[t.parent] : -1;
      b.leaf = t.child[0] < 0;
      for (int q = 0; q < 4; q++) b.child[q] = t.child[q] >= 0 ? idmap[t.child[q]] : -1;
      std::memcpy(b.corner, t.corner, sizeof(b.corner));
      double sd = side0;
      for (int l = 0; l < t.level; l++) sd /= 2.0;
      b.side = sd;
      if (!b.leaf) continue;
      b.original.resize(static_cast<size_t>(t.count) * sol_dim_);
      const int* src = perm.data() + t.begin;
      for (int i = 0; i < t.count; i++)
        for (int c = 0; c < sol_dim_; c++)
          b.original[static_cast<size_t>(i) * sol_dim_ + c] = sol_dim_ * src[i] + c;
    }
  });
  orig_pending_ = true;
}

void QuadTreeHost::materialize_originals() {
  // a split box's list is its points in index order (the reference pushes
  // every inserted dof into each box on the point's path): the merge of its
  // children's sorted lists, deepest level first
  if (!orig_pending_) return;
  for (int l = static_cast<int>(levels.size()) - 2; l >= 0; l--)
    for (int id : levels[l]) {
      Box& b = boxes[id];
      if (b.leaf) continue;
      std::vector<int> out;
      for (int q = 0; q < 4; q++) {
        const std::vector<int>& c = boxes[b.child[q]].original;
        std::vector<int> m(out.size() + c.size());
        std::merge(out.begin(), out.end(), c.begin(), c.end(), m.begin());
        out.swap(m);
      }
      b.original.swap(out);
    }
  orig_pending_ = false;
}

void QuadTreeHost::descendant_neighbors(int big, int small, std::vector<int>* found) const {
  // quadtree.cpp:119-161, including its "y < top && y < bottom" side test:
  // every descendant of `small` with a corner on an edge of `big`, in
  // depth-first order.
  const double top = boxes[big].corner[3], bottom = boxes[big].corner[1];
  const double left = boxes[big].corner[0], right = boxes[big].corner[4];
  // The corners of `small` and of all its descendants lie in small's closed
  // square; when no point of that square can pass either side test below,
  // the whole subtree is skipped (a widened 1e-12 band keeps the skip
  // conservative, so the result is unchanged).
  {
    const double sx0 = boxes[small].corner[0], sx1 = boxes[small].corner[4];
    const double sy0 = boxes[small].corner[1], sy1 = boxes[small].corner[3];
    const double eps = 1e-12;
    const bool xin = sx0 < right && sx1 > left;
    const bool horiz = xin && ((sy0 < top + eps && sy1 > top - eps) ||
                               (sy0 < bottom + eps && sy1 > bottom - eps));
    const bool vert = sy0 < bottom && ((sx0 < left + eps && sx1 > left - eps) ||
                                       (sx0 < right + eps && sx1 > right - eps));
    if (!horiz && !vert) return;
  }
  for (int q = 0; q < 8; q += 2) {
    const double x = boxes[small].corner[q], y = boxes[small].corner[q + 1];
    const bool horiz = x > left && x < right &&
                       (std::fabs(y - top) < 1e-14 || std::fabs(y - bottom) < 1e-14);
    const bool vert = y < top && y < bottom &&
                      (std::fabs(x - left) < 1e-14 || std::fabs(x - right) < 1e-14);
    if (horiz || vert) {
      found->push_back(small);
      break;
    }
  }
  for (int q = 0; q < 4; q++)
    if (boxes[small].child[q] >= 0) descendant_neighbors(big, boxes[small].child[q], found);
}

void QuadTreeHost::neighbor_lists() {
  // quadtree.cpp:27-69, level by level: a box's neighbours are the coarser
  // leaves that found it (appended while their own level was processed),
  // then its siblings, its same-level cousins whose lower-left corners lie
  // within side*sqrt(2), and (for leaves) the adjacent finer boxes, each of
  // which also records the leaf.  The per-box searches of a level only read
  // finished lists and append to their own box's list, so they run in
  // parallel; the finer boxes' records of the leaves that found them are
  // appended afterwards in the level's box order, as the reference makes
  // them.
  // per finer box: how many leaves of the level found it, where its
  // records start in `by`, how many are placed (reset after each level)
  std::vector<int> cnt(boxes.size(), 0), start(boxes.size(), 0), fill(boxes.size(), 0);
  std::vector<int> touched, by;
  for (size_t l = 0; l < levels.size(); l++) {
    const std::vector<int>& ids = levels[l];
    const int n = static_cast<int>(ids.size());
    std::vector<std::vector<int>> found(n);
    parallel_for(n, 8, [&](int b0, int b1) {
      for (int i = b0; i < b1; i++) {
        const int a = ids[i];
        Box& box = boxes[a];
        const int par = box.parent;
        std::vector<int>& nb = box.nbr;
        const size_t own0 = nb.size();
        if (par >= 0) {
          const Box& pb = boxes[par];
          nb.reserve(own0 + 8);
          for (int q = 0; q < 4; q++)
            if (pb.child[q] != a) nb.push_back(pb.child[q]);
          for (int o : pb.nbr) {
            for (int q = 0; q < 4; q++) {
              const int cz = boxes[o].child[q];
              if (cz < 0 || boxes[cz].level != box.level) continue;
              // (squares by multiplication: the corner distances are 0,
              // side, sqrt(2) side, ..., far from the 1e-5 margin, so the
              // outcome is that of the reference's pow form)
              const double dx = box.corner[0] - boxes[cz].corner[0];
              const double dy = box.corner[1] - boxes[cz].corner[1];
              const double dist = std::sqrt(dx * dx + dy * dy);
              if (dist < box.side * std::sqrt(2) + 1e-5) nb.push_back(cz);
            }
          }
        }
        if (box.leaf) {
          std::vector<int>& fd = found[i];
          const size_t own1 = nb.size();
          for (size_t u = own0; u < own1; u++) {  // all of the same level
            const int o = nb[u];
            for (int q = 0; q < 4; q++)
              if (boxes[o].child[q] >= 0) descendant_neighbors(a, boxes[o].child[q], &fd);
          }
          nb.insert(nb.end(), fd.begin(), fd.end());
        }
      }
    });
    // the records grouped by finer box, each group in the level's box order,
    // then appended box by box in parallel
    touched.clear();
    for (int i = 0; i < n; i++)
      for (int sm : found[i])
        if (cnt[sm]++ == 0) touched.push_back(sm);
    int total = 0;
    for (int sm : touched) {
      start[sm] = total;
      total += cnt[sm];
    }
    by.resize(total);
    for (int i = 0; i < n; i++)
      for (int sm : found[i]) by[start[sm] + fill[sm]++] = ids[i];
    parallel_for(static_cast<int>(touched.size()), 32, [&](int b0, int b1) {
      for (int u = b0; u < b1; u++) {
        const int sm = touched[u];
        std::vector<int>& nb = boxes[sm].nbr;
        nb.insert(nb.end(), by.begin() + start[sm], by.begin() + start[sm] + cnt[sm]);
        cnt[sm] = 0;
        fill[sm] = 0;
      }
    });
  }
}

void QuadTreeHost::build(const double* points, int n, int sol_dim,
                         int max_leaf_dofs) {
  build_forest(points, n, sol_dim, max_leaf_dofs, {0, n});
}

void QuadTreeHost::build_one(int p0, int p1, int tree_id) {
  // quadtree.cpp:72-114: root square [min - 0.01, max + 0.01]^2 over all
  // of the tree's coordinates, then the partition and the neighbour lists.
  double lo_v = pts_[2 * static_cast<size_t>(p0)], hi_v = lo_v;
  for (size_t i = 2 * static_cast<size_t>(p0); i < 2 * static_cast<size_t>(p1); i++) {
    if (pts_[i] < lo_v) lo_v = pts_[i];
    if (pts_[i] > hi_v) hi_v = pts_[i];
  }
  min_ = lo_v;
  max_ = hi_v;
  build_partition(p0, p1, tree_id, lo_v - 0.01, hi_v + 0.01);
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
  orig_pending_ = true;
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


// ---------------------------------------------------------------- perturb

void QuadTreeHost::unmark(int id) {
  Box& b = boxes[id];
  b.compressed = false;
  b.active.clear();
  b.skel.clear();
  b.redundant.clear();
  b.perm.clear();
  b.rank = 0;
}

void QuadTreeHost::mark_up(int id) {
  for (int b = id; b >= 0; b = boxes[b].parent) {
    unmark(b);
    for (int o : boxes[b].nbr) unmark(o);
  }
}

void QuadTreeHost::subdivide(int id) {
  boxes[id].leaf = false;
  const double mx = ((boxes[id].corner[6] - boxes[id].corner[0]) / 2.0) + boxes[id].corner[0];
  const double my = ((boxes[id].corner[3] - boxes[id].corner[1]) / 2.0) + boxes[id].corner[1];
  const double ev[4][4] = {{my, mx, my, mx}, {my, mx, mx, my}, {mx, my, mx, my}, {mx, mx, my, my}};
  const int lvl = boxes[id].level + 1;
  if (static_cast<int>(levels.size()) < lvl + 1) levels.resize(lvl + 1);
  int kids[4];
  for (int q = 0; q < 4; q++) {
    Box c;
    c.tree = boxes[id].tree;
    c.level = lvl;
    c.parent = id;
    c.side = boxes[id].side / 2.0;
    std::memcpy(c.corner, boxes[id].corner, sizeof(c.corner));
    for (int e = 0; e < 4; e++) c.corner[kEditIdx[q][e]] = ev[q][e];
    kids[q] = static_cast<int>(boxes.size());
    boxes.push_back(std::move(c));
    boxes[id].child[q] = kids[q];
    levels[lvl].push_back(kids[q]);
  }
  // the box keeps its own list; its dofs go down point by point in list order
  const std::vector<int>& orig = boxes[id].original;
  for (size_t i = 0; i < orig.size(); i += sol_dim_) {
    const int dof = orig[i];
    const int pt = dof / sol_dim_;
    const int q = pick_child(boxes[id], pts_[2 * static_cast<size_t>(pt)],
                             pts_[2 * static_cast<size_t>(pt) + 1]);
    for (int c = 0; c < sol_dim_; c++) boxes[kids[q]].original.push_back(dof + c);
  }
  for (int q = 0; q < 4; q++)
    if (static_cast<int>(boxes[kids[q]].original.size()) > max_leaf_) subdivide(kids[q]);
}

void QuadTreeHost::consolidate(int id) {
  // breadth-first over the subtree: the leaves' lists in that order
  std::vector<int> queue{id};
  std::vector<int> orig;
  for (size_t i = 0; i < queue.size(); i++) {
    const Box& c = boxes[queue[i]];
    if (c.leaf) {
      if (queue[i] != id) orig.insert(orig.end(), c.original.begin(), c.original.end());
    } else {
      for (int q = 0; q < 4; q++) queue.push_back(c.child[q]);
    }
  }
  boxes[id].original.swap(orig);
  for (size_t i = 1; i < queue.size(); i++) {
    std::vector<int>& lv = levels[boxes[queue[i]].level];
    auto it = std::find(lv.begin(), lv.end(), queue[i]);
    if (it != lv.end()) lv.erase(it);
    boxes[queue[i]].dead = true;
  }
  for (int q = 0; q < 4; q++) boxes[id].child[q] = -1;
  boxes[id].leaf = true;
}

namespace {
// Exact-coordinate key of a point (the reference hashes the pair of doubles,
// quadtree.cpp:369); -0.0 and 0.0 compare equal, so both hash as 0.0.
struct PointHash {
  size_t operator()(const std::pair<double, double>& p) const {
    auto bits = [](double v) {
      if (v == 0.0) v = 0.0;
      uint64_t u;
      std::memcpy(&u, &v, sizeof(u));
      return u;
    };
    const uint64_t a = bits(p.first), b = bits(p.second);
    return static_cast<size_t>(a * 0x9E3779B97F4A7C15ULL ^ (b + 0x632BE59BD9B4E019ULL + (a << 6)));
  }
};
}  // namespace

void QuadTreeHost::perturb(const double* old_pts, int n_old, const double* new_pts, int n_new) {
  // split boxes' lists as built, left stale afterwards as the reference
  // leaves them
  materialize_originals();
  const int sd = sol_dim_;
  // old point -> new point by exact coordinates (a repeated new point maps
  // to its last index); unmatched old points are deletions, unmatched new
  // points additions (quadtree.cpp:361-396)
  std::unordered_map<std::pair<double, double>, int, PointHash> to_new;
  to_new.reserve(2 * static_cast<size_t>(n_new) + 1);
  for (int i = 0; i < n_new; i++) to_new[{new_pts[2 * i], new_pts[2 * i + 1]}] = i;
  std::vector<int> old_to_new(n_old, -1), deletions, additions;
  std::vector<char> found(n_new, 0);
  for (int i = 0; i < n_old; i++) {
    auto it = to_new.find({old_pts[2 * i], old_pts[2 * i + 1]});
    if (it != to_new.end()) {
      old_to_new[i] = it->second;
      found[it->second] = 1;
    } else {
      deletions.push_back(i);
    }
  }
  for (int j = 0; j < n_new; j++)
    if (!found[j]) additions.push_back(j);

  // renumber the lists; a leaf's original list too (quadtree.cpp:402-458)
  auto remap = [&](std::vector<int>& v) {
    size_t w = 0;
    for (size_t r = 0; r < v.size(); r++) {
      const int nn = old_to_new[v[r] / sd];
      if (nn >= 0) v[w++] = sd * nn + v[r] % sd;
    }
    v.resize(w);
  };
  for (const std::vector<int>& lv : levels)
    for (int id : lv) {
      Box& b = boxes[id];
      if (b.leaf) remap(b.original);
      remap(b.active);
      remap(b.skel);
      remap(b.redundant);
    }

  const int root = roots.empty() ? 0 : roots[0];
  // additions: into their leaves (new coordinates), which lose their
  // compression with their neighbourhoods (quadtree.cpp:460-486)
  std::vector<int> bursting;
  for (int a : additions) {
    const double x = new_pts[2 * static_cast<size_t>(a)], y = new_pts[2 * static_cast<size_t>(a) + 1];
    int c = root;
    while (!boxes[c].leaf) c = boxes[c].child[pick_child(boxes[c], x, y)];
    for (int k = 0; k < sd; k++) boxes[c].original.push_back(sd * a + k);
    bursting.push_back(c);
    mark_up(c);
  }
  // dofs below every box after the additions (quadtree.cpp:488-502)
  std::vector<long long> below(boxes.size(), 0);
  for (const std::vector<int>& lv : levels)
    for (int id : lv) below[id] = boxes[id].leaf ? static_cast<long long>(boxes[id].original.size()) : 0;
  for (int l = static_cast<int>(levels.size()) - 1; l >= 1; l--)
    for (int id : levels[l]) below[boxes[id].parent] += below[id];
  // deletions: the first box under max_leaf dofs on the point's path (old
  // coordinates) is merged later; its leaf loses its compression
  // (quadtree.cpp:504-533)
  std::vector<int> sparse;
  std::vector<char> is_sparse(boxes.size(), 0);
  for (int d : deletions) {
    const double x = old_pts[2 * static_cast<size_t>(d)], y = old_pts[2 * static_cast<size_t>(d) + 1];
    int c = root;
    bool path_marked = false;
    while (!boxes[c].leaf) {
      if (below[c] < max_leaf_ && !path_marked) {
        path_marked = true;
        if (!is_sparse[c]) {
          is_sparse[c] = 1;
          sparse.push_back(c);
        }
      }
      c = boxes[c].child[pick_child(boxes[c], x, y)];
    }
    mark_up(c);
  }
  // split over-full leaves, merge sparse subtrees (their subtrees are
  // disjoint, so the order is immaterial), rebuild the neighbour lists
  // (quadtree.cpp:535-559)
  pts_ = new_pts;
  for (int b : bursting)
    if (boxes[b].leaf && static_cast<int>(boxes[b].original.size()) > max_leaf_) subdivide(b);
  for (int b : sparse) consolidate(b);
  for (Box& b : boxes) b.nbr.clear();
  neighbor_lists();
  pts_ = nullptr;
}

}  // namespace kib
