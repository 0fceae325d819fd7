// CPU restatement of the reference recursive-skeletonization solver.
//
// TEST INFRASTRUCTURE ONLY (the oracle).  Only tests/, __graft_entry__.smoke
// and bench.py's CPU arm load it; the GPU product never does.
//
// It restates, in plain C++ with no BLAS/LAPACK dependency, the reference
// path (paths relative to the reference repository):
//   * quadtree build + neighbour lists     quadtree.cpp:27-285
//   * active / near dof bookkeeping        quadtree.cpp:656-720
//   * kernel entries, ID matrix, proxies   kernel.cpp:11-357
//   * interpolative decomposition          ki_mat.cpp:502-541 (dgeqp3 + dtrtrs)
//   * skeletonize / decouple / updates     skel_factorization.cpp:32-294
//   * solve sweeps, multiply-connected     skel_factorization.cpp:297-551
//   * border matrices, solve API           linear_solve.cpp:18-180
// Floating-point expressions keep the reference's evaluation order so that
// matrix entries agree bit for bit with the reference build on the same
// compiler; LAPACK's dgeqp3 (via dlaqp2), dgetrf (via dgetf2) and dgetrs are
// restated from their published reference-LAPACK algorithms.
#include "ki_oracle.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

constexpr int kNumProxy = 128;          // kernel.h:10
constexpr double kRadiusRatio = 1.5;    // kernel.h:11
constexpr int kMinDofsToCompress = 16;  // skel_factorization.h:11

// ---------------------------------------------------------------- dense
struct Mat {
  int h = 0, w = 0;
  std::vector<double> a;
  Mat() = default;
  Mat(int h_, int w_) : h(h_), w(w_), a(static_cast<size_t>(h_) * w_, 0.0) {}
  double& operator()(int i, int j) { return a[i + static_cast<size_t>(h) * j]; }
  double operator()(int i, int j) const {
    return a[i + static_cast<size_t>(h) * j];
  }
};

Mat matmul(const Mat& A, const Mat& B) {  // cblas_dgemm NN (ki_mat.cpp:310-317)
  Mat C(A.h, B.w);
  for (int j = 0; j < B.w; j++) {
    for (int l = 0; l < A.w; l++) {
      double b = B(l, j);
      if (b == 0.0) continue;
      const double* ac = &A.a[static_cast<size_t>(A.h) * l];
      double* cc = &C.a[static_cast<size_t>(C.h) * j];
      for (int i = 0; i < A.h; i++) cc[i] += ac[i] * b;
    }
  }
  return C;
}

Mat transpose(const Mat& A) {
  Mat B(A.w, A.h);
  for (int j = 0; j < A.w; j++)
    for (int i = 0; i < A.h; i++) B(j, i) = A(i, j);
  return B;
}

Mat sub(const Mat& A, const Mat& B) {
  Mat C = A;
  for (size_t i = 0; i < C.a.size(); i++) C.a[i] = A.a[i] - B.a[i];
  return C;
}

Mat gather(const Mat& A, const std::vector<int>& I, const std::vector<int>& J) {
  Mat B(static_cast<int>(I.size()), static_cast<int>(J.size()));
  for (size_t j = 0; j < J.size(); j++)
    for (size_t i = 0; i < I.size(); i++) B(i, j) = A(I[i], J[j]);
  return B;
}

Mat rows(const Mat& A, const std::vector<int>& I) {
  Mat B(static_cast<int>(I.size()), A.w);
  for (int j = 0; j < A.w; j++)
    for (size_t i = 0; i < I.size(); i++) B(i, j) = A(I[i], j);
  return B;
}

void scatter_rows(Mat* A, const std::vector<int>& I, const Mat& B) {
  for (int j = 0; j < A->w; j++)
    for (size_t i = 0; i < I.size(); i++) (*A)(I[i], j) = B(i, j);
}

// dgetf2: unblocked right-looking LU with partial pivoting (first maximum).
void lu_factor(Mat* A, std::vector<int>* piv) {
  int n = A->h;
  piv->assign(n, 0);
  for (int j = 0; j < std::min(A->h, A->w); j++) {
    int p = j;
    double best = std::fabs((*A)(j, j));
    for (int i = j + 1; i < n; i++) {
      double v = std::fabs((*A)(i, j));
      if (v > best) { best = v; p = i; }
    }
    (*piv)[j] = p;
    if ((*A)(p, j) != 0.0) {
      if (p != j)
        for (int c = 0; c < A->w; c++) std::swap((*A)(j, c), (*A)(p, c));
      double inv = 1.0 / (*A)(j, j);
      for (int i = j + 1; i < n; i++) (*A)(i, j) *= inv;
    }
    for (int c = j + 1; c < A->w; c++) {
      double u = (*A)(j, c);
      if (u == 0.0) continue;
      for (int i = j + 1; i < n; i++) (*A)(i, c) -= (*A)(i, j) * u;
    }
  }
}

// dgetrs 'N': B <- A^{-1} B with A = P L U from lu_factor.
void lu_solve(const Mat& LU, const std::vector<int>& piv, Mat* B) {
  int n = LU.h;
  for (int c = 0; c < B->w; c++) {
    double* b = &B->a[static_cast<size_t>(B->h) * c];
    for (int i = 0; i < n; i++)
      if (piv[i] != i) std::swap(b[i], b[piv[i]]);
    for (int k = 0; k < n; k++) {
      double v = b[k];
      if (v != 0.0)
        for (int i = k + 1; i < n; i++) b[i] -= v * LU(i, k);
    }
    for (int k = n - 1; k >= 0; k--) {
      if (b[k] != 0.0) {
        b[k] /= LU(k, k);
        double v = b[k];
        for (int i = 0; i < k; i++) b[i] -= v * LU(i, k);
      }
    }
  }
}

// dgetrs 'T': B <- A^{-T} B.
void lu_solve_t(const Mat& LU, const std::vector<int>& piv, Mat* B) {
  int n = LU.h;
  for (int c = 0; c < B->w; c++) {
    double* b = &B->a[static_cast<size_t>(B->h) * c];
    for (int k = 0; k < n; k++) {  // U^T y = b
      double s = b[k];
      for (int i = 0; i < k; i++) s -= LU(i, k) * b[i];
      b[k] = s / LU(k, k);
    }
    for (int k = n - 1; k >= 0; k--) {  // L^T z = y
      double s = b[k];
      for (int i = k + 1; i < n; i++) s -= LU(i, k) * b[i];
      b[k] = s;
    }
    for (int i = n - 1; i >= 0; i--)
      if (piv[i] != i) std::swap(b[i], b[piv[i]]);
  }
}

// ---------------------------------------------- interpolative decomposition
double nrm2(int n, const double* x) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s += x[i] * x[i];
  return std::sqrt(s);
}

double lapy2(double x, double y) {  // dlapy2
  double xa = std::fabs(x), ya = std::fabs(y);
  double w = std::max(xa, ya), z = std::min(xa, ya);
  if (z == 0.0) return w;
  return w * std::sqrt(1.0 + (z / w) * (z / w));
}

// dgeqp3 through its unblocked kernel dlaqp2 on an m x n column-major A.
// Columns are physically swapped as LAPACK does; jpvt gets 0-based pivots.
void qrcp(int m, int n, double* A, std::vector<int>* jpvt) {
  const double tol3z = std::sqrt(0.5 * 2.220446049250313e-16);
  std::vector<double> vn1(n), vn2(n), work(n);
  jpvt->resize(n);
  for (int j = 0; j < n; j++) {
    vn1[j] = vn2[j] = nrm2(m, A + static_cast<size_t>(m) * j);
    (*jpvt)[j] = j;
  }
  auto col = [&](int j) { return A + static_cast<size_t>(m) * j; };
  int mn = std::min(m, n);
  for (int i = 0; i < mn; i++) {
    int pvt = i;
    for (int j = i + 1; j < n; j++)
      if (vn1[j] > vn1[pvt]) pvt = j;
    if (pvt != i) {
      std::swap_ranges(col(pvt), col(pvt) + m, col(i));
      std::swap((*jpvt)[pvt], (*jpvt)[i]);
      vn1[pvt] = vn1[i];
      vn2[pvt] = vn2[i];
    }
    // dlarfg on A(i:m, i)
    double* ci = col(i);
    double tau = 0.0;
    if (i < m - 1) {
      double alpha = ci[i];
      double xnorm = nrm2(m - i - 1, ci + i + 1);
      if (xnorm != 0.0) {
        double beta = -std::copysign(lapy2(alpha, xnorm), alpha);
        tau = (beta - alpha) / beta;
        double scal = 1.0 / (alpha - beta);
        for (int r = i + 1; r < m; r++) ci[r] *= scal;
        ci[i] = beta;
      }
    }
    // dlarf: apply H(i) = I - tau v v^T to A(i:m, i+1:n) from the left
    if (i < n - 1 && tau != 0.0) {
      double aii = ci[i];
      ci[i] = 1.0;
      for (int j = i + 1; j < n; j++) {
        const double* cj = col(j);
        double s = 0.0;
        for (int r = i; r < m; r++) s += cj[r] * ci[r];
        work[j] = s;
      }
      for (int j = i + 1; j < n; j++) {
        double* cj = col(j);
        double t = -tau * work[j];
        for (int r = i; r < m; r++) cj[r] += ci[r] * t;
      }
      ci[i] = aii;
    }
    // partial column norm update
    for (int j = i + 1; j < n; j++) {
      if (vn1[j] != 0.0) {
        double temp = std::fabs(col(j)[i]) / vn1[j];
        temp = 1.0 - temp * temp;
        temp = std::max(temp, 0.0);
        double q = vn1[j] / vn2[j];
        double temp2 = temp * (q * q);
        if (temp2 <= tol3z) {
          if (i < m - 1) {
            vn1[j] = nrm2(m - i - 1, col(j) + i + 1);
            vn2[j] = vn1[j];
          } else {
            vn1[j] = 0.0;
            vn2[j] = 0.0;
          }
        } else {
          vn1[j] *= std::sqrt(temp);
        }
      }
    }
  }
}

// ki_Mat::id (ki_mat.cpp:502-541): returns the rank k (0 = not compressible),
// the pivots p, and T = R11^{-1} R12 (k x (n-k)).
int interp_decomp(Mat A, double tol, std::vector<int>* p, Mat* T) {
  int m = A.h, n = A.w;
  std::vector<int> jpvt;
  qrcp(m, n, A.a.data(), &jpvt);
  int k = 0;
  double thresh = std::fabs(tol * A(0, 0));
  for (int i = 1; i < std::min(m, n); i++) {
    if (std::fabs(A(i, i)) < thresh) { k = i; break; }
  }
  if (k == 0) return 0;
  *p = jpvt;
  int r = n - k;
  *T = Mat(k, r);
  for (int c = 0; c < r; c++) {  // dtrsm Left/Upper/NoTrans/NonUnit
    double* b = &T->a[static_cast<size_t>(k) * c];
    for (int i = 0; i < k; i++) b[i] = A(i, k + c);
    for (int q = k - 1; q >= 0; q--) {
      if (b[q] != 0.0) {
        b[q] /= A(q, q);
        double v = b[q];
        for (int i = 0; i < q; i++) b[i] -= v * A(i, q);
      }
    }
  }
  return k;
}

// ------------------------------------------------------------------ geometry
struct Hole {
  double cx, cy, r;
  int num_nodes;
};

struct Problem {
  int pde = 0, sol_dim = 1;  // pde: 0 Laplace, 1 Laplace-Neumann, 2 Stokes
  std::vector<double> pts, nrm, curv, w;
  std::vector<Hole> holes;
  int n_points() const { return static_cast<int>(w.size()); }
  int n_dofs() const { return n_points() * sol_dim; }

  // Kernel::laplace (kernel.cpp:11-36), boundary or forward target.
  double laplace(double r1, double r2, double sw, double sc, double sn1,
                 double sn2, double tn1, double tn2, bool fwd) const {
    if (pde == 0) {
      if (r1 == 0. && r2 == 0.) return 0.5 + 0.5 * sc * sw * (1.0 / (2 * M_PI));
      return -sw * (1.0 / (2 * M_PI)) * (r1 * sn1 + r2 * sn2) /
             (r1 * r1 + r2 * r2);
    }
    if (fwd) return sw * (1.0 / (2 * M_PI)) * std::log(std::sqrt(r1 * r1 + r2 * r2));
    if (r1 == 0. && r2 == 0.) return sw - 0.5 + 0.5 * sc * sw * (1.0 / (2 * M_PI));
    return sw + sw * (1.0 / (2 * M_PI)) * (r1 * tn1 + r2 * tn2) /
                    (r1 * r1 + r2 * r2);
  }

  // Entry (tgt, src) of the boundary operator; tp/tn override the target
  // point for forward evaluation (tn = 0 there), kernel.cpp:47-96,114-150.
  double entry(int tgt, int src, const double* tp_fwd = nullptr) const {
    bool fwd = tp_fwd != nullptr;
    if (sol_dim == 1) {
      double sp0 = pts[2 * src], sp1 = pts[2 * src + 1];
      double tp0 = fwd ? tp_fwd[0] : pts[2 * tgt];
      double tp1 = fwd ? tp_fwd[1] : pts[2 * tgt + 1];
      double tn0 = fwd ? 0.0 : nrm[2 * tgt], tn1 = fwd ? 0.0 : nrm[2 * tgt + 1];
      return laplace(tp0 - sp0, tp1 - sp1, w[src], curv[src], nrm[2 * src],
                     nrm[2 * src + 1], tn0, tn1, fwd);
    }
    const double scale = 1.0 / (M_PI);
    int sj = src / 2, ti = tgt / 2;
    double sp[2] = {pts[2 * sj], pts[2 * sj + 1]};
    double sn[2] = {nrm[2 * sj], nrm[2 * sj + 1]};
    double sw = w[sj], sc = curv[sj];
    double tp[2], tn[2];
    if (fwd) {
      tp[0] = tp_fwd[0]; tp[1] = tp_fwd[1]; tn[0] = 0; tn[1] = 0;
    } else {
      tp[0] = pts[2 * ti]; tp[1] = pts[2 * ti + 1];
      tn[0] = nrm[2 * ti]; tn[1] = nrm[2 * ti + 1];
    }
    if (tp[0] == sp[0] && tp[1] == sp[1]) {
      int parity = (tgt + src + 1) % 2;
      return -0.5 * parity + (1 - 2 * parity) * 0.5 * sc * sw * scale *
                                 sn[(tgt + 1) % 2] * sn[(src + 1) % 2] +
             sw * tn[tgt % 2] * sn[src % 2];
    }
    double r[2] = {tp[0] - sp[0], tp[1] - sp[1]};
    double rr = r[0] * r[0] + r[1] * r[1];
    return sw * scale * (r[0] * sn[0] + r[1] * sn[1]) / (rr * rr) *
               r[tgt % 2] * r[src % 2] +
           sw * tn[tgt % 2] * sn[src % 2];
  }

  Mat block(const std::vector<int>& I, const std::vector<int>& J) const {
    Mat M(static_cast<int>(I.size()), static_cast<int>(J.size()));
    for (size_t j = 0; j < J.size(); j++)
      for (size_t i = 0; i < I.size(); i++) M(i, j) = entry(I[i], J[j]);
    return M;
  }

  // Proxy block (kernel.cpp:238-334): rows are proxy-point interactions in
  // both directions, columns the box dofs.
  Mat proxy(double cx, double cy, double r, const std::vector<int>& box) const {
    double pw = 2.0 * M_PI * r / kNumProxy;
    std::vector<double> pp, pn;
    for (int i = 0; i < kNumProxy; i++) {
      double ang = 2 * M_PI * i * (1.0 / kNumProxy);
      pp.push_back(cx + (r + 0.0) * std::cos(ang));
      pp.push_back(cy + (r + 0.0) * std::sin(ang));
      pn.push_back(std::cos(ang));
      pn.push_back(std::sin(ang));
    }
    int np = static_cast<int>(pp.size());
    if (sol_dim == 1) {
      Mat M(np, static_cast<int>(box.size()));
      for (size_t j = 0; j < box.size(); j++) {
        int b = box[j];
        double bp1 = pts[2 * b], bp2 = pts[2 * b + 1];
        double bn1 = nrm[2 * b], bn2 = nrm[2 * b + 1], bw = w[b];
        for (int i = 0; i < np; i += 2) {
          double r0 = pp[i] - bp1, r1 = pp[i + 1] - bp2;
          M(i / 2, j) = laplace(r0, r1, bw, 0, bn1, bn2, pn[i], pn[i + 1], false);
          M(np / 2 + i / 2, j) =
              laplace(-r0, -r1, pw, 0, pn[i], pn[i + 1], bn1, bn2, false);
        }
      }
      return M;
    }
    const double scale = 1.0 / (M_PI);
    Mat M(2 * np, static_cast<int>(box.size()));
    for (size_t j = 0; j < box.size(); j++) {
      int src = box[j], sj = src / 2;
      double sp[2] = {pts[2 * sj], pts[2 * sj + 1]};
      double sn[2] = {nrm[2 * sj], nrm[2 * sj + 1]};
      double sw = w[sj];
      for (int i = 0; i < np; i += 2) {
        double tn[2] = {pn[i], pn[i + 1]};
        double r[2] = {pp[i] - sp[0], pp[i + 1] - sp[1]};
        double rr = r[0] * r[0] + r[1] * r[1];
        double pot = sw * scale * (r[0] * sn[0] + r[1] * sn[1]) / (rr * rr);
        M(i, j) = pot * r[0] * r[src % 2] + sw * tn[0] * sn[src % 2];
        M(i + 1, j) = pot * r[1] * r[src % 2] + sw * tn[1] * sn[src % 2];
        pot = -pw * scale * (r[0] * tn[0] + r[1] * tn[1]) / (rr * rr);
        M(np + i, j) = pot * r[0] * r[src % 2] + pw * sn[src % 2] * tn[0];
        M(np + i + 1, j) = pot * r[1] * r[src % 2] + pw * sn[src % 2] * tn[1];
      }
    }
    return M;
  }
};

// ------------------------------------------------------------------ quadtree
struct Node {
  int level = 0, parent = -1;
  int children[4] = {-1, -1, -1, -1};
  bool is_leaf = true, compressed = false;
  double corners[8] = {0};
  double side = 0;
  std::vector<int> neighbors, original, active, near, skel, redundant, perm;
  Mat T, L, U, X_lu, schur;
  std::vector<int> X_piv;
  int id_m = 0;
};

struct Tree {
  int sol_dim = 1, max_leaf = 32;
  double min = 0, max = 0;
  std::vector<double> pts;
  std::vector<Node> nodes;
  std::vector<std::vector<int>> levels;

  int child_of(const Node& n, double x, double y) const {
    double midx = ((n.corners[6] - n.corners[0]) / 2.0) + n.corners[0];
    double midy = ((n.corners[3] - n.corners[1]) / 2.0) + n.corners[1];
    if (x < midx && y < midy) return 0;
    if (x < midx && y >= midy) return 1;
    if (x >= midx && y < midy) return 3;
    return 2;
  }

  void subdivide(int id) {  // quadtree.cpp:203-285
    nodes[id].is_leaf = false;
    double c[8];
    std::memcpy(c, nodes[id].corners, sizeof(c));
    double midx = ((c[6] - c[0]) / 2.0) + c[0];
    double midy = ((c[3] - c[1]) / 2.0) + c[1];
    int lvl = nodes[id].level + 1;
    if (static_cast<int>(levels.size()) < lvl + 1) levels.emplace_back();
    int kids[4];
    for (int i = 0; i < 4; i++) {
      Node ch;
      std::memcpy(ch.corners, c, sizeof(c));
      ch.level = lvl;
      ch.side = nodes[id].side / 2.0;
      ch.parent = id;
      kids[i] = static_cast<int>(nodes.size());
      nodes.push_back(ch);
      levels[lvl].push_back(kids[i]);
    }
    Node* k = &nodes[kids[0]];
    k->corners[3] = midy; k->corners[4] = midx; k->corners[5] = midy; k->corners[6] = midx;
    k = &nodes[kids[1]];
    k->corners[1] = midy; k->corners[4] = midx; k->corners[6] = midx; k->corners[7] = midy;
    k = &nodes[kids[2]];
    k->corners[0] = midx; k->corners[1] = midy; k->corners[2] = midx; k->corners[7] = midy;
    k = &nodes[kids[3]];
    k->corners[0] = midx; k->corners[2] = midx; k->corners[3] = midy; k->corners[5] = midy;
    for (int i = 0; i < 4; i++) nodes[id].children[i] = kids[i];
    const std::vector<int> orig = nodes[id].original;
    for (size_t q = 0; q < orig.size(); q += sol_dim) {
      int dof = orig[q];
      int pt = dof / sol_dim;
      int ci = child_of(nodes[id], pts[2 * pt], pts[2 * pt + 1]);
      for (int s = 0; s < sol_dim; s++)
        nodes[kids[ci]].original.push_back(dof + s);
    }
    for (int i = 0; i < 4; i++)
      if (static_cast<int>(nodes[kids[i]].original.size()) > max_leaf)
        subdivide(kids[i]);
  }

  void add(int id, double x, double y, int pt) {  // quadtree.cpp:164-197
    for (int s = 0; s < sol_dim; s++)
      nodes[id].original.push_back(sol_dim * pt + s);
    int ci = child_of(nodes[id], x, y);
    int ch = nodes[id].children[ci];
    if (ch >= 0) {
      add(ch, x, y, pt);
    } else if (nodes[id].is_leaf &&
               static_cast<int>(nodes[id].original.size()) > max_leaf) {
      subdivide(id);
    }
  }

  void descendant_neighbors(int big, int small) {  // quadtree.cpp:119-161
    const Node& B = nodes[big];
    double top = B.corners[3], bottom = B.corners[1];
    double left = B.corners[0], right = B.corners[4];
    for (int i = 0; i < 8; i += 2) {
      double x = nodes[small].corners[i], y = nodes[small].corners[i + 1];
      bool hit = false;
      if (x > left && x < right) {
        if (std::fabs(y - top) < 1e-14 || std::fabs(y - bottom) < 1e-14) hit = true;
      }
      // the reference tests y < top && y < bottom here (quadtree.cpp:143)
      if (!hit && y < top && y < bottom) {
        if (std::fabs(x - left) < 1e-14 || std::fabs(x - right) < 1e-14) hit = true;
      }
      if (hit) {
        nodes[big].neighbors.push_back(small);
        nodes[small].neighbors.push_back(big);
        break;
      }
    }
    for (int c = 0; c < 4; c++) {
      int ch = nodes[small].children[c];
      if (ch >= 0) descendant_neighbors(big, ch);
    }
  }

  void neighbor_lists() {  // quadtree.cpp:27-69
    for (size_t l = 0; l < levels.size(); l++) {
      for (int a : levels[l]) {
        int par = nodes[a].parent;
        if (par >= 0) {
          for (int c = 0; c < 4; c++) {
            int sib = nodes[par].children[c];
            if (sib != a) nodes[a].neighbors.push_back(sib);
          }
          std::vector<int> pn = nodes[par].neighbors;
          for (int q : pn) {
            for (int c = 0; c < 4; c++) {
              int cousin = nodes[q].children[c];
              if (cousin < 0) continue;
              if (nodes[cousin].level != nodes[a].level) continue;
              double dist = std::sqrt(
                  std::pow(nodes[a].corners[0] - nodes[cousin].corners[0], 2) +
                  std::pow(nodes[a].corners[1] - nodes[cousin].corners[1], 2));
              if (dist < nodes[a].side * std::sqrt(2) + 1e-5)
                nodes[a].neighbors.push_back(cousin);
            }
          }
        }
        if (nodes[a].is_leaf) {
          for (size_t q = 0; q < nodes[a].neighbors.size(); q++) {
            int nb = nodes[a].neighbors[q];
            if (nodes[nb].level != nodes[a].level) continue;
            for (int c = 0; c < 4; c++) {
              int ch = nodes[nb].children[c];
              if (ch >= 0) descendant_neighbors(a, ch);
            }
          }
        }
      }
    }
  }

  void build(const std::vector<double>& points, int sd, int leaf) {
    pts = points;
    sol_dim = sd;
    max_leaf = leaf;
    min = pts[0];
    max = pts[0];
    for (double v : pts) {
      if (v < min) min = v;
      if (v > max) max = v;
    }
    double lo = min - 0.01, hi = max + 0.01;
    Node root;
    double c[8] = {lo, lo, lo, hi, hi, hi, hi, lo};
    std::memcpy(root.corners, c, sizeof(c));
    root.side = hi - lo;
    nodes.push_back(root);
    levels.push_back({0});
    for (size_t i = 0; i < pts.size(); i += 2)
      add(0, pts[i], pts[i + 1], static_cast<int>(i / 2));
    neighbor_lists();
  }

  void refresh_box(int id) {  // quadtree.cpp:694-720
    Node& n = nodes[id];
    n.skel.clear();
    n.redundant.clear();
    n.active.clear();
    if (!n.is_leaf) {
      for (int c = 0; c < 4; c++) {
        const Node& ch = nodes[n.children[c]];
        const std::vector<int>& src = ch.compressed ? ch.skel : ch.active;
        n.active.insert(n.active.end(), src.begin(), src.end());
      }
    } else {
      n.active = n.original;
    }
  }

  void refresh_level(int l) {  // quadtree.cpp:664-691
    for (int id : levels[l])
      if (!nodes[id].compressed) refresh_box(id);
    for (int id : levels[l]) {
      Node& a = nodes[id];
      a.near.clear();
      for (int nb : a.neighbors) {
        const Node& b = nodes[nb];
        if (b.level > a.level) continue;
        const std::vector<int>& src = b.is_leaf ? b.original : b.active;
        a.near.insert(a.near.end(), src.begin(), src.end());
      }
    }
  }
};

// ---------------------------------------------------------------- solver
struct Solver {
  Problem pr;
  Tree tree;
  double tol = 1e-10;
  int threads = 1;
  std::vector<int> allskel, allred;
  Mat allskel_lu;
  std::vector<int> allskel_piv;
  Mat U, Psi, S_lu;  // border (holes only)
  std::vector<int> S_piv;
  bool holes() const { return U.w > 0; }

  // Kernel::get_id_mat (kernel.cpp:153-235).
  Mat id_matrix(int id) const {
    const Node& n = tree.nodes[id];
    double cx = n.corners[0] + n.side / 2.0;
    double cy = n.corners[1] + n.side / 2.0;
    std::vector<int> outside;
    if (n.level == 1 || n.level == 2) {
      for (int o : tree.levels[n.level])
        if (o != id)
          outside.insert(outside.end(), tree.nodes[o].active.begin(),
                         tree.nodes[o].active.end());
      if (n.level == 2)
        for (int o : tree.levels[1])
          if (tree.nodes[o].is_leaf)
            outside.insert(outside.end(), tree.nodes[o].original.begin(),
                           tree.nodes[o].original.end());
      int I = static_cast<int>(outside.size());
      Mat M(2 * I, static_cast<int>(n.active.size()));
      Mat a = pr.block(outside, n.active), b = pr.block(n.active, outside);
      for (int j = 0; j < M.w; j++)
        for (int i = 0; i < I; i++) {
          M(i, j) = a(i, j);
          M(I + i, j) = b(j, i);
        }
      return M;
    }
    std::vector<int> inner;
    for (int dof : n.near) {
      int pt = dof / pr.sol_dim;
      double x = pr.pts[2 * pt], y = pr.pts[2 * pt + 1];
      double dist = std::sqrt(std::pow(cx - x, 2) + std::pow(cy - y, 2));
      if (dist < kRadiusRatio * n.side) inner.push_back(dof);
    }
    Mat px = pr.proxy(cx, cy, n.side * kRadiusRatio, n.active);
    int I = static_cast<int>(inner.size());
    Mat M(2 * I + px.h, static_cast<int>(n.active.size()));
    Mat a = pr.block(inner, n.active), b = pr.block(n.active, inner);
    for (int j = 0; j < M.w; j++) {
      for (int i = 0; i < I; i++) {
        M(i, j) = a(i, j);
        M(I + i, j) = b(j, i);
      }
      for (int i = 0; i < px.h; i++) M(2 * I + i, j) = px(i, j);
    }
    return M;
  }

  // get_update / get_descendents_updates (skel_factorization.cpp:246-294).
  void add_update(Mat* upd, const std::vector<int>& BN, int id) const {
    const Node& d = tree.nodes[id];
    std::vector<int> bi, si;
    for (size_t s = 0; s < d.skel.size(); s++)
      for (size_t b = 0; b < BN.size(); b++)
        if (BN[b] == d.skel[s]) {
          si.push_back(static_cast<int>(s));
          bi.push_back(static_cast<int>(b));
        }
    for (size_t i = 0; i < bi.size(); i++)
      for (size_t j = 0; j < bi.size(); j++)
        (*upd)(bi[i], bi[j]) += d.schur(si[i], si[j]);
  }
  void descendant_updates(Mat* upd, const std::vector<int>& BN, int id) const {
    for (int c = 0; c < 4; c++) {
      int ch = tree.nodes[id].children[c];
      if (tree.nodes[ch].compressed) add_update(upd, BN, ch);
      if (!tree.nodes[ch].is_leaf) descendant_updates(upd, BN, ch);
    }
  }

  // id_compress + decouple (skel_factorization.cpp:32-91).
  void compress(int id) {
    Node& n = tree.nodes[id];
    Mat A = id_matrix(id);
    n.id_m = A.h;
    if (A.h == 0) return;
    std::vector<int> p;
    Mat T;
    int k = interp_decomp(A, tol, &p, &T);
    if (k == 0) return;
    n.T = T;
    n.perm = p;
    for (int i = 0; i < k; i++) n.skel.push_back(n.active[p[i]]);
    for (size_t i = k; i < p.size(); i++) n.redundant.push_back(n.active[p[i]]);
    int nb = static_cast<int>(n.active.size()), r = nb - k;
    Mat upd(nb, nb);
    if (!n.is_leaf) descendant_updates(&upd, n.active, id);
    Mat K = sub(pr.block(n.active, n.active), upd);
    std::vector<int> s(p.begin(), p.begin() + k), rr(p.begin() + k, p.end());
    Mat Tt = transpose(T);
    Mat K_r_sn = sub(gather(K, rr, s), matmul(Tt, gather(K, s, s)));
    Mat X = sub(sub(gather(K, rr, rr), matmul(Tt, gather(K, s, rr))),
                matmul(K_r_sn, T));
    Mat K_sn_r = sub(gather(K, s, rr), matmul(gather(K, s, s), T));
    lu_factor(&X, &n.X_piv);
    n.X_lu = X;
    Mat Lt = transpose(K_sn_r);  // L = K_sn_r X^{-1}: X^T L^T = K_sn_r^T
    lu_solve_t(n.X_lu, n.X_piv, &Lt);
    n.L = transpose(Lt);
    n.U = K_r_sn;
    lu_solve(n.X_lu, n.X_piv, &n.U);
    n.schur = matmul(n.L, K_r_sn);
    (void)r;
    n.compressed = true;
  }

  // apply_sweep_matrix (skel_factorization.cpp:297-318): vec(b) += M vec(a)
  // (M^T when transpose), for every column of vec.
  static void sweep(const Mat& M, Mat* vec, const std::vector<int>& a,
                    const std::vector<int>& b, bool tr, double sign) {
    if (a.empty() || b.empty()) return;
    Mat va = rows(*vec, a);
    Mat prod = tr ? matmul(transpose(M), va) : matmul(M, va);
    for (int j = 0; j < vec->w; j++)
      for (size_t i = 0; i < b.size(); i++) (*vec)(b[i], j) += sign * prod(i, j);
  }

  void diag_inv(const Node& n, Mat* vec, const std::vector<int>& range) const {
    if (range.empty()) return;
    Mat v = rows(*vec, range);
    lu_solve(n.X_lu, n.X_piv, &v);
    scatter_rows(vec, range, v);
  }

  void up_sweep(Mat* x, bool use_U_for_skel) const {
    for (int l = static_cast<int>(tree.levels.size()) - 1; l >= 0; l--) {
      const auto& lv = tree.levels[l];
#pragma omp parallel for num_threads(threads) schedule(dynamic)
      for (int q = 0; q < static_cast<int>(lv.size()); q++) {
        const Node& n = tree.nodes[lv[q]];
        if (!n.compressed) continue;
        sweep(n.T, x, n.skel, n.redundant, true, -1.0);
        if (use_U_for_skel)
          sweep(n.U, x, n.redundant, n.skel, true, -1.0);
        else
          sweep(n.L, x, n.redundant, n.skel, false, -1.0);
      }
    }
  }

  void down_sweep(Mat* x) const {
    for (size_t l = 0; l < tree.levels.size(); l++) {
      const auto& lv = tree.levels[l];
#pragma omp parallel for num_threads(threads) schedule(dynamic)
      for (int q = static_cast<int>(lv.size()) - 1; q >= 0; q--) {
        const Node& n = tree.nodes[lv[q]];
        if (!n.compressed) continue;
        sweep(n.U, x, n.skel, n.redundant, false, -1.0);
        sweep(n.T, x, n.redundant, n.skel, false, -1.0);
      }
    }
  }

  // D^{-1} on a matrix indexed by position in allred (skel_factorization.cpp:272-289).
  void dinv_red(Mat* v, const std::unordered_map<int, int>& red_pos) const {
    std::vector<int> all;
    for (int l = static_cast<int>(tree.levels.size()) - 1; l >= 0; l--)
      for (int id : tree.levels[l]) all.push_back(id);
#pragma omp parallel for num_threads(threads) schedule(dynamic)
    for (int q = 0; q < static_cast<int>(all.size()); q++) {
      const Node& n = tree.nodes[all[q]];
      if (n.redundant.empty() || !n.compressed) continue;
      std::vector<int> small;
      for (int d : n.redundant) small.push_back(red_pos.at(d));
      diag_inv(n, v, small);
    }
  }

  Mat mod_U, mod_PsiT;
  std::unordered_map<int, int> red_pos;

  void skeletonize() {  // skel_factorization.cpp:94-243
    int L = static_cast<int>(tree.levels.size());
    for (int l = L - 1; l > 0; l--) {
      tree.refresh_level(l);
      const auto& lv = tree.levels[l];
#pragma omp parallel for num_threads(threads) schedule(dynamic)
      for (int q = 0; q < static_cast<int>(lv.size()); q++) {
        Node& n = tree.nodes[lv[q]];
        if (n.compressed ||
            static_cast<int>(n.active.size()) < kMinDofsToCompress)
          continue;
        compress(lv[q]);
      }
    }
    for (int l = L - 1; l >= 0; l--) tree.refresh_level(l);
    allskel = tree.nodes[0].active;
    Mat allskel_mat;
    if (!allskel.empty()) {
      Mat upd(static_cast<int>(allskel.size()), static_cast<int>(allskel.size()));
      if (!tree.nodes[0].is_leaf) descendant_updates(&upd, allskel, 0);
      allskel_mat = sub(pr.block(allskel, allskel), upd);
    }
    allskel_lu = allskel_mat;
    if (!holes()) {
      lu_factor(&allskel_lu, &allskel_piv);
      return;
    }
    std::vector<int> sorted = allskel;
    std::sort(sorted.begin(), sorted.end());
    size_t si = 0;
    allred.clear();
    for (int i = 0; i < pr.n_dofs(); i++) {
      if (si < sorted.size() && i == sorted[si]) si++;
      else allred.push_back(i);
    }
    for (size_t i = 0; i < allred.size(); i++)
      red_pos[allred[i]] = static_cast<int>(i);
    mod_U = U;
    mod_PsiT = transpose(Psi);
    up_sweep(&mod_U, false);
    up_sweep(&mod_PsiT, true);
    Mat Dinv_C = rows(mod_U, allred);
    dinv_red(&Dinv_C, red_pos);
    int ns = static_cast<int>(allskel.size()), nh = Psi.h;
    Mat S(ns + nh, ns + nh);
    for (int j = 0; j < ns; j++)
      for (int i = 0; i < ns; i++) S(i, j) = allskel_mat(i, j);
    for (int j = 0; j < ns; j++)
      for (int i = 0; i < nh; i++) S(ns + i, j) = mod_PsiT(allskel[j], i);
    for (int j = 0; j < nh; j++)
      for (int i = 0; i < ns; i++) S(i, ns + j) = mod_U(allskel[i], j);
    Mat PsiR(nh, static_cast<int>(allred.size()));
    for (size_t c = 0; c < allred.size(); c++)
      for (int i = 0; i < nh; i++) PsiR(i, c) = mod_PsiT(allred[c], i);
    Mat corr = matmul(PsiR, Dinv_C);
    for (int j = 0; j < nh; j++)
      for (int i = 0; i < nh; i++)
        S(ns + i, ns + j) = (i == j ? -1.0 : 0.0) - corr(i, j);
    S_lu = S;
    lu_factor(&S_lu, &S_piv);
  }

  void solve(const double* f, double* mu, double* alpha) const {
    int N = pr.n_dofs();
    Mat x(N, 1);
    std::memcpy(x.a.data(), f, sizeof(double) * N);
    if (!holes()) {  // skel_factorization.cpp:341-403
      up_sweep(&x, false);
      std::vector<int> all;
      for (int l = static_cast<int>(tree.levels.size()) - 1; l >= 0; l--)
        for (int id : tree.levels[l]) all.push_back(id);
#pragma omp parallel for num_threads(threads) schedule(dynamic)
      for (int q = 0; q < static_cast<int>(all.size()); q++) {
        const Node& n = tree.nodes[all[q]];
        if (n.redundant.empty() || !n.compressed) continue;
        diag_inv(n, &x, n.redundant);
      }
      if (!allskel.empty()) {
        Mat v = rows(x, allskel);
        lu_solve(allskel_lu, allskel_piv, &v);
        scatter_rows(&x, allskel, v);
      }
      down_sweep(&x);
      std::memcpy(mu, x.a.data(), sizeof(double) * N);
      return;
    }
    // multiply_connected_solve (skel_factorization.cpp:406-551), with the
    // modified U / Psi of the factorization reused.
    up_sweep(&x, false);
    Mat w = rows(x, allred), z = rows(x, allskel);
    Mat Dinv_w = w;
    dinv_red(&Dinv_w, red_pos);
    int ns = static_cast<int>(allskel.size()), nh = Psi.h;
    Mat M(ns + nh, 1);
    for (int i = 0; i < ns; i++) M(i, 0) = z(i, 0);
    for (int i = 0; i < nh; i++) {
      double s = 0.0;
      for (size_t c = 0; c < allred.size(); c++)
        s += mod_PsiT(allred[c], i) * Dinv_w(c, 0);
      M(ns + i, 0) = -s;
    }
    lu_solve(S_lu, S_piv, &M);
    for (int i = 0; i < nh; i++) alpha[i] = M(ns + i, 0);
    Mat Nv = w;
    for (size_t c = 0; c < allred.size(); c++) {
      double s = 0.0;
      for (int j = 0; j < nh; j++) s += mod_U(allred[c], j) * alpha[j];
      Nv(c, 0) -= s;
    }
    dinv_red(&Nv, red_pos);
    scatter_rows(&x, allred, Nv);
    for (int i = 0; i < ns; i++) x(allskel[i], 0) = M(i, 0);
    down_sweep(&x);
    std::memcpy(mu, x.a.data(), sizeof(double) * N);
  }
};

// initialize_U_mat (linear_solve.cpp:18-64) on interleaved target points.
Mat make_U(const Problem& pr, const std::vector<double>& tgt) {
  int nh = static_cast<int>(pr.holes.size());
  if (nh == 0 || pr.pde == 1) return Mat();
  if (pr.pde == 0) {
    Mat U(static_cast<int>(tgt.size() / 2), nh);
    for (size_t i = 0; i < tgt.size(); i += 2)
      for (int h = 0; h < nh; h++) {
        double rx = tgt[i] - pr.holes[h].cx, ry = tgt[i + 1] - pr.holes[h].cy;
        U(i / 2, h) = std::log(std::sqrt(rx * rx + ry * ry));
      }
    return U;
  }
  Mat U(static_cast<int>(tgt.size()), 3 * nh);
  for (size_t i = 0; i < tgt.size(); i += 2)
    for (int h = 0; h < nh; h++) {
      double r0 = tgt[i] - pr.holes[h].cx, r1 = tgt[i + 1] - pr.holes[h].cy;
      double rn = std::sqrt(r0 * r0 + r1 * r1);
      double scale = 1.0 / (4 * M_PI);
      U(i, 3 * h) = scale * (std::log(1 / rn) + (1.0 / std::pow(rn, 2)) * r0 * r0);
      U(i + 1, 3 * h) = scale * ((1.0 / std::pow(rn, 2)) * r1 * r0);
      U(i, 3 * h + 1) = scale * ((1.0 / std::pow(rn, 2)) * r0 * r1);
      U(i + 1, 3 * h + 1) =
          scale * (std::log(1 / rn) + (1.0 / std::pow(rn, 2)) * r1 * r1);
      U(i, 3 * h + 2) = r1 * (scale / std::pow(rn, 2));
      U(i + 1, 3 * h + 2) = -r0 * (scale / std::pow(rn, 2));
    }
  return U;
}

// initialize_Psi_mat (linear_solve.cpp:67-110).
Mat make_Psi(const Problem& pr) {
  int nh = static_cast<int>(pr.holes.size());
  if (nh == 0 || pr.pde == 1) return Mat();
  int np = pr.n_points();
  Mat P(pr.pde == 0 ? nh : 3 * nh, pr.pde == 0 ? np : 2 * np);
  for (int q = 0; q < np; q++) {
    double x0 = pr.pts[2 * q], x1 = pr.pts[2 * q + 1];
    for (int h = 0; h < nh; h++) {
      double rx = x0 - pr.holes[h].cx, ry = x1 - pr.holes[h].cy;
      if (std::sqrt(rx * rx + ry * ry) < pr.holes[h].r + 1e-8) {
        if (pr.pde == 0) {
          P(h, q) = pr.w[q];
        } else {
          P(3 * h, 2 * q) = pr.w[q];
          P(3 * h + 1, 2 * q + 1) = pr.w[q];
          P(3 * h + 2, 2 * q) = pr.w[q] * x1;
          P(3 * h + 2, 2 * q + 1) = -pr.w[q] * x0;
        }
        break;
      }
    }
  }
  return P;
}

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

}  // namespace

extern "C" {

void* kiora_create(int pde, int n_points, const double* points,
                   const double* normals, const double* curvatures,
                   const double* weights, int n_holes, const double* holes,
                   int max_leaf_dofs, double id_tol, int threads,
                   double* t_factor) {
  Solver* s = new Solver();
  Problem& pr = s->pr;
  pr.pde = pde;
  pr.sol_dim = pde == 2 ? 2 : 1;
  pr.pts.assign(points, points + 2 * n_points);
  pr.nrm.assign(normals, normals + 2 * n_points);
  pr.curv.assign(curvatures, curvatures + n_points);
  pr.w.assign(weights, weights + n_points);
  for (int i = 0; i < n_holes; i++)
    pr.holes.push_back({holes[4 * i], holes[4 * i + 1], holes[4 * i + 2],
                        static_cast<int>(holes[4 * i + 3])});
  s->tol = id_tol;
  s->threads = std::max(1, threads);
  s->tree.build(pr.pts, pr.sol_dim, max_leaf_dofs);
  s->U = make_U(pr, pr.pts);
  s->Psi = make_Psi(pr);
  double t0 = now_s();
  s->skeletonize();
  if (t_factor) *t_factor = now_s() - t0;
  return s;
}

void kiora_destroy(void* h) { delete static_cast<Solver*>(h); }

int kiora_solve(void* h, const double* f, double* mu, double* alpha,
                double* t_solve) {
  Solver* s = static_cast<Solver*>(h);
  double t0 = now_s();
  s->solve(f, mu, alpha);
  if (t_solve) *t_solve = now_s() - t0;
  return s->holes() ? s->Psi.h : 0;
}

int kiora_num_levels(void* h) {
  return static_cast<int>(static_cast<Solver*>(h)->tree.levels.size());
}

int kiora_num_nodes(void* h, int level) {
  return static_cast<int>(static_cast<Solver*>(h)->tree.levels[level].size());
}

void kiora_node_info(void* h, int level, int idx, int* info, double* geom) {
  Solver* s = static_cast<Solver*>(h);
  const Node& n = s->tree.nodes[s->tree.levels[level][idx]];
  info[0] = n.is_leaf;
  info[1] = n.compressed;
  info[2] = static_cast<int>(n.original.size());
  info[3] = static_cast<int>(n.active.size());
  info[4] = static_cast<int>(n.skel.size());
  info[5] = static_cast<int>(n.redundant.size());
  info[6] = -1;
  if (n.parent >= 0) {
    const auto& pl = s->tree.levels[level - 1];
    for (size_t i = 0; i < pl.size(); i++)
      if (pl[i] == n.parent) info[6] = static_cast<int>(i);
  }
  info[7] = n.level;
  geom[0] = n.corners[0];
  geom[1] = n.corners[1];
  geom[2] = n.side;
}

void kiora_node_lists(void* h, int level, int idx, int* original, int* active,
                      int* skel, int* redundant) {
  Solver* s = static_cast<Solver*>(h);
  const Node& n = s->tree.nodes[s->tree.levels[level][idx]];
  auto cp = [](const std::vector<int>& v, int* out) {
    if (out && !v.empty()) std::memcpy(out, v.data(), sizeof(int) * v.size());
  };
  cp(n.original, original);
  cp(n.active, active);
  cp(n.skel, skel);
  cp(n.redundant, redundant);
}

void kiora_kernel_block(void* h, int nt, const int* tgt, int ns, const int* src,
                        double* out) {
  Solver* s = static_cast<Solver*>(h);
  std::vector<int> t(tgt, tgt + nt), q(src, src + ns);
  Mat m = s->pr.block(t, q);
  std::memcpy(out, m.a.data(), sizeof(double) * nt * ns);
}

void kiora_eval_targets(void* h, int nt, const double* targets,
                        const double* mu, const double* alpha, double* out) {
  Solver* s = static_cast<Solver*>(h);
  const Problem& pr = s->pr;
  int sd = pr.sol_dim, N = pr.n_dofs();
  for (int t = 0; t < nt; t++)
    for (int c = 0; c < sd; c++) {
      double acc = 0.0;
      for (int j = 0; j < N; j++)
        acc += pr.entry(sd * t + c, j, targets + 2 * t) * mu[j];
      out[sd * t + c] = acc;
    }
  if (s->holes() && alpha) {
    std::vector<double> tg(targets, targets + 2 * nt);
    Mat uf = make_U(pr, tg);
    for (int i = 0; i < uf.h; i++)
      for (int j = 0; j < uf.w; j++) out[i] += uf(i, j) * alpha[j];
  }
}

int kiora_border(void* h, double* U, double* Psi) {
  Solver* s = static_cast<Solver*>(h);
  if (!s->holes()) return 0;
  if (U) std::memcpy(U, s->U.a.data(), sizeof(double) * s->U.a.size());
  if (Psi) std::memcpy(Psi, s->Psi.a.data(), sizeof(double) * s->Psi.a.size());
  return s->U.w;
}

int kiora_allskel(void* h, int* out) {
  Solver* s = static_cast<Solver*>(h);
  if (out && !s->allskel.empty())
    std::memcpy(out, s->allskel.data(), sizeof(int) * s->allskel.size());
  return static_cast<int>(s->allskel.size());
}

void kiora_apply_dense(void* h, const double* x, double* y) {
  Solver* s = static_cast<Solver*>(h);
  const Problem& pr = s->pr;
  int N = pr.n_dofs();
  int nb = s->holes() ? s->U.w : 0;
#pragma omp parallel for num_threads(s->threads)
  for (int i = 0; i < N; i++) {
    double acc = 0.0;
    for (int j = 0; j < N; j++) acc += pr.entry(i, j) * x[j];
    for (int j = 0; j < nb; j++) acc += s->U(i, j) * x[N + j];
    y[i] = acc;
  }
  for (int i = 0; i < nb; i++) {
    double acc = -x[N + i];
    for (int j = 0; j < N; j++) acc += s->Psi(i, j) * x[j];
    y[N + i] = acc;
  }
}

int kiora_id_stats(void* h, int* out, int cap) {
  Solver* s = static_cast<Solver*>(h);
  int c = 0;
  for (size_t l = 0; l < s->tree.levels.size(); l++)
    for (int id : s->tree.levels[l]) {
      const Node& n = s->tree.nodes[id];
      if (n.id_m == 0) continue;
      if (out && c < cap) {
        out[4 * c] = static_cast<int>(l);
        out[4 * c + 1] = n.id_m;
        out[4 * c + 2] = static_cast<int>(n.active.size());
        out[4 * c + 3] = static_cast<int>(n.skel.size());
      }
      c++;
    }
  return c;
}
}
