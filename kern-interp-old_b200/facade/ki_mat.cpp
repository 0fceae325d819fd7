// kern_interp::ki_Mat of the C++ drop-in API: a host dense matrix with the
// reference's value semantics and method set (kern_interp/ki_mat.h:19-101).
// Plain loops; the solver's own dense work runs on the GPU.
#include "kern_interp/ki_mat.h"

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstring>
#include <limits>
#include <utility>

namespace kern_interp {

namespace {

double* alloc_zero(size_t n) {
  if (n == 0) return nullptr;
  double* p = new double[n];
  std::memset(p, 0, n * sizeof(double));
  return p;
}

// In-place LU with partial pivoting of the n x n column-major a (lda n):
// row k exchanged with piv[k] - 1 before step k (LAPACK dgetrf's
// convention).  Returns 0, or k + 1 if U(k, k) is exactly zero.
int lu_inplace(double* a, int n, int lda, int* piv) {
  int info = 0;
  for (int k = 0; k < n; k++) {
    int p = k;
    double best = std::fabs(a[k + static_cast<size_t>(lda) * k]);
    for (int i = k + 1; i < n; i++) {
      const double v = std::fabs(a[i + static_cast<size_t>(lda) * k]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    piv[k] = p + 1;
    if (p != k)
      for (int j = 0; j < n; j++) std::swap(a[k + static_cast<size_t>(lda) * j],
                                            a[p + static_cast<size_t>(lda) * j]);
    const double d = a[k + static_cast<size_t>(lda) * k];
    if (d == 0.0) {
      if (!info) info = k + 1;
      continue;
    }
    for (int i = k + 1; i < n; i++) a[i + static_cast<size_t>(lda) * k] /= d;
    for (int j = k + 1; j < n; j++) {
      const double f = a[k + static_cast<size_t>(lda) * j];
      if (f == 0.0) continue;
      double* cj = a + static_cast<size_t>(lda) * j;
      const double* ck = a + static_cast<size_t>(lda) * k;
      for (int i = k + 1; i < n; i++) cj[i] -= ck[i] * f;
    }
  }
  return info;
}

// Solves (LU) X = B (trans false) or (LU)^T X = B (trans true) in place for
// the nrhs columns of b (ldb), with the pivots of lu_inplace.
void lu_solve(const double* a, int n, int lda, const int* piv, double* b, int ldb, int nrhs,
              bool trans) {
  for (int c = 0; c < nrhs; c++) {
    double* x = b + static_cast<size_t>(ldb) * c;
    if (!trans) {
      for (int k = 0; k < n; k++)
        if (piv[k] - 1 != k) std::swap(x[k], x[piv[k] - 1]);
      for (int j = 0; j < n; j++) {  // L y = P b (unit lower)
        const double v = x[j];
        if (v != 0.0)
          for (int i = j + 1; i < n; i++) x[i] -= a[i + static_cast<size_t>(lda) * j] * v;
      }
      for (int j = n - 1; j >= 0; j--) {  // U x = y
        x[j] /= a[j + static_cast<size_t>(lda) * j];
        const double v = x[j];
        if (v != 0.0)
          for (int i = 0; i < j; i++) x[i] -= a[i + static_cast<size_t>(lda) * j] * v;
      }
    } else {
      for (int j = 0; j < n; j++) {  // U^T y = b
        double s = x[j];
        for (int i = 0; i < j; i++) s -= a[i + static_cast<size_t>(lda) * j] * x[i];
        x[j] = s / a[j + static_cast<size_t>(lda) * j];
      }
      for (int j = n - 1; j >= 0; j--) {  // L^T z = y
        double s = x[j];
        for (int i = j + 1; i < n; i++) s -= a[i + static_cast<size_t>(lda) * j] * x[i];
        x[j] = s;
      }
      for (int k = n - 1; k >= 0; k--)
        if (piv[k] - 1 != k) std::swap(x[k], x[piv[k] - 1]);
    }
  }
}

}  // namespace

ki_Mat::ki_Mat() : mat(nullptr), lda_(0), height_(0), width_(0) {}

ki_Mat::~ki_Mat() { delete[] mat; }

ki_Mat::ki_Mat(int h, int w) : lda_(h), height_(h), width_(w) {
  mat = alloc_zero(static_cast<size_t>(h) * w);
}

ki_Mat::ki_Mat(const ki_Mat& o) : lda_(o.lda_), height_(o.height_), width_(o.width_) {
  const size_t n = static_cast<size_t>(height_) * width_;
  mat = n ? new double[n] : nullptr;
  if (n) std::memcpy(mat, o.mat, n * sizeof(double));
}

ki_Mat& ki_Mat::operator=(const ki_Mat& o) {
  if (this == &o) return *this;
  const size_t n = static_cast<size_t>(o.height_) * o.width_;
  if (static_cast<size_t>(height_) * width_ != n) {
    delete[] mat;
    mat = n ? new double[n] : nullptr;
  }
  lda_ = o.lda_;
  height_ = o.height_;
  width_ = o.width_;
  if (n) std::memcpy(mat, o.mat, n * sizeof(double));
  return *this;
}

ki_Mat::ki_Mat(ki_Mat&& o) : mat(o.mat), lda_(o.lda_), height_(o.height_), width_(o.width_) {
  o.mat = nullptr;
  o.lda_ = o.height_ = o.width_ = 0;
}

ki_Mat& ki_Mat::operator=(ki_Mat&& o) {
  if (this == &o) return *this;
  delete[] mat;
  mat = o.mat;
  lda_ = o.lda_;
  height_ = o.height_;
  width_ = o.width_;
  o.mat = nullptr;
  o.lda_ = o.height_ = o.width_ = 0;
  return *this;
}

double ki_Mat::get(int i, int j) const {
  assert(i >= 0 && i < height_ && j >= 0 && j < width_);
  return mat[i + static_cast<size_t>(lda_) * j];
}

void ki_Mat::set(int i, int j, double a) {
  assert(i >= 0 && i < height_ && j >= 0 && j < width_);
  mat[i + static_cast<size_t>(lda_) * j] = a;
}

void ki_Mat::addset(int i, int j, double a) {
  assert(i >= 0 && i < height_ && j >= 0 && j < width_);
  mat[i + static_cast<size_t>(lda_) * j] += a;
}

void ki_Mat::set_submatrix(const std::vector<int>& I_, const std::vector<int>& J_,
                           const ki_Mat& A, bool transpose_A) {
  const int ni = static_cast<int>(I_.size()), nj = static_cast<int>(J_.size());
  for (int j = 0; j < nj; j++)
    for (int i = 0; i < ni; i++) set(I_[i], J_[j], transpose_A ? A.get(j, i) : A.get(i, j));
}

void ki_Mat::set_submatrix(int row_s, int row_e, int col_s, int col_e, const ki_Mat& A,
                           bool transpose_A, bool) {
  for (int j = col_s; j < col_e; j++)
    for (int i = row_s; i < row_e; i++)
      set(i, j, transpose_A ? A.get(j - col_s, i - row_s) : A.get(i - row_s, j - col_s));
}

void ki_Mat::set_submatrix(const std::vector<int>& I_, int col_s, int col_e, const ki_Mat& A,
                           bool transpose_A) {
  const int ni = static_cast<int>(I_.size());
  for (int j = col_s; j < col_e; j++)
    for (int i = 0; i < ni; i++)
      set(I_[i], j, transpose_A ? A.get(j - col_s, i) : A.get(i, j - col_s));
}

void ki_Mat::set_submatrix(int row_s, int row_e, const std::vector<int>& J_, const ki_Mat& A,
                           bool transpose_A) {
  const int nj = static_cast<int>(J_.size());
  for (int j = 0; j < nj; j++)
    for (int i = row_s; i < row_e; i++)
      set(i, J_[j], transpose_A ? A.get(j, i - row_s) : A.get(i - row_s, j));
}

void ki_Mat::transpose_into(ki_Mat* t) const {
  if (t->height_ != width_ || t->width_ != height_) *t = ki_Mat(width_, height_);
  for (int j = 0; j < width_; j++)
    for (int i = 0; i < height_; i++) t->set(j, i, get(i, j));
}

void ki_Mat::eye(int n) {
  *this = ki_Mat(n, n);
  for (int i = 0; i < n; i++) set(i, i, 1.0);
}

ki_Mat ki_Mat::transpose() const {
  ki_Mat t(width_, height_);
  transpose_into(&t);
  return t;
}

int ki_Mat::height() const { return height_; }
int ki_Mat::width() const { return width_; }

ki_Mat& ki_Mat::operator-=(const ki_Mat& o) {
  assert(height_ == o.height_ && width_ == o.width_);
  for (int j = 0; j < width_; j++)
    for (int i = 0; i < height_; i++) addset(i, j, -o.get(i, j));
  return *this;
}

ki_Mat& ki_Mat::operator+=(const ki_Mat& o) {
  assert(height_ == o.height_ && width_ == o.width_);
  for (int j = 0; j < width_; j++)
    for (int i = 0; i < height_; i++) addset(i, j, o.get(i, j));
  return *this;
}

ki_Mat& ki_Mat::operator*=(double o) {
  for (size_t q = 0; q < static_cast<size_t>(height_) * width_; q++) mat[q] *= o;
  return *this;
}

ki_Mat& ki_Mat::operator/=(double o) {
  for (size_t q = 0; q < static_cast<size_t>(height_) * width_; q++) mat[q] /= o;
  return *this;
}

ki_Mat ki_Mat::operator-() const {
  ki_Mat r(*this);
  r *= -1.0;
  return r;
}

ki_Mat ki_Mat::operator-(const ki_Mat& o) const {
  ki_Mat r(*this);
  r -= o;
  return r;
}

ki_Mat ki_Mat::operator+(const ki_Mat& o) const {
  ki_Mat r(*this);
  r += o;
  return r;
}

ki_Mat ki_Mat::operator*(const ki_Mat& o) const {
  assert(width_ == o.height_);
  ki_Mat r(height_, o.width_);
  for (int j = 0; j < o.width_; j++) {
    double* rc = r.mat + static_cast<size_t>(r.lda_) * j;
    for (int k = 0; k < width_; k++) {
      const double b = o.get(k, j);
      if (b == 0.0) continue;
      const double* ac = mat + static_cast<size_t>(lda_) * k;
      for (int i = 0; i < height_; i++) rc[i] += ac[i] * b;
    }
  }
  return r;
}

ki_Mat ki_Mat::operator*(double o) const {
  ki_Mat r(*this);
  r *= o;
  return r;
}

ki_Mat ki_Mat::operator/(double o) const {
  ki_Mat r(*this);
  r /= o;
  return r;
}

ki_Mat ki_Mat::operator()(const std::vector<int>& I_, const std::vector<int>& J_) const {
  ki_Mat r(static_cast<int>(I_.size()), static_cast<int>(J_.size()));
  for (size_t j = 0; j < J_.size(); j++)
    for (size_t i = 0; i < I_.size(); i++)
      r.set(static_cast<int>(i), static_cast<int>(j), get(I_[i], J_[j]));
  return r;
}

ki_Mat ki_Mat::operator()(const std::vector<int>& I_, int col_s, int col_e) const {
  ki_Mat r(static_cast<int>(I_.size()), col_e - col_s);
  for (int j = col_s; j < col_e; j++)
    for (size_t i = 0; i < I_.size(); i++) r.set(static_cast<int>(i), j - col_s, get(I_[i], j));
  return r;
}

ki_Mat ki_Mat::operator()(int row_s, int row_e, const std::vector<int>& J_) const {
  ki_Mat r(row_e - row_s, static_cast<int>(J_.size()));
  for (size_t j = 0; j < J_.size(); j++)
    for (int i = row_s; i < row_e; i++) r.set(i - row_s, static_cast<int>(j), get(i, J_[j]));
  return r;
}

ki_Mat ki_Mat::operator()(int row_s, int row_e, int col_s, int col_e) const {
  ki_Mat r(row_e - row_s, col_e - col_s);
  for (int j = col_s; j < col_e; j++)
    for (int i = row_s; i < row_e; i++) r.set(i - row_s, j - col_s, get(i, j));
  return r;
}

double ki_Mat::one_norm() const {
  double top = 0.0;
  for (int j = 0; j < width_; j++) {
    double s = 0.0;
    for (int i = 0; i < height_; i++) s += std::fabs(get(i, j));
    top = std::max(top, s);
  }
  return top;
}

double ki_Mat::vec_two_norm() const {
  assert(width_ == 1);
  return frob_norm();
}

double ki_Mat::frob_norm() const {
  double s = 0.0;
  for (int j = 0; j < width_; j++)
    for (int i = 0; i < height_; i++) s += get(i, j) * get(i, j);
  return std::sqrt(s);
}

double ki_Mat::max_entry_magnitude() const {
  double m = 0.0;
  for (int j = 0; j < width_; j++)
    for (int i = 0; i < height_; i++) m = std::max(m, std::fabs(get(i, j)));
  return m;
}

void ki_Mat::LU_factorize(ki_Mat* K_LU, std::vector<lapack_int>* piv) const {
  assert(height_ == width_);
  *K_LU = *this;
  piv->assign(height_, 0);
  lu_inplace(K_LU->mat, height_, K_LU->lda_, piv->data());
}

void ki_Mat::left_multiply_inverse(const ki_Mat& K, ki_Mat* U) const {
  ki_Mat lu;
  std::vector<lapack_int> piv;
  LU_factorize(&lu, &piv);
  lu.left_multiply_inverse(K, piv, U);
}

void ki_Mat::right_multiply_inverse(const ki_Mat& K, ki_Mat* L) const {
  ki_Mat lu;
  std::vector<lapack_int> piv;
  LU_factorize(&lu, &piv);
  lu.right_multiply_inverse(K, piv, L);
}

void ki_Mat::left_multiply_inverse(const ki_Mat& K, const std::vector<lapack_int>& piv,
                                   ki_Mat* U) const {
  // *this holds LU factors of X: U = X^-1 K
  assert(K.height_ == height_);
  *U = K;
  lu_solve(mat, height_, lda_, piv.data(), U->mat, U->lda_, U->width_, false);
}

void ki_Mat::right_multiply_inverse(const ki_Mat& K, const std::vector<lapack_int>& piv,
                                    ki_Mat* L) const {
  // *this holds LU factors of X: L = K X^-1, i.e. X^T L^T = K^T
  assert(K.width_ == height_);
  ki_Mat kt = K.transpose();
  lu_solve(mat, height_, lda_, piv.data(), kt.mat, kt.lda_, kt.width_, true);
  *L = kt.transpose();
}

int ki_Mat::id(std::vector<int>* p, ki_Mat* Z, double tol) const {
  // Householder QR with column pivoting (the largest remaining partial
  // column norm first, first index on ties; norms downdated after each
  // step and recomputed when cancellation makes the downdate unreliable),
  // then the rank rule and T = R11^-1 R12 (ki_mat.cpp:502-541).
  assert(height_ > 0 && width_ > 0);
  const int m = height_, n = width_, kmax = std::min(m, n);
  ki_Mat a(*this);
  std::vector<int> perm(n);
  std::vector<double> vn1(n), vn2(n);
  for (int j = 0; j < n; j++) {
    perm[j] = j;
    double s = 0.0;
    for (int i = 0; i < m; i++) s += a.get(i, j) * a.get(i, j);
    vn1[j] = vn2[j] = std::sqrt(s);
  }
  const double tol3z = std::sqrt(std::numeric_limits<double>::epsilon());
  std::vector<double> v(m);
  for (int k = 0; k < kmax; k++) {
    int pj = k;
    for (int j = k + 1; j < n; j++)
      if (vn1[j] > vn1[pj]) pj = j;
    if (pj != k) {
      for (int i = 0; i < m; i++) std::swap(a.mat[i + static_cast<size_t>(a.lda_) * k],
                                            a.mat[i + static_cast<size_t>(a.lda_) * pj]);
      std::swap(perm[k], perm[pj]);
      vn1[pj] = vn1[k];
      vn2[pj] = vn2[k];
    }
    // reflector for column k, rows k..m-1: beta = -sign(alpha) |x|
    double xn = 0.0;
    for (int i = k + 1; i < m; i++) xn += a.get(i, k) * a.get(i, k);
    const double alpha = a.get(k, k);
    double tau = 0.0;
    if (xn > 0.0) {
      const double beta = -std::copysign(std::sqrt(alpha * alpha + xn), alpha);
      tau = (beta - alpha) / beta;
      const double sc = 1.0 / (alpha - beta);
      v[k] = 1.0;
      for (int i = k + 1; i < m; i++) {
        v[i] = a.get(i, k) * sc;
        a.set(i, k, v[i]);
      }
      a.set(k, k, beta);
      for (int j = k + 1; j < n; j++) {
        double d = 0.0;
        for (int i = k; i < m; i++) d += v[i] * a.get(i, j);
        d *= tau;
        for (int i = k; i < m; i++) a.addset(i, j, -d * v[i]);
      }
    }
    for (int j = k + 1; j < n; j++) {
      if (vn1[j] == 0.0) continue;
      double t = std::fabs(a.get(k, j)) / vn1[j];
      t = std::max(0.0, (1.0 + t) * (1.0 - t));
      const double t2 = t * (vn1[j] / vn2[j]) * (vn1[j] / vn2[j]);
      if (t2 <= tol3z) {
        double s = 0.0;
        for (int i = k + 1; i < m; i++) s += a.get(i, j) * a.get(i, j);
        vn1[j] = vn2[j] = std::sqrt(s);
      } else {
        vn1[j] *= std::sqrt(t);
      }
    }
  }
  int skel = 0;
  const double thresh = std::fabs(tol * a.get(0, 0));
  for (int i = 1; i < kmax; i++)
    if (std::fabs(a.get(i, i)) < thresh) {
      skel = i;
      break;
    }
  if (skel == 0) return 0;
  for (int j = 0; j < n; j++) p->push_back(perm[j]);
  const int red = n - skel;
  ki_Mat z(skel, red);
  for (int j = 0; j < red; j++) {
    for (int i = skel - 1; i >= 0; i--) {
      double s = a.get(i, skel + j);
      for (int q = i + 1; q < skel; q++) s -= a.get(i, q) * z.get(q, j);
      z.set(i, j, s / a.get(i, i));
    }
  }
  *Z = std::move(z);
  return skel;
}

std::vector<double> ki_Mat::real_eigenvalues() {
  // Hessenberg reduction by Householder reflections, then the implicit
  // double-shift QR iteration (Francis) with deflation on negligible
  // subdiagonal entries; 1x1 blocks give real eigenvalues, 2x2 blocks a
  // real pair or a complex pair (Golub & Van Loan, Matrix Computations,
  // 7.4-7.5).
  assert(height_ == width_);
  const int n = width_;
  std::vector<double> out;
  if (n == 0) return out;
  std::vector<double> h(static_cast<size_t>(n) * n);
  auto H = [&](int i, int j) -> double& { return h[i + static_cast<size_t>(n) * j]; };
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) H(i, j) = get(i, j);
  std::vector<double> v(n);
  for (int k = 0; k + 2 < n; k++) {
    double xn = 0.0;
    for (int i = k + 1; i < n; i++) xn += H(i, k) * H(i, k);
    xn = std::sqrt(xn);
    if (xn == 0.0) continue;
    const double a0 = H(k + 1, k);
    const double beta = -std::copysign(xn, a0);
    for (int i = k + 1; i < n; i++) v[i] = H(i, k);
    v[k + 1] -= beta;
    double vv = 0.0;
    for (int i = k + 1; i < n; i++) vv += v[i] * v[i];
    if (vv == 0.0) continue;
    for (int j = 0; j < n; j++) {  // H = (I - 2vv^T/vv) H
      double d = 0.0;
      for (int i = k + 1; i < n; i++) d += v[i] * H(i, j);
      d *= 2.0 / vv;
      for (int i = k + 1; i < n; i++) H(i, j) -= d * v[i];
    }
    for (int i = 0; i < n; i++) {  // H = H (I - 2vv^T/vv)
      double d = 0.0;
      for (int j = k + 1; j < n; j++) d += H(i, j) * v[j];
      d *= 2.0 / vv;
      for (int j = k + 1; j < n; j++) H(i, j) -= d * v[j];
    }
  }
  const double eps = std::numeric_limits<double>::epsilon();
  std::vector<double> re(n, 0.0), im(n, 0.0);
  int hi = n - 1, iter = 0;
  while (hi >= 0) {
    int lo = hi;
    while (lo > 0) {
      const double s = std::fabs(H(lo - 1, lo - 1)) + std::fabs(H(lo, lo));
      if (std::fabs(H(lo, lo - 1)) <= eps * (s == 0.0 ? 1.0 : s)) {
        H(lo, lo - 1) = 0.0;
        break;
      }
      lo--;
    }
    if (lo == hi) {
      re[hi] = H(hi, hi);
      hi--;
      iter = 0;
      continue;
    }
    if (lo == hi - 1) {
      const double a = H(hi - 1, hi - 1), b = H(hi - 1, hi), c = H(hi, hi - 1), d = H(hi, hi);
      const double tr = a + d, det = a * d - b * c;
      const double disc = 0.25 * tr * tr - det;
      if (disc >= 0.0) {
        const double r = std::sqrt(disc);
        const double l1 = 0.5 * tr + (tr >= 0 ? r : -r);
        const double l2 = l1 != 0.0 ? det / l1 : 0.5 * tr - (tr >= 0 ? r : -r);
        re[hi - 1] = l1;
        re[hi] = l2;
      } else {
        re[hi - 1] = re[hi] = 0.5 * tr;
        im[hi - 1] = std::sqrt(-disc);
        im[hi] = -im[hi - 1];
      }
      hi -= 2;
      iter = 0;
      continue;
    }
    if (++iter > 60 * n) break;  // no convergence: report what deflated
    // double shift from the trailing 2x2 block (exceptional shift now and then)
    double s = H(hi - 1, hi - 1) + H(hi, hi);
    double t = H(hi - 1, hi - 1) * H(hi, hi) - H(hi - 1, hi) * H(hi, hi - 1);
    if (iter % 11 == 10) {
      const double w = std::fabs(H(hi, hi - 1)) + std::fabs(H(hi - 1, hi - 2));
      s = 1.5 * w;
      t = w * w;
    }
    double x = H(lo, lo) * H(lo, lo) + H(lo, lo + 1) * H(lo + 1, lo) - s * H(lo, lo) + t;
    double y = H(lo + 1, lo) * (H(lo, lo) + H(lo + 1, lo + 1) - s);
    double z = lo + 2 <= hi ? H(lo + 1, lo) * H(lo + 2, lo + 1) : 0.0;
    for (int k = lo; k <= hi - 1; k++) {
      const int nr = k + 2 <= hi ? 3 : 2;
      double u[3] = {x, y, nr == 3 ? z : 0.0};
      double un = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
      if (un != 0.0) {
        u[0] += std::copysign(un, u[0]);
        double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        const int c0 = std::max(lo, k - 1);
        for (int j = c0; j < n; j++) {
          double d = 0.0;
          for (int q = 0; q < nr; q++) d += u[q] * H(k + q, j);
          d *= 2.0 / uu;
          for (int q = 0; q < nr; q++) H(k + q, j) -= d * u[q];
        }
        const int r1 = std::min(hi, k + 3);
        for (int i = 0; i <= r1; i++) {
          double d = 0.0;
          for (int q = 0; q < nr; q++) d += H(i, k + q) * u[q];
          d *= 2.0 / uu;
          for (int q = 0; q < nr; q++) H(i, k + q) -= d * u[q];
        }
      }
      x = H(k + 1, k);
      y = k + 2 <= hi ? H(k + 2, k) : 0.0;
      z = k + 3 <= hi ? H(k + 3, k) : 0.0;
    }
  }
  for (int i = 0; i < n; i++)
    if (std::fabs(im[i]) < 1e-14) out.push_back(re[i]);
  return out;
}

}  // namespace kern_interp
