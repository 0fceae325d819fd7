// C++ drop-in API of the B200 solver: kern_interp::ki_Mat.
//
// The reference's dense matrix type (kern_interp/ki_mat.h:19-101): value
// semantics, column-major storage in `mat` with leading dimension lda_ =
// height, zero-initialised.  Callers use it for boundary data, solutions
// and small dense checks; the solver's own factors live on the GPU.  The
// arithmetic here is plain host code (no BLAS / LAPACK dependency): LU with
// partial pivoting (pivots 1-based, as LAPACK returns them) and the
// interpolative decomposition by Householder QR with column pivoting and
// the reference's rank rule.
#ifndef KERN_INTERP_KI_MAT_H_
#define KERN_INTERP_KI_MAT_H_

#include <string>
#include <vector>

#ifndef lapack_int
#define lapack_int int
#endif

#ifndef NORMAL
#define NORMAL 111     // CblasNoTrans's value
#endif
#ifndef TRANSPOSE
#define TRANSPOSE 112  // CblasTrans's value
#endif

namespace kern_interp {

struct ki_Mat {
  // column-major, lda_ = height_
  double* mat;

  int lda_, height_, width_;
  ki_Mat();
  ~ki_Mat();

  ki_Mat(int h, int w);

  ki_Mat(const ki_Mat& o);
  ki_Mat& operator=(const ki_Mat& copy);
  ki_Mat(ki_Mat&& move);
  ki_Mat& operator=(ki_Mat&& move);

  double get(int i, int j) const;
  void set(int i, int j, double a);
  void addset(int i, int j, double a);
  void set_submatrix(const std::vector<int>& I_, const std::vector<int>& J_, const ki_Mat& A,
                     bool transpose_A = false);
  void set_submatrix(int row_s, int row_e, int col_s, int col_e, const ki_Mat& A,
                     bool transpose_A = false, bool timing = false);
  void set_submatrix(const std::vector<int>& I_, int col_s, int col_e, const ki_Mat& A,
                     bool transpose_A = false);
  void set_submatrix(int row_s, int row_e, const std::vector<int>& J_, const ki_Mat& A,
                     bool transpose_A = false);

  void transpose_into(ki_Mat* transpose) const;
  void eye(int n);
  ki_Mat transpose() const;

  int height() const;
  int width() const;

  ki_Mat& operator-=(const ki_Mat& o);
  ki_Mat& operator+=(const ki_Mat& o);
  ki_Mat& operator*=(double o);
  ki_Mat& operator/=(double o);

  ki_Mat operator-() const;
  ki_Mat operator-(const ki_Mat& o) const;
  ki_Mat operator+(const ki_Mat& o) const;
  ki_Mat operator*(const ki_Mat& o) const;
  ki_Mat operator*(double o) const;
  ki_Mat operator/(double o) const;

  ki_Mat operator()(const std::vector<int>& I_, const std::vector<int>& J_) const;
  ki_Mat operator()(const std::vector<int>& I_, int col_s, int col_e) const;
  ki_Mat operator()(int row_s, int row_e, const std::vector<int>& J_) const;
  ki_Mat operator()(int row_s, int row_e, int col_s, int col_e) const;

  double one_norm() const;
  double vec_two_norm() const;
  double frob_norm() const;
  double max_entry_magnitude() const;

  // K_LU = the LU factors of *this (square), piv the 1-based row pivots
  void LU_factorize(ki_Mat* K_LU, std::vector<lapack_int>* piv) const;
  // *U = K^-1 U and *L = L K^-1 with K = *this (factored on the fly) or
  // with K an LU_factorize result and its pivots
  void left_multiply_inverse(const ki_Mat& K, ki_Mat* U) const;
  void right_multiply_inverse(const ki_Mat& K, ki_Mat* L) const;
  void left_multiply_inverse(const ki_Mat& K, const std::vector<lapack_int>& piv,
                             ki_Mat* U) const;
  void right_multiply_inverse(const ki_Mat& K, const std::vector<lapack_int>& piv,
                              ki_Mat* L) const;

  // Interpolative decomposition: p = the column pivots (0-based, skeleton
  // first), *Z = R11^-1 R12 (rank x (width - rank)); returns the rank: the
  // first i >= 1 with |R_ii| < tol |R_00|, none = 0 (not compressible).
  int id(std::vector<int>* p, ki_Mat* Z, double tol) const;
  // Real eigenvalues (imaginary part below 1e-14) of a square matrix.
  std::vector<double> real_eigenvalues();
};

}  // namespace kern_interp

#endif  // KERN_INTERP_KI_MAT_H_
