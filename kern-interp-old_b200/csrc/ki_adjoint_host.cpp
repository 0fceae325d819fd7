// Transposed solve and the backward pass of the target-potential map.
//
// The solve of SkelFactorization::solve (skel_factorization.cpp:341-403) is
// x = Down Top Diag Up b with, per compressed box (r redundant, s skeleton):
//   Up   = (x_s -= L x_r) o (x_r -= T^T x_s)      levels deepest first
//   Diag = x_r <- X_rr^-1 x_r
//   Down = (x_s -= T x_r) o (x_r -= U x_s)        levels root first
// so A^-T = Up^T Diag^T Top^T Down^T, applied right to left:
//   Down^T per box: x_r -= T^T x_s, then x_s -= U^T x_r   deepest level first
//   Top^T, Diag^T:  transposed LU solves
//   Up^T per box:   x_r -= L^T x_s, then x_s -= T x_r     root level first
// The reference has no transposed solve; it is what the adjoint needs.
#include "ki_solver.h"

namespace kib {

int Solver::solve_transpose_device(const double* d_b, double* d_x) {
  if (nb_ > 0) return fail("transposed solve: domains with holes are not supported");
  if (d_forest_) return fail("transposed solve: not available for a batch of problems");
  const int N = n_dofs_;
  if (d_b != d_x)
    KI_CUDA(cudaMemcpyAsync(d_x, d_b, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream_));
  const int L = static_cast<int>(levels_.size());
  for (int l = L - 1; l >= 0; l--) {
    const LevelFactors& lf = levels_[l];
    if (!lf.ntasks) continue;
    SweepParams sp{lf.d_tasks, lf.ntasks, d_x, N, 1, 0, nullptr, lf.cap};
    sp.kr = lf.kr;
    KI_CUDA(launch_sweep_up(sp, true, stream_));
  }
  SweepParams dp{all_compressed_.d_tasks, all_compressed_.ntasks, d_x, N, 1, 0, nullptr,
                 all_compressed_.cap};
  if (diag_all(dp, true)) return -2;
  const int ns = ns_;
  if (ns > 0) {
    KI_CUDA(launch_gather(d_x, N, d_allskel_, ns, 1, d_tmp_, ns, stream_));
    KI_CUDA(dense_lu_solve_rows(d_top_, ns, ns, d_top_piv_, d_tmp_, 1, 1, stream_));
    KI_CUDA(launch_scatter(d_x, N, d_allskel_, ns, 1, d_tmp_, ns, stream_));
  }
  for (int l = 0; l < L; l++) {
    const LevelFactors& lf = levels_[l];
    if (!lf.ntasks) continue;
    SweepParams sp{lf.d_tasks, lf.ntasks, d_x, N, 1, 0, nullptr, lf.cap};
    sp.kr = lf.kr;
    KI_CUDA(launch_transposed_up(sp, stream_));
  }
  return 0;
}

int Solver::adjoint_backward(int n_targets, const double* d_targets, const double* d_mu,
                             const double* d_grad_u, double* d_grad_f, double* d_grad_points,
                             double* d_grad_normals, double* d_grad_weights,
                             double* d_grad_curv) {
  if (opt_.pde != kLaplace || nb_ > 0 || d_forest_)
    return fail("adjoint: only the Laplace double layer on a single simply connected domain");
  const int n = n_points_;
  KI_CUDA(adj_.reserve(sizeof(double) * adjoint_work_doubles(n), stream_));
  double* work = static_cast<double*>(adj_.p);
  // g_mu = K_t^T grad_u (into grad_f), target-term node gradients
  KI_CUDA(launch_adjoint_laplace(d_nodes_, n, d_mu, n_targets, d_targets, d_grad_u, d_grad_f,
                                 work, stream_));
  // lam = A^-T g_mu = dJ/df
  if (solve_transpose_device(d_grad_f, d_grad_f)) return -2;
  KI_CUDA(launch_adjoint_laplace_finish(d_nodes_, n, d_mu, d_grad_f, work, d_grad_points,
                                        d_grad_normals, d_grad_weights, d_grad_curv, stream_));
  return 0;
}

}  // namespace kib
