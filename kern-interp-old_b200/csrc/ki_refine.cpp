// FP64 refinement of a (possibly low-accuracy) factorization on the
// bordered boundary operator
//
//     [ A  U ] [mu   ]   [f]
//     [Psi -I] [alpha] = [0]        (kern_interp_test.cpp:54-78 form; no
//                                    border when the domain has no holes)
//
// with the factorization's solve as the preconditioner M^-1 and the
// operator applied by the fast on-the-fly FP64 product.  Stationary
// refinement X += M^-1 (B - A X) runs first (the usual case: each step gains
// the factorization's accuracy); if it stalls, right-preconditioned GMRES
// continues from the current iterate.  The preconditioner application is a
// CUDA graph of the whole solve, captured once.  In GMRES the preconditioned
// directions Z_j = M^-1 V_j are kept (flexible-GMRES storage), so the
// correction is X += Z y without a further solve.  Orthogonalisation is
// classical Gram-Schmidt applied twice; the Hessenberg least-squares problem
// is tiny and solved on the host with Givens rotations.  The reference has no
// iterative solver; its direct solve is the X_0 = M^-1 b first step here.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "ki_solver.h"

namespace kib {

int Solver::mv_setup() {
  if (d_mv_tiles_) return 0;
  if (!num_sms_) {
    int dev = 0;
    KI_CUDA(cudaGetDevice(&dev));
    KI_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
  }
  seg_ = starts_.size() > 1 ? starts_ : std::vector<int>{0, n_points_};
  const int nseg = static_cast<int>(seg_.size()) - 1;
  // splits sized for the average problem, filling whole waves of the GPU
  mv_splits_ = matvec_splits(opt_.pde, std::max(1, n_points_ / nseg), nseg, num_sms_);
  std::vector<MvTile> tiles;
  matvec_tiles(seg_, mv_splits_, &tiles);
  n_mv_tiles_ = static_cast<int>(tiles.size());
  KI_ALLOC(d_mv_tiles_, MvTile, tiles.size());
  KI_ALLOC(d_seg_, int, seg_.size());
  KI_UPLOAD(d_mv_tiles_, tiles, stream_);
  KI_UPLOAD(d_seg_, seg_, stream_);
  return 0;
}

int Solver::solve_graph(const double* d_b, double* d_mu, double* d_alpha, const double* d_g) {
  const int N = n_dofs_, nb = nb_;
  // KI_SOLVE_GRAPH=0 launches the same kernels one by one instead (for tools
  // that cannot follow stream capture, e.g. kernel profilers)
  static const bool use_graph = [] {
    const char* e = std::getenv("KI_SOLVE_GRAPH");
    return !(e && e[0] == '0');
  }();
  if (!use_graph) return solve_device(d_b, d_mu, d_alpha, d_g);
  // capturing and instantiating costs more host time than a few solves
  // save: the graph is made once a factorization has served a few
  // preconditioner applications, i.e. when it is being reused
  if (!solve_exec_ && ++graph_uses_ < kGraphAfter) return solve_device(d_b, d_mu, d_alpha, d_g);
  if (!solve_exec_) {
    KI_ALLOC(g_x_, double, static_cast<size_t>(N) + 2 * nb);
    double* ga = g_x_ + N;
    double* gg = ga + nb;
    cudaGraph_t graph = nullptr;
    KI_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed));
    const int rc = solve_device(g_x_, g_x_, nb ? ga : nullptr, nb ? gg : nullptr);
    const cudaError_t e = cudaStreamEndCapture(stream_, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    KI_CUDA(e);
    const cudaError_t ei = cudaGraphInstantiate(&solve_exec_, graph, 0);
    cudaGraphDestroy(graph);
    KI_CUDA(ei);
  }
  KI_CUDA(cudaMemcpyAsync(g_x_, d_b, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream_));
  if (nb) {
    if (d_g)
      KI_CUDA(cudaMemcpyAsync(g_x_ + N + nb, d_g, sizeof(double) * nb, cudaMemcpyDeviceToDevice,
                              stream_));
    else
      KI_CUDA(cudaMemsetAsync(g_x_ + N + nb, 0, sizeof(double) * nb, stream_));
  }
  KI_CUDA(cudaGraphLaunch(solve_exec_, stream_));
  KI_CUDA(cudaMemcpyAsync(d_mu, g_x_, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream_));
  if (nb && d_alpha)
    KI_CUDA(cudaMemcpyAsync(d_alpha, g_x_ + N, sizeof(double) * nb, cudaMemcpyDeviceToDevice,
                            stream_));
  return 0;
}

int Solver::matvec_device(const double* d_x, double* d_y) {
  if (mv_setup()) return -2;
  const int nseg = static_cast<int>(seg_.size()) - 1;
  const size_t need = fast_matvec_scratch_doubles(n_dofs_, mv_splits_, nseg, nb_);
  // the product's partials live at the start of kry_; solve_refined places
  // its vectors after them
  if (kry_.bytes < sizeof(double) * need) KI_CUDA(kry_.reserve(sizeof(double) * need, stream_));
  KI_CUDA(launch_fast_matvec(opt_.pde, d_nodes_, d_mv_tiles_, n_mv_tiles_, d_seg_, nseg, n_dofs_,
                             mv_splits_, d_x, d_y, nb_, d_U_, d_Psi_, static_cast<double*>(kry_.p),
                             stream_));
  return 0;
}

int Solver::corr_matvec_device(const double* d_x, double* d_y, double dscale) {
  if (mv_setup()) return -2;
  const int nseg = static_cast<int>(seg_.size()) - 1;
  const size_t need = fast_matvec_scratch_doubles(n_dofs_, mv_splits_, nseg, nb_);
  if (kry_.bytes < sizeof(double) * need) KI_CUDA(kry_.reserve(sizeof(double) * need, stream_));
  KI_CUDA(launch_corr_matvec(opt_.pde, d_nodes_, d_mv_tiles_, n_mv_tiles_, d_seg_, nseg, n_dofs_,
                             mv_splits_, d_x, dscale, kCorrNearGap, d_y, nb_, d_U_, d_Psi_,
                             static_cast<double*>(kry_.p), stream_));
  return 0;
}

int Solver::solve_refined(const double* d_f, double* d_mu, double* d_alpha, double rel_tol,
                          int max_iters, int* iters_out, double* rel_res_out) {
  const int N = n_dofs_, nb = nb_, n = N + nb;
  const int m = std::max(1, std::min(max_iters, kMaxKrylov - 2));  // restart length
  if (mv_setup()) return -2;
  const int nseg = static_cast<int>(seg_.size()) - 1;
  const size_t mv = (fast_matvec_scratch_doubles(N, mv_splits_, nseg, nb) + 31) / 32 * 32;
  const size_t ldv = (static_cast<size_t>(n) + 31) / 32 * 32;
  const size_t dotp = static_cast<size_t>(kMaxKrylov) * multi_dot_blocks(n);
  // [mv partials][V: (m+1) ldv][Z: m ldv][B][X][W][dot partials][h: 3 kMaxKrylov]
  // [segment norms: nseg]
  const size_t total =
      mv + (2 * static_cast<size_t>(m) + 4) * ldv + dotp + 3 * kMaxKrylov + nseg + 1;
  KI_CUDA(kry_.reserve(sizeof(double) * total, stream_));
  double* base = static_cast<double*>(kry_.p);
  double* V = base + mv;
  double* Z = V + (m + 1) * ldv;
  double* B = Z + m * ldv;
  double* X = B + ldv;
  double* W = X + ldv;
  double* part = W + ldv;
  double* dh = part + dotp;  // [0, k) first pass, [kMax, kMax + k) second, [2 kMax] norm
  double* dseg = dh + 3 * kMaxKrylov;
  if (!h_kry_) {
    h_kry_ = keep_stage_.get<double>(3 * kMaxKrylov + nseg + 1);
    if (!h_kry_) return fail("pinned allocation failed: refinement coefficients");
  }
  double* hh = h_kry_;
  double* hseg = hh + 3 * kMaxKrylov;
  // largest per-problem relative residual of v (forest: every problem must
  // meet the tolerance on its own)
  std::vector<double> bseg;
  auto seg_norms = [&](const double* v, std::vector<double>* out) -> int {
    KI_CUDA(launch_segment_sumsq(v, d_seg_, nseg, sd_, dseg, stream_));
    KI_CUDA(cudaMemcpyAsync(hseg, dseg, sizeof(double) * nseg, cudaMemcpyDeviceToHost, stream_));
    KI_CUDA(cudaStreamSynchronize(stream_));
    out->assign(nseg, 0.0);
    for (int p = 0; p < nseg; p++) (*out)[p] = std::sqrt(hseg[p]);
    return 0;
  };

  // B = [f; 0], X = 0
  KI_CUDA(cudaMemcpyAsync(B, d_f, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream_));
  if (nb) KI_CUDA(cudaMemsetAsync(B + N, 0, sizeof(double) * nb, stream_));
  KI_CUDA(cudaMemsetAsync(X, 0, sizeof(double) * n, stream_));

  auto norm2 = [&](const double* v, double* out) -> int {
    KI_CUDA(launch_multi_dot(v, 0, 1, v, n, part, dh + 2 * kMaxKrylov, stream_));
    KI_CUDA(cudaMemcpyAsync(hh + 2 * kMaxKrylov, dh + 2 * kMaxKrylov, sizeof(double),
                            cudaMemcpyDeviceToHost, stream_));
    KI_CUDA(cudaStreamSynchronize(stream_));
    *out = std::sqrt(hh[2 * kMaxKrylov]);
    return 0;
  };

  double bnorm = 0;
  if (norm2(B, &bnorm)) return -2;
  // a forest stops on the global residual only once it is below every
  // problem's own share: ||r|| <= tol min_p ||b_p|| bounds each ||r_p||
  double tol_eff = rel_tol;
  if (nseg > 1) {
    if (seg_norms(B, &bseg)) return -2;
    double bmin = bnorm;
    for (double v : bseg)
      if (v > 0.0) bmin = std::min(bmin, v);
    tol_eff = rel_tol * bmin / bnorm;
  }
  int iters = 0;
  double rel = 0.0;
  if (bnorm == 0.0) {
    KI_CUDA(cudaMemsetAsync(d_mu, 0, sizeof(double) * N, stream_));
    if (nb && d_alpha) KI_CUDA(cudaMemsetAsync(d_alpha, 0, sizeof(double) * nb, stream_));
    if (iters_out) *iters_out = 0;
    if (rel_res_out) *rel_res_out = 0.0;
    return 0;
  }
  // relative residual of r = V (per problem for a forest), and ||r||
  auto residual = [&](double* beta, double* relr) -> int {
    if (norm2(V, beta)) return -2;
    *relr = *beta / bnorm;
    if (nseg > 1) {
      std::vector<double> rs;
      if (seg_norms(V, &rs)) return -2;
      double worst = 0.0;
      for (int p = 0; p < nseg; p++)
        if (bseg[p] > 0.0) worst = std::max(worst, rs[p] / bseg[p]);
      *relr = worst;
    }
    return 0;
  };

  // Stationary refinement first: X = M^-1 B, then X += M^-1 (B - A X) while
  // each step shrinks the residual at least tenfold (one solve and one
  // operator product per step, no inner products).  If it stalls, GMRES
  // continues from the current X and residual.  Once the residual r is
  // small, a step's correction D = M^-1 r is small too and the residual is
  // updated as r -= A D with the correction product: its relative error
  // (kCorrErr, see launch_corr_matvec) applies to |A D| ~ |r|, not to |X|,
  // so the updated residual stays within kCorrErr |r| of the true one; the
  // product is used only while that is below a tenth of the tolerance.
  static const bool corr_on = [] {
    const char* e = std::getenv("KI_CORR");
    return !(e && e[0] == '0');
  }();
  double beta = 0.0;
  bool done = false;
  {
    if (solve_graph(B, X, nb ? X + N : nullptr, nb ? B + N : nullptr)) return -2;
    iters++;
    if (matvec_device(X, W)) return -2;
    KI_CUDA(launch_sub(V, B, W, n, stream_));
    double prev = 1.0;
    for (;;) {
      if (residual(&beta, &rel)) return -2;
      if (rel <= rel_tol || iters >= max_iters || beta == 0.0) {
        done = true;
        break;
      }
      if (rel > 0.1 * prev) break;
      prev = rel;
      if (solve_graph(V, W, nb ? W + N : nullptr, nb ? V + N : nullptr)) return -2;
      KI_CUDA(launch_add(X, W, n, stream_));
      iters++;
      if (corr_on && kCorrErr * rel <= 0.1 * rel_tol) {
        // Z (unused until GMRES) receives A D
        if (corr_matvec_device(W, Z, 1.0 / beta)) return -2;
        KI_CUDA(launch_sub(V, V, Z, n, stream_));
      } else {
        if (matvec_device(X, W)) return -2;
        KI_CUDA(launch_sub(V, B, W, n, stream_));
      }
    }
  }
  bool have_r = true;  // V holds B - A X with norm beta
  for (; !done;) {
    if (!have_r) {
      if (matvec_device(X, W)) return -2;
      KI_CUDA(launch_sub(V, B, W, n, stream_));
      if (residual(&beta, &rel)) return -2;
    }
    have_r = false;
    if (rel <= rel_tol || iters >= max_iters || beta == 0.0) break;
    KI_CUDA(launch_scale_copy(V, V, n, 1.0 / beta, stream_));

    // Arnoldi with Givens rotations; H column-major (m+1) x m on the host
    std::vector<double> H(static_cast<size_t>(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1, 0.0);
    g[0] = beta;
    int k = 0;
    for (; k < m && iters < max_iters; k++) {
      double* vk = V + k * ldv;
      double* zk = Z + k * ldv;
      if (solve_graph(vk, zk, nb ? zk + N : nullptr, nb ? vk + N : nullptr)) return -2;
      if (matvec_device(zk, W)) return -2;
      iters++;
      // two passes of classical Gram-Schmidt against V_0..V_k
      KI_CUDA(launch_multi_dot(V, static_cast<long long>(ldv), k + 1, W, n, part, dh, stream_));
      KI_CUDA(launch_multi_axpy(W, V, static_cast<long long>(ldv), k + 1, dh, n, -1.0, stream_));
      KI_CUDA(launch_multi_dot(V, static_cast<long long>(ldv), k + 1, W, n, part, dh + kMaxKrylov,
                               stream_));
      KI_CUDA(launch_multi_axpy(W, V, static_cast<long long>(ldv), k + 1, dh + kMaxKrylov, n,
                                -1.0, stream_));
      KI_CUDA(launch_multi_dot(W, 0, 1, W, n, part, dh + 2 * kMaxKrylov, stream_));
      KI_CUDA(cudaMemcpyAsync(hh, dh, sizeof(double) * 3 * kMaxKrylov, cudaMemcpyDeviceToHost,
                              stream_));
      KI_CUDA(cudaStreamSynchronize(stream_));
      double* hk = &H[static_cast<size_t>(k) * (m + 1)];
      for (int i = 0; i <= k; i++) hk[i] = hh[i] + hh[kMaxKrylov + i];
      const double hnext = std::sqrt(hh[2 * kMaxKrylov]);
      hk[k + 1] = hnext;
      if (hnext > 0.0) KI_CUDA(launch_scale_copy(V + (k + 1) * ldv, W, n, 1.0 / hnext, stream_));
      for (int i = 0; i < k; i++) {  // apply the earlier rotations
        const double a = hk[i], b = hk[i + 1];
        hk[i] = cs[i] * a + sn[i] * b;
        hk[i + 1] = -sn[i] * a + cs[i] * b;
      }
      const double a = hk[k], b = hk[k + 1];
      const double r = std::hypot(a, b);
      cs[k] = r > 0 ? a / r : 1.0;
      sn[k] = r > 0 ? b / r : 0.0;
      hk[k] = r;
      hk[k + 1] = 0.0;
      g[k + 1] = -sn[k] * g[k];
      g[k] = cs[k] * g[k];
      if (std::fabs(g[k + 1]) <= tol_eff * bnorm || hnext == 0.0) {
        k++;
        break;
      }
    }
    // y = R^-1 g (upper triangular k x k), X += Z y
    std::vector<double> y(k, 0.0);
    for (int i = k - 1; i >= 0; i--) {
      double s = g[i];
      for (int j = i + 1; j < k; j++) s -= H[static_cast<size_t>(j) * (m + 1) + i] * y[j];
      const double d = H[static_cast<size_t>(i) * (m + 1) + i];
      y[i] = d != 0.0 ? s / d : 0.0;
    }
    if (k > 0) {
      for (int i = 0; i < k; i++) hh[i] = y[i];
      KI_CUDA(cudaMemcpyAsync(dh, hh, sizeof(double) * k, cudaMemcpyHostToDevice, stream_));
      KI_CUDA(launch_multi_axpy(X, Z, static_cast<long long>(ldv), k, dh, n, 1.0, stream_));
      // the host buffer is reused by the next cycle's download: keep the
      // upload ordered before it
      KI_CUDA(cudaStreamSynchronize(stream_));
    }
  }
  KI_CUDA(cudaMemcpyAsync(d_mu, X, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream_));
  if (nb && d_alpha)
    KI_CUDA(cudaMemcpyAsync(d_alpha, X + N, sizeof(double) * nb, cudaMemcpyDeviceToDevice,
                            stream_));
  if (iters_out) *iters_out = iters;
  if (rel_res_out) *rel_res_out = rel;
  return 0;
}

}  // namespace kib
