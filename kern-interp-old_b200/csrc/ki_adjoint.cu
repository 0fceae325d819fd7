// Adjoint of the target-potential map u = K_t mu, A mu = f, for the Laplace
// double-layer operator (kernel.cpp:11-36; forward/target entries
// kernel.cpp:337-357 with zero target normal).  The reference has no
// derivatives; these kernels supply the two contractions the backward pass
// needs besides the transposed solve:
//
//   source pass:  for every boundary node j as a SOURCE, with weights lam_t
//                 at evaluation points x_t (boundary nodes or targets):
//                   out_j = mu_j * sum_t lam_t dK(x_t, j)/d(x_j, n_j, w_j)
//                 and   kt_j = sum_t lam_t K(x_t, j)          (K^T lam)
//   target pass:  for every boundary node i as a TARGET:
//                   out_i = lam_i * sum_j mu_j dA_ij/dx_i
//
// with, for r = x_t - x_j != 0, rho = |r|^2, c = -w_j / (2 pi):
//   K       = c (r . n_j) / rho
//   dK/dx_t = c [n_j / rho - 2 (r . n_j) r / rho^2]  = -dK/dx_j
//   dK/dn_j = c r / rho
//   dK/dw_j = -(r . n_j) / (2 pi rho)
// Coincident pairs (the diagonal) are skipped; the diagonal entry
// 1/2 + kappa w / (4 pi) is differentiated on the host side of the pass.
// Layout as in the fast operator product: one thread per output node, the
// other side staged 256 at a time in shared memory, sums in a fixed order.
#include "ki_kernels.h"

namespace kib {

namespace {

constexpr int kAdjThreads = 256;

// eval points: xt (2 per point), lam (1 per point); sources: nodes[0, n).
// out: 6 per source node {d/dx, d/dy, d/dnx, d/dny, d/dw, K^T lam}.
__global__ void __launch_bounds__(kAdjThreads)
    adj_source_kernel(const Node* __restrict__ nodes, int n, const double* __restrict__ mu,
                      int nt, const double* __restrict__ xt, const double* __restrict__ lam,
                      double* __restrict__ out) {
  __shared__ double px[kAdjThreads], py[kAdjThreads], pl[kAdjThreads];
  const int j = blockIdx.x * kAdjThreads + threadIdx.x;
  double sx = 0, sy = 0, snx = 0, sny = 0, sw = 0;
  if (j < n) {
    const Node s = nodes[j];
    sx = s.x;
    sy = s.y;
    snx = s.nx;
    sny = s.ny;
    sw = s.w;
  }
  double gx = 0, gy = 0, gnx = 0, gny = 0, gw = 0, kt = 0;
  for (int base = 0; base < nt; base += kAdjThreads) {
    const int t = base + threadIdx.x;
    __syncthreads();
    if (t < nt) {
      px[threadIdx.x] = xt[2 * t];
      py[threadIdx.x] = xt[2 * t + 1];
      pl[threadIdx.x] = lam[t];
    } else {
      px[threadIdx.x] = 1e30;
      py[threadIdx.x] = 1e30;
      pl[threadIdx.x] = 0.0;
    }
    __syncthreads();
    const int cnt = min(kAdjThreads, nt - base);
#pragma unroll 4
    for (int q = 0; q < cnt; q++) {
      const double r0 = px[q] - sx, r1 = py[q] - sy;
      const double rho = r0 * r0 + r1 * r1;
      if (rho == 0.0) continue;
      const double inv = 1.0 / rho;
      const double rn = r0 * snx + r1 * sny;
      const double l = pl[q];
      const double a = l * rn * inv;        // lam (r.n) / rho
      kt += a;
      // dK/dx_j = -c [n / rho - 2 (r.n) r / rho^2]
      const double b = l * inv;             // lam / rho
      gx += b * snx - 2.0 * a * inv * r0;
      gy += b * sny - 2.0 * a * inv * r1;
      gnx += b * r0;
      gny += b * r1;
      gw += a;
    }
  }
  if (j < n) {
    const double c = -sw * KI_INV_2PI;
    const double m = mu[j];
    double* o = out + 6 * static_cast<long long>(j);
    o[0] = -c * m * gx;
    o[1] = -c * m * gy;
    o[2] = c * m * gnx;
    o[3] = c * m * gny;
    o[4] = -KI_INV_2PI * m * gw;
    o[5] = c * kt;
  }
}

// out: 2 per node {d/dx_i, d/dy_i} of lam_i sum_j A_ij mu_j (off-diagonal).
__global__ void __launch_bounds__(kAdjThreads)
    adj_target_kernel(const Node* __restrict__ nodes, int n, const double* __restrict__ mu,
                      const double* __restrict__ lam, double* __restrict__ out) {
  __shared__ double sx[kAdjThreads], sy[kAdjThreads], sa0[kAdjThreads], sa1[kAdjThreads];
  const int i = blockIdx.x * kAdjThreads + threadIdx.x;
  double tx = 0, ty = 0;
  if (i < n) {
    tx = nodes[i].x;
    ty = nodes[i].y;
  }
  double gx = 0, gy = 0;
  for (int base = 0; base < n; base += kAdjThreads) {
    const int j = base + threadIdx.x;
    __syncthreads();
    if (j < n) {
      const Node s = nodes[j];
      const double c = -s.w * KI_INV_2PI * mu[j];
      sx[threadIdx.x] = s.x;
      sy[threadIdx.x] = s.y;
      sa0[threadIdx.x] = c * s.nx;
      sa1[threadIdx.x] = c * s.ny;
    }
    __syncthreads();
    const int cnt = min(kAdjThreads, n - base);
#pragma unroll 4
    for (int q = 0; q < cnt; q++) {
      const double r0 = tx - sx[q], r1 = ty - sy[q];
      const double rho = r0 * r0 + r1 * r1;
      if (rho == 0.0) continue;
      const double inv = 1.0 / rho;
      const double rn = r0 * sa0[q] + r1 * sa1[q];  // c mu (r.n)
      // d/dx_t [c mu (r.n) / rho] = c mu n / rho - 2 c mu (r.n) r / rho^2
      gx += sa0[q] * inv - 2.0 * rn * inv * inv * r0;
      gy += sa1[q] * inv - 2.0 * rn * inv * inv * r1;
    }
  }
  if (i < n) {
    const double l = lam[i];
    out[2 * i] = l * gx;
    out[2 * i + 1] = l * gy;
  }
}

// Node gradients of J from the three pieces (all per node j):
//   target term  (source pass over the targets, weights g_u)      +
//   operator term (source pass over the nodes, weights lam;
//                  target pass; diagonal)                          -
__global__ void adj_combine_kernel(const Node* __restrict__ nodes, int n,
                                   const double* __restrict__ mu, const double* __restrict__ lam,
                                   const double* __restrict__ tgt_src,
                                   const double* __restrict__ op_src,
                                   const double* __restrict__ op_tgt, double* __restrict__ g_pts,
                                   double* __restrict__ g_nrm, double* __restrict__ g_w,
                                   double* __restrict__ g_k) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double* a = tgt_src + 6 * static_cast<long long>(j);
  const double* b = op_src + 6 * static_cast<long long>(j);
  const Node nd = nodes[j];
  const double lm = lam[j] * mu[j];
  g_pts[2 * j] = a[0] - b[0] - op_tgt[2 * j];
  g_pts[2 * j + 1] = a[1] - b[1] - op_tgt[2 * j + 1];
  g_nrm[2 * j] = a[2] - b[2];
  g_nrm[2 * j + 1] = a[3] - b[3];
  // diagonal 1/2 + kappa w / (4 pi)
  g_w[j] = a[4] - b[4] - lm * nd.k * (0.5 * KI_INV_2PI);
  g_k[j] = -lm * nd.w * (0.5 * KI_INV_2PI);
}

__global__ void adj_take_kt_kernel(const double* __restrict__ src6, int n,
                                   double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) out[j] = src6[6 * static_cast<long long>(j) + 5];
}

__global__ void node_xy_kernel(const Node* __restrict__ nodes, int n, double* __restrict__ xy) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) {
    xy[2 * j] = nodes[j].x;
    xy[2 * j + 1] = nodes[j].y;
  }
}

}  // namespace

cudaError_t launch_adjoint_laplace(const Node* nodes, int n, const double* mu, int nt,
                                   const double* targets, const double* grad_u, double* g_mu,
                                   double* work, cudaStream_t s) {
  // phase 1: g_mu = K_t^T grad_u and the target-term node gradients
  double* tgt_src = work;  // 6 n
  count_launches(2);
  adj_source_kernel<<<(n + kAdjThreads - 1) / kAdjThreads, kAdjThreads, 0, s>>>(
      nodes, n, mu, nt, targets, grad_u, tgt_src);
  adj_take_kt_kernel<<<(n + 255) / 256, 256, 0, s>>>(tgt_src, n, g_mu);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_laplace_finish(const Node* nodes, int n, const double* mu,
                                          const double* lam, double* work, double* g_pts,
                                          double* g_nrm, double* g_w, double* g_k,
                                          cudaStream_t s) {
  double* tgt_src = work;           // 6 n, from phase 1
  double* op_src = work + 6 * static_cast<long long>(n);   // 6 n
  double* op_tgt = op_src + 6 * static_cast<long long>(n); // 2 n
  double* xy = op_tgt + 2 * static_cast<long long>(n);     // 2 n
  const int nb = (n + kAdjThreads - 1) / kAdjThreads;
  count_launches(4);
  node_xy_kernel<<<(n + 255) / 256, 256, 0, s>>>(nodes, n, xy);
  adj_source_kernel<<<nb, kAdjThreads, 0, s>>>(nodes, n, mu, n, xy, lam, op_src);
  adj_target_kernel<<<nb, kAdjThreads, 0, s>>>(nodes, n, mu, lam, op_tgt);
  adj_combine_kernel<<<(n + 255) / 256, 256, 0, s>>>(nodes, n, mu, lam, tgt_src, op_src, op_tgt,
                                                     g_pts, g_nrm, g_w, g_k);
  return cudaGetLastError();
}

size_t adjoint_work_doubles(int n) { return 16 * static_cast<size_t>(n); }

}  // namespace kib
