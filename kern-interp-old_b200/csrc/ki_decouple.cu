// Decoupling of every compressed box of a level in one launch
// (SkelFactorization::decouple, skel_factorization.cpp:55-91), and the dense
// assembly of the top-level skeleton matrix (skel_factorization.cpp:116-122).
//
// Per box, in pivot order [s; r] of the ID:
//   K_BN     = K(act, act) - (accumulated Schur updates of compressed boxes
//              below, restricted to the active dofs)
//   K_r_sn   = K_rs - T^T K_ss
//   X_rr     = (K_rr - T^T K_sr) - K_r_sn T
//   K_sn_r   = K_sr - K_ss T
//   X_rr     = P L U                        (partial pivoting)
//   U        = X_rr^{-1} K_r_sn,  L = K_sn_r X_rr^{-1}
//   acc      = update(s, s) + L K_r_sn      (what the ancestors subtract)
// The reference re-searches every compressed descendant's skeleton inside
// the parent's index list (skel_factorization.cpp:246-294); here each box
// passes up one accumulated update on its skeleton, addressed through
// per-position block ids built on the host, so assembly is a direct lookup.
#include "ki_blockla.cuh"
#include "ki_kernels.h"

namespace kib {

namespace {

constexpr int kDecThreads = 256;

__device__ __forceinline__ double upd_lookup(const int* bid, const int* bpos,
                                             const UpdBlock* blocks, int a, int b) {
  const int ia = bid[a];
  if (ia < 0 || ia != bid[b]) return 0.0;
  const UpdBlock blk = blocks[ia];
  return blk.acc[bpos[a] + static_cast<long long>(blk.size) * bpos[b]];
}

__global__ void __launch_bounds__(kDecThreads) decouple_kernel(DecParams P) {
  __shared__ double red[64];
  const DecTask tk = P.tasks[blockIdx.x];
  const int n = tk.n, k = tk.k, r = n - k;
  const int* act = tk.act;
  const int* perm = tk.perm;
  const int* bid = tk.bid;
  const int* bpos = tk.bpos;
  const double* T = tk.T;
  double* K = tk.K;
  double* Krs = tk.Krs;
  double* L = tk.L;
  double* U = tk.U;
  double* X = tk.X;
  double* acc = tk.acc;
  int* piv = tk.piv;

  // K_BN in pivot order
  for (int e = threadIdx.x; e < n * n; e += kDecThreads) {
    const int a = e % n, b = e / n;
    const int pa = perm[a], pb = perm[b];
    const double kv = boundary_entry(P.pde, P.nodes, act[pa], act[pb]);
    K[e] = kv - upd_lookup(bid, bpos, tk.blocks, pa, pb);
  }
  __syncthreads();
  const double* Kss = K;
  const double* Krs_in = K + k;
  const double* Ksr = K + static_cast<long long>(n) * k;
  const double* Krr = K + k + static_cast<long long>(n) * k;
  // K_r_sn = K_rs - T^T K_ss            (r x k)
  cta_gemm_sub(Krs, r, Krs_in, n, T, k, true, Kss, n, false, r, k, k);
  // K_sn_r = K_sr - K_ss T  -> L buffer  (k x r)
  cta_gemm_sub(L, k, Ksr, n, Kss, n, false, T, k, false, k, r, k);
  // X = K_rr - T^T K_sr                  (r x r)
  cta_gemm_sub(X, r, Krr, n, T, k, true, Ksr, n, false, r, r, k);
  __syncthreads();
  // X -= K_r_sn T
  cta_gemm_sub(X, r, X, r, Krs, r, false, T, k, false, r, r, k);
  __syncthreads();
  const int info = cta_lu(X, r, r, piv, red);
  if (info && threadIdx.x == 0) atomicExch(P.status, 1);
  // U = X^{-1} K_r_sn (columns), L = K_sn_r X^{-1} (rows, through X^T)
  for (int e = threadIdx.x; e < r * k; e += kDecThreads) U[e] = Krs[e];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = kDecThreads / 32;
  for (int c = warp; c < k; c += nw) warp_lu_solve(X, r, r, piv, U + static_cast<long long>(r) * c, 1);
  for (int row = warp; row < k; row += nw) warp_lu_solve_t(X, r, r, piv, L + row, k);
  __syncthreads();
  // acc = update(s, s) + L K_r_sn
  for (int e = threadIdx.x; e < k * k; e += kDecThreads) {
    const int i = e % k, j = e / k;
    double s = 0.0;
    for (int l = 0; l < r; l++) s += L[i + static_cast<long long>(k) * l] * Krs[l + static_cast<long long>(r) * j];
    acc[e] = upd_lookup(bid, bpos, tk.blocks, perm[i], perm[j]) + s;
  }
  (void)lane;
}

__global__ void assemble_top_kernel(int pde, const Node* nodes, const int* dofs, int n,
                                    const int* bid, const int* bpos, const UpdBlock* blocks,
                                    double* out, int ld) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= static_cast<long long>(n) * n) return;
  const int a = static_cast<int>(e % n), b = static_cast<int>(e / n);
  out[a + static_cast<long long>(ld) * b] =
      boundary_entry(pde, nodes, dofs[a], dofs[b]) - upd_lookup(bid, bpos, blocks, a, b);
}

}  // namespace

cudaError_t launch_decouple(const DecParams& p, cudaStream_t s) {
  if (p.ntasks == 0) return cudaSuccess;
  decouple_kernel<<<p.ntasks, kDecThreads, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_assemble_top(int pde, const Node* nodes, const int* dofs, int n,
                                const int* bid, const int* bpos, const UpdBlock* blocks,
                                double* out, int ld, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const long long total = static_cast<long long>(n) * n;
  const int threads = 256;
  const int grid = static_cast<int>((total + threads - 1) / threads);
  assemble_top_kernel<<<grid, threads, 0, s>>>(pde, nodes, dofs, n, bid, bpos, blocks, out,
                                                ld);
  return cudaGetLastError();
}

}  // namespace kib
