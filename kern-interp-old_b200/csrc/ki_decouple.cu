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

// Boxes with n <= kSmemN keep K_BN, and then X_rr, in shared memory.
constexpr int kSmemN = kDecoupleSmemN;

__global__ void __launch_bounds__(kDecThreads) decouple_kernel(DecParams P) {
  extern __shared__ __align__(16) double dsm[];
  double* tile = dsm;                     // kGemmTileDoubles
  double* red = tile + kGemmTileDoubles;  // 64
  double* kbuf = red + 64;                // n*n when staged
  const DecTask tk = P.tasks[blockIdx.x];
  const int n = tk.n, k = tk.k, r = n - k;
  const bool staged = n <= kSmemN;
  const int* act = tk.act;
  const int* perm = tk.perm;
  const int* bid = tk.bid;
  const int* bpos = tk.bpos;
  const double* T = tk.T;
  double* K = staged ? kbuf : tk.K;
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
  // K_r_sn = K_rs - T^T K_ss   (r x k), kept in the U buffer until the end
  cta_gemm_tiled(U, r, Krs_in, n, T, k, true, Kss, n, false, r, k, k, tile);
  // K_sn_r = K_sr - K_ss T     (k x r), in the L buffer
  cta_gemm_tiled(L, k, Ksr, n, Kss, n, false, T, k, false, k, r, k, tile);
  // X = (K_rr - T^T K_sr) - K_r_sn T
  cta_gemm_tiled(X, r, Krr, n, T, k, true, Ksr, n, false, r, r, k, tile);
  cta_gemm_tiled(X, r, X, r, U, r, false, T, k, false, r, r, k, tile);
  // LU of X_rr, in shared memory when it fits (K is no longer needed)
  double* Xw = X;
  if (staged) {
    Xw = kbuf;
    for (int e = threadIdx.x; e < r * r; e += kDecThreads) Xw[e] = X[e];
    __syncthreads();
  }
  const int info = cta_lu(Xw, r, r, piv, red);
  if (info && threadIdx.x == 0) atomicExch(P.status, 1);
  if (staged) {
    for (int e = threadIdx.x; e < r * r; e += kDecThreads) X[e] = Xw[e];
  }
  __syncthreads();
  // L = K_sn_r X^{-1}, row by row through X^T
  const int warp = threadIdx.x >> 5;
  const int nw = kDecThreads / 32;
  for (int row = warp; row < k; row += nw) warp_lu_solve_t(Xw, r, r, piv, L + row, k);
  __syncthreads();
  // acc = update(s, s) + L K_r_sn
  cta_gemm_tiled(acc, k, nullptr, 0, L, k, false, U, r, false, k, k, r, tile);
  for (int e = threadIdx.x; e < k * k; e += kDecThreads) {
    const int i = e % k, j = e / k;
    acc[e] = upd_lookup(bid, bpos, tk.blocks, perm[i], perm[j]) - acc[e];
  }
  // U = X^{-1} K_r_sn, column by column
  for (int c = warp; c < k; c += nw) warp_lu_solve(Xw, r, r, piv, U + static_cast<long long>(r) * c, 1);
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

__global__ void assemble_perm_kernel(int pde, const Node* nodes, const int* act, const int* perm,
                                     int n, const int* bid, const int* bpos,
                                     const UpdBlock* blocks, double* K) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= static_cast<long long>(n) * n) return;
  const int a = static_cast<int>(e % n), b = static_cast<int>(e / n);
  const int pa = perm[a], pb = perm[b];
  K[e] = boundary_entry(pde, nodes, act[pa], act[pb]) - upd_lookup(bid, bpos, blocks, pa, pb);
}

__global__ void acc_finish_kernel(double* acc, int k, const int* perm, const int* bid,
                                  const int* bpos, const UpdBlock* blocks) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= k * k) return;
  const int i = e % k, j = e / k;
  acc[e] = upd_lookup(bid, bpos, blocks, perm[i], perm[j]) - acc[e];
}

}  // namespace

cudaError_t decouple_large(const DecTask& tk, int pde, const Node* nodes, int* status,
                           cudaStream_t s) {
  const int n = tk.n, k = tk.k, r = n - k;
  const long long nn = static_cast<long long>(n) * n;
  count_launches(2);
  assemble_perm_kernel<<<static_cast<int>((nn + 255) / 256), 256, 0, s>>>(
      pde, nodes, tk.act, tk.perm, n, tk.bid, tk.bpos, tk.blocks, tk.K);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const double* K = tk.K;
  const double* Kss = K;
  const double* Krs_in = K + k;
  const double* Ksr = K + static_cast<long long>(n) * k;
  const double* Krr = K + k + static_cast<long long>(n) * k;
  // K_r_sn in U, K_sn_r in L, X = (K_rr - T^T K_sr) - K_r_sn T
  if ((e = launch_gemm_sub(tk.U, r, Krs_in, n, tk.T, k, true, Kss, n, false, r, k, k, s))) return e;
  if ((e = launch_gemm_sub(tk.L, k, Ksr, n, Kss, n, false, tk.T, k, false, k, r, k, s))) return e;
  if ((e = launch_gemm_sub(tk.X, r, Krr, n, tk.T, k, true, Ksr, n, false, r, r, k, s))) return e;
  if ((e = launch_gemm_sub(tk.X, r, tk.X, r, tk.U, r, false, tk.T, k, false, r, r, k, s))) return e;
  if ((e = dense_lu(tk.X, r, r, tk.piv, status, s))) return e;
  if ((e = dense_lu_solve_rows(tk.X, r, r, tk.piv, tk.L, k, k, s))) return e;
  if ((e = launch_gemm_sub(tk.acc, k, nullptr, 0, tk.L, k, false, tk.U, r, false, k, k, r, s)))
    return e;
  acc_finish_kernel<<<(k * k + 255) / 256, 256, 0, s>>>(tk.acc, k, tk.perm, tk.bid, tk.bpos,
                                                         tk.blocks);
  if ((e = cudaGetLastError())) return e;
  return dense_lu_solve(tk.X, r, r, tk.piv, tk.U, k, r, s);
}

size_t decouple_smem_bytes(int n_max) {
  const int ns = n_max < kSmemN ? n_max : kSmemN;
  return sizeof(double) * (kGemmTileDoubles + 64 + static_cast<size_t>(ns) * ns);
}

cudaError_t launch_decouple(const DecParams& p, int n_max, cudaStream_t s) {
  if (p.ntasks == 0) return cudaSuccess;
  const size_t smem = decouple_smem_bytes(n_max);
  cudaError_t e = cudaFuncSetAttribute(decouple_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  count_launches(1);
  decouple_kernel<<<p.ntasks, kDecThreads, smem, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_assemble_top(int pde, const Node* nodes, const int* dofs, int n,
                                const int* bid, const int* bpos, const UpdBlock* blocks,
                                double* out, int ld, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const long long total = static_cast<long long>(n) * n;
  const int threads = 256;
  const int grid = static_cast<int>((total + threads - 1) / threads);
  count_launches(1);
  assemble_top_kernel<<<grid, threads, 0, s>>>(pde, nodes, dofs, n, bid, bpos, blocks, out,
                                                ld);
  return cudaGetLastError();
}

}  // namespace kib
