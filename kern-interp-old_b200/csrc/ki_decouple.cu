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
//   X_rr^-1  by Gauss-Jordan elimination with partial pivoting (kept: the
//            solve sweeps multiply by it instead of solving with LU factors)
//   U        = X_rr^{-1} K_r_sn,  L = K_sn_r X_rr^{-1}   (GEMMs)
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
  const int n = tk.n, k = tk.k, r = n - k;  // n <= kSmemN: the host sends larger boxes
  const int* act = tk.act;                  // through decouple_large
  const int* perm = tk.perm;
  const int* bid = tk.bid;
  const int* bpos = tk.bpos;
  const double* T = tk.T;
  double* K = kbuf;
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
  // K_r_sn = K_rs - T^T K_ss   (r x k), in the U buffer for now
  cta_gemm_tiled(U, r, Krs_in, n, T, k, true, Kss, n, false, r, k, k, tile);
  // K_sn_r = K_sr - K_ss T     (k x r), in the L buffer for now
  cta_gemm_tiled(L, k, Ksr, n, Kss, n, false, T, k, false, k, r, k, tile);
  // X = (K_rr - T^T K_sr) - K_r_sn T
  cta_gemm_tiled(X, r, Krr, n, T, k, true, Ksr, n, false, r, r, k, tile);
  cta_gemm_tiled(X, r, X, r, U, r, false, T, k, false, r, r, k, tile);
  // K is done with: stage X, K_r_sn and K_sn_r in its place (r ldx + 2 k r
  // <= n^2) and invert X there (Gauss-Jordan, partial pivoting).  X's
  // leading dimension is odd where that fits (r <= k^2): the elimination's
  // row operations, a thread per column, then hit distinct banks
  const int ldx = (r | 1) * r + 2 * k * r <= n * n ? (r | 1) : r;
  double* Xw = kbuf;
  double* Krsn = Xw + ldx * r;  // r x k
  double* Ksnr = Krsn + r * k;  // k x r
  for (int e = threadIdx.x; e < r * r; e += kDecThreads) Xw[e % r + ldx * (e / r)] = X[e];
  for (int e = threadIdx.x; e < r * k; e += kDecThreads) {
    Krsn[e] = U[e];
    Ksnr[e] = L[e];
  }
  __syncthreads();
  // Gauss-Jordan with the pivot rows left in place (one barrier per step);
  // the result B gives X^{-1}(j, q) = B(p_j, p^{-1}(q)), gathered into X
  // in global memory and read back into shared memory for the products
  int* prow = reinterpret_cast<int*>(tile);  // the tile is free until U, L
  int* pinv = prow + kSmemN;
  unsigned long long* slot_key = reinterpret_cast<unsigned long long*>(pinv + kSmemN);
  int* slot_row = reinterpret_cast<int*>(slot_key + 64);
  double* colj = reinterpret_cast<double*>(slot_row + 64);  // 2 r
  const int info = cta_gj_invert_inplace(Xw, r, ldx, prow, slot_key, slot_row, colj);
  if (info && threadIdx.x == 0) atomicExch(P.status, 1);
  for (int j = threadIdx.x; j < r; j += kDecThreads) {
    pinv[prow[j]] = j;
    piv[j] = prow[j];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < r * r; e += kDecThreads) {
    const int j = e % r, q = e / r;
    X[e] = Xw[prow[j] + ldx * pinv[q]];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < r * r; e += kDecThreads) Xw[e % r + ldx * (e / r)] = X[e];
  __syncthreads();
  // U = X^{-1} K_r_sn,  L = K_sn_r X^{-1}
  cta_gemm_tiled(U, r, nullptr, 0, Xw, ldx, false, Krsn, r, false, r, k, r, tile, 1.0);
  cta_gemm_tiled(L, k, nullptr, 0, Ksnr, k, false, Xw, ldx, false, k, r, r, tile, 1.0);
  // acc = update(s, s) + L K_r_sn
  cta_gemm_tiled(acc, k, nullptr, 0, L, k, false, Krsn, r, false, k, k, r, tile, 1.0);
  for (int e = threadIdx.x; e < k * k; e += kDecThreads) {
    const int i = e % k, j = e / k;
    acc[e] += upd_lookup(bid, bpos, tk.blocks, perm[i], perm[j]);
  }
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

__global__ void identity_kernel(double* y, int r) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < r * r) y[e] = (e % r == e / r) ? 1.0 : 0.0;
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
  // X^{-1}: LU, then the solve of X Y = I (one CTA per column), into X
  // through the K scratch (K is no longer needed); K_r_sn and K_sn_r are
  // kept behind it (r^2 + 2 k r <= n^2)
  double* Y = tk.K;
  double* Krsn = Y + static_cast<long long>(r) * r;
  double* Ksnr = Krsn + static_cast<long long>(r) * k;
  if ((e = cudaMemcpyAsync(Krsn, tk.U, sizeof(double) * r * k, cudaMemcpyDeviceToDevice, s)))
    return e;
  if ((e = cudaMemcpyAsync(Ksnr, tk.L, sizeof(double) * r * k, cudaMemcpyDeviceToDevice, s)))
    return e;
  if ((e = dense_lu(tk.X, r, r, tk.piv, status, s, reinterpret_cast<int*>(tk.K + nn)))) return e;
  count_launches(1);
  identity_kernel<<<(r * r + 255) / 256, 256, 0, s>>>(Y, r);
  if ((e = cudaGetLastError())) return e;
  if ((e = dense_lu_solve(tk.X, r, r, tk.piv, Y, r, r, s))) return e;
  if ((e = cudaMemcpyAsync(tk.X, Y, sizeof(double) * r * r, cudaMemcpyDeviceToDevice, s))) return e;
  // U = X^{-1} K_r_sn, L = K_sn_r X^{-1}, acc = update + L K_r_sn
  if ((e = launch_gemm_tiled(tk.U, r, nullptr, 0, tk.X, r, false, Krsn, r, false, r, k, r, 1.0,
                             s)))
    return e;
  if ((e = launch_gemm_tiled(tk.L, k, nullptr, 0, Ksnr, k, false, tk.X, r, false, k, r, r, 1.0,
                             s)))
    return e;
  if ((e = launch_gemm_sub(tk.acc, k, nullptr, 0, tk.L, k, false, Krsn, r, false, k, k, r, s)))
    return e;
  acc_finish_kernel<<<(k * k + 255) / 256, 256, 0, s>>>(tk.acc, k, tk.perm, tk.bid, tk.bpos,
                                                         tk.blocks);
  return cudaGetLastError();
}

size_t decouple_smem_bytes(int n_max) {
  const int ns = n_max < kSmemN ? n_max : kSmemN;
  return sizeof(double) * (kGemmTileDoubles + 64 + static_cast<size_t>(ns) * ns);
}

cudaError_t launch_decouple(const DecParams& p, int n_max, cudaStream_t s) {
  if (p.ntasks == 0) return cudaSuccess;
  const size_t smem = decouple_smem_bytes(n_max);
  cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&decouple_kernel),
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
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
