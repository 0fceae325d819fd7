// Level-synchronous solve sweeps (SkelFactorization::solve and
// multiply_connected_solve, skel_factorization.cpp:341-551).  Boxes of one
// level own disjoint dofs, so every box of a level is swept in the same
// launch, one warp per box, with the box's skeleton and redundant entries
// staged in shared memory:
//   up:    x[r] -= T^T x[s];  x[s] -= L x[r]      (apply_sweep_matrix :301-318)
//          (x[s] -= U^T x[r] when sweeping Psi^T, skel_factorization.cpp:253-270)
//   diag:  x[r] = X_rr^{-1} x[r]                  (apply_diag_inv_matrix :331-338)
//   down:  x[r] -= U x[s];    x[s] -= T x[r]
#include "ki_blockla.cuh"
#include "ki_kernels.h"

namespace kib {

namespace {

constexpr int kSweepWarps = 4;

__device__ __forceinline__ int row_of(const SweepParams& P, int dof) {
  return P.red_pos_map ? P.red_pos[dof] : dof;
}

template <int MODE>  // 0 up (L), 1 up (U^T), 2 down
__global__ void __launch_bounds__(32 * kSweepWarps) sweep_kernel(SweepParams P, int cap) {
  extern __shared__ double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * kSweepWarps + warp;
  if (b >= P.ntasks) return;
  const SweepTask tk = P.tasks[b];
  const int k = tk.k, r = tk.r;
  double* xs = sm + static_cast<long long>(warp) * cap;
  double* xr = xs + k;
  const int* S = tk.skel;
  const int* R = tk.red;
  const double* T = tk.T;
  const double* L = tk.L;
  const double* U = tk.U;
  for (int c = 0; c < P.nrhs; c++) {
    double* x = P.x + static_cast<long long>(P.ldx) * c;
    for (int i = lane; i < k; i += 32) xs[i] = x[S[i]];
    for (int j = lane; j < r; j += 32) xr[j] = x[R[j]];
    __syncwarp();
    if (MODE <= 1) {
      for (int j = lane; j < r; j += 32) {
        const double* tc = T + static_cast<long long>(k) * j;
        double s = 0.0;
        for (int l = 0; l < k; l++) s += tc[l] * xs[l];
        xr[j] -= s;
      }
      __syncwarp();
      for (int i = lane; i < k; i += 32) {
        double s = 0.0;
        if (MODE == 0) {
          for (int j = 0; j < r; j++) s += L[i + static_cast<long long>(k) * j] * xr[j];
        } else {
          const double* uc = U + static_cast<long long>(r) * i;
          for (int j = 0; j < r; j++) s += uc[j] * xr[j];
        }
        xs[i] -= s;
      }
    } else {
      for (int j = lane; j < r; j += 32) {
        double s = 0.0;
        for (int l = 0; l < k; l++) s += U[j + static_cast<long long>(r) * l] * xs[l];
        xr[j] -= s;
      }
      __syncwarp();
      for (int i = lane; i < k; i += 32) {
        double s = 0.0;
        for (int j = 0; j < r; j++) s += T[i + static_cast<long long>(k) * j] * xr[j];
        xs[i] -= s;
      }
    }
    __syncwarp();
    for (int i = lane; i < k; i += 32) x[S[i]] = xs[i];
    for (int j = lane; j < r; j += 32) x[R[j]] = xr[j];
    __syncwarp();
  }
}

__global__ void __launch_bounds__(32 * kSweepWarps) diag_kernel(SweepParams P, int cap) {
  extern __shared__ double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * kSweepWarps + warp;
  if (b >= P.ntasks) return;
  const SweepTask tk = P.tasks[b];
  const int r = tk.r;
  double* xr = sm + static_cast<long long>(warp) * cap;
  const int* R = tk.red;
  const double* X = tk.X;
  const int* piv = tk.piv;
  for (int c = 0; c < P.nrhs; c++) {
    double* x = P.x + static_cast<long long>(P.ldx) * c;
    for (int j = lane; j < r; j += 32) xr[j] = x[row_of(P, R[j])];
    __syncwarp();
    warp_lu_solve(X, r, r, piv, xr, 1);
    for (int j = lane; j < r; j += 32) x[row_of(P, R[j])] = xr[j];
    __syncwarp();
  }
}

}  // namespace

cudaError_t launch_sweep_up(const SweepParams& p, bool use_u, cudaStream_t s) {
  if (p.ntasks == 0) return cudaSuccess;
  const int cap = p.cap;
  const size_t smem = sizeof(double) * static_cast<size_t>(cap) * kSweepWarps;
  const int grid = (p.ntasks + kSweepWarps - 1) / kSweepWarps;
  if (use_u) {
    cudaFuncSetAttribute(sweep_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
    sweep_kernel<1><<<grid, 32 * kSweepWarps, smem, s>>>(p, cap);
  } else {
    cudaFuncSetAttribute(sweep_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
    sweep_kernel<0><<<grid, 32 * kSweepWarps, smem, s>>>(p, cap);
  }
  return cudaGetLastError();
}

cudaError_t launch_sweep_down(const SweepParams& p, cudaStream_t s) {
  if (p.ntasks == 0) return cudaSuccess;
  const int cap = p.cap;
  const size_t smem = sizeof(double) * static_cast<size_t>(cap) * kSweepWarps;
  cudaFuncSetAttribute(sweep_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  sweep_kernel<2><<<(p.ntasks + kSweepWarps - 1) / kSweepWarps, 32 * kSweepWarps, smem, s>>>(
      p, cap);
  return cudaGetLastError();
}

cudaError_t launch_diag_solve(const SweepParams& p, cudaStream_t s) {
  if (p.ntasks == 0) return cudaSuccess;
  const int cap = p.cap;
  const size_t smem = sizeof(double) * static_cast<size_t>(cap) * kSweepWarps;
  cudaFuncSetAttribute(diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  diag_kernel<<<(p.ntasks + kSweepWarps - 1) / kSweepWarps, 32 * kSweepWarps, smem, s>>>(p, cap);
  return cudaGetLastError();
}

}  // namespace kib
