// Level-synchronous solve sweeps (SkelFactorization::solve and
// multiply_connected_solve, skel_factorization.cpp:341-551).  Boxes of one
// level own disjoint dofs, so every box of a level is swept in the same
// launch, one CTA per box, with the box's skeleton and redundant entries of
// up to kRhsChunk right-hand sides staged in shared memory:
//   up:    x[r] -= T^T x[s];  x[s] -= L x[r]      (apply_sweep_matrix :301-318)
//          (x[s] -= U^T x[r] when sweeping Psi^T, skel_factorization.cpp:253-270)
//   diag:  x[r] = X_rr^{-1} x[r]                  (apply_diag_inv_matrix :331-338)
//   down:  x[r] -= U x[s];    x[s] -= T x[r]
// Staged vectors are stored dof-major (row * nc + rhs) so the threads that
// share a matrix entry read consecutive shared-memory words.
#include "ki_blockla.cuh"
#include "ki_kernels.h"

namespace kib {

namespace {

constexpr int kSweepThreads = 128;
constexpr int kRhsChunk = 8;
constexpr int kDiagWarps = 4;

__device__ __forceinline__ int row_of(const SweepParams& P, int dof) {
  return P.red_pos_map ? P.red_pos[dof] : dof;
}

// out[i, c] -= sum_l M(i, l) * in[l, c] with M(i, l) = A[i * si + l * sl].
__device__ __forceinline__ void apply_sub(double* out, const double* in, int rows, int inner,
                                          int nc, const double* A, long long si, long long sl) {
  for (int t = threadIdx.x; t < rows * nc; t += kSweepThreads) {
    const int i = t / nc, c = t - i * nc;
    const double* a = A + si * i;
    double s0 = 0.0, s1 = 0.0;
    int l = 0;
    for (; l + 1 < inner; l += 2) {
      s0 += a[sl * l] * in[l * nc + c];
      s1 += a[sl * (l + 1)] * in[(l + 1) * nc + c];
    }
    if (l < inner) s0 += a[sl * l] * in[l * nc + c];
    out[i * nc + c] -= s0 + s1;
  }
}

template <int MODE>  // 0 up (L), 1 up (U^T), 2 down
__global__ void __launch_bounds__(kSweepThreads) sweep_kernel(SweepParams P) {
  extern __shared__ double sm[];
  const SweepTask tk = P.tasks[blockIdx.x];
  const int k = tk.k, r = tk.r;
  const int* S = tk.skel;
  const int* R = tk.red;
  for (int c0 = 0; c0 < P.nrhs; c0 += kRhsChunk) {
    const int nc = min(kRhsChunk, P.nrhs - c0);
    double* xs = sm;
    double* xr = sm + k * nc;
    for (int t = threadIdx.x; t < k * nc; t += kSweepThreads) {
      const int i = t / nc, c = t - i * nc;
      xs[t] = P.x[S[i] + static_cast<long long>(P.ldx) * (c0 + c)];
    }
    for (int t = threadIdx.x; t < r * nc; t += kSweepThreads) {
      const int j = t / nc, c = t - j * nc;
      xr[t] = P.x[R[j] + static_cast<long long>(P.ldx) * (c0 + c)];
    }
    __syncthreads();
    if (MODE <= 1) {
      // xr -= T^T xs : (T^T)(j, l) = T[l + k j]
      apply_sub(xr, xs, r, k, nc, tk.T, k, 1);
      __syncthreads();
      if (MODE == 0) {
        // xs -= L xr : L(i, j) = L[i + k j]
        apply_sub(xs, xr, k, r, nc, tk.L, 1, k);
      } else {
        // xs -= U^T xr : (U^T)(i, j) = U[j + r i]
        apply_sub(xs, xr, k, r, nc, tk.U, r, 1);
      }
    } else {
      // xr -= U xs : U(j, l) = U[j + r l]
      apply_sub(xr, xs, r, k, nc, tk.U, 1, r);
      __syncthreads();
      // xs -= T xr : T(i, j) = T[i + k j]
      apply_sub(xs, xr, k, r, nc, tk.T, 1, k);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < k * nc; t += kSweepThreads) {
      const int i = t / nc, c = t - i * nc;
      P.x[S[i] + static_cast<long long>(P.ldx) * (c0 + c)] = xs[t];
    }
    for (int t = threadIdx.x; t < r * nc; t += kSweepThreads) {
      const int j = t / nc, c = t - j * nc;
      P.x[R[j] + static_cast<long long>(P.ldx) * (c0 + c)] = xr[t];
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(32 * kDiagWarps) diag_kernel(SweepParams P, int cap) {
  extern __shared__ double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * kDiagWarps + warp;
  if (b >= P.ntasks) return;
  const SweepTask tk = P.tasks[b];
  const int r = tk.r;
  double* xr = sm + static_cast<long long>(warp) * cap;
  const int* R = tk.red;
  for (int c = 0; c < P.nrhs; c++) {
    double* x = P.x + static_cast<long long>(P.ldx) * c;
    for (int j = lane; j < r; j += 32) xr[j] = x[row_of(P, R[j])];
    __syncwarp();
    warp_lu_solve(tk.X, r, r, tk.piv, xr, 1);
    for (int j = lane; j < r; j += 32) x[row_of(P, R[j])] = xr[j];
    __syncwarp();
  }
}

template <int MODE>
cudaError_t launch_mode(const SweepParams& p, cudaStream_t s) {
  const int nc = p.nrhs < kRhsChunk ? p.nrhs : kRhsChunk;
  const size_t smem = sizeof(double) * static_cast<size_t>(p.cap) * nc;
  cudaError_t e = cudaFuncSetAttribute(sweep_kernel<MODE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  sweep_kernel<MODE><<<p.ntasks, kSweepThreads, smem, s>>>(p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_sweep_up(const SweepParams& p, bool use_u, cudaStream_t s) {
  if (p.ntasks == 0 || p.nrhs == 0) return cudaSuccess;
  count_launches(1);
  return use_u ? launch_mode<1>(p, s) : launch_mode<0>(p, s);
}

cudaError_t launch_sweep_down(const SweepParams& p, cudaStream_t s) {
  if (p.ntasks == 0 || p.nrhs == 0) return cudaSuccess;
  count_launches(1);
  return launch_mode<2>(p, s);
}

cudaError_t launch_diag_solve(const SweepParams& p, cudaStream_t s) {
  if (p.ntasks == 0 || p.nrhs == 0) return cudaSuccess;
  const int cap = p.cap;
  const size_t smem = sizeof(double) * static_cast<size_t>(cap) * kDiagWarps;
  cudaError_t e = cudaFuncSetAttribute(diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  count_launches(1);
  diag_kernel<<<(p.ntasks + kDiagWarps - 1) / kDiagWarps, 32 * kDiagWarps, smem, s>>>(p, cap);
  return cudaGetLastError();
}

}  // namespace kib
