// Level-synchronous solve sweeps (SkelFactorization::solve and
// multiply_connected_solve, skel_factorization.cpp:341-551).  Boxes of one
// level own disjoint dofs, so every box of a level is swept in the same
// launch, one CTA per box, with the box's skeleton and redundant entries of
// up to 32 right-hand sides staged in shared memory:
//   up:    x[r] -= T^T x[s];  x[s] -= L x[r]      (apply_sweep_matrix :301-318)
//          (x[s] -= U^T x[r] when sweeping Psi^T, skel_factorization.cpp:253-270)
//   diag:  x[r] = X_rr^{-1} x[r]                  (apply_diag_inv_matrix :331-338)
//   down:  x[r] -= U x[s];    x[s] -= T x[r]
// Staged vectors are stored dof-major (row * nc + rhs) so the threads that
// share a matrix entry read consecutive shared-memory words.
#include <algorithm>

#include "ki_blockla.cuh"
#include "ki_kernels.h"

namespace kib {

namespace {

constexpr int kSweepThreads = 128;
constexpr int kRhsChunkMax = 32;
constexpr size_t kSweepSmemBudget = 96 * 1024;

// Right-hand sides staged per pass: as many as fit the shared-memory budget
// (up to 32), so a box's T, L, U are read once per pass.
inline int rhs_chunk(int nrhs, int cap) {
  const int fit = static_cast<int>(kSweepSmemBudget / (sizeof(double) * (cap > 0 ? cap : 1)));
  return std::max(1, std::min(std::min(nrhs, kRhsChunkMax), fit));
}
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

template <int MODE>  // 0 up (L), 1 up (U^T), 2 down, 3 transposed up (L^T, T)
__global__ void __launch_bounds__(kSweepThreads) sweep_kernel(SweepParams P, int chunk) {
  extern __shared__ double sm[];
  const SweepTask tk = P.tasks[blockIdx.x];
  const int k = tk.k, r = tk.r;
  const int* S = tk.skel;
  const int* R = tk.red;
  for (int c0 = 0; c0 < P.nrhs; c0 += chunk) {
    const int nc = min(chunk, P.nrhs - c0);
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
    } else if (MODE == 2) {
      // xr -= U xs : U(j, l) = U[j + r l]
      apply_sub(xr, xs, r, k, nc, tk.U, 1, r);
      __syncthreads();
      // xs -= T xr : T(i, j) = T[i + k j]
      apply_sub(xs, xr, k, r, nc, tk.T, 1, k);
    } else {
      // xr -= L^T xs : (L^T)(j, l) = L[l + k j]
      apply_sub(xr, xs, r, k, nc, tk.L, k, 1);
      __syncthreads();
      // xs -= T xr
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

// X_rr^{-1} on a box's redundant entries of up to `chunk` right-hand sides
// at once, one CTA per box, the entries staged dof-major in shared memory:
// pivots, then blocked unit-L and U substitution in 32-row blocks (warps
// take the right-hand sides of a diagonal block, all threads the updates
// below / above it).  The LU factors are read with coalesced column loads.
constexpr int kDiagCtaThreads = 256;
__global__ void __launch_bounds__(kDiagCtaThreads) diag_cta_kernel(SweepParams P, int chunk) {
  extern __shared__ double xs[];
  const SweepTask tk = P.tasks[blockIdx.x];
  const int r = tk.r;
  const double* lu = tk.X;
  const int* R = tk.red;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int nw = kDiagCtaThreads / 32;
  for (int c0 = 0; c0 < P.nrhs; c0 += chunk) {
    const int nc = min(chunk, P.nrhs - c0);
    for (int t = threadIdx.x; t < r * nc; t += kDiagCtaThreads) {
      const int j = t / nc, c = t - j * nc;
      xs[t] = P.x[row_of(P, R[j]) + static_cast<long long>(P.ldx) * (c0 + c)];
    }
    __syncthreads();
    if (threadIdx.x < nc)
      for (int i = 0; i < r; i++) {
        const int p = tk.piv[i];
        if (p != i) {
          const double t = xs[i * nc + threadIdx.x];
          xs[i * nc + threadIdx.x] = xs[p * nc + threadIdx.x];
          xs[p * nc + threadIdx.x] = t;
        }
      }
    __syncthreads();
    for (int kb = 0; kb < r; kb += 32) {  // unit L
      const int nbk = min(32, r - kb);
      double Lr[32];
#pragma unroll
      for (int k = 0; k < 32; k++)
        Lr[k] = (lane < nbk && k < lane) ? lu[kb + lane + static_cast<long long>(r) * (kb + k)] : 0.0;
      for (int c = warp; c < nc; c += nw) {
        double xv = lane < nbk ? xs[(kb + lane) * nc + c] : 0.0;
#pragma unroll
        for (int k = 0; k < 32; k++) xv -= Lr[k] * __shfl_sync(0xffffffffu, xv, k);
        if (lane < nbk) xs[(kb + lane) * nc + c] = xv;
      }
      __syncthreads();
      const int below = r - kb - nbk;
      for (int t = threadIdx.x; t < below * nc; t += kDiagCtaThreads) {
        const int i = kb + nbk + t / nc, c = t % nc;
        double s = 0.0;
        for (int k = 0; k < nbk; k++) s += lu[i + static_cast<long long>(r) * (kb + k)] * xs[(kb + k) * nc + c];
        xs[i * nc + c] -= s;
      }
      __syncthreads();
    }
    for (int kb = ((r - 1) / 32) * 32; kb >= 0; kb -= 32) {  // U
      const int nbk = min(32, r - kb);
      double Ur[32];
#pragma unroll
      for (int k = 0; k < 32; k++)
        Ur[k] = (lane < nbk && k < nbk && k >= lane)
                    ? lu[kb + lane + static_cast<long long>(r) * (kb + k)]
                    : 0.0;
      for (int c = warp; c < nc; c += nw) {
        double xv = lane < nbk ? xs[(kb + lane) * nc + c] : 0.0;
#pragma unroll
        for (int k = 31; k >= 0; k--) {
          if (k < nbk) {
            if (lane == k) xv /= Ur[k];
            const double xk = __shfl_sync(0xffffffffu, xv, k);
            if (lane < k) xv -= Ur[k] * xk;
          }
        }
        if (lane < nbk) xs[(kb + lane) * nc + c] = xv;
      }
      __syncthreads();
      for (int t = threadIdx.x; t < kb * nc; t += kDiagCtaThreads) {
        const int i = t / nc, c = t % nc;
        double s = 0.0;
        for (int k = 0; k < nbk; k++) s += lu[i + static_cast<long long>(r) * (kb + k)] * xs[(kb + k) * nc + c];
        xs[i * nc + c] -= s;
      }
      __syncthreads();
    }
    for (int t = threadIdx.x; t < r * nc; t += kDiagCtaThreads) {
      const int j = t / nc, c = t - j * nc;
      P.x[row_of(P, R[j]) + static_cast<long long>(P.ldx) * (c0 + c)] = xs[t];
    }
    __syncthreads();
  }
}

template <bool TRANS>
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
    if (TRANS)
      warp_lu_solve_t(tk.X, r, r, tk.piv, xr, 1);
    else
      warp_lu_solve(tk.X, r, r, tk.piv, xr, 1);
    for (int j = lane; j < r; j += 32) x[row_of(P, R[j])] = xr[j];
    __syncwarp();
  }
}

template <int MODE>
cudaError_t launch_mode(const SweepParams& p, cudaStream_t s) {
  const int nc = rhs_chunk(p.nrhs, p.cap);
  const size_t smem = sizeof(double) * static_cast<size_t>(p.cap) * nc;
  cudaError_t e = cudaFuncSetAttribute(sweep_kernel<MODE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  sweep_kernel<MODE><<<p.ntasks, kSweepThreads, smem, s>>>(p, nc);
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

cudaError_t launch_transposed_up(const SweepParams& p, cudaStream_t s) {
  if (p.ntasks == 0 || p.nrhs == 0) return cudaSuccess;
  count_launches(1);
  return launch_mode<3>(p, s);
}

namespace {
template <bool TRANS>
cudaError_t launch_diag(const SweepParams& p, cudaStream_t s) {
  if (p.ntasks == 0 || p.nrhs == 0) return cudaSuccess;
  const int cap = p.cap;
  const size_t smem = sizeof(double) * static_cast<size_t>(cap) * kDiagWarps;
  cudaError_t e = cudaFuncSetAttribute(diag_kernel<TRANS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  count_launches(1);
  diag_kernel<TRANS><<<(p.ntasks + kDiagWarps - 1) / kDiagWarps, 32 * kDiagWarps, smem, s>>>(
      p, cap);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_diag_solve(const SweepParams& p, cudaStream_t s) {
  if (p.ntasks == 0 || p.nrhs == 0) return cudaSuccess;
  const int nc = rhs_chunk(p.nrhs, p.cap);
  const size_t smem = sizeof(double) * static_cast<size_t>(p.cap > 0 ? p.cap : 1) * nc;
  cudaError_t e = cudaFuncSetAttribute(diag_cta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  count_launches(1);
  diag_cta_kernel<<<p.ntasks, kDiagCtaThreads, smem, s>>>(p, nc);
  return cudaGetLastError();
}

cudaError_t launch_diag_solve_t(const SweepParams& p, cudaStream_t s) { return launch_diag<true>(p, s); }

}  // namespace kib
