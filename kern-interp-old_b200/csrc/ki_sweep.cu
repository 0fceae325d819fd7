// Level-synchronous solve sweeps (SkelFactorization::solve and
// multiply_connected_solve, skel_factorization.cpp:341-551).  Boxes of one
// level own disjoint dofs, so every box of a level is swept in the same
// launch, one CTA per box, with the box's skeleton and redundant entries of
// up to 32 right-hand sides staged in shared memory:
//   up:    x[r] -= T^T x[s];  x[s] -= L x[r]      (apply_sweep_matrix :301-318)
//          (x[s] -= U^T x[r] when sweeping Psi^T, skel_factorization.cpp:253-270)
//   diag:  x[r] = X_rr^{-1} x[r]                  (apply_diag_inv_matrix :331-338;
//          the factorization keeps X_rr^{-1} itself, so this is a product)
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

// Asynchronous 8-byte copies global -> shared (cp.async; waited for with
// cp_async_wait_all before a barrier).
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void stage_async(double* dst, const double* src, int cnt) {
  for (int e = threadIdx.x; e < cnt; e += blockDim.x) cp_async8(dst + e, src + e);
}

__device__ __forceinline__ int row_of(const SweepParams& P, int dof) {
  return P.red_pos_map ? P.red_pos[dof] : dof;
}

// out[i, c] -= sum_l M(i, l) * in[l, c] with M(i, l) = A[i * si + l * sl].
__device__ __forceinline__ void apply_sub(double* out, const double* in, int rows, int inner,
                                          int nc, const double* A, long long si, long long sl) {
  for (int t = threadIdx.x; t < rows * nc; t += blockDim.x) {
    const int i = t / nc, c = t - i * nc;
    const double* a = A + si * i;
    // four independent loads in flight per thread
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int l = 0;
    for (; l + 3 < inner; l += 4) {
      const double a0 = a[sl * l], a1 = a[sl * (l + 1)], a2 = a[sl * (l + 2)],
                   a3 = a[sl * (l + 3)];
      s0 += a0 * in[l * nc + c];
      s1 += a1 * in[(l + 1) * nc + c];
      s2 += a2 * in[(l + 2) * nc + c];
      s3 += a3 * in[(l + 3) * nc + c];
    }
    for (; l < inner; l++) s0 += a[sl * l] * in[l * nc + c];
    out[i * nc + c] -= (s0 + s1) + (s2 + s3);
  }
}

// The same for several right-hand sides: a thread owns one output row and a
// group of up to kGrp right-hand sides, so each matrix entry is loaded once
// for the whole group (the lanes of a warp hold consecutive rows of one
// group and read the same staged vector entry).
constexpr int kGrp = 8;
__device__ __forceinline__ void apply_sub_multi(double* out, const double* in, int rows, int inner,
                                                int nc, const double* A, long long si,
                                                long long sl) {
  const int ng = (nc + kGrp - 1) / kGrp;
  for (int t = threadIdx.x; t < rows * ng; t += blockDim.x) {
    const int i = t % rows, g = t / rows;
    const int c0 = g * kGrp, m = min(kGrp, nc - c0);
    const double* a = A + si * i;
    double acc[kGrp];
#pragma unroll
    for (int c = 0; c < kGrp; c++) acc[c] = 0.0;
    int l = 0;
    for (; l + 3 < inner; l += 4) {
      const double av0 = a[sl * l], av1 = a[sl * (l + 1)], av2 = a[sl * (l + 2)],
                   av3 = a[sl * (l + 3)];
      const double* x = in + l * nc + c0;
#pragma unroll
      for (int c = 0; c < kGrp; c++)
        if (c < m)
          acc[c] += av0 * x[c] + av1 * x[nc + c] + av2 * x[2 * nc + c] + av3 * x[3 * nc + c];
    }
    for (; l < inner; l++) {
      const double av = a[sl * l];
      const double* x = in + l * nc + c0;
#pragma unroll
      for (int c = 0; c < kGrp; c++)
        if (c < m) acc[c] += av * x[c];
    }
#pragma unroll
    for (int c = 0; c < kGrp; c++)
      if (c < m) out[i * nc + c0 + c] -= acc[c];
  }
}

// One right-hand side on a wide CTA (a level of a few large boxes, the
// factors read from global memory): where the inner index is contiguous
// (sl = 1) a warp per output row, lanes over the inner index (coalesced,
// eight loads in flight per lane per pass); otherwise threads over the
// contiguous rows with the inner index cut into segments, partial sums
// through shared memory (part: segments x rows doubles) added in segment
// order.  Ends with a barrier.
constexpr int kWideThreads = 512;
__device__ __forceinline__ void apply_sub_wide(double* out, const double* in, int rows, int inner,
                                               const double* A, long long si, long long sl,
                                               double* part) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (sl == 1) {
    for (int i = warp; i < rows; i += nw) {
      const double* a = A + si * i;
      double acc[8];
#pragma unroll
      for (int u = 0; u < 8; u++) acc[u] = 0.0;
      for (int l0 = 0; l0 < inner; l0 += 256) {
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int l = l0 + 32 * u + lane;
          if (l < inner) acc[u] += a[l] * in[l];
        }
      }
      double s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) out[i] -= s;
    }
    __syncthreads();
    return;
  }
  const int rows32 = (rows + 31) & ~31;
  const int nseg = max(1, min(static_cast<int>(blockDim.x) / max(rows32, 1), 16));
  const int seg_len = (inner + nseg - 1) / nseg;
  for (int t = threadIdx.x; t < rows32 * nseg; t += blockDim.x) {
    const int i = t % rows32, g = t / rows32;
    double s = 0.0;
    if (i < rows) {
      const double* a = A + si * i;
      const int l1 = min(inner, (g + 1) * seg_len);
      double acc[8];
#pragma unroll
      for (int u = 0; u < 8; u++) acc[u] = 0.0;
      for (int l0 = g * seg_len; l0 < l1; l0 += 8) {
#pragma unroll
        for (int u = 0; u < 8; u++)
          if (l0 + u < l1) acc[u] += a[sl * (l0 + u)] * in[l0 + u];
      }
      s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    }
    part[g * rows32 + i] = s;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    double s = 0.0;
    for (int g = 0; g < nseg; g++) s += part[g * rows32 + i];
    out[i] -= s;
  }
  __syncthreads();
}

__device__ __forceinline__ void apply_any(double* out, const double* in, int rows, int inner,
                                          int nc, const double* A, long long si, long long sl,
                                          double* part = nullptr) {
  if (part) {
    apply_sub_wide(out, in, rows, inner, A, si, sl, part);
  } else if (nc == 1) {
    apply_sub(out, in, rows, inner, nc, A, si, sl);
  } else {
    apply_sub_multi(out, in, rows, inner, nc, A, si, sl);
  }
}

template <int MODE>  // 0 up (L), 1 up (U^T), 2 down, 3 transposed up (L^T, T)
__device__ __forceinline__ void sweep_body(const SweepParams& P, int chunk, double* sm,
                                           bool wide = false) {
  const SweepTask tk = P.tasks[blockIdx.x];
  const int k = tk.k, r = tk.r;
  const int* S = tk.skel;
  const int* R = tk.red;
  // the two factor matrices of this mode (each k r entries, contiguous)
  const double* F1 = MODE == 2 ? tk.U : MODE == 3 ? tk.L : tk.T;
  const double* F2 = MODE == 0 ? tk.L : MODE == 1 ? tk.U : tk.T;
  const bool staged = P.kr > 0 && chunk == 1;  // (uniform over the launch)
  if (staged) {
    double* f1 = sm + P.cap;
    stage_async(f1, F1, k * r);
    stage_async(f1 + P.kr, F2, k * r);
    F1 = f1;
    F2 = f1 + P.kr;
  }
  // wide CTA, one right-hand side: partial-sum scratch after the vector
  double* part = wide && chunk == 1 ? sm + P.cap : nullptr;
  for (int c0 = 0; c0 < P.nrhs; c0 += chunk) {
    const int nc = min(chunk, P.nrhs - c0);
    double* xs = sm;
    double* xr = sm + k * nc;
    for (int t = threadIdx.x; t < k * nc; t += blockDim.x) {
      const int i = t / nc, c = t - i * nc;
      xs[t] = P.x[static_cast<long long>(S[i]) * P.ldd + static_cast<long long>(P.ldx) * (c0 + c)];
    }
    for (int t = threadIdx.x; t < r * nc; t += blockDim.x) {
      const int j = t / nc, c = t - j * nc;
      xr[t] = P.x[static_cast<long long>(R[j]) * P.ldd + static_cast<long long>(P.ldx) * (c0 + c)];
    }
    if (staged) cp_async_wait_all();
    __syncthreads();
    if (MODE <= 1) {
      // xr -= T^T xs : (T^T)(j, l) = T[l + k j]
      apply_any(xr, xs, r, k, nc, F1, k, 1, part);
      __syncthreads();
      if (MODE == 0) {
        // xs -= L xr : L(i, j) = L[i + k j]
        apply_any(xs, xr, k, r, nc, F2, 1, k, part);
      } else {
        // xs -= U^T xr : (U^T)(i, j) = U[j + r i]
        apply_any(xs, xr, k, r, nc, F2, r, 1, part);
      }
    } else if (MODE == 2) {
      // xr -= U xs : U(j, l) = U[j + r l]
      apply_any(xr, xs, r, k, nc, F1, 1, r, part);
      __syncthreads();
      // xs -= T xr : T(i, j) = T[i + k j]
      apply_any(xs, xr, k, r, nc, F2, 1, k, part);
    } else {
      // xr -= L^T xs : (L^T)(j, l) = L[l + k j]
      apply_any(xr, xs, r, k, nc, F1, k, 1, part);
      __syncthreads();
      // xs -= T xr
      apply_any(xs, xr, k, r, nc, F2, 1, k, part);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < k * nc; t += blockDim.x) {
      const int i = t / nc, c = t - i * nc;
      P.x[static_cast<long long>(S[i]) * P.ldd + static_cast<long long>(P.ldx) * (c0 + c)] = xs[t];
    }
    for (int t = threadIdx.x; t < r * nc; t += blockDim.x) {
      const int j = t / nc, c = t - j * nc;
      P.x[static_cast<long long>(R[j]) * P.ldd + static_cast<long long>(P.ldx) * (c0 + c)] = xr[t];
    }
    __syncthreads();
  }
}

// The solve is a chain of short dependent launches (a few per level, up
// and down the tree).  They are launched as programmatic dependents of the
// kernel before them: the launch is processed while that kernel's last
// blocks drain, and each block first waits (griddepcontrol.wait) until the
// previous grid has completed and its writes are visible, so no read of x
// can overtake its producer.  Outside such a launch the wait returns at once.
__device__ __forceinline__ void wait_prior_grid() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... KArgs, typename... Args>
cudaError_t launch_chained(void (*kernel)(KArgs...), int blocks, int threads, size_t smem,
                           cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, args...);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <int MODE>
__global__ void __launch_bounds__(kSweepThreads) sweep_kernel(SweepParams P, int chunk) {
  wait_prior_grid();
  extern __shared__ double sm[];
  sweep_body<MODE>(P, chunk, sm);
}

// A level of a few large boxes, one right-hand side, factors not staged:
// 512 threads per box (see apply_sub_wide).
template <int MODE>
__global__ void __launch_bounds__(kWideThreads) sweep_wide_kernel(SweepParams P) {
  wait_prior_grid();
  extern __shared__ double sm[];
  sweep_body<MODE>(P, 1, sm, true);
}

// The two up sweeps of the hole border (U with L, Psi^T with U^T) of one
// level in one launch: blockIdx.y picks the sweep.
__global__ void __launch_bounds__(kSweepThreads) sweep_pair_kernel(SweepParams pu, SweepParams pp,
                                                                   int chunk) {
  extern __shared__ double sm[];
  if (blockIdx.y == 0) {
    sweep_body<0>(pu, chunk, sm);
  } else {
    sweep_body<1>(pp, chunk, sm);
  }
}

// x_r <- X_rr^{-1} x_r (TRANS: X_rr^{-T} x_r) on every box's redundant entries,
// one CTA per box, up to `chunk` right-hand sides per pass staged dof-major
// in shared memory; the decoupling stored X_rr^{-1} itself, so this is a
// small matrix product (coalesced column reads) with no sequential steps.
constexpr int kDiagThreads = 256;
template <bool TRANS>
__global__ void __launch_bounds__(kDiagThreads) diag_inv_kernel(SweepParams P, int chunk) {
  wait_prior_grid();
  extern __shared__ double sm[];
  const SweepTask tk = P.tasks[blockIdx.x];
  const int r = tk.r;
  const double* Xi = tk.X;
  const int* R = tk.red;
  // one right-hand side: X^{-1} staged in shared memory (P.kr = max r^2)
  const bool staged = P.kr > 0 && chunk == 1;
  if (staged) {
    double* xi = sm + 2 * P.cap;
    stage_async(xi, Xi, r * r);
    Xi = xi;
  }
  for (int c0 = 0; c0 < P.nrhs; c0 += chunk) {
    const int nc = min(chunk, P.nrhs - c0);
    double* xs = sm;
    double* ys = sm + static_cast<long long>(r) * nc;
    for (int t = threadIdx.x; t < r * nc; t += kDiagThreads) {
      const int j = t / nc, c = t - j * nc;
      xs[t] = P.x[static_cast<long long>(row_of(P, R[j])) * P.ldd + static_cast<long long>(P.ldx) * (c0 + c)];
    }
    if (staged) cp_async_wait_all();
    __syncthreads();
    if (nc > 1) {
      // a row and a group of right-hand sides per thread: each X^{-1}
      // entry is loaded once for the group
      const int ng = (nc + kGrp - 1) / kGrp;
      for (int t = threadIdx.x; t < r * ng; t += kDiagThreads) {
        const int i = t % r, g = t / r;
        const int cg = g * kGrp, m = min(kGrp, nc - cg);
        double acc[kGrp];
#pragma unroll
        for (int c = 0; c < kGrp; c++) acc[c] = 0.0;
        auto xa = [&](int j) {
          return TRANS ? Xi[j + static_cast<long long>(r) * i] : Xi[i + static_cast<long long>(r) * j];
        };
        int j = 0;
        for (; j + 3 < r; j += 4) {
          const double a0 = xa(j), a1 = xa(j + 1), a2 = xa(j + 2), a3 = xa(j + 3);
          const double* x = xs + j * nc + cg;
#pragma unroll
          for (int c = 0; c < kGrp; c++)
            if (c < m)
              acc[c] += a0 * x[c] + a1 * x[nc + c] + a2 * x[2 * nc + c] + a3 * x[3 * nc + c];
        }
        for (; j < r; j++) {
          const double a = xa(j);
          const double* x = xs + j * nc + cg;
#pragma unroll
          for (int c = 0; c < kGrp; c++)
            if (c < m) acc[c] += a * x[c];
        }
#pragma unroll
        for (int c = 0; c < kGrp; c++)
          if (c < m) ys[i * nc + cg + c] = acc[c];
      }
    } else
    for (int t = threadIdx.x; t < r * nc; t += kDiagThreads) {
      const int i = t % r, c = t / r;  // consecutive threads: consecutive rows i
      auto xa = [&](int j) {
        return TRANS ? Xi[j + static_cast<long long>(r) * i] : Xi[i + static_cast<long long>(r) * j];
      };
      double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
      int j = 0;
      for (; j + 3 < r; j += 4) {
        const double a0 = xa(j), a1 = xa(j + 1), a2 = xa(j + 2), a3 = xa(j + 3);
        s0 += a0 * xs[j * nc + c];
        s1 += a1 * xs[(j + 1) * nc + c];
        s2 += a2 * xs[(j + 2) * nc + c];
        s3 += a3 * xs[(j + 3) * nc + c];
      }
      for (; j < r; j++) s0 += xa(j) * xs[j * nc + c];
      ys[i * nc + c] = (s0 + s1) + (s2 + s3);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < r * nc; t += kDiagThreads) {
      const int j = t / nc, c = t - j * nc;
      P.x[static_cast<long long>(row_of(P, R[j])) * P.ldd + static_cast<long long>(P.ldx) * (c0 + c)] = ys[t];
    }
    __syncthreads();
  }
}

// A single right-hand side stages the factors when both fit next to the
// vector in this much shared memory.
constexpr size_t kStageSmemMax = 100 * 1024;
// Levels of at most this many boxes whose factors are not staged sweep a
// single right-hand side with wide CTAs.
constexpr int kWideMaxBoxes = 64;

template <int MODE>
cudaError_t launch_mode(const SweepParams& p0, cudaStream_t s) {
  SweepParams p = p0;
  const int nc = rhs_chunk(p.nrhs, p.cap);
  size_t smem = sizeof(double) * static_cast<size_t>(p.cap) * nc;
  if (nc == 1 && p.kr > 0 && smem + 2 * sizeof(double) * static_cast<size_t>(p.kr) <= kStageSmemMax)
    smem += 2 * sizeof(double) * static_cast<size_t>(p.kr);
  else
    p.kr = 0;
  if (nc == 1 && p.kr == 0 && p.ntasks <= kWideMaxBoxes) {
    // the partial sums: segments x rows rounded to 32, at most the larger
    // of kWideThreads and the rows rounded up (a single segment)
    const size_t wsmem =
        smem + sizeof(double) * (std::max(kWideThreads, (p.cap + 31) & ~31) + 64);
    cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&sweep_wide_kernel<MODE>),
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(wsmem));
    if (e != cudaSuccess) return e;
    return launch_chained(sweep_wide_kernel<MODE>, p.ntasks, kWideThreads, wsmem, s, p);
  }
  cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&sweep_kernel<MODE>),
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  return launch_chained(sweep_kernel<MODE>, p.ntasks, kSweepThreads, smem, s, p, nc);
}

}  // namespace

cudaError_t launch_sweep_up(const SweepParams& p, bool use_u, cudaStream_t s) {
  if (p.ntasks == 0 || p.nrhs == 0) return cudaSuccess;
  count_launches(1);
  return use_u ? launch_mode<1>(p, s) : launch_mode<0>(p, s);
}

cudaError_t launch_sweep_up_pair(const SweepParams& pu, const SweepParams& pp, cudaStream_t s) {
  if (pu.ntasks == 0 || pu.nrhs == 0) return cudaSuccess;
  const int nc = rhs_chunk(pu.nrhs, pu.cap);
  const size_t smem = sizeof(double) * static_cast<size_t>(pu.cap) * nc;
  cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&sweep_pair_kernel),
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  count_launches(1);
  sweep_pair_kernel<<<dim3(pu.ntasks, 2), kSweepThreads, smem, s>>>(pu, pp, nc);
  return cudaGetLastError();
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
// The diagonal step of a few large boxes, one right-hand side: 512 threads
// per box, x_r <- X^{-1} x_r through apply_sub_wide (ys = 0 - X^{-1} xs,
// stored negated).
template <bool TRANS>
__global__ void __launch_bounds__(kWideThreads) diag_wide_kernel(SweepParams P) {
  wait_prior_grid();
  extern __shared__ double sm[];
  const SweepTask tk = P.tasks[blockIdx.x];
  const int r = tk.r;
  const int* R = tk.red;
  double* xs = sm;
  double* ys = sm + P.cap;
  double* part = ys + P.cap;
  for (int j = threadIdx.x; j < r; j += blockDim.x) {
    xs[j] = P.x[static_cast<long long>(row_of(P, R[j])) * P.ldd];
    ys[j] = 0.0;
  }
  __syncthreads();
  if (TRANS) {
    apply_sub_wide(ys, xs, r, r, tk.X, r, 1, part);  // X^{-T}(i, j) = X[j + r i]
  } else {
    apply_sub_wide(ys, xs, r, r, tk.X, 1, r, part);  // X^{-1}(i, j) = X[i + r j]
  }
  for (int j = threadIdx.x; j < r; j += blockDim.x)
    P.x[static_cast<long long>(row_of(P, R[j])) * P.ldd] = -ys[j];
}

template <bool TRANS>
cudaError_t launch_diag(const SweepParams& p0, cudaStream_t s) {
  if (p0.ntasks == 0 || p0.nrhs == 0) return cudaSuccess;
  SweepParams p = p0;
  const int nc = rhs_chunk(p.nrhs, 2 * (p.cap > 0 ? p.cap : 1));
  size_t smem = 2 * sizeof(double) * static_cast<size_t>(p.cap > 0 ? p.cap : 1) * nc;
  if (nc == 1 && p.kr > 0 && smem + sizeof(double) * static_cast<size_t>(p.kr) <= kStageSmemMax)
    smem += sizeof(double) * static_cast<size_t>(p.kr);
  else
    p.kr = 0;
  if (nc == 1 && p.kr == 0 && p.ntasks <= kWideMaxBoxes) {
    const size_t wsmem = sizeof(double) * (2 * static_cast<size_t>(p.cap) +
                                           std::max(kWideThreads, (p.cap + 31) & ~31) + 64);
    cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&diag_wide_kernel<TRANS>),
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(wsmem));
    if (e != cudaSuccess) return e;
    count_launches(1);
    return launch_chained(diag_wide_kernel<TRANS>, p.ntasks, kWideThreads, wsmem, s, p);
  }
  cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&diag_inv_kernel<TRANS>),
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  count_launches(1);
  return launch_chained(diag_inv_kernel<TRANS>, p.ntasks, kDiagThreads, smem, s, p, nc);
}
}  // namespace

cudaError_t launch_diag_solve(const SweepParams& p, cudaStream_t s) { return launch_diag<false>(p, s); }

cudaError_t launch_diag_solve_t(const SweepParams& p, cudaStream_t s) { return launch_diag<true>(p, s); }

}  // namespace kib
