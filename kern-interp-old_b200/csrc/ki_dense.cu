// Dense FP64 building blocks on the device: blocked LU with partial pivoting
// for the top-level skeleton system (the reference's LU_factorize / dgetrf,
// ki_mat.cpp:427-433, applied at skel_factorization.cpp:124-128 and :308),
// its solve (dgetrs, ki_mat.cpp:467-480), small GEMMs and gather/scatter.
//
// The LU is right-looking with 32-column panels: one CTA factors the panel
// (pivot search over the whole column, dgetf2 steps), then the row
// interchanges are applied to the other columns, U12 = L11^{-1} A12 is formed
// per column, and the trailing matrix is updated by a tiled GEMM spread over
// the whole GPU.
#include <atomic>

#include "ki_blockla.cuh"
#include "ki_kernels.h"

namespace kib {

namespace {
std::atomic<long long> g_launches{0};
}  // namespace

void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_total() { return g_launches.load(std::memory_order_relaxed); }

namespace {

constexpr int kNb = 32;

// Panel factorization of a(j0:n, j0:j0+w) with partial pivoting over rows
// j0..n-1; swaps are applied inside the panel only.
__global__ void __launch_bounds__(1024) panel_lu_kernel(double* a, int n, int ld, int j0,
                                                        int w, int* ipiv, int* status) {
  __shared__ double red[32];
  __shared__ int redi[32];
  __shared__ int sp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  for (int jj = 0; jj < w; jj++) {
    const int j = j0 + jj;
    double bv = -1.0;
    int bp = 0x7fffffff;
    for (int i = j + threadIdx.x; i < n; i += blockDim.x) {
      const double v = fabs(a[i + static_cast<long long>(ld) * j]);
      if (v > bv || (v == bv && i < bp)) {
        bv = v;
        bp = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int op = __shfl_xor_sync(0xffffffffu, bp, o);
      if (ov > bv || (ov == bv && op < bp)) {
        bv = ov;
        bp = op;
      }
    }
    if (lane == 0) {
      red[warp] = bv;
      redi[warp] = bp;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = red[0];
      int p = redi[0];
      for (int q = 1; q < nw; q++)
        if (red[q] > v || (red[q] == v && redi[q] < p)) {
          v = red[q];
          p = redi[q];
        }
      sp = p;
      ipiv[j] = p;
    }
    __syncthreads();
    const int p = sp;
    const double piv = a[p + static_cast<long long>(ld) * j];
    if (piv != 0.0) {
      if (p != j && threadIdx.x < w) {
        double* x = a + static_cast<long long>(ld) * (j0 + threadIdx.x);
        const double t = x[j];
        x[j] = x[p];
        x[p] = t;
      }
      __syncthreads();
      const double inv = 1.0 / piv;
      for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x)
        a[i + static_cast<long long>(ld) * j] *= inv;
    } else if (threadIdx.x == 0) {
      atomicExch(status, 1);
    }
    __syncthreads();
    // rank-one update of the panel's remaining columns: a warp per column,
    // lanes over the rows
    for (int c = j0 + jj + 1 + warp; c < j0 + w; c += nw) {
      double* ac = a + static_cast<long long>(ld) * c;
      const double ajc = ac[j];
      if (ajc != 0.0) {
        const double* aj = a + static_cast<long long>(ld) * j;
        for (int i = j + 1 + lane; i < n; i += 32) ac[i] -= aj[i] * ajc;
      }
    }
    __syncthreads();
  }
}

// The same panel factorization with the panel staged in shared memory
// (rows n - j0, w columns, leading dimension ldp): the column steps touch
// only on-chip data, and the panel is written back once.
__global__ void __launch_bounds__(1024) panel_lu_smem_kernel(double* a, int n, int ld, int j0,
                                                             int w, int* ipiv, int* status) {
  extern __shared__ double P[];
  __shared__ double red[32];
  __shared__ int redi[32];
  __shared__ int sp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const int rows = n - j0, ldp = rows | 1;
  for (int e = threadIdx.x; e < rows * w; e += blockDim.x) {
    const int i = e % rows, c = e / rows;
    P[i + ldp * c] = a[j0 + i + static_cast<long long>(ld) * (j0 + c)];
  }
  __syncthreads();
  for (int jj = 0; jj < w; jj++) {
    const double* col = P + ldp * jj;
    double bv = -1.0;
    int bp = 0x7fffffff;
    for (int i = jj + threadIdx.x; i < rows; i += blockDim.x) {
      const double v = fabs(col[i]);
      if (v > bv || (v == bv && i < bp)) {
        bv = v;
        bp = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int op = __shfl_xor_sync(0xffffffffu, bp, o);
      if (ov > bv || (ov == bv && op < bp)) {
        bv = ov;
        bp = op;
      }
    }
    if (lane == 0) {
      red[warp] = bv;
      redi[warp] = bp;
    }
    __syncthreads();
    if (warp == 0) {
      double v = lane < nw ? red[lane] : -1.0;
      int q = lane < nw ? redi[lane] : 0x7fffffff;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oq = __shfl_xor_sync(0xffffffffu, q, o);
        if (ov > v || (ov == v && oq < q)) {
          v = ov;
          q = oq;
        }
      }
      if (lane == 0) {
        sp = q;
        ipiv[j0 + jj] = j0 + q;
      }
    }
    __syncthreads();
    const int p = sp;
    if (p != jj && threadIdx.x < w) {
      double* x = P + ldp * threadIdx.x;
      const double t = x[jj];
      x[jj] = x[p];
      x[p] = t;
    }
    __syncthreads();
    const double piv = col[jj];
    if (piv == 0.0) {
      if (threadIdx.x == 0) atomicExch(status, 1);
    } else {
      const double inv = 1.0 / piv;
      for (int i = jj + 1 + threadIdx.x; i < rows; i += blockDim.x) P[i + ldp * jj] *= inv;
    }
    __syncthreads();
    // rank-one update of the panel's remaining columns: a warp per column,
    // lanes over the rows
    for (int c = jj + 1 + warp; c < w; c += nw) {
      double* pc = P + ldp * c;
      const double pjc = pc[jj];
      if (pjc != 0.0) {
        const double* pj = P + ldp * jj;
        for (int i = jj + 1 + lane; i < rows; i += 32) pc[i] -= pj[i] * pjc;
      }
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < rows * w; e += blockDim.x) {
    const int i = e % rows, c = e / rows;
    a[j0 + i + static_cast<long long>(ld) * (j0 + c)] = P[i + ldp * c];
  }
}

// Row interchanges of panel j0 applied to every column outside the panel.
__global__ void swap_kernel(double* a, int n, int ld, int j0, int w, const int* ipiv) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || (c >= j0 && c < j0 + w)) return;
  double* x = a + static_cast<long long>(ld) * c;
  for (int jj = 0; jj < w; jj++) {
    const int j = j0 + jj, p = ipiv[j];
    if (p != j) {
      const double t = x[j];
      x[j] = x[p];
      x[p] = t;
    }
  }
}

// A12 <- L11^{-1} A12 (unit lower), one thread per column right of the panel.
__global__ void trsm_row_kernel(double* a, int n, int ld, int j0, int w) {
  const int c = j0 + w + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double* x = a + static_cast<long long>(ld) * c;
  double b[kNb];
#pragma unroll
  for (int i = 0; i < kNb; i++) b[i] = i < w ? x[j0 + i] : 0.0;
#pragma unroll
  for (int kk = 0; kk < kNb; kk++) {
    if (kk >= w) break;
    const double v = b[kk];
#pragma unroll
    for (int i = kk + 1; i < kNb; i++)
      if (i < w) b[i] -= v * a[j0 + i + static_cast<long long>(ld) * (j0 + kk)];
  }
#pragma unroll
  for (int i = 0; i < kNb; i++)
    if (i < w) x[j0 + i] = b[i];
}

// A22 -= A21 A12 for the trailing block, 64 x 64 tiles, inner dimension w.
__global__ void __launch_bounds__(256) trailing_kernel(double* a, int n, int ld, int j0, int w) {
  __shared__ double sa[kNb][64 + 1];
  __shared__ double sb[kNb][64 + 1];
  const int s0 = j0 + w;
  const int r0 = s0 + blockIdx.x * 64, c0 = s0 + blockIdx.y * 64;
  for (int e = threadIdx.x; e < 64 * kNb; e += 256) {
    const int i = e % 64, l = e / 64;
    const int gi = r0 + i, gc = c0 + i;
    sa[l][i] = (gi < n && l < w) ? a[gi + static_cast<long long>(ld) * (j0 + l)] : 0.0;
    sb[l][i] = (gc < n && l < w) ? a[j0 + l + static_cast<long long>(ld) * gc] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4] = {};
#pragma unroll 4
  for (int l = 0; l < kNb; l++) {
    double av[4], bv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      av[q] = sa[l][tx + 16 * q];
      bv[q] = sb[l][ty + 16 * q];
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int t = 0; t < 4; t++) acc[q][t] += av[q] * bv[t];
  }
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const int gi = r0 + tx + 16 * q, gc = c0 + ty + 16 * t;
      if (gi < n && gc < n) a[gi + static_cast<long long>(ld) * gc] -= acc[q][t];
    }
}

// B <- A^{-1} B, one CTA per right-hand side, the vector in shared memory.
constexpr int kSolveThreads = 512;
__global__ void __launch_bounds__(kSolveThreads)
    lu_solve_cta_kernel(const double* __restrict__ lu, int n, int ld, const int* __restrict__ ipiv,
                        double* b, int ldb) {
  extern __shared__ double x[];
  double* bc = b + static_cast<long long>(ldb) * blockIdx.x;
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = bc[i];
  __syncthreads();
  cta_lu_solve(lu, n, ld, ipiv, x);
  for (int i = threadIdx.x; i < n; i += blockDim.x) bc[i] = x[i];
}

// B <- A^{-1} B with one warp per right-hand side.
__global__ void lu_solve_kernel(const double* lu, int n, int ld, const int* ipiv, double* b,
                                int nrhs, int ldb) {
  const int c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (c >= nrhs) return;
  warp_lu_solve(lu, n, ld, ipiv, b + static_cast<long long>(ldb) * c, 1);
}

__global__ void gather_kernel(const double* x, int ldx, const int* idx, int n, int nrhs,
                              double* out, int ldo) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= static_cast<long long>(n) * nrhs) return;
  const int i = static_cast<int>(e % n), c = static_cast<int>(e / n);
  out[i + static_cast<long long>(ldo) * c] = x[idx[i] + static_cast<long long>(ldx) * c];
}

__global__ void gather_rows_kernel(const double* x, int ldd, const int* idx, int n, int nrhs,
                                   double* out, int ldo) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= static_cast<long long>(n) * nrhs) return;
  const int c = static_cast<int>(e % nrhs), i = static_cast<int>(e / nrhs);
  out[i + static_cast<long long>(ldo) * c] = x[static_cast<long long>(idx[i]) * ldd + c];
}

__global__ void scatter_kernel(double* x, int ldx, const int* idx, int n, int nrhs,
                               const double* in, int ldi) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= static_cast<long long>(n) * nrhs) return;
  const int i = static_cast<int>(e % n), c = static_cast<int>(e / n);
  x[idx[i] + static_cast<long long>(ldx) * c] = in[i + static_cast<long long>(ldi) * c];
}

__global__ void gemm_kernel(bool ta, bool tb, int m, int n, int k, double alpha,
                            const double* a, int lda, const double* b, int ldb, double beta,
                            double* c, int ldc) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= static_cast<long long>(m) * n) return;
  const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
  double s = 0.0;
  for (int l = 0; l < k; l++) {
    const double av = ta ? a[l + static_cast<long long>(lda) * i] : a[i + static_cast<long long>(lda) * l];
    const double bv = tb ? b[j + static_cast<long long>(ldb) * l] : b[l + static_cast<long long>(ldb) * j];
    s += av * bv;
  }
  double* cp = c + i + static_cast<long long>(ldc) * j;
  *cp = alpha * s + (beta == 0.0 ? 0.0 : beta * *cp);
}

// C(i, j) = alpha * sum_l A(l, i) B(l, j) + beta C(i, j) for a long inner
// dimension: one CTA per output entry, strided partial sums, block reduce.
__global__ void __launch_bounds__(256) gemm_tn_long_kernel(int m, int k, double alpha,
                                                           const double* a, int lda,
                                                           const double* b, int ldb,
                                                           double beta, double* c, int ldc) {
  __shared__ double red[8];
  const int i = blockIdx.x % m, j = blockIdx.x / m;
  const double* ac = a + static_cast<long long>(lda) * i;
  const double* bc = b + static_cast<long long>(ldb) * j;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int l = threadIdx.x;
  for (; l + 768 < k; l += 1024) {
    s0 += ac[l] * bc[l];
    s1 += ac[l + 256] * bc[l + 256];
    s2 += ac[l + 512] * bc[l + 512];
    s3 += ac[l + 768] * bc[l + 768];
  }
  for (; l < k; l += 256) s0 += ac[l] * bc[l];
  double t = warp_sum_d((s0 + s1) + (s2 + s3));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < 8; w++) v += red[w];
    double* cp = c + i + static_cast<long long>(ldc) * j;
    *cp = alpha * v + (beta == 0.0 ? 0.0 : beta * *cp);
  }
}

// One 64 x 64 tile of C = C0 - op(A) op(B) per CTA.
__global__ void __launch_bounds__(256) gemm_sub_kernel(double* C, int ldc, const double* C0,
                                                       int ldc0, const double* A, int lda,
                                                       bool ta, const double* B, int ldb,
                                                       bool tb, int m, int n, int kk) {
  __shared__ double tile[kGemmTileDoubles];
  const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 64;
  const int mt = min(64, m - i0), nt = min(64, n - j0);
  const double* Ab = ta ? A + static_cast<long long>(lda) * i0 : A + i0;
  const double* Bb = tb ? B + j0 : B + static_cast<long long>(ldb) * j0;
  cta_gemm_tiled(C + i0 + static_cast<long long>(ldc) * j0, ldc,
                 C0 ? C0 + i0 + static_cast<long long>(ldc0) * j0 : nullptr, ldc0, Ab, lda, ta, Bb,
                 ldb, tb, mt, nt, kk, tile);
}

// Rows of B (nrows rows, row stride 1, column stride ldb) <- rows of B A^{-1},
// i.e. each row r: solve A^T y = B(r, :)^T, one warp per row.
__global__ void lu_solve_rows_kernel(const double* lu, int n, int ld, const int* ipiv, double* b,
                                     int nrows, int ldb) {
  const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (r >= nrows) return;
  warp_lu_solve_t(lu, n, ld, ipiv, b + r, ldb);
}

}  // namespace

cudaError_t launch_gemm_sub(double* C, int ldc, const double* C0, int ldc0, const double* A,
                            int lda, bool ta, const double* B, int ldb, bool tb, int m, int n,
                            int k, cudaStream_t s) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  count_launches(1);
  gemm_sub_kernel<<<dim3((m + 63) / 64, (n + 63) / 64), 256, 0, s>>>(C, ldc, C0, ldc0, A, lda, ta,
                                                                      B, ldb, tb, m, n, k);
  return cudaGetLastError();
}

cudaError_t dense_lu_solve_rows(const double* lu, int n, int ld, const int* ipiv, double* b,
                                int nrows, int ldb, cudaStream_t s) {
  if (n == 0 || nrows == 0) return cudaSuccess;
  count_launches(1);
  lu_solve_rows_kernel<<<(nrows + 3) / 4, 128, 0, s>>>(lu, n, ld, ipiv, b, nrows, ldb);
  return cudaGetLastError();
}

namespace {
constexpr size_t kPanelSmemMax = 200 * 1024;
constexpr size_t kSolveSmemMax = 200 * 1024;
}  // namespace

cudaError_t dense_lu(double* a, int n, int ld, int* ipiv, int* status, cudaStream_t s) {
  for (int j0 = 0; j0 < n; j0 += kNb) {
    const int w = min(kNb, n - j0);
    count_launches(n - j0 - w > 0 ? 4 : 2);
    const size_t psmem = sizeof(double) * static_cast<size_t>((n - j0) | 1) * w;
    if (psmem <= kPanelSmemMax) {
      const cudaError_t e = cudaFuncSetAttribute(
          panel_lu_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPanelSmemMax);
      if (e != cudaSuccess) return e;
      panel_lu_smem_kernel<<<1, 1024, psmem, s>>>(a, n, ld, j0, w, ipiv, status);
    } else {
      panel_lu_kernel<<<1, 1024, 0, s>>>(a, n, ld, j0, w, ipiv, status);
    }
    swap_kernel<<<(n + 127) / 128, 128, 0, s>>>(a, n, ld, j0, w, ipiv);
    const int right = n - j0 - w;
    if (right > 0) {
      trsm_row_kernel<<<(right + 127) / 128, 128, 0, s>>>(a, n, ld, j0, w);
      const int tiles = (right + 63) / 64;
      trailing_kernel<<<dim3(tiles, tiles), 256, 0, s>>>(a, n, ld, j0, w);
    }
  }
  return cudaGetLastError();
}

cudaError_t dense_lu_solve(const double* lu, int n, int ld, const int* ipiv, double* b,
                           int nrhs, int ldb, cudaStream_t s) {
  if (n == 0 || nrhs == 0) return cudaSuccess;
  count_launches(1);
  const size_t smem = sizeof(double) * static_cast<size_t>(n);
  if (n >= 64 && smem <= kSolveSmemMax) {
    const cudaError_t e = cudaFuncSetAttribute(
        lu_solve_cta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSolveSmemMax);
    if (e != cudaSuccess) return e;
    lu_solve_cta_kernel<<<nrhs, kSolveThreads, smem, s>>>(lu, n, ld, ipiv, b, ldb);
    return cudaGetLastError();
  }
  const int per = 4;
  lu_solve_kernel<<<(nrhs + per - 1) / per, 32 * per, 0, s>>>(lu, n, ld, ipiv, b, nrhs, ldb);
  return cudaGetLastError();
}

cudaError_t launch_gather(const double* x, int ldx, const int* idx, int n, int nrhs,
                          double* out, int ldo, cudaStream_t s) {
  const long long tot = static_cast<long long>(n) * nrhs;
  if (tot == 0) return cudaSuccess;
  count_launches(1);
  gather_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, s>>>(x, ldx, idx, n, nrhs, out, ldo);
  return cudaGetLastError();
}

cudaError_t launch_gather_rows(const double* x, int ldd, const int* idx, int n, int nrhs,
                               double* out, int ldo, cudaStream_t s) {
  const long long tot = static_cast<long long>(n) * nrhs;
  if (tot == 0) return cudaSuccess;
  count_launches(1);
  gather_rows_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, s>>>(x, ldd, idx, n, nrhs, out,
                                                                          ldo);
  return cudaGetLastError();
}

cudaError_t launch_scatter(double* x, int ldx, const int* idx, int n, int nrhs,
                           const double* in, int ldi, cudaStream_t s) {
  const long long tot = static_cast<long long>(n) * nrhs;
  if (tot == 0) return cudaSuccess;
  count_launches(1);
  scatter_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, s>>>(x, ldx, idx, n, nrhs, in, ldi);
  return cudaGetLastError();
}

cudaError_t small_gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double* a,
                       int lda, const double* b, int ldb, double beta, double* c, int ldc,
                       cudaStream_t s) {
  const long long tot = static_cast<long long>(m) * n;
  if (tot == 0) return cudaSuccess;
  count_launches(1);
  if (ta && !tb && k > 2048 && tot <= 65536) {
    gemm_tn_long_kernel<<<static_cast<int>(tot), 256, 0, s>>>(m, k, alpha, a, lda, b, ldb, beta,
                                                              c, ldc);
    return cudaGetLastError();
  }
  gemm_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, s>>>(ta, tb, m, n, k, alpha, a, lda,
                                                                  b, ldb, beta, c, ldc);
  return cudaGetLastError();
}

}  // namespace kib

namespace kib {

namespace {

// Border blocks of S (skel_factorization.cpp:291-307): columns ns.. get the
// swept U rows of the skeleton, rows ns.. the swept Psi columns, and the
// corner -I - Psi_r D^{-1} U_r.
__global__ void fill_border_kernel(double* S, int ld, int ns, int nb, const double* us,
                                   const double* ps, const double* corr) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int side = ns * nb;
  if (e < side) {
    const int i = e % ns, j = e / ns;
    S[i + static_cast<long long>(ld) * (ns + j)] = us[i + static_cast<long long>(ns) * j];
    S[ns + j + static_cast<long long>(ld) * i] = ps[i + static_cast<long long>(ns) * j];
  } else if (e < side + nb * nb) {
    const int q = e - side, i = q % nb, j = q / nb;
    S[ns + i + static_cast<long long>(ld) * (ns + j)] = (i == j ? -1.0 : 0.0) - corr[i + nb * j];
  }
}

}  // namespace

cudaError_t launch_fill_border(double* S, int ld, int ns, int nb, const double* us,
                               const double* ps, const double* corr, cudaStream_t s) {
  const int tot = ns * nb + nb * nb;
  if (tot == 0) return cudaSuccess;
  count_launches(1);
  fill_border_kernel<<<(tot + 255) / 256, 256, 0, s>>>(S, ld, ns, nb, us, ps, corr);
  return cudaGetLastError();
}

}  // namespace kib
