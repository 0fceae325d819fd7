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
      if (p < j || p >= n) {  // no comparable entry (NaN column)
        p = j;
        atomicExch(status, 1);
      }
      sp = p;
      ipiv[j] = p;
    }
    __syncthreads();
    const int p = sp;
    const double piv = a[p + static_cast<long long>(ld) * j];
    if (piv != 0.0 && !isinf(piv)) {
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

// Panel factorization with the panel in registers: 512 threads, thread t
// holding rows t + 512 r (r < R) of the W-column panel; the column loop is
// unrolled, so every register index is a constant.  Per column: the pivot
// search over the owned rows and a warp reduction, one barrier, a second
// reduction over the 16 warp maxima (every warp does it), the owners of the
// pivot row and of row jj publish them in shared memory, a second barrier,
// then every thread exchanges (if it owns one of the two rows), forms its
// multipliers and applies the rank-one update in registers.  Rows are
// exchanged whole, as LAPACK's getf2 does; the pivot is the largest
// magnitude, the first such row on ties.
constexpr int kRegThreads = 512;
template <int R, int W>
__global__ void __launch_bounds__(kRegThreads) panel_lu_reg_kernel(double* a, int n, int ld,
                                                                    int j0, int w, int* ipiv,
                                                                    int* status) {
  __shared__ double rowP[W], rowJ[W];
  __shared__ double red[kRegThreads / 32];
  __shared__ int redi[kRegThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rows = n - j0;
  double x[R][W];
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = threadIdx.x + kRegThreads * r;
#pragma unroll
    for (int c = 0; c < W; c++)
      x[r][c] = (i < rows && c < w) ? a[j0 + i + static_cast<long long>(ld) * (j0 + c)] : 0.0;
  }
#pragma unroll
  for (int jj = 0; jj < W; jj++) {
    if (jj >= w) break;
    double bv = -1.0;
    int bp = 0x7fffffff;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int i = threadIdx.x + kRegThreads * r;
      const double v = fabs(x[r][jj]);
      if (i >= jj && i < rows && v > bv) {
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
    double v = lane < kRegThreads / 32 ? red[lane] : -1.0;
    int p = lane < kRegThreads / 32 ? redi[lane] : 0x7fffffff;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, v, o);
      const int op = __shfl_xor_sync(0xffffffffu, p, o);
      if (ov > v || (ov == v && op < p)) {
        v = ov;
        p = op;
      }
    }
    // no comparable entry (NaN column): keep the row, flag the factorization
    const bool bad = p < jj || p >= rows;
    if (bad) p = jj;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int i = threadIdx.x + kRegThreads * r;
      if (i == p) {
#pragma unroll
        for (int c = 0; c < W; c++) rowP[c] = x[r][c];
      }
      if (i == jj) {
#pragma unroll
        for (int c = 0; c < W; c++) rowJ[c] = x[r][c];
      }
    }
    __syncthreads();
    const double piv = rowP[jj];
    if (threadIdx.x == 0) {
      ipiv[j0 + jj] = j0 + p;
      if (piv == 0.0 || bad || isinf(piv)) atomicExch(status, 1);
    }
    const double inv = piv != 0.0 ? 1.0 / piv : 0.0;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int i = threadIdx.x + kRegThreads * r;
      if (i == jj) {
#pragma unroll
        for (int c = 0; c < W; c++) x[r][c] = rowP[c];
      } else if (i == p) {
#pragma unroll
        for (int c = 0; c < W; c++) x[r][c] = rowJ[c];
      }
      if (i > jj && i < rows) {
        const double li = x[r][jj] * inv;
#pragma unroll
        for (int c = jj + 1; c < W; c++) x[r][c] -= li * rowP[c];
        x[r][jj] = li;
      }
    }
    // the next step overwrites rowP / rowJ / red only after its first
    // barrier, which every thread reaches after this step's reads
  }
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = threadIdx.x + kRegThreads * r;
#pragma unroll
    for (int c = 0; c < W; c++)
      if (i < rows && c < w) a[j0 + i + static_cast<long long>(ld) * (j0 + c)] = x[r][c];
  }
}

// Panel factorization for panels of up to kFastRows rows, staged in shared
// memory, 512 threads and two barriers per column: after the pivot search
// (every thread then reads the 16 warp maxima and agrees on the pivot), and
// after the update.  Warp c % 16 owns panel column c; for step jj each lane
// forms the multipliers l_i of its rows from the unswapped column jj
// (l_i = x_i / pivot with rows jj and p exchanged), and the owners apply
// the row exchange and the rank-one update to their columns > jj and the
// row exchange to the finished columns < jj.  Column jj itself is exchanged
// and scaled by its owner during step jj + 1, when nobody reads it any more.  Pivot choice as in LAPACK: the largest
// magnitude, the first such row on ties.
constexpr int kFastThreads = 512;
constexpr int kFastQ = 26;  // rows per lane
constexpr int kFastRows = 32 * kFastQ;
__global__ void __launch_bounds__(kFastThreads) panel_lu_fast_kernel(double* a, int n, int ld,
                                                                     int j0, int w, int* ipiv,
                                                                     int* status) {
  extern __shared__ double P[];
  __shared__ double red[kFastThreads / 32];
  __shared__ int redi[kFastThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int nw = kFastThreads / 32;
  const int rows = n - j0, ldp = rows | 1;
  for (int e = threadIdx.x; e < rows * w; e += kFastThreads) {
    const int i = e % rows, c = e / rows;
    P[i + ldp * c] = a[j0 + i + static_cast<long long>(ld) * (j0 + c)];
  }
  __syncthreads();
  int prev_p = 0;
  double prev_inv = 0.0;
  for (int jj = 0; jj < w; jj++) {
    double* col = P + ldp * jj;
    double bv = -1.0;
    int bp = 0x7fffffff;
    for (int i = jj + threadIdx.x; i < rows; i += kFastThreads) {
      const double v = fabs(col[i]);
      if (v > bv) {
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
    double v = red[0];
    int p = redi[0];
#pragma unroll
    for (int q = 1; q < nw; q++) {
      const double ov = red[q];
      const int op = redi[q];
      if (ov > v || (ov == v && op < p)) {
        v = ov;
        p = op;
      }
    }
    const bool bad = p < jj || p >= rows;  // no comparable entry (NaN column)
    if (bad) p = jj;
    const double piv = col[p];
    if (threadIdx.x == 0) {
      ipiv[j0 + jj] = j0 + p;
      if (piv == 0.0 || bad || isinf(piv)) atomicExch(status, 1);
    }
    const double inv = piv != 0.0 ? 1.0 / piv : 0.0;
    // finished columns < jj (nobody reads them in this step): the previous
    // column's own exchange and scaling, then this step's row exchange
    for (int c = warp; c < jj; c += nw) {
      double* pc = P + ldp * c;
      if (c == jj - 1) {
        const double top = pc[jj - 1], other = pc[prev_p];
        __syncwarp();
        if (lane == 0 && prev_p != jj - 1) {
          pc[jj - 1] = other;
          pc[prev_p] = top;
        }
        __syncwarp();
        for (int i = jj + lane; i < rows; i += 32) pc[i] *= prev_inv;
        __syncwarp();
      }
      if (lane == 0 && p != jj) {
        const double t = pc[jj];
        pc[jj] = pc[p];
        pc[p] = t;
      }
      __syncwarp();
    }
    // multipliers of this lane's rows
    double l[kFastQ];
#pragma unroll
    for (int q = 0; q < kFastQ; q++) {
      const int i = lane + 32 * q;
      l[q] = 0.0;
      if (32 * q < rows && i > jj && i < rows) l[q] = (i == p ? col[jj] : col[i]) * inv;
    }
    for (int c = jj + 1; c < w; c++) {
      if (c % nw != warp) continue;
      double* pc = P + ldp * c;
      const double xj = pc[jj], xp = pc[p];
      __syncwarp();
      if (lane == 0) pc[jj] = xp;
      const double u = xp;
#pragma unroll
      for (int q = 0; q < kFastQ; q++) {
        if (32 * q >= rows) break;
        const int i = lane + 32 * q;
        if (i > jj && i < rows) {
          const double xi = i == p ? xj : pc[i];
          pc[i] = xi - l[q] * u;
        }
      }
      __syncwarp();
    }
    prev_p = p;
    prev_inv = inv;
    __syncthreads();
  }
  // the last column's exchange and scaling
  if (w > 0 && warp == (w - 1) % nw) {
    double* pc = P + ldp * (w - 1);
    const double top = pc[w - 1], other = pc[prev_p];
    __syncwarp();
    if (lane == 0 && prev_p != w - 1) {
      pc[w - 1] = other;
      pc[prev_p] = top;
    }
    __syncwarp();
    for (int i = w + lane; i < rows; i += 32) pc[i] *= prev_inv;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < rows * w; e += kFastThreads) {
    const int i = e % rows, c = e / rows;
    a[j0 + i + static_cast<long long>(ld) * (j0 + c)] = P[i + ldp * c];
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
        if (q < jj || q >= rows) {  // no comparable entry (NaN column)
          q = jj;
          atomicExch(status, 1);
        }
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
    if (piv == 0.0 || isinf(piv)) {
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
    if (p != j && p > j && p < n) {
      const double t = x[j];
      x[j] = x[p];
      x[p] = t;
    }
  }
}

// A12 <- L11^{-1} A12 (unit lower), one thread per column right of the
// panel, L11 staged in shared memory.
__global__ void trsm_row_kernel(double* a, int n, int ld, int j0, int w) {
  __shared__ double l11[kNb][kNb + 1];
  for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
    const int i = e % w, kk = e / w;
    l11[i][kk] = a[j0 + i + static_cast<long long>(ld) * (j0 + kk)];
  }
  __syncthreads();
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
      if (i < w) b[i] -= v * l11[i][kk];
  }
#pragma unroll
  for (int i = 0; i < kNb; i++)
    if (i < w) x[j0 + i] = b[i];
}

// The panel's row interchanges applied to every column outside the panel,
// fused with A12 <- L11^{-1} A12 for the columns right of it.  Each block
// first turns the interchange sequence into a list of (destination, source)
// rows (at most 2w entries; the rows below j0 are untouched), so a column's
// moved entries are all loaded before any is stored: independent loads
// instead of a chain of w dependent exchanges.  One thread per column;
// dynamic shared memory: n - j0 ints.
constexpr int kSwapThreads = 128;
__global__ void __launch_bounds__(kSwapThreads) swap_trsm_kernel(double* a, int n, int ld, int j0,
                                                                 int w, const int* ipiv) {
  extern __shared__ int perm[];
  __shared__ double l11[kNb][kNb + 1];
  __shared__ int dst[2 * kNb], src[2 * kNb], piv[kNb];
  __shared__ int cnt;
  const int rows = n - j0;
  for (int i = threadIdx.x; i < rows; i += kSwapThreads) perm[i] = i;
  for (int e = threadIdx.x; e < w * w; e += kSwapThreads) {
    const int i = e % w, kk = e / w;
    l11[i][kk] = a[j0 + i + static_cast<long long>(ld) * (j0 + kk)];
  }
  if (threadIdx.x < w) piv[threadIdx.x] = ipiv[j0 + threadIdx.x] - j0;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int jj = 0; jj < w; jj++) {
      const int p = piv[jj];
      if (p < jj || p >= rows) continue;
      const int t = perm[jj];
      perm[jj] = perm[p];
      perm[p] = t;
    }
  __syncthreads();
  for (int i = threadIdx.x; i < rows; i += kSwapThreads)
    if (perm[i] != i) {
      const int k = atomicAdd(&cnt, 1);
      dst[k] = i;
      src[k] = perm[i];
    }
  __syncthreads();
  const int m = cnt;
  const int q = blockIdx.x * kSwapThreads + threadIdx.x;
  if (q >= n - w) return;
  const int c = q < j0 ? q : q + w;
  double* x = a + static_cast<long long>(ld) * c + j0;
  // this thread's column alone: every moved entry loaded, then stored
  double v[2 * kNb];
#pragma unroll
  for (int k = 0; k < 2 * kNb; k++)
    if (k < m) v[k] = x[src[k]];
#pragma unroll
  for (int k = 0; k < 2 * kNb; k++)
    if (k < m) x[dst[k]] = v[k];
  if (c < j0) return;
  double b[kNb];
#pragma unroll
  for (int i = 0; i < kNb; i++) b[i] = i < w ? x[i] : 0.0;
#pragma unroll
  for (int kk = 0; kk < kNb; kk++) {
    if (kk >= w) break;
    const double bk = b[kk];
#pragma unroll
    for (int i = kk + 1; i < kNb; i++)
      if (i < w) b[i] -= bk * l11[i][kk];
  }
#pragma unroll
  for (int i = 0; i < kNb; i++)
    if (i < w) x[i] = b[i];
}

// A22 -= A21 A12 for the trailing block, 64 x 64 tiles, inner dimension w,
// on the FP64 tensor cores: 8 warps laid out 2 x 4, a warp's 32 x 16 block
// as 4 x 2 DMMA blocks (dmma_8x8x4 fragment layout).
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
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
  const int fr = lane >> 2, fk = lane & 3;
  double acc[4][2][2] = {};
#pragma unroll
  for (int ks = 0; ks < kNb / 4; ks++) {
    if (4 * ks >= w) break;
    double af[4], bf[2];
#pragma unroll
    for (int q = 0; q < 4; q++) af[q] = sa[4 * ks + fk][wm + 8 * q + fr];
#pragma unroll
    for (int t = 0; t < 2; t++) bf[t] = sb[4 * ks + fk][wn + 8 * t + fr];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int t = 0; t < 2; t++) dmma_8x8x4(acc[q][t][0], acc[q][t][1], af[q], bf[t]);
  }
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int t = 0; t < 2; t++)
#pragma unroll
      for (int v = 0; v < 2; v++) {
        const int gi = r0 + wm + 8 * q + fr, gc = c0 + wn + 8 * t + 2 * fk + v;
        if (gi < n && gc < n) a[gi + static_cast<long long>(ld) * gc] -= acc[q][t][v];
      }
}

// B <- A^{-1} B, one CTA per right-hand side, the vector in shared memory
// (then n ints staging the pivots).  perm (optional): the interchanges
// composed into one permutation (pivots_to_perm), applied as a gather.
constexpr int kSolveThreads = 512;
__global__ void __launch_bounds__(kSolveThreads)
    lu_solve_cta_kernel(const double* __restrict__ lu, int n, int ld, const int* __restrict__ ipiv,
                        const int* __restrict__ perm, double* b, int ldb) {
  extern __shared__ double x[];
  int* pv = reinterpret_cast<int*>(x + n);
  double* bc = b + static_cast<long long>(ldb) * blockIdx.x;
  // (the caller brings the LU into L2 beforehand: launch_l2_prefetch)
  if (perm) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = bc[perm[i]];
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = bc[i];
  }
  __syncthreads();
  cta_lu_solve(lu, n, ld, perm ? nullptr : ipiv, x, pv);
  for (int i = threadIdx.x; i < n; i += blockDim.x) bc[i] = x[i];
}

// The inverses of the 16 x 16 diagonal blocks of an LU's factors, a warp
// per block, lane j forming column j: L_kk^{-1} by forward substitution on
// e_j (unit diagonal), U_kk^{-1} by back substitution (the divisions by
// u_ii in full precision).  A last block of fewer rows is completed with
// the identity.  dinv: block k's L^{-1} then U^{-1}, each column-major,
// 2 * 256 doubles a block.
constexpr int kInvBlk = 16;
__global__ void lu_block_inv_kernel(const double* __restrict__ lu, int n, int ld,
                                    double* __restrict__ dinv) {
  const int blk = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int j = threadIdx.x & 31;
  if (blk >= (n + kInvBlk - 1) / kInvBlk || j >= kInvBlk) return;
  const int kb = blk * kInvBlk, nbk = min(kInvBlk, n - kb);
  auto A = [&](int i, int k) -> double {
    return i < nbk && k < nbk ? lu[kb + i + static_cast<long long>(ld) * (kb + k)]
                              : (i == k ? 1.0 : 0.0);
  };
  double* out = dinv + static_cast<long long>(blk) * 2 * kInvBlk * kInvBlk;
  double y[kInvBlk];
#pragma unroll
  for (int i = 0; i < kInvBlk; i++) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < i; k++) s += A(i, k) * y[k];
    y[i] = i < j ? 0.0 : (i == j ? 1.0 : -s);
  }
#pragma unroll
  for (int i = 0; i < kInvBlk; i++) out[j * kInvBlk + i] = y[i];
#pragma unroll
  for (int i = kInvBlk - 1; i >= 0; i--) {
    double s = i == j ? 1.0 : 0.0;
#pragma unroll
    for (int k = i + 1; k < kInvBlk; k++) s -= A(i, k) * y[k];
    y[i] = i > j ? 0.0 : s / A(i, i);
  }
#pragma unroll
  for (int i = 0; i < kInvBlk; i++) out[kInvBlk * kInvBlk + j * kInvBlk + i] = y[i];
}

// b <- A^{-1} b for the LU above, one CTA per right-hand side, a thread per
// row (n <= kInvSolveThreads), 16-row blocks: warp 0 applies the block's
// inverse L_kk^{-1} (forward) or U_kk^{-1} (backward) to the block's values,
// then every row still to be solved subtracts its 16 entries of the block
// column times them.  Each thread requests its row's entries of the next
// block column while the current block is applied, so the loads overlap the
// barrier and the block product.  The block inverses (lu_block_inv_kernel)
// are staged in shared memory at the start, behind them the vector.  perm:
// the interchanges composed into one permutation, applied as a gather.
constexpr int kInvSolveThreads = kLuBlockInvMaxN;
__global__ void __launch_bounds__(kInvSolveThreads, 1)
    lu_solve_inv_kernel(const double* __restrict__ lu, int n, int ld,
                        const double* __restrict__ dinv, const int* __restrict__ perm, double* b,
                        int ldb) {
  extern __shared__ __align__(16) double sm[];
  constexpr int NB = kInvBlk, BS = 2 * kInvBlk * kInvBlk;
  const int nblk = (n + NB - 1) / NB;
  double* di = sm;              // nblk x BS
  double* x = sm + nblk * BS;   // nblk x NB, zero past n
  double* bc = b + static_cast<long long>(ldb) * blockIdx.x;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int e = 2 * t; e < nblk * BS; e += 2 * kInvSolveThreads) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(di + e));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(dinv + e));
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int i = t; i < nblk * NB; i += kInvSolveThreads) x[i] = i < n ? bc[perm[i]] : 0.0;
  const bool mine = t < n;
  double l[NB];
  // rows below block 0: its column entries (L, unit lower)
#pragma unroll
  for (int k = 0; k < NB; k++)
    l[k] = mine && t >= NB && k < n ? lu[t + static_cast<long long>(ld) * k] : 0.0;
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  for (int kb = 0; kb < n; kb += NB) {  // L y = P b
    if (warp == 0) {
      const double* Li = di + (kb / NB) * BS;
      const int r = lane & (NB - 1);
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < NB; k++) acc += Li[k * NB + r] * x[kb + k];
      __syncwarp();
      if (lane < NB) x[kb + lane] = acc;
    }
    __syncthreads();
    if (mine && t >= kb + NB) {
      const double2* xv = reinterpret_cast<const double2*>(x + kb);
      double s = 0.0;
#pragma unroll
      for (int h = 0; h < NB / 2; h++) {
        const double2 u = xv[h];
        s += l[2 * h] * u.x;
        s += l[2 * h + 1] * u.y;
      }
      x[t] -= s;
    }
    const int kn = kb + NB;
    if (mine && t >= kn + NB) {
      const double* q = lu + t + static_cast<long long>(ld) * kn;
      if (kn + NB <= n) {
#pragma unroll
        for (int k = 0; k < NB; k++) l[k] = q[static_cast<long long>(ld) * k];
      } else {
#pragma unroll
        for (int k = 0; k < NB; k++) l[k] = kn + k < n ? q[static_cast<long long>(ld) * k] : 0.0;
      }
    }
    __syncthreads();
  }
  const int kb_last = (nblk - 1) * NB;
#pragma unroll
  for (int k = 0; k < NB; k++)
    l[k] = t < kb_last && kb_last + k < n ? lu[t + static_cast<long long>(ld) * (kb_last + k)]
                                          : 0.0;
  for (int kb = kb_last; kb >= 0; kb -= NB) {  // U x = y
    if (warp == 0) {
      const double* Ui = di + (kb / NB) * BS + NB * NB;
      const int r = lane & (NB - 1);
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < NB; k++) acc += Ui[k * NB + r] * x[kb + k];
      __syncwarp();
      if (lane < NB && kb + lane < n) x[kb + lane] = acc;
    }
    __syncthreads();
    if (t < kb) {
      const double2* xv = reinterpret_cast<const double2*>(x + kb);
      double s = 0.0;
#pragma unroll
      for (int h = 0; h < NB / 2; h++) {
        const double2 u = xv[h];
        s += l[2 * h] * u.x;
        s += l[2 * h + 1] * u.y;
      }
      x[t] -= s;
    }
    const int kp = kb - NB;
    if (kp >= 0 && t < kp) {
      const double* q = lu + t + static_cast<long long>(ld) * kp;
#pragma unroll
      for (int k = 0; k < NB; k++) l[k] = q[static_cast<long long>(ld) * k];
    }
    __syncthreads();
  }
  if (mine) bc[t] = x[t];
}

// Every 128-byte line of [p, p + bytes) into L2 with the evict-last
// priority, from the whole grid (the prefetches return at once; the lines
// arrive at HBM bandwidth while later kernels run).
__global__ void l2_prefetch_kernel(const char* p, long long lines) {
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < lines;
       e += static_cast<long long>(gridDim.x) * blockDim.x)
    asm volatile("prefetch.global.L2::evict_last [%0];" ::"l"(p + 128 * e));
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

// One 64 x 64 tile of C = C0 + alpha op(A) op(B) per CTA (FP64 tensor cores).
__global__ void __launch_bounds__(256) gemm_sub_kernel(double* C, int ldc, const double* C0,
                                                       int ldc0, const double* A, int lda,
                                                       bool ta, const double* B, int ldb,
                                                       bool tb, int m, int n, int kk,
                                                       double alpha) {
  __shared__ double tile[kGemmTileDoubles];
  const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 64;
  const int mt = min(64, m - i0), nt = min(64, n - j0);
  const double* Ab = ta ? A + static_cast<long long>(lda) * i0 : A + i0;
  const double* Bb = tb ? B + j0 : B + static_cast<long long>(ldb) * j0;
  cta_gemm_tiled(C + i0 + static_cast<long long>(ldc) * j0, ldc,
                 C0 ? C0 + i0 + static_cast<long long>(ldc0) * j0 : nullptr, ldc0, Ab, lda, ta, Bb,
                 ldb, tb, mt, nt, kk, tile, alpha);
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
                                                                      B, ldb, tb, m, n, k, -1.0);
  return cudaGetLastError();
}

cudaError_t launch_gemm_tiled(double* C, int ldc, const double* C0, int ldc0, const double* A,
                              int lda, bool ta, const double* B, int ldb, bool tb, int m, int n,
                              int k, double alpha, cudaStream_t s) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  count_launches(1);
  gemm_sub_kernel<<<dim3((m + 63) / 64, (n + 63) / 64), 256, 0, s>>>(C, ldc, C0, ldc0, A, lda, ta,
                                                                      B, ldb, tb, m, n, k, alpha);
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

// ---- single-launch LU for matrices of up to kLuFusedMaxN rows
//
// CTA b of the cooperative grid owns columns [32 b, 32 b + 32) in shared
// memory for the whole factorization.  For every panel k < b it waits for
// panel k's flag, then applies that step to its own columns exactly as the
// panel-by-panel path does (row interchanges, U12 = L11^{-1} A12 in the
// same order, A22 -= L21 U12 on the FP64 tensor cores: the same values up
// to the order of the sums over the panel's 32 columns); then it factors its own
// panel (the pivot search over its rows, one row interchange, the rank-one
// update: one barrier per column with the rows in registers up to 512 rows,
// two in shared memory beyond), publishes the block and its pivots and
// raises flag b.  The next panel's owner starts as soon as it has applied
// step b, while the others are still updating: the dependent chain is
// panel, one step's update on one CTA, panel, ...  Finished blocks apply
// the later steps' interchanges to their L rows and write them back at the
// end.  Every read of another CTA's data bypasses L1 (the lines may hold
// values from before the step).  Every wait is bounded: on a timeout (or
// another CTA's) the CTA sets *status = 2 and returns.
constexpr int kFusedThreads = 512;
constexpr unsigned long long kFusedWaitNs = 200ull * 1000 * 1000;

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Thread 0 waits (bounded) for flag k; false for every thread on an abort.
__device__ bool fused_wait(int* sync, int k, int G, int* status, int* s_ok) {
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned long long t0 = global_ns();
    while (ld_acquire_gpu(sync + k) == 0) {
      if (ld_acquire_gpu(sync + G) != 0 || global_ns() - t0 > kFusedWaitNs) {
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    if (!ok) {
      atomicExch(sync + G, 1);
      atomicExch(status, 2);
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// Row interchanges of one step on this CTA's columns (rows >= j0; one lane
// per column, in pivot order).
__device__ __forceinline__ void fused_swaps(double* blk, int np, int n, int j0, int wk, int wb,
                                            const int* pv) {
  if (threadIdx.x < wb) {
    const int c = threadIdx.x;
    for (int jj = 0; jj < wk; jj++) {
      const int p = pv[jj], r = j0 + jj;
      if (p > r && p < n) {
        const double t = blk[r + np * c];
        blk[r + np * c] = blk[p + np * c];
        blk[p + np * c] = t;
      }
    }
  }
}

// The slots through which a register panel's column step publishes, before
// its barrier, each warp's best candidate (key, row) and that row whole, and
// row `col` (the one the pivot row trades places with).  Double-buffered by
// column parity: column jj + 2 writes a slot only after the barrier of
// column jj + 1, which every panel thread reaches after its reads of column
// jj.
struct __align__(16) PanelSlots {
  double cand[2][kFusedThreads / 32][kNb];
  double crow[2][kNb];
  unsigned long long key[2][kFusedThreads / 32];
  int idx[2][kFusedThreads / 32];
};

// The 32-column panel is factored as two halves of 16 columns, as a
// recursive LU does: the left half in registers, its interchanges then
// applied to the right half, U12 = L11^{-1} A12 and A22 -= L21 U12 (FP64
// tensor cores) on the right half, the right half factored the same way,
// and its interchanges applied to the left half.  The pivots are those of
// the 32-column panel; the sums run in another order.
constexpr int kHalf = kNb / 2;

// The barrier of the panel threads (the first T of the block): the block's
// own when all take part, else named barrier 1 (the other warps wait at the
// block barrier that follows the half).
template <int T>
__device__ __forceinline__ void panel_sync() {
  if (T == kFusedThreads) {
    __syncthreads();
  } else {
    asm volatile("bar.sync 1, %0;" ::"n"(T) : "memory");
  }
}

// Factors block columns cb .. cb + wh - 1 (absolute c0 + cb + jj) over rows
// >= c0 + cb in registers, interchanges restricted to those columns; the
// pivots also go to hp[0 .. wh).  Called by threads t < T only, thread t
// holding rows t + T q (q < R; T R >= n).  Each column costs one barrier of
// the T threads: before it every warp publishes its best candidate and that
// row, and the owner of row col publishes row col; after it every thread
// agrees on the pivot p from the T / 32 warp maxima, reads the pivot row
// from the slot of the warp holding it, rows col and p trade values and the
// rows below apply the rank-one update.  Pivot rule: the largest |a(i, col)|
// over rows i >= col, the first such row on ties, a NaN no candidate.
// Arithmetic: l = x * (1 / piv), x_c -= l * prow_c.  Fewer panel threads than
// the block's 512 (256 with two or three rows each) shorten the column step:
// half the warps to reduce and to synchronise, the same rank-one work.
// Not inlined: the two calls share its code, and inside the fused kernel
// (128 registers a thread) an inlined copy spills in the column loop.
template <int T, int R>
__device__ __noinline__ void fused_half_rt(double* blk, int np, int n, int c0, int cb, int wh,
                                              int* ipiv, int* status, PanelSlots& S, int* hp) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  double x[R][kHalf];
#pragma unroll
  for (int q = 0; q < R; q++)
#pragma unroll
    for (int c = 0; c < kHalf; c++) {
      const int row = t + T * q;
      x[q][c] = row < n && c < wh ? blk[row + np * (cb + c)] : 0.0;
    }
#pragma unroll
  for (int jj = 0; jj < kHalf; jj++) {
    if (jj >= wh) break;
    const int col = c0 + cb + jj, buf = jj & 1;
    unsigned long long key = 0;
    int idx = 0x7fffffff;
#pragma unroll
    for (int q = 0; q < R; q++) {
      const int row = t + T * q;
      const double v = fabs(x[q][jj]);
      const unsigned long long k = static_cast<unsigned long long>(__double_as_longlong(v));
      if (row >= col && row < n && v == v && (idx == 0x7fffffff || k > key)) {
        key = k;
        idx = row;
      }
    }
    unsigned long long wkey;
    int widx;
    warp_argmax_bits(key, idx, &wkey, &widx);
    if (lane == 0) {
      S.key[buf][warp] = wkey;
      S.idx[buf][warp] = widx;
    }
    // (rows moved as pairs of doubles: half the shared-memory instructions)
#pragma unroll
    for (int q = 0; q < R; q++) {
      const int row = t + T * q;
      if (row == widx) {
        double2* d = reinterpret_cast<double2*>(S.cand[buf][warp]);
#pragma unroll
        for (int h = 0; h < kHalf / 2; h++) d[h] = make_double2(x[q][2 * h], x[q][2 * h + 1]);
      }
      if (row == col) {
        double2* d = reinterpret_cast<double2*>(S.crow[buf]);
#pragma unroll
        for (int h = 0; h < kHalf / 2; h++) d[h] = make_double2(x[q][2 * h], x[q][2 * h + 1]);
      }
    }
    panel_sync<T>();
    unsigned long long gkey;
    int p;
    warp_argmax_bits(lane < T / 32 ? S.key[buf][lane] : 0ull,
                     lane < T / 32 ? S.idx[buf][lane] : 0x7fffffff, &gkey, &p);
    // no comparable entry (NaN column): keep the row, flag the factorization
    const bool bad = p < col || p >= n;
    const double* prow = bad ? S.crow[buf] : S.cand[buf][(p % T) >> 5];
    if (bad) p = col;
    const double piv = prow[jj];
    if (t == 0) {
      ipiv[col] = p;
      hp[jj] = p;
      if (piv == 0.0 || bad || isinf(piv)) atomicExch(status, 1);
    }
    const double inv = piv != 0.0 ? 1.0 / piv : 0.0;
    const double2* prow2 = reinterpret_cast<const double2*>(prow);
    // interchange (rows col and p trade their values), then the update
#pragma unroll
    for (int q = 0; q < R; q++) {
      const int row = t + T * q;
      if (row == col || row == p) {
        const double2* src = row == col ? prow2 : reinterpret_cast<const double2*>(S.crow[buf]);
#pragma unroll
        for (int h = 0; h < kHalf / 2; h++) {
          const double2 u = src[h];
          x[q][2 * h] = u.x;
          x[q][2 * h + 1] = u.y;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < R; q++) {
      const int row = t + T * q;
      if (row > col && row < n) {
        const double li = x[q][jj] * inv;
#pragma unroll
        for (int h = (jj + 1) / 2; h < kHalf / 2; h++) {
          const double2 u = prow2[h];
          if (2 * h > jj) x[q][2 * h] -= li * u.x;
          x[q][2 * h + 1] -= li * u.y;
        }
        x[q][jj] = li;
      }
    }
  }
  const int rmin = c0 + cb;
#pragma unroll
  for (int q = 0; q < R; q++)
#pragma unroll
    for (int c = 0; c < kHalf; c++) {
      const int row = t + T * q;
      if (c < wh && row >= rmin && row < n) blk[row + np * (cb + c)] = x[q][c];
    }
}

// The row interchanges hp[0 .. cnt) of rows r0 + jj, on block columns
// [cfrom, cto): a thread per column, in pivot order.
__device__ __forceinline__ void half_swaps(double* blk, int np, int n, int r0, int cnt,
                                           const int* hp, int cfrom, int cto) {
  const int c = cfrom + static_cast<int>(threadIdx.x);
  if (c < cto) {
    for (int jj = 0; jj < cnt; jj++) {
      const int p = hp[jj], r = r0 + jj;
      if (p > r && p < n) {
        const double tmp = blk[r + np * c];
        blk[r + np * c] = blk[p + np * c];
        blk[p + np * c] = tmp;
      }
    }
  }
}

template <int T, int R>
__device__ __forceinline__ void fused_panel_split(double* blk, int np, int n, int c0, int wb,
                                                  int* ipiv, int* status, PanelSlots& S,
                                                  int* hp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wl = min(kHalf, wb), wr = wb - wl;
  if (threadIdx.x < T) fused_half_rt<T, R>(blk, np, n, c0, 0, wl, ipiv, status, S, hp);
  __syncthreads();
  if (wr <= 0) return;
  // the left half's interchanges on the right half
  half_swaps(blk, np, n, c0, wl, hp, kHalf, kHalf + wr);
  __syncthreads();
  // U12 = L11^{-1} A12: a warp per right-half column
  if (warp < wr) {
    const int c = kHalf + warp;
    double xv = lane < wl ? blk[c0 + lane + np * c] : 0.0;
#pragma unroll
    for (int kk = 0; kk < kHalf; kk++) {
      const double xk = __shfl_sync(0xffffffffu, xv, kk);
      if (kk < wl && lane > kk && lane < wl) xv -= xk * blk[c0 + lane + np * kk];
    }
    if (lane < wl) blk[c0 + lane + np * c] = xv;
  }
  __syncthreads();
  // A22 -= L21 U12 on the FP64 tensor cores: rows c0 + 16 .., 8-row tiles
  // over the warps, both 8-column tiles of the right half, k = 16
  {
    const int r0 = c0 + wl, nr = n - r0;
    const int fr = lane >> 2, fk = lane & 3;
    for (int tr = warp; 8 * tr < nr; tr += kFusedThreads / 32) {
      const int row = r0 + 8 * tr + fr;
      double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
      for (int ks = 0; ks < kHalf / 4; ks++) {
        const int kk = 4 * ks + fk;
        const double af = row < n && kk < wl ? blk[row + np * kk] : 0.0;
#pragma unroll
        for (int tc = 0; tc < 2; tc++) {
          const int cc = kHalf + 8 * tc + fr;
          const double bf = kk < wl && cc < kHalf + wr ? blk[c0 + kk + np * cc] : 0.0;
          dmma_8x8x4(acc[tc][0], acc[tc][1], af, bf);
        }
      }
      const int rowc = r0 + 8 * tr + fr;
      if (rowc < n) {
#pragma unroll
        for (int tc = 0; tc < 2; tc++)
#pragma unroll
          for (int v = 0; v < 2; v++) {
            const int cc = kHalf + 8 * tc + 2 * fk + v;
            if (cc < kHalf + wr) blk[rowc + np * cc] -= acc[tc][v];
          }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < T) fused_half_rt<T, R>(blk, np, n, c0, kHalf, wr, ipiv, status, S, hp + kHalf);
  __syncthreads();
  // the right half's interchanges on the left half
  half_swaps(blk, np, n, c0 + kHalf, wr, hp + kHalf, 0, wl);
}

// hold (a test hook, normally 0): thread block 0 keeps its flag down, so the
// other blocks' bounded waits run out and the launch ends with status 2.
// kPanel: the rows each of the 256 panel threads holds (2: n <= 512, 3: n
// <= 768; one instantiation per form keeps each one's registers to itself).
template <int kPanel>
__global__ void __launch_bounds__(kFusedThreads, 1)
    lu_fused_kernel(double* a, int n, int ld, int* ipiv, int* status, int* sync, int hold) {
  extern __shared__ double blk[];  // np x kNb, column-major
  __shared__ double l11[kNb][kNb + 1];
  __shared__ int pv[kNb];
  __shared__ int s_ok;
  __shared__ PanelSlots slots;
  __shared__ int half_piv[kNb];
  const int G = gridDim.x, b = blockIdx.x;
  const int np = n | 1;
  const int c0 = kNb * b, wb = min(kNb, n - c0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i0 = 0; i0 < n; i0 += kFusedThreads) {  // a row's 32 loads in flight at once
    const int i = i0 + tid;
    double v[kNb];
#pragma unroll
    for (int c = 0; c < kNb; c++)
      v[c] = i < n && c < wb ? a[i + static_cast<long long>(ld) * (c0 + c)] : 0.0;
#pragma unroll
    for (int c = 0; c < kNb; c++)
      if (i < n && c < wb) blk[i + np * c] = v[c];
  }
  __syncthreads();

  // the steps of the panels to the left
  for (int k = 0; k < b; k++) {
    if (!fused_wait(sync, k, G, status, &s_ok)) return;
    const int j0 = kNb * k, wk = min(kNb, n - j0);
    if (warp == 0) {
      // the step's interchanges on this block (a lane per column, pivots
      // by shuffle) while the other warps bring L11 in
      const int pr = lane < wk ? __ldcg(ipiv + j0 + lane) : 0;
      for (int jj = 0; jj < wk; jj++) {
        const int p = __shfl_sync(0xffffffffu, pr, jj), r = j0 + jj;
        if (lane < wb && p > r && p < n) {
          const double t = blk[r + np * lane];
          blk[r + np * lane] = blk[p + np * lane];
          blk[p + np * lane] = t;
        }
      }
    } else {
      for (int e = tid - 32; e < kNb * kNb; e += kFusedThreads - 32) {
        const int i = e & (kNb - 1), kk = e / kNb;
        if (i < wk && kk < wk)
          l11[i][kk] = __ldcg(a + j0 + i + static_cast<long long>(ld) * (j0 + kk));
      }
    }
    __syncthreads();
    // U12 = L11^{-1} A12, one warp per two columns (interleaved), in the kk
    // order of the panel-by-panel path
    static_assert(kNb == 2 * (kFusedThreads / 32), "two columns per warp");
    {
      const int ca = warp, cb = warp + kFusedThreads / 32;
      double xa = lane < wk && ca < wb ? blk[j0 + lane + np * ca] : 0.0;
      double xb = lane < wk && cb < wb ? blk[j0 + lane + np * cb] : 0.0;
#pragma unroll 8
      for (int kk = 0; kk < wk; kk++) {
        const double ya = __shfl_sync(0xffffffffu, xa, kk);
        const double yb = __shfl_sync(0xffffffffu, xb, kk);
        if (lane > kk && lane < wk) {
          const double l = l11[lane][kk];
          xa -= ya * l;
          xb -= yb * l;
        }
      }
      if (lane < wk && ca < wb) blk[j0 + lane + np * ca] = xa;
      if (lane < wk && cb < wb) blk[j0 + lane + np * cb] = xb;
    }
    __syncthreads();
    // A22 -= L21 U12 on the FP64 tensor cores (m8n8k4): warp w takes the
    // 8-row tiles w, w + 16, w + 32, w + 48 below the panel against the
    // block's 8-column tiles, L21 fragments from global memory (L2), U12
    // fragments from the block; the sum over kk first, then subtracted
    {
      const int r0 = j0 + wk, nr = n - r0;
      const int fr = lane >> 2, fk = lane & 3;
      constexpr int nw = kFusedThreads / 32;
      for (int t0 = warp; 8 * t0 < nr; t0 += 4 * nw) {
        // every L21 fragment of the warp's rows requested at once (one L2
        // round trip), then the block's columns in two halves of 16
        double af[kNb / 4][4];
#pragma unroll
        for (int ks = 0; ks < kNb / 4; ks++)
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int row = r0 + 8 * (t0 + nw * q) + fr, kk = 4 * ks + fk;
            af[ks][q] = row < n && kk < wk
                            ? __ldcg(a + row + static_cast<long long>(ld) * (j0 + kk))
                            : 0.0;
          }
#pragma unroll 1
        for (int h = 0; h < 2; h++) {
          double acc[4][2][2];
#pragma unroll
          for (int q = 0; q < 4; q++)
#pragma unroll
            for (int t = 0; t < 2; t++) acc[q][t][0] = acc[q][t][1] = 0.0;
#pragma unroll
          for (int ks = 0; ks < kNb / 4; ks++) {
            const int kk = 4 * ks + fk;
            double bf[2];
#pragma unroll
            for (int t = 0; t < 2; t++) {
              const int col = 16 * h + 8 * t + fr;
              bf[t] = kk < wk && col < wb ? blk[j0 + kk + np * col] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
              for (int t = 0; t < 2; t++)
                dmma_8x8x4(acc[q][t][0], acc[q][t][1], af[ks][q], bf[t]);
          }
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int row = r0 + 8 * (t0 + nw * q) + fr;
            if (row >= n) continue;
#pragma unroll
            for (int t = 0; t < 2; t++)
#pragma unroll
              for (int v = 0; v < 2; v++) {
                const int col = 16 * h + 8 * t + 2 * fk + v;
                if (col < wb) blk[row + np * col] -= acc[q][t][v];
              }
          }
        }
      }
    }
    __syncthreads();
  }

  // this CTA's panel, in registers
  fused_panel_split<256, kPanel>(blk, np, n, c0, wb, ipiv, status, slots, half_piv);
  __syncthreads();
  // the rows the later blocks read (this panel's L11, L21 and U11) before
  // the flag, the U12 rows above after it
  for (int i = c0 + tid; i < n; i += kFusedThreads)
#pragma unroll 4
    for (int c = 0; c < wb; c++) __stcg(a + i + static_cast<long long>(ld) * (c0 + c), blk[i + np * c]);
  __syncthreads();
  if (tid == 0 && !(hold && b == 0)) {
    __threadfence();
    st_release_gpu(sync + b, 1);
  }
  for (int i = tid; i < c0; i += kFusedThreads)
#pragma unroll 4
    for (int c = 0; c < wb; c++) __stcg(a + i + static_cast<long long>(ld) * (c0 + c), blk[i + np * c]);
  if (b + 1 == G) return;

  // the later steps' interchanges on this block's L rows, then those rows
  // written again (every CTA that reads this panel has done so before the
  // last flag is raised)
  for (int k = b + 1; k < G; k++) {
    if (!fused_wait(sync, k, G, status, &s_ok)) return;
    const int j0 = kNb * k, wk = min(kNb, n - j0);
    if (tid < wk) pv[tid] = __ldcg(ipiv + j0 + tid);
    __syncthreads();
    fused_swaps(blk, np, n, j0, wk, wb, pv);
    __syncthreads();
  }
  const int r1 = c0 + kNb;
  for (int i = r1 + tid; i < n; i += kFusedThreads)
#pragma unroll 4
    for (int c = 0; c < wb; c++) __stcg(a + i + static_cast<long long>(ld) * (c0 + c), blk[i + np * c]);
}
}  // namespace

namespace {
std::atomic<int> g_lu_inject{0};
}  // namespace

void inject_lu_fault(int mode) { g_lu_inject.store(mode); }

cudaError_t dense_lu(double* a, int n, int ld, int* ipiv, int* status, cudaStream_t s,
                     int* sync, bool top_level) {
  if (sync && n > 0 && n <= kLuFusedMaxN) {
    int G = (n + kNb - 1) / kNb;
    const size_t smem = sizeof(double) * static_cast<size_t>(n | 1) * kNb;
    static_assert(kLuFusedMaxN <= 3 * 256, "three rows per panel thread at most");
    const void* fn = n <= 512 ? reinterpret_cast<const void*>(&lu_fused_kernel<2>)
                              : reinterpret_cast<const void*>(&lu_fused_kernel<3>);
    cudaError_t e = raise_func_attr(fn,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(sync, 0, sizeof(int) * (G + 1), s)) != cudaSuccess) return e;
    // test hook (inject_lu_fault): the abort word raised before the start,
    // or block 0's flag held down; one top-level launch of more than one block
    int hold = 0;
    if (top_level && G > 1 && g_lu_inject.load() != 0) {
      const int mode = g_lu_inject.exchange(0);
      if (mode == 1 && (e = cudaMemsetAsync(sync + G, 0x7f, sizeof(int), s)) != cudaSuccess)
        return e;
      hold = mode == 2 ? 1 : 0;
    }
    void* args[] = {&a, &n, &ld, &ipiv, &status, &sync, &hold};
    count_launches(1);
    return cudaLaunchCooperativeKernel(fn, dim3(G), dim3(kFusedThreads), args, smem, s);
  }
  for (int j0 = 0; j0 < n;) {
    // register-resident panels: 32 columns while a thread holds one row,
    // 16 columns for two rows
    const int rows = n - j0;
    const int wmax = rows <= kRegThreads ? kNb : rows <= 2 * kRegThreads ? kNb / 2 : kNb;
    const int w = min(wmax, n - j0);
    count_launches(n - j0 - w > 0 ? 3 : 2);
    const size_t psmem = sizeof(double) * static_cast<size_t>((n - j0) | 1) * w;
    if (rows <= kRegThreads) {
      panel_lu_reg_kernel<1, kNb><<<1, kRegThreads, 0, s>>>(a, n, ld, j0, w, ipiv, status);
    } else if (rows <= 2 * kRegThreads) {
      panel_lu_reg_kernel<2, kNb / 2><<<1, kRegThreads, 0, s>>>(a, n, ld, j0, w, ipiv, status);
    } else if (psmem <= kPanelSmemMax && n - j0 <= kFastRows) {
      const cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&panel_lu_fast_kernel),
                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            kPanelSmemMax);
      if (e != cudaSuccess) return e;
      panel_lu_fast_kernel<<<1, kFastThreads, psmem, s>>>(a, n, ld, j0, w, ipiv, status);
    } else if (psmem <= kPanelSmemMax) {
      const cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&panel_lu_smem_kernel),
                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            kPanelSmemMax);
      if (e != cudaSuccess) return e;
      panel_lu_smem_kernel<<<1, 1024, psmem, s>>>(a, n, ld, j0, w, ipiv, status);
    } else {
      panel_lu_kernel<<<1, 1024, 0, s>>>(a, n, ld, j0, w, ipiv, status);
    }
    const int right = n - j0 - w;
    if (n - w > 0) {
      const size_t ssmem = sizeof(int) * static_cast<size_t>(n - j0);
      if (ssmem <= 48 * 1024) {
        swap_trsm_kernel<<<(n - w + kSwapThreads - 1) / kSwapThreads, kSwapThreads, ssmem, s>>>(
            a, n, ld, j0, w, ipiv);
      } else {
        swap_kernel<<<(n + 127) / 128, 128, 0, s>>>(a, n, ld, j0, w, ipiv);
        if (right > 0) trsm_row_kernel<<<(right + 127) / 128, 128, 0, s>>>(a, n, ld, j0, w);
      }
    }
    if (right > 0) {
      const int tiles = (right + 63) / 64;
      trailing_kernel<<<dim3(tiles, tiles), 256, 0, s>>>(a, n, ld, j0, w);
    }
    j0 += w;
  }
  return cudaGetLastError();
}

// The row interchanges of an LU composed into one permutation: (P b)[i] =
// b[perm[i]].  One thread walks the interchanges in order over shared
// memory (the pivots staged there first).
__global__ void pivots_to_perm_kernel(const int* __restrict__ ipiv, int n, int* perm) {
  extern __shared__ int sh[];
  int* pv = sh;
  int* idx = sh + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    pv[i] = ipiv[i];
    idx[i] = i;
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int i = 0; i < n; i++) {
      const int p = pv[i];
      if (p != i && static_cast<unsigned>(p) < static_cast<unsigned>(n)) {
        const int t = idx[i];
        idx[i] = idx[p];
        idx[p] = t;
      }
    }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = idx[i];
}

cudaError_t launch_pivots_to_perm(const int* ipiv, int n, int* perm, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const size_t smem = 2 * sizeof(int) * static_cast<size_t>(n);
  if (smem > 48 * 1024) {
    const cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&pivots_to_perm_kernel),
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem));
    if (e != cudaSuccess) return e;
  }
  count_launches(1);
  pivots_to_perm_kernel<<<1, 256, smem, s>>>(ipiv, n, perm);
  return cudaGetLastError();
}

cudaError_t launch_l2_prefetch(const void* p, size_t bytes, cudaStream_t s) {
  const long long lines = static_cast<long long>((bytes + 127) / 128);
  if (lines == 0) return cudaSuccess;
  const int blocks = static_cast<int>(std::min<long long>(592, (lines + 255) / 256));
  count_launches(1);
  l2_prefetch_kernel<<<blocks, 256, 0, s>>>(static_cast<const char*>(p), lines);
  return cudaGetLastError();
}

cudaError_t dense_lu_solve(const double* lu, int n, int ld, const int* ipiv, double* b,
                           int nrhs, int ldb, cudaStream_t s, const int* perm,
                           const double* dinv) {
  if (n == 0 || nrhs == 0) return cudaSuccess;
  count_launches(1);
  if (dinv && perm && n <= kInvSolveThreads) {
    const int nblk = (n + kInvBlk - 1) / kInvBlk;
    const size_t ism = sizeof(double) * static_cast<size_t>(nblk) * (2 * kInvBlk * kInvBlk + kInvBlk);
    const cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&lu_solve_inv_kernel),
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(ism));
    if (e != cudaSuccess) return e;
    lu_solve_inv_kernel<<<nrhs, kInvSolveThreads, ism, s>>>(lu, n, ld, dinv, perm, b, ldb);
    return cudaGetLastError();
  }
  const size_t smem = (sizeof(double) + sizeof(int)) * static_cast<size_t>(n);
  if (n >= 64 && smem <= kSolveSmemMax) {
    const cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&lu_solve_cta_kernel),
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kSolveSmemMax);
    if (e != cudaSuccess) return e;
    lu_solve_cta_kernel<<<nrhs, kSolveThreads, smem, s>>>(lu, n, ld, ipiv, perm, b, ldb);
    return cudaGetLastError();
  }
  const int per = 4;
  lu_solve_kernel<<<(nrhs + per - 1) / per, 32 * per, 0, s>>>(lu, n, ld, ipiv, b, nrhs, ldb);
  return cudaGetLastError();
}

cudaError_t launch_lu_block_inv(const double* lu, int n, int ld, double* dinv, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launches(1);
  const int nblk = (n + kInvBlk - 1) / kInvBlk;
  lu_block_inv_kernel<<<(nblk + 3) / 4, 128, 0, s>>>(lu, n, ld, dinv);
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

// Redundant-dof index of the bordered system (skel_factorization.cpp:
// 130-160 splits the dofs into the top level's skeletons and the rest):
// allred = the dofs outside the ascending, repeat-free skeleton list, in
// ascending order; red_pos[d] = d's position in allred, -1 for a skeleton.
// A dof's position is d minus the skeletons below it (binary search), so
// the lists are made where they are used instead of on the host.
__global__ void red_index_kernel(const int* __restrict__ skel_sorted, int ns, int n,
                                 int* __restrict__ allred, int* __restrict__ red_pos) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n) return;
  int lo = 0, hi = ns;  // the first skeleton >= d
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (skel_sorted[mid] < d) lo = mid + 1; else hi = mid;
  }
  if (lo < ns && skel_sorted[lo] == d) {
    red_pos[d] = -1;
    return;
  }
  red_pos[d] = d - lo;
  allred[d - lo] = d;
}

cudaError_t launch_red_index(const int* skel_sorted, int ns, int n, int* allred, int* red_pos,
                             cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launches(1);
  red_index_kernel<<<(n + 255) / 256, 256, 0, s>>>(skel_sorted, ns, n, allred, red_pos);
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

// The bordered system's row gathers in one pass (skel_factorization.cpp:
// 146-170): U, Psi^T and X_rr^{-1} U (dof-major, nb entries a dof) at the
// redundant dofs into Ured, Pred and dinv, U and Psi^T at the top-level
// skeletons into us, ps; all outputs column-major.
__global__ void border_gather_kernel(const double* __restrict__ modU,
                                     const double* __restrict__ modP,
                                     const double* __restrict__ modD, int nb,
                                     const int* __restrict__ allred, int nr,
                                     const int* __restrict__ allskel, int ns,
                                     double* __restrict__ Ured, double* __restrict__ Pred,
                                     double* __restrict__ dinv, double* __restrict__ us,
                                     double* __restrict__ ps) {
  // the row index runs fastest: the column-major writes coalesce, and a
  // dof's nb entries, read by nb neighbouring passes, come from cache
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= static_cast<long long>(nr + ns) * nb) return;
  const int c = static_cast<int>(e / (nr + ns)), i = static_cast<int>(e % (nr + ns));
  if (i < nr) {
    const long long src = static_cast<long long>(allred[i]) * nb + c;
    const long long dst = i + static_cast<long long>(nr) * c;
    Ured[dst] = modU[src];
    dinv[dst] = modD[src];
    Pred[dst] = modP[src];
  } else {
    const int j = i - nr;
    const long long src = static_cast<long long>(allskel[j]) * nb + c;
    const long long dst = j + static_cast<long long>(ns) * c;
    us[dst] = modU[src];
    ps[dst] = modP[src];
  }
}

cudaError_t launch_border_gather(const double* modU, const double* modP, const double* modD,
                                 int nb, const int* allred, int nr, const int* allskel, int ns,
                                 double* Ured, double* Pred, double* dinv, double* us,
                                 double* ps, cudaStream_t s) {
  const long long tot = static_cast<long long>(nr + ns) * nb;
  if (tot == 0) return cudaSuccess;
  count_launches(1);
  border_gather_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, s>>>(
      modU, modP, modD, nb, allred, nr, allskel, ns, Ured, Pred, dinv, us, ps);
  return cudaGetLastError();
}

// dst rows idx[0..n) <- src rows (dof-major, nb entries a dof)
__global__ void copy_rows_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                 int nb, const int* __restrict__ idx, int n) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= static_cast<long long>(n) * nb) return;
  const long long o = static_cast<long long>(idx[e / nb]) * nb + e % nb;
  dst[o] = src[o];
}

cudaError_t launch_copy_rows(const double* src, double* dst, int nb, const int* idx, int n,
                             cudaStream_t s) {
  const long long tot = static_cast<long long>(n) * nb;
  if (tot == 0) return cudaSuccess;
  count_launches(1);
  copy_rows_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, s>>>(src, dst, nb, idx, n);
  return cudaGetLastError();
}

// C = alpha A^T B + beta C for a long inner dimension k and a small C (m, n
// <= kLongTnMax): split over k, every CTA reading its rows of A and B once
// (64 at a time through shared memory) and summing all m n entries of its
// part; the parts are then added in split order (deterministic).  Replaces
// a CTA per entry of C, which read A and B m n times over through L2.
constexpr int kLongTnMax = 32;
constexpr int kLongTnRows = 64;

// A thread owns a 2 x 2 block of C (four independent FMA chains, four
// shared-memory loads per four FMAs); the tiles' columns past m and n are
// zero, so an odd m or n needs no test in the loop.
__global__ void __launch_bounds__(256) gemm_tn_split_kernel(int m, int n, int k, const double* a,
                                                            int lda, const double* b, int ldb,
                                                            int rows_per, double* part) {
  // tile loads staged in registers: a tile's loads are all in flight at
  // once, and the next tile's while this one is summed (one memory round
  // trip per CTA instead of one per load and tile)
  constexpr int kLoads = kLongTnRows * (kLongTnMax + 1) / 256 + 1;
  __shared__ double As[kLongTnRows][kLongTnMax + 2], Bs[kLongTnRows][kLongTnMax + 2];
  const int l0 = blockIdx.x * rows_per, l1 = min(k, l0 + rows_per);
  const int mb = (m + 1) / 2, nbk = (n + 1) / 2;
  const int ea = kLongTnRows * 2 * mb, eb = kLongTnRows * 2 * nbk;  // tile entries
  const bool owner = threadIdx.x < mb * nbk;
  const int i0 = 2 * (threadIdx.x % mb), j0 = 2 * (threadIdx.x / mb);
  double ra[kLoads], rb[kLoads];
  auto fetch = [&](int r0) {
    const int rn = min(kLongTnRows, l1 - r0);
#pragma unroll
    for (int q = 0; q < kLoads; q++) {
      const int e = threadIdx.x + 256 * q;
      const int r = e % kLongTnRows, c = e / kLongTnRows;
      ra[q] = e < ea && r < rn && c < m ? a[r0 + r + static_cast<long long>(lda) * c] : 0.0;
      rb[q] = e < eb && r < rn && c < n ? b[r0 + r + static_cast<long long>(ldb) * c] : 0.0;
    }
  };
  double c00 = 0.0, c01 = 0.0, c10 = 0.0, c11 = 0.0;
  if (l0 < l1) fetch(l0);
  for (int r0 = l0; r0 < l1; r0 += kLongTnRows) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kLoads; q++) {
      const int e = threadIdx.x + 256 * q;
      const int r = e % kLongTnRows, c = e / kLongTnRows;
      if (e < ea) As[r][c] = ra[q];
      if (e < eb) Bs[r][c] = rb[q];
    }
    __syncthreads();
    if (r0 + kLongTnRows < l1) fetch(r0 + kLongTnRows);
    if (owner) {
#pragma unroll 16
      for (int r = 0; r < kLongTnRows; r++) {
        const double a0 = As[r][i0], a1 = As[r][i0 + 1];
        const double b0 = Bs[r][j0], b1 = Bs[r][j0 + 1];
        c00 += a0 * b0;
        c01 += a0 * b1;
        c10 += a1 * b0;
        c11 += a1 * b1;
      }
    }
  }
  if (!owner) return;
  double* pp = part + static_cast<long long>(blockIdx.x) * m * n;
  if (i0 < m && j0 < n) pp[i0 + m * j0] = c00;
  if (i0 < m && j0 + 1 < n) pp[i0 + m * (j0 + 1)] = c01;
  if (i0 + 1 < m && j0 < n) pp[i0 + 1 + m * j0] = c10;
  if (i0 + 1 < m && j0 + 1 < n) pp[i0 + 1 + m * (j0 + 1)] = c11;
}

__global__ void gemm_tn_split_finish_kernel(int m, int n, int splits, const double* part,
                                            double alpha, double beta, double* c, int ldc) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  const int mn = m * n;
  if (o >= mn) return;
  double v = 0.0;
  for (int q = 0; q < splits; q++) v += part[static_cast<long long>(q) * mn + o];
  double* cp = c + (o % m) + static_cast<long long>(ldc) * (o / m);
  *cp = alpha * v + (beta == 0.0 ? 0.0 : beta * *cp);
}

int long_gemm_tn_splits(int m, int n, int k) {
  if (m < 1 || n < 1 || m > kLongTnMax || n > kLongTnMax || k < 1) return 0;
  return std::max(1, std::min(296, (k + 255) / 256));
}

cudaError_t long_gemm_tn(int m, int n, int k, double alpha, const double* a, int lda,
                         const double* b, int ldb, double beta, double* c, int ldc,
                         double* part, cudaStream_t s) {
  const int splits = long_gemm_tn_splits(m, n, k);
  if (splits < 1) return cudaErrorInvalidValue;
  const int rows_per = (k + splits - 1) / splits;
  const int used = (k + rows_per - 1) / rows_per;  // (every split gets rows)
  count_launches(2);
  gemm_tn_split_kernel<<<used, 256, 0, s>>>(m, n, k, a, lda, b, ldb, rows_per, part);
  gemm_tn_split_finish_kernel<<<(m * n + 255) / 256, 256, 0, s>>>(m, n, used, part, alpha, beta,
                                                                 c, ldc);
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
