// CTA- and warp-level FP64 dense routines on column-major matrices, used
// inside the per-box kernels (decouple, sweeps, diagonal solves).  They
// restate the LAPACK/BLAS steps the reference calls through ki_Mat
// (ki_mat.cpp:310-317 dgemm, :427-493 dgetrf/dgetrs).
#ifndef KI_BLOCKLA_CUH_
#define KI_BLOCKLA_CUH_

#include <cuda_runtime.h>

namespace kib {

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// C (m x n) = C0 - op(A) op(B) over the CTA, with op(A) m x kk, op(B) kk x n.
// C may alias C0.  ta/tb select the transposes (A stored kk x m when ta).
__device__ inline void cta_gemm_sub(double* C, int ldc, const double* C0, int ldc0,
                                    const double* A, int lda, bool ta, const double* B,
                                    int ldb, bool tb, int m, int n, int kk) {
  for (int e = threadIdx.x; e < m * n; e += blockDim.x) {
    const int i = e % m, j = e / m;
    double s = 0.0;
    for (int l = 0; l < kk; l++) {
      const double a = ta ? A[l + static_cast<long long>(lda) * i]
                          : A[i + static_cast<long long>(lda) * l];
      const double b = tb ? B[j + static_cast<long long>(ldb) * l]
                          : B[l + static_cast<long long>(ldb) * j];
      s += a * b;
    }
    C[i + static_cast<long long>(ldc) * j] = C0[i + static_cast<long long>(ldc0) * j] - s;
  }
}

// One FP64 tensor-core step (DMMA, mma.sync m8n8k4 .f64): the warp's 8 x 8
// block C += A (8 x 4) B (4 x 8).  Fragments: lane l holds A(l / 4, l % 4),
// B(l % 4, l / 4) and C(l / 4, 2 (l % 4) + v), v = 0, 1.
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%4,%5};\n"
               : "=d"(c0), "=d"(c1)
               : "d"(a), "d"(b), "d"(c0), "d"(c1));
}

// Tiled CTA GEMM on the FP64 tensor cores: C (m x n) = C0 + alpha op(A)
// op(B) (alpha = -1 unless given), op(A) m x kk, op(B) kk x n, 64 x 64
// output tiles, the inner dimension staged 16 at a time in `tile` (2 * 16 *
// kTileLd doubles, zero-padded past the matrix edges; kTileLd = 68, 4 mod
// 16 doubles: a half-warp's fragment loads, rows 4 fk apart and columns fr
// apart, then land on 16 distinct banks).  The 8 warps of the
// (256-thread) CTA are laid out 2 x 4 over a tile: each warp owns a 32 x 16
// block, i.e. 4 x 2 DMMA blocks of 8 x 8 with their accumulators in
// registers, and takes 6 fragment loads from shared memory per 8 DMMAs
// (2048 FMAs), where a 4 x 4 register tile per thread needs a load per two
// FMAs, more than shared memory delivers at the FP64 rate.  C0 may be null
// (taken as zero) or alias C; C must not alias A or B.  Operands may live in
// shared or global memory.  Ends with a barrier.
constexpr int kTileLd = 68;
constexpr int kGemmTileDoubles = 2 * 16 * kTileLd;

__device__ inline void cta_gemm_tiled(double* C, int ldc, const double* C0, int ldc0,
                                      const double* A, int lda, bool ta, const double* B,
                                      int ldb, bool tb, int m, int n, int kk, double* tile,
                                      double alpha = -1.0) {
  double* sa = tile;                 // [16][kTileLd]: sa[l kTileLd + i] = op(A)(i0 + i, l0 + l)
  double* sb = tile + 16 * kTileLd;  // [16][kTileLd]: sb[l kTileLd + j] = op(B)(l0 + l, j0 + j)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;  // this warp's block in the tile
  const int fr = lane >> 2, fk = lane & 3;                 // fragment row / inner index
  for (int i0 = 0; i0 < m; i0 += 64) {
    for (int j0 = 0; j0 < n; j0 += 64) {
      double acc[4][2][2];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 2; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
      for (int l0 = 0; l0 < kk; l0 += 16) {
        for (int e = threadIdx.x; e < 16 * 64; e += 256) {
          // A: element (row i0 + q, inner l0 + l); B: (inner l0 + l, col j0 + q)
          int q, l;
          if (ta) {  // op(A)(i, l) = A[l + lda i]: inner index fastest in memory
            l = e & 15;
            q = e >> 4;
          } else {
            q = e & 63;
            l = e >> 6;
          }
          const int gi = i0 + q, gl = l0 + l;
          double va = 0.0;
          if (gi < m && gl < kk)
            va = ta ? A[gl + static_cast<long long>(lda) * gi] : A[gi + static_cast<long long>(lda) * gl];
          sa[l * kTileLd + q] = va;
          int qb, lb;
          if (tb) {  // op(B)(l, j) = B[j + ldb l]: output index fastest
            qb = e & 63;
            lb = e >> 6;
          } else {
            lb = e & 15;
            qb = e >> 4;
          }
          const int gj = j0 + qb, glb = l0 + lb;
          double vb = 0.0;
          if (gj < n && glb < kk)
            vb = tb ? B[gj + static_cast<long long>(ldb) * glb] : B[glb + static_cast<long long>(ldb) * gj];
          sb[lb * kTileLd + qb] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < 4; ks++) {
          const int lrow = (ks * 4 + fk) * kTileLd;
          double af[4], bf[2];
#pragma unroll
          for (int a = 0; a < 4; a++) af[a] = sa[lrow + wm + 8 * a + fr];
#pragma unroll
          for (int b = 0; b < 2; b++) bf[b] = sb[lrow + wn + 8 * b + fr];
#pragma unroll
          for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) dmma_8x8x4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
        }
        __syncthreads();
      }
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
          for (int v = 0; v < 2; v++) {
            const int gi = i0 + wm + 8 * a + fr, gj = j0 + wn + 8 * b + 2 * fk + v;
            if (gi < m && gj < n) {
              const double c0 = C0 ? C0[gi + static_cast<long long>(ldc0) * gj] : 0.0;
              C[gi + static_cast<long long>(ldc) * gj] = c0 + alpha * acc[a][b][v];
            }
          }
    }
  }
  __syncthreads();
}

// In-place LU with partial pivoting (dgetf2) of an n x n matrix over the
// CTA.  ipiv[j] = row exchanged with row j.  `red` needs 2 * 32 doubles.
// Returns nonzero if an exactly zero or infinite pivot was met, or a column
// held no comparable entry (NaN).
__device__ inline int cta_lu(double* a, int n, int ld, int* ipiv, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  int* redi = reinterpret_cast<int*>(red + 32);
  int info = 0;
  for (int j = 0; j < n; j++) {
    // first maximum of |a(j:n, j)|
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
      for (int w = 1; w < nw; w++)
        if (red[w] > v || (red[w] == v && redi[w] < p)) {
          v = red[w];
          p = redi[w];
        }
      // no comparable entry (a NaN column): keep the row, report failure
      redi[30] = p < j || p >= n;
      if (redi[30]) p = j;
      ipiv[j] = p;
      redi[31] = p;
    }
    __syncthreads();
    const int p = redi[31];
    if (redi[30]) info = 1;
    const double piv = a[p + static_cast<long long>(ld) * j];
    if (piv != 0.0) {
      if (p != j) {
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
          double* x = a + static_cast<long long>(ld) * c;
          const double t = x[j];
          x[j] = x[p];
          x[p] = t;
        }
        __syncthreads();
      }
      const double inv = 1.0 / piv;
      for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x)
        a[i + static_cast<long long>(ld) * j] *= inv;
      if (isinf(piv)) info = 1;
    } else {
      info = 1;
    }
    __syncthreads();
    // rank-one update of the trailing block: warps take columns, lanes rows
    for (int c = j + 1 + warp; c < n; c += nw) {
      double* ac = a + static_cast<long long>(ld) * c;
      const double ajc = ac[j];
      if (ajc != 0.0) {
        const double* aj = a + static_cast<long long>(ld) * j;
        for (int i = j + 1 + lane; i < n; i += 32) ac[i] -= aj[i] * ajc;
      }
    }
    __syncthreads();
  }
  return info;
}

// Warp argmax of non-negative doubles (first index on ties) with three
// integer reductions instead of shuffle rounds: a non-negative double's bit
// pattern orders like the value, so the maximum is found on its high word,
// then its low word, then the smallest index holding it.  A lane with no
// candidate passes key 0 and index INT_MAX.
__device__ __forceinline__ void warp_argmax_bits(unsigned long long key, int idx,
                                                 unsigned long long* kmax, int* imin) {
  const unsigned hi = static_cast<unsigned>(key >> 32), lo = static_cast<unsigned>(key);
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const bool top = hi == mhi && lo == mlo;
  *imin = static_cast<int>(__reduce_min_sync(0xffffffffu, top ? static_cast<unsigned>(idx)
                                                              : 0x7fffffffu));
  *kmax = (static_cast<unsigned long long>(mhi) << 32) | mlo;
}

// Gauss-Jordan inversion of the n x n matrix a (column-major, ld; n <=
// blockDim.x) in place, partial pivoting, one barrier per pivot step.  Row
// i is updated by S = blockDim.x / n threads (at most 8), thread (i, s)
// owning the columns of segment s.  Rows are never exchanged: step j
// eliminates column j with row p_j (the largest |a(i, j)| among the rows
// not yet pivots, the first on ties; a NaN counts as 0).  Before the step's
// barrier the owner of a(i, j) keeps it in colj (double-buffered by step
// parity) and each warp publishes its best candidate (key, row) in a slot;
// after it every thread reduces the slots to the same p_j and updates its
// segment with the arithmetic of the row-swapping form: a(i, c) -= a(i, j)
// (a(p, c) / piv) via the reciprocal, a(i, j) <- -a(i, j) / piv, while row
// p_j waits until the next step's barrier, when nobody reads it any more,
// to scale itself (a(p, c) / piv, a(p, j) <- 1 / piv).  On return the
// result B holds A^{-1}(j, q) = B(p_j, p^{-1}(q)); pivot_row[j] = p_j.
// Returns nonzero when a pivot was 0, infinite or NaN.  Slots: 2 x 32 keys
// and rows; colj: 2 n doubles.
__device__ inline int cta_gj_invert_inplace(double* a, int n, int ld, int* pivot_row,
                                            unsigned long long* slot_key, int* slot_row,
                                            double* colj) {
  if (n <= 0) return 0;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nw = blockDim.x >> 5;
  const int S = max(1, min(static_cast<int>(blockDim.x) / n, 8));
  const int i = t % n, sg = t / n;
  const bool live = sg < S;
  const int L = (n + S - 1) / S, cb = sg * L, ce = min(n, cb + L);
  double* ar = a + i;
  bool used = false, pending = false;
  int jprev = 0;
  double own_inv = 0.0;
  int info = 0;
  for (int j = 0; j < n; j++) {
    const int buf = j & 1;
    const bool owner = live && j >= cb && j < ce;
    double aij = 0.0;
    if (owner) {
      aij = ar[static_cast<long long>(ld) * j];
      if (pending) aij *= own_inv;  // (the row scales itself after the barrier)
      colj[buf * n + i] = aij;
    }
    const bool cand = owner && !used;
    double v = cand ? fabs(aij) : 0.0;
    if (v != v) v = 0.0;
    unsigned long long wk;
    int wi;
    warp_argmax_bits(cand ? static_cast<unsigned long long>(__double_as_longlong(v)) : 0ull,
                     cand ? i : 0x7fffffff, &wk, &wi);
    if (lane == 0) {
      slot_key[32 * buf + warp] = wk;
      slot_row[32 * buf + warp] = wi;
    }
    __syncthreads();
    unsigned long long gk;
    int p;
    warp_argmax_bits(lane < nw ? slot_key[32 * buf + lane] : 0ull,
                     lane < nw ? slot_row[32 * buf + lane] : 0x7fffffff, &gk, &p);
    if (pending) {  // the previous step's pivot row, scaled now
      for (int c = cb; c < ce; c++) {
        double* e = ar + static_cast<long long>(ld) * c;
        *e = c == jprev ? own_inv : *e * own_inv;
      }
      pending = false;
    }
    const double* ap = a + p;
    const double piv = ap[static_cast<long long>(ld) * j];
    if (!(fabs(piv) > 0.0) || isinf(piv)) info = 1;  // (0, NaN or infinite)
    const double inv = 1.0 / piv;
    if (t == 0) pivot_row[j] = p;
    if (i == p) {
      if (live) {
        used = true;
        pending = true;
        own_inv = inv;
        jprev = j;
      }
    } else if (live) {
      const double f = colj[buf * n + i];
#pragma unroll 4
      for (int c = cb; c < ce; c++) {
        double* e = ar + static_cast<long long>(ld) * c;
        *e = c == j ? -f * inv : *e - f * (ap[static_cast<long long>(ld) * c] * inv);
      }
    }
  }
  __syncthreads();  // (every read of the last pivot row done)
  if (pending) {
    for (int c = cb; c < ce; c++) {
      double* e = ar + static_cast<long long>(ld) * c;
      *e = c == jprev ? own_inv : *e * own_inv;
    }
  }
  __syncthreads();
  return info;
}


// b (length n, stride inc) <- A^{-1} b for the LU above, by one warp.
__device__ inline void warp_lu_solve(const double* lu, int n, int ld, const int* ipiv,
                                     double* b, int inc) {
  const int lane = threadIdx.x & 31;
  if (lane == 0)
    for (int i = 0; i < n; i++) {
      const int p = ipiv[i];
      // (a pivot out of range, left by an LU that stopped early, is skipped)
      if (p != i && static_cast<unsigned>(p) < static_cast<unsigned>(n)) {
        const double t = b[static_cast<long long>(inc) * i];
        b[static_cast<long long>(inc) * i] = b[static_cast<long long>(inc) * p];
        b[static_cast<long long>(inc) * p] = t;
      }
    }
  __syncwarp();
  for (int k = 0; k < n; k++) {  // unit lower, column sweep
    const double v = b[static_cast<long long>(inc) * k];
    if (v != 0.0)
      for (int i = k + 1 + lane; i < n; i += 32)
        b[static_cast<long long>(inc) * i] -= v * lu[i + static_cast<long long>(ld) * k];
    __syncwarp();
  }
  for (int k = n - 1; k >= 0; k--) {  // upper, column sweep
    const double bk = b[static_cast<long long>(inc) * k];
    __syncwarp();
    if (bk != 0.0) {
      const double v = bk / lu[k + static_cast<long long>(ld) * k];
      if (lane == 0) b[static_cast<long long>(inc) * k] = v;
      for (int i = lane; i < k; i += 32)
        b[static_cast<long long>(inc) * i] -= v * lu[i + static_cast<long long>(ld) * k];
    }
    __syncwarp();
  }
}

// b <- A^{-T} b for the LU above (dgetrs 'T'), by one warp.
__device__ inline void warp_lu_solve_t(const double* lu, int n, int ld, const int* ipiv,
                                       double* b, int inc) {
  const int lane = threadIdx.x & 31;
  for (int k = 0; k < n; k++) {  // U^T y = b: row k of U dotted with y(0:k)
    double s = 0.0;
    for (int i = lane; i < k; i += 32)
      s += lu[i + static_cast<long long>(ld) * k] * b[static_cast<long long>(inc) * i];
    s = warp_sum_d(s);
    if (lane == 0) {
      const long long o = static_cast<long long>(inc) * k;
      b[o] = (b[o] - s) / lu[k + static_cast<long long>(ld) * k];
    }
    __syncwarp();
  }
  for (int k = n - 1; k >= 0; k--) {  // L^T z = y (unit)
    double s = 0.0;
    for (int i = k + 1 + lane; i < n; i += 32)
      s += lu[i + static_cast<long long>(ld) * k] * b[static_cast<long long>(inc) * i];
    s = warp_sum_d(s);
    if (lane == 0) b[static_cast<long long>(inc) * k] -= s;
    __syncwarp();
  }
  if (lane == 0)
    for (int i = n - 1; i >= 0; i--) {
      const int p = ipiv[i];
      // (a pivot out of range, left by an LU that stopped early, is skipped)
      if (p != i && static_cast<unsigned>(p) < static_cast<unsigned>(n)) {
        const double t = b[static_cast<long long>(inc) * i];
        b[static_cast<long long>(inc) * i] = b[static_cast<long long>(inc) * p];
        b[static_cast<long long>(inc) * p] = t;
      }
    }
  __syncwarp();
}

// x <- A^{-1} x for the LU above, x in shared memory (n values), by the
// whole CTA (blockDim >= 32): row interchanges, then blocked forward (unit
// L) and backward (U) substitution in 32-row blocks; warp 0 solves each
// diagonal block from registers, then every thread updates its rows with
// the block's 32 values.  Ends with a barrier.
// x (length n, in shared memory) <- A^{-1} x for the LU above, by the whole
// CTA, in 32-row blocks.  ipiv: the row interchanges, applied first in
// order (nullptr: x is already permuted); piv_smem (optional, n ints of
// shared memory) stages ipiv so that the sequential interchanges wait on
// shared memory, not on a global load each.  Per block: the diagonal
// triangle by warp 0 in registers (loaded one block ahead, during the
// previous block's update), then the update of the remaining rows, a
// thread per row with the block's 32 entries requested at once.
__device__ inline void cta_lu_solve(const double* __restrict__ lu, int n, int ld,
                                    const int* __restrict__ ipiv, double* x,
                                    int* piv_smem = nullptr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (ipiv) {
    const int* pv = ipiv;
    if (piv_smem) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) piv_smem[i] = ipiv[i];
      __syncthreads();
      pv = piv_smem;
    }
    if (threadIdx.x == 0)
      for (int i = 0; i < n; i++) {
        const int p = pv[i];
        // (a pivot out of range, left by an LU that stopped early, is skipped)
        if (p != i && static_cast<unsigned>(p) < static_cast<unsigned>(n)) {
          const double t = x[i];
          x[i] = x[p];
          x[p] = t;
        }
      }
  }
  __syncthreads();
  auto lower_block = [&](int kb, double* Lr) {  // warp 0: rows kb.., strictly lower
    const int nbk = min(32, n - kb);
#pragma unroll
    for (int k = 0; k < 32; k++)
      Lr[k] = (lane < nbk && k < lane) ? lu[kb + lane + static_cast<long long>(ld) * (kb + k)]
                                       : 0.0;
  };
  double Dr[32];
  if (warp == 0) lower_block(0, Dr);
  for (int kb = 0; kb < n; kb += 32) {  // L y = P b
    const int nbk = min(32, n - kb);
    if (warp == 0) {
      double xv = lane < nbk ? x[kb + lane] : 0.0;
#pragma unroll
      for (int k = 0; k < 32; k++) {
        const double xk = __shfl_sync(0xffffffffu, xv, k);
        xv -= Dr[k] * xk;  // Dr[k] = 0 unless k < lane
      }
      if (lane < nbk) x[kb + lane] = xv;
    }
    __syncthreads();
    if (warp == 0 && kb + 32 < n) lower_block(kb + 32, Dr);
    for (int i = kb + nbk + threadIdx.x; i < n; i += blockDim.x) {
      double l[32];
#pragma unroll
      for (int k = 0; k < 32; k++)
        l[k] = k < nbk ? lu[i + static_cast<long long>(ld) * (kb + k)] : 0.0;
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 32; k++) s += l[k] * x[kb + (k < nbk ? k : 0)];
      x[i] -= s;
    }
    __syncthreads();
  }
  auto upper_block = [&](int kb, double* Ur, double* rd) {  // warp 0
    const int nbk = min(32, n - kb);
#pragma unroll
    for (int k = 0; k < 32; k++)
      Ur[k] = (lane < nbk && k < nbk && k > lane)
                  ? lu[kb + lane + static_cast<long long>(ld) * (kb + k)]
                  : 0.0;
    // the diagonal's reciprocal, formed off the substitution's chain
    *rd = lane < nbk ? 1.0 / lu[kb + lane + static_cast<long long>(ld) * (kb + lane)] : 0.0;
  };
  const int kb_last = ((n - 1) / 32) * 32;
  double rd = 0.0;
  if (warp == 0 && n > 0) upper_block(kb_last, Dr, &rd);
  for (int kb = kb_last; kb >= 0; kb -= 32) {  // U x = y
    const int nbk = min(32, n - kb);
    if (warp == 0) {
      double xv = lane < nbk ? x[kb + lane] : 0.0;
#pragma unroll
      for (int k = 31; k >= 0; k--) {
        if (k < nbk) {
          if (lane == k) xv *= rd;
          const double xk = __shfl_sync(0xffffffffu, xv, k);
          xv -= Dr[k] * xk;  // Dr[k] = 0 unless lane < k
        }
      }
      if (lane < nbk) x[kb + lane] = xv;
    }
    __syncthreads();
    if (warp == 0 && kb > 0) upper_block(kb - 32, Dr, &rd);
    for (int i = threadIdx.x; i < kb; i += blockDim.x) {
      double u[32];
#pragma unroll
      for (int k = 0; k < 32; k++)
        u[k] = k < nbk ? lu[i + static_cast<long long>(ld) * (kb + k)] : 0.0;
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 32; k++) s += u[k] * x[kb + (k < nbk ? k : 0)];
      x[i] -= s;
    }
    __syncthreads();
  }
}

}  // namespace kib

#endif  // KI_BLOCKLA_CUH_
