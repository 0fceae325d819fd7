// Interpolative decomposition of every box of one quadtree level in one
// launch: fused ID-matrix generation, column-pivoted Householder QR with the
// reference's rank rule, and T = R11^{-1} R12.
//
// Reference semantics (paths relative to the reference repository):
//   * ID matrix rows: Kernel::get_id_mat, kernel.cpp:153-235 (proxy circle
//     of radius 1.5 side with 128 points; levels 1-2 use all other boxes).
//   * Pivoting and Householder steps: LAPACK dgeqp3/dlaqp2 as called by
//     ki_Mat::id (ki_mat.cpp:502-541): first-maximum column pivot on the
//     partial column norms, dlarfg reflector (beta = -sign(alpha) |x|), the
//     norm downdate with recomputation when it loses accuracy (tol3z).
//   * Rank: first i >= 1 with |R_ii| < tol |R_00|; none => 0 (no compression).
//   * T = R11^{-1} R12 by column back substitution (dtrtrs).
// The factorization stops at the rank: R_ii never changes after step i and
// T only needs R's first k rows, so steps k..n-1 of dgeqp3 are skipped.  The
// skeleton (pivots 0..k-1, in order) is unchanged by this; the redundant
// columns come out in their order at step k instead of dgeqp3's later pivot
// order, which only permutes the redundant set inside the box.
//
// B200 layout: one box is owned by a cluster of G CTAs (G = 1 for the many
// small boxes of deep levels, up to 8 for the few tall boxes near the root).
// Columns are dealt round-robin to the CTAs (physical column j belongs to
// CTA j % G), the matrix lives in HBM/L2 in column-major order, each warp
// streams whole columns, and one cluster barrier per pivot step publishes
// the updated columns and each CTA's best pivot candidate through
// distributed shared memory.  Every CTA recomputes the Householder vector of
// the pivot column itself, so no extra broadcast barrier is needed.
#include <cooperative_groups.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "ki_kernels.h"

namespace cg = cooperative_groups;

namespace kib {

namespace {

constexpr int kIdThreads = 256;
constexpr int kIdWarps = kIdThreads / 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// 32-bit integer hash (the "lowbias32" finalizer published by C. Wellons):
// the sketch takes its row choice from the low bits and its sign from the
// top bit.
__device__ __forceinline__ unsigned sketch_hash(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Block-wide sum; `red` holds kIdWarps doubles.  Ends with a barrier so
// `red` may be reused immediately.
__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = lane < kIdWarps ? red[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) red[0] = t;
  }
  __syncthreads();
  t = red[0];
  __syncthreads();
  return t;
}

struct Cand {
  double val;
  int pos;
  int pad;
};

// Lexicographic pivot order: larger norm first, then smaller position.
__device__ __forceinline__ bool better(double v, int p, double bv, int bp) {
  return v > bv || (v == bv && p < bp);
}

__device__ __forceinline__ void warp_best(double& v, int& p) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int op = __shfl_xor_sync(0xffffffffu, p, o);
    if (better(ov, op, v, p)) {
      v = ov;
      p = op;
    }
  }
}

// Stokes entries of one ID-matrix row for both dofs (components 0, 1) of a
// column node, with the arithmetic of the fast single-entry path
// (pair_entry<true> / proxy_entry_node<true>) and the pair's shared part (r,
// |r|^2, its reciprocal, r.n) formed once.  kind 0: row = target dof rdof
// of node rn, the column node the source; kind 1: the transposed block
// (the column node the target, rn/rdof the source); kind 2: proxy row pr.
__device__ __forceinline__ void stokes_entries2(int kind, const Node& rn, int rdof, const Node& cn,
                                                int cdof0, int pr, const double* dir, double cx,
                                                double cy, double rad, double pw, int ps,
                                                double* e0, double* e1) {
  if (kind == 2) {
    const int np = kNumProxy >> ps;
    const bool second = pr >= 2 * np;
    const int rr_ = second ? pr - 2 * np : pr;
    const int q = (rr_ >> 1) << ps, comp = rr_ & 1;
    const double tn0 = dir[q], tn1 = dir[kNumProxy + q];
    const double r0 = (cx + rad * tn0) - cn.x, r1 = (cy + rad * tn1) - cn.y;
    const double rr = r0 * r0 + r1 * r1;
    const double rc = comp ? r1 : r0, tnc = comp ? tn1 : tn0;
    if (!second) {
      const double pot = ((cn.w * KI_INV_PI) * (r0 * cn.nx + r1 * cn.ny)) * nr_rcp(rr * rr);
      *e0 = (pot * rc) * r0 + (cn.w * tnc) * cn.nx;
      *e1 = (pot * rc) * r1 + (cn.w * tnc) * cn.ny;
    } else {
      const double pot = ((-pw * KI_INV_PI) * (r0 * tn0 + r1 * tn1)) * nr_rcp(rr * rr);
      *e0 = (pot * rc) * r0 + (pw * cn.nx) * tnc;
      *e1 = (pot * rc) * r1 + (pw * cn.ny) * tnc;
    }
    return;
  }
  if (rn.x == cn.x && rn.y == cn.y) {  // a node with itself: the diagonal formula
    if (kind == 0) {
      *e0 = pair_entry<true>(kStokes, rn, rdof, cn, cdof0);
      *e1 = pair_entry<true>(kStokes, rn, rdof, cn, cdof0 + 1);
    } else {
      *e0 = pair_entry<true>(kStokes, cn, cdof0, rn, rdof);
      *e1 = pair_entry<true>(kStokes, cn, cdof0 + 1, rn, rdof);
    }
    return;
  }
  const Node& t = kind == 0 ? rn : cn;  // target node
  const Node& s = kind == 0 ? cn : rn;  // source node
  const double r0 = t.x - s.x, r1 = t.y - s.y;
  const double inv = nr_rcp(r0 * r0 + r1 * r1);
  const double pot = (s.w * KI_INV_PI) * (r0 * s.nx + r1 * s.ny) * (inv * inv);
  if (kind == 0) {  // the row's component fixed, the source component varies
    const int tc = rdof & 1;
    const double rt = tc ? r1 : r0, tn = tc ? t.ny : t.nx;
    *e0 = (pot * rt) * r0 + (s.w * tn) * s.nx;
    *e1 = (pot * rt) * r1 + (s.w * tn) * s.ny;
  } else {  // the row's (source) component fixed, the target component varies
    const int sc = rdof & 1;
    const double rs = sc ? r1 : r0, sn = sc ? s.ny : s.nx;
    *e0 = (pot * r0) * rs + (s.w * t.nx) * sn;
    *e1 = (pot * r1) * rs + (s.w * t.ny) * sn;
  }
}

__device__ __forceinline__ double lapy2(double x, double y) {
  const double xa = fabs(x), ya = fabs(y);
  const double w = fmax(xa, ya), z = fmin(xa, ya);
  if (z == 0.0) return w;
  const double q = z / w;
  return w * sqrt(1.0 + q * q);
}

// Column pass helpers: four independent loads in flight per lane.
__device__ __forceinline__ double col_dot(const double* __restrict__ col,
                                          const double* __restrict__ v, int r0, int m) {
  double w0 = 0.0, w1 = 0.0;
  int r = r0;
  for (; r + 96 < m; r += 128) {
    const double a0 = col[r], a1 = col[r + 32], a2 = col[r + 64], a3 = col[r + 96];
    w0 += v[r] * a0 + v[r + 64] * a2;
    w1 += v[r + 32] * a1 + v[r + 96] * a3;
  }
  for (; r < m; r += 32) w0 += v[r] * col[r];
  return w0 + w1;
}

__device__ __forceinline__ void col_axpy(double* __restrict__ col, const double* __restrict__ v,
                                         int r0, int m, double t) {
  int r = r0;
  for (; r + 96 < m; r += 128) {
    const double a0 = col[r], a1 = col[r + 32], a2 = col[r + 64], a3 = col[r + 96];
    col[r] = a0 + v[r] * t;
    col[r + 32] = a1 + v[r + 32] * t;
    col[r + 64] = a2 + v[r + 64] * t;
    col[r + 96] = a3 + v[r + 96] * t;
  }
  for (; r < m; r += 32) col[r] += v[r] * t;
}

__device__ __forceinline__ double col_sumsq(const double* __restrict__ col, int r0, int m) {
  double s0 = 0.0, s1 = 0.0;
  int r = r0;
  for (; r + 96 < m; r += 128) {
    const double a0 = col[r], a1 = col[r + 32], a2 = col[r + 64], a3 = col[r + 96];
    s0 += a0 * a0 + a2 * a2;
    s1 += a1 * a1 + a3 * a3;
  }
  for (; r < m; r += 32) s0 += col[r] * col[r];
  return s0 + s1;
}

// sum over r = r0, r0 + L, ... < r1 of a[r] b[r], four loads in flight.
__device__ __forceinline__ double strided_dot(const double* a, const double* b, int r0, int r1,
                                              int L) {
  double s0 = 0.0, s1 = 0.0;
  int r = r0;
  for (; r + 3 * L < r1; r += 4 * L) {
    const double x0 = a[r], x1 = a[r + L], x2 = a[r + 2 * L], x3 = a[r + 3 * L];
    const double y0 = b[r], y1 = b[r + L], y2 = b[r + 2 * L], y3 = b[r + 3 * L];
    s0 += x0 * y0 + x2 * y2;
    s1 += x1 * y1 + x3 * y3;
  }
  for (; r < r1; r += L) s0 += a[r] * b[r];
  return s0 + s1;
}

// col[r] += v[r] t over r = r0, r0 + L, ... < r1, loads ahead of stores.
__device__ __forceinline__ void strided_axpy(double* col, const double* v, int r0, int r1, int L,
                                             double t) {
  int r = r0;
  for (; r + 3 * L < r1; r += 4 * L) {
    const double x0 = col[r], x1 = col[r + L], x2 = col[r + 2 * L], x3 = col[r + 3 * L];
    const double y0 = v[r], y1 = v[r + L], y2 = v[r + 2 * L], y3 = v[r + 3 * L];
    col[r] = x0 + y0 * t;
    col[r + L] = x1 + y1 * t;
    col[r + 2 * L] = x2 + y2 * t;
    col[r + 3 * L] = x3 + y3 * t;
  }
  for (; r < r1; r += L) col[r] += v[r] * t;
}

// T column = R11^{-1} b by one warp (dtrsm column sweep), b = R(0:k, col)
// and the result held in registers (k <= 32 kTRegs); colq(q) is column q of
// R in pivot order.  Returns false when k is too large for the registers.
constexpr int kTRegs = 8;
constexpr int kTRegsOc = 4;  // the on-chip kernel's register T solve: ranks <= 128
template <class ColFn>
__device__ __forceinline__ bool warp_tsolve(const double* bcol, int k, const double* rdiag,
                                            ColFn colq, double* out) {
  if (k > 32 * kTRegs) return false;
  const int lane = threadIdx.x & 31;
  double b[kTRegs];
#pragma unroll
  for (int t = 0; t < kTRegs; t++) {
    const int l = lane + 32 * t;
    b[t] = l < k ? bcol[l] : 0.0;
  }
  for (int q = k - 1; q >= 0; q--) {
    const int tq = q >> 5;
    double bq = 0.0;
#pragma unroll
    for (int t = 0; t < kTRegs; t++)
      if (t == tq) bq = b[t];
    bq = __shfl_sync(0xffffffffu, bq, q & 31);
    if (bq != 0.0) {
      const double xq = bq / rdiag[q];
      const double* rq = colq(q);
#pragma unroll
      for (int t = 0; t < kTRegs; t++) {
        const int l = lane + 32 * t;
        if (l == q) b[t] = xq;
        else if (l < q) b[t] -= xq * rq[l];
      }
    }
  }
#pragma unroll
  for (int t = 0; t < kTRegs; t++) {
    const int l = lane + 32 * t;
    if (l < k) out[l] = b[t];
  }
  return true;
}

// Streaming variant: the matrix lives in HBM/L2 (boxes too large for a
// cluster's shared memory); G CTAs per box.
template <int G>
__global__ void __launch_bounds__(kIdThreads, 1) id_kernel(IdParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int task = blockIdx.x / G;
  int g = 0;
  if constexpr (G > 1) g = static_cast<int>(cg::this_cluster().block_rank());
  const IdTask tk = P.tasks[task];
  const int n = tk.n, m = tk.m, lda = tk.lda, I = tk.n_row;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  double* v = reinterpret_cast<double*>(smem_raw);     // m_cap: Householder vector
  double* rdiag = v + P.m_cap;                        // n_cap: R_ii
  double* vn1 = rdiag + P.n_cap;                      // n_cap: partial norms (physical)
  double* vn2 = vn1 + P.n_cap;                        // n_cap
  double* red = vn2 + P.n_cap;                        // 32
  Cand* wbest = reinterpret_cast<Cand*>(red + 32);    // kIdWarps
  Cand* slot = wbest + kIdWarps;                      // 2 (cluster exchange)
  int* pos2col = reinterpret_cast<int*>(slot + 2);    // n_cap
  int* own = pos2col + P.n_cap;                       // n_cap
  int* si = own + P.n_cap;                            // [0] own count, [1] pivot column

  double* A = P.work + tk.a_off;
  auto colp = [&](int j) -> double* { return A + static_cast<long long>(j) * lda; };
  const int* act = P.act + tk.act_off;
  const int* rowd = P.rowdofs + tk.row_off;
  const Node* nodes = P.nodes;
  const int pde = P.pde;
  const int mn = min(m, n);

  // Warp 0: choose the pivot for step i from the candidates (own CTA's warp
  // bests for G == 1, every CTA's slot otherwise), swap it into position i
  // and list this CTA's columns at positions > i.
  auto select_pivot = [&](int i, bool from_slots) {
    double bv = -1.0;
    int bp = 0x7fffffff;
    if (from_slots) {
      if (lane < G) {
        Cand c;
        if constexpr (G > 1) {
          c = cg::this_cluster().map_shared_rank(slot, lane)[i & 1];
        } else {
          c = slot[i & 1];
        }
        bv = c.val;
        bp = c.pos;
      }
    } else if (lane < kIdWarps) {
      bv = wbest[lane].val;
      bp = wbest[lane].pos;
    }
    warp_best(bv, bp);
    // no comparable candidate (every remaining norm NaN, from non-finite
    // entries): keep column i in place rather than index past the columns
    const int pvt = bp >= i && bp < n ? bp : i;
    const int ci = pos2col[i];
    const int cp = pos2col[pvt];
    __syncwarp();
    if (lane == 0) {
      pos2col[i] = cp;
      pos2col[pvt] = ci;
      si[1] = cp;
    }
    __syncwarp();
    int cnt = 0;
    for (int base = i + 1; base < n; base += 32) {
      const int p = base + lane;
      const bool mine = p < n && (pos2col[p] % G == g);
      const unsigned bal = __ballot_sync(0xffffffffu, mine);
      if (mine) own[cnt + __popc(bal & ((1u << lane) - 1u))] = p;
      cnt += __popc(bal);
    }
    if (lane == 0) si[0] = cnt;
  };

  // ---- generation of the owned columns + their initial norms
  for (int t = warp; g + G * t < n; t += kIdWarps) {
    const int j = g + G * t;
    const int cd = act[j];
    double* col = colp(j);
    double ss = 0.0;
    for (int r = lane; r < m; r += 32) {
      double val;
      if (r < I) {
        val = boundary_entry(pde, nodes, rowd[r], cd);
      } else if (r < 2 * I) {
        val = boundary_entry(pde, nodes, cd, rowd[r - I]);
      } else {
        val = proxy_entry(pde, nodes, P.proxy_dir, r - 2 * I, cd, tk.cx, tk.cy, tk.rad, tk.pw);
      }
      col[r] = val;
      ss += val * val;
    }
    ss = warp_sum(ss);
    if (lane == 0) {
      vn1[j] = sqrt(ss);
      vn2[j] = vn1[j];
    }
  }
  for (int p = threadIdx.x; p < n; p += kIdThreads) pos2col[p] = p;
  __syncthreads();
  {
    double bv = -1.0;
    int bp = 0x7fffffff;
    for (int t = warp; g + G * t < n; t += kIdWarps) {
      const int j = g + G * t;
      if (better(vn1[j], j, bv, bp)) {
        bv = vn1[j];
        bp = j;
      }
    }
    if (lane == 0) wbest[warp] = Cand{bv, bp, 0};
  }
  __syncthreads();
  if constexpr (G > 1) {
    if (warp == 0) {
      double bv = lane < kIdWarps ? wbest[lane].val : -1.0;
      int bp = lane < kIdWarps ? wbest[lane].pos : 0x7fffffff;
      warp_best(bv, bp);
      if (lane == 0) slot[0] = Cand{bv, bp, 0};
    }
    cg::this_cluster().sync();
  }
  if (warp == 0 && mn > 0) select_pivot(0, G > 1);
  __syncthreads();

  const double tol3z = sqrt(0.5 * 2.220446049250313e-16);
  int rank = 0;
  double thresh = 0.0;
  for (int i = 0; i < mn; i++) {
    const int c = si[1];
    const double* colc = colp(c);
    // ---- Householder reflector of the pivot column (redundantly per CTA);
    // the column's rows below the diagonal are staged in v as they are read.
    double part = 0.0;
    {
      int r = i + 1 + threadIdx.x;
      for (; r + 3 * kIdThreads < m; r += 4 * kIdThreads) {
        const double a0 = colc[r], a1 = colc[r + kIdThreads];
        const double a2 = colc[r + 2 * kIdThreads], a3 = colc[r + 3 * kIdThreads];
        v[r] = a0;
        v[r + kIdThreads] = a1;
        v[r + 2 * kIdThreads] = a2;
        v[r + 3 * kIdThreads] = a3;
        part += (a0 * a0 + a1 * a1) + (a2 * a2 + a3 * a3);
      }
      for (; r < m; r += kIdThreads) {
        const double a0 = colc[r];
        v[r] = a0;
        part += a0 * a0;
      }
    }
    part = warp_sum(part);
    if (lane == 0) red[warp] = part;
    __syncthreads();
    double xs = 0.0;
#pragma unroll
    for (int w = 0; w < kIdWarps; w++) xs += red[w];
    const double xnorm = sqrt(xs);
    const double alpha = colc[i];
    double beta = alpha, tau = 0.0, scal = 0.0;
    if (i < m - 1 && xnorm != 0.0) {
      beta = -copysign(lapy2(alpha, xnorm), alpha);
      tau = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    if (i == 0) thresh = fabs(P.tol * beta);
    if (i >= 1 && fabs(beta) < thresh) {
      rank = i;
      break;
    }
    if (threadIdx.x == 0) {
      rdiag[i] = beta;
      v[i] = 1.0;
    }
    for (int r = i + 1 + threadIdx.x; r < m; r += kIdThreads) v[r] *= scal;
    __syncthreads();
    // ---- apply H to the owned trailing columns, downdate their norms and
    // track this warp's best candidate for the next pivot
    const int nown = si[0];
    double bv = -1.0;
    int bp = 0x7fffffff;
    for (int t = warp; t < nown; t += kIdWarps) {
      const int p = own[t];
      const int j = pos2col[p];
      double* col = colp(j);
      if (tau != 0.0) {
        const double w = warp_sum(col_dot(col, v, i + lane, m));
        col_axpy(col, v, i + lane, m, -tau * w);
      }
      __syncwarp();
      const double aij = col[i];
      double nv1 = vn1[j];
      const double nv2 = vn2[j];
      bool recompute = false;
      if (nv1 != 0.0) {
        double temp = fabs(aij) / nv1;
        temp = fmax(1.0 - temp * temp, 0.0);
        const double q = nv1 / nv2;
        const double temp2 = temp * (q * q);
        if (temp2 <= tol3z) {
          recompute = true;
        } else {
          nv1 *= sqrt(temp);
        }
      }
      if (recompute) {
        const double ss = warp_sum(col_sumsq(col, i + 1 + lane, m));
        nv1 = (i < m - 1) ? sqrt(ss) : 0.0;
        if (lane == 0) vn2[j] = nv1;
      }
      if (lane == 0) vn1[j] = nv1;
      if (better(nv1, p, bv, bp)) {
        bv = nv1;
        bp = p;
      }
    }
    if (lane == 0) wbest[warp] = Cand{bv, bp, 0};
    __syncthreads();
    if (i + 1 < mn) {
      if constexpr (G > 1) {
        if (warp == 0) {
          double cv = lane < kIdWarps ? wbest[lane].val : -1.0;
          int cpos = lane < kIdWarps ? wbest[lane].pos : 0x7fffffff;
          warp_best(cv, cpos);
          if (lane == 0) slot[(i + 1) & 1] = Cand{cv, cpos, 0};
        }
        cg::this_cluster().sync();
      }
      if (warp == 0) select_pivot(i + 1, G > 1);
      __syncthreads();
    }
  }

  // No CTA may leave while a peer can still read its pivot slot.
  if constexpr (G > 1) cg::this_cluster().sync();

  // ---- outputs: rank, pivots, T = R11^{-1} R12 for the owned columns
  if (g == 0) {
    if (threadIdx.x == 0) P.rank[task] = rank;
    for (int p = threadIdx.x; p < n; p += kIdThreads) P.perm[tk.perm_off + p] = pos2col[p];
  }
  const int k = rank;
  double* T = P.tout + tk.t_off;
  for (int p = k + warp; k > 0 && p < n; p += kIdWarps) {
    const int j = pos2col[p];
    if (j % G != g) continue;
    const double* col = colp(j);
    double* tc = T + static_cast<long long>(p - k) * k;
    if (warp_tsolve(col, k, rdiag, [&](int q) { return colp(pos2col[q]); }, tc)) continue;
    for (int l = lane; l < k; l += 32) tc[l] = col[l];
    __syncwarp();
    for (int q = k - 1; q >= 0; q--) {
      const double bq = tc[q];
      __syncwarp();
      if (bq != 0.0) {
        const double xq = bq / rdiag[q];
        const double* rq = colp(pos2col[q]);
        if (lane == 0) tc[q] = xq;
        for (int l = lane; l < q; l += 32) tc[l] -= xq * rq[l];
      }
      __syncwarp();
    }
  }
}

constexpr int kOcThreads = 512;  // on-chip variant: 16 warps per CTA
constexpr int kOcWarps = kOcThreads / 32;

// On-chip variant: the whole ID matrix sits in the shared memory of a
// G-CTA cluster (CTA g holds the physical columns j with j % G == g) and a
// peer's pivot column is read through distributed shared memory.  In every
// pivot step the trailing columns are spread over all warps: each column is
// worked by a group of L lanes (L = 256 / columns, a power of two) that walk
// interleaved rows, so a group reads consecutive rows and every warp of the
// CTA has independent work to hide shared-memory and FP64 latency.

template <int G>
__global__ void __launch_bounds__(kOcThreads, 2) id_onchip_kernel(IdParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int task = blockIdx.x / G;
  int g = 0;
  if constexpr (G > 1) g = static_cast<int>(cg::this_cluster().block_rank());
  const IdTask tk = P.tasks[task];
  // sketched box: the working matrix is the sk x n sketch S A
  const bool sketch = tk.sk > 0;
  const int n = tk.n, m = sketch ? tk.sk : tk.m, lda = tk.lda, I = tk.n_row;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  // layout of this task (every CTA of the cluster has the same task)
  double* cols = reinterpret_cast<double*>(smem_raw);   // owned columns
  const int nloc = (n - g + G - 1) / G;  // columns j = g + G t owned by this CTA
  // (the layout must be the same in every CTA of the cluster, whose peers
  // read `slot` at the local offset: sized for the largest share)
  double* v = cols + static_cast<long long>((n + G - 1) / G) * lda;  // m
  double* rdiag = v + m;                                 // n
  double* vn1 = rdiag + n;                               // n
  double* vn2 = vn1 + n;                                 // n
  double* red = vn2 + n;                                 // 32
  Cand* wbest = reinterpret_cast<Cand*>(red + 32);       // kOcWarps
  Cand* slot = wbest + kOcWarps;                         // 2
  int* pos2col = reinterpret_cast<int*>(slot + 2);       // n
  int* own = pos2col + n;                                // n
  int* si = own + n;                                     // [0] own count, [1] pivot

  auto colp = [&](int j) -> double* {
    double* base = cols + static_cast<long long>(j / G) * lda;
    if constexpr (G > 1) {
      if (j % G != g) return cg::this_cluster().map_shared_rank(base, j % G);
    }
    return base;
  };
  const int* act = P.act + tk.act_off;
  const int* rowd = P.rowdofs + tk.row_off;
  const Node* nodes = P.nodes;
  const int pde = P.pde;
  const int mn = min(m, n);

  auto select_pivot = [&](int i, bool from_slots) {
    double bv = -1.0;
    int bp = 0x7fffffff;
    if (from_slots) {
      if (lane < G) {
        Cand c;
        if constexpr (G > 1) {
          c = cg::this_cluster().map_shared_rank(slot, lane)[i & 1];
        } else {
          c = slot[i & 1];
        }
        bv = c.val;
        bp = c.pos;
      }
    } else if (lane < kOcWarps) {
      bv = wbest[lane].val;
      bp = wbest[lane].pos;
    }
    warp_best(bv, bp);
    // no comparable candidate (every remaining norm NaN, from non-finite
    // entries): keep column i in place rather than index past the columns
    const int pvt = bp >= i && bp < n ? bp : i;
    const int ci = pos2col[i];
    const int cp = pos2col[pvt];
    __syncwarp();
    if (lane == 0) {
      pos2col[i] = cp;
      pos2col[pvt] = ci;
      si[1] = cp;
    }
    __syncwarp();
    if constexpr (G == 1) {
      // a single CTA owns every column: the positions > i, in order (the
      // trailing update takes p = i + 1 + q without the list)
      if (lane == 0) si[0] = n - i - 1;
      return;
    }
    int cnt = 0;
    for (int base = i + 1; base < n; base += 32) {
      const int p = base + lane;
      const bool mine = p < n && (pos2col[p] % G == g);
      const unsigned bal = __ballot_sync(0xffffffffu, mine);
      if (mine) own[cnt + __popc(bal & ((1u << lane) - 1u))] = p;
      cnt += __popc(bal);
    }
    if (lane == 0) si[0] = cnt;
  };

  // ---- generation of the owned columns + their initial norms (two rows per
  // lane per iteration for instruction-level parallelism)
  auto entry_at = [&](int r, int cd) -> double {
    if (r < I) return boundary_entry(pde, nodes, rowd[r], cd);
    if (r < 2 * I) return boundary_entry(pde, nodes, cd, rowd[r - I]);
    return proxy_entry(pde, nodes, P.proxy_dir, r - 2 * I, cd, tk.cx, tk.cy, tk.rad, tk.pw);
  };
  if (sketch) {
    // Y = S A for this CTA's columns.  Warp w owns columns t = w, w + 16, ...
    // and walks the rows of A 32 at a time, lane l generating row r0 + l in
    // registers and adding it, with its row's hashed sign, into row
    // (h(block) + l) mod sk of Y: a sparse sign embedding whose buckets are
    // runs of 32 from a hashed start, so the lanes of a block never hit the
    // same row (sk >= 32) and each adds its entry directly.  A column is only
    // touched by its warp, pass after pass in row order, so the result is
    // deterministic, and no barrier is needed.  Columns never mix, so the
    // CTAs of a cluster need no exchange here.
    const int mA = tk.m;
    const int sh = pde == kStokes ? 1 : 0;
    // this CTA's column node records and dofs, staged once
    Node* cn = reinterpret_cast<Node*>(
        (reinterpret_cast<uintptr_t>(si + 8) + 15) & ~uintptr_t{15});
    int* cdof = reinterpret_cast<int*>(cn + nloc);
    // work units: a column, or (Stokes, G = 1) the two dofs of one node in
    // consecutive columns, whose entries share r, |r|^2 and r.n
    int* unit = cdof + nloc;  // 2 t + (pair ? 1 : 0)
    for (int t = threadIdx.x; t < nloc; t += kOcThreads) {
      const int cd = act[g + G * t];
      cdof[t] = cd;
      cn[t] = nodes[cd >> sh];
    }
    for (long long e = threadIdx.x; e < static_cast<long long>(lda) * nloc; e += kOcThreads)
      cols[e] = 0.0;
    __syncthreads();
    const bool pairs = G == 1 && pde == kStokes;
    if (warp == 0) {
      int cnt = 0;
      for (int base = 0; base < nloc; base += 32) {
        const int t = base + lane;
        bool start = t < nloc, two = false;
        if (start && pairs) {
          const int cd = cdof[t];
          start = !((cd & 1) && t > 0 && cdof[t - 1] == cd - 1);
          two = !(cd & 1) && t + 1 < nloc && cdof[t + 1] == cd + 1;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, start);
        if (start) unit[cnt + __popc(bal & ((1u << lane) - 1u))] = 2 * t + (two ? 1 : 0);
        cnt += __popc(bal);
      }
      if (lane == 0) si[3] = cnt;
    }
    __syncthreads();
    const int nunits = si[3];
    if (warp < nunits) {
      for (int r0 = 0; r0 < mA; r0 += 32) {
        const int r = r0 + lane;
        const bool valid = r < mA;
        Node rnode = {};
        int rdof = 0;
        if (valid && r < 2 * I) {
          rdof = rowd[r < I ? r : r - I];
          rnode = nodes[rdof >> sh];
        }
        // the block of 32 rows lands on 32 consecutive rows of Y (mod sk)
        // from a hashed start, so the lanes of a block never collide; the
        // sign comes from the row's own hash
        int idx = static_cast<int>(sketch_hash(static_cast<unsigned>(r0 >> 5) ^ 0x9e3779b9u) %
                                   static_cast<unsigned>(m)) + lane;
        if (idx >= m) idx -= m;
        const bool neg = (sketch_hash(static_cast<unsigned>(r)) & 0x80000000u) != 0;
        for (int u = warp; u < nunits; u += kOcWarps) {
          const int t = unit[u] >> 1;
          if (unit[u] & 1) {
            if (valid) {
              double e0, e1;
              stokes_entries2(r < I ? 0 : r < 2 * I ? 1 : 2, rnode, rdof, cn[t], cdof[t],
                              r - 2 * I, P.proxy_dir, tk.cx, tk.cy, tk.rad, tk.pw, tk.pshift,
                              &e0, &e1);
              cols[static_cast<long long>(lda) * t + idx] += neg ? -e0 : e0;
              cols[static_cast<long long>(lda) * (t + 1) + idx] += neg ? -e1 : e1;
            }
            continue;
          }
          double val = 0.0;
          if (valid) {
            if (r < I) {
              val = pair_entry<true>(pde, rnode, rdof, cn[t], cdof[t]);
            } else if (r < 2 * I) {
              val = pair_entry<true>(pde, cn[t], cdof[t], rnode, rdof);
            } else {
              val = proxy_entry_node<true>(pde, cn[t], P.proxy_dir, r - 2 * I, cdof[t], tk.cx,
                                           tk.cy, tk.rad, tk.pw, tk.pshift);
            }
          }
          if (valid) cols[static_cast<long long>(lda) * t + idx] += neg ? -val : val;
        }
      }
    }
    __syncthreads();
    for (int t = warp; t < nloc; t += kOcWarps) {
      const double* col = cols + static_cast<long long>(lda) * t;
      double ss = 0.0;
      for (int r = lane; r < m; r += 32) ss += col[r] * col[r];
      ss = warp_sum(ss);
      if (lane == 0) {
        const int j = g + G * t;
        vn1[j] = sqrt(ss);
        vn2[j] = vn1[j];
      }
    }
  } else {
  for (int t = warp; g + G * t < n; t += kOcWarps) {
    const int j = g + G * t;
    const int cd = act[j];
    double* col = colp(j);
    double ss = 0.0;
    int r = lane;
    for (; r + 96 < m; r += 128) {
      const double a0 = entry_at(r, cd);
      const double a1 = entry_at(r + 32, cd);
      const double a2 = entry_at(r + 64, cd);
      const double a3 = entry_at(r + 96, cd);
      col[r] = a0;
      col[r + 32] = a1;
      col[r + 64] = a2;
      col[r + 96] = a3;
      ss += (a0 * a0 + a1 * a1) + (a2 * a2 + a3 * a3);
    }
    for (; r < m; r += 32) {
      const double a0 = entry_at(r, cd);
      col[r] = a0;
      ss += a0 * a0;
    }
    ss = warp_sum(ss);
    if (lane == 0) {
      vn1[j] = sqrt(ss);
      vn2[j] = vn1[j];
    }
  }
  }
  for (int p = threadIdx.x; p < n; p += kOcThreads) pos2col[p] = p;
  __syncthreads();
  {
    double bv = -1.0;
    int bp = 0x7fffffff;
    for (int t = warp; g + G * t < n; t += kOcWarps) {
      const int j = g + G * t;
      if (better(vn1[j], j, bv, bp)) {
        bv = vn1[j];
        bp = j;
      }
    }
    if (lane == 0) wbest[warp] = Cand{bv, bp, 0};
  }
  __syncthreads();
  if constexpr (G > 1) {
    if (warp == 0) {
      double bv = lane < kOcWarps ? wbest[lane].val : -1.0;
      int bp = lane < kOcWarps ? wbest[lane].pos : 0x7fffffff;
      warp_best(bv, bp);
      if (lane == 0) slot[0] = Cand{bv, bp, 0};
    }
    cg::this_cluster().sync();
  }
  if (warp == 0 && mn > 0) select_pivot(0, G > 1);
  __syncthreads();

  const double tol3z = sqrt(0.5 * 2.220446049250313e-16);
  int rank = 0;
  double thresh = 0.0;
  // Sketched boxes (rows sk = n + 16): warp 0 forms step i's Householder
  // vector right after choosing its pivot, so a step costs two CTA barriers
  // (after the trailing update, after warp 0) instead of four.
  double* hh = red + 16;  // [0] tau, [1] |tol R_00|; si[2]: the rank once found
  auto householder_w0 = [&](int i) {
    const double* colc = colp(si[1]);
    double part = 0.0;
    for (int r = i + 1 + lane; r < m; r += 32) {
      const double a0 = colc[r];
      v[r] = a0;
      part += a0 * a0;
    }
    const double xnorm = sqrt(warp_sum(part));
    const double alpha = colc[i];
    double beta = alpha, tau = 0.0, scal = 0.0;
    if (i < m - 1 && xnorm != 0.0) {
      // (sketched boxes only: reciprocals by Newton-refined estimates)
      beta = -copysign(lapy2(alpha, xnorm), alpha);
      tau = (beta - alpha) * nr_rcp(beta);
      scal = nr_rcp(alpha - beta);
    }
    for (int r = i + 1 + lane; r < m; r += 32) v[r] *= scal;
    if (lane == 0) {
      if (i == 0) hh[1] = fabs(P.tol * beta);
      if (i >= 1 && fabs(beta) < hh[1]) si[2] = i;
      rdiag[i] = beta;
      v[i] = 1.0;
      hh[0] = tau;
    }
  };
  if (sketch) {
    if (warp == 0) {
      if (lane == 0) si[2] = 0;
      __syncwarp();
      if (mn > 0) householder_w0(0);
    }
    __syncthreads();
  }
  for (int i = 0; i < mn; i++) {
    const int c = si[1];
    const double* colc = colp(c);
    double tau = 0.0;
    if (sketch) {
      if (si[2] != 0) {
        rank = si[2];
        break;
      }
      tau = hh[0];
    } else {
    double part = 0.0;
    for (int r = i + 1 + threadIdx.x; r < m; r += kOcThreads) {
      const double a0 = colc[r];
      v[r] = a0;
      part += a0 * a0;
    }
    part = warp_sum(part);
    if (lane == 0) red[warp] = part;
    __syncthreads();
    double xs = 0.0;
#pragma unroll
    for (int w = 0; w < kOcWarps; w++) xs += red[w];
    const double xnorm = sqrt(xs);
    const double alpha = colc[i];
    double beta = alpha, scal = 0.0;
    if (i < m - 1 && xnorm != 0.0) {
      beta = -copysign(lapy2(alpha, xnorm), alpha);
      tau = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    if (i == 0) thresh = fabs(P.tol * beta);
    if (i >= 1 && fabs(beta) < thresh) {
      rank = i;
      break;
    }
    if (threadIdx.x == 0) {
      rdiag[i] = beta;
      v[i] = 1.0;
    }
    for (int r = i + 1 + threadIdx.x; r < m; r += kOcThreads) v[r] *= scal;
    __syncthreads();
    }
    const int nown = si[0];
    // lanes per column for this step: spread the trailing columns over all
    // warps (L = 1 .. 32, a power of two); lane s of a group walks rows
    // i + s, i + s + L, ... so a group reads consecutive rows
    int L = 32;
    while (L > 1 && nown * L > kOcThreads) L >>= 1;
    const int gl = threadIdx.x & (L - 1);         // lane within the group
    const int gi = threadIdx.x / L;               // group index
    const int ngroups = kOcThreads / L;
    double bv = -1.0;
    int bp = 0x7fffffff;
    for (int q0 = 0; q0 < nown; q0 += ngroups) {
      const int q = q0 + gi;
      const bool active = q < nown;
      const int p = active ? (G == 1 ? i + 1 + q : own[q]) : 0;
      const int j = active ? pos2col[p] : g;
      double* col = colp(j);
      double w = 0.0;
      if (active && tau != 0.0) w = strided_dot(col, v, i + gl, m, L);
      for (int o = 1; o < L; o <<= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
      if (active && tau != 0.0) strided_axpy(col, v, i + gl, m, L, -tau * w);
      __syncwarp();
      // partial-norm downdate (dlaqp2), recomputed when it lost accuracy
      double nv1 = 0.0;
      bool recompute = false;
      if (active) {
        const double aij = col[i];
        nv1 = vn1[j];
        const double nv2 = vn2[j];
        if (nv1 != 0.0) {
          // sketched boxes need not follow dlaqp2's rounding: reciprocal
          // estimates instead of divisions on this per-step chain
          double temp = sketch ? fabs(aij) * nr_rcp(nv1) : fabs(aij) / nv1;
          temp = fmax(1.0 - temp * temp, 0.0);
          const double qq = sketch ? nv1 * nr_rcp(nv2) : nv1 / nv2;
          const double temp2 = temp * (qq * qq);
          if (temp2 <= tol3z) {
            recompute = true;
          } else {
            nv1 *= sqrt(temp);
          }
        }
      }
      if (__any_sync(0xffffffffu, recompute)) {
        double ss = 0.0;
        if (recompute) ss = strided_dot(col, col, i + 1 + gl, m, L);
        for (int o = 1; o < L; o <<= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
        if (recompute) {
          nv1 = (i < m - 1) ? sqrt(ss) : 0.0;
          if (gl == 0) vn2[j] = nv1;
        }
      }
      if (active) {
        if (gl == 0) vn1[j] = nv1;
        if (better(nv1, p, bv, bp)) {
          bv = nv1;
          bp = p;
        }
      }
      __syncwarp();
    }
    warp_best(bv, bp);
    if (lane == 0) wbest[warp] = Cand{bv, bp, 0};
    __syncthreads();
    if (i + 1 < mn) {
      if constexpr (G > 1) {
        if (warp == 0) {
          double cv = lane < kOcWarps ? wbest[lane].val : -1.0;
          int cpos = lane < kOcWarps ? wbest[lane].pos : 0x7fffffff;
          warp_best(cv, cpos);
          if (lane == 0) slot[(i + 1) & 1] = Cand{cv, cpos, 0};
        }
        cg::this_cluster().sync();
      }
      if (warp == 0) {
        select_pivot(i + 1, G > 1);
        if (sketch) {
          __syncwarp();
          householder_w0(i + 1);
        }
      }
      __syncthreads();
    }
  }
  if constexpr (G > 1) cg::this_cluster().sync();
  // a sketch shorter than n + 16 rows certifies a rank only well below its
  // row count; otherwise the box is reported (-1) for the full sketch
  if (sketch && m < n + 16 && (rank == 0 || rank > m - 16)) rank = -1;

  if (g == 0) {
    if (threadIdx.x == 0) P.rank[task] = rank;
    for (int p = threadIdx.x; p < n; p += kOcThreads) P.perm[tk.perm_off + p] = pos2col[p];
  }
  // T = R11^{-1} R12 for this CTA's redundant columns, solved in place in
  // their first k rows (dtrsm column sweep)
  const int k = rank;
  double* T = P.tout + tk.t_off;
  if (k > 0) {
    if (threadIdx.x < 32) {
      int cnt = 0;
      for (int base = k; base < n; base += 32) {
        const int p = base + lane;
        const bool mine = p < n && (pos2col[p] % G == g);
        const unsigned bal = __ballot_sync(0xffffffffu, mine);
        if (mine) own[cnt + __popc(bal & ((1u << lane) - 1u))] = p;
        cnt += __popc(bal);
      }
      if (lane == 0) si[0] = cnt;
    }
    // reciprocals of R's diagonal, off the substitutions' dependent chains
    // (vn2 is free once the factorization has stopped)
    for (int q = threadIdx.x; q < k; q += kOcThreads) vn2[q] = 1.0 / rdiag[q];
    __syncthreads();
    // one warp per redundant column: the column's back substitution runs
    // in its warp with no CTA barrier (columns are independent).  Up to
    // 32 kTRegsOc rows (a budget that leaves the 64-register launch bound
    // without local memory) the column lives in registers (lane l holding rows l,
    // l + 32, ...): per step one shuffle on the dependent chain, T written
    // once at the end
    const int nr = si[0];
    for (int t = warp; t < nr; t += kOcWarps) {
      const int p = own[t];
      double* col = colp(pos2col[p]);
      double* Tp = T + static_cast<long long>(p - k) * k;
      if (k <= 32 * kTRegsOc) {
        double b[kTRegsOc];
#pragma unroll
        for (int u = 0; u < kTRegsOc; u++) {
          const int l = lane + 32 * u;
          b[u] = l < k ? col[l] : 0.0;
        }
        // rows q in [32 u, 32 u + 32) sit in slot u: the slot loop outside
        // (unrolled), so every register index is a constant
#pragma unroll
        for (int u = kTRegsOc - 1; u >= 0; u--) {
          for (int q = min(k, 32 * u + 32) - 1; q >= 32 * u; q--) {
            const double* rq = colp(pos2col[q]);
            const double bq = __shfl_sync(0xffffffffu, b[u], q & 31);
            const double xq = bq * vn2[q];
#pragma unroll
            for (int v = 0; v <= u; v++) {
              const int l = lane + 32 * v;
              if (l == q) {
                b[v] = xq;
              } else if (l < q && bq != 0.0) {
                b[v] -= xq * rq[l];
              }
            }
          }
        }
#pragma unroll
        for (int u = 0; u < kTRegsOc; u++) {
          const int l = lane + 32 * u;
          if (l < k) Tp[l] = b[u];
        }
        continue;
      }
      for (int q = k - 1; q >= 0; q--) {
        const double bq = col[q];
        __syncwarp();
        const double xq = bq * vn2[q];
        if (lane == 0) Tp[q] = xq;
        if (bq != 0.0) {
          const double* rq = colp(pos2col[q]);
          for (int l = lane; l < q; l += 32) col[l] -= xq * rq[l];
        }
        __syncwarp();
      }
    }
    __syncthreads();
  }
  if constexpr (G > 1) cg::this_cluster().sync();
}

template <int G>
cudaError_t launch_onchip(const IdParams& p, cudaStream_t s) {
  const size_t smem = static_cast<size_t>(p.onchip_smem);
  if (smem == 0 || smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&id_onchip_kernel<G>),
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  if (G > 8) {
    e = raise_func_attr(reinterpret_cast<const void*>(&id_onchip_kernel<G>),
                        cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G * p.ntasks);
  cfg.blockDim = dim3(kOcThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  int na = 0;
  if (G > 1) {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = G;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    na = 1;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  return cudaLaunchKernelEx(&cfg, id_onchip_kernel<G>, p);
}

template <int G>
cudaError_t launch_g(const IdParams& p, cudaStream_t s) {
  const size_t smem = id_smem_bytes(p.m_cap, p.n_cap);
  cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&id_kernel<G>),
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G * p.ntasks);
  cfg.blockDim = dim3(kIdThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  int na = 0;
  if (G > 1) {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = G;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    na = 1;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  return cudaLaunchKernelEx(&cfg, id_kernel<G>, p);
}

}  // namespace

size_t id_sketch_smem_bytes(int sk, int n, int G) {
  const size_t nloc = static_cast<size_t>((n + G - 1) / G);
  // matrix share, staged node records and dofs of the columns (+ alignment)
  return id_smem_bytes(sk, n) + sizeof(double) * nloc * onchip_lda(sk) +
         (sizeof(Node) + 2 * sizeof(int)) * nloc + 16;
}

size_t id_onchip_smem_bytes(int m, int n, int G) {
  return id_smem_bytes(m, n) +
         sizeof(double) * static_cast<size_t>((n + G - 1) / G) * onchip_lda(m);
}

size_t id_smem_bytes(int m_cap, int n_cap) {
  return sizeof(double) * (static_cast<size_t>(m_cap) + 3 * n_cap + 32) +
         sizeof(Cand) * (kOcWarps + 2) + sizeof(int) * (2 * static_cast<size_t>(n_cap) + 8);
}

cudaError_t launch_id(const IdParams& p, int group, cudaStream_t s) {
  if (p.ntasks == 0) return cudaSuccess;
  count_launches(1);
  switch (group) {
    case 1: return launch_g<1>(p, s);
    case 2: return launch_g<2>(p, s);
    case 4: return launch_g<4>(p, s);
    case 8: return launch_g<8>(p, s);
    case kOnChip + 1: return launch_onchip<1>(p, s);
    case kOnChip + 2: return launch_onchip<2>(p, s);
    case kOnChip + 4: return launch_onchip<4>(p, s);
    case kOnChip + 8: return launch_onchip<8>(p, s);
    case kOnChip + 16: return launch_onchip<16>(p, s);
    default: return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------------------
// Interpolative decomposition without any device allocation.
//
// Some callers cannot call cudaMalloc: their device memory belongs to another
// allocator (a framework's caching allocator or a pool reserved up front)
// and a raw cudaMalloc/cudaFree would both bypass it and synchronise the
// whole device.  For them the ID of one box runs with its m x n working
// matrix in the file-scope array below, which every GPU that loads this
// library holds (8 MiB) until the process exits.  All calls share the
// array, the one-task descriptor and the proxy table, and each keeps the
// previous call's contents: the working matrix is fully regenerated before
// it is read, so nothing needs clearing, but calls that overlap on the GPU
// (different streams, or several host threads) race on it.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];
static __device__ __align__(256) IdTask g_noalloc_task[1];
static __device__ __align__(256) double g_noalloc_dir[2 * kNumProxy];

namespace {

__global__ void noalloc_set_task_kernel(IdTask tk) { g_noalloc_task[0] = tk; }

struct NoAllocSlot {
  bool ready = false;
  double* scratch = nullptr;
  IdTask* task = nullptr;
  double* dir = nullptr;
};
constexpr int kMaxDevices = 64;
NoAllocSlot g_noalloc_slot[kMaxDevices];
std::mutex g_noalloc_mu;

}  // namespace

// Resolves the device addresses of the static arrays for the current device
// (host code may not pass the array names to a kernel: they are host-side
// stand-ins) and fills the proxy table.  Runs once per device, on the first
// call made with that device current.
cudaError_t noalloc_setup(NoAllocSlot** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocSlot& sl = g_noalloc_slot[dev];
  if (!sl.ready) {
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&sl.scratch), g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&sl.task), g_noalloc_task);
    if (e != cudaSuccess) return e;
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&sl.dir), g_noalloc_dir);
    if (e != cudaSuccess) return e;
    double dir[2 * kNumProxy];
    for (int i = 0; i < kNumProxy; i++) {
      const double ang = 2 * M_PI * i * (1.0 / kNumProxy);
      dir[i] = std::cos(ang);
      dir[kNumProxy + i] = std::sin(ang);
    }
    e = cudaMemcpyToSymbol(g_noalloc_dir, dir, sizeof(dir));
    if (e != cudaSuccess) return e;
    sl.ready = true;
  }
  *out = &sl;
  return cudaSuccess;
}

cudaError_t launch_id_noalloc(int pde, const Node* nodes, const int* act, int n,
                              const int* rows, int n_rows, int proxy_rows, double cx,
                              double cy, double radius, double tol, int* rank, int* perm,
                              double* T, cudaStream_t s) {
  NoAllocSlot* sl = nullptr;
  cudaError_t e = noalloc_setup(&sl);
  if (e != cudaSuccess) return e;
  IdTask tk{};
  tk.n = n;
  tk.m = 2 * n_rows + proxy_rows;
  tk.n_row = n_rows;
  tk.proxy = proxy_rows;
  tk.lda = (tk.m + 3) & ~3;
  tk.cx = cx;
  tk.cy = cy;
  tk.rad = radius;
  tk.pw = 2.0 * M_PI * radius / kNumProxy;
  // the descriptor travels as a kernel argument (copied at launch, so the
  // host's copy may go out of scope at once) and is stored by one thread
  count_launches(1);
  noalloc_set_task_kernel<<<1, 1, 0, s>>>(tk);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  IdParams p{};
  p.tasks = sl->task;
  p.ntasks = 1;
  p.pde = pde;
  p.nodes = nodes;
  p.act = act;
  p.rowdofs = rows;
  p.work = sl->scratch;
  p.tout = T;
  p.perm = perm;
  p.rank = rank;
  p.proxy_dir = sl->dir;
  p.tol = tol;
  p.m_cap = tk.m;
  p.n_cap = n;
  return launch_id(p, 1, s);
}

int id_cluster_fits(int group, int m_cap, int n_cap, size_t col_cap) {
  if (group < kOnChip) return 1;
  const int G = group - kOnChip;
  const size_t smem = id_smem_bytes(m_cap, n_cap) + sizeof(double) * col_cap;
  if (smem > 227 * 1024) return 0;
  if (G == 1) return 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G);
  cfg.blockDim = dim3(kOcThreads);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = G;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  cudaError_t e;
  switch (G) {
    case 2: e = raise_func_attr(reinterpret_cast<const void*>(&id_onchip_kernel<2>), cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&clusters, id_onchip_kernel<2>, &cfg); break;
    case 4: e = raise_func_attr(reinterpret_cast<const void*>(&id_onchip_kernel<4>), cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&clusters, id_onchip_kernel<4>, &cfg); break;
    case 8: e = raise_func_attr(reinterpret_cast<const void*>(&id_onchip_kernel<8>), cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&clusters, id_onchip_kernel<8>, &cfg); break;
    case 16: e = raise_func_attr(reinterpret_cast<const void*>(&id_onchip_kernel<16>), cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e == cudaSuccess) e = raise_func_attr(reinterpret_cast<const void*>(&id_onchip_kernel<16>), cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&clusters, id_onchip_kernel<16>, &cfg); break;
    default: return 0;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return clusters > 0 ? 1 : 0;
}

}  // namespace kib
