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

template <int G>
__global__ void __launch_bounds__(kIdThreads) id_kernel(IdParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int task = blockIdx.x / G;
  int g = 0;
  if constexpr (G > 1) g = static_cast<int>(cg::this_cluster().block_rank());
  const IdTask tk = P.tasks[task];
  const int n = tk.n, m = tk.m, lda = tk.lda, I = tk.n_row;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  double* v = reinterpret_cast<double*>(smem_raw);   // m_cap: Householder vector
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
    const int pvt = bp;
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
    double* col = A + static_cast<long long>(j) * lda;
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
    const double* colc = A + static_cast<long long>(c) * lda;
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
      double* col = A + static_cast<long long>(j) * lda;
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
  if (rank == 0) return;
  const int k = rank;
  double* T = P.tout + tk.t_off;
  for (int p = k + warp; p < n; p += kIdWarps) {
    const int j = pos2col[p];
    if (j % G != g) continue;
    const double* col = A + static_cast<long long>(j) * lda;
    double* tc = T + static_cast<long long>(p - k) * k;
    for (int l = lane; l < k; l += 32) tc[l] = col[l];
    __syncwarp();
    for (int q = k - 1; q >= 0; q--) {
      const double bq = tc[q];
      __syncwarp();
      if (bq != 0.0) {
        const double xq = bq / rdiag[q];
        const double* rq = A + static_cast<long long>(pos2col[q]) * lda;
        if (lane == 0) tc[q] = xq;
        for (int l = lane; l < q; l += 32) tc[l] -= xq * rq[l];
      }
      __syncwarp();
    }
  }
}

template <int G>
cudaError_t launch_g(const IdParams& p, cudaStream_t s) {
  const size_t smem = id_smem_bytes(p.m_cap, p.n_cap);
  cudaError_t e = cudaFuncSetAttribute(id_kernel<G>,
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

size_t id_smem_bytes(int m_cap, int n_cap) {
  return sizeof(double) * (static_cast<size_t>(m_cap) + 3 * n_cap + 32) +
         sizeof(Cand) * (kIdWarps + 2) + sizeof(int) * (2 * static_cast<size_t>(n_cap) + 8);
}

cudaError_t launch_id(const IdParams& p, int group, cudaStream_t s) {
  if (p.ntasks == 0) return cudaSuccess;
  count_launches(1);
  switch (group) {
    case 1: return launch_g<1>(p, s);
    case 2: return launch_g<2>(p, s);
    case 4: return launch_g<4>(p, s);
    case 8: return launch_g<8>(p, s);
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
  e = cudaMemcpyToSymbolAsync(g_noalloc_task, &tk, sizeof(IdTask), 0, cudaMemcpyHostToDevice, s);
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

}  // namespace kib
