// The solution on a set of domain points, as boundary_integral_solve
// computes it (linear_solve.cpp:142-180): out = K_domain mu + U_forward alpha
// with the forward kernel (kernel.cpp:337-357) and the hole border columns
// (linear_solve.cpp:18-64), then zero wherever Boundary::is_in_domain says
// the point lies outside the domain.
//
// The reference forms K_domain as a dense |targets| x N matrix (16 GB for a
// 350^2 grid on 16,384 nodes) and multiplies it.  Here each thread owns one
// target and sweeps the source nodes staged in shared memory, forming the
// entries on the fly (FP64, reciprocal by a refined FP32 estimate, so the
// sums agree with the exact entries to FP64 rounding); the sources are split
// across CTAs when there are too few targets to fill the GPU, and a finish
// kernel adds the split sums in a fixed order, the border term and the mask.
//
// Domain tests (kept apart from the sums so they are exact):
//   * nodes: CubicBoundary::is_in_domain (cubic_boundary.cpp:182-230), the
//     test of every node-defined boundary: outside when within 1e-2 of any
//     node, when the crossing count of the outer curve is even, or when a
//     hole's crossing count is +1 modulo 2 (C remainder semantics: a count
//     of -1 does not exclude).  A crossing is counted for the edge from node
//     i to the next node of its curve when node i lies right of the point
//     and the edge's end heights straddle it.
//   * disk: Circle / Annulus / Donut::is_in_domain (circle.cpp:34-42,
//     annulus.cpp:66-79, donut.cpp:67-80): outside when |x - c| + 1e-2 > R or
//     |x - hole center| - 1e-2 < hole radius for any hole.
#include "ki_kernels.h"

namespace kib {

namespace {

constexpr int kDomThreads = 256;
constexpr double kDomainEps = 1e-2;  // cubic_boundary.cpp:185, circle.cpp:37

// Per-source values staged in shared memory, as in the operator product:
//   Laplace:          a = -(w / 2 pi) mu (n_x, n_y)
//   Laplace-Neumann:  a0 = (w / 2 pi) mu        (forward entry (w/2pi) log|r|)
//   Stokes:           a = (w / pi) (n_x, n_y), density (mu_0, mu_1)
template <int PDE>
__global__ void __launch_bounds__(kDomThreads)
    domain_partial_kernel(const Node* __restrict__ nodes, int np, int nt,
                          const double* __restrict__ tg, const double* __restrict__ mu,
                          int chunk, long long stride, double* __restrict__ part) {
  __shared__ double sx[kDomThreads], sy[kDomThreads], sa0[kDomThreads], sa1[kDomThreads];
  __shared__ double sd0[kDomThreads], sd1[kDomThreads];
  const int t = blockIdx.x * kDomThreads + threadIdx.x;
  const bool live = t < nt;
  const double tx = live ? tg[2 * t] : 0.0, ty = live ? tg[2 * t + 1] : 0.0;
  const int s0 = blockIdx.y * chunk;
  const int s1 = min(np, s0 + chunk);
  double y0 = 0.0, y1 = 0.0;
  for (int base = s0; base < s1; base += kDomThreads) {
    const int j = base + threadIdx.x;
    __syncthreads();
    if (j < s1) {
      const Node s = nodes[j];
      sx[threadIdx.x] = s.x;
      sy[threadIdx.x] = s.y;
      if (PDE == kLaplace) {
        const double c = -s.w * KI_INV_2PI * mu[j];
        sa0[threadIdx.x] = c * s.nx;
        sa1[threadIdx.x] = c * s.ny;
      } else if (PDE == kLaplaceNeumann) {
        sa0[threadIdx.x] = s.w * KI_INV_2PI * mu[j];
      } else {
        const double c = s.w * KI_INV_PI;
        sa0[threadIdx.x] = c * s.nx;
        sa1[threadIdx.x] = c * s.ny;
        sd0[threadIdx.x] = mu[2 * j];
        sd1[threadIdx.x] = mu[2 * j + 1];
      }
    } else {
      // padding: a far source of zero strength (|r|^2 stays inside the FP32
      // range of the reciprocal estimate; every numerator is zero)
      sx[threadIdx.x] = 1e15;
      sy[threadIdx.x] = 1e15;
      sa0[threadIdx.x] = 0.0;
      sa1[threadIdx.x] = 0.0;
      sd0[threadIdx.x] = 0.0;
      sd1[threadIdx.x] = 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < kDomThreads; q++) {
      const double r0 = tx - sx[q], r1 = ty - sy[q];
      const double rr = r0 * r0 + r1 * r1;
      if (PDE == kLaplaceNeumann) {
        y0 += sa0[q] * (0.5 * log(rr));
      } else {
        const double inv = rr > 0.0 ? nr_rcp(rr) : 0.0;
        if (PDE == kLaplace) {
          y0 += (r0 * sa0[q] + r1 * sa1[q]) * inv;
        } else {
          const double rn = r0 * sa0[q] + r1 * sa1[q];
          const double rx = r0 * sd0[q] + r1 * sd1[q];
          const double pq = (rn * rx) * (inv * inv);
          y0 += pq * r0;
          y1 += pq * r1;
        }
      }
    }
  }
  if (!live) return;
  if (PDE == kStokes) {
    part[stride * blockIdx.y + 2 * t] = y0;
    part[stride * blockIdx.y + 2 * t + 1] = y1;
  } else {
    part[stride * blockIdx.y + t] = y0;
  }
}

// CubicBoundary::is_in_domain, in two steps.
//
// curve_prep_kernel, one thread per node: the node's position, the height of
// the next node of its curve, and a code marking the last node of the outer
// curve (1) or of a hole (2), as structure-of-arrays; and per tile of 32
// consecutive nodes (one warp) the bounds a point must meet for the tile to
// matter: the nodes' box, the lowest and highest edge end, whether a curve
// ends in it.
//
// domain_mask_nodes_kernel, one warp per 32 targets, no block barriers: the
// warp walks the tiles in order; a tile that no target of the warp can be
// within 1e-2 of (box distance) and that no target lies strictly between
// the tile's edge ends and left of its rightmost node contributes nothing
// and is skipped, unless it ends a curve.  Other tiles are staged in the
// warp's shared-memory slice and every lane runs the reference's tests on
// the 32 nodes.  mask[t] = 1 inside, 0 outside.
struct CurveTile {
  double bx0, bx1, by0, by1, ey0, ey1;
  int code, pad;
};

__global__ void curve_prep_kernel(const Node* __restrict__ nodes, int np,
                                  const double* __restrict__ holes, int nh,
                                  double* __restrict__ cx, double* __restrict__ cy,
                                  double* __restrict__ cyn, int* __restrict__ ccode,
                                  CurveTile* __restrict__ tiles) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  int n_outer = np;
  for (int h = 0; h < nh; h++) n_outer -= static_cast<int>(holes[4 * h + 3]);
  double bx0 = NAN, bx1 = NAN, by0 = NAN, by1 = NAN, ey0 = NAN, ey1 = NAN;
  int code = 0;
  if (j < np) {
    int start = 0, end = n_outer;
    code = 1;
    if (j >= n_outer) {
      start = n_outer;
      code = 2;
      for (int h = 0; h < nh; h++) {
        end = start + static_cast<int>(holes[4 * h + 3]);
        if (j < end) break;
        start = end;
      }
    }
    const Node s = nodes[j];
    const double yn = nodes[j + 1 < end ? j + 1 : start].y;
    code = j == end - 1 ? code : 0;
    cx[j] = s.x;
    cy[j] = s.y;
    cyn[j] = yn;
    ccode[j] = code;
    bx0 = bx1 = s.x;
    by0 = by1 = s.y;
    ey0 = fmin(s.y, yn);
    ey1 = fmax(s.y, yn);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    bx0 = fmin(bx0, __shfl_xor_sync(0xffffffffu, bx0, o));
    bx1 = fmax(bx1, __shfl_xor_sync(0xffffffffu, bx1, o));
    by0 = fmin(by0, __shfl_xor_sync(0xffffffffu, by0, o));
    by1 = fmax(by1, __shfl_xor_sync(0xffffffffu, by1, o));
    ey0 = fmin(ey0, __shfl_xor_sync(0xffffffffu, ey0, o));
    ey1 = fmax(ey1, __shfl_xor_sync(0xffffffffu, ey1, o));
    code |= __shfl_xor_sync(0xffffffffu, code, o);
  }
  if (lane == 0 && j < np) tiles[j >> 5] = CurveTile{bx0, bx1, by0, by1, ey0, ey1, code, 0};
}

constexpr int kMaskWarps = 8;
__global__ void __launch_bounds__(32 * kMaskWarps)
    domain_mask_nodes_kernel(const double* __restrict__ cx, const double* __restrict__ cy,
                             const double* __restrict__ cyn, const int* __restrict__ ccode,
                             const CurveTile* __restrict__ tiles, int np, int nt,
                             const double* __restrict__ tg, unsigned char* __restrict__ mask) {
  __shared__ double sx[kMaskWarps][32], sy[kMaskWarps][32], syn[kMaskWarps][32];
  __shared__ int scode[kMaskWarps][32];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int t = (blockIdx.x * kMaskWarps + wl) * 32 + lane;
  const bool live = t < nt;
  const double tx = live ? tg[2 * t] : 0.0, ty = live ? tg[2 * t + 1] : 0.0;
  int wind = 0;
  bool out = false;
  const int ntiles = (np + 31) >> 5;
  for (int k = 0; k < ntiles; k++) {
    const CurveTile tl = tiles[k];
    const double dx = fmax(fmax(tl.bx0 - tx, tx - tl.bx1), 0.0);
    const double dy = fmax(fmax(tl.by0 - ty, ty - tl.by1), 0.0);
    const bool near_box = dx * dx + dy * dy < 1.0004e-4;
    const bool cross = ty > tl.ey0 && ty < tl.ey1 && tx < tl.bx1;
    if (!__any_sync(0xffffffffu, live && (near_box || cross)) && tl.code == 0) continue;
    const int j = (k << 5) + lane;
    __syncwarp();
    if (j < np) {
      sx[wl][lane] = cx[j];
      sy[wl][lane] = cy[j];
      syn[wl][lane] = cyn[j];
      scode[wl][lane] = ccode[j];
    } else {
      // padding: left of every point (no crossing), infinitely far
      sx[wl][lane] = -INFINITY;
      sy[wl][lane] = 0.0;
      syn[wl][lane] = 0.0;
      scode[wl][lane] = 0;
    }
    __syncwarp();
    for (int q = 0; q < 32; q++) {
      const double px = sx[wl][q], py = sy[wl][q];
      const double ddx = subd(tx, px), ddy = subd(ty, py);
      const double d2 = add(mul(ddx, ddx), mul(ddy, ddy));
      // sqrt(d2) < eps needs d2 < eps^2 (1 + 2^-50); test the root exactly
      if (d2 < 1.0001e-4 && __dsqrt_rn(d2) < kDomainEps) out = true;
      if (px > tx) {
        const double pyn = syn[wl][q];
        if (py < ty && pyn > ty) {
          wind++;
        } else if (py > ty && pyn < ty) {
          wind--;
        }
      }
      const int cq = scode[wl][q];
      if (cq) {
        if (cq == 1 ? wind % 2 == 0 : wind % 2 == 1) out = true;
        wind = 0;
      }
    }
  }
  if (live) mask[t] = out ? 0 : 1;
}

// Circle / Annulus / Donut::is_in_domain with the disk (cx, cy, R).
__global__ void domain_mask_disk_kernel(double cx, double cy, double R,
                                        const double* __restrict__ holes, int nh, int nt,
                                        const double* __restrict__ tg,
                                        unsigned char* __restrict__ mask) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const double tx = tg[2 * t], ty = tg[2 * t + 1];
  const double x = subd(tx, cx), y = subd(ty, cy);
  bool out = add(__dsqrt_rn(add(mul(x, x), mul(y, y))), kDomainEps) > R;
  for (int h = 0; h < nh && !out; h++) {
    const double rx = subd(tx, holes[4 * h]), ry = subd(ty, holes[4 * h + 1]);
    if (subd(__dsqrt_rn(add(mul(rx, rx), mul(ry, ry))), kDomainEps) < holes[4 * h + 2])
      out = true;
  }
  mask[t] = out ? 0 : 1;
}

// Split sums in a fixed order, + U_forward alpha, masked.
__global__ void domain_finish_kernel(int pde, int nt, int splits, long long stride,
                                     const double* __restrict__ part,
                                     const double* __restrict__ tg, int nh,
                                     const double* __restrict__ holes,
                                     const double* __restrict__ alpha,
                                     const unsigned char* __restrict__ mask,
                                     double* __restrict__ out) {
  const int sd = pde == kStokes ? 2 : 1;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= nt * sd) return;
  const int t = row / sd, comp = row % sd;
  double s = part[row];
  for (int k = 1; k < splits; k++) s += part[stride * k + row];
  if (alpha && pde != kLaplaceNeumann) {
    const double tx = tg[2 * t], ty = tg[2 * t + 1];
    for (int h = 0; h < nh; h++) {
      double u[3];
      border_u(pde, tx, ty, holes + 4 * h, comp, u);
      if (pde == kLaplace) {
        s += u[0] * alpha[h];
      } else {
        s += u[0] * alpha[3 * h] + u[1] * alpha[3 * h + 1] + u[2] * alpha[3 * h + 2];
      }
    }
  }
  if (mask && !mask[t]) s = 0.0;
  out[row] = s;
}

}  // namespace

int domain_splits(int nt, int np, int num_sms) {
  const int tiles = (nt + kDomThreads - 1) / kDomThreads;
  const int want = (2 * num_sms + tiles - 1) / tiles;
  return std::max(1, std::min(want, (np + 1023) / 1024));
}

size_t domain_mask_scratch_bytes(int np) {
  const size_t tiles = (static_cast<size_t>(np) + 31) / 32;
  return 3 * sizeof(double) * np + sizeof(int) * np + sizeof(CurveTile) * tiles + 256;
}

cudaError_t launch_domain_mask(int kind, const Node* nodes, int np, const double* holes, int nh,
                               const double* disk, int nt, const double* targets,
                               unsigned char* mask, void* scratch, cudaStream_t s) {
  if (nt == 0) return cudaSuccess;
  if (kind == kDomainNodes) {
    // scratch: x, y, next y (np doubles each), tiles (16-byte aligned), codes
    double* cx = static_cast<double*>(scratch);
    double* cy = cx + np;
    double* cyn = cy + np;
    CurveTile* tiles = reinterpret_cast<CurveTile*>(cyn + np + (np & 1));
    int* ccode = reinterpret_cast<int*>(tiles + (np + 31) / 32);
    count_launches(2);
    curve_prep_kernel<<<(np + 255) / 256, 256, 0, s>>>(nodes, np, holes, nh, cx, cy, cyn, ccode,
                                                       tiles);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int per_block = 32 * kMaskWarps;
    domain_mask_nodes_kernel<<<(nt + per_block - 1) / per_block, per_block, 0, s>>>(
        cx, cy, cyn, ccode, tiles, np, nt, targets, mask);
  } else {
    count_launches(1);
    const int grid = (nt + kDomThreads - 1) / kDomThreads;
    domain_mask_disk_kernel<<<grid, kDomThreads, 0, s>>>(disk[0], disk[1], disk[2], holes, nh,
                                                        nt, targets, mask);
  }
  return cudaGetLastError();
}

cudaError_t launch_domain_eval(int pde, const Node* nodes, int np, int nt,
                               const double* targets, const double* mu, int nh,
                               const double* holes, const double* alpha,
                               const unsigned char* mask, int splits, double* part,
                               double* out, cudaStream_t s) {
  if (nt == 0) return cudaSuccess;
  const int sd = pde == kStokes ? 2 : 1;
  const long long rows = static_cast<long long>(nt) * sd;
  double* dst = splits > 1 ? part : out;
  const int chunk = (np + splits - 1) / splits;
  const dim3 grid((nt + kDomThreads - 1) / kDomThreads, splits);
  count_launches(2);
  if (pde == kLaplace) {
    domain_partial_kernel<kLaplace><<<grid, kDomThreads, 0, s>>>(nodes, np, nt, targets, mu,
                                                                chunk, rows, dst);
  } else if (pde == kLaplaceNeumann) {
    domain_partial_kernel<kLaplaceNeumann><<<grid, kDomThreads, 0, s>>>(nodes, np, nt, targets,
                                                                       mu, chunk, rows, dst);
  } else {
    domain_partial_kernel<kStokes><<<grid, kDomThreads, 0, s>>>(nodes, np, nt, targets, mu,
                                                               chunk, rows, dst);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  domain_finish_kernel<<<static_cast<int>((rows + 255) / 256), 256, 0, s>>>(
      pde, nt, splits, rows, dst, targets, nh, holes, alpha, mask, out);
  return cudaGetLastError();
}

}  // namespace kib
