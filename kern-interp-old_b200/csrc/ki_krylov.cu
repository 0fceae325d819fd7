// FP64 kernels of the iterative-refinement / GMRES solve:
//   * a fast dense operator product y = A x with entries formed on the fly
//     (the boundary operator of kernel.cpp:11-96, bordered by the hole
//     columns U and rows Psi when the domain has holes, as in the residual
//     check of kern_interp_test.cpp:54-78).  Unlike apply_kernel it is free
//     to fuse and reassociate: it is the refinement residual, accurate to
//     FP64 rounding, not the bit-exact entry path of the factorization;
//   * the few vector operations GMRES needs (several dot products in one
//     pass, several axpys in one pass, scaling), all with a fixed reduction
//     order so a solve is reproducible.
//
// Operator product layout: one thread per target node, 256 targets per CTA,
// sources staged 256 at a time in shared memory as structure-of-arrays with
// the density folded in; the source range is split over gridDim.y so the
// grid covers every SM, and the splits' partial sums are added in order by
// a second kernel (no atomics).
#include <algorithm>
#include <vector>

#include "ki_kernels.h"

namespace kib {

namespace {

constexpr int kMvThreads = 256;

// Per-source values staged in shared memory.
//   Laplace:          a = -(w / 2 pi) x (n_x, n_y)
//   Laplace-Neumann:  a = (w / 2 pi) x (1, 1)      (target normal applied later)
//   Stokes:           a = (w / pi) (n_x, n_y), density (x0, x1)
template <int PDE>
__global__ void __launch_bounds__(kMvThreads)
    mv_partial_kernel(const Node* __restrict__ nodes, const MvTile* __restrict__ tiles,
                      long long part_stride, const double* __restrict__ x,
                      double* __restrict__ part, double* __restrict__ part_rank1) {
  __shared__ double sx[kMvThreads], sy[kMvThreads], sa0[kMvThreads], sa1[kMvThreads];
  __shared__ double sd0[kMvThreads], sd1[kMvThreads];
  __shared__ double red[kMvThreads / 32];
  const MvTile tile = tiles[blockIdx.x];
  const int t = tile.t0 + threadIdx.x;
  const int s0 = tile.s0, s1 = tile.s1;
  const bool live = t < tile.t1;
  double tx = 0, ty = 0, tnx = 0, tny = 0;
  if (live) {
    const Node nt = nodes[t];
    tx = nt.x;
    ty = nt.y;
    tnx = nt.nx;
    tny = nt.ny;
  }
  double y0 = 0.0, y1 = 0.0, r1 = 0.0;
  for (int base = s0; base < s1; base += kMvThreads) {
    const int j = base + threadIdx.x;
    __syncthreads();
    if (j < s1) {
      const Node s = nodes[j];
      sx[threadIdx.x] = s.x;
      sy[threadIdx.x] = s.y;
      if (PDE == kLaplace) {
        const double c = -s.w * KI_INV_2PI * x[j];
        sa0[threadIdx.x] = c * s.nx;
        sa1[threadIdx.x] = c * s.ny;
      } else if (PDE == kLaplaceNeumann) {
        sa0[threadIdx.x] = s.w * KI_INV_2PI * x[j];
        // rank-one part: sum_j w_j x_j (the "+ w_s" of every entry)
        if (tile.first) r1 += s.w * x[j];
      } else {
        const double c = s.w * KI_INV_PI;
        sa0[threadIdx.x] = c * s.nx;
        sa1[threadIdx.x] = c * s.ny;
        const double d0 = x[2 * j], d1 = x[2 * j + 1];
        sd0[threadIdx.x] = d0;
        sd1[threadIdx.x] = d1;
        // rank-one part: sum_j w_j (n_j . x_j), applied as tn_t * sum
        if (tile.first) r1 += s.w * (s.nx * d0 + s.ny * d1);
      }
    } else {
      // padding: a source far away with zero strength (|r|^2 stays within
      // the FP32 range of the reciprocal estimate; its numerators are zero)
      sx[threadIdx.x] = 1e15;
      sy[threadIdx.x] = 1e15;
      sa0[threadIdx.x] = 0.0;
      sa1[threadIdx.x] = 0.0;
      sd0[threadIdx.x] = 0.0;
      sd1[threadIdx.x] = 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < kMvThreads; q++) {
      const double r0 = tx - sx[q], rr1 = ty - sy[q];
      const double rr = r0 * r0 + rr1 * rr1;
      const double inv = rr > 0.0 ? nr_rcp(rr) : 0.0;
      if (PDE == kLaplace) {
        y0 += (r0 * sa0[q] + rr1 * sa1[q]) * inv;
      } else if (PDE == kLaplaceNeumann) {
        y0 += ((r0 * tnx + rr1 * tny) * sa0[q]) * inv;
      } else {
        const double rn = r0 * sa0[q] + rr1 * sa1[q];
        const double rx = r0 * sd0[q] + rr1 * sd1[q];
        const double pq = (rn * rx) * (inv * inv);
        y0 += pq * r0;
        y1 += pq * rr1;
      }
    }
  }
  if (live) {
    if (PDE == kStokes) {
      part[part_stride * tile.split + 2 * t] = y0;
      part[part_stride * tile.split + 2 * t + 1] = y1;
    } else {
      part[part_stride * tile.split + t] = y0;
    }
  }
  if (PDE != kLaplace && tile.first) {
    // fixed-order block sum of the rank-one coefficient of this split
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r1 += __shfl_xor_sync(0xffffffffu, r1, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = r1;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = 0.0;
      for (int w = 0; w < kMvThreads / 32; w++) v += red[w];
      part_rank1[tile.rank1_slot] = v;
    }
  }
}

// Operator product of a refinement correction, y = A d, where d is small
// next to the iterate (|d| ~ the preconditioner's accuracy times |x|), so a
// relative error eps in A d moves the updated residual r - A d by eps |d|
// only.  The pair sums run in FP32 (twice the FP64 pipe's rate, one MUFU
// reciprocal per pair) on coordinates taken relative to the target tile's
// first node, with the densities scaled by `dscale` (~1/|d|) to keep them
// in FP32's normal range; each 256-source block's FP32 sums are added to
// FP64 accumulators.  A source block whose bounding box comes within
// sqrt(near2) of the target tile's is summed in FP64 exactly as in
// mv_partial_kernel: for nearby nodes of one curve r.n_s is a small
// difference of O(|r|) terms (it behaves like kappa |r|^2 / 2), which FP32
// coordinates cannot resolve.  With gap g, the FP32 pairs' entries err by
// about u32 (|s - o| + |t - o|) w / (pi r^2); summed along a curve of node
// spacing h beyond the gap this is ~ u32 diam w / (h g) per unit density,
// 1e-6 for g = 0.01 on the workloads here.  Partials, rank-one slots and the
// finish are those of the FP64 product.
//
// A thread owns two targets of the 256-target tile, t and t + 128, as the two
// lanes of Blackwell's packed FP32 instructions (FADD2 / FMUL2 / FFMA2, one
// issue for both lanes): each source's values sit in shared memory twice,
// {v, v}, so a 16-byte load yields the packed operands of both lanes.  Every
// lane rounds exactly as the scalar fmaf, product or sum it stands for, so a
// target's sums are those of one target per thread; the packing halves the
// FP32 instructions the issue slots carry (loads, MUFU and FP32 shared them).
constexpr int kCorrThreads = kMvThreads / 2;

template <int PDE>
__global__ void __launch_bounds__(kCorrThreads)
    mv_corr_partial_kernel(const Node* __restrict__ nodes, const MvTile* __restrict__ tiles,
                           long long part_stride, const double* __restrict__ x, double dscale,
                           float near2, double* __restrict__ part,
                           double* __restrict__ part_rank1) {
  __shared__ double sx[kMvThreads], sy[kMvThreads], sa0[kMvThreads], sa1[kMvThreads];
  __shared__ double sd0[kMvThreads], sd1[kMvThreads];
  // FP32 source values relative to the tile origin, each twice:
  // pos {-x, -x, -y, -y}, amp {a0, a0, a1, a1}, den {d0, d0, d1, d1}
  __shared__ float4 fpos[kMvThreads], famp[kMvThreads], fden[kMvThreads];
  __shared__ float wbox[2][4][kCorrThreads / 32];  // per-warp box: [target|source][x0,y0,-x1,-y1]
  __shared__ double red[kCorrThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const MvTile tile = tiles[blockIdx.x];
  const int s0 = tile.s0, s1 = tile.s1;
  const Node org = nodes[tile.t0];
  const double ox = org.x, oy = org.y;
  const double inv_scale = 1.0 / dscale;
  double tx[2], ty[2], tnx[2], tny[2];
  bool live[2];
  float ftx[2], fty[2], ftnx[2], ftny[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int t = tile.t0 + threadIdx.x + h * kCorrThreads;
    live[h] = t < tile.t1;
    tx[h] = ty[h] = tnx[h] = tny[h] = 0.0;
    if (live[h]) {
      const Node nt = nodes[t];
      tx[h] = nt.x;
      ty[h] = nt.y;
      tnx[h] = nt.nx;
      tny[h] = nt.ny;
    }
    ftx[h] = static_cast<float>(tx[h] - ox);
    fty[h] = static_cast<float>(ty[h] - oy);
    ftnx[h] = static_cast<float>(tnx[h]);
    ftny[h] = static_cast<float>(tny[h]);
  }
  // bounding box of a thread's two points over the CTA: warp min/max here,
  // the per-warp results combined by every thread after the next barrier
  auto warp_box = [&](int which, bool v0, float px0, float py0, bool v1, float px1,
                      float py1) {
    float b0 = fminf(v0 ? px0 : 3e38f, v1 ? px1 : 3e38f);
    float b1 = fminf(v0 ? py0 : 3e38f, v1 ? py1 : 3e38f);
    float b2 = fminf(v0 ? -px0 : 3e38f, v1 ? -px1 : 3e38f);
    float b3 = fminf(v0 ? -py0 : 3e38f, v1 ? -py1 : 3e38f);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      b0 = fminf(b0, __shfl_xor_sync(0xffffffffu, b0, o));
      b1 = fminf(b1, __shfl_xor_sync(0xffffffffu, b1, o));
      b2 = fminf(b2, __shfl_xor_sync(0xffffffffu, b2, o));
      b3 = fminf(b3, __shfl_xor_sync(0xffffffffu, b3, o));
    }
    if (lane == 0) {
      wbox[which][0][warp] = b0;
      wbox[which][1][warp] = b1;
      wbox[which][2][warp] = b2;
      wbox[which][3][warp] = b3;
    }
  };
  auto cta_box = [&](int which, int c) {
    float b = 3e38f;
#pragma unroll
    for (int w = 0; w < kCorrThreads / 32; w++) b = fminf(b, wbox[which][c][w]);
    return b;
  };
  warp_box(0, live[0], ftx[0], fty[0], live[1], ftx[1], fty[1]);
  const float2 tx2 = make_float2(ftx[0], ftx[1]), ty2 = make_float2(fty[0], fty[1]);
  const float2 tnx2 = make_float2(ftnx[0], ftnx[1]), tny2 = make_float2(ftny[0], ftny[1]);
  double y0[2] = {0.0, 0.0}, y1[2] = {0.0, 0.0}, r1 = 0.0;
  for (int base = s0; base < s1; base += kMvThreads) {
    __syncthreads();
    bool valid[2];
    float fsx[2], fsy[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int k = threadIdx.x + h * kCorrThreads;  // staging slot
      const int j = base + k;
      valid[h] = j < s1;
      float fa0 = 0.f, fa1 = 0.f, fd0 = 0.f, fd1 = 0.f;
      if (valid[h]) {
        const Node s = nodes[j];
        sx[k] = s.x;
        sy[k] = s.y;
        fsx[h] = static_cast<float>(s.x - ox);
        fsy[h] = static_cast<float>(s.y - oy);
        if (PDE == kLaplace) {
          const double c = -s.w * KI_INV_2PI * x[j];
          sa0[k] = c * s.nx;
          sa1[k] = c * s.ny;
          fa0 = static_cast<float>(c * dscale * s.nx);
          fa1 = static_cast<float>(c * dscale * s.ny);
        } else if (PDE == kLaplaceNeumann) {
          sa0[k] = s.w * KI_INV_2PI * x[j];
          fa0 = static_cast<float>(s.w * KI_INV_2PI * (x[j] * dscale));
          if (tile.first) r1 += s.w * x[j];
        } else {
          const double c = s.w * KI_INV_PI;
          sa0[k] = c * s.nx;
          sa1[k] = c * s.ny;
          fa0 = static_cast<float>(c * s.nx);
          fa1 = static_cast<float>(c * s.ny);
          const double d0 = x[2 * j], d1 = x[2 * j + 1];
          sd0[k] = d0;
          sd1[k] = d1;
          fd0 = static_cast<float>(d0 * dscale);
          fd1 = static_cast<float>(d1 * dscale);
          if (tile.first) r1 += s.w * (s.nx * d0 + s.ny * d1);
        }
      } else {
        // padding: a far source of zero strength
        sx[k] = 1e15;
        sy[k] = 1e15;
        sa0[k] = sa1[k] = 0.0;
        sd0[k] = sd1[k] = 0.0;
        fsx[h] = fsy[h] = 1e15f;
      }
      fpos[k] = make_float4(-fsx[h], -fsx[h], -fsy[h], -fsy[h]);
      famp[k] = make_float4(fa0, fa0, fa1, fa1);
      if (PDE == kStokes) fden[k] = make_float4(fd0, fd0, fd1, fd1);
    }
    warp_box(1, valid[0], fsx[0], fsy[0], valid[1], fsx[1], fsy[1]);
    __syncthreads();
    // gap between the boxes (0 when they overlap)
    const float gx = fmaxf(0.f, fmaxf(cta_box(1, 0) + cta_box(0, 2), cta_box(0, 0) + cta_box(1, 2)));
    const float gy = fmaxf(0.f, fmaxf(cta_box(1, 1) + cta_box(0, 3), cta_box(0, 1) + cta_box(1, 3)));
    if (gx * gx + gy * gy < near2) {
#pragma unroll 2
      for (int q = 0; q < kMvThreads; q++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const double r0 = tx[h] - sx[q], rr1 = ty[h] - sy[q];
          const double rr = r0 * r0 + rr1 * rr1;
          const double inv = rr > 0.0 ? nr_rcp(rr) : 0.0;
          if (PDE == kLaplace) {
            y0[h] += (r0 * sa0[q] + rr1 * sa1[q]) * inv;
          } else if (PDE == kLaplaceNeumann) {
            y0[h] += ((r0 * tnx[h] + rr1 * tny[h]) * sa0[q]) * inv;
          } else {
            const double rn = r0 * sa0[q] + rr1 * sa1[q];
            const double rx = r0 * sd0[q] + rr1 * sd1[q];
            const double pq = (rn * rx) * (inv * inv);
            y0[h] += pq * r0;
            y1[h] += pq * rr1;
          }
        }
      }
    } else {
      float2 f0 = make_float2(0.f, 0.f), f1 = make_float2(0.f, 0.f);
#pragma unroll 8
      for (int q = 0; q < kMvThreads; q++) {
        const float4 p = fpos[q], a = famp[q];
        const float2 r0 = __fadd2_rn(tx2, make_float2(p.x, p.y));
        const float2 rr1 = __fadd2_rn(ty2, make_float2(p.z, p.w));
        const float2 rr = __ffma2_rn(r0, r0, __fmul2_rn(rr1, rr1));
        float2 inv;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(inv.x) : "f"(rr.x));
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(inv.y) : "f"(rr.y));
        const float2 a0 = make_float2(a.x, a.y), a1 = make_float2(a.z, a.w);
        if (PDE == kLaplace) {
          f0 = __ffma2_rn(__ffma2_rn(r0, a0, __fmul2_rn(rr1, a1)), inv, f0);
        } else if (PDE == kLaplaceNeumann) {
          f0 = __ffma2_rn(__fmul2_rn(__ffma2_rn(r0, tnx2, __fmul2_rn(rr1, tny2)), a0), inv, f0);
        } else {
          const float4 d = fden[q];
          const float2 rn = __ffma2_rn(r0, a0, __fmul2_rn(rr1, a1));
          const float2 rx = __ffma2_rn(r0, make_float2(d.x, d.y),
                                       __fmul2_rn(rr1, make_float2(d.z, d.w)));
          const float2 pq = __fmul2_rn(__fmul2_rn(rn, rx), __fmul2_rn(inv, inv));
          f0 = __ffma2_rn(pq, r0, f0);
          f1 = __ffma2_rn(pq, rr1, f1);
        }
      }
      y0[0] += static_cast<double>(f0.x) * inv_scale;
      y0[1] += static_cast<double>(f0.y) * inv_scale;
      y1[0] += static_cast<double>(f1.x) * inv_scale;
      y1[1] += static_cast<double>(f1.y) * inv_scale;
    }
  }
#pragma unroll
  for (int h = 0; h < 2; h++) {
    if (!live[h]) continue;
    const int t = tile.t0 + threadIdx.x + h * kCorrThreads;
    if (PDE == kStokes) {
      part[part_stride * tile.split + 2 * t] = y0[h];
      part[part_stride * tile.split + 2 * t + 1] = y1[h];
    } else {
      part[part_stride * tile.split + t] = y0[h];
    }
  }
  if (PDE != kLaplace && tile.first) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r1 += __shfl_xor_sync(0xffffffffu, r1, o);
    if (lane == 0) red[warp] = r1;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = 0.0;
      for (int w = 0; w < kCorrThreads / 32; w++) v += red[w];
      part_rank1[tile.rank1_slot] = v;
    }
  }
}

// y_i = sum of the splits' partials + diagonal correction + rank-one term +
// U x_border; the border rows are done by mv_border_partial_kernel.
__device__ __forceinline__ int segment_of(const int* __restrict__ seg, int nseg, int node) {
  int lo = 0, hi = nseg - 1;  // seg[lo] <= node < seg[hi + 1]
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg[mid] <= node) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void mv_finish_kernel(int pde, const Node* __restrict__ nodes, int n_dofs,
                                 int splits, const double* __restrict__ part,
                                 const double* __restrict__ part_rank1,
                                 const int* __restrict__ seg, int nseg,
                                 const double* __restrict__ x, double* __restrict__ y, int nb,
                                 const double* __restrict__ U) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_dofs) return;
  double s = 0.0;
  for (int p = 0; p < splits; p++) s += part[static_cast<long long>(p) * n_dofs + i];
  double g = 0.0;
  if (pde != kLaplace) {
    const int q = segment_of(seg, nseg, pde == kStokes ? i >> 1 : i);
    for (int p = 0; p < splits; p++) g += part_rank1[static_cast<long long>(q) * splits + p];
  }
  if (pde == kLaplace) {
    const Node nd = nodes[i];
    s += (0.5 + 0.5 * nd.k * nd.w * KI_INV_2PI) * x[i];
  } else if (pde == kLaplaceNeumann) {
    const Node nd = nodes[i];
    s += g + (-0.5 + 0.5 * nd.k * nd.w * KI_INV_2PI) * x[i];
  } else {
    const Node nd = nodes[i >> 1];
    const int c = i & 1;
    const double tn = c ? nd.ny : nd.nx;
    // -1/2 x - (kappa w / 2 pi) t (t . x), t = (-n_y, n_x), and tn_c * g
    const double tc = c ? nd.nx : -nd.ny;
    const double tdotx = -nd.ny * x[i & ~1] + nd.nx * x[i | 1];
    s += -0.5 * x[i] - nd.k * nd.w * KI_INV_2PI * tc * tdotx + tn * g;
  }
  for (int b = 0; b < nb; b++) s += U[i + static_cast<long long>(n_dofs) * b] * x[n_dofs + b];
  y[i] = s;
}

// Border rows y_{N+h} = Psi(h, :) x(0:N) - x_{N+h} in one pass over Psi:
// Psi is nb x N column-major, so a dof's nb entries are contiguous; each
// thread walks dofs, accumulating up to 32 rows at a time in registers, and
// each CTA writes its partial sums (kBorderBlocks x nb), added in a fixed
// order by mv_border_finish_kernel.
constexpr int kBorderBlocks = 64;
__global__ void __launch_bounds__(256)
    mv_border_partial_kernel(int n_dofs, int nb, const double* __restrict__ Psi,
                             const double* __restrict__ x, double* __restrict__ part) {
  __shared__ double red[8][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int per = (n_dofs + gridDim.x - 1) / gridDim.x;
  const int j0 = blockIdx.x * per, j1 = min(n_dofs, j0 + per);
  for (int h0 = 0; h0 < nb; h0 += 32) {
    const int hn = min(32, nb - h0);
    double acc[32];
#pragma unroll
    for (int h = 0; h < 32; h++) acc[h] = 0.0;
    for (int j = j0 + threadIdx.x; j < j1; j += 256) {
      const double xj = x[j];
      const double* pc = Psi + static_cast<long long>(nb) * j + h0;
#pragma unroll
      for (int h = 0; h < 32; h++)
        if (h < hn) acc[h] += pc[h] * xj;
    }
#pragma unroll
    for (int h = 0; h < 32; h++) {
      double v = acc[h];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][h] = v;
    }
    __syncthreads();
    if (threadIdx.x < hn) {
      double v = 0.0;
      for (int w = 0; w < 8; w++) v += red[w][threadIdx.x];
      part[static_cast<long long>(blockIdx.x) * nb + h0 + threadIdx.x] = v;
    }
    __syncthreads();
  }
}

__global__ void mv_border_finish_kernel(int n_dofs, int nb, int nblk,
                                        const double* __restrict__ part,
                                        const double* __restrict__ x, double* __restrict__ y) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= nb) return;
  double v = 0.0;
  for (int b = 0; b < nblk; b++) v += part[static_cast<long long>(b) * nb + h];
  y[n_dofs + h] = v - x[n_dofs + h];
}

// ---- vector kernels (n up to a few million; k <= kMaxKrylov vectors)

constexpr int kVecThreads = 256;

// part[j * gridDim.x + b] = sum over this CTA's slice of V_j . w
// Partial sums of V(:, j) . w over this block's rows for j < k: a thread
// per row, the columns 16 at a time with their loads in flight together,
// then a fixed-order reduction over the block.
constexpr int kDotChunk = 16;
__global__ void multi_dot_kernel(const double* __restrict__ V, long long ldv, int k,
                                 const double* __restrict__ w, int n, double* __restrict__ part) {
  __shared__ double red[kVecThreads / 32][kDotChunk];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int per = (n + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(n, i0 + per);
  for (int j0 = 0; j0 < k; j0 += kDotChunk) {
    double s[kDotChunk];
#pragma unroll
    for (int u = 0; u < kDotChunk; u++) s[u] = 0.0;
    for (int i = i0 + threadIdx.x; i < i1; i += kVecThreads) {
      const double wi = w[i];
#pragma unroll
      for (int u = 0; u < kDotChunk; u++)
        if (j0 + u < k) s[u] += V[ldv * (j0 + u) + i] * wi;
    }
#pragma unroll
    for (int u = 0; u < kDotChunk; u++) {
      double v = s[u];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][u] = v;
    }
    __syncthreads();
    if (threadIdx.x < kDotChunk && j0 + threadIdx.x < k) {
      double v = 0.0;
      for (int q = 0; q < kVecThreads / 32; q++) v += red[q][threadIdx.x];
      part[static_cast<long long>(j0 + threadIdx.x) * gridDim.x + blockIdx.x] = v;
    }
    __syncthreads();
  }
}

// out[j] = the sum of column j's partials: a warp per column (lanes over
// the blocks, then a shuffle tree: a fixed order).
__global__ void multi_dot_finish_kernel(const double* __restrict__ part, int nblk, int k,
                                        double* __restrict__ out) {
  const int j = blockIdx.x, lane = threadIdx.x;
  if (j >= k) return;
  const double* p = part + static_cast<long long>(j) * nblk;
  double v0 = 0.0, v1 = 0.0;
  int b = lane;
  for (; b + 32 < nblk; b += 64) {
    v0 += p[b];
    v1 += p[b + 32];
  }
  if (b < nblk) v0 += p[b];
  double v = v0 + v1;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) out[j] = v;
}

// w -= V h (h on the device, k entries)
__global__ void multi_axpy_kernel(double* __restrict__ w, const double* __restrict__ V,
                                  long long ldv, int k, const double* __restrict__ h, int n,
                                  double sign) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int j = 0; j < k; j++) s += V[ldv * j + i] * h[j];
  w[i] += sign * s;
}

__global__ void scale_copy_kernel(double* __restrict__ dst, const double* __restrict__ src,
                                  int n, double a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = a * src[i];
}

__global__ void add_kernel(double* __restrict__ x, const double* __restrict__ y, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += y[i];
}

__global__ void rsub_kernel(double* __restrict__ y, const double* __restrict__ g, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = (g ? g[i] : 0.0) - y[i];
}

__global__ void sub_kernel(double* __restrict__ r, const double* __restrict__ b,
                           const double* __restrict__ ax, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = b[i] - ax[i];
}

// out[p] = sum of v^2 over dofs [seg[p] * sd, seg[p + 1] * sd), one CTA per
// segment, fixed order.
__global__ void segment_sumsq_kernel(const double* __restrict__ v, const int* __restrict__ seg,
                                     int sd, double* __restrict__ out) {
  __shared__ double red[32];
  const long long a = static_cast<long long>(seg[blockIdx.x]) * sd;
  const long long b = static_cast<long long>(seg[blockIdx.x + 1]) * sd;
  double s = 0.0;
  for (long long i = a + threadIdx.x; i < b; i += blockDim.x) s += v[i] * v[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); w++) t += red[w];
    out[blockIdx.x] = t;
  }
}

}  // namespace

int matvec_splits(int pde, int n_nodes, int nseg, int num_sms) {
  // resident CTAs of the product kernel on the whole GPU
  int per_sm = 0;
  const void* fn = pde == kLaplace ? reinterpret_cast<const void*>(&mv_partial_kernel<kLaplace>)
                   : pde == kLaplaceNeumann
                       ? reinterpret_cast<const void*>(&mv_partial_kernel<kLaplaceNeumann>)
                       : reinterpret_cast<const void*>(&mv_partial_kernel<kStokes>);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kMvThreads, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long slots = static_cast<long long>(per_sm) * std::max(1, num_sms);
  const int per_seg = (n_nodes + kMvThreads - 1) / kMvThreads;  // target tiles
  const long long tblocks = static_cast<long long>(per_seg) * std::max(1, nseg);
  const int max_split = std::max(1, std::min(per_seg, kMaxMatvecSplits));  // >= 256 sources each
  // time ~ waves x (sources per split): minimise ceil(tblocks S / slots) / S
  int best = 1;
  double best_t = 1e300;
  for (int S = 1; S <= max_split; S++) {
    const double t = static_cast<double>((tblocks * S + slots - 1) / slots) / S;
    if (t < best_t * (1.0 - 1e-9)) {
      best_t = t;
      best = S;
    }
  }
  return best;
}

void matvec_tiles(const std::vector<int>& seg, int splits, std::vector<MvTile>* tiles) {
  // per segment: target tiles of 256 nodes x source chunks; every (target,
  // split) pair gets a tile, so each partial is written exactly once
  tiles->clear();
  const int nseg = static_cast<int>(seg.size()) - 1;
  for (int p = 0; p < nseg; p++) {
    const int a = seg[p], b = seg[p + 1];
    const int chunk = ((b - a + splits - 1) / splits + kMvThreads - 1) / kMvThreads * kMvThreads;
    for (int q = 0; q < splits; q++) {
      const int s0 = std::min(b, a + q * chunk), s1 = std::min(b, s0 + chunk);
      for (int t0 = a; t0 < b; t0 += kMvThreads)
        tiles->push_back(MvTile{t0, std::min(b, t0 + kMvThreads), s0, s1, q, p * splits + q,
                                t0 == a ? 1 : 0, 0});
    }
  }
}

cudaError_t launch_fast_matvec(int pde, const Node* nodes, const MvTile* tiles, int ntiles,
                               const int* seg, int nseg, int n_dofs, int splits, const double* x,
                               double* y, int nb, const double* U, const double* Psi,
                               double* part, cudaStream_t s) {
  if (splits < 1 || splits > kMaxMatvecSplits) return cudaErrorInvalidValue;
  double* part_rank1 = part + static_cast<long long>(splits) * n_dofs;
  count_launches(nb ? 3 : 2);
  if (pde == kLaplace)
    mv_partial_kernel<kLaplace><<<ntiles, kMvThreads, 0, s>>>(nodes, tiles, n_dofs, x, part,
                                                               part_rank1);
  else if (pde == kLaplaceNeumann)
    mv_partial_kernel<kLaplaceNeumann><<<ntiles, kMvThreads, 0, s>>>(nodes, tiles, n_dofs, x,
                                                                      part, part_rank1);
  else
    mv_partial_kernel<kStokes><<<ntiles, kMvThreads, 0, s>>>(nodes, tiles, n_dofs, x, part,
                                                              part_rank1);
  mv_finish_kernel<<<(n_dofs + 255) / 256, 256, 0, s>>>(pde, nodes, n_dofs, splits, part,
                                                        part_rank1, seg, nseg, x, y, nb, U);
  if (nb) {
    double* bpart = part_rank1 + static_cast<long long>(splits) * nseg;
    count_launches(1);
    mv_border_partial_kernel<<<kBorderBlocks, 256, 0, s>>>(n_dofs, nb, Psi, x, bpart);
    mv_border_finish_kernel<<<(nb + 63) / 64, 64, 0, s>>>(n_dofs, nb, kBorderBlocks, bpart, x, y);
  }
  return cudaGetLastError();
}

cudaError_t launch_corr_matvec(int pde, const Node* nodes, const MvTile* tiles, int ntiles,
                               const int* seg, int nseg, int n_dofs, int splits, const double* x,
                               double dscale, double near_gap, double* y, int nb,
                               const double* U, const double* Psi, double* part,
                               cudaStream_t s) {
  if (splits < 1 || splits > kMaxMatvecSplits || !(dscale > 0.0)) return cudaErrorInvalidValue;
  double* part_rank1 = part + static_cast<long long>(splits) * n_dofs;
  const float near2 = static_cast<float>(near_gap * near_gap);
  count_launches(nb ? 3 : 2);
  if (pde == kLaplace)
    mv_corr_partial_kernel<kLaplace><<<ntiles, kCorrThreads, 0, s>>>(
        nodes, tiles, n_dofs, x, dscale, near2, part, part_rank1);
  else if (pde == kLaplaceNeumann)
    mv_corr_partial_kernel<kLaplaceNeumann><<<ntiles, kCorrThreads, 0, s>>>(
        nodes, tiles, n_dofs, x, dscale, near2, part, part_rank1);
  else
    mv_corr_partial_kernel<kStokes><<<ntiles, kCorrThreads, 0, s>>>(
        nodes, tiles, n_dofs, x, dscale, near2, part, part_rank1);
  mv_finish_kernel<<<(n_dofs + 255) / 256, 256, 0, s>>>(pde, nodes, n_dofs, splits, part,
                                                        part_rank1, seg, nseg, x, y, nb, U);
  if (nb) {
    double* bpart = part_rank1 + static_cast<long long>(splits) * nseg;
    count_launches(1);
    mv_border_partial_kernel<<<kBorderBlocks, 256, 0, s>>>(n_dofs, nb, Psi, x, bpart);
    mv_border_finish_kernel<<<(nb + 63) / 64, 64, 0, s>>>(n_dofs, nb, kBorderBlocks, bpart, x, y);
  }
  return cudaGetLastError();
}

size_t fast_matvec_scratch_doubles(int n_dofs, int splits, int nseg, int nb) {
  return static_cast<size_t>(splits) * n_dofs + static_cast<size_t>(splits) * nseg +
         static_cast<size_t>(kBorderBlocks) * nb;
}

int multi_dot_blocks(int n) { return std::max(1, std::min(592, (n + 255) / 256)); }

cudaError_t launch_multi_dot(const double* V, long long ldv, int k, const double* w, int n,
                             double* part, double* out, cudaStream_t s) {
  if (k < 1 || k > kMaxKrylov) return cudaErrorInvalidValue;
  const int nblk = multi_dot_blocks(n);
  count_launches(2);
  multi_dot_kernel<<<nblk, kVecThreads, 0, s>>>(V, ldv, k, w, n, part);
  multi_dot_finish_kernel<<<k, 32, 0, s>>>(part, nblk, k, out);
  return cudaGetLastError();
}

cudaError_t launch_multi_axpy(double* w, const double* V, long long ldv, int k, const double* h,
                              int n, double sign, cudaStream_t s) {
  if (k < 1) return cudaSuccess;
  count_launches(1);
  multi_axpy_kernel<<<(n + 255) / 256, 256, 0, s>>>(w, V, ldv, k, h, n, sign);
  return cudaGetLastError();
}

cudaError_t launch_scale_copy(double* dst, const double* src, int n, double a, cudaStream_t s) {
  count_launches(1);
  scale_copy_kernel<<<(n + 255) / 256, 256, 0, s>>>(dst, src, n, a);
  return cudaGetLastError();
}

cudaError_t launch_segment_sumsq(const double* v, const int* seg, int nseg, int sd, double* out,
                                 cudaStream_t s) {
  count_launches(1);
  segment_sumsq_kernel<<<nseg, 256, 0, s>>>(v, seg, sd, out);
  return cudaGetLastError();
}

cudaError_t launch_add(double* x, const double* y, int n, cudaStream_t s) {
  count_launches(1);
  add_kernel<<<(n + 255) / 256, 256, 0, s>>>(x, y, n);
  return cudaGetLastError();
}

cudaError_t launch_rsub(double* y, const double* g, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launches(1);
  rsub_kernel<<<(n + 255) / 256, 256, 0, s>>>(y, g, n);
  return cudaGetLastError();
}

cudaError_t launch_sub(double* r, const double* b, const double* ax, int n, cudaStream_t s) {
  count_launches(1);
  sub_kernel<<<(n + 255) / 256, 256, 0, s>>>(r, b, ax, n);
  return cudaGetLastError();
}

}  // namespace kib
