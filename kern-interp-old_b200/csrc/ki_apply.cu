// Dense operator products with on-the-fly FP64 entries:
//   * y = A x for the full boundary operator (and, for domains with holes,
//     the bordered system [K U; Psi -I] of the reference's residual check,
//     kern_interp_test.cpp:54-78), used by iterative refinement / GMRES;
//   * target evaluation, schur_solve's K_domain mu + U_forward alpha
//     (linear_solve.cpp:126-140, kernel.cpp:337-357, linear_solve.cpp:18-64);
//   * explicit kernel blocks K(tgt, src) (Kernel::operator(), kernel.cpp:99-111).
// One thread per output row; the source nodes are read in the same order by
// all lanes of a warp, so each load is a broadcast.
#include <map>
#include <mutex>
#include <tuple>

#include "ki_kernels.h"

namespace kib {

namespace {

// Segment (problem) of a node: seg[p] <= node < seg[p + 1].
__device__ __forceinline__ int apply_segment(const int* __restrict__ seg, int nseg, int node) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg[mid] <= node) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void apply_kernel(int pde, const Node* __restrict__ nodes, int n,
                             const int* __restrict__ seg, int nseg,
                             const double* __restrict__ x, double* __restrict__ y, int nb,
                             const double* __restrict__ U, const double* __restrict__ Psi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    // a forest's operator is block diagonal: sources of the row's problem
    const int sd = pde == kStokes ? 2 : 1;
    int j0 = 0, j1 = n;
    if (seg) {
      const int p = apply_segment(seg, nseg, i / sd);
      j0 = seg[p] * sd;
      j1 = seg[p + 1] * sd;
    }
    double s = 0.0;
    for (int j = j0; j < j1; j++) s += boundary_entry(pde, nodes, i, j) * x[j];
    for (int b = 0; b < nb; b++) s += U[i + static_cast<long long>(n) * b] * x[n + b];
    y[i] = s;
  } else if (i < n + nb) {
    const int h = i - n;
    double s = -x[i];
    for (int j = 0; j < n; j++) s += Psi[h + static_cast<long long>(nb) * j] * x[j];
    y[i] = s;
  }
}

// The hole border of a multiply-connected domain (initialize_U_mat and
// initialize_Psi_mat, linear_solve.cpp:18-110), one thread per node: U
// (dofs x nb, column-major) holds each hole's log / Stokeslet + rotlet
// columns at the node (and Urow the same dof-major), Psi (nb x dofs) the
// quadrature weights (and w (y, -x) for Stokes rotation) of the nodes on
// each hole.  Psi must be zero on entry.
__global__ void border_fill_kernel(int pde, const Node* __restrict__ nodes, int np,
                                   const double* __restrict__ holes, int nh, double* U,
                                   double* Psi, double* Urow) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  const Node nd = nodes[q];
  const long long N = pde == kStokes ? 2LL * np : np;
  const int rows = pde == kStokes ? 3 * nh : nh;
  for (int h = 0; h < nh; h++) {
    if (pde == kLaplace) {
      double u[3];
      border_u(pde, nd.x, nd.y, holes + 4 * h, 0, u);
      U[q + N * h] = u[0];
      Urow[static_cast<long long>(q) * rows + h] = u[0];
    } else {
      for (int c = 0; c < 2; c++) {
        double u[3];
        border_u(pde, nd.x, nd.y, holes + 4 * h, c, u);
        for (int j = 0; j < 3; j++) {
          U[2 * q + c + N * (3 * h + j)] = u[j];
          Urow[(2LL * q + c) * rows + 3 * h + j] = u[j];
        }
      }
    }
  }
  for (int h = 0; h < nh; h++) {
    const double rx = nd.x - holes[4 * h], ry = nd.y - holes[4 * h + 1];
    if (sqrt(rx * rx + ry * ry) < holes[4 * h + 2] + 1e-8) {
      auto put = [&](int i, long long j, double v) { Psi[i + rows * j] = v; };
      if (pde == kLaplace) {
        put(h, q, nd.w);
      } else {
        put(3 * h, 2 * q, nd.w);
        put(3 * h + 1, 2 * q + 1, nd.w);
        put(3 * h + 2, 2 * q, nd.w * nd.y);
        put(3 * h + 2, 2 * q + 1, -nd.w * nd.x);
      }
      break;
    }
  }
}

// One CTA per target row: the threads stride over the source dofs and the
// partial sums are reduced in a fixed order (each entry is the exact
// forward entry; only the summation order differs from a serial sum).
constexpr int kTgtThreads = 256;
__global__ void __launch_bounds__(kTgtThreads)
    targets_kernel(int pde, const Node* __restrict__ nodes, int n, int nt,
                   const double* __restrict__ tg, const double* __restrict__ mu, int nh,
                   const double* __restrict__ holes, const double* __restrict__ alpha,
                   double* __restrict__ out) {
  __shared__ double red[kTgtThreads / 32];
  const int sd = pde == kStokes ? 2 : 1;
  const int row = blockIdx.x;
  const int t = row / sd, comp = row % sd;
  const double tx = tg[2 * t], ty = tg[2 * t + 1];
  double s = 0.0;
  for (int j = threadIdx.x; j < n; j += kTgtThreads)
    s += forward_entry(pde, nodes, tx, ty, comp, j) * mu[j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x != 0) return;
  s = 0.0;
  for (int w = 0; w < kTgtThreads / 32; w++) s += red[w];
  if (alpha && pde != kLaplaceNeumann) {
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
  out[row] = s;
}

__global__ void block_kernel(int pde, const Node* __restrict__ nodes, const int* tgt, int nt,
                             const int* src, int ns, double* out) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= static_cast<long long>(nt) * ns) return;
  const int i = static_cast<int>(e % nt), j = static_cast<int>(e / nt);
  out[e] = boundary_entry(pde, nodes, tgt[i], src[j]);
}

// Forward entries (Kernel::forward, kernel.cpp:337-357): row i is domain
// dof tgt[i] (the point tgt[i] / sd, velocity component tgt[i] % sd),
// column j boundary dof src[j]; column-major nt x ns.
__global__ void forward_block_kernel(int pde, const Node* __restrict__ nodes,
                                     const double* __restrict__ tp, const int* tgt, int nt,
                                     const int* src, int ns, double* out) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= static_cast<long long>(nt) * ns) return;
  const int i = static_cast<int>(e % nt), j = static_cast<int>(e / nt);
  const int sd = pde == kStokes ? 2 : 1;
  const int pt = tgt[i] / sd, comp = tgt[i] % sd;
  out[e] = forward_entry(pde, nodes, tp[2 * pt], tp[2 * pt + 1], comp, src[j]);
}

}  // namespace

cudaError_t launch_forward_block(int pde, const Node* nodes, const double* targets,
                                 const int* tgt, int nt, const int* src, int ns, double* out,
                                 cudaStream_t s) {
  const long long tot = static_cast<long long>(nt) * ns;
  if (tot == 0) return cudaSuccess;
  count_launches(1);
  forward_block_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, s>>>(pde, nodes, targets,
                                                                           tgt, nt, src, ns, out);
  return cudaGetLastError();
}

cudaError_t launch_apply_operator(int pde, const Node* nodes, int n_dofs, const int* seg,
                                  int nseg, const double* x, double* y, int nb, const double* U,
                                  const double* Psi, cudaStream_t s) {
  const int rows = n_dofs + nb;
  count_launches(1);
  apply_kernel<<<(rows + 127) / 128, 128, 0, s>>>(pde, nodes, n_dofs, seg, nseg, x, y, nb, U,
                                                  Psi);
  return cudaGetLastError();
}

cudaError_t launch_eval_targets(int pde, const Node* nodes, int n_dofs, int nt,
                                const double* targets, const double* mu, int nh,
                                const double* holes, const double* alpha, double* out,
                                cudaStream_t s) {
  const int rows = nt * (pde == kStokes ? 2 : 1);
  if (rows == 0) return cudaSuccess;
  count_launches(1);
  targets_kernel<<<rows, kTgtThreads, 0, s>>>(pde, nodes, n_dofs, nt, targets, mu, nh, holes,
                                               alpha, out);
  return cudaGetLastError();
}

cudaError_t launch_border_fill(int pde, const Node* nodes, int np, const double* holes, int nh,
                               double* U, double* Psi, double* Urow, cudaStream_t s) {
  const long long N = pde == kStokes ? 2LL * np : np;
  const long long nb = pde == kStokes ? 3LL * nh : nh;
  const cudaError_t e = cudaMemsetAsync(Psi, 0, sizeof(double) * N * nb, s);
  if (e != cudaSuccess) return e;
  count_launches(1);
  border_fill_kernel<<<(np + 255) / 256, 256, 0, s>>>(pde, nodes, np, holes, nh, U, Psi, Urow);
  return cudaGetLastError();
}

cudaError_t launch_kernel_block(int pde, const Node* nodes, const int* tgt, int nt,
                                const int* src, int ns, double* out, cudaStream_t s) {
  const long long tot = static_cast<long long>(nt) * ns;
  if (tot == 0) return cudaSuccess;
  count_launches(1);
  block_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, s>>>(pde, nodes, tgt, nt, src, ns,
                                                                   out);
  return cudaGetLastError();
}

namespace {
__global__ void copy_segments_kernel(const CopySeg* __restrict__ segs) {
  const CopySeg sg = segs[blockIdx.x];
  for (long long i = threadIdx.x; i < sg.words; i += blockDim.x) sg.dst[i] = sg.src[i];
}
}  // namespace

cudaError_t launch_copy_segments(const CopySeg* segs, int n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  count_launches(1);
  copy_segments_kernel<<<n, 256, 0, s>>>(segs);
  return cudaGetLastError();
}

cudaError_t raise_func_attr(const void* func, cudaFuncAttribute attr, int value) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, int>, int> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_tuple(dev, func, static_cast<int>(attr));
  auto it = done.find(key);
  if (it != done.end() && it->second >= value) return cudaSuccess;
  e = cudaFuncSetAttribute(func, attr, value);
  if (e == cudaSuccess) done[key] = value;
  return e;
}

}  // namespace kib
