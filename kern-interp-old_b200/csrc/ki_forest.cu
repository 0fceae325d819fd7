// Top level of a forest of independent problems (many boundaries factored
// together): each tree's root skeleton matrix (skel_factorization.cpp:
// 116-128, one per problem) is assembled, LU-factored and solved by one CTA
// per tree in a single launch each, instead of one dense LU per problem.
#include "ki_blockla.cuh"
#include "ki_kernels.h"

namespace kib {

namespace {

__device__ __forceinline__ double top_upd(const TopTask& t, int a, int b) {
  const int ia = t.bid[a];
  if (ia < 0 || ia != t.bid[b]) return 0.0;
  const UpdBlock blk = t.blocks[ia];
  return blk.acc[t.bpos[a] + static_cast<long long>(blk.size) * t.bpos[b]];
}

__global__ void forest_assemble_kernel(int pde, const Node* __restrict__ nodes,
                                       const TopTask* __restrict__ tasks) {
  const TopTask t = tasks[blockIdx.y];
  const int nn = t.n * t.n;  // top skeletons are far below 46341 dofs
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += gridDim.x * blockDim.x) {
    const int a = e % t.n, b = e / t.n;
    t.a[e] = boundary_entry(pde, nodes, t.dofs[a], t.dofs[b]) - top_upd(t, a, b);
  }
}

constexpr int kForestThreads = 512;

__global__ void __launch_bounds__(kForestThreads)
    forest_lu_kernel(const TopTask* __restrict__ tasks, int* status) {
  __shared__ double red[64];
  const TopTask t = tasks[blockIdx.x];
  if (t.n == 0) return;
  if (cta_lu(t.a, t.n, t.n, t.piv, red) && threadIdx.x == 0) atomicExch(status, 1);
}

__global__ void __launch_bounds__(kForestThreads)
    forest_solve_kernel(const TopTask* __restrict__ tasks, double* __restrict__ x) {
  extern __shared__ double xs[];
  const TopTask t = tasks[blockIdx.x];
  if (t.n == 0) return;
  for (int i = threadIdx.x; i < t.n; i += blockDim.x) xs[i] = x[t.dofs[i]];
  __syncthreads();
  cta_lu_solve(t.a, t.n, t.n, t.piv, xs);
  for (int i = threadIdx.x; i < t.n; i += blockDim.x) x[t.dofs[i]] = xs[i];
}

}  // namespace

cudaError_t launch_forest_top(int pde, const Node* nodes, const TopTask* tasks, int ntasks,
                              int n_max, int* status, cudaStream_t s) {
  if (ntasks == 0 || n_max == 0) return cudaSuccess;
  const long long nn = static_cast<long long>(n_max) * n_max;
  const int gx = static_cast<int>(std::min<long long>((nn + 255) / 256, 64));
  count_launches(2);
  forest_assemble_kernel<<<dim3(gx, ntasks), 256, 0, s>>>(pde, nodes, tasks);
  forest_lu_kernel<<<ntasks, kForestThreads, 0, s>>>(tasks, status);
  return cudaGetLastError();
}

cudaError_t launch_forest_top_solve(const TopTask* tasks, int ntasks, int n_max, double* x,
                                    cudaStream_t s) {
  if (ntasks == 0 || n_max == 0) return cudaSuccess;
  const size_t smem = sizeof(double) * static_cast<size_t>(n_max);
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  const cudaError_t e = raise_func_attr(reinterpret_cast<const void*>(&forest_solve_kernel),
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e != cudaSuccess) return e;
  count_launches(1);
  forest_solve_kernel<<<ntasks, kForestThreads, smem, s>>>(tasks, x);
  return cudaGetLastError();
}

}  // namespace kib
