// C ABI of the B200 solver (declarations and reference citations in
// include/kinterp.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/kinterp.h"
#include "ki_kernels.h"
#include "ki_solver.h"

struct ki_solver_s {
  std::unique_ptr<kib::Solver> solver;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  double* d_io = nullptr;  // staging for host-buffer calls
  size_t io_bytes = 0;
  bool tree_only = false;  // ki_partition handle: no factors on the device
  bool geom_only = false;  // ki_geometry handle: device boundary arrays only
  ~ki_solver_s() {
    solver.reset();  // synchronises the stream: nothing queued uses d_io
    if (d_io) kib::chunk_pool::put(d_io, io_bytes, false);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

namespace {

thread_local std::string g_err;

int set_err(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int from_solver(ki_solver_t s, int rc) {
  if (rc == 0) return KI_OK;
  return set_err(rc == -2 ? KI_ERR_CUDA : KI_ERR_NUMERIC, s->solver->error);
}

int staging(ki_solver_t s, size_t bytes) {
  // device staging of the host-buffer calls, from the process-wide chunk
  // cache (a fresh handle per solve then costs no cudaMalloc / cudaFree)
  if (bytes <= s->io_bytes) return KI_OK;
  if (s->d_io) {
    const cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return set_err(KI_ERR_CUDA, cudaGetErrorString(e));
    kib::chunk_pool::put(s->d_io, s->io_bytes, false);
  }
  s->d_io = nullptr;
  s->io_bytes = 0;
  size_t got = 0;
  void* p = kib::chunk_pool::get(bytes, false, &got);
  if (!p) return set_err(KI_ERR_CUDA, "device staging allocation failed");
  s->d_io = static_cast<double*>(p);
  s->io_bytes = got;
  return KI_OK;
}

int cuda_err(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return KI_OK;
  return set_err(KI_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define KI_TRY(expr)               \
  do {                             \
    const int rc_ = (expr);        \
    if (rc_ != KI_OK) return rc_;  \
  } while (0)

bool box_ref(ki_solver_t s, int level, int idx, const kib::Box** out, int* parent_idx) {
  if (!s || !s->solver) return false;
  s->solver->tree.materialize_originals();
  const auto& lv = s->solver->tree.levels;
  if (level < 0 || level >= static_cast<int>(lv.size())) return false;
  if (idx < 0 || idx >= static_cast<int>(lv[level].size())) return false;
  const int id = lv[level][idx];
  *out = &s->solver->tree.boxes[id];
  *parent_idx = -1;
  const int par = (*out)->parent;
  if (par >= 0) {
    const auto& pl = lv[level - 1];
    for (size_t i = 0; i < pl.size(); i++)
      if (pl[i] == par) *parent_idx = static_cast<int>(i);
  }
  return true;
}

// Every value finite (NaN and infinities fail): boundary data with a
// non-finite value would only surface as NaN factors.
bool all_finite(const double* a, size_t n) {
  bool ok = true;
  for (size_t i = 0; i < n; i++) ok &= std::isfinite(a[i]);
  return ok;
}

bool geometry_finite(int n_points, const double* points, const double* normals,
                     const double* curvatures, const double* weights) {
  const size_t n = static_cast<size_t>(n_points);
  return all_finite(points, 2 * n) && all_finite(normals, 2 * n) && all_finite(curvatures, n) &&
         all_finite(weights, n);
}

int factor_impl(int pde, int n_points, const double* points, const double* normals,
                const double* curvatures, const double* weights, int n_holes,
                const double* holes, int max_leaf_dofs, double id_tol, void* stream,
                ki_solver_t* out, bool timed, const std::vector<int>* starts = nullptr,
                int mode = KI_MODE_REFERENCE) {
  if (!out) return set_err(KI_ERR_ARG, "ki_factor: out is NULL");
  *out = nullptr;
  if (pde < KI_LAPLACE || pde > KI_STOKES) return set_err(KI_ERR_ARG, "ki_factor: bad pde");
  if (n_points <= 0 || !points || !normals || !curvatures || !weights)
    return set_err(KI_ERR_ARG, "number of boundary points to init tree cannot be 0");
  if (n_holes < 0 || (n_holes > 0 && !holes)) return set_err(KI_ERR_ARG, "ki_factor: bad holes");
  if (max_leaf_dofs < 1) return set_err(KI_ERR_ARG, "ki_factor: max_leaf_dofs must be >= 1");
  if (!geometry_finite(n_points, points, normals, curvatures, weights) ||
      (n_holes > 0 && !all_finite(holes, 4 * static_cast<size_t>(n_holes))))
    return set_err(KI_ERR_ARG, "ki_factor: non-finite boundary data (NaN or infinity)");
  if (!(id_tol > 0)) return set_err(KI_ERR_ARG, "id_tol must be greater than 0");
  if (mode != KI_MODE_REFERENCE && mode != KI_MODE_PRECONDITIONER)
    return set_err(KI_ERR_ARG, "ki_factor: bad mode");
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
    return set_err(KI_ERR_CUDA, "no CUDA device available");
  std::unique_ptr<ki_solver_s> h(new (std::nothrow) ki_solver_s());
  if (!h) return set_err(KI_ERR_ARG, "out of host memory");
  if (stream) {
    h->stream = static_cast<cudaStream_t>(stream);
  } else {
    KI_TRY(cuda_err(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking),
                    "cudaStreamCreate"));
    h->own_stream = true;
  }
  kib::SolverOptions opt;
  opt.pde = pde;
  opt.max_leaf_dofs = max_leaf_dofs;
  opt.id_tol = id_tol;
  opt.sketch_id = mode == KI_MODE_PRECONDITIONER;
  opt.proxy_shift = opt.sketch_id ? 1 : 0;  // 64 proxy points for sketched boxes
  opt.top_keep_max = opt.sketch_id ? kib::kLuFusedMaxN : 0;
  h->solver.reset(new kib::Solver(opt, n_points, points, normals, curvatures, weights, n_holes,
                                  holes, h->stream));
  h->solver->time_phases = timed;
  if (starts) h->solver->set_forest(*starts);
  const int rc = h->solver->factor();
  if (rc) return from_solver(h.get(), rc);
  *out = h.release();
  return KI_OK;
}

}  // namespace

extern "C" {

const char* ki_last_error(void) { return g_err.c_str(); }

int ki_version(void) { return 100; }

long long ki_kernel_launches(void) { return kib::launch_total(); }

long long ki_cached_bytes(void) { return static_cast<long long>(kib::chunk_pool::cached_bytes()); }

void ki_release_cache(void) { kib::chunk_pool::release_all(); }

int ki_factor(int pde, int n_points, const double* points, const double* normals,
              const double* curvatures, const double* weights, int n_holes,
              const double* holes, int max_leaf_dofs, double id_tol, void* stream,
              ki_solver_t* out) {
  return factor_impl(pde, n_points, points, normals, curvatures, weights, n_holes, holes,
                     max_leaf_dofs, id_tol, stream, out, false);
}

int ki_factor_timed(int pde, int n_points, const double* points, const double* normals,
                    const double* curvatures, const double* weights, int n_holes,
                    const double* holes, int max_leaf_dofs, double id_tol, void* stream,
                    ki_solver_t* out) {
  return factor_impl(pde, n_points, points, normals, curvatures, weights, n_holes, holes,
                     max_leaf_dofs, id_tol, stream, out, true);
}

int ki_factor_ex(int pde, int n_points, const double* points, const double* normals,
                 const double* curvatures, const double* weights, int n_holes,
                 const double* holes, int max_leaf_dofs, double id_tol, int mode, int timed,
                 void* stream, ki_solver_t* out) {
  return factor_impl(pde, n_points, points, normals, curvatures, weights, n_holes, holes,
                     max_leaf_dofs, id_tol, stream, out, timed != 0, nullptr, mode);
}

int ki_factor_batch(int pde, int n_problems, const int* n_points, const double* points,
                    const double* normals, const double* curvatures, const double* weights,
                    int max_leaf_dofs, double id_tol, int mode, void* stream, ki_solver_t* out) {
  if (!out) return set_err(KI_ERR_ARG, "ki_factor_batch: out is NULL");
  *out = nullptr;
  if (n_problems < 1 || !n_points) return set_err(KI_ERR_ARG, "ki_factor_batch: no problems");
  std::vector<int> starts(1, 0);
  long long total = 0;
  for (int p = 0; p < n_problems; p++) {
    if (n_points[p] <= 0)
      return set_err(KI_ERR_ARG, "number of boundary points to init tree cannot be 0");
    total += n_points[p];
    if (total > (1LL << 30)) return set_err(KI_ERR_ARG, "ki_factor_batch: too many points");
    starts.push_back(static_cast<int>(total));
  }
  return factor_impl(pde, static_cast<int>(total), points, normals, curvatures, weights, 0,
                     nullptr, max_leaf_dofs, id_tol, stream, out, false, &starts, mode);
}

int ki_num_problems(ki_solver_t s) { return s && s->solver ? s->solver->n_trees() : -KI_ERR_ARG; }

int ki_box_tree(ki_solver_t s, int level, int idx) {
  const kib::Box* b;
  int par;
  if (!box_ref(s, level, idx, &b, &par)) return -set_err(KI_ERR_ARG, "ki_box_tree: bad box");
  return b->tree;
}

int ki_partition(int n_points, const double* points, int sol_dim, int max_leaf_dofs,
                 ki_solver_t* out) {
  if (!out) return set_err(KI_ERR_ARG, "ki_partition: out is NULL");
  *out = nullptr;
  if (n_points <= 0 || !points)
    return set_err(KI_ERR_ARG, "number of boundary points to init tree cannot be 0");
  if (sol_dim != 1 && sol_dim != 2) return set_err(KI_ERR_ARG, "ki_partition: sol_dim must be 1 or 2");
  if (max_leaf_dofs < 1) return set_err(KI_ERR_ARG, "ki_partition: max_leaf_dofs must be >= 1");
  std::unique_ptr<ki_solver_s> h(new (std::nothrow) ki_solver_s());
  if (!h) return set_err(KI_ERR_ARG, "out of host memory");
  kib::SolverOptions opt;
  opt.pde = sol_dim == 2 ? KI_STOKES : KI_LAPLACE;
  opt.max_leaf_dofs = max_leaf_dofs;
  std::vector<double> zeros(2 * static_cast<size_t>(n_points), 0.0);
  h->solver.reset(new kib::Solver(opt, n_points, points, zeros.data(), zeros.data(),
                                  zeros.data(), 0, nullptr, nullptr));
  h->solver->build_tree_only();
  h->tree_only = true;
  *out = h.release();
  return KI_OK;
}

int ki_partition_update(ki_solver_t s, int n_points, const double* points) {
  if (!s || !s->solver || !s->tree_only)
    return set_err(KI_ERR_ARG, "ki_partition_update: needs a ki_partition handle");
  if (n_points <= 0 || !points)
    return set_err(KI_ERR_ARG, "number of boundary points to init tree cannot be 0");
  if (s->solver->n_trees() > 1)
    return set_err(KI_ERR_ARG, "ki_partition_update: not available for a batch of problems");
  s->solver->perturb_tree_only(n_points, points);
  return KI_OK;
}

int ki_partition_batch(int n_problems, const int* n_points, const double* points, int sol_dim,
                       int max_leaf_dofs, ki_solver_t* out) {
  if (!out) return set_err(KI_ERR_ARG, "ki_partition_batch: out is NULL");
  *out = nullptr;
  if (n_problems < 1 || !n_points || !points)
    return set_err(KI_ERR_ARG, "ki_partition_batch: no problems");
  if (sol_dim != 1 && sol_dim != 2)
    return set_err(KI_ERR_ARG, "ki_partition_batch: sol_dim must be 1 or 2");
  if (max_leaf_dofs < 1) return set_err(KI_ERR_ARG, "ki_partition_batch: max_leaf_dofs must be >= 1");
  std::vector<int> starts(1, 0);
  long long total = 0;
  for (int p = 0; p < n_problems; p++) {
    if (n_points[p] <= 0)
      return set_err(KI_ERR_ARG, "number of boundary points to init tree cannot be 0");
    total += n_points[p];
    if (total > (1LL << 30)) return set_err(KI_ERR_ARG, "ki_partition_batch: too many points");
    starts.push_back(static_cast<int>(total));
  }
  std::unique_ptr<ki_solver_s> h(new (std::nothrow) ki_solver_s());
  if (!h) return set_err(KI_ERR_ARG, "out of host memory");
  kib::SolverOptions opt;
  opt.pde = sol_dim == 2 ? KI_STOKES : KI_LAPLACE;
  opt.max_leaf_dofs = max_leaf_dofs;
  const int n = static_cast<int>(total);
  std::vector<double> zeros(2 * static_cast<size_t>(n), 0.0);
  h->solver.reset(new kib::Solver(opt, n, points, zeros.data(), zeros.data(), zeros.data(), 0,
                                  nullptr, nullptr));
  h->solver->set_forest(starts);
  h->solver->build_tree_only();
  h->tree_only = true;
  *out = h.release();
  return KI_OK;
}

int ki_update(ki_solver_t s, int n_points, const double* points, const double* normals,
              const double* curvatures, const double* weights, int n_holes, const double* holes,
              int* n_reused) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver) return set_err(KI_ERR_ARG, "ki_update: bad handle");
  if (n_points <= 0 || !points || !normals || !curvatures || !weights)
    return set_err(KI_ERR_ARG, "number of boundary points to init tree cannot be 0");
  if (n_holes < 0 || (n_holes > 0 && !holes)) return set_err(KI_ERR_ARG, "ki_update: bad holes");
  if (!geometry_finite(n_points, points, normals, curvatures, weights) ||
      (n_holes > 0 && !all_finite(holes, 4 * static_cast<size_t>(n_holes))))
    return set_err(KI_ERR_ARG, "ki_update: non-finite boundary data (NaN or infinity)");
  if (s->solver->n_trees() > 1)
    return set_err(KI_ERR_ARG, "ki_update: not available for a batch of problems");
  return from_solver(s, s->solver->update(n_points, points, normals, curvatures, weights,
                                          n_holes, holes, n_reused));
}

int ki_copy(ki_solver_t s, void* stream, ki_solver_t* out) {
  if (!out) return set_err(KI_ERR_ARG, "ki_copy: out is NULL");
  *out = nullptr;
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver) return set_err(KI_ERR_ARG, "ki_copy: bad handle");
  if (s->solver->n_trees() > 1)
    return set_err(KI_ERR_ARG, "ki_copy: not available for a batch of problems");
  std::unique_ptr<ki_solver_s> h(new (std::nothrow) ki_solver_s());
  if (!h) return set_err(KI_ERR_ARG, "out of host memory");
  if (stream) {
    h->stream = static_cast<cudaStream_t>(stream);
  } else {
    KI_TRY(cuda_err(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking),
                    "cudaStreamCreate"));
    h->own_stream = true;
  }
  int rc = 0;
  kib::Solver* c = s->solver->copy(h->stream, &rc);
  if (!c) return set_err(rc == -2 ? KI_ERR_CUDA : KI_ERR_NUMERIC, s->solver->error);
  h->solver.reset(c);
  *out = h.release();
  return KI_OK;
}

void ki_destroy(ki_solver_t s) { delete s; }

int ki_num_dofs(ki_solver_t s) { return s && s->solver ? s->solver->n_dofs() : -KI_ERR_ARG; }

int ki_num_border(ki_solver_t s) { return s && s->solver ? s->solver->n_border() : -KI_ERR_ARG; }

int ki_solve_device(ki_solver_t s, const double* d_f, double* d_mu, double* d_alpha) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || !d_f || !d_mu) return set_err(KI_ERR_ARG, "ki_solve_device: bad args");
  if (s->solver->n_border() > 0 && !d_alpha)
    return set_err(KI_ERR_ARG, "ki_solve_device: alpha required for a domain with holes");
  return from_solver(s, s->solver->solve_device(d_f, d_mu, d_alpha));
}

int ki_solve(ki_solver_t s, const double* f, double* mu, double* alpha) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || !f || !mu) return set_err(KI_ERR_ARG, "ki_solve: bad args");
  const int N = s->solver->n_dofs(), nb = s->solver->n_border();
  if (nb > 0 && !alpha) return set_err(KI_ERR_ARG, "ki_solve: alpha required for a domain with holes");
  KI_TRY(staging(s, sizeof(double) * (N + nb + 1)));
  double* d_x = s->d_io;
  double* d_a = d_x + N;
  KI_TRY(cuda_err(cudaMemcpyAsync(d_x, f, sizeof(double) * N, cudaMemcpyHostToDevice, s->stream),
                  "copy f"));
  KI_TRY(from_solver(s, s->solver->solve_device(d_x, d_x, nb ? d_a : nullptr)));
  KI_TRY(cuda_err(cudaMemcpyAsync(mu, d_x, sizeof(double) * N, cudaMemcpyDeviceToHost, s->stream),
                  "copy mu"));
  if (nb > 0)
    KI_TRY(cuda_err(cudaMemcpyAsync(alpha, d_a, sizeof(double) * nb, cudaMemcpyDeviceToHost,
                                    s->stream),
                    "copy alpha"));
  return cuda_err(cudaStreamSynchronize(s->stream), "ki_solve");
}

int ki_solve_bordered_device(ki_solver_t s, const double* d_f, const double* d_g, double* d_mu,
                             double* d_alpha) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || !d_f || !d_mu) return set_err(KI_ERR_ARG, "ki_solve_bordered_device: bad args");
  if (s->solver->n_border() > 0 && !d_alpha)
    return set_err(KI_ERR_ARG, "ki_solve_bordered_device: alpha required for a domain with holes");
  return from_solver(s, s->solver->solve_device(d_f, d_mu, d_alpha,
                                                s->solver->n_border() ? d_g : nullptr));
}

int ki_solve_refined_device(ki_solver_t s, const double* d_f, double* d_mu, double* d_alpha,
                            double rel_tol, int max_iters, int* iters, double* rel_res) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || !d_f || !d_mu || !(rel_tol >= 0.0) || max_iters < 1)
    return set_err(KI_ERR_ARG, "ki_solve_refined_device: bad args");
  if (s->solver->n_border() > 0 && !d_alpha)
    return set_err(KI_ERR_ARG, "ki_solve_refined_device: alpha required for a domain with holes");
  return from_solver(s, s->solver->solve_refined(d_f, d_mu, d_alpha, rel_tol, max_iters, iters,
                                                 rel_res));
}

int ki_solve_refined(ki_solver_t s, const double* f, double* mu, double* alpha, double rel_tol,
                     int max_iters, int* iters, double* rel_res) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || !f || !mu || !(rel_tol >= 0.0) || max_iters < 1)
    return set_err(KI_ERR_ARG, "ki_solve_refined: bad args");
  const int N = s->solver->n_dofs(), nb = s->solver->n_border();
  if (nb > 0 && !alpha)
    return set_err(KI_ERR_ARG, "ki_solve_refined: alpha required for a domain with holes");
  KI_TRY(staging(s, sizeof(double) * (2 * static_cast<size_t>(N) + nb + 1)));
  double* d_f = s->d_io;
  double* d_x = d_f + N;
  double* d_a = d_x + N;
  KI_TRY(cuda_err(cudaMemcpyAsync(d_f, f, sizeof(double) * N, cudaMemcpyHostToDevice, s->stream),
                  "copy f"));
  KI_TRY(from_solver(s, s->solver->solve_refined(d_f, d_x, nb ? d_a : nullptr, rel_tol,
                                                 max_iters, iters, rel_res)));
  KI_TRY(cuda_err(cudaMemcpyAsync(mu, d_x, sizeof(double) * N, cudaMemcpyDeviceToHost, s->stream),
                  "copy mu"));
  if (nb > 0)
    KI_TRY(cuda_err(cudaMemcpyAsync(alpha, d_a, sizeof(double) * nb, cudaMemcpyDeviceToHost,
                                    s->stream),
                    "copy alpha"));
  return cuda_err(cudaStreamSynchronize(s->stream), "ki_solve_refined");
}

int ki_matvec_device(ki_solver_t s, const double* d_x, double* d_y) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || !d_x || !d_y) return set_err(KI_ERR_ARG, "ki_matvec_device: bad args");
  return from_solver(s, s->solver->matvec_device(d_x, d_y));
}

int ki_matvec_correction_device(ki_solver_t s, const double* d_x, double* d_y, double dscale) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || !d_x || !d_y || !(dscale > 0.0))
    return set_err(KI_ERR_ARG, "ki_matvec_correction_device: bad args");
  return from_solver(s, s->solver->corr_matvec_device(d_x, d_y, dscale));
}

int ki_solve_transpose_device(ki_solver_t s, const double* d_b, double* d_x) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || !d_b || !d_x) return set_err(KI_ERR_ARG, "ki_solve_transpose_device: bad args");
  if (s->solver->n_border() > 0)
    return set_err(KI_ERR_ARG, "ki_solve_transpose_device: domains with holes are not supported");
  return from_solver(s, s->solver->solve_transpose_device(d_b, d_x));
}

int ki_eval_targets_device(ki_solver_t s, int n_targets, const double* d_targets,
                           const double* d_mu, const double* d_alpha, double* d_out) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || n_targets < 0 || (n_targets > 0 && (!d_targets || !d_out)) || !d_mu)
    return set_err(KI_ERR_ARG, "ki_eval_targets_device: bad args");
  if (n_targets == 0) return KI_OK;
  if (s->solver->n_trees() > 1)
    return set_err(KI_ERR_ARG, "ki_eval_targets_device: not available for a batch of problems");
  kib::Solver& sv = *s->solver;
  const bool use_alpha = sv.n_border() > 0 && d_alpha;
  return cuda_err(kib::launch_eval_targets(sv.pde(), sv.d_nodes(), sv.n_dofs(), n_targets,
                                           d_targets, d_mu, sv.n_holes(), sv.d_holes(),
                                           use_alpha ? d_alpha : nullptr, d_out, s->stream),
                  "ki_eval_targets_device");
}

int ki_adjoint_forward(ki_solver_t s, const double* d_f, int n_targets, const double* d_targets,
                       double* d_mu, double* d_u) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || !d_f || !d_mu || n_targets < 0 || (n_targets > 0 && (!d_targets || !d_u)))
    return set_err(KI_ERR_ARG, "ki_adjoint_forward: bad args");
  if (s->solver->pde() != KI_LAPLACE || s->solver->n_border() > 0)
    return set_err(KI_ERR_ARG,
                   "ki_adjoint_forward: only the Laplace double layer on a simply connected domain");
  KI_TRY(from_solver(s, s->solver->solve_device(d_f, d_mu, nullptr)));
  return ki_eval_targets_device(s, n_targets, d_targets, d_mu, nullptr, d_u);
}

int ki_adjoint_backward(ki_solver_t s, int n_targets, const double* d_targets, const double* d_mu,
                        const double* d_grad_u, double* d_grad_f, double* d_grad_points,
                        double* d_grad_normals, double* d_grad_weights,
                        double* d_grad_curvatures) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || n_targets < 0 || (n_targets > 0 && (!d_targets || !d_grad_u)) ||
      !d_mu || !d_grad_f || !d_grad_points || !d_grad_normals || !d_grad_weights ||
      !d_grad_curvatures)
    return set_err(KI_ERR_ARG, "ki_adjoint_backward: bad args");
  if (s->solver->pde() != KI_LAPLACE || s->solver->n_border() > 0)
    return set_err(KI_ERR_ARG,
                   "ki_adjoint_backward: only the Laplace double layer on a simply connected domain");
  return from_solver(s, s->solver->adjoint_backward(n_targets, d_targets, d_mu, d_grad_u,
                                                    d_grad_f, d_grad_points, d_grad_normals,
                                                    d_grad_weights, d_grad_curvatures));
}

int ki_apply_device(ki_solver_t s, const double* d_x, double* d_y) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || !d_x || !d_y) return set_err(KI_ERR_ARG, "ki_apply_device: bad args");
  return from_solver(s, s->solver->apply_device(d_x, d_y));
}

int ki_eval_targets(ki_solver_t s, int n_targets, const double* targets, const double* mu,
                    const double* alpha, double* out) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || n_targets < 0 || (n_targets > 0 && (!targets || !out)) || !mu)
    return set_err(KI_ERR_ARG, "ki_eval_targets: bad args");
  if (n_targets == 0) return KI_OK;
  if (s->solver->n_trees() > 1)
    return set_err(KI_ERR_ARG, "ki_eval_targets: not available for a batch of problems");
  kib::Solver& sv = *s->solver;
  const int N = sv.n_dofs(), nb = sv.n_border(), sd = sv.sol_dim();
  const bool use_alpha = nb > 0 && alpha;
  const size_t need = static_cast<size_t>(N) + nb + 2 * static_cast<size_t>(n_targets) +
                      static_cast<size_t>(sd) * n_targets;
  KI_TRY(staging(s, sizeof(double) * need));
  double* d_mu = s->d_io;
  double* d_al = d_mu + N;
  double* d_tg = d_al + nb;
  double* d_out = d_tg + 2 * static_cast<size_t>(n_targets);
  KI_TRY(cuda_err(cudaMemcpyAsync(d_mu, mu, sizeof(double) * N, cudaMemcpyHostToDevice, s->stream),
                  "copy mu"));
  if (use_alpha)
    KI_TRY(cuda_err(cudaMemcpyAsync(d_al, alpha, sizeof(double) * nb, cudaMemcpyHostToDevice,
                                    s->stream),
                    "copy alpha"));
  KI_TRY(cuda_err(cudaMemcpyAsync(d_tg, targets, sizeof(double) * 2 * n_targets,
                                  cudaMemcpyHostToDevice, s->stream),
                  "copy targets"));
  KI_TRY(cuda_err(kib::launch_eval_targets(sv.pde(), sv.d_nodes(), N, n_targets, d_tg, d_mu,
                                           sv.n_holes(), sv.d_holes(),
                                           use_alpha ? d_al : nullptr, d_out, s->stream),
                  "eval targets"));
  KI_TRY(cuda_err(cudaMemcpyAsync(out, d_out, sizeof(double) * sd * n_targets,
                                  cudaMemcpyDeviceToHost, s->stream),
                  "copy out"));
  return cuda_err(cudaStreamSynchronize(s->stream), "ki_eval_targets");
}

static int domain_args(ki_solver_t s, int n_targets, int kind, const double* disk,
                       const char* who) {
  if (s && s->tree_only) return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || n_targets < 0)
    return set_err(KI_ERR_ARG, std::string(who) + ": bad args");
  if (kind != KI_DOMAIN_ALL && kind != KI_DOMAIN_NODES && kind != KI_DOMAIN_DISK)
    return set_err(KI_ERR_ARG, std::string(who) + ": unknown domain test");
  if (kind == KI_DOMAIN_DISK && !disk)
    return set_err(KI_ERR_ARG, std::string(who) + ": the disk test needs {cx, cy, R}");
  if (s->solver->n_trees() > 1)
    return set_err(KI_ERR_ARG, std::string(who) + ": not available for a batch of problems");
  return KI_OK;
}

int ki_eval_domain_device(ki_solver_t s, int n_targets, const double* d_targets,
                          const double* d_mu, const double* d_alpha, int kind, const double* disk,
                          double* d_out) {
  KI_TRY(domain_args(s, n_targets, kind, disk, "ki_eval_domain_device"));
  if (n_targets == 0) return KI_OK;
  if (!d_targets || !d_mu || !d_out)
    return set_err(KI_ERR_ARG, "ki_eval_domain_device: bad args");
  return from_solver(s, s->solver->eval_domain(n_targets, d_targets, d_mu, d_alpha, kind, disk,
                                               d_out));
}

int ki_domain_mask_device(ki_solver_t s, int n_targets, const double* d_targets, int kind,
                          const double* disk, unsigned char* d_mask) {
  KI_TRY(domain_args(s, n_targets, kind, disk, "ki_domain_mask_device"));
  if (kind == KI_DOMAIN_ALL)
    return set_err(KI_ERR_ARG, "ki_domain_mask_device: needs KI_DOMAIN_NODES or KI_DOMAIN_DISK");
  if (n_targets == 0) return KI_OK;
  if (!d_targets || !d_mask) return set_err(KI_ERR_ARG, "ki_domain_mask_device: bad args");
  return from_solver(s, s->solver->domain_mask(n_targets, d_targets, kind, disk, d_mask));
}

int ki_eval_domain(ki_solver_t s, int n_targets, const double* targets, const double* mu,
                   const double* alpha, int kind, const double* disk, double* out) {
  KI_TRY(domain_args(s, n_targets, kind, disk, "ki_eval_domain"));
  if (n_targets == 0) return KI_OK;
  if (!targets || !mu || !out) return set_err(KI_ERR_ARG, "ki_eval_domain: bad args");
  kib::Solver& sv = *s->solver;
  const int N = sv.n_dofs(), nb = sv.n_border(), sd = sv.sol_dim();
  const bool use_alpha = nb > 0 && alpha;
  const size_t need = static_cast<size_t>(N) + nb + 2 * static_cast<size_t>(n_targets) +
                      static_cast<size_t>(sd) * n_targets;
  KI_TRY(staging(s, sizeof(double) * need));
  double* d_mu = s->d_io;
  double* d_al = d_mu + N;
  double* d_tg = d_al + nb;
  double* d_out = d_tg + 2 * static_cast<size_t>(n_targets);
  KI_TRY(cuda_err(cudaMemcpyAsync(d_mu, mu, sizeof(double) * N, cudaMemcpyHostToDevice, s->stream),
                  "copy mu"));
  if (use_alpha)
    KI_TRY(cuda_err(cudaMemcpyAsync(d_al, alpha, sizeof(double) * nb, cudaMemcpyHostToDevice,
                                    s->stream),
                    "copy alpha"));
  KI_TRY(cuda_err(cudaMemcpyAsync(d_tg, targets, sizeof(double) * 2 * n_targets,
                                  cudaMemcpyHostToDevice, s->stream),
                  "copy targets"));
  KI_TRY(from_solver(s, sv.eval_domain(n_targets, d_tg, d_mu, use_alpha ? d_al : nullptr, kind,
                                       disk, d_out)));
  KI_TRY(cuda_err(cudaMemcpyAsync(out, d_out, sizeof(double) * sd * n_targets,
                                  cudaMemcpyDeviceToHost, s->stream),
                  "copy out"));
  return cuda_err(cudaStreamSynchronize(s->stream), "ki_eval_domain");
}

int ki_domain_points(int domain_size, double x_min, double x_max, double y_min, double y_max,
                     double* points) {
  if (domain_size < 0 || (domain_size > 0 && !points))
    return set_err(KI_ERR_ARG, "ki_domain_points: bad args");
  size_t k = 0;
  for (int i = 0; i < domain_size; i++) {
    const double x = x_min + ((i + 0.0) / (domain_size - 1)) * (x_max - x_min);
    for (int j = 0; j < domain_size; j++) {
      points[k++] = x;
      points[k++] = y_min + ((j + 0.0) / (domain_size - 1)) * (y_max - y_min);
    }
  }
  return KI_OK;
}

int ki_test_inject_fault(int what) {
  if (what < KI_INJECT_NONE || what > KI_INJECT_LU_STALL)
    return set_err(KI_ERR_ARG, "ki_test_inject_fault: unknown fault");
  kib::inject_lu_fault(what);
  return KI_OK;
}

int ki_geometry(int pde, int n_points, const double* points, const double* normals,
                const double* curvatures, const double* weights, void* stream,
                ki_solver_t* out) {
  if (!out) return set_err(KI_ERR_ARG, "ki_geometry: out is NULL");
  *out = nullptr;
  if (pde < KI_LAPLACE || pde > KI_STOKES) return set_err(KI_ERR_ARG, "ki_geometry: bad pde");
  if (n_points <= 0 || !points || !normals || !curvatures || !weights)
    return set_err(KI_ERR_ARG, "ki_geometry: no boundary points");
  if (!geometry_finite(n_points, points, normals, curvatures, weights))
    return set_err(KI_ERR_ARG, "ki_geometry: non-finite boundary data (NaN or infinity)");
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
    return set_err(KI_ERR_CUDA, "no CUDA device available");
  std::unique_ptr<ki_solver_s> h(new (std::nothrow) ki_solver_s());
  if (!h) return set_err(KI_ERR_ARG, "out of host memory");
  if (stream) {
    h->stream = static_cast<cudaStream_t>(stream);
  } else {
    KI_TRY(cuda_err(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking),
                    "cudaStreamCreate"));
    h->own_stream = true;
  }
  kib::SolverOptions opt;
  opt.pde = pde;
  h->solver.reset(new kib::Solver(opt, n_points, points, normals, curvatures, weights, 0,
                                  nullptr, h->stream));
  const int rc = h->solver->prepare_geometry();
  if (rc) return from_solver(h.get(), rc);
  h->tree_only = true;
  h->geom_only = true;
  *out = h.release();
  return KI_OK;
}

int ki_forward_block(ki_solver_t s, int n_targets, const double* targets, int nt, const int* tgt,
                     int ns, const int* src, double* out) {
  if (s && s->tree_only && !s->geom_only)
    return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || n_targets < 0 || nt < 0 || ns < 0 ||
      (nt * ns > 0 && (!tgt || !src || !out || !targets)))
    return set_err(KI_ERR_ARG, "ki_forward_block: bad args");
  if (nt == 0 || ns == 0) return KI_OK;
  const int N = s->solver->n_dofs();
  const int sd = s->solver->pde() == KI_STOKES ? 2 : 1;
  for (int i = 0; i < nt; i++)
    if (tgt[i] < 0 || tgt[i] >= sd * n_targets)
      return set_err(KI_ERR_ARG, "ki_forward_block: tgt out of range");
  for (int j = 0; j < ns; j++)
    if (src[j] < 0 || src[j] >= N) return set_err(KI_ERR_ARG, "ki_forward_block: src out of range");
  const size_t ints = static_cast<size_t>(nt) + ns;
  const size_t need = sizeof(double) * (static_cast<size_t>(nt) * ns + 2 * n_targets) +
                      sizeof(int) * ints + 64;
  KI_TRY(staging(s, need));
  double* d_out = s->d_io;
  double* d_tp = d_out + static_cast<size_t>(nt) * ns;
  int* d_t = reinterpret_cast<int*>(d_tp + 2 * static_cast<size_t>(n_targets));
  int* d_s = d_t + nt;
  KI_TRY(cuda_err(cudaMemcpyAsync(d_tp, targets, sizeof(double) * 2 * n_targets,
                                  cudaMemcpyHostToDevice, s->stream), "copy"));
  KI_TRY(cuda_err(cudaMemcpyAsync(d_t, tgt, sizeof(int) * nt, cudaMemcpyHostToDevice, s->stream), "copy"));
  KI_TRY(cuda_err(cudaMemcpyAsync(d_s, src, sizeof(int) * ns, cudaMemcpyHostToDevice, s->stream), "copy"));
  KI_TRY(cuda_err(kib::launch_forward_block(s->solver->pde(), s->solver->d_nodes(), d_tp, d_t,
                                            nt, d_s, ns, d_out, s->stream),
                  "forward block"));
  KI_TRY(cuda_err(cudaMemcpyAsync(out, d_out, sizeof(double) * nt * ns, cudaMemcpyDeviceToHost,
                                  s->stream),
                  "copy out"));
  return cuda_err(cudaStreamSynchronize(s->stream), "ki_forward_block");
}

int ki_kernel_block(ki_solver_t s, int nt, const int* tgt, int ns, const int* src, double* out) {
  if (s && s->tree_only && !s->geom_only)
    return set_err(KI_ERR_STATE, "handle holds a partition only");
  if (!s || !s->solver || nt < 0 || ns < 0 || (nt * ns > 0 && (!tgt || !src || !out)))
    return set_err(KI_ERR_ARG, "ki_kernel_block: bad args");
  if (nt == 0 || ns == 0) return KI_OK;
  const int N = s->solver->n_dofs();
  for (int i = 0; i < nt; i++)
    if (tgt[i] < 0 || tgt[i] >= N) return set_err(KI_ERR_ARG, "ki_kernel_block: tgt out of range");
  for (int j = 0; j < ns; j++)
    if (src[j] < 0 || src[j] >= N) return set_err(KI_ERR_ARG, "ki_kernel_block: src out of range");
  const size_t ints = static_cast<size_t>(nt) + ns;
  const size_t need = sizeof(double) * static_cast<size_t>(nt) * ns + sizeof(int) * ints + 64;
  KI_TRY(staging(s, need));
  double* d_out = s->d_io;
  int* d_t = reinterpret_cast<int*>(d_out + static_cast<size_t>(nt) * ns);
  int* d_s = d_t + nt;
  KI_TRY(cuda_err(cudaMemcpyAsync(d_t, tgt, sizeof(int) * nt, cudaMemcpyHostToDevice, s->stream), "copy"));
  KI_TRY(cuda_err(cudaMemcpyAsync(d_s, src, sizeof(int) * ns, cudaMemcpyHostToDevice, s->stream), "copy"));
  KI_TRY(cuda_err(kib::launch_kernel_block(s->solver->pde(), s->solver->d_nodes(), d_t, nt, d_s, ns,
                                           d_out, s->stream),
                  "kernel block"));
  KI_TRY(cuda_err(cudaMemcpyAsync(out, d_out, sizeof(double) * nt * ns, cudaMemcpyDeviceToHost,
                                  s->stream),
                  "copy out"));
  return cuda_err(cudaStreamSynchronize(s->stream), "ki_kernel_block");
}

int ki_num_levels(ki_solver_t s) {
  if (!s || !s->solver) return -KI_ERR_ARG;
  return static_cast<int>(s->solver->tree.levels.size());
}

int ki_num_boxes(ki_solver_t s, int level) {
  if (!s || !s->solver || level < 0 ||
      level >= static_cast<int>(s->solver->tree.levels.size()))
    return -KI_ERR_ARG;
  return static_cast<int>(s->solver->tree.levels[level].size());
}

int ki_box_info(ki_solver_t s, int level, int idx, int* info, double* geom) {
  const kib::Box* b;
  int par;
  if (!box_ref(s, level, idx, &b, &par) || !info) return set_err(KI_ERR_ARG, "ki_box_info: bad box");
  info[0] = b->leaf;
  info[1] = b->compressed;
  info[2] = static_cast<int>(b->original.size());
  info[3] = static_cast<int>(b->active.size());
  info[4] = static_cast<int>(b->skel.size());
  info[5] = static_cast<int>(b->redundant.size());
  info[6] = par;
  info[7] = b->level;
  if (geom) {
    geom[0] = b->corner[0];
    geom[1] = b->corner[1];
    geom[2] = b->side;
  }
  return KI_OK;
}

int ki_box_lists(ki_solver_t s, int level, int idx, int* original, int* active, int* skel,
                 int* redundant) {
  const kib::Box* b;
  int par;
  if (!box_ref(s, level, idx, &b, &par)) return set_err(KI_ERR_ARG, "ki_box_lists: bad box");
  auto cp = [](const std::vector<int>& v, int* o) {
    if (o && !v.empty()) std::memcpy(o, v.data(), sizeof(int) * v.size());
  };
  cp(b->original, original);
  cp(b->active, active);
  cp(b->skel, skel);
  cp(b->redundant, redundant);
  return KI_OK;
}

int ki_box_neighbors(ki_solver_t s, int level, int idx, int* nbr_level, int* nbr_idx) {
  const kib::Box* b;
  int par;
  if (!box_ref(s, level, idx, &b, &par)) return -set_err(KI_ERR_ARG, "ki_box_neighbors: bad box");
  const auto& lv = s->solver->tree.levels;
  const auto& boxes = s->solver->tree.boxes;
  int q = 0;
  for (int o : b->nbr) {
    const int ol = boxes[o].level;
    int pos = -1;
    for (size_t i = 0; i < lv[ol].size() && pos < 0; i++)
      if (lv[ol][i] == o) pos = static_cast<int>(i);
    if (nbr_level) nbr_level[q] = ol;
    if (nbr_idx) nbr_idx[q] = pos;
    q++;
  }
  return q;
}

int ki_allskel(ki_solver_t s, int* out) {
  if (!s || !s->solver) return -KI_ERR_ARG;
  const auto& v = s->solver->allskel;
  if (out && !v.empty()) std::memcpy(out, v.data(), sizeof(int) * v.size());
  return static_cast<int>(v.size());
}

int ki_launch_log(ki_solver_t s, double* out, int cap) {
  if (!s || !s->solver) return -KI_ERR_ARG;
  const auto& log = s->solver->launch_log;
  for (int i = 0; out && i < cap && i < static_cast<int>(log.size()); i++) {
    const auto& r = log[i];
    const double row[7] = {double(r.level), double(r.kind), double(r.group), double(r.ntasks),
                           double(r.m_cap), double(r.n_cap), r.ms};
    std::memcpy(out + 7 * i, row, sizeof(row));
  }
  return static_cast<int>(log.size());
}

int ki_timeline(ki_solver_t s, double* out, int cap) {
  if (!s || !s->solver) return -KI_ERR_ARG;
  const auto& log = s->solver->launch_log;
  const auto& hm = s->solver->host_marks;
  const int total = static_cast<int>(log.size() + hm.size());
  int i = 0;
  for (const auto& r : log) {
    if (out && i < cap) {
      const double row[4] = {double(r.kind), double(r.level), r.t0, r.t1};
      std::memcpy(out + 4 * i, row, sizeof(row));
    }
    i++;
  }
  for (const auto& m : hm) {
    if (out && i < cap) {
      const double row[4] = {100.0 + m.code, double(m.level), m.ms, m.ms};
      std::memcpy(out + 4 * i, row, sizeof(row));
    }
    i++;
  }
  return total;
}

int ki_stats(ki_solver_t s, double* out, int n) {
  if (!s || !s->solver || !out) return -KI_ERR_ARG;
  const kib::Solver& v = *s->solver;
  const double vals[] = {v.t_factor_ms,    v.t_id_ms,        static_cast<double>(v.id_launches),
                         v.id_flops,       v.id_bytes,       v.t_decouple_ms,
                         v.t_top_ms,       v.t_wait_ms,      v.t_host_prep_ms,
                         v.t_host_post_ms, v.t_upload_ms,    v.t_host_top_ms,
                         v.id_onchip_flops, static_cast<double>(v.staging_bytes()),
                         v.dec_flops,      v.top_flops,      v.solve_bytes};
  const int cnt = n < 17 ? n : 17;
  for (int i = 0; i < cnt; i++) out[i] = vals[i];
  return cnt;
}

int ki_id_noalloc(int pde, const double* d_nodes, int n_points, const int* d_active,
                  int n_active, const int* d_rows, int n_rows, int proxy, double cx,
                  double cy, double radius, double id_tol, int* d_rank, int* d_perm,
                  double* d_T, void* stream) {
  if (pde < KI_LAPLACE || pde > KI_STOKES) return set_err(KI_ERR_ARG, "ki_id_noalloc: bad pde");
  if (!d_nodes || n_points <= 0 || !d_active || n_active <= 0 || n_rows < 0 ||
      (n_rows > 0 && !d_rows) || !d_rank || !d_perm || !d_T)
    return set_err(KI_ERR_ARG, "ki_id_noalloc: bad arguments");
  if (!(id_tol > 0)) return set_err(KI_ERR_ARG, "id_tol must be greater than 0");
  const int proxy_rows = proxy ? (pde == KI_STOKES ? 4 : 2) * kib::kNumProxy : 0;
  const long long m = 2LL * n_rows + proxy_rows;
  if (m == 0) return set_err(KI_ERR_ARG, "ki_id_noalloc: the ID matrix has no rows");
  const long long lda = (m + 3) / 4 * 4;
  if (lda * n_active > kib::kNoAllocScratchDoubles)
    return set_err(KI_ERR_ARG, "ki_id_noalloc: the " + std::to_string(m) + " x " +
                                   std::to_string(n_active) +
                                   " ID matrix exceeds the 8 MiB static scratch "
                                   "(1048576 doubles, rows padded to a multiple of 4)");
  if (kib::id_smem_bytes(static_cast<int>(m), n_active) > 227 * 1024)
    return set_err(KI_ERR_ARG, "ki_id_noalloc: too many rows for the shared staging");
  return cuda_err(kib::launch_id_noalloc(pde, reinterpret_cast<const kib::Node*>(d_nodes),
                                         d_active, n_active, d_rows, n_rows, proxy_rows, cx,
                                         cy, radius, id_tol, d_rank, d_perm, d_T,
                                         static_cast<cudaStream_t>(stream)),
                  "ki_id_noalloc");
}

}  // extern "C"
