// The B200 recursive-skeletonization factorization object.
//
// One Solver holds what the reference spreads over QuadTree (the tree and
// every box's T, L, U, X_rr factors, quadtree.h:44-102) and
// SkelFactorization (skeletonize/solve, skel_factorization.h:19-62): the
// host quadtree and index lists, and device storage for the geometry, the
// per-level factors and the top-level (bordered) skeleton LU.
#ifndef KI_SOLVER_H_
#define KI_SOLVER_H_

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "ki_kernels.h"
#include "ki_tree.h"

namespace kib {

// Process-wide cache of device chunks and pinned host chunks.  A solver
// takes chunks while it factors and hands them back when it is destroyed
// (after its streams are idle), so repeated factorizations neither call
// cudaMalloc/cudaHostAlloc again nor pay cudaFree's device synchronisation.
// Cached memory is kept until ki_release_cache() or process exit.
namespace chunk_pool {
void* get(size_t bytes, bool pinned, size_t* got);
void put(void* p, size_t bytes, bool pinned);
void release_all();
size_t cached_bytes();
}  // namespace chunk_pool

// Bump allocator over pooled chunks (device memory, or pinned host memory
// for upload staging); pointers stay valid until the arena is destroyed.
class Arena {
 public:
  explicit Arena(bool pinned = false) : pinned_(pinned) {}
  ~Arena();
  void* alloc(size_t bytes);
  template <class T>
  T* get(size_t count) { return static_cast<T*>(alloc(sizeof(T) * (count ? count : 1))); }
  size_t reserved() const { return reserved_; }

 private:
  bool pinned_;
  std::vector<std::pair<void*, size_t>> chunks_;
  char* cur_ = nullptr;
  size_t left_ = 0;
  size_t reserved_ = 0;
};

// Reusable device scratch that only grows.
struct Scratch {
  void* p = nullptr;
  size_t bytes = 0;
  ~Scratch();
  cudaError_t reserve(size_t want, cudaStream_t s);
};

struct SolverOptions {
  int pde = 0;              // 0 Laplace, 1 Laplace-Neumann, 2 Stokes
  int max_leaf_dofs = 32;   // MAX_LEAF_DOFS (quadtree.h:10)
  double id_tol = 1e-6;
  int min_dofs_to_compress = 16;  // MIN_DOFS_TO_COMPRESS (skel_factorization.h:11)
};

struct LevelFactors {
  int level = 0;
  int ntasks = 0;
  int cap = 0;
  SweepTask* d_tasks = nullptr;
  std::vector<SweepTask> h_tasks;  // host copy of d_tasks
  int* d_skel = nullptr;
  int* d_red = nullptr;
  std::vector<int> boxes;  // compressed boxes of this level
};

struct BoxBlock {  // accumulated update living at positions [pos, pos + size)
  const double* acc;
  int size;
  int pos;
};

class Solver {
 public:
  Solver(const SolverOptions& opt, int n_points, const double* points,
         const double* normals, const double* curvatures, const double* weights,
         int n_holes, const double* holes, cudaStream_t stream);
  ~Solver();

  // QuadTree::initialize_tree + SkelFactorization::skeletonize.
  int factor();
  // QuadTree::initialize_tree only, active lists as before compression.
  void build_tree_only();
  // linear_solve on device buffers: d_mu (dofs), d_alpha (border, may be
  // null when there are no holes).  d_b and d_mu may be the same buffer.
  int solve_device(const double* d_b, double* d_mu, double* d_alpha);
  // y = A x on device (bordered when there are holes).
  int apply_device(const double* d_x, double* d_y);

  int n_dofs() const { return n_dofs_; }
  int n_border() const { return nb_; }
  int pde() const { return opt_.pde; }
  int sol_dim() const { return sd_; }
  cudaStream_t stream() const { return stream_; }
  const Node* d_nodes() const { return d_nodes_; }
  const double* d_holes() const { return d_holes_; }
  int n_holes() const { return static_cast<int>(holes_.size() / 4); }

  QuadTreeHost tree;
  std::vector<int> allskel;
  std::vector<int> allred;

  // Phase times of the last factor/solve (ms, CUDA events); id_ms is the
  // summed duration of the ID launches, id_launches their count.
  double t_factor_ms = 0, t_id_ms = 0, t_decouple_ms = 0, t_top_ms = 0;
  int id_launches = 0;
  double id_flops = 0, id_bytes = 0;  // algorithmic work of the streamed ID launches
  double id_fold_flops = 0;           // FP64 work of the on-chip fold ID launches
  bool time_phases = false;
  // Per-launch record of the timed factorization: kind 0 ID, 1 decouple,
  // 2 top-level assembly + LU; ms from CUDA events on the solver stream.
  struct LaunchRecord {
    int level, kind, group, ntasks, m_cap, n_cap;
    double ms;
  };
  std::vector<LaunchRecord> launch_log;
  double t_wait_ms = 0;  // host time blocked on the per-level rank download
  // host-side phases (steady clock): level list building before the ID
  // launch, skeleton/decouple bookkeeping after it, uploads, top level
  double t_host_prep_ms = 0, t_host_post_ms = 0, t_upload_ms = 0, t_host_top_ms = 0;
  std::string error;

 private:
  // Event pairs of the timed factorization, resolved after its final
  // synchronisation so timing adds no extra waits.
  struct PendingTimer {
    cudaEvent_t e0, e1;
    LaunchRecord rec;
  };
  std::vector<PendingTimer> pending_;
  int timer_begin(cudaEvent_t* e0, cudaStream_t s = nullptr);
  int timer_end(cudaEvent_t e0, const LaunchRecord& rec, cudaStream_t s = nullptr);
  int timers_resolve();
  int fail(const std::string& msg);
  int cuda_check(cudaError_t e, const char* what);
  int process_level(int level);
  int factor_top();
  int factor_border();
  std::vector<BoxBlock> blocks_of(int box) const;
  void build_block_map(const std::vector<BoxBlock>& blocks, int n, std::vector<int>* bid,
                       std::vector<int>* bpos, std::vector<UpdBlock>* tab) const;

  SolverOptions opt_;
  int sd_ = 1, n_points_ = 0, n_dofs_ = 0, nb_ = 0;
  std::vector<double> pts_, nrm_, curv_, wts_, holes_;
  cudaStream_t stream_;
  // Decoupling of level l runs on dstream_ while the host prepares, and the
  // GPU runs, the interpolative decompositions of level l - 1.
  cudaStream_t dstream_ = nullptr;
  cudaEvent_t ev_id_ = nullptr, ev_dec_ = nullptr;

  bool onchip_ok_[17] = {};  // a G-CTA cluster with full shared memory fits
  Arena arena_;
  Arena stage_{true};  // pinned staging of every host-to-device upload
  template <class T>
  int upload(T* dst, const std::vector<T>& src, cudaStream_t s);
  Scratch work_, scratch2_;
  Node* d_nodes_ = nullptr;
  double* d_proxy_dir_ = nullptr;
  double* d_holes_ = nullptr;
  int* d_status_ = nullptr;

  // per-box device factors (indexed by box id)
  struct BoxDev {
    double* T = nullptr;
    double* L = nullptr;
    double* U = nullptr;
    double* X = nullptr;
    double* acc = nullptr;
    int* piv = nullptr;
  };
  std::vector<BoxDev> boxdev_;
  std::vector<LevelFactors> levels_;
  LevelFactors all_compressed_;

  // top level
  int ns_ = 0;
  double* d_top_ = nullptr;  // LU of allskel_mat, or of S with holes
  int* d_top_piv_ = nullptr;
  int* d_allskel_ = nullptr;
  int* d_allred_ = nullptr;
  int* d_red_pos_ = nullptr;
  double* d_U_ = nullptr;     // N x nb
  double* d_Psi_ = nullptr;   // nb x N
  std::vector<double> h_PsiT_;  // Psi^T (N x nb), host
  double* d_Ured_ = nullptr;  // modified U rows of allred (|red| x nb)
  double* d_Pred_ = nullptr;  // modified Psi^T rows of allred (|red| x nb)
  double* d_tmp_ = nullptr;   // solve scratch
};

}  // namespace kib

#endif  // KI_SOLVER_H_
