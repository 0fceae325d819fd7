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
#include <utility>
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
  size_t used() const { return used_; }  // bytes handed out since construction
  void swap(Arena& o) {
    std::swap(pinned_, o.pinned_);
    chunks_.swap(o.chunks_);
    std::swap(cur_, o.cur_);
    std::swap(left_, o.left_);
    std::swap(reserved_, o.reserved_);
    std::swap(used_, o.used_);
  }

 private:
  bool pinned_;
  std::vector<std::pair<void*, size_t>> chunks_;
  char* cur_ = nullptr;
  size_t left_ = 0;
  size_t reserved_ = 0;
  size_t used_ = 0;
};

// Reusable device scratch that only grows.
struct Scratch {
  void* p = nullptr;
  size_t bytes = 0;
  // buffers outgrown without waiting for the stream (returned to the pool
  // when the scratch is destroyed, after its owner synchronized)
  std::vector<std::pair<void*, size_t>> retired;
  ~Scratch();
  // Grows to at least `want` bytes; the old buffer is released after `s`
  // has drained (a synchronization), or, with retire, kept until the end.
  cudaError_t reserve(size_t want, cudaStream_t s, bool retire = false);
};

struct SolverOptions {
  int pde = 0;              // 0 Laplace, 1 Laplace-Neumann, 2 Stokes
  int max_leaf_dofs = 32;   // MAX_LEAF_DOFS (quadtree.h:10)
  double id_tol = 1e-6;
  int min_dofs_to_compress = 16;  // MIN_DOFS_TO_COMPRESS (skel_factorization.h:11)
  // Preconditioner mode: boxes whose ID matrix is much taller than wide are
  // decomposed through a sparse row sketch (different skeletons from the
  // reference, same accuracy class); for factorizations used with the
  // refinement, never for reference-identical results.
  bool sketch_id = false;
  // Sketched boxes sample the proxy circle at every 2^proxy_shift-th of the
  // reference's kNumProxy points: the circle's representation error decays
  // like (box radius / circle radius)^points, far below a preconditioner's
  // tolerance at 64 points.
  int proxy_shift = 0;
  // Preconditioner mode, one tree: level 1 is left uncompressed when its
  // active dofs (with the hole border) are at most this many (0: never).
  // The top-level matrix grows from level 1's skeletons to its active dofs,
  // which the single-launch LU factors in less time than the level-1 IDs
  // and decouplings take (their pivoted QRs are the factorization's longest
  // dependent chains); the factorization only gets more accurate.
  int top_keep_max = 0;
};

// Device factors of one compressed box, for copying between solvers.
struct BoxDevView {
  const double *T, *L, *U, *X, *acc;
  const int* piv;
  int k, r;
};

struct LevelFactors {
  int level = 0;
  int ntasks = 0;
  int cap = 0;
  int kr = 0;  // max over the level's boxes of k r (rank x redundant); all_compressed_: max r^2 of the staged boxes
  int nbig = 0;  // all_compressed_: the first nbig tasks (largest r) stage nothing
  SweepTask* d_tasks = nullptr;
  std::vector<SweepTask> h_tasks;  // host copy of d_tasks
  int* d_skel = nullptr;
  int* d_red = nullptr;
  int nred = 0;  // entries of d_red (the level's redundant dofs)
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

  // Many independent problems in one factorization (a forest): problem p
  // owns points [starts[p], starts[p + 1]); its dofs are numbered after the
  // previous problems'.  Call before factor(); no holes.
  void set_forest(const std::vector<int>& starts) { starts_ = starts; }
  int n_trees() const { return starts_.size() > 1 ? static_cast<int>(starts_.size()) - 1 : 1; }
  size_t staging_bytes() const { return stage_.used() + keep_stage_.used(); }
  const std::vector<int>& starts() const { return starts_; }

  // QuadTree::initialize_tree + SkelFactorization::skeletonize.
  int factor();
  // QuadTree::perturb (quadtree.cpp:359-560) to a new boundary, then
  // skeletonize: compressed boxes whose points and neighbourhoods did not
  // change keep their factors (renumbered); the others, and the top level,
  // are factored again.  One problem; n_reused reports the kept boxes.
  int update(int n_points, const double* points, const double* normals,
             const double* curvatures, const double* weights, int n_holes, const double* holes,
             int* n_reused);
  // QuadTree::copy_into (quadtree.cpp:584-641) followed by skeletonize:
  // a factorization of the same boundary in a new solver on `stream`, its
  // tree a copy of this one and every compressed box's factors copied on
  // the device; only the uncompressed boxes and the top level are factored.
  Solver* copy(cudaStream_t stream, int* rc);
  // QuadTree::initialize_tree only, active lists as before compression.
  void build_tree_only();
  // Device copies of the boundary arrays only (no quadtree, no factors),
  // for dense entry blocks; returns after the copies are done.
  int prepare_geometry() {
    const int rc = setup_geometry();
    return rc ? rc : cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
  }
  // The partition half of QuadTree::perturb on a tree-only solver.
  void perturb_tree_only(int n_points, const double* points);
  // linear_solve on device buffers: d_mu (dofs), d_alpha (border, may be
  // null when there are no holes).  d_b and d_mu may be the same buffer.
  // d_g (nb values, may be null = zero) is the right-hand side of the
  // border rows [Psi -I][mu; alpha] = g; the reference always has g = 0.
  int solve_device(const double* d_b, double* d_mu, double* d_alpha,
                   const double* d_g = nullptr);
  // FP64 refinement / GMRES on the (bordered) boundary operator,
  // preconditioned by this factorization, entries of A formed on the fly:
  // stops when ||[f; 0] - A [mu; alpha]|| <= rel_tol ||f|| or after
  // max_iters preconditioned products.  The first residual is formed with
  // the FP64 product; once the residual r is small enough that the
  // correction product's error (kCorrErr |r|) stays below a tenth of
  // rel_tol ||f||, a stationary step updates it as r -= A d with the
  // correction product of its correction d (corr_matvec_device).  iters /
  // rel_res report the work and the final residual.
  int solve_refined(const double* d_f, double* d_mu, double* d_alpha, double rel_tol,
                    int max_iters, int* iters, double* rel_res);
  // Fast FP64 product y = A x (bordered), the refinement's residual operator.
  int matvec_device(const double* d_x, double* d_y);
  // y = A d for a small correction d: far source blocks summed in FP32 with
  // d scaled by dscale, near blocks in FP64 (launch_corr_matvec).
  int corr_matvec_device(const double* d_x, double* d_y, double dscale);
  // Relative error bound of the correction product (measured below 2e-6 of
  // |A d| on every test geometry); KI_CORR=0 turns the product off.
  static constexpr double kCorrErr = 2e-6;
  // Bounding-box gap below which a source block is summed in FP64.
  static constexpr double kCorrNearGap = 0.01;
  // x = A^-T b with the same factorization (simply connected domains):
  // the sweeps of solve_device transposed and run in reverse order.
  int solve_transpose_device(const double* d_b, double* d_x);
  // Backward pass of u = K_t A^-1 f (Laplace, no holes): given mu = A^-1 f
  // and grad_u at n_targets points, writes grad_f = A^-T K_t^T grad_u and
  // the gradients with respect to the node positions (2 per node), normals
  // (2 per node), weights and curvatures.
  int adjoint_backward(int n_targets, const double* d_targets, const double* d_mu,
                       const double* d_grad_u, double* d_grad_f, double* d_grad_points,
                       double* d_grad_normals, double* d_grad_weights, double* d_grad_curv);
  // y = A x on device (bordered when there are holes).
  int apply_device(const double* d_x, double* d_y);
  // boundary_integral_solve's evaluation (linear_solve.cpp:142-180):
  // d_out = K_domain mu + U_forward alpha at nt points, zero outside the
  // domain of test `kind` (DomainKind; disk = host {cx, cy, R} for
  // kDomainDisk).  domain_mask writes the test alone (1 inside).
  int eval_domain(int nt, const double* d_targets, const double* d_mu, const double* d_alpha,
                  int kind, const double* disk, double* d_out);
  int domain_mask(int nt, const double* d_targets, int kind, const double* disk,
                  unsigned char* d_mask);

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
  int n_red_ = 0;  // dofs outside allskel (the bordered system's redundant rows)

  // Phase times of the last factor/solve (ms, CUDA events); id_ms is the
  // summed duration of the ID launches, id_launches their count.
  double t_factor_ms = 0, t_id_ms = 0, t_decouple_ms = 0, t_top_ms = 0;
  int id_launches = 0;
  double id_flops = 0, id_bytes = 0;  // algorithmic FP64 flops / HBM bytes of all ID launches
  double id_onchip_flops = 0;         // the part of id_flops done by on-chip launches
  // algorithmic FP64 flops of the decoupling launches (entries of K_BN, the
  // products with T, X_rr^-1, L, U and the accumulated update) and of the
  // top level (assembly + LU); FP64 factor bytes one solve reads (T twice,
  // L, U, X_rr^-1, the top LU) plus its vector passes
  double dec_flops = 0, top_flops = 0, solve_bytes = 0;
  bool time_phases = false;
  // Per-launch record of the timed factorization: kind 0 ID, 1 decouple,
  // 2 top-level assembly + LU; ms from CUDA events on the solver stream.
  struct LaunchRecord {
    int level, kind, group, ntasks, m_cap, n_cap;
    double ms;
    double t0 = 0, t1 = 0;  // start / end, ms after the factorization began (GPU clock)
  };
  std::vector<LaunchRecord> launch_log;
  // Host side of the timed factorization: code (7 geometry queued, 8
  // partition built, 0 tree checked, 9 a level's active lists, 10 its ID
  // rows, 11 its ID groups ordered, 1 level lists ready / ID launched, 2
  // ranks received, 3 decouple launched, 4 top level started, 5 top level
  // launched, 6 factorization synchronised), level,
  // ms after the factorization began (host clock).
  struct HostMark {
    int code, level;
    double ms;
  };
  std::vector<HostMark> host_marks;
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
  cudaEvent_t ev_start_ = nullptr;  // GPU time origin of the timed factorization
  double host_start_ = 0;           // host time origin
  void mark(int code, int level);
  int timer_begin(cudaEvent_t* e0, cudaStream_t s = nullptr);
  int timer_end(cudaEvent_t e0, const LaunchRecord& rec, cudaStream_t s = nullptr);
  int timers_resolve();
  int fail(const std::string& msg);
  int cuda_check(cudaError_t e, const char* what);
  // One level's IDs between their launch and its decoupling: the next
  // level's IDs are launched before this level's decouple bookkeeping.
  struct IdCand {
    int box = -1, n = 0, m = 0, I = 0, g = 0, sk = 0;
    int g_full = 0;  // sketched with fewer than n + 16 rows: the cluster for n + 16
    std::vector<int> rows;
  };
  struct PendingLevel {
    int level = 0;
    std::vector<int> boxes;  // compressed boxes of the level (earlier ones first)
    std::vector<IdCand> cand;
    std::vector<IdTask> tasks;
    std::vector<int> comp;  // candidates that compressed
    int* rank = nullptr;  // pinned device-to-host targets
    int* perm = nullptr;
    int* d_act = nullptr;
    int* d_rows = nullptr;
    int* d_perm = nullptr;
    double* d_T = nullptr;
    int perm_total = 0;
    bool ids_queued = false;  // ev_id_[level & 1] marks the end of its IDs
  };
  int id_launch(int level, PendingLevel* pl);
  int id_finish(PendingLevel* pl);
  // Boxes whose short sketch could not certify their rank (rank -1 from
  // the kernel) decomposed again with the full n + 16 rows.
  int id_rerun_full(PendingLevel* pl);
  // Largest rank of the previous (deeper) level of this factorization
  // (-1 before the first level): sizes the next level's sketches.
  int rank_hint_ = -1;
  int decouple_level(PendingLevel* pl);
  int decouple_boxes(PendingLevel* pl);
  int level_sweeps(int level, const std::vector<int>& boxes, cudaStream_t s);
  int begin_factor(cudaEvent_t* ev0);
  int setup_geometry();
  int check_coincident();  // refuse nodes at the same position
  bool geom_ready_ = false;  // setup_geometry done for this factorization
  int finish_factor(cudaEvent_t ev0);
  // Copies the factors of `boxes` (T, L, U, X^-1, update, pivots) from
  // `src` into this solver's arena, one batched copy on stream_.
  int adopt_factors(const std::vector<int>& boxes, const std::vector<BoxDevView>& src);
  void drop_device_state();
  int build_all_compressed();
  bool level1_stays();
  int diag_all(SweepParams dp, bool trans);
  int factor_top();
  int factor_top_forest();
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
  cudaEvent_t ev_id_[2] = {}, ev_dec_ = nullptr;  // ev_id_: per level parity
  // A level's ID launches of different cluster sizes are independent: the
  // second and later ones run on these streams, concurrently with the first.
  static constexpr int kIdStreams = 3;
  cudaStream_t id_streams_[kIdStreams] = {};
  cudaEvent_t id_fork_ = nullptr, id_join_[kIdStreams] = {};
  // The few boxes too big for the batched decouple (one multi-kernel
  // sequence each) run on these, concurrently with each other.
  static constexpr int kDecStreams = 3;
  cudaStream_t dl_streams_[kDecStreams] = {};
  cudaEvent_t dl_fork_ = nullptr, dl_join_[kDecStreams] = {};
  // the border columns' level sweeps (U, Psi^T), beside the decouplings
  cudaStream_t bstream_ = nullptr;
  cudaEvent_t ev_lvl_ = nullptr, ev_bdr_ = nullptr;
  // a level's decoupling uploads (block maps, task lists, sweep
  // descriptors): queued on their own stream, they copy while the level
  // below is still decoupling, and the decoupling stream waits on ev_up_
  // (long complete by then) instead of running the copies between two
  // levels' decouplings, the factorization's longest chain
  cudaStream_t ustream_ = nullptr;
  cudaEvent_t ev_up_ = nullptr;

  bool onchip_ok_[17] = {};  // a G-CTA cluster with full shared memory fits
  Arena arena_;
  // pinned staging of every host-to-device upload and of the per-level rank
  // readbacks; replaced by a fresh arena at each update() (after the
  // streams are synchronised), so a long sequence of updates keeps it bounded
  Arena stage_{true};
  Arena keep_stage_{true};  // long-lived pinned buffers (refinement coefficients)
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

  // forest
  std::vector<int> starts_;       // point offsets of the problems (empty: one problem)
  TopTask* d_forest_ = nullptr;   // per-tree top systems
  int forest_nmax_ = 0;

  // top level
  int ns_ = 0;
  double* d_top_ = nullptr;  // LU of allskel_mat, or of S with holes
  int* d_top_piv_ = nullptr;
  int* d_top_perm_ = nullptr;  // the top LU's interchanges as one permutation
  double* d_top_dinv_ = nullptr;  // its inverted 16 x 16 diagonal blocks (or nullptr)
  int* d_allskel_ = nullptr;
  int* d_allred_ = nullptr;
  int* d_red_pos_ = nullptr;
  double* d_U_ = nullptr;     // N x nb
  double* d_Psi_ = nullptr;   // nb x N
  double* d_Urow_ = nullptr;  // U dof-major (N x nb, row i contiguous)
  double* d_modU_ = nullptr;  // U and Psi^T dof-major, swept up level by level
  double* d_modP_ = nullptr;
  // X_rr^{-1} U at every compressed box's redundant rows (dof-major), filled
  // level by level on the border stream
  double* d_modD_ = nullptr;
  double* d_Ured_ = nullptr;  // modified U rows of allred (|red| x nb)
  double* d_Pred_ = nullptr;  // modified Psi^T rows of allred (|red| x nb)
  double* d_tmp_ = nullptr;   // solve scratch
  // refinement workspace: Krylov basis V, preconditioned basis Z, vectors,
  // operator-product and dot-product partials
  Scratch kry_;
  Scratch adj_;  // adjoint contraction partials
  Scratch dom_;  // domain evaluation: split partials and the mask
  int mv_setup();  // tile table of the operator product (once)
  // The solve as a CUDA graph on fixed buffers (captured once the
  // factorization has served a few preconditioner applications, replayed
  // for every later one): copies in, one graph launch, copies out.
  int solve_graph(const double* d_b, double* d_mu, double* d_alpha, const double* d_g);
  cudaGraphExec_t solve_exec_ = nullptr;
  static constexpr int kGraphAfter = 6;  // preconditioner applications before capture
  int graph_uses_ = 0;
  double* g_x_ = nullptr;  // graph buffers: dofs, then border alpha, then border g
  MvTile* d_mv_tiles_ = nullptr;
  int n_mv_tiles_ = 0, mv_splits_ = 0;
  int* d_seg_ = nullptr;  // node offsets of the problems
  std::vector<int> seg_;
  double* h_kry_ = nullptr;  // pinned host copy of the Arnoldi coefficients
  int num_sms_ = 0;
  int smem_per_sm_ = 0;  // shared memory of an SM, bytes
};

}  // namespace kib

// Error propagation inside Solver members: a failing CUDA call or allocation
// records the message in `error` and returns a nonzero status.
#define KI_CUDA(expr)                                   \
  do {                                                  \
    const int rc_ = cuda_check((expr), #expr);          \
    if (rc_) return rc_;                                \
  } while (0)

#define KI_UPLOAD(...)                     \
  do {                                     \
    const int urc_ = upload(__VA_ARGS__);  \
    if (urc_) return urc_;                 \
  } while (0)

#define KI_ALLOC(ptr, type, count)                                  \
  do {                                                              \
    (ptr) = arena_.get<type>(count);                                \
    if (!(ptr)) return fail("device allocation failed: " #ptr);     \
  } while (0)

#endif  // KI_SOLVER_H_
