// Device work descriptors and kernel launchers of the B200 solver.
#ifndef KI_KERNELS_H_
#define KI_KERNELS_H_

#include <cuda_runtime.h>

#include <algorithm>

#include <vector>

#include "ki_entries.cuh"

namespace kib {

// Number of kernels this library has launched in the process (every launch
// wrapper below adds its launches).
void count_launches(int n);
long long launch_total();

// ---------------------------------------------------------------- ID
// One interpolative decomposition (Kernel::get_id_mat + ki_Mat::id,
// kernel.cpp:153-235, ki_mat.cpp:502-541).  Rows of the ID matrix:
//   [0, I)      K(rowdof[r], act[j])          near/outside dofs as targets
//   [I, 2I)     K(act[j], rowdof[r - I])      the transposed block
//   [2I, m)     proxy rows (proxy = 256 Laplace / 512 Stokes, 0 on levels 1-2)
struct IdTask {
  int n;          // active dofs (columns)
  int m;          // rows = 2 I + proxy
  int n_row;      // I
  int proxy;      // proxy rows
  int act_off;    // into IdParams::act
  int row_off;    // into IdParams::rowdofs
  int lda;        // leading dimension of A in the workspace
  int perm_off;   // into IdParams::perm (n ints)
  long long a_off;  // A in the workspace (doubles)
  long long t_off;  // T output (doubles), capacity n*n/4 + 1
  double cx, cy, rad, pw;  // proxy circle centre, radius, weight
  int sk;         // > 0: on-chip CTA factors the sk x n row sketch S A instead of A
  int pshift;     // sketched tasks: proxy circle of kNumProxy >> pshift points
};

// Row sketch of an ID matrix (on-chip): every row of A is added with a
// hashed sign into one row of the sk-row sketch, the rows of each 32-row
// block of A into a run of 32 consecutive sketch rows (mod sk) from a hashed
// start (a sparse sign embedding; sk >= 32).
constexpr int kSketchBlocks = 1;
// Sketch rows for an m x n matrix: n + 16 rounded up to the block count.
inline int sketch_rows(int n) { return (n + 16 + kSketchBlocks - 1) / kSketchBlocks * kSketchBlocks; }
// Sketch rows when the box's rank is expected near rank_hint (the largest
// rank of the level below; 0 when unknown): rank_hint + 40, at least 64 and
// at most n + 16, a multiple of 8.  A rank found above rows - 16, or none,
// is not trusted (the kernel reports -1 and the box is decomposed again
// with n + 16 rows).
// Levels of at most this many boxes take the full sketch directly.
constexpr int kShortSketchMinBoxes = 32;
inline int sketch_rows_hint(int n, int rank_hint) {
  const int want = ((rank_hint > 24 ? rank_hint : 24) + 40 + 7) / 8 * 8;
  const int full = sketch_rows(n);
  return want < full ? want : full;
}

struct IdParams {
  const IdTask* tasks;
  int ntasks;
  int pde;
  const Node* nodes;
  const int* act;
  const int* rowdofs;
  double* work;
  double* tout;
  int* perm;
  int* rank;
  const double* proxy_dir;  // cos/sin table, 2 * kNumProxy doubles
  double tol;
  int m_cap, n_cap;  // streaming launches: maxima over the launch (shared-memory layout)
  long long col_cap;  // unused by the kernels (kept for the host's bookkeeping)
  long long onchip_smem;  // on-chip launches: dynamic shared memory per CTA, the
                          // largest id_onchip_smem_bytes over the launch's tasks
};
// Shared memory of one on-chip CTA for an m x n box in a G-CTA cluster (the
// layout is per task, so boxes of different sizes share a launch).
size_t id_onchip_smem_bytes(int m, int n, int G);
// ... and for a sketched box (sk sketch rows) in a G-CTA cluster.
size_t id_sketch_smem_bytes(int sk, int n, int G);

// launch_id group codes: G (1, 2, 4, 8) streams the matrix through HBM/L2
// with G CTAs per box; kOnChip + G (G = 1 .. 16) keeps it in the shared
// memory of a G-CTA cluster.
constexpr int kOnChip = 100;
// Column stride of an on-chip ID matrix with m rows: the smallest >= m
// that is 4 mod 16 doubles.  The trailing update gives each column a group
// of L lanes (L = 4 .. 32) reading consecutive rows; with the stride 4 mod
// 16 the four 4-lane groups of a half-warp start 4 banks apart (disjoint),
// the two 8-lane groups overlap in half their banks.  Measured on a B200
// (deep-level IDs of the Stokes workload): the QR loop 23% faster than with
// an odd stride, 9% faster than with 8 mod 16.
inline int onchip_lda(int m) { return m + ((4 - m % 16) + 16) % 16; }
// Nonzero if an on-chip launch of this size can be scheduled on the device.
int id_cluster_fits(int group, int m_cap, int n_cap, size_t col_cap);

// Launches one ID per task with a cluster of CTAs per task (group codes above).
cudaError_t launch_id(const IdParams& p, int group, cudaStream_t s);
size_t id_smem_bytes(int m_cap, int n_cap);

// One ID whose working matrix lives in a static device array (no device
// allocation anywhere); lda * n must not exceed kNoAllocScratchDoubles.
constexpr long long kNoAllocScratchDoubles = 1LL << 20;  // 8 MiB
cudaError_t launch_id_noalloc(int pde, const Node* nodes, const int* act, int n,
                              const int* rows, int n_rows, int proxy_rows, double cx,
                              double cy, double radius, double tol, int* rank, int* perm,
                              double* T, cudaStream_t s);

// ---------------------------------------------------------------- decouple
// Assembly + decouple of one compressed box (skel_factorization.cpp:55-91).
// The box's K_BN = K(act, act) - (children's accumulated Schur updates) is
// formed in pivot order [skel; redundant]; update blocks are addressed per
// active position: upd(a, b) = blocks[bid[a]] (bpos[a], bpos[b]) when
// bid[a] == bid[b] >= 0.
struct UpdBlock {
  const double* acc;  // accumulated update matrix, size x size, ld size
  int size;
  int pad;
};

struct DecTask {
  int n, k;              // active, skeleton count (r = n - k)
  const int* act;        // n active dofs, active order
  const int* perm;       // ID pivots: column p of the ID is active[perm[p]]
  const int* bid;        // per active position: update block id or -1
  const int* bpos;       // per active position: row inside that block
  const UpdBlock* blocks;
  const double* T;       // k x r, ld k (from the ID)
  double* K;             // scratch n x n + kLuSyncInts (boxes too large for shared memory)
  double* L;             // k x r, ld k
  double* U;             // r x k, ld r
  double* X;             // X_rr^{-1}, r x r, ld r (written by the decoupling)
  double* acc;           // accumulated update on the skeleton, k x k
  int* piv;              // r ints of scratch (pivots of the inversion)
};

struct DecParams {
  const DecTask* tasks;
  int ntasks;
  int pde;
  const Node* nodes;
  int* status;  // set nonzero on an exactly zero pivot
};

// n_max: largest box of the launch (sizes the shared-memory staging).
// Boxes with n > kDecoupleSmemN must go through decouple_large instead.
constexpr int kDecoupleSmemN = 160;
cudaError_t launch_decouple(const DecParams& p, int n_max, cudaStream_t s);
// Dynamic shared memory of a decouple launch whose largest box has n_max dofs.
size_t decouple_smem_bytes(int n_max);
// The same decoupling for one large box as a sequence of GPU-wide kernels
// (tk is the host copy of the box's descriptor; tk.K must hold n x n).
cudaError_t decouple_large(const DecTask& tk, int pde, const Node* nodes, int* status,
                           cudaStream_t s);

// Dense assembly of the top-level skeleton matrix K(allskel, allskel) minus
// the accumulated updates (skel_factorization.cpp:116-122), n x n, ld ld.
cudaError_t launch_assemble_top(int pde, const Node* nodes, const int* dofs, int n,
                                const int* bid, const int* bpos, const UpdBlock* blocks,
                                double* out, int ld, cudaStream_t s);

// ---------------------------------------------------------------- forest
// Per-tree top-level system of a forest: the tree's root skeleton dofs, the
// update-block lookup of its children, and its n x n matrix / pivots.
struct TopTask {
  int n;
  int pad;
  const int* dofs;
  const int* bid;
  const int* bpos;
  const UpdBlock* blocks;
  double* a;
  int* piv;
};
// Assemble and LU-factor every tree's top matrix (one CTA per tree).
cudaError_t launch_forest_top(int pde, const Node* nodes, const TopTask* tasks, int ntasks,
                              int n_max, int* status, cudaStream_t s);
// x[dofs_t] <- A_t^{-1} x[dofs_t] for every tree t (one CTA per tree).
cudaError_t launch_forest_top_solve(const TopTask* tasks, int ntasks, int n_max, double* x,
                                    cudaStream_t s);

// ---------------------------------------------------------------- dense LU
// In-place LU with partial pivoting of an n x n matrix (ld), pivots 0-based
// row indices as LAPACK's (ipiv[j] = row swapped with j).  With `sync`
// (kLuSyncInts ints of device scratch, used by this call alone until it
// completes) a matrix of up to kLuFusedMaxN rows is factored by one
// cooperative launch; otherwise, or when larger, panel by panel (the same
// pivot rule and values, the trailing sums in another order).  *status: 1 zero pivot, 2 a bounded wait between the
// cooperative launch's thread blocks ran out.
constexpr int kLuFusedMaxN = 768;
constexpr int kLuSyncInts = kLuFusedMaxN / 32 + 8;
cudaError_t dense_lu(double* a, int n, int ld, int* ipiv, int* status, cudaStream_t s,
                     int* sync = nullptr, bool top_level = false);
// Test hook for the failure path of the cooperative LU: the next top-level
// launch (dense_lu with top_level) of more than one thread block starts with
// its abort word raised (mode 1) or with block 0's flag held down so that
// the other blocks' bounded waits run out (mode 2); either way it ends with
// *status = 2.  0 clears it.
void inject_lu_fault(int mode);
// Multi-CTA tiled C = C0 + alpha op(A) op(B) (64 x 64 tiles, FP64 tensor
// cores); C0 may be null.
cudaError_t launch_gemm_tiled(double* C, int ldc, const double* C0, int ldc0, const double* A,
                              int lda, bool ta, const double* B, int ldb, bool tb, int m, int n,
                              int k, double alpha, cudaStream_t s);
// Multi-CTA tiled C = C0 - op(A) op(B) (64 x 64 tiles); C0 may be null.
cudaError_t launch_gemm_sub(double* C, int ldc, const double* C0, int ldc0, const double* A,
                            int lda, bool ta, const double* B, int ldb, bool tb, int m, int n,
                            int k, cudaStream_t s);
// Each of the nrows rows of B (column stride ldb) <- row * A^{-1}.
cudaError_t dense_lu_solve_rows(const double* lu, int n, int ld, const int* ipiv, double* b,
                                int nrows, int ldb, cudaStream_t s);
// B <- A^{-1} B (n x nrhs, ldb) for the LU above; perm (optional, from
// launch_pivots_to_perm) replaces the sequential interchanges by a gather;
// dinv (optional, with perm, n <= kLuBlockInvMaxN: launch_lu_block_inv)
// the inverted 16 x 16 diagonal blocks, applied as products in place of
// the in-block substitutions.
cudaError_t dense_lu_solve(const double* lu, int n, int ld, const int* ipiv, double* b,
                           int nrhs, int ldb, cudaStream_t s, const int* perm = nullptr,
                           const double* dinv = nullptr);
// The inverses of the 16 x 16 diagonal blocks of L and U of an n x n LU:
// lu_block_inv_doubles(n) doubles at dinv.
constexpr int kLuBlockInvMaxN = 768;
inline size_t lu_block_inv_doubles(int n) { return static_cast<size_t>((n + 15) / 16) * 512; }
cudaError_t launch_lu_block_inv(const double* lu, int n, int ld, double* dinv, cudaStream_t s);
// Brings [p, p + bytes) into L2 (evict-last priority) from a whole grid of
// prefetches; returns as soon as they are issued.
cudaError_t launch_l2_prefetch(const void* p, size_t bytes, cudaStream_t s);
// The interchanges ipiv[0..n) of an LU composed into one permutation:
// (P b)[i] = b[perm[i]].
cudaError_t launch_pivots_to_perm(const int* ipiv, int n, int* perm, cudaStream_t s);

// Border blocks of the bordered top-level system S (ld >= ns + nb).
cudaError_t launch_fill_border(double* S, int ld, int ns, int nb, const double* us,
                               const double* ps, const double* corr, cudaStream_t s);

// ---------------------------------------------------------------- sweeps
// Per-box sweep descriptors for SkelFactorization::solve
// (skel_factorization.cpp:341-403) and the multiply-connected variant.
struct SweepTask {
  int k, r;
  const int* skel;   // k dofs
  const int* red;    // r dofs
  const double* T;   // k x r
  const double* L;   // k x r
  const double* U;   // r x k
  const double* X;   // X_rr^{-1} (r x r)
  const int* piv;    // unused by the sweeps (kept with the factors)
};

struct SweepParams {
  const SweepTask* tasks;
  int ntasks;
  double* x;
  int ldx, nrhs;
  int red_pos_map;      // nonzero: redundant dofs index rows of x via red_pos
  const int* red_pos;
  int cap;              // per-box staging: max over tasks of k + r
  int ldd = 1;          // dof stride of x: entry (dof, rhs c) is x[dof ldd + c ldx]
  // nonzero: max over tasks of k r; a single right-hand side then stages the
  // box's two factor matrices in shared memory (asynchronous copies issued
  // with the gather: one memory round trip instead of one per few entries)
  int kr = 0;
};
// Boxes up to this many redundant dofs stage X^{-1} in a single-right-hand-
// side diagonal solve (r^2 doubles next to the vector).
constexpr int kDiagStageMaxR = 104;

// x[red] -= T^T x[skel]; then x[skel] -= L x[red]   (or U^T when use_u)
cudaError_t launch_sweep_up(const SweepParams& p, bool use_u, cudaStream_t s);
// x[red] -= U x[skel]; then x[skel] -= T x[red]
// Both border up sweeps of a level at once: pu (MODE L) and pp (MODE U^T),
// same tasks, rhs count and capacity, different vectors.
cudaError_t launch_sweep_up_pair(const SweepParams& pu, const SweepParams& pp, cudaStream_t s);
cudaError_t launch_sweep_down(const SweepParams& p, cudaStream_t s);
// x[red] = X_rr^{-1} x[red]
cudaError_t launch_diag_solve(const SweepParams& p, cudaStream_t s);
// Transposed solve pieces (A^-T = Up^T Diag^T Top^T Down^T): the transposed
// down step x_r -= T^T x_s, x_s -= U^T x_r is launch_sweep_up(use_u = true);
// the transposed up step is x_r -= L^T x_s, x_s -= T x_r; the transposed
// diagonal solve is X_rr^-T.
cudaError_t launch_transposed_up(const SweepParams& p, cudaStream_t s);
cudaError_t launch_diag_solve_t(const SweepParams& p, cudaStream_t s);

// ---------------------------------------------------------------- misc
// out[i] = x[idx[i]] (gather) / x[idx[i]] = in[i] (scatter), nrhs columns.
cudaError_t launch_gather(const double* x, int ldx, const int* idx, int n, int nrhs,
                          double* out, int ldo, cudaStream_t s);
// out[i + ldo c] = x[idx[i] ldd + c]: rows of a dof-major matrix
cudaError_t launch_gather_rows(const double* x, int ldd, const int* idx, int n, int nrhs,
                               double* out, int ldo, cudaStream_t s);
// Ured, Pred, dinv <- rows allred of U, Psi^T, X^{-1} U (dof-major, nb a
// dof); us, ps <- rows allskel of U, Psi^T; outputs column-major (ld nr, ns)
cudaError_t launch_border_gather(const double* modU, const double* modP, const double* modD,
                                 int nb,
                                 const int* allred, int nr, const int* allskel, int ns,
                                 double* Ured, double* Pred, double* dinv, double* us,
                                 double* ps, cudaStream_t s);
// dst rows idx[0..n) <- the same rows of src (dof-major, nb entries a dof)
cudaError_t launch_copy_rows(const double* src, double* dst, int nb, const int* idx, int n,
                             cudaStream_t s);
// C (m x n, m, n <= 32) = alpha A^T B + beta C, A k x m, B k x n column-major,
// split over k; `part` holds long_gemm_tn_splits(m, n, k) * m * n doubles
// (0: sizes not supported)
int long_gemm_tn_splits(int m, int n, int k);
cudaError_t long_gemm_tn(int m, int n, int k, double alpha, const double* a, int lda,
                         const double* b, int ldb, double beta, double* c, int ldc,
                         double* part, cudaStream_t s);
// allred (the n - ns dofs outside skel_sorted, ascending) and red_pos (n:
// position in allred, -1 for a skeleton) from the ascending, repeat-free
// skeleton dofs skel_sorted[0..ns), all below n
cudaError_t launch_red_index(const int* skel_sorted, int ns, int n, int* allred, int* red_pos,
                             cudaStream_t s);
cudaError_t launch_scatter(double* x, int ldx, const int* idx, int n, int nrhs,
                           const double* in, int ldi, cudaStream_t s);
// C = alpha * op(A) * op(B) + beta * C, small dense FP64 (column-major).
cudaError_t small_gemm(bool ta, bool tb, int m, int n, int k, double alpha,
                       const double* a, int lda, const double* b, int ldb, double beta,
                       double* c, int ldc, cudaStream_t s);

// y = K x for the full boundary operator (on-the-fly entries), plus the
// hole border terms when U/Psi are given (nb border columns).  seg (node
// offsets of nseg problems, may be null) makes it block diagonal.
cudaError_t launch_apply_operator(int pde, const Node* nodes, int n_dofs, const int* seg,
                                  int nseg, const double* x, double* y, int nb, const double* U,
                                  const double* Psi, cudaStream_t s);
// Target evaluation out = K_fwd(targets) mu (+ U_fwd alpha).
cudaError_t launch_eval_targets(int pde, const Node* nodes, int n_dofs, int nt,
                                const double* targets, const double* mu, int nh,
                                const double* holes, const double* alpha, double* out,
                                cudaStream_t s);
// Solution on domain points with the domain mask (boundary_integral_solve,
// linear_solve.cpp:142-180).  kind: kDomainAll (no mask), kDomainNodes
// (CubicBoundary::is_in_domain on the node curves), kDomainDisk (the
// Circle / Annulus / Donut test with disk = {cx, cy, R}).  mask: 1 inside,
// 0 outside.  launch_domain_eval zeroes outside points when mask is given;
// `part` holds splits x rows doubles when splits > 1 (domain_splits).
enum DomainKind : int { kDomainAll = 0, kDomainNodes = 1, kDomainDisk = 2 };
int domain_splits(int nt, int np, int num_sms);
// The node-curve test needs domain_mask_scratch_bytes(np) of device scratch.
size_t domain_mask_scratch_bytes(int np);
cudaError_t launch_domain_mask(int kind, const Node* nodes, int np, const double* holes, int nh,
                               const double* disk, int nt, const double* targets,
                               unsigned char* mask, void* scratch, cudaStream_t s);
cudaError_t launch_domain_eval(int pde, const Node* nodes, int np, int nt,
                               const double* targets, const double* mu, int nh,
                               const double* holes, const double* alpha,
                               const unsigned char* mask, int splits, double* part,
                               double* out, cudaStream_t s);
// cudaFuncSetAttribute(func, attr, value) unless this process already
// raised the attribute to at least `value` on the current device: the call
// costs microseconds of host time, which level loops with many short
// launches otherwise pay on every launch.
cudaError_t raise_func_attr(const void* func, cudaFuncAttribute attr, int value);

// Batched device-to-device copy: segment i moves words[i] 32-bit words from
// src to dst (one CTA per segment).
struct CopySeg {
  const unsigned* src;
  unsigned* dst;
  long long words;
};
cudaError_t launch_copy_segments(const CopySeg* segs, int n, cudaStream_t s);
// Hole border of a multiply-connected domain (initialize_U_mat /
// initialize_Psi_mat): U (dofs x nb, column-major), Urow the same U stored
// dof-major (entry (i, b) at i nb + b), Psi (nb x dofs, column-major, which
// is Psi^T stored dof-major).
cudaError_t launch_border_fill(int pde, const Node* nodes, int np, const double* holes, int nh,
                               double* U, double* Psi, double* Urow, cudaStream_t s);
// Forward block: domain dofs tgt (point tgt / sd of `targets`, component
// tgt % sd) against boundary dofs src, column-major nt x ns.
cudaError_t launch_forward_block(int pde, const Node* nodes, const double* targets,
                                 const int* tgt, int nt, const int* src, int ns, double* out,
                                 cudaStream_t s);
// Dense kernel block K(tgt, src), column-major nt x ns.
cudaError_t launch_kernel_block(int pde, const Node* nodes, const int* tgt, int nt,
                                const int* src, int ns, double* out, cudaStream_t s);

// ---------------------------------------------------------------- Krylov
// Fast FP64 operator product y = A x (fused, reassociated: accurate to FP64
// rounding, not bit-identical to the entry kernels), bordered by U / Psi
// when nb > 0.  `part` needs fast_matvec_scratch_doubles(n_dofs, splits, nseg, nb).
constexpr int kMaxMatvecSplits = 64;
constexpr int kMaxKrylov = 64;  // vectors per multi-dot
// One CTA of the operator product: targets [t0, t1) (nodes) against sources
// [s0, s1) of the same segment (problem); partial `split`; the first target
// tile of a (segment, split) also sums the rank-one coefficient into slot
// rank1_slot.
struct MvTile {
  int t0, t1, s0, s1, split, rank1_slot, first, pad;
};
// Source splits for nseg segments of about n_nodes nodes each: the count
// whose tiles fill whole waves of the resident CTAs best (a last, partly
// filled wave costs as much time as a full one).
int matvec_splits(int pde, int n_nodes, int nseg, int num_sms);
// seg: node offsets of the segments (size nseg + 1); one segment = one
// problem, so a forest's operator is block diagonal.
void matvec_tiles(const std::vector<int>& seg, int splits, std::vector<MvTile>* tiles);
size_t fast_matvec_scratch_doubles(int n_dofs, int splits, int nseg, int nb);
cudaError_t launch_fast_matvec(int pde, const Node* nodes, const MvTile* tiles, int ntiles,
                               const int* seg, int nseg, int n_dofs, int splits, const double* x,
                               double* y, int nb, const double* U, const double* Psi,
                               double* part, cudaStream_t s);
// The same product for a small correction d (see ki_krylov.cu): source
// blocks whose bounding box comes within near_gap of the target tile's in
// FP64, the others in FP32 with the densities scaled by dscale (> 0).
cudaError_t launch_corr_matvec(int pde, const Node* nodes, const MvTile* tiles, int ntiles,
                               const int* seg, int nseg, int n_dofs, int splits, const double* x,
                               double dscale, double near_gap, double* y, int nb,
                               const double* U, const double* Psi, double* part,
                               cudaStream_t s);
// out[j] = V_j . w for j < k (V column j at V + ldv j); part needs
// k * multi_dot_blocks(n) doubles.  Fixed reduction order.
int multi_dot_blocks(int n);
cudaError_t launch_multi_dot(const double* V, long long ldv, int k, const double* w, int n,
                             double* part, double* out, cudaStream_t s);
// w += sign * V h
cudaError_t launch_multi_axpy(double* w, const double* V, long long ldv, int k, const double* h,
                              int n, double sign, cudaStream_t s);
// ---------------------------------------------------------------- adjoint
// Laplace double-layer adjoint contractions (see ki_adjoint.cu).  work needs
// adjoint_work_doubles(n).  Phase 1: g_mu = K_t^T grad_u and the target
// term; phase 2 (after lam = A^-T g_mu): node gradients of J.
size_t adjoint_work_doubles(int n);
cudaError_t launch_adjoint_laplace(const Node* nodes, int n, const double* mu, int nt,
                                   const double* targets, const double* grad_u, double* g_mu,
                                   double* work, cudaStream_t s);
cudaError_t launch_adjoint_laplace_finish(const Node* nodes, int n, const double* mu,
                                          const double* lam, double* work, double* g_pts,
                                          double* g_nrm, double* g_w, double* g_k,
                                          cudaStream_t s);

cudaError_t launch_scale_copy(double* dst, const double* src, int n, double a, cudaStream_t s);
// out[p] = squared norm of segment p of v (dofs seg[p] sd .. seg[p + 1] sd)
cudaError_t launch_segment_sumsq(const double* v, const int* seg, int nseg, int sd, double* out,
                                 cudaStream_t s);
// x += y
cudaError_t launch_add(double* x, const double* y, int n, cudaStream_t s);
// r = b - ax
cudaError_t launch_sub(double* r, const double* b, const double* ax, int n, cudaStream_t s);
// y = g - y (g null: y = -y)
cudaError_t launch_rsub(double* y, const double* g, int n, cudaStream_t s);

}  // namespace kib

#endif  // KI_KERNELS_H_
