/* kinterp: C ABI of the B200 recursive-skeletonization solver for 2-D
 * Laplace / Stokes boundary integral equations.
 *
 * Every entry point replaces one call of the reference C++ API
 * (jpryan1/kern-interp-old; paths relative to that repository) and takes
 * plain pointers and sizes only.  Unless a name ends in _device, buffers are
 * host memory and the call returns after its results are in them.  The
 * `stream` argument of ki_factor is a cudaStream_t (NULL: the library creates
 * its own non-blocking stream); every later call on the handle is ordered on
 * that stream.  All calls return KI_OK (0) or an error code, with the message
 * in ki_last_error(); nothing ever aborts the process.
 *
 * Geometry arrays follow the reference Boundary (boundaries/boundary.h:35-51):
 * points and normals interleaved xy (2 n_points doubles), curvatures and
 * weights (n_points), holes as n_holes rows of (cx, cy, radius, num_nodes).
 * A Stokes dof is 2 * point + component, as in Kernel::stokes_get
 * (kernel/kernel.cpp:47-96).
 */
#ifndef KINTERP_H_
#define KINTERP_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ki_solver_s* ki_solver_t;

enum {
  KI_OK = 0,
  KI_ERR_ARG = 1,      /* invalid argument or handle */
  KI_ERR_CUDA = 2,     /* CUDA runtime error (no device, launch failure, ...) */
  KI_ERR_NUMERIC = 3,  /* singular block, no compression possible */
  KI_ERR_STATE = 4     /* call out of order (e.g. solve before factor) */
};

enum { KI_LAPLACE = 0, KI_LAPLACE_NEUMANN = 1, KI_STOKES = 2 };

/* Factorization modes.  KI_MODE_REFERENCE: the reference's method exactly
 * (same partition, ranks and skeletons).  KI_MODE_PRECONDITIONER: for a
 * factorization used by ki_solve_refined: boxes whose ID matrix is much
 * taller than wide are decomposed through a sparse random row sketch
 * whose proxy circle has 64 of the reference's 128 points (cheaper,
 * different skeletons, same accuracy class). */
enum { KI_MODE_REFERENCE = 0, KI_MODE_PRECONDITIONER = 1 };

/* Message of the last failing call on this thread ("" if none). */
const char* ki_last_error(void);
/* Library version, major * 10000 + minor * 100 + patch. */
int ki_version(void);
/* Number of CUDA kernels this library has launched in the process. */
long long ki_kernel_launches(void);
/* Device and pinned host memory that destroyed handles left in the
 * library's cache for later factorizations, in bytes; ki_release_cache()
 * returns it to CUDA (call it with no handle alive). */
long long ki_cached_bytes(void);
void ki_release_cache(void);

/* Builds the quadtree and skeletonizes the boundary operator.
 * Replaces QuadTree::initialize_tree (quadtree/quadtree.h:85-86), the U/Psi
 * set-up of boundary_integral_solve (linear_solve.cpp:155-163) and
 * SkelFactorization(id_tol, threads).skeletonize (skel_factorization/
 * skel_factorization.h:25,40).  max_leaf_dofs is the reference's
 * MAX_LEAF_DOFS (quadtree.h:10; 32 there). */
int ki_factor(int pde, int n_points, const double* points, const double* normals,
              const double* curvatures, const double* weights, int n_holes,
              const double* holes, int max_leaf_dofs, double id_tol, void* stream,
              ki_solver_t* out);

/* Builds only the quadtree (host side, no GPU work): QuadTree::
 * initialize_tree (quadtree.h:85-86) with every box's active list set as
 * before any compression.  The handle answers the introspection calls below;
 * solve calls on it return KI_ERR_STATE. */
int ki_partition(int n_points, const double* points, int sol_dim, int max_leaf_dofs,
                 ki_solver_t* out);

/* Releases every device buffer of the handle. */
void ki_destroy(ki_solver_t s);

/* Dof count (n_points or 2 n_points) and border size (holes: 1 per hole for
 * Laplace, 3 per hole for Stokes; 0 without holes). */
int ki_num_dofs(ki_solver_t s);
int ki_num_border(ki_solver_t s);

/* linear_solve (linear_solve.h:27-29): mu = A^{-1} f with the factors; alpha
 * receives the border unknowns (multiply_connected_solve,
 * skel_factorization.h:60-61) and may be NULL when there are no holes. */
int ki_solve(ki_solver_t s, const double* f, double* mu, double* alpha);

/* ki_solve on device buffers, stream ordered, no host synchronisation.
 * d_f and d_mu may be the same buffer. */
int ki_solve_device(ki_solver_t s, const double* d_f, double* d_mu, double* d_alpha);

/* y = A x with on-the-fly FP64 entries of the full operator (the dense
 * matrix the reference test forms, kern_interp_test.cpp:54-90), bordered by
 * [U; Psi, -I] when there are holes; device buffers of dofs + border. */
int ki_apply_device(ki_solver_t s, const double* d_x, double* d_y);

/* The bordered solve with a nonzero border right-hand side g (nb values,
 * NULL = zero): [A U; Psi -I][mu; alpha] = [f; g].  The reference solves
 * only g = 0 (skel_factorization.cpp:406-551); the refinement needs the
 * general form to precondition residuals. */
int ki_solve_bordered_device(ki_solver_t s, const double* d_f, const double* d_g, double* d_mu,
                             double* d_alpha);

/* FP64 refinement (no counterpart in the reference, whose linear_solve is
 * the direct solve only, linear_solve.cpp:113-124): right-preconditioned
 * GMRES on the operator of ki_apply_device with this factorization as the
 * preconditioner, stopping when the true relative residual
 * ||[f; 0] - A [mu; alpha]|| / ||f|| <= rel_tol or after max_iters
 * preconditioned products (each = one solve + one operator product).
 * iters and rel_res (may be NULL) report the products used and the final
 * true residual.  Use with a factorization at a looser id_tol (or the
 * reduced-precision one of ki_factor_ex) to reach FP64 accuracy. */
int ki_solve_refined_device(ki_solver_t s, const double* d_f, double* d_mu, double* d_alpha,
                            double rel_tol, int max_iters, int* iters, double* rel_res);
/* Same with host buffers (copies inside the call; returns when mu and alpha
 * are in host memory). */
int ki_solve_refined(ki_solver_t s, const double* f, double* mu, double* alpha, double rel_tol,
                     int max_iters, int* iters, double* rel_res);
/* The refinement's operator product: same y as ki_apply_device up to FP64
 * rounding (fused and reassociated, not bit-identical to the entries). */
int ki_matvec_device(ki_solver_t s, const double* d_x, double* d_y);
/* The refinement's product for a small correction d (no reference
 * counterpart): source blocks far from a target tile summed in FP32 (d
 * scaled by dscale > 0 on the way, to keep it in FP32's normal range), near
 * ones in FP64; relative error ~1e-6 of |A| |d|.  ki_solve_refined uses it
 * to update small residuals. */
int ki_matvec_correction_device(ki_solver_t s, const double* d_x, double* d_y, double dscale);

/* x = A^-T b with the factorization (no reference counterpart: the
 * reference solves only with A, skel_factorization.cpp:341-403).  Simply
 * connected domains only.  d_b and d_x may be the same buffer. */
int ki_solve_transpose_device(ki_solver_t s, const double* d_b, double* d_x);

/* Differentiable target potential u = K_t A^-1 f (Laplace double layer,
 * simply connected; the target map of linear_solve.cpp:126-140), as the
 * forward/backward pair of an autograd function.  Forward: d_mu = A^-1 d_f
 * (kept by the caller for the backward) and d_u = K_t d_mu at n_targets
 * points (interleaved xy).  Backward: given d_grad_u = dJ/du, writes
 * dJ/df = A^-T K_t^T grad_u (n dofs) and dJ/d(points) (2n), dJ/d(normals)
 * (2n), dJ/d(weights) (n), dJ/d(curvatures) (n), the node geometry held
 * by the handle; chain them to any shape parameters on the caller's side.
 * No reference counterpart (the reference has no derivatives). */
int ki_adjoint_forward(ki_solver_t s, const double* d_f, int n_targets, const double* d_targets,
                       double* d_mu, double* d_u);
int ki_adjoint_backward(ki_solver_t s, int n_targets, const double* d_targets, const double* d_mu,
                        const double* d_grad_u, double* d_grad_f, double* d_grad_points,
                        double* d_grad_normals, double* d_grad_weights,
                        double* d_grad_curvatures);

/* schur_solve's target evaluation (linear_solve.cpp:126-140): out = K_domain
 * mu + U_forward alpha at n_targets points (interleaved xy). */
int ki_eval_targets(ki_solver_t s, int n_targets, const double* targets,
                    const double* mu, const double* alpha, double* out);
/* Same on device buffers (targets, mu, alpha, out), stream-ordered. */
int ki_eval_targets_device(ki_solver_t s, int n_targets, const double* d_targets,
                           const double* d_mu, const double* d_alpha, double* d_out);

/* boundary_integral_solve's evaluation on domain points
 * (linear_solve.cpp:142-180): out = K_domain mu + U_forward alpha, set to
 * zero at every point outside the domain.  The domain test `kind`:
 *   KI_DOMAIN_ALL    no test (every point kept);
 *   KI_DOMAIN_NODES  CubicBoundary::is_in_domain (cubic_boundary.cpp:182-230)
 *                    on the handle's node curves (outer nodes first, then
 *                    each hole's nodes): outside within 1e-2 of a node, or
 *                    by the crossing counts of the outer curve and holes;
 *   KI_DOMAIN_DISK   Circle / Annulus / Donut::is_in_domain (circle.cpp:34-42,
 *                    annulus.cpp:66-79, donut.cpp:67-80) with disk = host
 *                    {cx, cy, R}: outside when |x - c| + 1e-2 > R or within
 *                    1e-2 of a hole's circle or inside it.
 * Entries are formed on the fly (no |targets| x N matrix); the sums agree
 * with the exact entries to FP64 rounding.  Points exactly on a node get
 * no contribution from that node (such points are outside every test).
 * Device variant: targets (interleaved xy), mu, alpha, out on the device,
 * stream-ordered; host variant copies in and out and returns when out is
 * in host memory. */
enum { KI_DOMAIN_ALL = 0, KI_DOMAIN_NODES = 1, KI_DOMAIN_DISK = 2 };
int ki_eval_domain_device(ki_solver_t s, int n_targets, const double* d_targets,
                          const double* d_mu, const double* d_alpha, int kind, const double* disk,
                          double* d_out);
int ki_eval_domain(ki_solver_t s, int n_targets, const double* targets, const double* mu,
                   const double* alpha, int kind, const double* disk, double* out);
/* The domain test alone: d_mask[t] = 1 inside, 0 outside (kind NODES or DISK). */
int ki_domain_mask_device(ki_solver_t s, int n_targets, const double* d_targets, int kind,
                          const double* disk, unsigned char* d_mask);
/* get_domain_points (linear_solve.cpp:183-193): domain_size^2 points,
 * x = x_min + i/(domain_size-1) (x_max - x_min) in the outer loop and y
 * likewise in the inner loop, interleaved xy into points (2 domain_size^2). */
int ki_domain_points(int domain_size, double x_min, double x_max, double y_min, double y_max,
                     double* points);

/* Test hook for the failure path (no reference counterpart; the reference
 * has no bounded waits).  KI_INJECT_LU_ABORT: the next top-level LU done
 * by the cooperative launch (33 to 768 rows) starts with its abort word
 * raised; KI_INJECT_LU_STALL: its first block
 * keeps its flag down, so the other blocks' bounded waits (200 ms) run out.
 * Either way that factorization returns KI_ERR_NUMERIC ("a bounded wait
 * timed out") and the device stays usable.  One-shot, process-wide;
 * KI_INJECT_NONE clears it. */
enum { KI_INJECT_NONE = 0, KI_INJECT_LU_ABORT = 1, KI_INJECT_LU_STALL = 2 };
int ki_test_inject_fault(int what);
/* A handle holding device copies of the boundary arrays only, without a
 * quadtree or factors: the Kernel object of the reference (kernel.h:15-41,
 * its boundary copies) for dense entry blocks (ki_kernel_block,
 * ki_forward_block); every other call refuses it.  Free with ki_destroy. */
int ki_geometry(int pde, int n_points, const double* points, const double* normals,
                const double* curvatures, const double* weights, void* stream,
                ki_solver_t* out);
/* Kernel::operator() with forward = true (kernel.cpp:114-150, 337-357): the
 * column-major nt x ns block of forward entries, row i the domain dof tgt[i]
 * (point tgt[i] / sol_dim of the n_targets interleaved xy targets, velocity
 * component tgt[i] % sol_dim), column j the boundary dof src[j]. */
int ki_forward_block(ki_solver_t s, int n_targets, const double* targets, int nt, const int* tgt,
                     int ns, const int* src, double* out);
/* Kernel::operator() (kernel/kernel.cpp:99-111): column-major nt x ns block
 * K(tgt, src) evaluated on the GPU. */
int ki_kernel_block(ki_solver_t s, int nt, const int* tgt, int ns, const int* src,
                    double* out);

/* Tree / skeleton introspection (QuadTree levels and InteractionLists,
 * quadtree.h:14-102).  info[8] = is_leaf, compressed, |original|, |active|,
 * |skel|, |redundant|, parent index in its level (-1 root), level;
 * geom[3] = lower-left corner x, y and side length.  Lists may be NULL. */
int ki_num_levels(ki_solver_t s);
int ki_num_boxes(ki_solver_t s, int level);
int ki_box_info(ki_solver_t s, int level, int idx, int* info, double* geom);
int ki_box_lists(ki_solver_t s, int level, int idx, int* original, int* active,
                 int* skel, int* redundant);
/* Neighbour list of a box (QuadTreeNode::neighbors, computed by
 * compute_neighbor_lists, quadtree.cpp:27-69), in the reference's order:
 * neighbour q is box nbr_idx[q] of level nbr_level[q].  Returns the count
 * (negative on error); either output may be NULL. */
int ki_box_neighbors(ki_solver_t s, int level, int idx, int* nbr_level, int* nbr_idx);
/* Top-level skeleton (root active box); returns its size, fills out if given. */
int ki_allskel(ki_solver_t s, int* out);

/* Statistics of the last factorization: out[0] factor ms, [1] ID kernel ms,
 * [2] ID launches, [3] ID algorithmic FP64 flops (entry generation,
 * Householder steps taken, T solve), [4] ID algorithmic HBM bytes (inputs,
 * outputs, and the working matrix of launches that stream it),
 * [5] decouple ms, [6] top-level LU ms, [7] host ms blocked on rank
 * downloads, host ms spent on [8] level lists before the ID launches,
 * [9] skeleton/decouple bookkeeping, [10] uploads, [11] the top level,
 * [12] the part of [3] done by on-chip launches, [13] pinned staging bytes
 * the handle has used since it was made or last updated, [14] decoupling
 * algorithmic FP64 flops (K_BN entries, the products with T, X_rr^-1, L,
 * U and the accumulated update), [15] top-level flops (assembly + 2/3 n^3
 * LU), [16] factor bytes one solve reads (T twice, L, U, X_rr^-1, top LU,
 * 8 vector passes) (timed factorizations only for [1], [5], [6]).
 * Returns the number of values written (at most n, at most 17). */
int ki_stats(ki_solver_t s, double* out, int n);
/* Launch log of a ki_factor_timed factorization: rows of 7 doubles
 * (level, kind 0 ID / 1 decouple / 2 top LU, cluster size, boxes, max rows,
 * max columns, ms).  Returns the row count; writes at most cap rows. */
int ki_launch_log(ki_solver_t s, double* out, int cap);
/* Timeline of a ki_factor_timed factorization: rows of 4 doubles
 * (what, level, start ms, end ms) after the factorization began: `what` <
 * 100 is a launch kind of ki_launch_log timed on the GPU clock; `what` =
 * 100 + code is a host mark (7 geometry queued, 8 partition built, 0 tree
 * checked, 9 a level's active lists, 10 its ID rows, 11 its ID groups
 * ordered, 1 level lists ready and ID launched, 2 ranks received, 3 decouple
 * launched, 4 top level started, 5 top level launched, 6 synchronised) on
 * the host clock.  Returns the row
 * count; writes at most cap rows. */
int ki_timeline(ki_solver_t s, double* out, int cap);

/* Enables CUDA-event timing of the ID launches for the next ki_factor calls
 * made through ki_factor_timed. */
int ki_factor_timed(int pde, int n_points, const double* points, const double* normals,
                    const double* curvatures, const double* weights, int n_holes,
                    const double* holes, int max_leaf_dofs, double id_tol, void* stream,
                    ki_solver_t* out);

/* ki_factor with a mode (KI_MODE_*) and phase timing (timed != 0, as
 * ki_factor_timed). */
int ki_factor_ex(int pde, int n_points, const double* points, const double* normals,
                 const double* curvatures, const double* weights, int n_holes,
                 const double* holes, int max_leaf_dofs, double id_tol, int mode, int timed,
                 void* stream, ki_solver_t* out);

/* QuadTree::perturb (quadtree/quadtree.cpp:359-560) followed by
 * SkelFactorization::skeletonize (skel_factorization.cpp:94-243), as the
 * reference's boundary-update loops run them (kern_interp_test.cpp:491-530,
 * experiment_two.cpp:55-60): the handle follows its boundary to new node
 * arrays (any number of points; holes as in ki_factor).  Points are matched
 * to the old ones by exact coordinates.  Leaves that gain or lose points,
 * their neighbours, their ancestors and the ancestors' neighbours are
 * factored again, over-full leaves are split and sparse subtrees merged;
 * every other compressed box keeps its factors (its dofs renumbered).
 * n_reused (may be NULL) receives the number of boxes kept.  One problem
 * per handle (not a batch).  On failure the handle is unusable. */
int ki_update(ki_solver_t s, int n_points, const double* points, const double* normals,
              const double* curvatures, const double* weights, int n_holes, const double* holes,
              int* n_reused);

/* The partition half of QuadTree::perturb on a ki_partition handle (no
 * GPU): the tree follows its points to new ones exactly as ki_update's does. */
int ki_partition_update(ki_solver_t s, int n_points, const double* points);

/* QuadTree::copy_into (quadtree/quadtree.cpp:584-641) followed by
 * skeletonize, as kern_interp_test.cpp:533-567 runs them: a new handle on
 * `stream` (NULL: its own) with a copy of the tree and of every compressed
 * box's factors; only the boxes without compression and the top level are
 * factored again, so its solves equal this handle's.  The two handles are
 * independent afterwards (ki_update on one leaves the other as it is). */
int ki_copy(ki_solver_t s, void* stream, ki_solver_t* out);

/* Many independent problems factored together (no reference counterpart:
 * the reference factors one boundary per QuadTree).  Problem p has
 * n_points[p] nodes; the geometry arrays are the problems' arrays laid end
 * to end (points/normals interleaved xy), and so are the dofs of every
 * later call (ki_solve, ki_solve_device, ki_solve_refined[_device]): the
 * handle holds one quadtree per problem, and every level of every tree is
 * processed by the same launches.  Each problem gets exactly the partition,
 * skeletons and factors it would get alone.  Simply connected domains only
 * (no holes); n_problems >= 1. */
int ki_factor_batch(int pde, int n_problems, const int* n_points, const double* points,
                    const double* normals, const double* curvatures, const double* weights,
                    int max_leaf_dofs, double id_tol, int mode, void* stream, ki_solver_t* out);
/* The partition of a batch only (host; like ki_partition per problem). */
int ki_partition_batch(int n_problems, const int* n_points, const double* points, int sol_dim,
                       int max_leaf_dofs, ki_solver_t* out);
/* Number of problems in the handle (1 for ki_factor). */
int ki_num_problems(ki_solver_t s);
/* Problem index of box idx of level `level` (negative on error). */
int ki_box_tree(ki_solver_t s, int level, int idx);

/* Interpolative decomposition of one box that allocates no device memory,
 * for callers that cannot call cudaMalloc (their device memory is owned by
 * another allocator, such as a framework's caching allocator or a pool
 * reserved up front, and a cudaMalloc/cudaFree would also synchronise the
 * device).  No counterpart in the reference: it is the per-box step of
 * skeletonize (Kernel::get_id_mat + ki_Mat::id) exposed on its own.
 *
 * Device inputs: d_nodes holds n_points records of 8 doubles (x, y, n_x,
 * n_y, weight, curvature, 0, 0); d_active the n_active column dofs; d_rows
 * the n_rows near dofs.  The ID matrix is [K(rows, active); K(active,
 * rows)^T], followed, when proxy is nonzero, by the 128-point proxy-circle
 * rows of centre (cx, cy) and the given radius (256 rows for Laplace, 512
 * for Stokes).  Every dof in d_active and d_rows must be below n_points
 * (Laplace) or 2 n_points (Stokes): the device does not check them.  Device outputs: *d_rank (0: not compressible), d_perm
 * (n_active pivots, active positions), d_T (k x (n_active - k), ld k;
 * capacity n_active^2 / 4 + 1 doubles).
 * The m x n working matrix lives in one static 8 MiB device array: calls
 * with ((m + 3) / 4 * 4) * n_active > 1048576 are rejected with KI_ERR_ARG.
 * The first call on a device resolves that array's address (make it before
 * any stream capture).  All calls share the array: calls that overlap on the
 * GPU race.  Stream ordered; returns without synchronising. */
int ki_id_noalloc(int pde, const double* d_nodes, int n_points, const int* d_active,
                  int n_active, const int* d_rows, int n_rows, int proxy, double cx,
                  double cy, double radius, double id_tol, int* d_rank, int* d_perm,
                  double* d_T, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* KINTERP_H_ */
