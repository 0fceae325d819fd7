/* CPU restatement of the reference's recursive-skeletonization solver.
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle the GPU product is checked
 * against (tests/, __graft_entry__.smoke and bench.py's CPU arm).  The product
 * never links, loads or calls it.
 *
 * Every entry point restates a reference routine (paths relative to the
 * reference repository):
 *   kiora_create      QuadTree::initialize_tree  quadtree.cpp:72-114
 *                     SkelFactorization::skeletonize skel_factorization.cpp:94-243
 *   kiora_solve       linear_solve               linear_solve.cpp:113-123
 *                     SkelFactorization::solve   skel_factorization.cpp:341-403
 *                     multiply_connected_solve   skel_factorization.cpp:406-551
 *   kiora_kernel_block Kernel::operator()        kernel.cpp:99-111
 *   kiora_eval_targets schur_solve               linear_solve.cpp:126-140
 *   kiora_border       initialize_U_mat / _Psi_mat linear_solve.cpp:18-110
 * The column-pivoted QR restates LAPACK dgeqp3/dlaqp2 (unblocked) and the LU
 * restates dgetf2, the published reference-LAPACK algorithms that the
 * reference reaches through LAPACKE (ki_mat.cpp:427-541).
 */
#ifndef ORACLE_KI_ORACLE_H_
#define ORACLE_KI_ORACLE_H_
#ifdef __cplusplus
extern "C" {
#endif

void* kiora_create(int pde, int n_points, const double* points,
                   const double* normals, const double* curvatures,
                   const double* weights, int n_holes, const double* holes,
                   int max_leaf_dofs, double id_tol, int threads,
                   double* t_factor);
void kiora_destroy(void* h);
int kiora_solve(void* h, const double* f, double* mu, double* alpha,
                double* t_solve);
int kiora_num_levels(void* h);
int kiora_num_nodes(void* h, int level);
void kiora_node_info(void* h, int level, int idx, int* info, double* geom);
void kiora_node_lists(void* h, int level, int idx, int* original, int* active,
                      int* skel, int* redundant);
void kiora_kernel_block(void* h, int nt, const int* tgt, int ns,
                        const int* src, double* out);
void kiora_eval_targets(void* h, int nt, const double* targets,
                        const double* mu, const double* alpha, double* out);
int kiora_border(void* h, double* U, double* Psi);
int kiora_allskel(void* h, int* out);
/* y = A x with A the full dense boundary operator (plus the [K U; Psi -I]
 * border when the domain has holes); x and y have dofs (+ border) entries. */
void kiora_apply_dense(void* h, const double* x, double* y);
/* Per compressed box ID statistics: rows of (level, m, n, k). Returns count. */
int kiora_id_stats(void* h, int* out, int cap);

#ifdef __cplusplus
}
#endif
#endif
