// C++ drop-in API of the B200 solver: kern_interp::SkelFactorization.
//
// Same class, constructor and public entry points as the reference's
// kern_interp/skel_factorization/skel_factorization.h:19-62.  skeletonize
// runs the whole recursive skeletonization on the GPU (ki_factor, or
// ki_update after QuadTree::perturb) and leaves the factors in the tree;
// solve and multiply_connected_solve run the level sweeps on the GPU
// (ki_solve).  fact_threads is accepted for compatibility (the GPU
// schedules boxes itself).  The per-box steps of the reference (decouple,
// id_compress, the Schur-update gathers, the sweep helpers) happen inside
// those calls and are not exposed one by one.  Failures print the
// library's error and abort, where the reference asserts or exits.
#ifndef KERN_INTERP_SKEL_FACTORIZATION_SKEL_FACTORIZATION_H_
#define KERN_INTERP_SKEL_FACTORIZATION_SKEL_FACTORIZATION_H_

#include <vector>

#include "kern_interp/kernel/kernel.h"
#include "kern_interp/ki_mat.h"
#include "kern_interp/quadtree/quadtree.h"

#define MIN_DOFS_TO_COMPRESS 16

namespace kern_interp {

class SkelFactorization {
 public:
  double id_tol;
  int fact_threads;

  SkelFactorization() {}
  SkelFactorization(double id_tol, int fact_threads);
  ~SkelFactorization() {}

  void skeletonize(const Kernel& K, QuadTree* tree);
  void solve(const QuadTree& quadtree, ki_Mat* x, const ki_Mat& b) const;
  void multiply_connected_solve(const QuadTree& quadtree, ki_Mat* x, ki_Mat* alpha,
                                const ki_Mat& b) const;
};

}  // namespace kern_interp

#endif  // KERN_INTERP_SKEL_FACTORIZATION_SKEL_FACTORIZATION_H_
