// C++ drop-in API of the B200 solver: the reference's solve entry points
// (kern_interp/linear_solve.h:15-35), same names, arguments and results.
#ifndef KERN_INTERP_LINEAR_SOLVE_H_
#define KERN_INTERP_LINEAR_SOLVE_H_

#include <string>
#include <vector>

#include "kern_interp/boundaries/boundary.h"
#include "kern_interp/kernel/kernel.h"
#include "kern_interp/quadtree/quadtree.h"
#include "kern_interp/skel_factorization/skel_factorization.h"

#define TIMING_ITERATIONS 5

namespace kern_interp {

// Factor, solve and evaluate at the kernel's domain points; points outside
// the domain (Boundary::is_in_domain) get 0 (linear_solve.cpp:142-180).
ki_Mat boundary_integral_solve(const Kernel& kernel, const Boundary& boundary,
                               QuadTree* quadtree, double id_tol, int fact_threads,
                               const std::vector<double>& domain_points);
// Hole columns U (log / Stokeslet + rotlet per hole) and rows Psi
// (quadrature weights on each hole's nodes), linear_solve.cpp:18-110.
ki_Mat initialize_U_mat(const Kernel::Pde pde, const std::vector<Hole>& holes,
                        const std::vector<double>& tgt_points);
ki_Mat initialize_Psi_mat(const Kernel::Pde pde, const std::vector<Hole>& holes,
                          const Boundary& boundary);
// domain_size^2 points of a grid over [x_min, x_max] x [y_min, y_max], x
// outer, as interleaved xy (linear_solve.cpp:183-194)
void get_domain_points(int domain_size, std::vector<double>* points, double x_min,
                       double x_max, double y_min, double y_max);
// mu = A^-1 f (and alpha for a multiply-connected domain), linear_solve.cpp:113-123
void linear_solve(const SkelFactorization& skel_factorization, const QuadTree& quadtree,
                  const ki_Mat& f, ki_Mat* mu, ki_Mat* alpha = nullptr);
// solution = K_domain mu (+ U_forward alpha), linear_solve.cpp:126-140
void schur_solve(const SkelFactorization& skel_factorization, const QuadTree& quadtree,
                 const ki_Mat& U, const ki_Mat& Psi, const ki_Mat& f, const ki_Mat& K_domain,
                 const ki_Mat& U_forward, ki_Mat* solution);

}  // namespace kern_interp

#endif  // KERN_INTERP_LINEAR_SOLVE_H_
