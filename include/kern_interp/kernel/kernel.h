// C++ drop-in API of the B200 solver: kern_interp::Kernel.
//
// Same type, fields and constructor as the reference's kern_interp/kernel/
// kernel.h:15-86: the PDE and copies of the boundary arrays.  operator()
// returns the dense block of boundary-operator entries (Kernel::laplace /
// stokes_get, kernel.cpp:11-150; bit-identical to the reference's), and
// forward() the domain-evaluation matrix (kernel.cpp:337-357); both are
// formed by the library's GPU entry kernels.  The per-box ID and proxy
// matrices of the reference's Kernel are built on the GPU inside
// SkelFactorization::skeletonize and are not exposed here.
#ifndef KERN_INTERP_KERNEL_KERNEL_H_
#define KERN_INTERP_KERNEL_KERNEL_H_

#include <memory>
#include <vector>

#include "kern_interp/boundaries/boundary.h"
#include "kern_interp/ki_mat.h"
#include "kern_interp/quadtree/quadtree.h"

#define NUM_PROXY_POINTS 128
#define RADIUS_RATIO 1.5

namespace kern_interp {

struct Kernel {
  enum Pde { LAPLACE, LAPLACE_NEUMANN, STOKES };
  Kernel() {}
  Kernel(int solution_dimension_, int domain_dimension_, Kernel::Pde pde_, Boundary* boundary,
         std::vector<double> domain_points_)
      : solution_dimension(solution_dimension_),
        domain_dimension(domain_dimension_),
        pde(pde_),
        boundary_points(boundary->points),
        boundary_normals(boundary->normals),
        boundary_weights(boundary->weights),
        boundary_curvatures(boundary->curvatures),
        domain_points(domain_points_) {}

  int solution_dimension, domain_dimension;
  Kernel::Pde pde;
  std::vector<double> boundary_points, boundary_normals, boundary_weights, boundary_curvatures,
      domain_points;

  // K(tgt, src) for boundary dofs (forward = false), or for domain-point
  // dofs against boundary dofs (forward = true: rows index the domain
  // points' dofs)
  ki_Mat operator()(const std::vector<int>& tgt_inds, const std::vector<int>& src_inds,
                    bool forward = false) const;
  void update_boundary(Boundary* boundary);
  ki_Mat laplace_get(const std::vector<int>& tgt_inds, const std::vector<int>& src_inds,
                     bool forward = false) const;
  ki_Mat stokes_get(const std::vector<int>& tgt_inds, const std::vector<int>& src_inds,
                    bool forward = false) const;
  // every domain-point dof against every boundary dof
  ki_Mat forward() const;

 private:
  // device copy of the boundary arrays, made on first use (shared by copies
  // of this Kernel; dropped by update_boundary)
  mutable std::shared_ptr<void> geometry_;
  void* geometry() const;
};

}  // namespace kern_interp

#endif  // KERN_INTERP_KERNEL_KERNEL_H_
