// Solver side of the domain evaluation (boundary_integral_solve,
// linear_solve.cpp:142-180): the split choice, the scratch for the split
// partials and the mask, and the launches of ki_domain.cu.
#include <algorithm>
#include <vector>

#include "ki_solver.h"

namespace kib {

namespace {
// The node-curve test walks the outer nodes and then each hole's nodes:
// the hole node counts must be non-negative and fit in the node array.
bool curves_fit(const std::vector<double>& holes, int n_points) {
  double used = 0;
  for (size_t h = 0; h + 3 < holes.size(); h += 4) {
    if (!(holes[h + 3] >= 0)) return false;
    used += holes[h + 3];
  }
  return used <= n_points;
}
}  // namespace

int Solver::domain_mask(int nt, const double* d_targets, int kind, const double* disk,
                        unsigned char* d_mask) {
  if (kind != kDomainNodes && kind != kDomainDisk) return fail("domain_mask: unknown test");
  if (kind == kDomainDisk && !disk) return fail("domain_mask: the disk test needs {cx, cy, R}");
  if (n_trees() > 1) return fail("domain_mask: not available for a batch of problems");
  if (kind == kDomainNodes && !curves_fit(holes_, n_points_))
    return fail("domain_mask: hole node counts exceed the number of nodes");
  KI_CUDA(dom_.reserve(domain_mask_scratch_bytes(n_points_), stream_));
  KI_CUDA(launch_domain_mask(kind, d_nodes_, n_points_, d_holes_, n_holes(), disk, nt, d_targets,
                             d_mask, dom_.p, stream_));
  return 0;
}

int Solver::eval_domain(int nt, const double* d_targets, const double* d_mu,
                        const double* d_alpha, int kind, const double* disk, double* d_out) {
  if (kind != kDomainAll && kind != kDomainNodes && kind != kDomainDisk)
    return fail("eval_domain: unknown domain test");
  if (kind == kDomainDisk && !disk) return fail("eval_domain: the disk test needs {cx, cy, R}");
  if (n_trees() > 1) return fail("eval_domain: not available for a batch of problems");
  if (kind == kDomainNodes && !curves_fit(holes_, n_points_))
    return fail("eval_domain: hole node counts exceed the number of nodes");
  if (nt == 0) return 0;
  if (!num_sms_) {
    int dev = 0;
    KI_CUDA(cudaGetDevice(&dev));
    KI_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
  }
  const int splits = domain_splits(nt, n_points_, num_sms_);
  const size_t rows = static_cast<size_t>(nt) * sd_;
  // scratch: [split partials][node-curve test][mask], 256-byte aligned parts
  auto up = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  const size_t part_bytes = up(splits > 1 ? sizeof(double) * rows * splits : 0);
  const size_t curve_bytes = up(kind == kDomainNodes ? domain_mask_scratch_bytes(n_points_) : 0);
  const size_t mask_bytes = kind != kDomainAll ? static_cast<size_t>(nt) : 0;
  KI_CUDA(dom_.reserve(part_bytes + curve_bytes + mask_bytes + 16, stream_));
  char* base = static_cast<char*>(dom_.p);
  double* part = reinterpret_cast<double*>(base);
  unsigned char* mask =
      mask_bytes ? reinterpret_cast<unsigned char*>(base + part_bytes + curve_bytes) : nullptr;
  if (mask) KI_CUDA(launch_domain_mask(kind, d_nodes_, n_points_, d_holes_, n_holes(), disk, nt,
                                       d_targets, mask, base + part_bytes, stream_));
  const bool use_alpha = nb_ > 0 && d_alpha;
  KI_CUDA(launch_domain_eval(opt_.pde, d_nodes_, n_points_, nt, d_targets, d_mu, n_holes(),
                             d_holes_, use_alpha ? d_alpha : nullptr, mask, splits, part, d_out,
                             stream_));
  return 0;
}

}  // namespace kib
