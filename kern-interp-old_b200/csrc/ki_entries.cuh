// Boundary-integral matrix entries on the device.
//
// The double-layer entries of the reference Kernel (kern_interp/kernel/
// kernel.cpp): Laplace (kernel.cpp:11-36, 114-150), Laplace-Neumann
// (kernel.cpp:23-33) and the Stokes 2x2 blocks with the rank-one completion
// (kernel.cpp:47-96), plus the proxy-circle rows used by the interpolative
// decomposition (kernel.cpp:238-334).  Every product and sum is issued with
// an explicit round-to-nearest intrinsic in the reference's C evaluation
// order, so no FMA contraction happens and an entry equals the reference's
// double-precision value bit for bit (the reference is built without FMA).
#ifndef KI_ENTRIES_CUH_
#define KI_ENTRIES_CUH_

#include <cuda_runtime.h>

namespace kib {

enum Pde : int { kLaplace = 0, kLaplaceNeumann = 1, kStokes = 2 };

// One boundary node: position, unit normal, quadrature weight, curvature.
struct __align__(16) Node {
  double x, y, nx, ny, w, k, pad0, pad1;
};

constexpr int kNumProxy = 128;        // kernel.h:10
constexpr double kRadiusRatio = 1.5;  // kernel.h:11

// Proxy directions cos/sin(2 pi q / 128) are evaluated by the host's libm
// (so the proxy points match the reference's, kernel.cpp:244-251) and passed
// to the kernels as a 256-entry table: cos in [0, 128), sin in [128, 256).

#define KI_INV_2PI (1.0 / (2 * 3.14159265358979323846))
#define KI_INV_PI (1.0 / (3.14159265358979323846))

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double subd(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double divd(double a, double b) { return __ddiv_rn(a, b); }

// 1 / x for normal x > 0: the hardware's approximate FP64 reciprocal (PTX
// rcp.approx.ftz.f64, an estimate good to roughly 20 bits) refined by two
// Newton-Raphson steps y <- y + y (1 - x y) in FP64, each squaring the
// relative error, so the result is accurate to FP64 rounding.  x = 0 gives
// an infinite estimate: callers exclude it.
__device__ __forceinline__ double nr_rcp(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// The arithmetic of the entry formulas.  Exact: every product, sum and
// quotient a round-to-nearest intrinsic in the reference's evaluation order
// (no contraction), so entries equal the reference's bits.  Fast: plain
// expressions (contracted to FMA) and reciprocals by nr_rcp, accurate to a
// few FP64 ulps: for the sketched IDs of the preconditioner mode, whose
// skeletons differ from the reference's anyway.
template <bool FAST>
struct EM {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};
template <>
struct EM<true> {
  static __device__ __forceinline__ double mul(double a, double b) { return a * b; }
  static __device__ __forceinline__ double add(double a, double b) { return a + b; }
  static __device__ __forceinline__ double sub(double a, double b) { return a - b; }
  static __device__ __forceinline__ double div(double a, double b) { return a * nr_rcp(b); }
};

// Kernel::laplace for r = t - s (not the forward/target variant).
template <bool FAST = false>
__device__ __forceinline__ double laplace_entry(int pde, double r1, double r2,
                                                double sw, double sc,
                                                double sn1, double sn2,
                                                double tn1, double tn2) {
  using M = EM<FAST>;
  const double rr = M::add(M::mul(r1, r1), M::mul(r2, r2));
  if (pde == kLaplace) {
    if (r1 == 0. && r2 == 0.) return M::add(0.5, M::mul(M::mul(M::mul(0.5, sc), sw), KI_INV_2PI));
    return M::div(M::mul(M::mul(-sw, KI_INV_2PI), M::add(M::mul(r1, sn1), M::mul(r2, sn2))), rr);
  }
  if (r1 == 0. && r2 == 0.)
    return M::add(M::sub(sw, 0.5), M::mul(M::mul(M::mul(0.5, sc), sw), KI_INV_2PI));
  return M::add(sw, M::div(M::mul(M::mul(sw, KI_INV_2PI), M::add(M::mul(r1, tn1), M::mul(r2, tn2))), rr));
}

// Boundary operator entry for target dof `tgt` at node t and source dof
// `src` at node s (the dofs give the Stokes components; for Stokes a dof is
// 2*node + component).
template <bool FAST = false>
__device__ __forceinline__ double pair_entry(int pde, const Node& t, int tgt, const Node& s,
                                             int src) {
  using M = EM<FAST>;
  if (pde != kStokes)
    return laplace_entry<FAST>(pde, M::sub(t.x, s.x), M::sub(t.y, s.y), s.w, s.k, s.nx, s.ny,
                               t.nx, t.ny);
  const int tc = tgt & 1, sc = src & 1;
  const double sn_s = sc ? s.ny : s.nx;   // sn[src % 2]
  const double tn_t = tc ? t.ny : t.nx;   // tn[tgt % 2]
  if (t.x == s.x && t.y == s.y) {
    // kernel.cpp:80-85: -1/2 delta - (kappa w / 2 pi) t t^T + w n n^T
    const int parity = (tgt + src + 1) & 1;
    const double snA = tc ? s.nx : s.ny;  // sn[(tgt + 1) % 2]
    const double snB = sc ? s.nx : s.ny;  // sn[(src + 1) % 2]
    const double a = M::mul(-0.5, static_cast<double>(parity));
    const double b = M::mul(M::mul(M::mul(M::mul(M::mul(static_cast<double>(1 - 2 * parity), 0.5), s.k), s.w),
                                   KI_INV_PI), snA);
    return M::add(M::add(a, M::mul(b, snB)), M::mul(M::mul(s.w, tn_t), sn_s));
  }
  const double r0 = M::sub(t.x, s.x), r1 = M::sub(t.y, s.y);
  const double rr = M::add(M::mul(r0, r0), M::mul(r1, r1));
  double pot;
  if (FAST) {
    const double inv = nr_rcp(rr);  // rr (not rr^2) stays in the estimate's range
    pot = (s.w * KI_INV_PI) * (r0 * s.nx + r1 * s.ny) * (inv * inv);
  } else {
    pot = M::div(M::mul(M::mul(s.w, KI_INV_PI), M::add(M::mul(r0, s.nx), M::mul(r1, s.ny))),
                 M::mul(rr, rr));
  }
  const double rt = tc ? r1 : r0, rs = sc ? r1 : r0;
  return M::add(M::mul(M::mul(pot, rt), rs), M::mul(M::mul(s.w, tn_t), sn_s));
}

// Boundary operator entry (tgt dof, src dof) from the node array.
template <bool FAST = false>
__device__ __forceinline__ double boundary_entry(int pde, const Node* __restrict__ nodes,
                                                 int tgt, int src) {
  const int sh = pde == kStokes ? 1 : 0;
  return pair_entry<FAST>(pde, nodes[tgt >> sh], tgt, nodes[src >> sh], src);
}

// Proxy-block row `row` (0 <= row < 2*128 for Laplace, 4*128 for Stokes) for
// box column dof `src` (kernel.cpp:268-334); circle centre (cx, cy), radius r.
template <bool FAST = false>
__device__ __forceinline__ double proxy_entry_node(int pde, const Node& nd,
                                                   const double* __restrict__ dir, int row,
                                                   int src, double cx, double cy, double r,
                                                   double pw, int ps = 0) {
  using M = EM<FAST>;
  const double* c_proxy_cos = dir;
  const double* c_proxy_sin = dir + kNumProxy;
  const int np = kNumProxy >> ps;  // every 2^ps-th point of the table
  if (pde != kStokes) {
    const Node& b = nd;
    const int q = (row & (np - 1)) << ps;
    const double px = M::add(cx, M::mul(r, c_proxy_cos[q]));
    const double py = M::add(cy, M::mul(r, c_proxy_sin[q]));
    const double r0 = M::sub(px, b.x), r1 = M::sub(py, b.y);
    if (row < np)
      return laplace_entry<FAST>(pde, r0, r1, b.w, 0.0, b.nx, b.ny, c_proxy_cos[q],
                                 c_proxy_sin[q]);
    return laplace_entry<FAST>(pde, -r0, -r1, pw, 0.0, c_proxy_cos[q], c_proxy_sin[q], b.nx,
                               b.ny);
  }
  const Node& s = nd;
  const int scomp = src & 1;
  const bool second = row >= 2 * np;
  const int rr_ = second ? row - 2 * np : row;
  const int q = (rr_ >> 1) << ps, comp = rr_ & 1;
  const double tn0 = c_proxy_cos[q], tn1 = c_proxy_sin[q];
  const double px = M::add(cx, M::mul(r, tn0));
  const double py = M::add(cy, M::mul(r, tn1));
  const double r0 = M::sub(px, s.x), r1 = M::sub(py, s.y);
  const double rr = M::add(M::mul(r0, r0), M::mul(r1, r1));
  const double rs = scomp ? r1 : r0;
  const double rc = comp ? r1 : r0;
  const double sns = scomp ? s.ny : s.nx;
  const double tnc = comp ? tn1 : tn0;
  if (!second) {
    const double pot = M::div(M::mul(M::mul(s.w, KI_INV_PI), M::add(M::mul(r0, s.nx), M::mul(r1, s.ny))),
                              M::mul(rr, rr));
    return M::add(M::mul(M::mul(pot, rc), rs), M::mul(M::mul(s.w, tnc), sns));
  }
  const double pot = M::div(M::mul(M::mul(-pw, KI_INV_PI), M::add(M::mul(r0, tn0), M::mul(r1, tn1))),
                            M::mul(rr, rr));
  return M::add(M::mul(M::mul(pot, rc), rs), M::mul(M::mul(pw, sns), tnc));
}

// The same with the box dof's node taken from the node array.
template <bool FAST = false>
__device__ __forceinline__ double proxy_entry(int pde, const Node* __restrict__ nodes,
                                              const double* __restrict__ dir,
                                              int row, int src, double cx, double cy,
                                              double r, double pw) {
  return proxy_entry_node<FAST>(pde, nodes[pde == kStokes ? src >> 1 : src], dir, row, src, cx,
                                cy, r, pw);
}

// Forward (target-point) entry of Kernel::forward (kernel.cpp:337-357) with
// target normal zero; tgt_comp is the velocity component for Stokes.
__device__ __forceinline__ double forward_entry(int pde, const Node* __restrict__ nodes,
                                                double tx, double ty, int tgt_comp,
                                                int src) {
  if (pde == kLaplace) {
    const Node s = nodes[src];
    return laplace_entry(kLaplace, subd(tx, s.x), subd(ty, s.y), s.w, s.k, s.nx, s.ny,
                         0.0, 0.0);
  }
  if (pde == kLaplaceNeumann) {
    const Node s = nodes[src];
    const double r1 = subd(tx, s.x), r2 = subd(ty, s.y);
    return mul(mul(s.w, KI_INV_2PI), log(sqrt(add(mul(r1, r1), mul(r2, r2)))));
  }
  const Node s = nodes[src >> 1];
  const int sc = src & 1;
  const double r0 = subd(tx, s.x), r1 = subd(ty, s.y);
  if (r0 == 0.0 && r1 == 0.0) {
    // target on a node: the diagonal formula with zero target normal
    const int parity = (tgt_comp + src + 1) & 1;
    const double snA = tgt_comp ? s.nx : s.ny;
    const double snB = sc ? s.nx : s.ny;
    const double b = mul(mul(mul(mul(mul(static_cast<double>(1 - 2 * parity), 0.5), s.k), s.w),
                             KI_INV_PI), snA);
    return add(mul(-0.5, static_cast<double>(parity)), mul(b, snB));
  }
  const double rr = add(mul(r0, r0), mul(r1, r1));
  const double pot = divd(mul(mul(s.w, KI_INV_PI), add(mul(r0, s.nx), mul(r1, s.ny))),
                          mul(rr, rr));
  return mul(mul(pot, tgt_comp ? r1 : r0), sc ? r1 : r0);
}

// Border columns for one target point (initialize_U_mat, linear_solve.cpp:18-64).
__device__ __forceinline__ void border_u(int pde, double tx, double ty, const double* hole, int comp,
                         double* out) {
  const double rx = tx - hole[0], ry = ty - hole[1];
  const double rn = sqrt(rx * rx + ry * ry);
  if (pde == kLaplace) {
    out[0] = log(rn);
    return;
  }
  const double scale = 1.0 / (4 * 3.14159265358979323846);
  const double inv2 = 1.0 / (rn * rn);
  const double lg = log(1 / rn);
  if (comp == 0) {
    out[0] = scale * (lg + inv2 * rx * rx);
    out[1] = scale * (inv2 * rx * ry);
    out[2] = ry * (scale * inv2);
  } else {
    out[0] = scale * (inv2 * ry * rx);
    out[1] = scale * (lg + inv2 * ry * ry);
    out[2] = -rx * (scale * inv2);
  }
}

}  // namespace kib

#endif  // KI_ENTRIES_CUH_
