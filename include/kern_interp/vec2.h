// C++ drop-in API of the B200 solver: kern_interp::Vec2.
// Same type and members as the reference's kern_interp/vec2.h:6-17.
#ifndef KERN_INTERP_VEC2_H_
#define KERN_INTERP_VEC2_H_

#include <cmath>

namespace kern_interp {

struct Vec2 {
  double a[2];

  Vec2() : a{0.0, 0.0} {}
  Vec2(double m, double n) : a{m, n} {}
  double norm() const { return std::sqrt(a[0] * a[0] + a[1] * a[1]); }
  double dot(const Vec2& o) const { return a[0] * o.a[0] + a[1] * o.a[1]; }
  Vec2 operator-(const Vec2& o) const { return Vec2(a[0] - o.a[0], a[1] - o.a[1]); }
  Vec2 operator*(const double d) const { return Vec2(a[0] * d, a[1] * d); }
};

}  // namespace kern_interp

#endif  // KERN_INTERP_VEC2_H_
