// Boundary data helpers and the analytic test boundaries of the C++ drop-in
// API (kern_interp/boundaries/boundary.cpp, circle.cpp, annulus.cpp,
// donut.cpp of the reference): the same node placement, normals,
// curvatures, trapezoid weights, boundary conditions and domain tests.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "kern_interp/boundaries/annulus.h"
#include "kern_interp/boundaries/boundary.h"
#include "kern_interp/boundaries/circle.h"
#include "kern_interp/boundaries/donut.h"

namespace kern_interp {

namespace {

bool vector_condition(BoundaryCondition bc) {
  switch (bc) {
    case TANGENT_VEC:
    case REVERSE_TANGENT_VEC:
    case NORMAL_VEC:
    case REVERSE_NORMAL_VEC:
    case LEFT_TO_RIGHT_FLOW:
    case EX3B:
    case HORIZONTAL_VEC:
    case NO_SLIP:
      return true;
    default:
      return false;
  }
}

// Nodes of an outer unit circle about (0.5, 0.5) followed by each hole's
// circle (normals pointing out of the domain: inward on the holes, curvature
// -1/r), hole_nodes = N / 5 per hole (annulus.cpp:9-51, donut.cpp:9-51).
void circle_with_holes(Boundary* b, int N) {
  b->points.clear();
  b->normals.clear();
  b->weights.clear();
  b->curvatures.clear();
  for (int i = 0; i < N; i++) {
    const double ang = i * 2.0 * M_PI / N;
    b->points.push_back(0.5 + std::cos(ang));
    b->points.push_back(0.5 + std::sin(ang));
    b->normals.push_back(std::cos(ang));
    b->normals.push_back(std::sin(ang));
    b->curvatures.push_back(1);
    b->weights.push_back(2 * M_PI / N);
  }
  const int hn = N / 5;
  for (size_t h = 0; h < b->holes.size(); h++) {
    const Hole hole = b->holes[h];
    for (int q = 0; q < hn; q++) {
      const double ang = q * 2.0 * M_PI / hn;
      b->points.push_back(hole.center.a[0] + hole.radius * std::cos(ang));
      b->points.push_back(hole.center.a[1] + hole.radius * std::sin(ang));
      b->normals.push_back(-std::cos(ang));
      b->normals.push_back(-std::sin(ang));
      b->curvatures.push_back(-1.0 / hole.radius);
      b->weights.push_back((2 * hole.radius * M_PI) / hn);
    }
  }
}

bool outside_holes(const std::vector<Hole>& holes, const Vec2& a, double eps) {
  for (const Hole& hole : holes)
    if ((a - hole.center).norm() - eps < hole.radius) return false;
  return true;
}

}  // namespace

void Boundary::set_boundary_values_size(BoundaryCondition bc) {
  if (bc == DEFAULT) {
    std::fprintf(stderr, "set_boundary_values_size: DEFAULT names the boundary's own data\n");
    std::exit(-1);
  }
  const int n = static_cast<int>(weights.size());
  boundary_values = ki_Mat(vector_condition(bc) ? 2 * n : n, 1);
}

void Boundary::apply_boundary_condition(int start_idx, int end_idx, BoundaryCondition bc) {
  for (int p = start_idx; p < end_idx; p++) {
    const double x = points[2 * p], y = points[2 * p + 1];
    const double nx = normals[2 * p], ny = normals[2 * p + 1];
    switch (bc) {
      case SINGLE_ELECTRON:
        // potential of a unit charge at (-3, -2)
        boundary_values.set(p, 0,
                            std::log(std::sqrt(std::pow(x + 3, 2) + std::pow(y + 2, 2))) /
                                (2 * M_PI));
        break;
      case ALL_ONES:
        boundary_values.set(p, 0, 1.0);
        break;
      case ALL_NEG_ONES:
        boundary_values.set(p, 0, -1.0);
        break;
      case ALL_ZEROS:
        boundary_values.set(p, 0, 0.0);
        break;
      case TANGENT_VEC:
        boundary_values.set(2 * p, 0, -ny);
        boundary_values.set(2 * p + 1, 0, nx);
        break;
      case REVERSE_TANGENT_VEC:
        boundary_values.set(2 * p, 0, ny);
        boundary_values.set(2 * p + 1, 0, -nx);
        break;
      case NORMAL_VEC:
        boundary_values.set(2 * p, 0, nx);
        boundary_values.set(2 * p + 1, 0, ny);
        break;
      case REVERSE_NORMAL_VEC:
        boundary_values.set(2 * p, 0, -nx);
        boundary_values.set(2 * p + 1, 0, -ny);
        break;
      case HORIZONTAL_VEC:
        boundary_values.set(2 * p, 0, 1.0);
        boundary_values.set(2 * p + 1, 0, 0.0);
        break;
      case LEFT_TO_RIGHT_FLOW: {
        const bool inflow = x < -0.99 || x > 1.99;
        boundary_values.set(2 * p, 0, inflow ? 1.0 : 0.0);
        boundary_values.set(2 * p + 1, 0, 0.0);
        break;
      }
      case NO_SLIP:
        boundary_values.set(2 * p, 0, 0.0);
        boundary_values.set(2 * p + 1, 0, 0.0);
        break;
      default:
        std::fprintf(stderr, "apply_boundary_condition: condition %d is an experiment's own\n",
                     static_cast<int>(bc));
        std::exit(-1);
    }
  }
}

// circle.cpp:9-34: radius 0.25 about (0.5, 0.5)
void Circle::initialize(int N, BoundaryCondition bc) {
  points.clear();
  normals.clear();
  weights.clear();
  curvatures.clear();
  for (int i = 0; i < N; i++) {
    const double ang = i * 2.0 * M_PI / N;
    points.push_back(0.5 + 0.25 * std::cos(ang));
    points.push_back(0.5 + 0.25 * std::sin(ang));
    normals.push_back(std::cos(ang));
    normals.push_back(std::sin(ang));
    curvatures.push_back(4);
    weights.push_back(M_PI / (N * 2));
  }
  if (bc == DEFAULT) {
    boundary_values = ki_Mat(N, 1);
    apply_boundary_condition(0, N, SINGLE_ELECTRON);
  } else {
    set_boundary_values_size(bc);
    apply_boundary_condition(0, N, bc);
  }
}

bool Circle::is_in_domain(const Vec2& a) const {
  const double x = a.a[0] - 0.5, y = a.a[1] - 0.5;
  return !(std::sqrt(std::pow(x, 2) + std::pow(y, 2)) + 1e-2 > 0.25);
}

// annulus.cpp:9-65: two holes of radius 0.2 at (0.9, 0.5) and (0.1, 0.5)
void Annulus::initialize(int N, BoundaryCondition bc) {
  if (holes.empty()) {
    Hole hole;
    hole.center = Vec2(0.9, 0.5);
    hole.radius = 0.2;
    hole.num_nodes = N / 5;
    holes.push_back(hole);
    hole.center = Vec2(0.1, 0.5);
    holes.push_back(hole);
  }
  circle_with_holes(this, N);
  const int hn = N / 5;
  const int total = N + hn * static_cast<int>(holes.size());
  if (bc == DEFAULT) {
    boundary_values = ki_Mat(total, 1);
    apply_boundary_condition(0, N, ALL_ZEROS);
    apply_boundary_condition(N, N + hn, ALL_ONES);
    apply_boundary_condition(N + hn, N + 2 * hn, ALL_NEG_ONES);
  } else {
    set_boundary_values_size(bc);
    apply_boundary_condition(0, total, bc);
  }
}

bool Annulus::is_in_domain(const Vec2& a) const {
  const double x = a.a[0] - 0.5, y = a.a[1] - 0.5;
  if (std::sqrt(std::pow(x, 2) + std::pow(y, 2)) + 1e-2 > 1) return false;
  return outside_holes(holes, a, 1e-2);
}

// donut.cpp:9-65: one hole of radius 0.5 at the centre
void Donut::initialize(int N, BoundaryCondition bc) {
  if (holes.empty()) {
    Hole hole;
    hole.center = Vec2(0.5, 0.5);
    hole.radius = 0.5;
    hole.num_nodes = N / 5;
    holes.push_back(hole);
  }
  circle_with_holes(this, N);
  const int hn = N / 5;
  const int total = N + hn * static_cast<int>(holes.size());
  if (bc == DEFAULT) {
    boundary_values = ki_Mat(total, 1);
    for (int i = 0; i < N; i++) boundary_values.set(i, 0, 1);
    for (int i = N; i < total; i++) boundary_values.set(i, 0, -1. / holes[0].radius);
  } else {
    set_boundary_values_size(bc);
    apply_boundary_condition(0, total, bc);
  }
}

bool Donut::is_in_domain(const Vec2& a) const {
  const double x = a.a[0] - 0.5, y = a.a[1] - 0.5;
  if (std::sqrt(std::pow(x, 2) + std::pow(y, 2)) + 1e-2 > 1) return false;
  return outside_holes(holes, a, 1e-2);
}

}  // namespace kern_interp
