// Host geometry of the engine: closed-curve evaluation and the exact
// axis-aligned boxes of spline pieces. Discretize's output depends on these
// boxes bit for bit (a piece is refined exactly when its closed box meets a
// box of another loop), so they follow the reference's arithmetic and
// evaluation order: src/curve.cpp:20-43 (bases), :156-184 (get_point),
// :197-277 (compute_box_1d), :293-324 (get_segment_bounding_box). This file
// is compiled with -ffp-contract=off so no product or sum is fused.
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

namespace fln {

struct Vec3 {
  double x, y, z;
};
inline Vec3 operator-(const Vec3 &a, const Vec3 &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }

// Closed-interval box; the default is empty (intersects nothing), like
// Eigen::AlignedBox's null box.
struct Box3 {
  double lo[3] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max(),
                  std::numeric_limits<double>::max()};
  double hi[3] = {-std::numeric_limits<double>::max(), -std::numeric_limits<double>::max(),
                  -std::numeric_limits<double>::max()};
};
inline bool overlaps(const Box3 &a, const Box3 &b) {
  return a.lo[0] <= b.hi[0] && a.lo[1] <= b.hi[1] && a.lo[2] <= b.hi[2] && b.lo[0] <= a.hi[0] &&
         b.lo[1] <= a.hi[1] && b.lo[2] <= a.hi[2];
}
inline double min_of(double a, double b) { return (b < a) ? b : a; }
inline double max_of(double a, double b) { return (a < b) ? b : a; }
inline void grow(Box3 &a, const Box3 &b) {
  for (int d = 0; d < 3; ++d) {
    a.lo[d] = min_of(a.lo[d], b.lo[d]);
    a.hi[d] = max_of(a.hi[d], b.hi[d]);
  }
}
inline double diag_length(const Box3 &b) {
  const double dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
  return std::sqrt(dx * dx + dy * dy + dz * dz);
}

enum SegKind : int { kBSpline = 0, kCatmullRom = 1, kBezier = 2, kPolyline = 3 };

// A curve of the model: control points (closed or open) and a segment kind.
struct CurveData {
  std::vector<Vec3> q;
  SegKind kind = kBSpline;
  bool closed = false;

  int segments() const {
    const int n = (int)q.size();
    if (closed) return n;
    return kind == kPolyline ? n - 1 : n - 3;
  }

  // Cubic coefficients (t^3, t^2, t, 1) of one coordinate of a spline segment
  // given its four control values; the monomial forms of curve.cpp:205-233.
  static void cubic(SegKind k, double q1, double q2, double q3, double q4, double c[4]) {
    if (k == kBSpline) {
      c[0] = -(1.0 / 6.0) * q1 + 0.5 * q2 - 0.5 * q3 + (1.0 / 6.0) * q4;
      c[1] = 0.5 * q1 - q2 + 0.5 * q3;
      c[2] = -0.5 * q1 + 0.5 * q3;
      c[3] = (1.0 / 6.0) * q1 + (2.0 / 3.0) * q2 + (1.0 / 6.0) * q3;
    } else if (k == kCatmullRom) {
      c[0] = -0.5 * q1 + 1.5 * q2 - 1.5 * q3 + 0.5 * q4;
      c[1] = 1.0 * q1 - 2.5 * q2 + 2.0 * q3 - 0.5 * q4;
      c[2] = -0.5 * q1 + 0.5 * q3;
      c[3] = 1.0 * q2;
    } else {
      c[0] = -1.0 * q1 + 3.0 * q2 - 3.0 * q3 + 1.0 * q4;
      c[1] = 3.0 * q1 - 6.0 * q2 + 3.0 * q3;
      c[2] = -3.0 * q1 + 3.0 * q2;
      c[3] = 1.0 * q1;
    }
  }

  // Point on segment `seg` at parameter t (Horner bases of curve.cpp:20-43).
  Vec3 at(int seg, double t) const {
    const size_t n = q.size();
    if (kind == kPolyline) {
      const Vec3 &s = q[seg], &e = q[(seg + 1) % n];
      const double u = 1.0 - t;
      return {u * s.x + t * e.x, u * s.y + t * e.y, u * s.z + t * e.z};
    }
    double B[4];
    if (kind == kBSpline) {
      B[0] = ((-(1.0 / 6) * t + (1.0 / 2)) * t - (1.0 / 2)) * t + (1.0 / 6);
      B[1] = ((1.0 / 2) * t - 1.0) * (t * t) + (2.0 / 3);
      B[2] = ((-(1.0 / 2) * t + (1.0 / 2)) * t + (1.0 / 2)) * t + (1.0 / 6);
      B[3] = (1.0 / 6) * (t * t) * t;
    } else if (kind == kCatmullRom) {
      B[0] = ((-0.5 * t + 1.0) * t - 0.5) * t;
      B[1] = (1.5 * t - 2.5) * (t * t) + 1.0;
      B[2] = ((-1.5 * t + 2.0) * t + 0.5) * t;
      B[3] = (0.5 * t - 0.5) * (t * t);
    } else {
      B[0] = ((-1.0 * t + 3.0) * t - 3.0) * t + 1.0;
      B[1] = ((3.0 * t - 6.0) * t + 3.0) * t;
      B[2] = (-3.0 * t + 3.0) * (t * t);
      B[3] = 1.0 * t * t * t;
    }
    const Vec3 &a = q[seg], &b = q[(seg + 1) % n], &c = q[(seg + 2) % n], &d = q[(seg + 3) % n];
    return {((B[0] * a.x + B[1] * b.x) + B[2] * c.x) + B[3] * d.x,
            ((B[0] * a.y + B[1] * b.y) + B[2] * c.y) + B[3] * d.y,
            ((B[0] * a.z + B[1] * b.z) + B[2] * c.z) + B[3] * d.z};
  }

  // Extent of one cubic coordinate over [t0, t1]: the endpoint values and any
  // interior stationary point (roots of the derivative by the stable
  // quadratic formula), as curve.cpp:234-276 evaluates them.
  static void extent(const double c[4], double t0, double t1, double &lo, double &hi) {
    auto ev = [&](double s) { return ((c[0] * s + c[1]) * s + c[2]) * s + c[3]; };
    lo = ev(t0);
    hi = ev(t1);
    if (hi < lo) {
      const double tmp = lo;
      lo = hi;
      hi = tmp;
    }
    auto take = [&](double s) {
      if (s >= t0 && s <= t1) {
        const double v = ev(s);
        lo = min_of(lo, v);
        hi = max_of(hi, v);
      }
    };
    const double disc = 4 * c[1] * c[1] - 12 * c[2] * c[0];
    if (disc == 0) {
      take(-2 * c[1] / (6 * c[0]));
      return;
    }
    const double rad = (c[1] >= 0) ? -2 * c[1] - std::sqrt(disc) : -2 * c[1] + std::sqrt(disc);
    take(rad / (6 * c[0]));
    take(2 * c[2] / rad);
  }

  Box3 piece_box(int seg, double t0 = 0.0, double t1 = 1.0) const {
    Box3 b;
    if (kind == kPolyline) {
      const Vec3 a = at(seg, t0), e = at(seg, t1);
      const double av[3] = {a.x, a.y, a.z}, ev[3] = {e.x, e.y, e.z};
      for (int d = 0; d < 3; ++d) {
        b.lo[d] = min_of(av[d], ev[d]);
        b.hi[d] = max_of(av[d], ev[d]);
      }
      return b;
    }
    const size_t n = q.size();
    const Vec3 &p0 = q[seg], &p1 = q[(seg + 1) % n], &p2 = q[(seg + 2) % n], &p3 = q[(seg + 3) % n];
    const double v[3][4] = {{p0.x, p1.x, p2.x, p3.x}, {p0.y, p1.y, p2.y, p3.y}, {p0.z, p1.z, p2.z, p3.z}};
    for (int d = 0; d < 3; ++d) {
      double c[4];
      cubic(kind, v[d][0], v[d][1], v[d][2], v[d][3], c);
      extent(c, t0, t1, b.lo[d], b.hi[d]);
    }
    return b;
  }

  Box3 whole_box() const {
    Box3 b;
    const int ns = segments();
    for (int s = 0; s < ns; ++s) grow(b, piece_box(s));
    return b;
  }
};

}  // namespace fln
