// Host geometry of the engine: closed-curve evaluation and the exact
// axis-aligned boxes of spline pieces. Discretize's output depends on these
// boxes bit for bit (a piece is refined exactly when its closed box meets a
// box of another loop), so they follow the reference's arithmetic and
// evaluation order: src/curve.cpp:20-43 (bases), :156-184 (get_point),
// :197-277 (compute_box_1d), :293-324 (get_segment_bounding_box). This file
// is compiled with -ffp-contract=off so no product or sum is fused.
//
// The raw piece functions (seg_point, seg_box) are also compiled for the GPU
// (discretize.cu, built with --fmad=false; CUDA's division and square root
// are correctly rounded), so the device Discretize reproduces these boxes
// bit for bit.
#pragma once

#ifdef __CUDACC__
#define FLN_HD __host__ __device__
#else
#define FLN_HD
#endif

#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

namespace fln {

struct Vec3 {
  double x, y, z;
};
static_assert(sizeof(Vec3) == 3 * sizeof(double), "Vec3 is three packed doubles");
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
FLN_HD inline double min_of(double a, double b) { return (b < a) ? b : a; }
FLN_HD inline double max_of(double a, double b) { return (a < b) ? b : a; }
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

// Cubic coefficients (t^3, t^2, t, 1) of one coordinate of a spline segment
// given its four control values; the monomial forms of curve.cpp:205-233.
FLN_HD inline void seg_cubic(int k, double q1, double q2, double q3, double q4, double c[4]) {
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

// Point on segment `seg` of a curve with n control points q (3 doubles
// each) at parameter t (Horner bases of curve.cpp:20-43).
FLN_HD inline void seg_point(int kind, const double *q, int64_t n, int64_t seg, double t, double out[3]) {
  if (kind == kPolyline) {
    const double *s = q + 3 * seg, *e = q + 3 * ((seg + 1) % n);
    const double u = 1.0 - t;
    for (int d = 0; d < 3; ++d) out[d] = u * s[d] + t * e[d];
    return;
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
  const double *a = q + 3 * seg, *b = q + 3 * ((seg + 1) % n), *c = q + 3 * ((seg + 2) % n),
               *dd = q + 3 * ((seg + 3) % n);
  for (int d = 0; d < 3; ++d) out[d] = ((B[0] * a[d] + B[1] * b[d]) + B[2] * c[d]) + B[3] * dd[d];
}

// Extent of one cubic coordinate over [t0, t1]: the endpoint values and any
// interior stationary point (roots of the derivative by the stable
// quadratic formula), as curve.cpp:234-276 evaluates them.
FLN_HD inline double cubic_at(const double c[4], double s) { return ((c[0] * s + c[1]) * s + c[2]) * s + c[3]; }
FLN_HD inline void cubic_take(const double c[4], double s, double t0, double t1, double &lo, double &hi) {
  if (s >= t0 && s <= t1) {
    const double v = cubic_at(c, s);
    lo = min_of(lo, v);
    hi = max_of(hi, v);
  }
}
FLN_HD inline void cubic_extent(const double c[4], double t0, double t1, double &lo, double &hi) {
  lo = cubic_at(c, t0);
  hi = cubic_at(c, t1);
  if (hi < lo) {
    const double tmp = lo;
    lo = hi;
    hi = tmp;
  }
  const double disc = 4 * c[1] * c[1] - 12 * c[2] * c[0];
  if (disc == 0) {
    cubic_take(c, -2 * c[1] / (6 * c[0]), t0, t1, lo, hi);
    return;
  }
  const double rad = (c[1] >= 0) ? -2 * c[1] - sqrt(disc) : -2 * c[1] + sqrt(disc);
  cubic_take(c, rad / (6 * c[0]), t0, t1, lo, hi);
  cubic_take(c, 2 * c[2] / rad, t0, t1, lo, hi);
}

// Closed box of piece [t0, t1] of segment `seg` (curve.cpp:293-324).
FLN_HD inline void seg_box(int kind, const double *q, int64_t n, int64_t seg, double t0, double t1, double lo[3],
                           double hi[3]) {
  if (kind == kPolyline) {
    double a[3], e[3];
    seg_point(kind, q, n, seg, t0, a);
    seg_point(kind, q, n, seg, t1, e);
    for (int d = 0; d < 3; ++d) {
      lo[d] = min_of(a[d], e[d]);
      hi[d] = max_of(a[d], e[d]);
    }
    return;
  }
  const double *p0 = q + 3 * seg, *p1 = q + 3 * ((seg + 1) % n), *p2 = q + 3 * ((seg + 2) % n),
               *p3 = q + 3 * ((seg + 3) % n);
  for (int d = 0; d < 3; ++d) {
    double c[4];
    seg_cubic(kind, p0[d], p1[d], p2[d], p3[d], c);
    cubic_extent(c, t0, t1, lo[d], hi[d]);
  }
}

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

  // Point on segment `seg` at parameter t.
  Vec3 at(int seg, double t) const {
    double o[3];
    seg_point(kind, &q[0].x, (int64_t)q.size(), seg, t, o);
    return {o[0], o[1], o[2]};
  }

  Box3 piece_box(int seg, double t0 = 0.0, double t1 = 1.0) const {
    Box3 b;
    seg_box(kind, &q[0].x, (int64_t)q.size(), seg, t0, t1, b.lo, b.hi);
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
