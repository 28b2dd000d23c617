// Test infrastructure only: the CPU oracle that checks the product.
//
// This is a plain C++17 + OpenMP restatement of the reference's CPU path for
// the linking-number hot path (antequ/fastlinkingnumbers, `verifycurves`).
// It is the checker and the timed CPU baseline. Nothing in the product
// (`fastlinkingnumbers_b200/`) links, imports or calls it; only `tests/`,
// `__graft_entry__.smoke()` and the CPU legs of `bench.py` do.
//
// Each routine cites the reference file:line it restates. Eigen is absent in
// this image, so the small 3-vector / box algebra the reference takes from
// Eigen 3.3 (dot, cross, norm = sqrt(squaredNorm), AlignedBox intersects /
// merged / center / sizes) is restated here with the same evaluation order.
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace fln_oracle {

struct V3 {
  double x = 0, y = 0, z = 0;
};
inline V3 operator+(const V3 &a, const V3 &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(const V3 &a, const V3 &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, const V3 &a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(const V3 &a, const V3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(const V3 &a, const V3 &b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
double norm(const V3 &a);

// Axis-aligned box with Eigen::AlignedBox semantics (closed intervals; the
// default box is "null": lo = +max, hi = lowest, so it intersects nothing).
struct Box {
  V3 lo{1.7976931348623157e308, 1.7976931348623157e308, 1.7976931348623157e308};
  V3 hi{-1.7976931348623157e308, -1.7976931348623157e308, -1.7976931348623157e308};
};
bool box_intersects(const Box &a, const Box &b);
Box box_merged(const Box &a, const Box &b);
V3 box_center(const Box &b);
double box_diag(const Box &b);  // sizes().norm()

enum class SegType : int { BSpline = 0, CatmullRom = 1, Bezier = 2, Polyline = 3 };

// include/curve.h:41-195, src/curve.cpp
struct Curve {
  std::vector<V3> q;
  SegType type = SegType::BSpline;
  bool looped = false;
  int num_segments() const;                                   // curve.h:61-66
  V3 point(int seg, double t) const;                          // curve.cpp:156-184
  Box seg_box(int seg, double tlo = 0.0, double thi = 1.0) const;  // curve.cpp:293-324
  Box curve_box() const;                                      // curve.cpp:331-343
  std::vector<V3> start_points() const;                       // curve.cpp:125-134
  std::vector<V3> midpoints() const;                          // curve.cpp:99-108
  std::vector<V3> tangents() const;                           // curve.cpp:110-123
};

// src/model.cpp:280-364 (BCC import; float32 -> double).
std::vector<Curve> load_bcc(const std::string &path);
void save_bcc(const std::string &path, const std::vector<Curve> &curves);

// src/ModifiedKdBVH.h:101-237 — kd-median tree over object boxes; objects
// are permuted, internal nodes numbered in construction order, root last.
struct KdTree {
  std::vector<int> children;  // 2 per internal node; >= nboxes means object
  std::vector<Box> boxes;     // internal node boxes
  std::vector<int> objects;   // permuted object ids (position -> original id)
  std::vector<Box> obj_boxes; // box of object at each position
  int nboxes() const { return (int)boxes.size(); }
  int root() const { return (int)boxes.size() - 1; }
  void build(const std::vector<Box> &boxes_in);
};

// src/potential_link_search.cpp:88-165.
std::vector<std::pair<int, int>> potential_links_unique(const std::vector<Curve> &curves);
std::vector<std::vector<int>> per_curve_symmetric(const std::vector<std::pair<int, int>> &u, int n);
std::vector<std::vector<int>> per_curve_unique(const std::vector<std::pair<int, int>> &u, int n);

// src/discretize.cpp:103-281. Throws std::runtime_error like the reference.
std::vector<Curve> discretize(const std::vector<Curve> &curves,
                              const std::vector<std::vector<int>> &links, int *rounds_out = nullptr);

// src/compute_link.cpp:126-178 and :200-280.
double direct_one_arctan(const Curve &c1, const Curve &c2, bool parallel);
double direct_fast(const Curve &c1, const Curve &c2);

// src/compute_link.h:95-114
struct Moment {
  double q0[9] = {0}, q1[9] = {0}, q2[9] = {0};  // row-major 3x3
  double dip[9] = {0};                           // row-major 3x3
  V3 tan, mid;
  double tannorm = 0, dipnorm = 0, quadnorm = 0;
};

struct SegTree {
  KdTree kd;                 // objects are segment ids
  std::vector<Moment> mom;   // nboxes internal + n leaves
};
// src/compute_link.cpp:295-389
SegTree make_seg_tree(const Curve &c);
// src/compute_link.cpp:547-666 + :695-934. `as_float` reproduces the
// reference's serial path returning through a float (compute_link.cpp:927).
double bh_eval(const SegTree &t1, const SegTree &t2, double epssq, double itolsq, double &err,
               bool parallel, uint64_t *far_count = nullptr, uint64_t *leaf_count = nullptr);

// The product's curve-order tree (no counterpart in the reference): node =
// contiguous segment range; internal id = split - 1, leaf id = n - 1 + segment.
struct CurveTree {
  int n = 0, root = 0;
  std::vector<int> lo, cnt, left, right;  // left < 0: leaf
  std::vector<Box> box;
  std::vector<Moment> mom;
};
CurveTree make_curve_tree(const Curve &c);
// One Barnes–Hut pass over the two curve-order trees at itolsq = beta^2;
// node pairs of at most `bucket` segments a side are summed exactly.
double curve_bh_eval(const CurveTree &t1, const CurveTree &t2, double epssq, double itolsq, int bucket,
                     double &err, uint64_t *far_count = nullptr, uint64_t *exact_count = nullptr);
// The same pass at itolsq1, continued from an itolsq0 pass's far node pairs
// and reusing its exact terms (the node pairs are the same).
double curve_bh_eval_continued(const CurveTree &t1, const CurveTree &t2, double epssq, double itolsq0,
                               double itolsq1, int bucket, double &err, uint64_t *far_count = nullptr,
                               uint64_t *exact_count = nullptr);

struct PairResult {
  int i, j;
  double lk;
  double err;  // BH error estimate after scaling (0 for direct sum)
};

// src/linking_number_certificate.cpp:102-229, :241-338, :358-394.
struct Certificate {
  int ncurves = 0;
  std::vector<std::pair<std::pair<int, int>, int>> entries;  // ((i,j),lk) i<j, sorted
  std::vector<PairResult> pairs;
  double mean_off = 0, max_off = 0;
  std::string text() const;  // lnc.cpp:441-454
};
Certificate compute_certificate(const std::vector<Curve> &model, bool direct, bool disc,
                                double beta0, double betamax,
                                std::vector<Curve> *discretized_out = nullptr);

}  // namespace fln_oracle
