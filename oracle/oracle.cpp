// Test infrastructure only: CPU restatement of the reference's linking-number
// path, used as the checker for the product and as the timed CPU baseline.
// See oracle.hpp for the scope rules. Citations are to files of
// antequ/fastlinkingnumbers.
#include "oracle.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <tuple>
#include <unordered_set>

namespace fln_oracle {

// compute_link.cpp:11-18
static const double kInvRt3 = 0.5773502691896257645091487805019574556476017512701268760186023264;
static const double kInvTwoPi = 0.1591549430918953357688837633725143620344596457404564487476673440;
static const double kInvFourPi = 0.0795774715459476678844418816862571810172298228702282243738336720;
static const double kFourPi = 12.566370614359172953850573533118011536788677597500423283899778369;

double norm(const V3 &a) { return std::sqrt(dot(a, a)); }

bool box_intersects(const Box &a, const Box &b) {
  return a.lo.x <= b.hi.x && a.lo.y <= b.hi.y && a.lo.z <= b.hi.z && b.lo.x <= a.hi.x &&
         b.lo.y <= a.hi.y && b.lo.z <= a.hi.z;
}
static inline double mn(double a, double b) { return (b < a) ? b : a; }  // std::min
static inline double mx(double a, double b) { return (a < b) ? b : a; }  // std::max
Box box_merged(const Box &a, const Box &b) {
  Box r;
  r.lo = {mn(a.lo.x, b.lo.x), mn(a.lo.y, b.lo.y), mn(a.lo.z, b.lo.z)};
  r.hi = {mx(a.hi.x, b.hi.x), mx(a.hi.y, b.hi.y), mx(a.hi.z, b.hi.z)};
  return r;
}
V3 box_center(const Box &b) {
  return {(b.lo.x + b.hi.x) / 2.0, (b.lo.y + b.hi.y) / 2.0, (b.lo.z + b.hi.z) / 2.0};
}
double box_diag(const Box &b) { return norm(b.hi - b.lo); }

// ---------------------------------------------------------------- curves
// Spline bases in the Horner forms of curve.cpp:20-43.
static void basis(SegType t, double s, double *B) {
  if (t == SegType::BSpline) {
    B[0] = ((-(1.0 / 6) * s + (1.0 / 2)) * s - (1.0 / 2)) * s + (1.0 / 6);
    B[1] = ((1.0 / 2) * s - 1.0) * (s * s) + (2.0 / 3);
    B[2] = ((-(1.0 / 2) * s + (1.0 / 2)) * s + (1.0 / 2)) * s + (1.0 / 6);
    B[3] = (1.0 / 6) * (s * s) * s;
  } else if (t == SegType::CatmullRom) {
    B[0] = ((-0.5 * s + 1.0) * s - 0.5) * s;
    B[1] = (1.5 * s - 2.5) * (s * s) + 1.0;
    B[2] = ((-1.5 * s + 2.0) * s + 0.5) * s;
    B[3] = (0.5 * s - 0.5) * (s * s);
  } else {
    B[0] = ((-1.0 * s + 3.0) * s - 3.0) * s + 1.0;
    B[1] = ((3.0 * s - 6.0) * s + 3.0) * s;
    B[2] = (-3.0 * s + 3.0) * (s * s);
    B[3] = 1.0 * s * s * s;
  }
}

int Curve::num_segments() const {
  const int n = (int)q.size();
  if (looped) return n;
  return type == SegType::Polyline ? n - 1 : n - 3;
}

V3 Curve::point(int seg, double t) const {
  if (t < 0.0 || t > 1.0 || seg < 0 || seg >= num_segments())
    throw std::runtime_error("Curve::get_point() has an invalid i or t.");
  const size_t n = q.size();
  if (type == SegType::Polyline) {
    const V3 &s = q[seg], &e = q[(seg + 1) % n];
    return (1.0 - t) * s + t * e;
  }
  double B[4];
  basis(type, t, B);
  const V3 &q0 = q[seg], &q1 = q[(seg + 1) % n], &q2 = q[(seg + 2) % n], &q3 = q[(seg + 3) % n];
  return ((B[0] * q0 + B[1] * q1) + B[2] * q2) + B[3] * q3;
}

// curve.cpp:197-277 — exact extent of one cubic coordinate over [t0, t1].
static void box_1d(SegType t, double q1, double q2, double q3, double q4, double t0, double t1,
                   double &lo, double &hi) {
  double x0, x1, x2, x3;
  if (t == SegType::BSpline) {
    x0 = -(1.0 / 6.0) * q1 + 0.5 * q2 - 0.5 * q3 + (1.0 / 6.0) * q4;
    x1 = 0.5 * q1 - q2 + 0.5 * q3;
    x2 = -0.5 * q1 + 0.5 * q3;
    x3 = (1.0 / 6.0) * q1 + (2.0 / 3.0) * q2 + (1.0 / 6.0) * q3;
  } else if (t == SegType::CatmullRom) {
    x0 = -0.5 * q1 + 1.5 * q2 - 1.5 * q3 + 0.5 * q4;
    x1 = 1.0 * q1 - 2.5 * q2 + 2.0 * q3 - 0.5 * q4;
    x2 = -0.5 * q1 + 0.5 * q3;
    x3 = 1.0 * q2;
  } else {
    x0 = -1.0 * q1 + 3.0 * q2 - 3.0 * q3 + 1.0 * q4;
    x1 = 3.0 * q1 - 6.0 * q2 + 3.0 * q3;
    x2 = -3.0 * q1 + 3.0 * q2;
    x3 = 1.0 * q1;
  }
  auto ev = [&](double s) { return ((x0 * s + x1) * s + x2) * s + x3; };
  lo = ev(t0);
  hi = ev(t1);
  if (hi < lo) std::swap(lo, hi);
  auto take = [&](double s) {
    if (s >= t0 && s <= t1) {
      double v = ev(s);
      lo = mn(lo, v);
      hi = mx(hi, v);
    }
  };
  const double disc = 4 * x1 * x1 - 12 * x2 * x0;
  if (disc == 0) {
    take(-2 * x1 / (6 * x0));
  } else {
    double radical;
    if (x1 >= 0) {
      radical = -2 * x1 - std::sqrt(disc);
    } else {
      radical = -2 * x1 + std::sqrt(disc);
    }
    take(radical / (6 * x0));
    take(2 * x2 / radical);
  }
}

Box Curve::seg_box(int seg, double tlo, double thi) const {
  if (seg < 0 || seg >= num_segments() || tlo < 0 || thi > 1 || tlo > thi)
    throw std::runtime_error("Curve::get_segment_bounding_box() has an invalid i or t.");
  Box b;
  if (type == SegType::Polyline) {
    const V3 a = point(seg, tlo), c = point(seg, thi);
    b.lo = {mn(a.x, c.x), mn(a.y, c.y), mn(a.z, c.z)};
    b.hi = {mx(a.x, c.x), mx(a.y, c.y), mx(a.z, c.z)};
  } else {
    const size_t n = q.size();
    const V3 &q0 = q[seg], &q1 = q[(seg + 1) % n], &q2 = q[(seg + 2) % n], &q3 = q[(seg + 3) % n];
    box_1d(type, q0.x, q1.x, q2.x, q3.x, tlo, thi, b.lo.x, b.hi.x);
    box_1d(type, q0.y, q1.y, q2.y, q3.y, tlo, thi, b.lo.y, b.hi.y);
    box_1d(type, q0.z, q1.z, q2.z, q3.z, tlo, thi, b.lo.z, b.hi.z);
  }
  return b;
}

Box Curve::curve_box() const {
  const int ns = num_segments();
  if (ns <= 0) return Box();
  Box b = seg_box(0);
  for (int i = 1; i < ns; ++i) b = box_merged(b, seg_box(i));
  return b;
}

std::vector<V3> Curve::start_points() const {
  if (!looped) throw std::runtime_error("Curve::GetStartPoints() does not support unlooped curves.");
  std::vector<V3> r(q.size());
  for (size_t i = 0; i < q.size(); ++i) r[i] = point((int)i, 0.0);
  return r;
}
std::vector<V3> Curve::midpoints() const {
  if (!looped) throw std::runtime_error("Curve::GetMidpoints() does not support unlooped curves.");
  std::vector<V3> r(q.size());
  for (size_t i = 0; i < q.size(); ++i) r[i] = point((int)i, 0.5);
  return r;
}
std::vector<V3> Curve::tangents() const {
  std::vector<V3> s = start_points();
  const size_t n = s.size();
  std::vector<V3> t(n);
  for (size_t i = 0; i + 1 < n; ++i) t[i] = s[i + 1] - s[i];
  if (n) t[n - 1] = s[0] - s[n - 1];
  return t;
}

// ---------------------------------------------------------------- BCC I/O
#pragma pack(push, 1)
struct BccHeader {  // model.cpp:268-277
  char sign[3];
  unsigned char byte_count;
  char curve_type[2];
  char dimensions;
  char up_dimension;
  uint64_t curve_count;
  uint64_t total_points;
  char info[40];
};
#pragma pack(pop)
static_assert(sizeof(BccHeader) == 64, "BCC header is 64 bytes");

std::vector<Curve> load_bcc(const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("Unable to load BCC file.");
  BccHeader h;
  if (std::fread(&h, sizeof h, 1, f) != 1 || h.sign[0] != 'B' || h.sign[1] != 'C' ||
      h.sign[2] != 'C' || h.byte_count != 0x44 || h.dimensions != 3) {
    std::fclose(f);
    throw std::runtime_error("Unable to load BCC file.");
  }
  SegType t;
  if (h.curve_type[0] == 'C' && h.curve_type[1] == '0') t = SegType::CatmullRom;
  else if (h.curve_type[0] == 'B' && h.curve_type[1] == 'S') t = SegType::BSpline;
  else if (h.curve_type[0] == 'B' && h.curve_type[1] == 'Z') t = SegType::Bezier;
  else if (h.curve_type[0] == 'P' && h.curve_type[1] == 'L') t = SegType::Polyline;
  else {
    std::fclose(f);
    throw std::runtime_error("Unable to load BCC file.");
  }
  std::vector<Curve> curves;
  std::vector<float> buf;
  for (uint64_t i = 0; i < h.curve_count; ++i) {
    int32_t cnt;
    if (std::fread(&cnt, 4, 1, f) != 1) {
      std::fclose(f);
      throw std::runtime_error("Unable to load BCC file.");
    }
    Curve c;
    c.type = t;
    c.looped = cnt < 0;
    int64_t n = cnt < 0 ? -(int64_t)cnt : cnt;
    buf.resize(3 * n);
    if (n && std::fread(buf.data(), 4, 3 * n, f) != (size_t)(3 * n)) {
      std::fclose(f);
      throw std::runtime_error("Unable to load BCC file.");
    }
    c.q.resize(n);
    for (int64_t k = 0; k < n; ++k) c.q[k] = {(double)buf[3 * k], (double)buf[3 * k + 1], (double)buf[3 * k + 2]};
    curves.push_back(std::move(c));
  }
  std::fclose(f);
  return curves;
}

void save_bcc(const std::string &path, const std::vector<Curve> &curves) {
  BccHeader h;
  std::memset(&h, 0, sizeof h);
  h.sign[0] = 'B';
  h.sign[1] = 'C';
  h.sign[2] = 'C';
  h.byte_count = 0x44;
  const char *tc = "C0";
  if (!curves.empty()) {
    switch (curves[0].type) {
      case SegType::BSpline: tc = "BS"; break;
      case SegType::Bezier: tc = "BZ"; break;
      case SegType::Polyline: tc = "PL"; break;
      default: tc = "C0";
    }
  }
  h.curve_type[0] = tc[0];
  h.curve_type[1] = tc[1];
  h.dimensions = 3;
  h.up_dimension = 1;
  h.curve_count = curves.size();
  for (auto &c : curves) h.total_points += c.q.size();
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("Unable to export BCC file.");
  std::fwrite(&h, sizeof h, 1, f);
  std::vector<float> buf;
  for (auto &c : curves) {
    int32_t cnt = (int32_t)c.q.size();
    if (c.looped) cnt = -cnt;
    std::fwrite(&cnt, 4, 1, f);
    buf.resize(3 * c.q.size());
    for (size_t k = 0; k < c.q.size(); ++k) {
      buf[3 * k] = (float)c.q[k].x;
      buf[3 * k + 1] = (float)c.q[k].y;
      buf[3 * k + 2] = (float)c.q[k].z;
    }
    if (!buf.empty()) std::fwrite(buf.data(), 4, buf.size(), f);
  }
  std::fclose(f);
}

// ---------------------------------------------------------------- kd tree
// ModifiedKdBVH.h:101-132 (init) and :207-237 (build). The partition is
// std::nth_element on box centres along dim, cycling x, y, z per level, with
// the special case of 3 objects (2 + 1). Internal nodes are numbered in the
// order they are completed; object children are encoded as (n - 1) + position.
void KdTree::build(const std::vector<Box> &in) {
  const int n = (int)in.size();
  children.clear();
  boxes.clear();
  objects.resize(n);
  std::iota(objects.begin(), objects.end(), 0);
  obj_boxes = in;
  if (n < 2) return;
  std::vector<V3> centre(n);
  for (int i = 0; i < n; ++i) centre[i] = box_center(in[i]);
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  boxes.reserve(n - 1);
  children.reserve(2 * n - 2);
  auto coord = [&](int id, int dim) {
    const V3 &c = centre[id];
    return dim == 0 ? c.x : (dim == 1 ? c.y : c.z);
  };
  // Explicit recursion mirrors the reference's post-order numbering.
  struct Rec {
    KdTree *self;
    const std::vector<Box> &in;
    std::vector<int> &idx;
    decltype(coord) &cd;
    int n;
    void go(int from, int to, int dim) {
      const int size = to - from;
      auto cmp = [&](int a, int b) { return cd(a, dim) < cd(b, dim); };
      if (size == 2) {
        self->boxes.push_back(box_merged(in[idx[from]], in[idx[from + 1]]));
        self->children.push_back(from + n - 1);
        self->children.push_back(from + n);
      } else if (size == 3) {
        const int mid = from + 2;
        std::nth_element(idx.begin() + from, idx.begin() + mid, idx.begin() + to, cmp);
        go(from, mid, (dim + 1) % 3);
        const int i1 = (int)self->boxes.size() - 1;
        self->boxes.push_back(box_merged(self->boxes[i1], in[idx[mid]]));
        self->children.push_back(i1);
        self->children.push_back(mid + n - 1);
      } else {
        const int mid = from + size / 2;
        std::nth_element(idx.begin() + from, idx.begin() + mid, idx.begin() + to, cmp);
        go(from, mid, (dim + 1) % 3);
        const int i1 = (int)self->boxes.size() - 1;
        go(mid, to, (dim + 1) % 3);
        const int i2 = (int)self->boxes.size() - 1;
        self->boxes.push_back(box_merged(self->boxes[i1], self->boxes[i2]));
        self->children.push_back(i1);
        self->children.push_back(i2);
      }
    }
  } rec{this, in, idx, coord, n};
  rec.go(0, n, 0);
  for (int p = 0; p < n; ++p) {
    objects[p] = idx[p];
    obj_boxes[p] = in[idx[p]];
  }
}

// All (object of t1, object of t2) position pairs whose boxes intersect; the
// set is what Eigen's BVIntersect (BVAlgorithms.h:95-145) reaches, because
// merged parent boxes contain their children exactly.
template <class F>
static void kd_overlap(const KdTree &t1, const KdTree &t2, F &&emit) {
  const int n1 = (int)t1.objects.size(), n2 = (int)t2.objects.size();
  if (!n1 || !n2) return;
  const int nb1 = t1.nboxes(), nb2 = t2.nboxes();
  auto box1 = [&](int id) -> const Box & { return id < nb1 ? t1.boxes[id] : t1.obj_boxes[id - nb1]; };
  auto box2 = [&](int id) -> const Box & { return id < nb2 ? t2.boxes[id] : t2.obj_boxes[id - nb2]; };
  // n == 1 trees have no internal node; their root is object position 0.
  const int r1 = n1 == 1 ? nb1 : t1.root(), r2 = n2 == 1 ? nb2 : t2.root();
  std::vector<std::pair<int, int>> todo{{r1, r2}};
  while (!todo.empty()) {
    auto [a, b] = todo.back();
    todo.pop_back();
    if (!box_intersects(box1(a), box2(b))) continue;
    const bool la = a >= nb1, lb = b >= nb2;
    if (la && lb) {
      emit(a - nb1, b - nb2);
    } else if (la) {
      todo.push_back({a, t2.children[2 * b]});
      todo.push_back({a, t2.children[2 * b + 1]});
    } else if (lb) {
      todo.push_back({t1.children[2 * a], b});
      todo.push_back({t1.children[2 * a + 1], b});
    } else {
      for (int x = 0; x < 2; ++x)
        for (int y = 0; y < 2; ++y) todo.push_back({t1.children[2 * a + x], t2.children[2 * b + y]});
    }
  }
}

// ---------------------------------------------------------------- PLS
// potential_link_search.cpp:88-127: the sorted set of (i < j) with
// intersecting whole-curve boxes (both the KdBVH and the O(n^2) branches
// produce exactly this set).
std::vector<std::pair<int, int>> potential_links_unique(const std::vector<Curve> &curves) {
  const int n = (int)curves.size();
  std::vector<Box> b(n);
#pragma omp parallel for
  for (int i = 0; i < n; ++i) b[i] = curves[i].curve_box();
  std::vector<std::pair<int, int>> out;
  if (n >= 50) {
    KdTree t;
    t.build(b);
    kd_overlap(t, t, [&](int pa, int pb) {
      const int i = t.objects[pa], j = t.objects[pb];
      if (i < j) out.emplace_back(i, j);
    });
    std::sort(out.begin(), out.end());
  } else {
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        if (box_intersects(b[i], b[j])) out.emplace_back(i, j);
  }
  return out;
}

std::vector<std::vector<int>> per_curve_symmetric(const std::vector<std::pair<int, int>> &u, int n) {
  std::vector<std::vector<int>> r(n);
  for (auto &p : u) {
    r[p.first].push_back(p.second);
    r[p.second].push_back(p.first);
  }
  for (auto &v : r) std::sort(v.begin(), v.end());
  return r;
}
std::vector<std::vector<int>> per_curve_unique(const std::vector<std::pair<int, int>> &u, int n) {
  std::vector<std::vector<int>> r(n);
  for (auto &p : u) r[p.first].push_back(p.second);
  return r;
}

// ---------------------------------------------------------------- discretize
// discretize.cpp:103-281.
namespace {
struct Piece {
  int curve, seg;
  double tlo, thi;
  bool operator<(const Piece &o) const {
    return std::tie(curve, seg, tlo, thi) < std::tie(o.curve, o.seg, o.tlo, o.thi);
  }
  bool operator==(const Piece &o) const {
    return curve == o.curve && seg == o.seg && tlo == o.tlo && thi == o.thi;
  }
};
}  // namespace

std::vector<Curve> discretize(const std::vector<Curve> &curves, const std::vector<std::vector<int>> &links,
                              int *rounds_out) {
  const int nc = (int)curves.size();
  const double eps = std::numeric_limits<double>::epsilon();
  std::vector<std::vector<Piece>> live(nc);
  std::vector<std::vector<Box>> live_box(nc);
  double min_diag = std::numeric_limits<double>::infinity();
  double avg = 0.0;
  long long entrycount = 0;
  for (int i = 0; i < nc; ++i) {
    const int ns = curves[i].num_segments();
    for (int j = 0; j < ns; ++j) {
      Box bb = curves[i].seg_box(j);
      live[i].push_back({i, j, 0.0, 1.0});
      live_box[i].push_back(bb);
      avg += norm(curves[i].q[j]);
      const double d = box_diag(bb);
      if (!(d >= min_diag)) min_diag = d;
    }
    entrycount += ns > 0 ? ns : 0;
  }
  avg /= entrycount * 1.73205080757;
  const double thresh = eps * avg;
  if (!(min_diag >= thresh))
    throw std::runtime_error("Discretize: Smallest input segment is smaller than eps * avg coordinate. Consider combining.");

  std::vector<std::vector<Piece>> done(nc);
  std::vector<KdTree> trees(nc);
  long long npairs = 0;
  int rounds = 0;
  const int kMaxRounds = 55;
  for (int it = 0; it < kMaxRounds; ++it) {
    ++rounds;
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nc; ++i) trees[i].build(live_box[i]);
    std::vector<std::vector<Piece>> next(nc);
    std::vector<std::vector<Box>> next_box(nc);
    npairs = 0;
    bool too_small = false;
#pragma omp parallel for schedule(dynamic) reduction(+ : npairs)
    for (int i = 0; i < nc; ++i) {
      std::vector<char> hit(live[i].size(), 0);
      long long np = 0;
      for (int j : links[i]) {
        kd_overlap(trees[i], trees[j], [&](int pa, int) {
          ++np;
          hit[trees[i].objects[pa]] = 1;
        });
      }
      double md = std::numeric_limits<double>::infinity();
      for (size_t k = 0; k < live[i].size(); ++k) {
        const Piece &p = live[i][k];
        if (hit[k]) {
          const double tm = 0.5 * (p.tlo + p.thi);
          Box b1 = curves[p.curve].seg_box(p.seg, p.tlo, tm);
          Box b2 = curves[p.curve].seg_box(p.seg, tm, p.thi);
          next[i].push_back({p.curve, p.seg, p.tlo, tm});
          next_box[i].push_back(b1);
          next[i].push_back({p.curve, p.seg, tm, p.thi});
          next_box[i].push_back(b2);
          md = mn(md, mn(box_diag(b1), box_diag(b2)));
        } else {
          done[i].push_back(p);
        }
      }
      npairs += np;
      if (!(md >= thresh)) {
#pragma omp atomic write
        too_small = true;
      }
    }
    if (too_small)
      throw std::runtime_error("Discretize: Smallest segment is smaller than eps * avg coordinate. Perhaps curves are too close.");
    if (npairs == 0) break;
    live.swap(next);
    live_box.swap(next_box);
  }
  if (rounds_out) *rounds_out = rounds;
  if (npairs > 0) throw std::runtime_error("Reached max recursion (curves are too close) in Discretize().");
  std::vector<Curve> out(nc);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nc; ++i) {
    out[i].type = SegType::Polyline;
    out[i].looped = true;
    std::sort(done[i].begin(), done[i].end());
    for (const Piece &p : done[i]) out[i].q.push_back(curves[i].point(p.seg, p.tlo));
    if (!curves[i].looped && !done[i].empty()) {
      const Piece &p = done[i].back();
      out[i].q.push_back(curves[i].point(p.seg, p.thi));
      out[i].looped = false;
    }
  }
  return out;
}

// ---------------------------------------------------------------- direct sum
// compute_link.cpp:126-178.
double direct_one_arctan(const Curve &c1, const Curve &c2, bool parallel) {
  const std::vector<V3> P = c1.start_points();
  std::vector<V3> Q = c2.start_points();
  const int n1 = (int)P.size(), n2 = (int)Q.size();
  if (n2) Q.push_back(Q[0]);
  double lk = 0;
#pragma omp parallel for reduction(+ : lk) if (parallel)
  for (int i = 0; i < n1; ++i) {
    const V3 p0 = P[i], p1 = P[(i + 1) % n1];
    double row = 0;
    for (int k = 0; k < n2; ++k) {
      const V3 a = Q[k] - p0, b = Q[k] - p1, c = Q[k + 1] - p1, d = Q[k + 1] - p0;
      const double la = norm(a), lb = norm(b), lc = norm(c);
      const double ca = dot(c, a);
      const double div1 = la * lb * lc + dot(a, b) * lc + ca * lb + dot(c, b) * la;
      const double ld = norm(d);
      const double div2 = la * ld * lc + dot(a, d) * lc + ca * ld + dot(c, d) * la;
      const double det = a.x * (b.y * c.z - b.z * c.y) + a.z * (b.x * c.y - b.y * c.x) +
                         a.y * (b.z * c.x - b.x * c.z);
      const double xp = div1 * div2 - det * det;
      const double yp = det * (div1 + div2);
      double t = 2.0 * std::atan2(yp, xp);
      const double sg = (double)((det > 0) - (det < 0));
      t = t + ((yp * det < 0) ? kFourPi * sg : 0.0);
      row += t;
    }
    lk += row;
  }
  return lk * kInvFourPi;
}

// compute_link.cpp:200-280 (Bertolazzi arctan addition along curve 1 for each
// curve-2 segment k, with the negative-x-axis crossing count in `off`).
double direct_fast(const Curve &c1, const Curve &c2) {
  const std::vector<V3> P = c1.start_points();
  std::vector<V3> Qv = c2.start_points();
  const int n1 = (int)P.size(), n2 = (int)Qv.size();
  if (!n1 || !n2) return 0.0;
  Qv.push_back(Qv[0]);
  std::vector<double> qx(n2 + 1), qy(n2 + 1), qz(n2 + 1);
  for (int k = 0; k <= n2; ++k) {
    qx[k] = Qv[k].x;
    qy[k] = Qv[k].y;
    qz[k] = Qv[k].z;
  }
  std::vector<double> S(n2, -1.0), xs(n2, 1.0), ys(n2, 0.0), off(n2, 0.0);
  for (int i = 0; i < n1; ++i) {
    const V3 p0 = P[i], p1 = P[(i + 1) % n1];
    double *__restrict Sp = S.data(), *__restrict xsp = xs.data(), *__restrict ysp = ys.data(),
                       *__restrict offp = off.data();
    for (int k = 0; k < n2; ++k) {
      const double ax = qx[k] - p0.x, ay = qy[k] - p0.y, az = qz[k] - p0.z;
      const double bx = qx[k] - p1.x, by = qy[k] - p1.y, bz = qz[k] - p1.z;
      const double cx = qx[k + 1] - p1.x, cy = qy[k + 1] - p1.y, cz = qz[k + 1] - p1.z;
      const double dx = qx[k + 1] - p0.x, dy = qy[k + 1] - p0.y, dz = qz[k + 1] - p0.z;
      const double la = std::sqrt(ax * ax + ay * ay + az * az);
      const double lb = std::sqrt(bx * bx + by * by + bz * bz);
      const double lc = std::sqrt(cx * cx + cy * cy + cz * cz);
      const double ca = cx * ax + cy * ay + cz * az;
      const double div1 = la * lb * lc + (ax * bx + ay * by + az * bz) * lc + ca * lb +
                          (cx * bx + cy * by + cz * bz) * la;
      const double ld = std::sqrt(dx * dx + dy * dy + dz * dz);
      const double div2 = la * ld * lc + (ax * dx + ay * dy + az * dz) * lc + ca * ld +
                          (cx * dx + cy * dy + cz * dz) * la;
      const double det = ax * (by * cz - bz * cy) + az * (bx * cy - by * cx) + ay * (bz * cx - bx * cz);
      const double xp = div1 * div2 - det * det;
      const double yp = det * (div1 + div2);
      const double x0 = xsp[k], y0 = ysp[k], s0 = Sp[k];
      double ny = x0 * yp + xp * y0;
      double nx = x0 * xp - y0 * yp;
      const double m = mx(std::fabs(nx), std::fabs(ny));
      nx = nx / m;
      ny = ny / m;
      const double sg = (double)((det > 0) - (det < 0));
      double o = offp[k] + ((yp * det < 0) ? sg : 0.0);
      const double s3 = ((ny > 0.0) || (ny == 0.0 && nx < 0.0)) ? 1.0 : -1.0;
      const double t1 = s3 * s0, t2 = yp * s0;
      o += s0 * (((t1 < 0) && (t2 >= 0)) ? 1.0 : 0.0);
      offp[k] = o;
      xsp[k] = nx;
      ysp[k] = ny;
      Sp[k] = s3;
    }
  }
  double lk = 0;
  for (int k = 0; k < n2; ++k) lk += (2.0 * kInvFourPi) * std::atan2(ys[k], xs[k]);
  double os = 0;
  for (int k = 0; k < n2; ++k) os += off[k];
  return lk + os;
}

// ---------------------------------------------------------------- Barnes–Hut
// compute_link.cpp:295-315 (one kd tree of segment boxes per loop) and
// :333-389 (recursive moment build with the shift of Eqs. 21-23).
SegTree make_seg_tree(const Curve &c) {
  SegTree t;
  const int n = (int)c.q.size();
  std::vector<Box> bx(n);
  for (int j = 0; j < n; ++j) bx[j] = c.seg_box(j);
  t.kd.build(bx);
  if (n < 2) return t;
  const std::vector<V3> mids = c.midpoints(), tans = c.tangents();
  t.mom.assign(t.kd.nboxes() + n, Moment());
  const int nb = t.kd.nboxes();
  struct B {
    SegTree &t;
    const std::vector<V3> &mids, &tans;
    int nb;
    void go(int node) {
      const Box &bb = t.kd.boxes[node];
      const V3 mid = 0.5 * (bb.hi + bb.lo);
      Moment &M = t.mom[node];
      M.mid = mid;
      for (int s = 0; s < 2; ++s) {
        const int ch = t.kd.children[2 * node + s];
        Moment &C = t.mom[ch];
        if (ch < nb) {
          go(ch);
        } else {
          const int seg = t.kd.objects[ch - nb];
          C.mid = mids[seg];
          const V3 c1 = tans[seg];
          C.tan = c1;
          C.tannorm = norm(c1);
          const double cc[3] = {c1.x, c1.y, c1.z};
          for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) {
              const double o = cc[r] * cc[q];
              C.q0[3 * r + q] = ((1.0 / 12.0) * cc[0]) * o;
              C.q1[3 * r + q] = ((1.0 / 12.0) * cc[1]) * o;
              C.q2[3 * r + q] = ((1.0 / 12.0) * cc[2]) * o;
            }
          C.quadnorm = (1.0 / 36.0) * C.tannorm * C.tannorm * C.tannorm;
        }
        const V3 cv = C.tan;
        M.tan = M.tan + cv;
        const V3 rc = C.mid - mid;
        const double c3[3] = {cv.x, cv.y, cv.z}, r3[3] = {rc.x, rc.y, rc.z};
        for (int r = 0; r < 3; ++r)
          for (int q = 0; q < 3; ++q) M.dip[3 * r + q] += C.dip[3 * r + q] + c3[r] * r3[q];
        double *MQ[3] = {M.q0, M.q1, M.q2};
        const double *CQ[3] = {C.q0, C.q1, C.q2};
        for (int k = 0; k < 3; ++k) {
          // tmp = rc * C.dip.row(k); Q_k += C.Q_k + tmp^T + tmp + c_k rc rc^T
          for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) {
              const double tmp_rq = r3[r] * C.dip[3 * k + q];
              const double tmp_qr = r3[q] * C.dip[3 * k + r];
              MQ[k][3 * r + q] += ((CQ[k][3 * r + q] + tmp_qr) + tmp_rq) + c3[k] * (r3[r] * r3[q]);
            }
        }
      }
      M.tannorm = norm(M.tan);
      double sd = 0;
      for (int e = 0; e < 9; ++e) sd += M.dip[e] * M.dip[e];
      M.dipnorm = std::sqrt(sd) * kInvRt3;
      double sq = 0;
      for (int e = 0; e < 9; ++e) sq += M.q0[e] * M.q0[e];
      double sq1 = 0;
      for (int e = 0; e < 9; ++e) sq1 += M.q1[e] * M.q1[e];
      double sq2 = 0;
      for (int e = 0; e < 9; ++e) sq2 += M.q2[e] * M.q2[e];
      M.quadnorm = (1.0 / 3.0) * std::sqrt(sq + sq1 + sq2);
    }
  } b{t, mids, tans, nb};
  b.go(t.kd.root());
  return t;
}

static inline V3 matvec(const double *m, const V3 &v) {
  return {m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
          m[6] * v.x + m[7] * v.y + m[8] * v.z};
}
static inline V3 matTvec(const double *m, const V3 &v) {
  return {m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
          m[2] * v.x + m[5] * v.y + m[8] * v.z};
}
static inline V3 row(const double *m, int r) { return {m[3 * r], m[3 * r + 1], m[3 * r + 2]}; }
static inline double trace(const double *m) { return m[0] + m[4] + m[8]; }

// compute_link.cpp:411-524 — dipole (Eq. 29) and quadrupole (Eq. 30) terms
// of the far-field expansion, times 4 pi |r|^3, plus the Eq. 14 estimate.
static double far_ho(const Moment &m1, const Moment &m2, const V3 &dr, double rdist2, double rad1,
                     double rad2, double &err) {
  double res = 0;
  const double *D3 = m2.dip, *C3 = m1.dip;
  const V3 D1 = m2.tan, C1 = m1.tan;
  const V3 D2{D3[5] - D3[7], D3[6] - D3[2], D3[1] - D3[3]};
  const V3 C2{C3[5] - C3[7], C3[6] - C3[2], C3[1] - C3[3]};
  res -= dot(C1, D2) + dot(C2, D1);
  res -= 3.0 * rdist2 * (dot(cross(matvec(D3, dr), C1), dr) + dot(cross(matvec(C3, dr), D1), dr));
  {
    const V3 ppp{trace(m1.q0), trace(m1.q1), trace(m1.q2)};
    const V3 qpq{trace(m2.q0), trace(m2.q1), trace(m2.q2)};
    const double tqs1 = -dot(dr, cross(ppp, D1) + cross(C1, qpq));
    const double p01 = dot(row(C3, 0), row(D3, 1)), p02 = dot(row(C3, 0), row(D3, 2));
    const double p10 = dot(row(C3, 1), row(D3, 0)), p12 = dot(row(C3, 1), row(D3, 2));
    const double p20 = dot(row(C3, 2), row(D3, 0)), p21 = dot(row(C3, 2), row(D3, 1));
    const double tqs2 = 2.0 * (dr.x * (p12 - p21) + dr.y * (p20 - p02) + dr.z * (p01 - p10));
    const double tqs = tqs1 + tqs2;
    const V3 pX{dot(row(m1.q1, 2) - row(m1.q2, 1), dr), dot(row(m1.q2, 0) - row(m1.q0, 2), dr),
                dot(row(m1.q0, 1) - row(m1.q1, 0), dr)};
    double tqt = dot(D1, pX);
    const V3 qX{dot(row(m2.q1, 2) - row(m2.q2, 1), dr), dot(row(m2.q2, 0) - row(m2.q0, 2), dr),
                dot(row(m2.q0, 1) - row(m2.q1, 0), dr)};
    tqt += -dot(C1, qX);
    tqt += dot(dr, matTvec(C3, D2) - matTvec(D3, C2));
    const V3 tpp{dot(dr, matvec(m1.q0, dr)), dot(dr, matvec(m1.q1, dr)), dot(dr, matvec(m1.q2, dr))};
    const double tfpp = -dot(dr, cross(D1, tpp));
    const V3 tqq{dot(dr, matvec(m2.q0, dr)), dot(dr, matvec(m2.q1, dr)), dot(dr, matvec(m2.q2, dr))};
    const double tfqq = dot(dr, cross(C1, tqq));
    const double tfpq = 2.0 * dot(matvec(C3, dr), cross(dr, matvec(D3, dr)));
    const double tf = tfpp + tfqq + tfpq;
    res -= 1.5 * rdist2 * ((tqs + 2.0 * tqt) + 5.0 * rdist2 * tf);
  }
  err = rdist2 * (m1.quadnorm * (rad1 * m2.tannorm + 3 * m2.dipnorm) +
                  m2.quadnorm * (rad2 * m1.tannorm + 3 * m1.dipnorm));
  return res;
}

namespace {
struct BHCtx {
  double epssq, itolsq;
  uint64_t nfar = 0, nleaf = 0;
};
}  // namespace

static inline const Box &node_box(const SegTree &t, int node) {
  const int nb = t.kd.nboxes();
  return node < nb ? t.kd.boxes[node] : t.kd.obj_boxes[node - nb];
}

// compute_link.cpp:576-606 — exact one-arctan term of two leaf segments.
static double leaf_term(const Moment &m1, const Moment &m2) {
  const V3 dr = m2.mid - m1.mid;
  const double det = dot(dr, cross(m2.tan, m1.tan));
  const V3 al = dr + 0.5 * (m1.tan - m2.tan);
  // The reference writes dr + 0.5 * (-t2 + t1) etc.; same rounding as above.
  const V3 be = dr + 0.5 * ((-1.0) * m2.tan - m1.tan);
  const V3 ga = dr + 0.5 * (m2.tan - m1.tan);
  double la = norm(al), lb = norm(be), lc = norm(ga);
  double ac = dot(al, ga);
  const double div1 = la * lb * lc + dot(al, be) * lc + ac * lb + dot(be, ga) * la;
  const V3 de = dr + 0.5 * (m2.tan + m1.tan);
  const double ld = norm(de);
  const double div2 = la * ld * lc + dot(al, de) * lc + ac * ld + dot(de, ga) * la;
  la = div1 * div2 - det * det;
  ac = (det == 0) ? std::copysign(1.0, div1) + std::copysign(1.0, div2) : (div1 + div2);
  lb = det * ac;
  lc = (det == 0) ? -std::copysign(1.0, div1) : std::copysign(1.0, det);
  return kInvTwoPi * std::atan2(lb, la) + (((ac < 0) || ((ac == 0) && (det < 0))) ? lc : 0.0);
}

// compute_link.cpp:547-666 — depth-first two-tree traversal; the roles of the
// two trees swap at every split, as in the reference.
static double bh_rec(const SegTree &t1, const SegTree &t2, int n1, int n2, double &err, BHCtx &cx) {
  const int o1 = n1 - t1.kd.nboxes(), o2 = n2 - t2.kd.nboxes();
  const Box &b1 = node_box(t1, n1), &b2 = node_box(t2, n2);
  const double r1sq = 0.25 * dot(b1.hi - b1.lo, b1.hi - b1.lo);
  const double r2sq = 0.25 * dot(b2.hi - b2.lo, b2.hi - b2.lo);
  const double r1 = std::sqrt(r1sq), r2 = std::sqrt(r2sq);
  const double rs = (r1 + r2) * (r1 + r2);
  const Moment &m1 = t1.mom[n1], &m2 = t2.mom[n2];
  const V3 dr = m2.mid - m1.mid;
  const double dsq = dot(dr, dr) + cx.epssq;
  const double thr = rs * cx.itolsq + cx.epssq;
  if (o1 >= 0 && o2 >= 0) {
    ++cx.nleaf;
    return leaf_term(m1, m2);
  }
  if (dsq > thr) {
    ++cx.nfar;
    double res = dot(dr, cross(m2.tan, m1.tan));
    const double rdist2 = 1.0 / dsq;
    const double mult = rdist2 / std::sqrt(dsq) * kInvFourPi;
    double e;
    res += far_ho(m1, m2, dr, rdist2, r1, r2, e);
    err += e * mult;
    return mult * res;
  }
  bool split2;
  if (o1 < 0 && o2 < 0) split2 = r2sq > r1sq;
  else split2 = o2 < 0;
  if (split2) {
    // keep = node1 (tree 1), split node2: recurse(tree1, tree2, n1, child)
    const int c0 = t2.kd.children[2 * n2], c1 = t2.kd.children[2 * n2 + 1];
    return bh_rec(t1, t2, n1, c0, err, cx) + bh_rec(t1, t2, n1, c1, err, cx);
  }
  // keep = node2 (tree 2), split node1: recurse(tree2, tree1, n2, child)
  const int c0 = t1.kd.children[2 * n1], c1 = t1.kd.children[2 * n1 + 1];
  return bh_rec(t2, t1, n2, c0, err, cx) + bh_rec(t2, t1, n2, c1, err, cx);
}

// compute_link.cpp:695-841 — one breadth-first pass (tree roles fixed).
static double bh_iter(const SegTree &t1, const SegTree &t2, const std::vector<int> &a,
                      const std::vector<int> &b, std::vector<int> &na, std::vector<int> &nb_,
                      double &err, BHCtx &cx) {
  const int ni = (int)a.size();
  na.assign(2 * ni, 0);
  nb_.assign(2 * ni, 0);
  int next = 0;
  double res = 0, lerr = 0;
  uint64_t nfar = 0, nleaf = 0;
#pragma omp parallel for reduction(+ : res, lerr, nfar, nleaf) if (ni >= 100)
  for (int x = 0; x < ni; ++x) {
    const int n1 = a[x], n2 = b[x];
    const int o1 = n1 - t1.kd.nboxes(), o2 = n2 - t2.kd.nboxes();
    const Box &b1 = node_box(t1, n1), &b2 = node_box(t2, n2);
    const double r1sq = 0.25 * dot(b1.hi - b1.lo, b1.hi - b1.lo);
    const double r2sq = 0.25 * dot(b2.hi - b2.lo, b2.hi - b2.lo);
    const double r1 = std::sqrt(r1sq), r2 = std::sqrt(r2sq);
    const double rs = (r1 + r2) * (r1 + r2);
    const Moment &m1 = t1.mom[n1], &m2 = t2.mom[n2];
    const V3 dr = m2.mid - m1.mid;
    const double dsq = dot(dr, dr) + cx.epssq;
    const double thr = rs * cx.itolsq + cx.epssq;
    if (o1 >= 0 && o2 >= 0) {
      ++nleaf;
      res += leaf_term(m1, m2);
    } else if (dsq > thr) {
      ++nfar;
      double lr = dot(dr, cross(m2.tan, m1.tan));
      const double rdist2 = 1.0 / dsq;
      const double mult = rdist2 / std::sqrt(dsq) * kInvFourPi;
      double e;
      lr += far_ho(m1, m2, dr, rdist2, r1, r2, e);
      lerr += e * mult;
      res += mult * lr;
    } else {
      bool split1 = true;
      if (o1 < 0 && o2 < 0) {
        if (r2sq > r1sq) split1 = false;
      } else if (o2 < 0) {
        split1 = false;
      }
      int h;
#pragma omp atomic capture
      h = next++;
      if (split1) {
        na[2 * h] = t1.kd.children[2 * n1];
        na[2 * h + 1] = t1.kd.children[2 * n1 + 1];
        nb_[2 * h] = n2;
        nb_[2 * h + 1] = n2;
      } else {
        na[2 * h] = n1;
        na[2 * h + 1] = n1;
        nb_[2 * h] = t2.kd.children[2 * n2];
        nb_[2 * h + 1] = t2.kd.children[2 * n2 + 1];
      }
    }
  }
  na.resize(2 * next);
  nb_.resize(2 * next);
  err = lerr;
  cx.nfar += nfar;
  cx.nleaf += nleaf;
  return res;
}

// compute_link.cpp:866-934.
double bh_eval(const SegTree &t1, const SegTree &t2, double epssq, double itolsq, double &err_total,
               bool parallel, uint64_t *far_count, uint64_t *leaf_count) {
  if (t1.mom.empty() || t2.mom.empty())
    throw std::runtime_error("Barnes-Hut needs loops of at least two segments.");
  BHCtx cx{epssq, itolsq};
  err_total = 0;
  double out;
  if (parallel) {
    std::vector<int> a, b, na{t1.kd.root()}, nb{t2.kd.root()};
    double res = 0, e = 0;
    int cur = 1;
    while (cur > 0 && cur < 75000) {
      std::swap(na, a);
      std::swap(nb, b);
      res += bh_iter(t1, t2, a, b, na, nb, e, cx);
      cur = (int)na.size();
      err_total += e;
    }
    double e2 = 0;
    uint64_t nfar = 0, nleaf = 0;
#pragma omp parallel for reduction(+ : res, e2, nfar, nleaf) schedule(dynamic)
    for (int x = 0; x < cur; ++x) {
      BHCtx lc{epssq, itolsq};
      res += bh_rec(t1, t2, na[x], nb[x], e2, lc);
      nfar += lc.nfar;
      nleaf += lc.nleaf;
    }
    cx.nfar += nfar;
    cx.nleaf += nleaf;
    err_total += e2;
    out = res;
  } else {
    double e = 0;
    const float r = (float)bh_rec(t1, t2, t1.kd.root(), t2.kd.root(), e, cx);
    err_total += e;
    out = r;
  }
  if (far_count) *far_count = cx.nfar;
  if (leaf_count) *leaf_count = cx.nleaf;
  return out;
}

// ------------------------------------------------- curve-order Barnes–Hut
// The product's default Barnes–Hut (no counterpart in the reference; its
// pieces follow the reference): a curve-order tree per loop (node = a
// contiguous segment range, split at lo + (hi - lo) / 2; the internal node
// that splits at s has id s - 1, the leaf of segment p has id n - 1 + p), the
// moment build and shift of compute_link.cpp:333-389, the far field and
// Eq. 14 estimate of :411-524, the exact term of :576-606. Node pairs that are
// neither far nor leaf pairs and have at most `bucket` segments a side are
// summed exactly over their segment pairs; bucket 1 is the reference's rule.
// The roles of the two trees stay fixed (the product's traversal); the split
// rule is the reference's (larger squared radius, or the internal node of an
// internal/leaf pair). Everything in FP64, one pass at the given beta.
CurveTree make_curve_tree(const Curve &c) {
  if (c.type != SegType::Polyline) throw std::runtime_error("curve-order trees take polylines.");
  CurveTree t;
  const int n = (int)c.q.size();
  t.n = n;
  if (n < 2) throw std::runtime_error("Barnes-Hut needs loops of at least two segments.");
  t.lo.assign(2 * n - 1, 0);
  t.cnt.assign(2 * n - 1, 0);
  t.left.assign(2 * n - 1, -1);
  t.right.assign(2 * n - 1, -1);
  t.box.assign(2 * n - 1, Box());
  t.mom.assign(2 * n - 1, Moment());
  const std::vector<V3> mids = c.midpoints(), tans = c.tangents();
  struct B {
    CurveTree &t;
    const Curve &c;
    const std::vector<V3> &mids, &tans;
    int go(int lo, int hi) {
      const int n = t.n;
      if (hi - lo == 1) {
        const int id = n - 1 + lo;
        t.lo[id] = lo;
        t.cnt[id] = 1;
        t.box[id] = c.seg_box(lo);
        Moment &C = t.mom[id];
        C.mid = mids[lo];
        const V3 c1 = tans[lo];
        C.tan = c1;
        C.tannorm = norm(c1);
        const double cc[3] = {c1.x, c1.y, c1.z};
        for (int r = 0; r < 3; ++r)
          for (int q = 0; q < 3; ++q) {
            const double o = cc[r] * cc[q];
            C.q0[3 * r + q] = ((1.0 / 12.0) * cc[0]) * o;
            C.q1[3 * r + q] = ((1.0 / 12.0) * cc[1]) * o;
            C.q2[3 * r + q] = ((1.0 / 12.0) * cc[2]) * o;
          }
        C.quadnorm = (1.0 / 36.0) * C.tannorm * C.tannorm * C.tannorm;
        return id;
      }
      const int s = lo + (hi - lo) / 2, id = s - 1;
      const int l = go(lo, s), r = go(s, hi);
      t.lo[id] = lo;
      t.cnt[id] = hi - lo;
      t.left[id] = l;
      t.right[id] = r;
      t.box[id] = box_merged(t.box[l], t.box[r]);
      const Box &bb = t.box[id];
      const V3 mid = 0.5 * (bb.hi + bb.lo);
      Moment &M = t.mom[id];
      M.mid = mid;
      for (int ch : {l, r}) {
        const Moment &C = t.mom[ch];
        const V3 cv = C.tan;
        M.tan = M.tan + cv;
        const V3 rc = C.mid - mid;
        const double c3[3] = {cv.x, cv.y, cv.z}, r3[3] = {rc.x, rc.y, rc.z};
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) M.dip[3 * a + b] += C.dip[3 * a + b] + c3[a] * r3[b];
        double *MQ[3] = {M.q0, M.q1, M.q2};
        const double *CQ[3] = {C.q0, C.q1, C.q2};
        for (int k = 0; k < 3; ++k)
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
              MQ[k][3 * a + b] += ((CQ[k][3 * a + b] + r3[b] * C.dip[3 * k + a]) + r3[a] * C.dip[3 * k + b]) +
                                  c3[k] * (r3[a] * r3[b]);
      }
      M.tannorm = norm(M.tan);
      double sd = 0, sq = 0;
      for (int e = 0; e < 9; ++e) sd += M.dip[e] * M.dip[e];
      for (int e = 0; e < 9; ++e) sq += M.q0[e] * M.q0[e] + M.q1[e] * M.q1[e] + M.q2[e] * M.q2[e];
      M.dipnorm = std::sqrt(sd) * kInvRt3;
      M.quadnorm = (1.0 / 3.0) * std::sqrt(sq);
      return id;
    }
  } b{t, c, mids, tans};
  t.root = b.go(0, n);
  return t;
}

namespace {
struct CurveBH {
  const CurveTree &t1, &t2;
  double epssq, itolsq;
  int bucket;
  double err = 0;
  uint64_t nfar = 0, nexact = 0;
  double exsum = 0;                                // the exact terms alone
  std::vector<std::pair<int, int>> *far_pairs = nullptr;  // records the far node pairs if set
  double exact(int s1, int s2) {
    ++nexact;
    const double v = leaf_term(t1.mom[t1.n - 1 + s1], t2.mom[t2.n - 1 + s2]);
    exsum += v;
    return v;
  }
  double rec(int a, int b) {
    const Box &b1 = t1.box[a], &b2 = t2.box[b];
    const double r1sq = 0.25 * dot(b1.hi - b1.lo, b1.hi - b1.lo);
    const double r2sq = 0.25 * dot(b2.hi - b2.lo, b2.hi - b2.lo);
    const double r1 = std::sqrt(r1sq), r2 = std::sqrt(r2sq);
    const Moment &m1 = t1.mom[a], &m2 = t2.mom[b];
    const V3 dr = m2.mid - m1.mid;
    const double dsq = dot(dr, dr) + epssq;
    const bool leaf1 = t1.left[a] < 0, leaf2 = t2.left[b] < 0;
    if (leaf1 && leaf2) return exact(t1.lo[a], t2.lo[b]);
    if (dsq > (r1 + r2) * (r1 + r2) * itolsq + epssq) {
      ++nfar;
      if (far_pairs) far_pairs->push_back({a, b});
      double res = dot(dr, cross(m2.tan, m1.tan));
      const double rdist2 = 1.0 / dsq;
      const double mult = rdist2 / std::sqrt(dsq) * kInvFourPi;
      double e;
      res += far_ho(m1, m2, dr, rdist2, r1, r2, e);
      err += e * mult;
      return mult * res;
    }
    if (t1.cnt[a] <= bucket && t2.cnt[b] <= bucket) {
      double s = 0;
      for (int i = 0; i < t1.cnt[a]; ++i)
        for (int j = 0; j < t2.cnt[b]; ++j) s += exact(t1.lo[a] + i, t2.lo[b] + j);
      return s;
    }
    const bool split2 = (!leaf1 && !leaf2) ? (r2sq > r1sq) : !leaf2;
    if (split2) return rec(a, t2.left[b]) + rec(a, t2.right[b]);
    return rec(t1.left[a], b) + rec(t1.right[a], b);
  }
};
}  // namespace

// The same traversal at beta1 >= beta0, continued from a beta0 pass: a node
// pair opened at beta0 is opened at beta1 (far at beta1 implies far at
// beta0), and an exact pair stays exact (the bucket test does not depend on
// beta). So the beta1 sum is the beta0 pass's exact terms plus the beta1
// traversal of the beta0 pass's far pairs, node pair for node pair; err and
// far_count are the continuation's, exact_count counts both passes.
double curve_bh_eval_continued(const CurveTree &t1, const CurveTree &t2, double epssq, double itolsq0,
                               double itolsq1, int bucket, double &err, uint64_t *far_count,
                               uint64_t *exact_count) {
  if (itolsq1 < itolsq0) throw std::runtime_error("the continued pass needs beta1 >= beta0");
  std::vector<std::pair<int, int>> frontier;
  CurveBH p0{t1, t2, epssq, itolsq0, std::max(bucket, 1)};
  p0.far_pairs = &frontier;
  p0.rec(t1.root, t2.root);
  CurveBH p1{t1, t2, epssq, itolsq1, std::max(bucket, 1)};
  double v = p0.exsum;
  for (const auto &fp : frontier) v += p1.rec(fp.first, fp.second);
  err = p1.err;
  if (far_count) *far_count = p1.nfar;
  if (exact_count) *exact_count = p0.nexact + p1.nexact;
  return v;
}

double curve_bh_eval(const CurveTree &t1, const CurveTree &t2, double epssq, double itolsq, int bucket,
                     double &err, uint64_t *far_count, uint64_t *exact_count) {
  CurveBH cx{t1, t2, epssq, itolsq, std::max(bucket, 1)};
  const double v = cx.rec(t1.root, t2.root);
  err = cx.err;
  if (far_count) *far_count = cx.nfar;
  if (exact_count) *exact_count = cx.nexact;
  return v;
}

// ---------------------------------------------------------------- certificate
std::string Certificate::text() const {
  std::ostringstream s;
  s << ncurves << "\n";
  for (auto &e : entries) s << e.first.first << "," << e.first.second << "," << e.second << "\n";
  return s.str();
}

// linking_number_certificate.cpp:358-394 with the method drivers at
// :102-229 (Barnes–Hut, beta retry) and :241-338 (direct sum).
Certificate compute_certificate(const std::vector<Curve> &model, bool direct, bool disc, double beta0,
                                double betamax, std::vector<Curve> *discretized_out) {
  const int nc = (int)model.size();
  std::vector<Curve> dc;
  std::vector<std::vector<int>> uniq;
  if (disc) {
    auto links = per_curve_symmetric(potential_links_unique(model), nc);
    dc = discretize(model, links);
    uniq = per_curve_unique(potential_links_unique(dc), nc);
  } else {
    uniq = per_curve_unique(potential_links_unique(model), nc);
    dc = model;
  }
  Certificate cert;
  cert.ncurves = nc;
  std::vector<std::pair<int, int>> plist;
  for (int i = 0; i < nc; ++i)
    for (int j : uniq[i]) plist.emplace_back(i, j);
  const int np = (int)plist.size();
  cert.pairs.resize(np);
  const bool small = nc < 6;  // NCURVES_PARALLEL_THRESHOLD (lnc.cpp:22)
  const double kEpsSq = 1e-24, kTarget = 0.1, kScale = 0.05;  // lnc.cpp:24-26
  std::vector<SegTree> trees;
  if (!direct) {
    trees.resize(nc);
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nc; ++i) trees[i] = make_seg_tree(dc[i]);
  }
#pragma omp parallel for schedule(dynamic) if (!small)
  for (int p = 0; p < np; ++p) {
    const int i = plist[p].first, j = plist[p].second;
    double lk, err = 0;
    if (direct) {
      lk = small ? direct_one_arctan(dc[i], dc[j], true) : direct_fast(dc[i], dc[j]);
    } else {
      lk = bh_eval(trees[i], trees[j], kEpsSq, beta0 * beta0, err, small);
      err *= kScale;
      const double tb = std::min(std::pow(err / kTarget, 0.25) * beta0, betamax);
      if (tb > beta0) {
        err = 0;
        lk = bh_eval(trees[i], trees[j], kEpsSq, tb * tb, err, small);
      }
    }
    cert.pairs[p] = {i, j, lk, err};
  }
  double off = 0, mxo = 0;
  for (auto &r : cert.pairs) {
    const double nearest = std::round(r.lk);
    const double o = std::fabs(r.lk - nearest);
    off += o;
    mxo = mx(mxo, o);
    if (!(std::fabs(nearest) < 0.25)) {
      // NaN -> int is undefined in the reference; x86 yields INT_MIN.
      const int v = std::isnan(nearest) ? std::numeric_limits<int>::min() : (int)nearest;
      if (std::isnan(nearest)) std::fprintf(stderr, "Linking number (%d,%d) is NaN.\n", r.i, r.j);
      if (v != 0) cert.entries.push_back({{r.i, r.j}, v});
    }
  }
  std::sort(cert.entries.begin(), cert.entries.end());
  cert.mean_off = np ? off / np : 0;
  cert.max_off = mxo;
  if (discretized_out) *discretized_out = std::move(dc);
  return cert;
}

}  // namespace fln_oracle
