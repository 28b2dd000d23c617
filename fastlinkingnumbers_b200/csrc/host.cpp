// Host stages of the engine: BCC I/O, potential-link search, Discretize and
// certificates. Compiled with -ffp-contract=off (see geometry.hpp).
#include "host.hpp"

#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <tuple>
#include <unordered_set>

namespace fln {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// ------------------------------------------------------------------ BCC
// Binary Curve Collection (model.cpp:266-452): a 64-byte header, then per
// curve an int32 point count (negative = closed loop) and float32 xyz.
namespace {
#pragma pack(push, 1)
struct BccHeader {
  char sign[3];
  uint8_t bytes;
  char type[2];
  uint8_t dims;
  uint8_t up;
  uint64_t ncurves;
  uint64_t npoints;
  char info[40];
};
#pragma pack(pop)
static_assert(sizeof(BccHeader) == 64, "BCC header size");
}  // namespace

// BCC reader (model.cpp:280-364): the file is mapped, one serial pass finds
// where each curve's points start (the counts chain the records), and the
// float32 points are widened to double in parallel. The same checks, in the
// same order, as a record-by-record read.
void load_bcc(const std::string &path, Model &m) {
  const int fd = ::open(path.c_str(), O_RDONLY);
  if (fd < 0) throw Error(FLN_ERR_IO, "Unable to open BCC file: " + path);
  struct stat st;
  if (::fstat(fd, &st) != 0) {
    ::close(fd);
    throw Error(FLN_ERR_IO, "Unable to open BCC file: " + path);
  }
  const uint64_t fsize = (uint64_t)st.st_size;
  const unsigned char *base = nullptr;
  if (fsize > 0) {
    void *mp = ::mmap(nullptr, fsize, PROT_READ, MAP_PRIVATE, fd, 0);
    if (mp == MAP_FAILED) {
      ::close(fd);
      throw Error(FLN_ERR_IO, "Unable to map BCC file: " + path);
    }
    base = static_cast<const unsigned char *>(mp);
  }
  ::close(fd);
  struct Unmap {
    const unsigned char *p;
    uint64_t n;
    ~Unmap() {
      if (p) ::munmap(const_cast<unsigned char *>(p), n);
    }
  } unmap{base, fsize};
  auto fail = [&](fln_status s, const std::string &msg) { throw Error(s, msg + ": " + path); };
  BccHeader h;
  if (fsize < sizeof h) fail(FLN_ERR_IO, "Incomplete BCC header");
  std::memcpy(&h, base, sizeof h);
  if (h.sign[0] != 'B' || h.sign[1] != 'C' || h.sign[2] != 'C') fail(FLN_ERR_FORMAT, "Invalid BCC header");
  if (h.bytes != 0x44) fail(FLN_ERR_FORMAT, "Invalid BCC bytecount (only 32-bit ints and floats)");
  if (h.dims != 3) fail(FLN_ERR_FORMAT, "Invalid BCC dimensions (only 3D)");
  SegKind kind;
  if (h.type[0] == 'C' && h.type[1] == '0') kind = kCatmullRom;
  else if (h.type[0] == 'B' && h.type[1] == 'S') kind = kBSpline;
  else if (h.type[0] == 'B' && h.type[1] == 'Z') kind = kBezier;
  else if (h.type[0] == 'P' && h.type[1] == 'L') kind = kPolyline;
  else fail(FLN_ERR_FORMAT, "Invalid BCC curve type (only C0, BS, BZ, PL)");
  // Every curve needs at least its 4-byte count: reject impossible counts
  // before allocating.
  if (h.ncurves > (fsize - 64) / 4) fail(FLN_ERR_FORMAT, "BCC curve count exceeds file size");
  std::vector<uint64_t> at(h.ncurves);  // byte offset of each curve's points
  std::vector<int64_t> npts(h.ncurves);
  std::vector<CurveData> curves(h.ncurves);
  uint64_t p = sizeof h;
  for (uint64_t i = 0; i < h.ncurves; ++i) {
    if (p + 4 > fsize) fail(FLN_ERR_IO, "Cannot read curve control point count");
    int32_t cnt;
    std::memcpy(&cnt, base + p, 4);
    const int64_t n = cnt < 0 ? -(int64_t)cnt : cnt;
    if ((uint64_t)n * 12 > fsize) fail(FLN_ERR_FORMAT, "BCC point count exceeds file size");
    if (p + 4 + (uint64_t)n * 12 > fsize) fail(FLN_ERR_IO, "Invalid number of control points read");
    curves[i].kind = kind;
    curves[i].closed = cnt < 0;
    at[i] = p + 4;
    npts[i] = n;
    p += 4 + (uint64_t)n * 12;
  }
  // Allocate here, serially: an allocation failure inside the parallel
  // region could not leave it as an exception.
  std::vector<int64_t> first(h.ncurves + 1, 0);  // first point of each curve
  for (uint64_t i = 0; i < h.ncurves; ++i) {
    curves[i].q.resize(npts[i]);
    first[i + 1] = first[i] + npts[i];
  }
  FloatArray f32(3 * (size_t)first[h.ncurves]);
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < (int64_t)h.ncurves; ++i) {
    CurveData &c = curves[i];
    const int64_t n = npts[i];
    const unsigned char *src = base + at[i];
    if (n) std::memcpy(&f32[3 * first[i]], src, 12 * (size_t)n);
    for (int64_t k = 0; k < n; ++k) {
      float v[3];
      std::memcpy(v, src + 12 * k, 12);
      c.q[k] = {(double)v[0], (double)v[1], (double)v[2]};
    }
  }
  m.curves.swap(curves);
  m.bcc_xyz.swap(f32);
  m.prepared = false;
}

void save_bcc(const std::string &path, const Model &m) {
  BccHeader h;
  std::memset(&h, 0, sizeof h);
  h.sign[0] = 'B';
  h.sign[1] = 'C';
  h.sign[2] = 'C';
  h.bytes = 0x44;
  const char *t = "C0";
  if (!m.curves.empty()) {
    const SegKind k = m.curves[0].kind;
    t = k == kBSpline ? "BS" : k == kBezier ? "BZ" : k == kPolyline ? "PL" : "C0";
  }
  h.type[0] = t[0];
  h.type[1] = t[1];
  h.dims = 3;
  h.up = 1;
  h.ncurves = m.curves.size();
  for (auto &c : m.curves) h.npoints += c.q.size();
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) throw Error(FLN_ERR_IO, "Error creating output file: " + path);
  bool ok = std::fwrite(&h, sizeof h, 1, f) == 1;
  std::vector<float> buf;
  for (auto &c : m.curves) {
    int32_t cnt = (int32_t)c.q.size();
    if (c.closed) cnt = -cnt;
    ok = ok && std::fwrite(&cnt, 4, 1, f) == 1;
    buf.resize(3 * c.q.size());
    for (size_t k = 0; k < c.q.size(); ++k) {
      buf[3 * k] = (float)c.q[k].x;
      buf[3 * k + 1] = (float)c.q[k].y;
      buf[3 * k + 2] = (float)c.q[k].z;
    }
    if (!buf.empty()) ok = ok && std::fwrite(buf.data(), 4, buf.size(), f) == buf.size();
  }
  std::fclose(f);
  if (!ok) throw Error(FLN_ERR_IO, "Cannot write BCC file: " + path);
}

// ------------------------------------------------------------------ PLS
// Sweep along x over boxes sorted by their low x; emits every intersecting
// (i < j) once, then sorts — the same set the reference's KdBVH
// self-intersection or its O(n^2) loop produces.
std::vector<std::pair<int, int>> box_pairs(const std::vector<Box3> &boxes) {
  const int n = (int)boxes.size();
  std::vector<int> order;
  order.reserve(n);
  for (int i = 0; i < n; ++i)
    if (boxes[i].lo[0] <= boxes[i].hi[0]) order.push_back(i);  // empty boxes meet nothing
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    return boxes[a].lo[0] < boxes[b].lo[0] || (boxes[a].lo[0] == boxes[b].lo[0] && a < b);
  });
  const int m = (int)order.size();
  std::vector<std::vector<std::pair<int, int>>> part(omp_get_max_threads());
#pragma omp parallel for schedule(dynamic, 64)
  for (int s = 0; s < m; ++s) {
    auto &out = part[omp_get_thread_num()];
    const Box3 &a = boxes[order[s]];
    for (int t = s + 1; t < m && boxes[order[t]].lo[0] <= a.hi[0]; ++t) {
      if (overlaps(a, boxes[order[t]])) {
        const int i = order[s], j = order[t];
        out.emplace_back(std::min(i, j), std::max(i, j));
      }
    }
  }
  std::vector<std::pair<int, int>> all;
  for (auto &p : part) all.insert(all.end(), p.begin(), p.end());
  std::sort(all.begin(), all.end());
  return all;
}

// ------------------------------------------------------------------ Discretize
// Adaptive refinement of spline pieces (discretize.cpp:103-281): each round,
// every live piece whose closed box meets a live piece box of another,
// potentially linked curve is halved in t; the others become final. The
// output polyline of a curve is the start point of each final piece, in
// (segment, t) order. The broad phase here is our own: one curve-order box
// tree per curve (pieces stay sorted along the curve, so contiguous ranges
// are spatially compact) and a dual-tree walk per potential pair i < j that
// marks both sides. The refined set depends only on the box predicate, so it
// equals the reference's whatever tree is used.
namespace {
struct Piece {
  int32_t seg;
  double t0, t1;
};

constexpr int kLeaf = 4;

struct RangeTree {
  // Node k covers [lo[k], hi[k]) of the curve's live pieces; children 2k, 2k+1.
  std::vector<int32_t> lo, hi;
  std::vector<Box3> box;
  void build(const std::vector<Box3> &pb) {
    const int n = (int)pb.size();
    lo.assign(1, 0);
    hi.assign(1, 0);
    box.assign(1, Box3());
    if (!n) return;
    size_t cap = 2;
    while ((int)(cap / 2) * kLeaf < 2 * n) cap *= 2;
    lo.assign(2 * cap, -1);
    hi.assign(2 * cap, -1);
    box.assign(2 * cap, Box3());
    rec(1, 0, n, pb);
  }
  void rec(int k, int a, int b, const std::vector<Box3> &pb) {
    lo[k] = a;
    hi[k] = b;
    if (b - a <= kLeaf) {
      Box3 bb;
      for (int i = a; i < b; ++i) grow(bb, pb[i]);
      box[k] = bb;
      return;
    }
    const int mid = a + (b - a) / 2;
    rec(2 * k, a, mid, pb);
    rec(2 * k + 1, mid, b, pb);
    box[k] = box[2 * k];
    grow(box[k], box[2 * k + 1]);
  }
  bool leaf(int k) const { return hi[k] - lo[k] <= kLeaf; }
};

// Marks pieces of trees A and B whose boxes meet; returns the number of
// meeting piece pairs.
int64_t dual_walk(const RangeTree &A, const std::vector<Box3> &ba, std::atomic<uint8_t> *ha,
                  const RangeTree &B, const std::vector<Box3> &bb, std::atomic<uint8_t> *hb) {
  if (ba.empty() || bb.empty()) return 0;
  int64_t count = 0;
  std::vector<std::pair<int, int>> stack{{1, 1}};
  while (!stack.empty()) {
    auto [x, y] = stack.back();
    stack.pop_back();
    if (!overlaps(A.box[x], B.box[y])) continue;
    const bool lx = A.leaf(x), ly = B.leaf(y);
    if (lx && ly) {
      for (int i = A.lo[x]; i < A.hi[x]; ++i)
        for (int j = B.lo[y]; j < B.hi[y]; ++j)
          if (overlaps(ba[i], bb[j])) {
            ++count;
            ha[i].store(1, std::memory_order_relaxed);
            hb[j].store(1, std::memory_order_relaxed);
          }
    } else if (ly || (!lx && (A.hi[x] - A.lo[x]) >= (B.hi[y] - B.lo[y]))) {
      stack.push_back({2 * x, y});
      stack.push_back({2 * x + 1, y});
    } else {
      stack.push_back({x, 2 * y});
      stack.push_back({x, 2 * y + 1});
    }
  }
  return count;
}
}  // namespace

void discretize(const std::vector<CurveData> &curves, const std::vector<std::vector<int>> &links,
                std::vector<int64_t> &offsets, DoubleArray &xyz, int32_t &rounds) {
  const int nc = (int)curves.size();
  std::vector<std::vector<Piece>> live(nc), done(nc);
  std::vector<std::vector<Box3>> lbox(nc);
  // Input sanity (discretize.cpp:126-160): mean |control point| over the
  // segment-indexed points, and the smallest segment box diagonal.
  double norm_sum = 0, min_diag = std::numeric_limits<double>::infinity();
  int64_t nseg = 0;
  for (int i = 0; i < nc; ++i) {
    const int ns = curves[i].segments();
    if (ns <= 0) continue;
    live[i].resize(ns);
    lbox[i].resize(ns);
    for (int s = 0; s < ns; ++s) {
      live[i][s] = {s, 0.0, 1.0};
      lbox[i][s] = curves[i].piece_box(s);
      const Vec3 &p = curves[i].q[s];
      norm_sum += std::sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
      const double d = diag_length(lbox[i][s]);
      if (!(d >= min_diag)) min_diag = d;
    }
    nseg += ns;
  }
  const double avg = norm_sum / ((double)nseg * 1.73205080757);
  const double thresh = std::numeric_limits<double>::epsilon() * avg;
  if (!(min_diag >= thresh))
    throw Error(FLN_ERR_SEGMENT_TOO_SMALL,
                "Discretize: Smallest input segment is smaller than eps * avg coordinate. Consider combining.");
  // Unique potential pairs i < j from the symmetric lists.
  std::vector<std::pair<int, int>> plist;
  for (int i = 0; i < nc; ++i)
    for (int j : links[i])
      if (i < j) plist.emplace_back(i, j);

  const int kMaxRounds = 55;  // MAX_RECURSION (discretize.cpp:174)
  int64_t overlaps_total = 0;
  rounds = 0;
  std::vector<RangeTree> trees(nc);
  for (int it = 0; it < kMaxRounds; ++it) {
    ++rounds;
    std::vector<std::unique_ptr<std::atomic<uint8_t>[]>> hit(nc);
    for (int i = 0; i < nc; ++i) {
      hit[i].reset(new std::atomic<uint8_t>[std::max<size_t>(1, live[i].size())]);
      for (size_t k = 0; k < live[i].size(); ++k) hit[i][k].store(0, std::memory_order_relaxed);
    }
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nc; ++i) trees[i].build(lbox[i]);
    int64_t count = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : count)
    for (int64_t p = 0; p < (int64_t)plist.size(); ++p) {
      const int i = plist[p].first, j = plist[p].second;
      count += dual_walk(trees[i], lbox[i], hit[i].get(), trees[j], lbox[j], hit[j].get());
    }
    overlaps_total = count;
    std::vector<char> small(nc, 0);
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nc; ++i) {
      std::vector<Piece> next;
      std::vector<Box3> nbox;
      double md = std::numeric_limits<double>::infinity();
      for (size_t k = 0; k < live[i].size(); ++k) {
        const Piece &p = live[i][k];
        if (!hit[i][k].load(std::memory_order_relaxed)) {
          done[i].push_back(p);
          continue;
        }
        const double tm = 0.5 * (p.t0 + p.t1);
        const Box3 b1 = curves[i].piece_box(p.seg, p.t0, tm), b2 = curves[i].piece_box(p.seg, tm, p.t1);
        next.push_back({p.seg, p.t0, tm});
        nbox.push_back(b1);
        next.push_back({p.seg, tm, p.t1});
        nbox.push_back(b2);
        md = min_of(md, min_of(diag_length(b1), diag_length(b2)));
      }
      if (!(md >= thresh)) small[i] = 1;
      live[i].swap(next);
      lbox[i].swap(nbox);
    }
    for (int i = 0; i < nc; ++i)
      if (small[i])
        throw Error(FLN_ERR_SEGMENT_TOO_SMALL,
                    "Discretize: Smallest segment is smaller than eps * avg coordinate. Perhaps curves are too close.");
    if (count == 0) break;
  }
  if (overlaps_total > 0)
    throw Error(FLN_ERR_MAX_RECURSION, "Reached max recursion (curves are too close) in Discretize().");
  offsets.assign(nc + 1, 0);
  for (int i = 0; i < nc; ++i) {
    std::sort(done[i].begin(), done[i].end(), [](const Piece &a, const Piece &b) {
      return std::tie(a.seg, a.t0, a.t1) < std::tie(b.seg, b.t0, b.t1);
    });
    offsets[i + 1] = offsets[i] + (int64_t)done[i].size() + ((!curves[i].closed && !done[i].empty()) ? 1 : 0);
  }
  xyz.assign(3 * offsets[nc], 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nc; ++i) {
    int64_t at = offsets[i];
    for (const Piece &p : done[i]) {
      const Vec3 v = curves[i].at(p.seg, p.t0);
      xyz[3 * at] = v.x;
      xyz[3 * at + 1] = v.y;
      xyz[3 * at + 2] = v.z;
      ++at;
    }
    if (!curves[i].closed && !done[i].empty()) {
      const Piece &p = done[i].back();
      const Vec3 v = curves[i].at(p.seg, p.t1);
      xyz[3 * at] = v.x;
      xyz[3 * at + 1] = v.y;
      xyz[3 * at + 2] = v.z;
    }
  }
}

void prepare(Model &m, bool discretize_on) {
  const int nc = (int)m.curves.size();
  std::vector<Box3> boxes(nc);
  if (discretize_on) {
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nc; ++i) boxes[i] = m.curves[i].whole_box();
    const auto pl = box_pairs(boxes);
    std::vector<std::vector<int>> links(nc);
    for (auto &p : pl) {
      links[p.first].push_back(p.second);
      links[p.second].push_back(p.first);
    }
    for (auto &l : links) std::sort(l.begin(), l.end());
    discretize(m.curves, links, m.poly_offsets, m.poly_xyz, m.rounds);
    // Potential pairs of the polylines (boxes of their segments).
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nc; ++i) {
      Box3 b;
      const int64_t a = m.poly_offsets[i], e = m.poly_offsets[i + 1], n = e - a;
      for (int64_t k = 0; k < n; ++k) {
        const double *p = &m.poly_xyz[3 * (a + k)], *q = &m.poly_xyz[3 * (a + (k + 1) % n)];
        Box3 s;
        for (int d = 0; d < 3; ++d) {
          s.lo[d] = min_of(p[d], q[d]);
          s.hi[d] = max_of(p[d], q[d]);
        }
        grow(b, s);
      }
      boxes[i] = b;
    }
  } else {
    // Without Discretize (lnc.cpp:371-379) the potential pairs come from the
    // curves' own boxes, and the linking-number stage reads each looped curve
    // as the closed polyline of its segment start points
    // (Curve::GetStartPoints, curve.cpp:133-143: get_point(k, 0) for every
    // segment k; a polyline's control points themselves). An open curve
    // keeps its control points: it may not reach that stage.
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nc; ++i) boxes[i] = m.curves[i].whole_box();
    m.poly_offsets.assign(nc + 1, 0);
    for (int i = 0; i < nc; ++i) m.poly_offsets[i + 1] = m.poly_offsets[i] + (int64_t)m.curves[i].q.size();
    m.poly_xyz.resize(3 * m.poly_offsets[nc]);
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nc; ++i) {
      const CurveData &c = m.curves[i];
      for (size_t k = 0; k < c.q.size(); ++k) {
        const Vec3 v = (c.closed && c.kind != kPolyline) ? c.at((int)k, 0.0) : c.q[k];
        double *o = &m.poly_xyz[3 * (m.poly_offsets[i] + (int64_t)k)];
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
      }
    }
    m.rounds = 0;
  }
  const auto pl = box_pairs(boxes);
  // An open curve that reaches the linking-number stage is an error there
  // (Curve::GetStartPoints, curve.cpp:126-128); one without pairs is not.
  for (auto &p : pl)
    if (!m.curves[p.first].closed || !m.curves[p.second].closed)
      throw Error(FLN_ERR_UNLOOPED, "Curve::GetStartPoints() does not support unlooped curves.");
  m.pairs.resize(2 * pl.size());
  for (size_t p = 0; p < pl.size(); ++p) {
    m.pairs[2 * p] = pl[p].first;
    m.pairs[2 * p + 1] = pl[p].second;
  }
  m.prepared = true;
}

// ------------------------------------------------------------------ certificates
std::string Certificate::text() const {
  std::string s = std::to_string(ncurves) + "\n";
  for (auto &e : entries) s += std::to_string(e.i) + "," + std::to_string(e.j) + "," + std::to_string(e.lk) + "\n";
  return s;
}

void fill_certificate(Certificate &c, int32_t ncurves, const std::vector<int32_t> &pairs,
                      const std::vector<double> &lk) {
  c.ncurves = ncurves;
  c.entries.clear();
  const size_t np = lk.size();
  double off = 0, mx = 0;
  for (size_t p = 0; p < np; ++p) {
    const double r = std::round(lk[p]);
    const double o = std::fabs(lk[p] - r);
    off += o;
    mx = max_of(mx, o);
    if (!(std::fabs(r) < 0.25)) {
      if (std::isnan(r)) throw Error(FLN_ERR_NONFINITE, "Linking number (" + std::to_string(pairs[2 * p]) + "," +
                                                            std::to_string(pairs[2 * p + 1]) + ") is NaN.");
      int32_t i = pairs[2 * p], j = pairs[2 * p + 1];
      if (i > j) std::swap(i, j);
      c.entries.push_back({i, j, (int32_t)r});
    }
  }
  std::sort(c.entries.begin(), c.entries.end(),
            [](const CertEntry &a, const CertEntry &b) { return std::tie(a.i, a.j) < std::tie(b.i, b.j); });
  c.mean_off = np ? off / (double)np : 0.0;
  c.max_off = mx;
}

// ReadMatrix: first line the size, then "col,row,value" triplets; duplicate
// coordinates sum (setFromTriplets) and zeros are dropped.
Certificate read_certificate(const std::string &path) {
  std::ifstream f(path);
  if (!f) throw Error(FLN_ERR_IO, "Unable to open certificate: " + path);
  Certificate c;
  std::string line;
  if (!std::getline(f, line)) throw Error(FLN_ERR_FORMAT, "Empty certificate: " + path);
  c.ncurves = std::atoi(line.c_str());
  std::map<std::pair<int, int>, long long> acc;
  while (std::getline(f, line)) {
    std::stringstream ss(line);
    std::string a, b, v;
    if (std::getline(ss, a, ',') && std::getline(ss, b, ',') && std::getline(ss, v, ','))
      acc[{std::atoi(a.c_str()), std::atoi(b.c_str())}] += std::atoi(v.c_str());
  }
  for (auto &kv : acc)
    if (kv.second != 0) c.entries.push_back({kv.first.first, kv.first.second, (int32_t)kv.second});
  return c;
}

// ExportDiffsToFiles: pairs whose values differ (self - other, zeros pruned)
// without the size line; and, as the reference does, every curve index that
// has a nonzero entry in *this* certificate (lnc.cpp:548-559).
void export_diffs(const Certificate &self, const Certificate &other, const std::string &pairs_path,
                  const std::string &curves_path) {
  if (self.ncurves != other.ncurves) {
    const std::string msg = "Unable to compare: The two models have different numbers of curves: " +
                            std::to_string(self.ncurves) + " vs. " + std::to_string(other.ncurves) + ".\n";
    if (!pairs_path.empty() && pairs_path != "[none]") std::ofstream(pairs_path) << msg;
    if (!curves_path.empty() && curves_path != "[none]") std::ofstream(curves_path) << msg;
    return;
  }
  if (!pairs_path.empty() && pairs_path != "[none]") {
    std::map<std::pair<int, int>, long long> d;
    for (auto &e : self.entries) d[{e.i, e.j}] += e.lk;
    for (auto &e : other.entries) d[{e.i, e.j}] -= e.lk;
    std::ofstream f(pairs_path);
    if (!f) throw Error(FLN_ERR_IO, "Cannot write " + pairs_path);
    for (auto &kv : d)
      if (kv.second != 0) f << kv.first.first << "," << kv.first.second << "," << kv.second << "\n";
  }
  if (!curves_path.empty() && curves_path != "[none]") {
    std::vector<char> active(std::max(0, self.ncurves), 0);
    for (auto &e : self.entries) {
      if (e.i >= 0 && e.i < self.ncurves) active[e.i] = 1;
      if (e.j >= 0 && e.j < self.ncurves) active[e.j] = 1;
    }
    std::ofstream f(curves_path);
    if (!f) throw Error(FLN_ERR_IO, "Cannot write " + curves_path);
    for (int i = 0; i < self.ncurves; ++i)
      if (active[i]) f << i << "\n";
  }
}

}  // namespace fln
