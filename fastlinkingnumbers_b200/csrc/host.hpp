// Host side of the engine: models, the BCC format, potential-link search,
// Discretize, certificates. Internal C++ API behind the C ABI of fln.h.
#pragma once

#include <cstdint>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/fln.h"
#include "geometry.hpp"

namespace fln {

// An error carrying its fln_status across the C++ layers; the C ABI turns it
// into the returned status and fln_last_error().
struct Error : std::runtime_error {
  fln_status status;
  Error(fln_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

// An allocator that default-initialises: resize() leaves doubles unwritten,
// so a large array's pages are first touched by whoever fills it (all
// threads of a parallel copy) instead of being zeroed by one thread.
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <class U>
  NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
  template <class U>
  void construct(U *p) noexcept {
    ::new (static_cast<void *>(p)) U;
  }
  template <class U, class... A>
  void construct(U *p, A &&...a) {
    ::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
  }
};
using DoubleArray = std::vector<double, NoInitAlloc<double>>;
using FloatArray = std::vector<float, NoInitAlloc<float>>;

struct Model {
  std::vector<CurveData> curves;
  // The control points as a BCC file stores them (float32, x y z, curves in
  // order), kept by load_bcc so that the GPU prepare can upload 12 bytes per
  // point and widen them on the device (exact). Empty once the curves are
  // replaced by other means.
  FloatArray bcc_xyz;
  // Prepared (discretized) closed polylines, CSR over loops, and the sorted
  // unique potential pairs (i < j) of those polylines.
  std::vector<int64_t> poly_offsets;
  DoubleArray poly_xyz;
  std::vector<int32_t> pairs;  // 2 per pair
  int32_t rounds = 0;
  bool prepared = false;
};

// model.cpp:280-364 / :367-452.
void load_bcc(const std::string &path, Model &m);
void save_bcc(const std::string &path, const Model &m);

// Sorted unique (i < j) pairs of intersecting boxes (potential_link_search.cpp:88-127).
std::vector<std::pair<int, int>> box_pairs(const std::vector<Box3> &boxes);

// discretize.cpp:103-281; `links[i]` lists every curve whose box meets curve
// i's (both directions). Throws Error on the reference's failure conditions.
void discretize(const std::vector<CurveData> &curves, const std::vector<std::vector<int>> &links,
                std::vector<int64_t> &offsets, DoubleArray &xyz, int32_t &rounds);

// PLS -> Discretize -> PLS (lnc.cpp:61-83 and :367-381).
void prepare(Model &m, bool discretize_on);

struct CertEntry {
  int32_t i, j, lk;
};
struct Certificate {
  int32_t ncurves = 0;
  std::vector<CertEntry> entries;  // i < j, sorted by (i, j), lk != 0
  // Per evaluated pair (empty for a loaded certificate).
  std::vector<int32_t> pairs;
  std::vector<double> lk, err;
  std::vector<int32_t> flags;
  double mean_off = 0, max_off = 0;
  std::string text() const;  // lnc.cpp:441-454
};

// Rounds real sums into the certificate (lnc.cpp:185-213, :294-322, :336-337, :393).
void fill_certificate(Certificate &c, int32_t ncurves, const std::vector<int32_t> &pairs,
                      const std::vector<double> &lk);
Certificate read_certificate(const std::string &path);  // lnc.cpp:402-430
void export_diffs(const Certificate &self, const Certificate &other, const std::string &pairs_path,
                  const std::string &curves_path);  // lnc.cpp:520-561

double now_ms();

}  // namespace fln
