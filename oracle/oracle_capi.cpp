// Test infrastructure only: C entry points of the CPU oracle for ctypes
// (tests/, __graft_entry__.smoke() and the CPU legs of bench.py).
#include <omp.h>

#include <cstring>
#include <exception>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "oracle.hpp"

using namespace fln_oracle;

namespace {
thread_local std::string g_err;
struct OrcModel {
  std::vector<Curve> curves;      // as loaded
  std::vector<Curve> poly;        // after discretize (or copy)
  std::vector<std::pair<int, int>> pairs;  // unique potential links of `poly`
  std::vector<SegTree> trees;
  std::vector<CurveTree> ctrees;  // curve-order trees of `poly`, built on first use
  int rounds = 0;
  std::string cert_text;
};
template <class F>
int guard(F &&f) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    g_err = e.what();
    return 1;
  }
}
}  // namespace

extern "C" {

const char *orc_last_error() { return g_err.c_str(); }

void *orc_create() { return new OrcModel(); }
void orc_destroy(void *m) { delete static_cast<OrcModel *>(m); }

int orc_load_bcc(void *m, const char *path) {
  return guard([&] { static_cast<OrcModel *>(m)->curves = load_bcc(path); });
}

// counts[i] < 0 marks a closed loop (BCC convention); xyz packs all points.
int orc_set_curves(void *m, int type, int ncurves, const int32_t *counts, const double *xyz) {
  return guard([&] {
    auto *o = static_cast<OrcModel *>(m);
    o->curves.assign(ncurves, Curve());
    size_t at = 0;
    for (int i = 0; i < ncurves; ++i) {
      Curve &c = o->curves[i];
      c.type = (SegType)type;
      c.looped = counts[i] < 0;
      const int n = counts[i] < 0 ? -counts[i] : counts[i];
      c.q.resize(n);
      for (int k = 0; k < n; ++k, ++at) c.q[k] = {xyz[3 * at], xyz[3 * at + 1], xyz[3 * at + 2]};
    }
  });
}

int orc_save_bcc(void *m, const char *path) {
  return guard([&] { save_bcc(path, static_cast<OrcModel *>(m)->curves); });
}

int orc_num_curves(void *m) { return (int)static_cast<OrcModel *>(m)->curves.size(); }

// PLS -> Discretize -> PLS (lnc.cpp:358-381).
int orc_prepare(void *m, int disc) {
  return guard([&] {
    auto *o = static_cast<OrcModel *>(m);
    const int nc = (int)o->curves.size();
    if (disc) {
      auto links = per_curve_symmetric(potential_links_unique(o->curves), nc);
      o->poly = discretize(o->curves, links, &o->rounds);
    } else {
      o->poly = o->curves;
    }
    o->pairs = potential_links_unique(o->poly);
    o->trees.clear();
    o->ctrees.clear();
  });
}

int orc_rounds(void *m) { return static_cast<OrcModel *>(m)->rounds; }
int64_t orc_num_pairs(void *m) { return (int64_t)static_cast<OrcModel *>(m)->pairs.size(); }
void orc_get_pairs(void *m, int32_t *out) {
  auto *o = static_cast<OrcModel *>(m);
  for (size_t p = 0; p < o->pairs.size(); ++p) {
    out[2 * p] = o->pairs[p].first;
    out[2 * p + 1] = o->pairs[p].second;
  }
}
int64_t orc_poly_total(void *m) {
  int64_t t = 0;
  for (auto &c : static_cast<OrcModel *>(m)->poly) t += (int64_t)c.q.size();
  return t;
}
// offsets: ncurves + 1 entries; xyz: 3 * total doubles.
void orc_get_poly(void *m, int64_t *offsets, double *xyz) {
  auto *o = static_cast<OrcModel *>(m);
  int64_t at = 0;
  for (size_t i = 0; i < o->poly.size(); ++i) {
    offsets[i] = at;
    for (auto &v : o->poly[i].q) {
      xyz[3 * at] = v.x;
      xyz[3 * at + 1] = v.y;
      xyz[3 * at + 2] = v.z;
      ++at;
    }
  }
  offsets[o->poly.size()] = at;
}
// Replace the polylines directly (closed loops), skipping Discretize.
int orc_set_poly(void *m, int ncurves, const int64_t *offsets, const double *xyz) {
  return guard([&] {
    auto *o = static_cast<OrcModel *>(m);
    o->poly.assign(ncurves, Curve());
    for (int i = 0; i < ncurves; ++i) {
      Curve &c = o->poly[i];
      c.type = SegType::Polyline;
      c.looped = true;
      for (int64_t k = offsets[i]; k < offsets[i + 1]; ++k) c.q.push_back({xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]});
    }
    o->pairs = potential_links_unique(o->poly);
    o->trees.clear();
    o->ctrees.clear();
  });
}

// method 0 = DirectFast (compute_link.cpp:200), 1 = OneArctanPerPair (:126),
// 2 = Barnes–Hut with the reference's per-pair beta retry (lnc.cpp:158-184);
// bh_parallel selects the BFS+DFS path (double result) instead of the serial
// DFS (float result). Pairs are given as indices into the (i, j) arrays.
int orc_eval_pairs(void *m, int method, const int32_t *pi, const int32_t *pj, int64_t n,
                   double beta0, double betamax, int bh_parallel, int nthreads, double *out_lk,
                   double *out_err, uint64_t *out_far, uint64_t *out_leaf) {
  return guard([&] {
    auto *o = static_cast<OrcModel *>(m);
    const int nc = (int)o->poly.size();
    if (nthreads > 0) omp_set_num_threads(nthreads);
    if (method == 2) {
      // Trees are built once per loop, on first use.
      if ((int)o->trees.size() != nc) o->trees.assign(nc, SegTree());
      std::vector<char> need(nc, 0);
      for (int64_t p = 0; p < n; ++p) need[pi[p]] = need[pj[p]] = 1;
#pragma omp parallel for schedule(dynamic)
      for (int i = 0; i < nc; ++i)
        if (need[i] && o->trees[i].mom.empty()) o->trees[i] = make_seg_tree(o->poly[i]);
    }
    std::string err;
#pragma omp parallel for schedule(dynamic) if (!(method == 2 && bh_parallel) && !(method == 1))
    for (int64_t p = 0; p < n; ++p) {
      try {
        const Curve &c1 = o->poly[pi[p]], &c2 = o->poly[pj[p]];
        double e = 0;
        uint64_t nf = 0, nl = 0;
        double lk;
        if (method == 0) {
          lk = direct_fast(c1, c2);
        } else if (method == 1) {
          lk = direct_one_arctan(c1, c2, true);
        } else {
          const SegTree &t1 = o->trees[pi[p]], &t2 = o->trees[pj[p]];
          lk = bh_eval(t1, t2, 1e-24, beta0 * beta0, e, bh_parallel, &nf, &nl);
          e *= 0.05;
          const double tb = std::min(std::pow(e / 0.1, 0.25) * beta0, betamax);
          if (tb > beta0) {
            uint64_t nf2 = 0, nl2 = 0;
            e = 0;
            lk = bh_eval(t1, t2, 1e-24, tb * tb, e, bh_parallel, &nf2, &nl2);
            e *= 0.05;  // reported on the first run's scale
            nf += nf2;
            nl += nl2;
          }
        }
        out_lk[p] = lk;
        if (out_err) out_err[p] = e;
        if (out_far) out_far[p] = nf;
        if (out_leaf) out_leaf[p] = nl;
      } catch (const std::exception &ex) {
#pragma omp critical
        err = ex.what();
      }
    }
    if (!err.empty()) throw std::runtime_error(err);
  });
}

int orc_eval_curve_bh2(void *m, const int32_t *pi, const int32_t *pj, int64_t n, double beta0, double beta,
                       int bucket, int nthreads, double *out_lk, double *out_err, uint64_t *out_far,
                       uint64_t *out_exact);

// One pass of the product's curve-order Barnes–Hut (see curve_bh_eval) per
// pair at beta; out_err is the Eq. 14 estimate times 0.05 (lnc.cpp:165).
int orc_eval_curve_bh(void *m, const int32_t *pi, const int32_t *pj, int64_t n, double beta, int bucket,
                      int nthreads, double *out_lk, double *out_err, uint64_t *out_far, uint64_t *out_exact) {
  return orc_eval_curve_bh2(m, pi, pj, n, beta, beta, bucket, nthreads, out_lk, out_err, out_far, out_exact);
}

// As orc_eval_curve_bh at beta1, continued from a pass at beta0 < beta1
// (curve_bh_eval_continued); beta0 == beta1 is one plain pass.
int orc_eval_curve_bh2(void *m, const int32_t *pi, const int32_t *pj, int64_t n, double beta0, double beta,
                       int bucket, int nthreads, double *out_lk, double *out_err, uint64_t *out_far,
                       uint64_t *out_exact) {
  return guard([&] {
    auto *o = static_cast<OrcModel *>(m);
    const int nc = (int)o->poly.size();
    if (nthreads > 0) omp_set_num_threads(nthreads);
    if ((int)o->ctrees.size() != nc) o->ctrees.assign(nc, CurveTree());
    std::vector<char> need(nc, 0);
    for (int64_t p = 0; p < n; ++p) {
      if (pi[p] < 0 || pi[p] >= nc || pj[p] < 0 || pj[p] >= nc) throw std::runtime_error("pair out of range");
      need[pi[p]] = need[pj[p]] = 1;
    }
    std::string err;
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nc; ++i) {
      try {
        if (need[i] && o->ctrees[i].mom.empty()) o->ctrees[i] = make_curve_tree(o->poly[i]);
      } catch (const std::exception &ex) {
#pragma omp critical
        err = ex.what();
      }
    }
    if (!err.empty()) throw std::runtime_error(err);
#pragma omp parallel for schedule(dynamic)
    for (int64_t p = 0; p < n; ++p) {
      double e = 0;
      uint64_t nf = 0, nx = 0;
      out_lk[p] = beta0 < beta ? curve_bh_eval_continued(o->ctrees[pi[p]], o->ctrees[pj[p]], 1e-24, beta0 * beta0,
                                                         beta * beta, bucket, e, &nf, &nx)
                               : curve_bh_eval(o->ctrees[pi[p]], o->ctrees[pj[p]], 1e-24, beta * beta, bucket, e,
                                               &nf, &nx);
      if (out_err) out_err[p] = 0.05 * e;
      if (out_far) out_far[p] = nf;
      if (out_exact) out_exact[p] = nx;
    }
  });
}

// Full reference pipeline (lnc.cpp:358-394). Stores the certificate text
// (lnc.cpp:441-454); returns its length, or -1 on error.
int64_t orc_certificate(void *m, int direct, int disc, double beta0, double betamax,
                        double *mean_off, double *max_off) {
  int64_t len = -1;
  guard([&] {
    auto *o = static_cast<OrcModel *>(m);
    Certificate c = compute_certificate(o->curves, direct != 0, disc != 0, beta0, betamax, &o->poly);
    o->cert_text = c.text();
    len = (int64_t)o->cert_text.size();
    if (mean_off) *mean_off = c.mean_off;
    if (max_off) *max_off = c.max_off;
  });
  return len;
}
void orc_certificate_text(void *m, char *buf) {
  auto *o = static_cast<OrcModel *>(m);
  std::memcpy(buf, o->cert_text.data(), o->cert_text.size());
}

int orc_max_threads() { return omp_get_max_threads(); }

}  // extern "C"
