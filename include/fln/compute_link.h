/*
 * Per-pair linking numbers with the reference's signatures, header-only over
 * the C ABI of fln.h: the functions of antequ/fastlinkingnumbers
 * src/compute_link.h:62-87 (ComputeLinkingNumberDirectOneArctanPerPair,
 * ComputeLinkingNumberDirectFast) and :176-181 (EvalLinkingNumberBarnesHut),
 * on closed polylines held as plain arrays instead of Eigen vectors.
 *
 * The reference builds the Barnes–Hut segment trees and their moments on the
 * host (MakeSegmentTrees, BuildTreeMoments) and passes them in; here the
 * engine builds both on the GPU inside the call, so EvalLinkingNumberBarnesHut
 * takes the two curves where the reference takes their trees and moments.
 * It runs the reference's tree (the kd-median ModifiedKdBVH) and traversal
 * (leaf pairs summed exactly) at beta = sqrt(itolsq), without the retry of
 * the certificate driver, and adds the raw Eq. 14 error estimate to
 * eval_errs_total, as the reference does.
 *
 * Every call runs on the device of Engine::Default() (device 0) unless an
 * Engine is given. Errors throw FlnStatusError (a std::runtime_error).
 */
#ifndef FLN_COMPUTE_LINK_H_
#define FLN_COMPUTE_LINK_H_

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <utility>
#include <vector>

#include "linking_number_certificate.h"

namespace VerifyCurves {

struct Vector3 {
  double x, y, z;
};

/* A polyline (include/curve.h:41-195, the polyline case): control points q,
 * looped = closed. num_segments() follows curve.h:61-66. */
class Curve {
 public:
  Curve() {}
  explicit Curve(std::vector<Vector3> q, bool looped = true) : q_(std::move(q)), looped_(looped) {}
  int num_segments() const { return looped_ ? (int)q_.size() : (int)q_.size() - 1; }
  bool looped() const { return looped_; }
  const std::vector<Vector3> &q() const { return q_; }
  std::vector<Vector3> &q() { return q_; }

 private:
  std::vector<Vector3> q_;
  bool looped_ = true;
};

namespace fln_detail {
inline const double *flat(const Curve &c) {
  static_assert(sizeof(Vector3) == 3 * sizeof(double), "Vector3 is three packed doubles");
  if (!c.looped()) throw std::runtime_error("The curve must be a closed polyline (looped).");
  if (c.q().size() < 2) throw std::runtime_error("A closed polyline needs at least two points.");
  return &c.q()[0].x;
}
}  // namespace fln_detail

/* compute_link.h:62-64. The GPU evaluates the closed-form segment-pair terms
 * of the direct sum in FP64; `parallel` has no effect (the kernel always
 * runs on the whole device). */
inline double ComputeLinkingNumberDirectOneArctanPerPair(const Curve &curve1, const Curve &curve2,
                                                         bool parallel = false, Engine &engine = Engine::Default()) {
  (void)parallel;
  double lk = 0.0;
  fln_throw_if(fln_direct_pair(engine.get(), fln_detail::flat(curve1), (int64_t)curve1.q().size(),
                               fln_detail::flat(curve2), (int64_t)curve2.q().size(), FLN_PREC_FP64, &lk));
  return lk;
}

/* compute_link.h:86-87: the same integral, the same FP64 kernel. */
inline double ComputeLinkingNumberDirectFast(const Curve &curve1, const Curve &curve2, bool parallel = false,
                                             Engine &engine = Engine::Default()) {
  return ComputeLinkingNumberDirectOneArctanPerPair(curve1, curve2, parallel, engine);
}

/* compute_link.h:176-181 (trees and moments built inside the call, see the
 * top of this file). */
inline double EvalLinkingNumberBarnesHut(const Curve &curve1, const Curve &curve2, const double epssq,
                                         const double itolsq, double &eval_errs_total, bool parallel = true,
                                         Engine &engine = Engine::Default()) {
  (void)parallel;
  if (!(itolsq > 0)) throw std::runtime_error("itolsq (beta squared) must be positive.");
  const double *a = fln_detail::flat(curve1), *b = fln_detail::flat(curve2);
  const int64_t n1 = (int64_t)curve1.q().size(), n2 = (int64_t)curve2.q().size();
  std::vector<double> xyz((size_t)(3 * (n1 + n2)));
  std::copy(a, a + 3 * n1, xyz.begin());
  std::copy(b, b + 3 * n2, xyz.begin() + 3 * n1);
  const int64_t off[3] = {0, n1, n1 + n2};
  const int32_t pair[2] = {0, 1};
  fln_params p;
  fln_default_params(&p);
  p.barnes_hut_init_beta = std::sqrt(itolsq);
  p.barnes_hut_beta_limit = p.barnes_hut_init_beta;
  p.epssq = epssq;
  p.error_est_scale = 1.0;   // the raw estimate, as EvalLinkingNumberBarnesHut accumulates it
  p.target_error = 1e300;    // one pass: the retry belongs to the certificate driver
  p.bh_escalations = 0;
  p.fp64_margin = 0.0;       // no FP64 recompute
  p.bh_err_limit = 1e300;
  p.bh_tree = 1;             // the reference's kd-median tree, leaf pairs summed exactly
  double lk = 0.0, err = 0.0;
  int32_t flags = 0;
  fln_throw_if(fln_linking_numbers(engine.get(), xyz.data(), off, 2, pair, 1, FLN_METHOD_BARNESHUT, &p, &lk, &err,
                                   &flags));
  eval_errs_total += err;
  return lk;
}

}  // namespace VerifyCurves

#endif  // FLN_COMPUTE_LINK_H_
