/*
 * C++ drop-in for the reference's public classes, header-only over the C ABI
 * of fln.h: VerifyCurves::Model (include/model.h:24-75) and
 * VerifyCurves::LinkingNumberCertificate (include/linking_number_certificate.h:25-131),
 * with the same method names, defaults and error behaviour (std::runtime_error).
 * Curves are exposed as plain arrays instead of Eigen vectors.
 */
#ifndef FLN_LINKING_NUMBER_CERTIFICATE_H_
#define FLN_LINKING_NUMBER_CERTIFICATE_H_

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../fln.h"

namespace VerifyCurves {

class FlnStatusError : public std::runtime_error {
 public:
  FlnStatusError(fln_status s, const std::string &m) : std::runtime_error(m), status(s) {}
  fln_status status;
};

inline void fln_throw_if(fln_status s) {
  if (s != FLN_OK) throw FlnStatusError(s, std::string(fln_status_string(s)) + ": " + fln_last_error());
}

/* One CUDA device + stream shared by the certificates of a process. */
class Engine {
 public:
  explicit Engine(int device = 0) { fln_throw_if(fln_ctx_create(device, nullptr, &ctx_)); }
  ~Engine() { fln_ctx_destroy(ctx_); }
  Engine(const Engine &) = delete;
  Engine &operator=(const Engine &) = delete;
  fln_ctx *get() const { return ctx_; }
  fln_stats stats() const {
    fln_stats s;
    fln_throw_if(fln_ctx_stats(ctx_, &s));
    return s;
  }
  static Engine &Default() {
    static Engine e(0);
    return e;
  }

 private:
  fln_ctx *ctx_ = nullptr;
};

enum class SegmentType { BSpline = FLN_SEG_BSPLINE, CatmullRom = FLN_SEG_CATMULLROM, Bezier = FLN_SEG_BEZIER,
                         Polyline = FLN_SEG_POLYLINE };

class Model {
 public:
  Model() { fln_throw_if(fln_model_create(&m_)); }
  ~Model() { fln_model_destroy(m_); }
  Model(const Model &) = delete;
  Model &operator=(const Model &) = delete;
  /* Model::ImportFromFile (model.cpp:44-54): BCC only. */
  void ImportFromFile(const std::string &filename) { fln_throw_if(fln_model_load_bcc(m_, filename.c_str())); }
  /* Model::ExportToFile (model.cpp:61-71). */
  void ExportToFile(const std::string &filename) const { fln_throw_if(fln_model_save_bcc(m_, filename.c_str())); }
  /* counts[c] control points of curve c, negative for a closed loop; xyz packed. */
  void SetCurves(SegmentType type, const std::vector<int32_t> &counts, const std::vector<double> &xyz) {
    fln_throw_if(fln_model_set_curves(m_, (fln_seg_type)type, (int32_t)counts.size(), counts.data(), xyz.data()));
  }
  int NumCurves() const { return fln_model_num_curves(m_); }
  fln_model *get() const { return m_; }

 private:
  fln_model *m_ = nullptr;
};

class LinkingNumberCertificate {
 public:
  LinkingNumberCertificate() {}
  explicit LinkingNumberCertificate(const std::string &filename) { ImportFromFile(filename); }

  /* ComputeFromModel (linking_number_certificate.h:63-66): Barnes–Hut by
   * default; force_direct_sum selects direct summation. */
  void ComputeFromModel(const Model &model, bool force_direct_sum = false, bool discretize = true,
                        double barnes_hut_init_beta = 2.0, double barnes_hut_beta_limit = 10.0,
                        Engine &engine = Engine::Default()) {
    fln_params p;
    fln_default_params(&p);
    p.barnes_hut_init_beta = barnes_hut_init_beta;
    p.barnes_hut_beta_limit = barnes_hut_beta_limit;
    ComputeFromModel(model, force_direct_sum, discretize, p, engine);
  }
  /* The same with every engine parameter (fln_params: precision, tree,
   * schedule, ...). */
  void ComputeFromModel(const Model &model, bool force_direct_sum, bool discretize, const fln_params &params,
                        Engine &engine = Engine::Default()) {
    fln_certificate *c = nullptr;
    fln_throw_if(fln_certificate_compute(engine.get(), model.get(), force_direct_sum, discretize, &params, &c));
    c_.reset(c);
  }
  void ExportToFile(const std::string &filename) const { fln_throw_if(fln_certificate_save(need(), filename.c_str())); }
  void ImportFromFile(const std::string &filename) {
    fln_certificate *c = nullptr;
    fln_throw_if(fln_certificate_load(filename.c_str(), &c));
    c_.reset(c);
  }
  void ExportDiffsToFiles(const std::string &out_diff_links_filename, const std::string &out_diff_curves_filename,
                          const LinkingNumberCertificate &other) const {
    fln_throw_if(fln_certificate_export_diffs(need(), other.need(), out_diff_links_filename.c_str(),
                                              out_diff_curves_filename.c_str()));
  }
  bool Equals(const LinkingNumberCertificate &other) const { return fln_certificate_equals(need(), other.need()) != 0; }
  bool operator==(const LinkingNumberCertificate &other) const { return Equals(other); }
  bool operator!=(const LinkingNumberCertificate &other) const { return !Equals(other); }
  std::string Text() const {
    const int64_t n = fln_certificate_text(need(), nullptr, 0);
    std::string s((size_t)n + 1, '\0');
    fln_certificate_text(need(), &s[0], n + 1);
    s.resize((size_t)n);
    return s;
  }

 private:
  struct Del {
    void operator()(fln_certificate *c) const { fln_certificate_destroy(c); }
  };
  const fln_certificate *need() const {
    if (!c_) throw std::runtime_error("LinkingNumberCertificate is empty.");
    return c_.get();
  }
  std::unique_ptr<fln_certificate, Del> c_;
};

}  // namespace VerifyCurves

#endif  // FLN_LINKING_NUMBER_CERTIFICATE_H_
