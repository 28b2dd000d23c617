// Compiles against the C++ drop-in headers (include/fln/*.h) and links
// libfln.so, as a reference user's program would after switching over.
//
//   shim_check host <golden dir> <tmp dir>   certificate I/O, comparison and
//                                            diffs, BCC round trip, errors
//   shim_check gpu  <golden dir> <tmp dir>   ComputeFromModel on a golden
//                                            input (both methods) and the
//                                            per-pair functions of compute_link.h
// Prints one line per check and exits non-zero at the first failure.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>

#include "fln/compute_link.h"
#include "fln/linking_number_certificate.h"

using namespace VerifyCurves;

static int failures = 0;
static void check(bool ok, const std::string &what) {
  std::cout << (ok ? "ok   " : "FAIL ") << what << std::endl;
  if (!ok) ++failures;
}

static std::string slurp(const std::string &path) {
  std::ifstream f(path);
  std::stringstream s;
  s << f.rdbuf();
  return s.str();
}

static int host_checks(const std::string &golden, const std::string &tmp) {
  // README.md:100-126: knittubebroken against knittubeinit.
  LinkingNumberCertificate broken(golden + "/certificates/knittubebroken.txt");
  LinkingNumberCertificate init(golden + "/certificates/knittubeinit.txt");
  check(broken.Text() == "39\n5,6,-2\n", "certificate import and text");
  check(broken != init, "operator!=");
  LinkingNumberCertificate again(golden + "/certificates/knittubebroken.txt");
  check(broken == again, "operator==");
  broken.ExportDiffsToFiles(tmp + "/dp.txt", tmp + "/dc.txt", init);
  check(slurp(tmp + "/dp.txt") == "5,6,-2\n", "ExportDiffsToFiles: pairs");
  check(slurp(tmp + "/dc.txt") == "5\n6\n", "ExportDiffsToFiles: curves");
  broken.ExportToFile(tmp + "/out.txt");
  check(slurp(tmp + "/out.txt") == "39\n5,6,-2\n", "ExportToFile");
  // BCC round trip through the model.
  Model m;
  m.ImportFromFile(tmp + "/knittubebroken.bcc");
  check(m.NumCurves() == 39, "Model::ImportFromFile");
  m.ExportToFile(tmp + "/rt.bcc");
  Model m2;
  m2.ImportFromFile(tmp + "/rt.bcc");
  m2.ExportToFile(tmp + "/rt2.bcc");
  check(m2.NumCurves() == 39 && slurp(tmp + "/rt.bcc") == slurp(tmp + "/rt2.bcc") &&
            slurp(tmp + "/rt.bcc").size() == slurp(tmp + "/knittubebroken.bcc").size(),
        "Model::ExportToFile round trip");
  // Errors surface as std::runtime_error, as the reference throws them.
  bool threw = false;
  try {
    Model bad;
    bad.ImportFromFile(tmp + "/does-not-exist.bcc");
  } catch (const FlnStatusError &e) {
    threw = e.status == FLN_ERR_IO && dynamic_cast<const std::runtime_error *>(&e) != nullptr;
  }
  check(threw, "missing file throws std::runtime_error");
  threw = false;
  try {
    LinkingNumberCertificate empty;
    empty.Text();
  } catch (const std::runtime_error &) {
    threw = true;
  }
  check(threw, "empty certificate throws");
  return failures;
}

// A circle of radius r in the plane spanned by unit vectors u, v about c.
static Curve circle(Vector3 c, Vector3 u, Vector3 v, double r, int n) {
  std::vector<Vector3> q(n);
  for (int k = 0; k < n; ++k) {
    const double t = 2.0 * M_PI * k / n, a = r * std::cos(t), b = r * std::sin(t);
    q[k] = {c.x + a * u.x + b * v.x, c.y + a * u.y + b * v.y, c.z + a * u.z + b * v.z};
  }
  return Curve(q, true);
}

static int gpu_checks(const std::string &golden, const std::string &tmp) {
  const std::string want = slurp(golden + "/certificates/knittubebroken.txt");
  for (bool direct : {true, false}) {
    Model m;
    m.ImportFromFile(tmp + "/knittubebroken.bcc");
    LinkingNumberCertificate c;
    c.ComputeFromModel(m, direct);
    check(c.Text() == want, std::string("ComputeFromModel ") + (direct ? "directsum" : "barneshut"));
    c.ExportToFile(tmp + "/cert.txt");
    check(slurp(tmp + "/cert.txt") == want, "ExportToFile after compute");
  }
  // The params overload: FP64 precision, the reference's tree.
  {
    Model m;
    m.ImportFromFile(tmp + "/knittubebroken.bcc");
    fln_params p;
    fln_default_params(&p);
    p.precision = FLN_PREC_FP64;
    p.bh_tree = 1;
    LinkingNumberCertificate c;
    c.ComputeFromModel(m, false, true, p);
    check(c.Text() == want, "ComputeFromModel with fln_params");
  }
  // Hopf link: two unit circles through each other's centres, Lk = +-1;
  // far apart: 0; one orientation reversed: the sign flips.
  const Curve a = circle({0, 0, 0}, {1, 0, 0}, {0, 1, 0}, 1.0, 400);
  const Curve b = circle({1, 0, 0}, {1, 0, 0}, {0, 0, 1}, 1.0, 400);
  const Curve far = circle({10, 0, 0}, {1, 0, 0}, {0, 0, 1}, 1.0, 400);
  std::vector<Vector3> rq(b.q().rbegin(), b.q().rend());
  const Curve brev(rq, true);
  const double d1 = ComputeLinkingNumberDirectFast(a, b);
  const double d2 = ComputeLinkingNumberDirectOneArctanPerPair(a, b);
  check(std::fabs(std::fabs(d1) - 1.0) < 1e-9 && d1 == d2, "ComputeLinkingNumberDirectFast: Hopf link");
  check(std::fabs(ComputeLinkingNumberDirectFast(a, far)) < 1e-9, "direct sum: separate circles");
  check(std::fabs(ComputeLinkingNumberDirectFast(a, brev) + d1) < 1e-9, "direct sum: reversed orientation");
  double err = 0.0;
  const double bh = EvalLinkingNumberBarnesHut(a, b, 1e-24, 4.0, err);
  check(std::fabs(bh - d1) < 1e-3 && err > 0.0, "EvalLinkingNumberBarnesHut: Hopf link, error accumulated");
  const double before = err;
  const double bh_far = EvalLinkingNumberBarnesHut(a, far, 1e-24, 4.0, err);
  check(std::fabs(bh_far) < 1e-3 && err >= before, "EvalLinkingNumberBarnesHut: separate circles");
  bool threw = false;
  try {
    ComputeLinkingNumberDirectFast(Curve(a.q(), false), b);
  } catch (const std::runtime_error &) {
    threw = true;
  }
  check(threw, "open curve rejected");
  return failures;
}

int main(int argc, char **argv) {
  if (argc != 4) {
    std::cerr << "usage: shim_check host|gpu <golden dir> <tmp dir>" << std::endl;
    return 2;
  }
  const std::string mode = argv[1];
  try {
    const int f = mode == "host" ? host_checks(argv[2], argv[3]) : gpu_checks(argv[2], argv[3]);
    return f ? 1 : 0;
  } catch (const std::exception &e) {
    std::cout << "FAIL exception: " << e.what() << std::endl;
    return 1;
  }
}
