// verifycurves: the reference's command line (src/main.cpp:14-99) on the B200
// engine, flag-compatible with src/define_args.h:9-55 (gflags is not used:
// --flag=value, --flag value, --flag / --noflag for booleans).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <map>
#include <string>

#include "fln/linking_number_certificate.h"

using namespace VerifyCurves;

static double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

int main(int argc, char **argv) {
  std::map<std::string, std::string> f = {{"input", "data/glove.bcc"},       {"output", "results/out.txt"},
                                          {"comparewith", "[none]"},         {"diffpairs", "[none]"},
                                          {"diffcurves", "[none]"},          {"method", "barneshut"},
                                          {"discretize", "true"},            {"barnes_hut_init_beta", "2.0"},
                                          {"barnes_hut_beta_limit", "10.0"}, {"precision", "mixed"},
                                          {"device", "0"}};
  const std::string bools[] = {"discretize"};
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a.rfind("--", 0) != 0 && a.rfind("-", 0) == 0) a = "-" + a;  // -flag like gflags
    if (a.rfind("--", 0) != 0) {
      std::cerr << "Unknown argument: " << a << std::endl;
      return 2;
    }
    a = a.substr(2);
    const size_t eq = a.find('=');
    std::string key = eq == std::string::npos ? a : a.substr(0, eq);
    bool is_bool = false;
    for (auto &b : bools) is_bool |= (key == b || key == "no" + b);
    if (!f.count(key) && !(is_bool && key.rfind("no", 0) == 0)) {
      std::cerr << "ERROR: unknown command line flag '" << key << "'" << std::endl;
      return 2;
    }
    if (eq != std::string::npos) {
      f[key] = a.substr(eq + 1);
    } else if (is_bool) {
      if (key.rfind("no", 0) == 0) f[key.substr(2)] = "false";
      else f[key] = "true";
    } else if (i + 1 < argc) {
      f[key] = argv[++i];
    } else {
      std::cerr << "ERROR: flag '" << key << "' is missing its argument" << std::endl;
      return 2;
    }
  }
  try {
    Model model;
    std::cout << "Importing from " << f["input"] << "." << std::endl;
    auto t0 = std::chrono::steady_clock::now();
    model.ImportFromFile(f["input"]);
    std::cout << "Import runtime: " << ms_since(t0) << " ms." << std::endl;
    bool direct;
    if (f["method"] == "directsum") direct = true;
    else if (f["method"] == "barneshut") direct = false;
    else {
      std::cerr << "Invalid method: '" << f["method"] << "'." << std::endl;
      throw std::runtime_error("Invalid method encountered.");
    }
    const std::string d = f["discretize"];
    const bool disc = !(d == "false" || d == "0" || d == "no");
    Engine engine(std::stoi(f["device"]));
    std::cout << "Computing the certificate using the " << (direct ? "Direct Summation" : "Barnes–Hut")
              << " Method." << std::endl;
    t0 = std::chrono::steady_clock::now();
    LinkingNumberCertificate cert;
    fln_params p;
    fln_default_params(&p);
    p.barnes_hut_init_beta = std::stod(f["barnes_hut_init_beta"]);
    p.barnes_hut_beta_limit = std::stod(f["barnes_hut_beta_limit"]);
    if (f["precision"] == "fp64") p.precision = FLN_PREC_FP64;
    else if (f["precision"] != "mixed") throw std::runtime_error("Invalid precision: '" + f["precision"] + "'.");
    cert.ComputeFromModel(model, direct, disc, p, engine);
    const fln_stats s = engine.stats();
    std::cout << "Linking-Number Computation, Mean Off-Integer Error: " << s.mean_off_integer << std::endl;
    std::cout << "Linking-Number Computation, Max  Off-Integer Error: " << s.max_off_integer << std::endl;
    std::cout << "Pairs: " << s.pairs << ", segment pairs: " << s.segment_pairs << ", FP64 recomputed: "
              << s.fp64_recomputed << ", discretize rounds: " << s.discretize_rounds << ", kernels: " << s.ms_kernels
              << " ms" << std::endl;
    std::cout << "Computation runtime: " << ms_since(t0) << " ms. This includes all 3 stages." << std::endl;
    std::cout << "Exporting the certificate to " << f["output"] << "." << std::endl;
    cert.ExportToFile(f["output"]);
    if (f["comparewith"] != "[none]" && (f["diffpairs"] != "[none]" || f["diffcurves"] != "[none]")) {
      LinkingNumberCertificate reference(f["comparewith"]);
      cert.ExportDiffsToFiles(f["diffpairs"], f["diffcurves"], reference);
      std::cout << "Compared and exported the difference between the model and the reference certificate."
                << std::endl;
    }
  } catch (const std::exception &e) {
    std::cerr << "verifycurves: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
