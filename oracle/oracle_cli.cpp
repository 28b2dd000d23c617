// Test infrastructure only: a `verifycurves`-style command line around the
// CPU oracle (src/main.cpp:14-99, flags of src/define_args.h:9-55), used to
// pin the oracle against the reference's golden certificates.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <string>

#include "oracle.hpp"

int main(int argc, char **argv) {
  std::map<std::string, std::string> f = {{"input", "data/glove.bcc"},
                                          {"output", "results/out.txt"},
                                          {"method", "barneshut"},
                                          {"discretize", "true"},
                                          {"barnes_hut_init_beta", "2.0"},
                                          {"barnes_hut_beta_limit", "10.0"}};
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a.rfind("--", 0) != 0) continue;
    a = a.substr(2);
    const size_t eq = a.find('=');
    if (eq != std::string::npos) {
      f[a.substr(0, eq)] = a.substr(eq + 1);
    } else if (a.rfind("no", 0) == 0 && f.count(a.substr(2))) {
      f[a.substr(2)] = "false";
    } else if (i + 1 < argc && std::strncmp(argv[i + 1], "--", 2) != 0) {
      f[a] = argv[++i];
    } else {
      f[a] = "true";
    }
  }
  try {
    const bool direct = f["method"] == "directsum";
    if (!direct && f["method"] != "barneshut") throw std::runtime_error("Invalid method encountered.");
    auto t0 = std::chrono::steady_clock::now();
    auto curves = fln_oracle::load_bcc(f["input"]);
    auto t1 = std::chrono::steady_clock::now();
    const bool disc = !(f["discretize"] == "false" || f["discretize"] == "0");
    auto cert = fln_oracle::compute_certificate(curves, direct, disc, std::stod(f["barnes_hut_init_beta"]),
                                                std::stod(f["barnes_hut_beta_limit"]));
    auto t2 = std::chrono::steady_clock::now();
    std::ofstream(f["output"]) << cert.text();
    std::printf("import %.3f ms, compute %.3f ms, pairs %zu, mean off-integer %.9g, max %.9g\n",
                1e-3 * std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count(),
                1e-3 * std::chrono::duration_cast<std::chrono::microseconds>(t2 - t1).count(),
                cert.pairs.size(), cert.mean_off, cert.max_off);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
