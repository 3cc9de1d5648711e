// Command-line driver in the shape of the reference's CLI test
// (fmm3d/tt.cpp:40-111), written against the reference-compatible facade:
//   tt_b200 <optionsfile> [seed]
// The option file uses the reference's format, one "-key value" per line
// with optional trailing "%comment" (fmm3d/options_0):
//   -numsrc, -numtrg, -kt, -fmm3d_np, -fmm3d_let3d_ptsmax, -fmm3d_let3d_maxlevel
// Sources and targets are uniform in [-1,1]^3 with U[0,1] densities, the
// normals are the positions (as the reference's driver does), eval runs three
// times and check() samples 20 targets against the direct sum.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <random>
#include <sstream>
#include <string>

#include "kifmm_fmm3d.hpp"

using namespace kifmm_compat;

static bool read_options(const char* path, std::map<std::string, std::string>& opts) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::string key;
    if (!(ss >> key) || key[0] != '-') continue;
    std::string rest;
    std::getline(ss, rest);
    opts[key] = rest;
  }
  return true;
}

static int int_opt(std::map<std::string, std::string>& o, const char* k) {
  auto it = o.find(k);
  if (it == o.end()) {
    std::fprintf(stderr, "missing option %s\n", k);
    std::exit(2);
  }
  return std::atoi(it->second.c_str());
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <optionsfile> [seed]\n", argv[0]);
    return 2;
  }
  std::map<std::string, std::string> opts;
  if (!read_options(argv[1], opts)) {
    std::fprintf(stderr, "cannot read option file %s\n", argv[1]);
    return 2;
  }
  unsigned long seed = argc > 2 ? std::strtoul(argv[2], nullptr, 10) : 1;
  int ns = int_opt(opts, "-numsrc"), nt = int_opt(opts, "-numtrg"), kt = int_opt(opts, "-kt");
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> box(-1.0, 1.0), unit(0.0, 1.0);
  DblNumMat srcpos(3, ns), trgpos(3, nt);
  for (int i = 0; i < ns; i++)
    for (int d = 0; d < 3; d++) srcpos(d, i) = box(rng);
  for (int i = 0; i < nt; i++)
    for (int d = 0; d < 3; d++) trgpos(d, i) = box(rng);
  Kernel3d knl(kt, std::vector<double>{1.0, 0.25});
  DblNumVec srcden(knl.sdof() * ns), trgval(knl.tdof() * nt);
  for (int i = 0; i < srcden.m(); i++) srcden(i) = unit(rng);

  FMM3d* fmm = new FMM3d("fmm3d_");
  fmm->srcpos() = &srcpos;
  fmm->srcnor() = &srcpos;
  fmm->trgpos() = &trgpos;
  fmm->ctr() = Point3(0, 0, 0);
  fmm->rootlvl() = 0;
  fmm->knl() = knl;
  using clk = std::chrono::steady_clock;
  auto t0 = clk::now();
  int rc = fmm->setup(opts);
  double ts = std::chrono::duration<double>(clk::now() - t0).count();
  if (rc) {
    std::fprintf(stderr, "setup failed (%d): %s\n", rc, fmm->lastError());
    delete fmm;
    return rc;
  }
  std::printf("fmm setup used %g secs\n", ts);
  for (int r = 0; r < 3; r++) {
    t0 = clk::now();
    rc = fmm->eval(srcden, trgval);
    double te = std::chrono::duration<double>(clk::now() - t0).count();
    if (rc) {
      std::fprintf(stderr, "eval failed (%d): %s\n", rc, fmm->lastError());
      delete fmm;
      return rc;
    }
    std::printf("fmm eval used %g secs\n", te);
  }
  double err = 0;
  rc = fmm->check(srcden, trgval, 20, &err);
  std::printf("relative error %g\n", err);
  delete fmm;
  return rc;
}
