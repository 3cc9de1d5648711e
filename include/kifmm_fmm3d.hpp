// kifmm_fmm3d.hpp -- C++ facade with the reference's FMM3d interface,
// header-only, over the C ABI in kifmm.h.  A driver written against the
// reference (fmm3d/tt.cpp:85-106) keeps its calls:
//
//   FMM3d* fmm = new FMM3d("fmm3d_");
//   fmm->srcpos() = &srcpos;  fmm->srcnor() = &srcnor;  fmm->trgpos() = &trgpos;
//   fmm->ctr() = Point3(0,0,0);  fmm->rootlvl() = 0;  fmm->knl() = Kernel3d(kt, coefs);
//   fmm->setup(opts);  fmm->eval(srcden, trgval);  fmm->check(srcden, trgval, 20);
//
// The containers mirror the reference's layouts: DblNumMat is column-major
// (common/nummat.hpp:79-83), so a 3 x n position matrix holds xyz per
// point; DblNumVec is contiguous.  Methods return 0 on success like the
// reference; on failure they return the kifmm_status code (the reference
// asserts instead, common/commoninc.hpp:59-60) and lastError() explains.
#pragma once

#include <cmath>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "kifmm.h"

namespace kifmm_compat {

class DblNumVec {
 public:
  explicit DblNumVec(int m = 0) : v_(m, 0.0) {}
  int m() const { return (int)v_.size(); }
  void resize(int m) { v_.assign(m, 0.0); }
  double& operator()(int i) { return v_[i]; }
  double operator()(int i) const { return v_[i]; }
  double* data() { return v_.data(); }
  const double* data() const { return v_.data(); }

 private:
  std::vector<double> v_;
};

class DblNumMat {  // column-major m x n
 public:
  DblNumMat(int m = 0, int n = 0) : m_(m), n_(n), v_((size_t)m * n, 0.0) {}
  int m() const { return m_; }
  int n() const { return n_; }
  void resize(int m, int n) {
    m_ = m;
    n_ = n;
    v_.assign((size_t)m * n, 0.0);
  }
  double& operator()(int i, int j) { return v_[i + (size_t)j * m_]; }
  double operator()(int i, int j) const { return v_[i + (size_t)j * m_]; }
  double* data() { return v_.data(); }
  const double* data() const { return v_.data(); }
  double* clmdata(int j) { return v_.data() + (size_t)j * m_; }

 private:
  int m_, n_;
  std::vector<double> v_;
};

struct Point3 {
  double x[3];
  Point3(double a = 0, double b = 0, double c = 0) : x{a, b, c} {}
  double& operator()(int i) { return x[i]; }
  double operator()(int i) const { return x[i]; }
};

// Kernel ids of fmm3d/kernel3d.hpp:29-53 (the FMM3d-supported ones).
enum { KNL_LAP_S_U = 111, KNL_LAP_D_U = 121, KNL_STK_S_U = 311, KNL_STK_S_P = 312, KNL_STK_D_U = 321,
       KNL_STK_D_P = 322, KNL_NAV_S_U = 511, KNL_NAV_D_U = 521 };

class Kernel3d {
 public:
  Kernel3d() : kt_(-1) {}
  Kernel3d(int kt, const std::vector<double>& coefs) : kt_(kt), coefs_(coefs) {}
  int& kt() { return kt_; }
  int kt() const { return kt_; }
  std::vector<double>& coefs() { return coefs_; }
  const std::vector<double>& coefs() const { return coefs_; }
  int sdof() const { return (kt_ == 111 || kt_ == 121) ? 1 : 3; }
  int tdof() const { return (kt_ == 111 || kt_ == 121 || kt_ == 312 || kt_ == 322) ? 1 : 3; }

 private:
  int kt_;
  std::vector<double> coefs_;
};

class FMM3d {
 public:
  explicit FMM3d(const std::string& prefix) : prefix_(prefix) { kifmm_create(prefix.c_str(), &h_); }
  ~FMM3d() {
    if (h_) kifmm_destroy(h_);
  }
  FMM3d(const FMM3d&) = delete;
  FMM3d& operator=(const FMM3d&) = delete;

  // member access, fmm3d/knlmat3d.hpp:38-41 and fmm3d/fmm3d.hpp:73-75
  DblNumMat*& srcpos() { return srcpos_; }
  DblNumMat*& srcnor() { return srcnor_; }
  DblNumMat*& trgpos() { return trgpos_; }
  Kernel3d& knl() { return knl_; }
  Point3& ctr() { return ctr_; }
  int& rootlvl() { return rootlvl_; }
  int sdof() const { return knl_.sdof(); }
  int tdof() const { return knl_.tdof(); }

  // FMM3d::setup, fmm3d/fmm3d_setup.cpp:26-63
  int setup(std::map<std::string, std::string>& opts) {
    if (!srcpos_ || !srcnor_ || !trgpos_ || srcpos_->m() != 3 || trgpos_->m() != 3) return KIFMM_ERR_ARG;
    int rc = kifmm_set_geometry(h_, srcpos_->n(), srcpos_->data(), srcnor_->data(), trgpos_->n(), trgpos_->data());
    if (rc) return rc;
    rc = kifmm_set_kernel(h_, knl_.kt(), (int)knl_.coefs().size(), knl_.coefs().data());
    if (rc) return rc;
    rc = kifmm_set_box(h_, ctr_.x, rootlvl_);
    if (rc) return rc;
    for (auto& kv : opts)
      if ((rc = kifmm_set_option(h_, kv.first.c_str(), kv.second.c_str()))) return rc;
    return kifmm_setup(h_);
  }

  // FMM3d::eval, fmm3d/fmm3d_eval.cpp:24-243 (trgval pre-sized, overwritten)
  int eval(const DblNumVec& srcden, DblNumVec& trgval) {
    if (srcden.m() != sdof() * srcpos_->n() || trgval.m() != tdof() * trgpos_->n()) return KIFMM_ERR_ARG;
    return kifmm_eval(h_, srcden.data(), trgval.data());
  }

  // FMM3d::check, fmm3d/fmm3d_check.cpp:25-73; prints like the reference and
  // also returns the relative error through relerr when given.
  int check(const DblNumVec& srcden, DblNumVec& trgval, int numchk, double* relerr = nullptr) {
    double e = 0.0;
    int rc = kifmm_check(h_, srcden.data(), trgval.data(), numchk, 0, &e);
    if (rc) return rc;
    std::fprintf(stderr, "relative error: %g\n", e);
    if (relerr) *relerr = e;
    return 0;
  }

  const char* lastError() const { return kifmm_last_error(h_); }
  kifmm_handle handle() const { return h_; }

 private:
  std::string prefix_;
  kifmm_handle h_ = nullptr;
  DblNumMat* srcpos_ = nullptr;
  DblNumMat* srcnor_ = nullptr;
  DblNumMat* trgpos_ = nullptr;
  Kernel3d knl_;
  Point3 ctr_;
  int rootlvl_ = 0;
};

}  // namespace kifmm_compat
