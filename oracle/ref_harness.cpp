// Test infrastructure (oracle only): a C-ABI harness around the UNMODIFIED
// reference KIFMM, compiled from the reference's own sources by
// oracle/Makefile into oracle/_ref/libkifmm_ref.so.  Used only by tests/,
// the golden-fixture script and bench.py's CPU-baseline leg; never by the
// product library.
//
// It drives the reference exactly as its CLI driver does (fmm3d/tt.cpp:85-101):
// FMM3d("fmm3d_"), srcpos/srcnor/trgpos, ctr, rootlvl, knl, setup(opts) with
// -fmm3d_np / -fmm3d_let3d_ptsmax / -fmm3d_let3d_maxlevel, then eval().
// It also exposes the reference's Let3d tree and U/V/W/X lists
// (fmm3d/let3d.cpp:56-281) and the Dense3d direct sum (fmm3d/dense3d.cpp:38-57).
#include <chrono>
#include <cstring>
#include <cstdio>

#include "fmm3d/dense3d.hpp"
#include "fmm3d/fmm3d.hpp"

namespace {

double now_s() {
  using clk = std::chrono::steady_clock;
  return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

// Two different (kernel, np) pairs in one process reallocate the reference's
// operator cache vector, whose elements own raw FFT plans
// (fmm3d/matmgnt3d.cpp:446 push_back, :32-37 destructor).  Reserving room
// first keeps every cached MatMgnt3d in place.
void reserve_mm_cache() {
  if (MatMgnt3d::_mmvec.capacity() < 64) MatMgnt3d::_mmvec.reserve(64);
}

std::string itos(int v) {
  char buf[32];
  std::snprintf(buf, sizeof(buf), "%d", v);
  return std::string(buf);
}

struct TreeHandle {
  DblNumMat src;
  DblNumMat trg;
  Let3d* let = nullptr;
};

}  // namespace

extern "C" {

int kref_fmm(int kt, int ncoef, const double* coefs, int np, int ptsmax, int maxlevel,
             const double* ctr, int rootlvl, int ns, const double* srcpos, const double* srcnor,
             int nt, const double* trgpos, const double* srcden, double* trgval, int neval,
             double* times) {
  reserve_mm_cache();
  DblNumMat sp(3, ns), sn(3, ns), tp(3, nt);
  std::memcpy(sp.data(), srcpos, sizeof(double) * 3 * (size_t)ns);
  std::memcpy(sn.data(), srcnor, sizeof(double) * 3 * (size_t)ns);
  std::memcpy(tp.data(), trgpos, sizeof(double) * 3 * (size_t)nt);
  std::vector<double> cf(coefs, coefs + ncoef);
  Kernel3d knl(kt, cf);
  DblNumVec sd(knl.sdof() * ns);
  std::memcpy(sd.data(), srcden, sizeof(double) * (size_t)knl.sdof() * ns);
  DblNumVec tv(knl.tdof() * nt);

  std::map<std::string, std::string> opts;
  opts["-fmm3d_np"] = itos(np);
  opts["-fmm3d_let3d_ptsmax"] = itos(ptsmax);
  opts["-fmm3d_let3d_maxlevel"] = itos(maxlevel);

  FMM3d* fmm = new FMM3d("fmm3d_");
  fmm->srcpos() = &sp;
  fmm->srcnor() = &sn;
  fmm->trgpos() = &tp;
  fmm->ctr() = Point3(ctr[0], ctr[1], ctr[2]);
  fmm->rootlvl() = rootlvl;
  fmm->knl() = knl;
  double t0 = now_s();
  int rc = fmm->setup(opts);
  double t1 = now_s();
  if (times) times[0] = t1 - t0;
  for (int e = 0; e < neval && rc == 0; e++) {
    t0 = now_s();
    rc = fmm->eval(sd, tv);
    t1 = now_s();
    if (times) times[1 + e] = t1 - t0;
  }
  std::memcpy(trgval, tv.data(), sizeof(double) * (size_t)knl.tdof() * nt);
  delete fmm;
  return rc;
}

int kref_direct(int kt, int ncoef, const double* coefs, int ns, const double* srcpos,
                const double* srcnor, const double* srcden, int nt, const double* trgpos,
                double* trgval) {
  DblNumMat sp(3, ns), sn(3, ns), tp(3, nt);
  std::memcpy(sp.data(), srcpos, sizeof(double) * 3 * (size_t)ns);
  std::memcpy(sn.data(), srcnor, sizeof(double) * 3 * (size_t)ns);
  std::memcpy(tp.data(), trgpos, sizeof(double) * 3 * (size_t)nt);
  std::vector<double> cf(coefs, coefs + ncoef);
  Kernel3d knl(kt, cf);
  DblNumVec sd(knl.sdof() * ns);
  std::memcpy(sd.data(), srcden, sizeof(double) * (size_t)knl.sdof() * ns);
  DblNumVec tv(knl.tdof() * nt);
  Dense3d dense("dense3d_");
  dense.srcpos() = &sp;
  dense.srcnor() = &sn;
  dense.trgpos() = &tp;
  dense.knl() = knl;
  std::map<std::string, std::string> opts;
  int rc = dense.setup(opts);
  if (rc == 0) rc = dense.eval(sd, tv);
  std::memcpy(trgval, tv.data(), sizeof(double) * (size_t)knl.tdof() * nt);
  return rc;
}

void* kref_tree_build(int ptsmax, int maxlevel, const double* ctr, int rootlvl, int ns,
                      const double* srcpos, int nt, const double* trgpos) {
  TreeHandle* h = new TreeHandle;
  h->src.resize(3, ns);
  h->trg.resize(3, nt);
  std::memcpy(h->src.data(), srcpos, sizeof(double) * 3 * (size_t)ns);
  std::memcpy(h->trg.data(), trgpos, sizeof(double) * 3 * (size_t)nt);
  h->let = new Let3d("fmm3d_let3d_");
  h->let->srcpos() = &h->src;
  h->let->trgpos() = &h->trg;
  h->let->ctr() = Point3(ctr[0], ctr[1], ctr[2]);
  h->let->rootlvl() = rootlvl;
  std::map<std::string, std::string> opts;
  opts["-fmm3d_let3d_ptsmax"] = itos(ptsmax);
  opts["-fmm3d_let3d_maxlevel"] = itos(maxlevel);
  h->let->setup(opts);
  return h;
}

int kref_tree_nnodes(void* hp) { return (int)((TreeHandle*)hp)->let->ndevec().size(); }

int kref_tree_nodes(void* hp, int* depth, int* path, int* par, int* chd, int* tag, int* sbeg,
                    int* snum, int* tbeg, int* tnum) {
  Let3d* let = ((TreeHandle*)hp)->let;
  int n = (int)let->ndevec().size();
  for (int i = 0; i < n; i++) {
    Let3d::Node& nd = let->node(i);
    depth[i] = nd.depth();
    path[3 * i + 0] = nd.path()(0);
    path[3 * i + 1] = nd.path()(1);
    path[3 * i + 2] = nd.path()(2);
    par[i] = nd.par();
    chd[i] = nd.chd();
    tag[i] = nd.tag();
    sbeg[i] = nd.sextbeg();
    snum[i] = nd.sextnum();
    tbeg[i] = nd.textbeg();
    tnum[i] = nd.textnum();
  }
  return 0;
}

static std::vector<int>& pick_list(Let3d::Node& nd, int which) {
  switch (which) {
    case 0: return nd.Unodes();
    case 1: return nd.Vnodes();
    case 2: return nd.Wnodes();
    case 3: return nd.Xnodes();
    case 4: return nd.sownvis();
    default: return nd.townvis();
  }
}

// which: 0=U 1=V 2=W 3=X 4=source point ids per node 5=target point ids per node
long kref_tree_list_total(void* hp, int which) {
  Let3d* let = ((TreeHandle*)hp)->let;
  long tot = 0;
  for (size_t i = 0; i < let->ndevec().size(); i++) tot += (long)pick_list(let->node((int)i), which).size();
  return tot;
}

int kref_tree_lists(void* hp, int which, long* ptr, int* idx) {
  Let3d* let = ((TreeHandle*)hp)->let;
  int n = (int)let->ndevec().size();
  long pos = 0;
  for (int i = 0; i < n; i++) {
    ptr[i] = pos;
    std::vector<int>& v = pick_list(let->node(i), which);
    for (size_t k = 0; k < v.size(); k++) idx[pos++] = v[k];
  }
  ptr[n] = pos;
  return 0;
}

void kref_tree_free(void* hp) {
  TreeHandle* h = (TreeHandle*)hp;
  delete h->let;
  delete h;
}

}  // extern "C"
