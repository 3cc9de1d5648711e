// C ABI of libkifmm_b200.so; see include/kifmm.h for the reference
// interface each entry point replaces.
#include <cstring>
#include <string>

#include "../../include/kifmm.h"
#include "engine.hpp"

using kifmm::Engine;

namespace {

kifmm_status fail(kifmm_handle h, kifmm_status s, const char* msg) {
  if (h) h->e.err = msg;
  return s;
}

}  // namespace

extern "C" {

kifmm_status kifmm_create(const char* prefix, kifmm_handle* out) {
  if (!out) return KIFMM_ERR_ARG;
  kifmm_handle h = new (std::nothrow) kifmm_engine;
  if (!h) return KIFMM_ERR_ALLOC;
  h->e.prefix = prefix ? prefix : "fmm3d_";
  *out = h;
  return KIFMM_OK;
}

kifmm_status kifmm_destroy(kifmm_handle h) {
  if (!h) return KIFMM_ERR_ARG;
  delete h;
  return KIFMM_OK;
}

kifmm_status kifmm_set_geometry(kifmm_handle h, int ns, const double* srcpos, const double* srcnor, int nt,
                                const double* trgpos) {
  if (!h) return KIFMM_ERR_ARG;
  if (ns < 0 || nt < 0 || (ns > 0 && (!srcpos || !srcnor)) || (nt > 0 && !trgpos))
    return fail(h, KIFMM_ERR_ARG, "bad geometry arguments");
  Engine& e = h->e;
  e.ns = ns;
  e.nt = nt;
  e.srcpos.assign(srcpos, srcpos + 3 * (size_t)ns);
  e.srcnor.assign(srcnor, srcnor + 3 * (size_t)ns);
  e.trgpos.assign(trgpos, trgpos + 3 * (size_t)nt);
  e.have_geom = true;
  e.ready = false;
  return KIFMM_OK;
}

kifmm_status kifmm_set_kernel(kifmm_handle h, int kt, int ncoef, const double* coefs) {
  if (!h) return KIFMM_ERR_ARG;
  if (ncoef < 0 || (ncoef > 0 && !coefs)) return fail(h, KIFMM_ERR_ARG, "bad coefficient arguments");
  kifmm::KernelDesc k;
  if (!kifmm::kernel_desc(kt, coefs, ncoef, &k)) return fail(h, KIFMM_ERR_KERNEL, "unsupported kernel or coefficients");
  kifmm::KernelDesc mm;
  if (!kifmm::equivalent_kernel(k, &mm)) return fail(h, KIFMM_ERR_KERNEL, "kernel not supported by FMM3d");
  h->e.user = k;
  h->e.have_kernel = true;
  h->e.ready = false;
  return KIFMM_OK;
}

kifmm_status kifmm_set_box(kifmm_handle h, const double ctr[3], int rootlvl) {
  if (!h || !ctr) return KIFMM_ERR_ARG;
  if (rootlvl < -30 || rootlvl > 30) return fail(h, KIFMM_ERR_ARG, "rootlvl out of range");
  std::memcpy(h->e.ctr, ctr, 3 * sizeof(double));
  h->e.rootlvl = rootlvl;
  h->e.ready = false;
  return KIFMM_OK;
}

kifmm_status kifmm_set_option(kifmm_handle h, const char* key, const char* value) {
  if (!h || !key || !value) return KIFMM_ERR_ARG;
  h->e.opts[key] = value;
  return KIFMM_OK;
}

kifmm_status kifmm_setup(kifmm_handle h) {
  if (!h) return KIFMM_ERR_ARG;
  return (kifmm_status)h->e.setup();
}

kifmm_status kifmm_eval(kifmm_handle h, const double* srcden, double* trgval) {
  if (!h) return KIFMM_ERR_ARG;
  return (kifmm_status)h->e.eval_host(srcden, trgval, 1);
}

kifmm_status kifmm_eval_multi(kifmm_handle h, int nrhs, const double* srcden, double* trgval) {
  if (!h) return KIFMM_ERR_ARG;
  return (kifmm_status)h->e.eval_host(srcden, trgval, nrhs);
}

kifmm_status kifmm_eval_device(kifmm_handle h, int nrhs, const double* d_srcden, double* d_trgval, void* stream,
                               int sync) {
  if (!h) return KIFMM_ERR_ARG;
  return (kifmm_status)h->e.eval_device(d_srcden, d_trgval, nrhs, (cudaStream_t)stream, sync != 0);
}

kifmm_status kifmm_poll_status(kifmm_handle h) {
  if (!h) return KIFMM_ERR_ARG;
  return (kifmm_status)h->e.poll_status();
}

kifmm_status kifmm_check(kifmm_handle h, const double* srcden, const double* trgval, int numchk, uint64_t seed,
                         double* relerr) {
  if (!h || !srcden || !trgval || !relerr) return KIFMM_ERR_ARG;
  return (kifmm_status)h->e.check(srcden, trgval, numchk, seed, relerr);
}

kifmm_status kifmm_direct(kifmm_handle h, const double* srcden, int nt, const double* trgpos, double* trgval) {
  if (!h || nt < 0 || (nt > 0 && (!trgpos || !trgval)) || !srcden) return KIFMM_ERR_ARG;
  if (nt == 0) return KIFMM_OK;
  return (kifmm_status)h->e.direct(srcden, nt, trgpos, trgval);
}

kifmm_status kifmm_tree_size(kifmm_handle h, int* nnodes, int* maxdepth) {
  if (!h || !nnodes || !maxdepth) return KIFMM_ERR_ARG;
  if (!h->e.tree_ready) return fail(h, KIFMM_ERR_STATE, "no tree before setup");
  *nnodes = h->e.tree.nnodes;
  *maxdepth = h->e.tree.maxdepth;
  return KIFMM_OK;
}

kifmm_status kifmm_tree_nodes(kifmm_handle h, int* depth, int* path, int* parent, int* child, int* tag, int* snum,
                              int* tnum) {
  if (!h) return KIFMM_ERR_ARG;
  if (!h->e.tree_ready) return fail(h, KIFMM_ERR_STATE, "no tree before setup");
  const kifmm::Tree& t = h->e.tree;
  size_t n = (size_t)t.nnodes;
  if (depth) std::memcpy(depth, t.depth.data(), n * sizeof(int));
  if (path) std::memcpy(path, t.path.data(), 3 * n * sizeof(int));
  if (parent) std::memcpy(parent, t.par.data(), n * sizeof(int));
  if (child) std::memcpy(child, t.chd.data(), n * sizeof(int));
  if (tag) std::memcpy(tag, t.tag.data(), n * sizeof(int));
  // sextnum/textnum are the leaf counts (0 on interior nodes), fmm3d/let3d.cpp:122-124
  for (size_t g = 0; g < n; g++) {
    bool leaf = t.chd[g] == -1;
    if (snum) snum[g] = leaf ? t.scnt[g] : 0;
    if (tnum) tnum[g] = leaf ? t.tcnt[g] : 0;
  }
  return KIFMM_OK;
}

kifmm_status kifmm_tree_lists(kifmm_handle h, int which, int64_t* total, int64_t* ptr, int* idx) {
  if (!h || which < 0 || which > 3) return KIFMM_ERR_ARG;
  if (!h->e.tree_ready) return fail(h, KIFMM_ERR_STATE, "no tree before setup");
  const kifmm::Csr& c = h->e.tree.lists[which];
  if (total) *total = (int64_t)c.idx.size();
  if (ptr) std::memcpy(ptr, c.ptr.data(), c.ptr.size() * sizeof(int64_t));
  if (idx && !c.idx.empty()) std::memcpy(idx, c.idx.data(), c.idx.size() * sizeof(int));
  return KIFMM_OK;
}

kifmm_status kifmm_tree_points(kifmm_handle h, int which, int64_t* ptr, int* idx) {
  if (!h || which < 0 || which > 1 || !ptr) return KIFMM_ERR_ARG;
  if (!h->e.tree_ready) return fail(h, KIFMM_ERR_STATE, "no tree before setup");
  const kifmm::Tree& t = h->e.tree;
  const std::vector<int>& beg = which == 0 ? t.sbeg : t.tbeg;
  const std::vector<int>& cnt = which == 0 ? t.scnt : t.tcnt;
  const std::vector<int>& perm = which == 0 ? t.sperm : t.tperm;
  int64_t pos = 0;
  for (int g = 0; g < t.nnodes; g++) {
    ptr[g] = pos;
    if (t.chd[g] == -1) {
      for (int i = 0; i < cnt[g]; i++) {
        if (idx) idx[pos] = perm[beg[g] + i];
        pos++;
      }
    }
  }
  ptr[t.nnodes] = pos;
  return KIFMM_OK;
}

kifmm_status kifmm_dofs(kifmm_handle h, int* sdof, int* tdof) {
  if (!h || !sdof || !tdof) return KIFMM_ERR_ARG;
  if (!h->e.have_kernel) return fail(h, KIFMM_ERR_STATE, "kernel not set");
  *sdof = h->e.user.sd;
  *tdof = h->e.user.td;
  return KIFMM_OK;
}

kifmm_status kifmm_phase_times(kifmm_handle h, double* ms, int* n) {
  if (!h || !ms || !n) return KIFMM_ERR_ARG;
  if (!h->e.ready) return fail(h, KIFMM_ERR_STATE, "no timings before setup");
  h->e.impl->phase_times(ms);
  *n = 9;
  return KIFMM_OK;
}

kifmm_status kifmm_setup_times(kifmm_handle h, double* ms, int* n) {
  if (!h || !ms || !n) return KIFMM_ERR_ARG;
  if (!h->e.tree_ready) return fail(h, KIFMM_ERR_STATE, "no setup times before setup");
  for (int i = 0; i < 4; i++) ms[i] = h->e.setup_ms[i];
  *n = 4;
  return KIFMM_OK;
}

kifmm_status kifmm_schedule(kifmm_handle h, double* values, int* n) {
  if (!h || !values || !n) return KIFMM_ERR_ARG;
  if (!h->e.ready) return fail(h, KIFMM_ERR_STATE, "no schedule before setup");
  for (int i = 0; i < 6; i++) values[i] = h->e.schedule[i];
  *n = 6;
  return KIFMM_OK;
}

kifmm_status kifmm_set_profiling(kifmm_handle h, int on) {
  if (!h) return KIFMM_ERR_ARG;
  h->e.profiling = on != 0;
  return KIFMM_OK;
}

kifmm_status kifmm_work_counters(kifmm_handle h, double* counts, int* n) {
  if (!h || !counts || !n) return KIFMM_ERR_ARG;
  if (!h->e.ready) return fail(h, KIFMM_ERR_STATE, "no counters before setup");
  for (size_t i = 0; i < h->e.counters.size(); i++) counts[i] = h->e.counters[i];
  *n = (int)h->e.counters.size();
  return KIFMM_OK;
}

kifmm_status kifmm_last_launch_count(kifmm_handle h, int* nlaunch) {
  if (!h || !nlaunch) return KIFMM_ERR_ARG;
  if (!h->e.ready) return fail(h, KIFMM_ERR_STATE, "no launches before setup");
  *nlaunch = h->e.impl->launches();
  return KIFMM_OK;
}

const char* kifmm_status_string(kifmm_status s) {
  switch (s) {
    case KIFMM_OK: return "ok";
    case KIFMM_ERR_ARG: return "invalid argument";
    case KIFMM_ERR_KERNEL: return "unsupported kernel";
    case KIFMM_ERR_OUT_OF_BOX: return "point outside the root box";
    case KIFMM_ERR_STATE: return "invalid call order";
    case KIFMM_ERR_OPTION: return "missing or malformed option";
    case KIFMM_ERR_CUDA: return "CUDA error";
    case KIFMM_ERR_ALLOC: return "allocation failed";
    case KIFMM_ERR_NUMERIC: return "operator precompute failed";
    case KIFMM_ERR_NO_DEVICE: return "no CUDA device";
    case KIFMM_ERR_CAPACITY: return "request exceeds the fixed scratch capacity";
  }
  return "unknown status";
}

const char* kifmm_last_error(kifmm_handle h) {
  if (!h) return "null handle";
  return h->e.err.c_str();
}

}  // extern "C"
