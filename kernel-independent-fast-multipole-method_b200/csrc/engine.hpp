// The evaluation engine behind the C ABI: one FMM3d-equivalent object.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "operators.hpp"
#include "tree.hpp"

namespace kifmm {

struct ImplBase {
  virtual ~ImplBase() = default;
  // device-resident densities/potentials (double, original point order)
  virtual int eval(const double* d_srcden, double* d_trgval, int nrhs, cudaStream_t st) = 0;
  // grows the per-rhs buffers (no allocation may happen inside a stream capture)
  virtual void reserve(int nrhs) = 0;
  // reads and clears the device-side error word (bit 0: a bounded wait timed out)
  virtual int take_status() = 0;
  virtual void phase_times(double* ms) const = 0;
  virtual int launches() const = 0;
  // the most density vectors one pass of the surface contractions may carry
  virtual int max_rhs_chunk() const = 0;
  // the FP16 tensor-core Hadamard runs, so its producer groups can be tuned
  virtual bool tunable_groups() const = 0;
};

struct Engine {
  std::string prefix = "fmm3d_";
  std::map<std::string, std::string> opts;
  // geometry (host copies)
  int ns = 0, nt = 0;
  std::vector<double> srcpos, srcnor, trgpos;
  bool have_geom = false;
  KernelDesc user, mm;
  bool have_kernel = false;
  double ctr[3] = {0, 0, 0};
  int rootlvl = 0;
  // options
  int np = 6, ptsmax = 150, maxlevel = 10;
  bool mixed = false;
  bool tensor_cores = true;  // mixed mode: surface contractions on tcgen05 (split TF32)
  bool m2l_toeplitz = false;  // V-list Hadamard in the 2x2x2 block-Toeplitz factored form
  bool m2l_tc = false;        // mixed, single-dof kernels: V-list Hadamard on tcgen05
  bool m2l_tc_tf32 = false;   // ... with split-TF32 operands instead of FP16 pairs
  int wait_limit = 1 << 22;   // polls before a device-side pipeline wait gives up (-<prefix>wait_limit;
                              // 0: every such wait gives up at once, to exercise the time-out path)
  int had_groups = 3;         // producer groups of the FP16 tensor-core Hadamard (-<prefix>had_groups)
  // -<prefix>operators per_level: the reference's non-homogeneous operator
  // path (one operator set per level at that level's radius, no 2^(+-l deg)
  // scaling; fmm3d/matmgnt3d.cpp:93-361 with _hom == false)
  bool per_level = false;
  int rhs_chunk = 0;          // density vectors per pass (-<prefix>rhs_chunk; 0: as many as memory allows, <= 8)
  int autotune = 0;           // time the candidate schedules at setup and keep the fastest (-<prefix>autotune)
  int autotune_rhs = 1;       // density vectors per eval the schedule is tuned for (-<prefix>autotune_rhs)
  bool had_groups_set = false, rhs_chunk_set = false;  // given as options: not tuned
  // the schedule in use: [0] Hadamard producer groups, [1] density vectors
  // per pass, [2] autotuned, [3] taken from the process-wide cache,
  // [4] candidates timed, [5] best ms per eval of autotune_rhs vectors
  double schedule[6] = {3, 0, 0, 0, 0, 0};
  bool profiling = false;
  // state
  bool ready = false;       // device state built, eval allowed
  bool tree_ready = false;  // host tree + lists built (introspection allowed)
  std::string err;
  Tree tree;
  std::shared_ptr<const Operators> ops;
  std::shared_ptr<const LevelOperators> lops;  // per_level: operators by depth (absolute level rootlvl + depth)
  std::unique_ptr<ImplBase> impl;
  int device = 0;
  cudaStream_t stream = nullptr;
  // work counters (kifmm_work_counters)
  std::vector<double> counters;
  // setup phases (ms): tree + lists, operators, device data and work lists,
  // schedule autotuning
  double setup_ms[4] = {0, 0, 0, 0};
  // host-API staging (grown on demand)
  double* d_in = nullptr;
  double* d_out = nullptr;
  size_t d_in_cap = 0, d_out_cap = 0;
  // original-order copies for the direct sum (uploaded on first use)
  double *d_spos = nullptr, *d_snor = nullptr, *d_sden = nullptr, *d_tchk = nullptr, *d_vchk = nullptr;
  size_t d_sden_cap = 0, d_tchk_cap = 0;

  ~Engine();
  int setup();  // returns a kifmm_status
  // times the candidate schedules on the set-up engine (autotune option)
  int autotune_run();
  // Instances that can share one concatenated forest engine give the same
  // key (kernel, equivalent kernel, np, precision, V-list form, root level,
  // wait limit); empty for instances that cannot be merged.
  std::string forest_key() const;
  // Sets this engine up as the concatenation of set-up members with one
  // forest_key: their trees side by side (node ids level by level, every
  // sibling group kept aligned), their points one after another, one work
  // list per pass over all of them.  Member k's sources are points
  // [src_off[k], src_off[k] + ns_k) of the forest, its targets likewise.
  int setup_forest(const std::vector<const Engine*>& members);
  std::vector<int> src_off, trg_off;
  int eval_host(const double* srcden, double* trgval, int nrhs);
  int eval_device(const double* d_srcden, double* d_trgval, int nrhs, cudaStream_t st, bool sync);
  // Enqueues the evaluation passes on st without any host synchronisation
  // or error query (usable inside a stream capture).
  int enqueue(const double* d_srcden, double* d_trgval, int nrhs, cudaStream_t st);
  int reserve(int nrhs);
  // KIFMM_ERR_CUDA if a device-side wait of an evaluation that has completed
  // since the last poll timed out (the status word is read and cleared)
  int poll_status();
  int direct(const double* srcden, int nt_chk, const double* tpos, double* out);
  int check(const double* srcden, const double* trgval, int numchk, uint64_t seed, double* relerr);
  void release_device();
};

}  // namespace kifmm

// The opaque handle of the C ABI (kifmm_handle in kifmm.h).
struct kifmm_engine {
  kifmm::Engine e;
};
