/* kifmm.h -- C ABI of the B200 KIFMM evaluation engine (libkifmm_b200.so).
 *
 * Drop-in boundary for the reference's FMM3d path
 * (lexingying/Kernel-independent-fast-multipole-method).  Every entry point
 * below names the reference interface it replaces.  Plain pointers and
 * sizes only; no C++ or torch types.  Positions and normals are 3 x n
 * column-major doubles (xyz interleaved per point), exactly the reference's
 * DblNumMat(3, n) (common/nummat.hpp:79-83); densities are sdof values per
 * point and potentials tdof values per point (fmm3d/fmm3d_eval.cpp:57-59,
 * :229-230).
 *
 * Every call returns a kifmm_status; the reference's assert paths
 * (iA/iC, common/commoninc.hpp:59-60) become codes.  A handle is owned by
 * one caller; calls on distinct handles may come from different threads.
 */
#ifndef KIFMM_B200_H
#define KIFMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct kifmm_engine* kifmm_handle;

typedef enum {
  KIFMM_OK = 0,
  KIFMM_ERR_ARG = 1,         /* null pointer, bad size or count */
  KIFMM_ERR_KERNEL = 2,      /* kernel id not supported by FMM3d::setup (fmm3d/fmm3d_setup.cpp:41-54) */
  KIFMM_ERR_OUT_OF_BOX = 3,  /* a point outside the root box (fmm3d/let3d.cpp:73,155) */
  KIFMM_ERR_STATE = 4,       /* call order (eval before setup, geometry missing, ...) */
  KIFMM_ERR_OPTION = 5,      /* missing or malformed -fmm3d_* option (fmm3d/fmm3d_setup.cpp:30, let3d.cpp:45-48) */
  KIFMM_ERR_CUDA = 6,        /* a CUDA runtime error (message in kifmm_last_error) */
  KIFMM_ERR_ALLOC = 7,       /* device or host allocation failed */
  KIFMM_ERR_NUMERIC = 8,     /* operator precompute failed (e.g. SVD did not converge) */
  KIFMM_ERR_NO_DEVICE = 9,   /* no CUDA device: there is no CPU fallback */
  KIFMM_ERR_CAPACITY = 10    /* request larger than kifmm_direct_noalloc's fixed scratch */
} kifmm_status;

typedef enum {
  KIFMM_PREC_FP64 = 0,   /* plain FP64 throughout (the reference's arithmetic) */
  KIFMM_PREC_MIXED = 1   /* FP32 bulk sums and surface products; FP64 pseudo-inverses */
} kifmm_precision;

/* Replaces FMM3d::FMM3d(const string& prefix) (fmm3d/fmm3d.cpp:24-28).
 * prefix is the option-key prefix ("fmm3d_" in fmm3d/tt.cpp:85). */
kifmm_status kifmm_create(const char* prefix, kifmm_handle* out);

/* Replaces FMM3d::~FMM3d (fmm3d/fmm3d.cpp:30-33). */
kifmm_status kifmm_destroy(kifmm_handle h);

/* Replaces KnlMat3d::srcpos()/srcnor()/trgpos() (fmm3d/knlmat3d.hpp:38-40).
 * The arrays are read during kifmm_setup; unlike the reference the engine
 * keeps its own copies afterwards. */
kifmm_status kifmm_set_geometry(kifmm_handle h, int ns, const double* srcpos, const double* srcnor, int nt,
                                const double* trgpos);

/* Replaces KnlMat3d::knl() = Kernel3d(kt, coefs) (fmm3d/kernel3d.hpp:64).
 * kt in {111,121,311,321,312,322,511,521}; coefs[0]=mu, coefs[1]=nu. */
kifmm_status kifmm_set_kernel(kifmm_handle h, int kt, int ncoef, const double* coefs);

/* Replaces FMM3d::ctr() and FMM3d::rootlvl() (fmm3d/fmm3d.hpp:73-74):
 * root box centre and level (box radius 2^-rootlvl). */
kifmm_status kifmm_set_box(kifmm_handle h, const double ctr[3], int rootlvl);

/* One entry of the reference's option map (map<string,string>, fmm3d/tt.cpp:23-38).
 * Keys the reference requires: -<prefix>np, -<prefix>let3d_ptsmax,
 * -<prefix>let3d_maxlevel.  Engine keys: -<prefix>precision (fp64|mixed),
 * -<prefix>tree (device|host: where the octree and lists are built),
 * -<prefix>m2l_form (tensor|tensor_tf32|toeplitz|direct: the V-list
 * Hadamard's form), -<prefix>tensor_cores (0|1), -<prefix>wait_limit,
 * -<prefix>had_groups (2|3), -<prefix>rhs_chunk (0..8), -<prefix>autotune
 * (0|1) and -<prefix>autotune_rhs (1..64): see kifmm_poll_status and
 * kifmm_schedule.  -<prefix>operators (scaled|per_level) selects the
 * reference's homogeneous operators (built once, rescaled by 2^(+-l deg)
 * per level) or its non-homogeneous branch (built at every level's radius,
 * fmm3d/matmgnt3d.cpp:93-361 with _hom == false; np 4, 6 or 8, direct
 * V-list form). */
kifmm_status kifmm_set_option(kifmm_handle h, const char* key, const char* value);

/* Replaces FMM3d::setup(map<string,string>&) (fmm3d/fmm3d_setup.cpp:26-63):
 * octree, U/V/W/X lists (fmm3d/let3d.cpp:56-281), translation operators
 * (fmm3d/matmgnt3d.cpp:91-361, built eagerly here), device buffers. */
kifmm_status kifmm_setup(kifmm_handle h);

/* Replaces FMM3d::eval(const DblNumVec& srcden, DblNumVec& trgval)
 * (fmm3d/fmm3d_eval.cpp:24-243).  Host pointers: srcden has sdof*ns values,
 * trgval receives tdof*nt values (overwritten, as :34 zeroes it). */
kifmm_status kifmm_eval(kifmm_handle h, const double* srcden, double* trgval);

/* Same evaluation for nrhs density vectors laid out one after another
 * (srcden[r*sdof*ns + ...], trgval[r*tdof*nt + ...]).  Host pointers. */
kifmm_status kifmm_eval_multi(kifmm_handle h, int nrhs, const double* srcden, double* trgval);

/* Device-resident form: d_srcden / d_trgval are device pointers (double,
 * same layout as kifmm_eval_multi); the work is enqueued on `stream`
 * (a cudaStream_t; NULL is the legacy default stream, as everywhere in
 * CUDA) and the call returns without synchronising when sync == 0. */
kifmm_status kifmm_eval_device(kifmm_handle h, int nrhs, const double* d_srcden, double* d_trgval, void* stream,
                               int sync);

/* No counterpart in the reference (its eval is synchronous and asserts).
 * Every pipeline wait inside this library's kernels is bounded; a wait that
 * runs out sets a bit of the handle's device status word and the kernel
 * returns without faulting.  Synchronous calls report it as
 * KIFMM_ERR_CUDA; for kifmm_eval_device(sync = 0) it is reported by the
 * handle's next kifmm_eval_device call or by this poll, once the stream
 * has been synchronised: KIFMM_ERR_CUDA if an eval that has completed since
 * the last poll timed out (the word is read and cleared).  The option
 * -<prefix>wait_limit (polls per wait, default 4194304) bounds the pipeline
 * waits of the tensor-core V-list kernel; 0 makes each of them give up at
 * once, which exercises this path without a fault. */
kifmm_status kifmm_poll_status(kifmm_handle h);

/* Batched evaluation of independent instances (no counterpart in the
 * reference, which runs one FMM3d::eval at a time, fmm3d/tt.cpp:97-101).
 * A batch groups already set-up handles (any kernels and sizes); each
 * kifmm_batch_eval_device call evaluates nrhs density vectors for every
 * instance (device pointers d_srcden[i] / d_trgval[i], layouts as in
 * kifmm_eval_device).  Instances with the same kernel, np, precision,
 * V-list form and root level are concatenated at creation into one
 * forest (their trees side by side, their points one after another), so each
 * pass of the evaluation is one launch over all of them; their results agree
 * with a kifmm_eval_device per instance to rounding (the summation order of
 * some passes changes with the merged work lists; the mixed engine's FP16
 * scale is shared by the forest).  Forests and the remaining instances run
 * concurrently, and the whole batch is captured into one CUDA graph on the
 * first call and replayed while nrhs and the pointers stay the same.  The
 * forest holds its own device copy of the members' set-up data. */
typedef struct kifmm_batch_s* kifmm_batch;
kifmm_status kifmm_batch_create(int n, const kifmm_handle* handles, kifmm_batch* out);
/* kifmm_batch_create with concatenate = 0: every instance evaluated by its own
 * engine on its own stream (each result bit-identical to its own
 * kifmm_eval_device). */
kifmm_status kifmm_batch_create_opts(int n, const kifmm_handle* handles, int concatenate, kifmm_batch* out);
/* The batch's units (forests + single instances), forests among them, and the
 * kernel launches of one replay of the captured evaluation (0 before the
 * first kifmm_batch_eval_device). */
kifmm_status kifmm_batch_info(kifmm_batch b, int* nunits, int* nforests, int* launches);
kifmm_status kifmm_batch_destroy(kifmm_batch b);
kifmm_status kifmm_batch_eval_device(kifmm_batch b, int nrhs, const double* const* d_srcden,
                                     double* const* d_trgval, void* stream, int sync);
const char* kifmm_batch_last_error(kifmm_batch b);
/* kifmm_poll_status over the batch's instances (synchronous replays poll
 * themselves; an asynchronous replay's time-out is reported by the next
 * kifmm_batch_eval_device or by this call after the stream is synchronised). */
kifmm_status kifmm_batch_poll_status(kifmm_batch b);

/* Replaces FMM3d::check(srcden, trgval, numchk) (fmm3d/fmm3d_check.cpp:25-73):
 * FP64 direct sum at numchk targets picked with `seed`; returns
 * ||fmm - direct|| / ||fmm|| in *relerr (the reference's metric, :61-71). */
kifmm_status kifmm_check(kifmm_handle h, const double* srcden, const double* trgval, int numchk, uint64_t seed,
                         double* relerr);

/* Replaces Dense3d::eval (fmm3d/dense3d.cpp:38-57) on the device: FP64
 * direct sum from the handle's sources to arbitrary targets (host arrays). */
kifmm_status kifmm_direct(kifmm_handle h, const double* srcden, int nt, const double* trgpos, double* trgval);

/* No counterpart in the reference.  FP64 direct sum (the kernels of
 * kifmm_direct) for callers that cannot allocate device memory: a process
 * whose GPU memory is owned by a framework's caching allocator or a fixed
 * budget reserved at start-up cannot call cudaMalloc between its steps.
 * All pointers are device pointers the caller allocated (layouts as in
 * kifmm_direct); the work is enqueued on `stream` (NULL = legacy default
 * stream) and the call does not synchronise.  The call allocates nothing:
 * its partial sums live in one fixed device array of
 * KIFMM_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB, held on every GPU that loads
 * the library until exit), so nt * tdof above that limit returns
 * KIFMM_ERR_CAPACITY.  Every call looks the array up on the current device
 * (cudaGetSymbolAddress, which allocates nothing); the first call on a
 * device loads the module there and should come before any stream capture.
 * An error already pending from the caller's earlier work is returned as
 * KIFMM_ERR_CUDA before anything is launched, and left pending.  All calls
 * share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
#define KIFMM_NOALLOC_SCRATCH_DOUBLES (1 << 20)
kifmm_status kifmm_direct_noalloc(int kt, int ncoef, const double* coefs, int ns, const double* d_srcpos,
                                  const double* d_srcnor, const double* d_srcden, int nt, const double* d_trgpos,
                                  double* d_trgval, void* stream);

/* Tree introspection (Let3d, fmm3d/let3d.hpp:38-74), for list parity tests.
 * Nodes are numbered exactly as the reference's breadth-first ndevec. */
kifmm_status kifmm_tree_size(kifmm_handle h, int* nnodes, int* maxdepth);
kifmm_status kifmm_tree_nodes(kifmm_handle h, int* depth, int* path, int* parent, int* child, int* tag,
                              int* snum, int* tnum);
/* which: 0=U 1=V 2=W 3=X.  total receives the list length sum; ptr (nnodes+1)
 * and idx (total) may be NULL to query the size first. */
kifmm_status kifmm_tree_lists(kifmm_handle h, int which, int64_t* total, int64_t* ptr, int* idx);
/* Original point ids per node, grouped by leaf: 0=sources (sownvis) 1=targets (townvis). */
kifmm_status kifmm_tree_points(kifmm_handle h, int which, int64_t* ptr, int* idx);

/* sdof / tdof of the handle's kernel (Kernel3d::sdof/tdof, fmm3d/kernel3d.cpp:24-86). */
kifmm_status kifmm_dofs(kifmm_handle h, int* sdof, int* tdof);

/* Per-phase device times (ms) of the last eval, measured with CUDA events
 * on the engine stream: [0] upward, [1] M2L, [2] X/S2L, [3] downward,
 * [4] leaf (U/W/X/L2T), [5] total, and inside [1]: [6] forward spectra,
 * [7] Hadamard accumulation, [8] inverse spectra.  n = entries written. */
kifmm_status kifmm_phase_times(kifmm_handle h, double* ms, int* n);
/* Host wall-clock times (ms) of the last kifmm_setup: [0] octree and
 * U/V/W/X lists (built on the GPU unless -<prefix>tree host), [1] the
 * translation operators (cached per kernel and np), [2] device data and
 * work lists, [3] schedule autotuning (-<prefix>autotune 1).  n = entries
 * written. */
kifmm_status kifmm_setup_times(kifmm_handle h, double* ms, int* n);
/* The evaluation schedule in use (no counterpart in the reference, whose
 * eval has a single fixed schedule): [0] producer warp groups of the FP16
 * tensor-core V-list Hadamard (2 or 3), [1] density vectors carried by one
 * pass of the surface contractions (0: as many as fit, at most 8), [2] 1 if
 * setup autotuned them (-<prefix>autotune 1: every candidate timed on
 * -<prefix>autotune_rhs synthetic density vectors, the fastest kept), [3] 1
 * if the choice came from the process-wide cache of an earlier setup with
 * the same kernel, np, precision, V-list form, tree size class and vector
 * count, [4] candidates timed, [5] the best candidate's ms per eval.
 * n = entries written (6). */
kifmm_status kifmm_schedule(kifmm_handle h, double* values, int* n);
/* Enables (1) or disables (0) per-phase event timing (off by default). */
kifmm_status kifmm_set_profiling(kifmm_handle h, int on);

/* Work counters of the setup, for roofline accounting:
 * [0] U-list point-point interactions, [1] V-list node pairs,
 * [2] W/X direct interactions, [3] nodes, [4] leaves, [5] surface GEMM flops
 * per eval, [6] forward spectra per eval, [7] inverse spectra per eval,
 * [8] S2M + L2T + M2T + S2L point-surface interactions, [9] tensor-core flops
 * per eval of the V-list Hadamard (0 unless that form is used). */
kifmm_status kifmm_work_counters(kifmm_handle h, double* counts, int* n);

/* Number of this library's kernel launches issued by the last eval. */
kifmm_status kifmm_last_launch_count(kifmm_handle h, int* nlaunch);

const char* kifmm_status_string(kifmm_status s);
/* Last error message of the handle (valid until the next call on it). */
const char* kifmm_last_error(kifmm_handle h);

#ifdef __cplusplus
}
#endif
#endif
