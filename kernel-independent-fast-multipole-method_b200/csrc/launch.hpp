// Host-callable launchers of the device passes (one stream argument each;
// no synchronisation inside).  Argument structs hold device pointers only.
#pragma once

#include <cuda_runtime.h>
#include <complex>

#include <vector>
#include <stdint.h>

#include "kernels_common.cuh"

namespace kifmm {

// Device view of the tree, points and per-node surface data of one engine.
template <typename T>
struct P2PArgs {
  int nnodes = 0, ns = 0, nt = 0, nsurf = 0, nuc = 0;
  const int *sbeg = nullptr, *scnt = nullptr, *tbeg = nullptr, *tcnt = nullptr, *depth = nullptr;
  const double *center = nullptr, *radius = nullptr;
  // sorted points, coordinates relative to their leaf centre
  const T *sx = nullptr, *sy = nullptr, *sz = nullptr, *snx = nullptr, *sny = nullptr, *snz = nullptr;
  const T* sden = nullptr;  // [rhs][ns][sd]
  const T *tx = nullptr, *ty = nullptr, *tz = nullptr;
  T* tval = nullptr;  // [rhs][nt][td]
  // unit surface grids (3 per point): UE radius 1, UC radius 3, DE radius 3, DC radius 1
  const T *ue_unit = nullptr, *uc_unit = nullptr, *de_unit = nullptr, *dc_unit = nullptr;
  // per-node surface data [node][point][dof] (one density vector at a time)
  const T* supeden = nullptr;
  const T* tdneden = nullptr;
  T* supcval = nullptr;
  T* tdncval = nullptr;
  KConst<T> ku{}, km{};  // user and equivalent kernel constants
  // leaves at this depth and below add L2T from their downward equivalent
  // surface in the leaf pass (a pass with near-field sources only sets it
  // beyond the deepest level)
  int l2t_depth = 2;
};

enum { P2P_S2M = 0, P2P_S2L = 1, P2P_LEAF = 2 };

struct P2PWork {
  const int* work = nullptr;  // node ids, one CTA each
  int n = 0;
  const int64_t* ptr = nullptr;  // CSR over work items (S2L: X leaves; LEAF: point-source leaves)
  const int* idx = nullptr;
  const int64_t* ptr2 = nullptr;  // LEAF: M2T source nodes
  const int* idx2 = nullptr;
};

template <typename T>
void launch_p2p(int kt, const P2PArgs<T>& a, const P2PWork& w, int which, int rhs, cudaStream_t st);

void launch_direct(int kt, const double* spos, const double* snor, const double* sden, int ns, const double* tpos,
                   int nt, double* out, const double* kc3, cudaStream_t st);

template <typename T>
void launch_scatter_den(const double* srcden, const int* perm, int ns, int sd, int nrhs, T* out, cudaStream_t st);
template <typename T>
void launch_gather_val(const T* tval, const int* perm, int nt, int td, int nrhs, double* trgval, cudaStream_t st);
// the same gather of tval + near (an FP64 near-field sum beside FP32 passes)
void launch_gather_val_sum(const float* tval, const double* near, const int* perm, int nt, int td, int nrhs,
                           double* trgval, cudaStream_t st);

// Batched node GEMM: for j < ncol,
//   C[cidx[j]*ldc + r] (=|+=) rs(j, r) * sum_k A[r*K + k] * B[bidx[j]*ldb + k]
// A is M x K row-major.  rs(j, r) = 2^(-(col_lvl[j] + lvl_base) * deg[r % sd])
// when col_lvl is set (homogeneous level scaling, one launch covering nodes of
// every level), else 1.
struct GemmScale {
  int sd = 1;
  int deg[4] = {0, 0, 0, 0};
  const int* col_lvl = nullptr;
  int lvl_base = 0;
};

// ws (FP64, ws_len doubles) lets a launch with few columns split K over
// several CTAs; pass nullptr to disable.
template <typename T>
int launch_node_gemm(int M, int K, const T* A, const T* B, int64_t ldb, const int* bidx, T* C, int64_t ldc,
                      const int* cidx, int ncol, bool accumulate, const GemmScale& sc, double* ws, size_t ws_len,
                      int num_sms, cudaStream_t st);

// The same product on the tensor cores (tcgen05, kind::tf32) for FP32 data,
// with both operands split into a TF32 head and a TF32 tail and three MMAs
// (head*head + head*tail + tail*head) accumulating in FP32: about 2^-21
// relative per product, the FP32 rounding class.  The operator is split on
// the host into shared-memory images, one per (N tile, 32-wide K chunk):
// head then tail, each 160 rows x 32 columns in the no-swizzle K-major
// core-matrix layout (zero padded), so that one bulk copy moves a chunk.
// Requires K, ldb, ldc multiples of 4 and 16-byte aligned B and C.  Launches
// with fewer tiles than SMs split K over CTAs into ws (FP64, ws_len doubles)
// and reduce it deterministically.  A bounded wait that times out sets bit 1
// of *status.  Returns the number of launches.
struct TcOperator {
  const float* img = nullptr;  // [ntiles][Kp/32][2][160 x 32]
  int M = 0, K = 0, Np = 0, Kp = 0;
  int ntile = 0, ntiles = 0;  // rows per N tile (multiple of 16, <= 160), number of N tiles
};
int launch_node_gemm_tc(const TcOperator& A, const float* B, int64_t ldb, const int* bidx, float* C, int64_t ldc,
                        const int* cidx, int ncol, bool accumulate, const GemmScale& sc, double* ws, size_t ws_len,
                        int num_sms, int* status, cudaStream_t st);
// host side: the images of a row-major M x K operator (fills A's sizes; img
// is left to the caller to upload)
void tc_operator_images(int M, int K, const double* A, std::vector<float>* img, TcOperator* desc);
// C[cidx[j]] (=|+=) scaled sum over nslice of partial[z][j][0..M) (gemm.cu)
void launch_node_gemm_reduce_f(int M, int ncol, int nslice, const double* partial, float* C, int64_t ldc,
                               const int* cidx, bool accumulate, const GemmScale& sc, int num_sms, cudaStream_t st);
// host-side split of a row-major M x K operator into the padded hi/lo pair
void split_tf32(int M, int K, const double* A, std::vector<float>* hi, std::vector<float>* lo, int* Np, int* Kp);

// FFT-based M2L (MatMgnt3d::plnden2effden / UE2DC_dgemv / effval2plnval,
// fmm3d/matmgnt3d.cpp:223-361).
struct M2LGeom {
  int np = 0, n = 0, nh = 0, nfreq = 0, nsurf = 0;
  int nfc = 0;                // stored (Hermitian-canonical) frequencies per spectrum
  const int* fc2f = nullptr;  // device: compact -> full frequency index
  const int* ff2c = nullptr;  // device: full -> compact c, or -c-1 for conj(compact c)
  const int* surf_ijk = nullptr;  // device, 3 per surface point
  int sd = 1, td = 1;
  int deg[4] = {0, 0, 0, 0};
  int rootlvl = 0;
  // 2: the sibling-group-major layout holding FP16 pairs (below)
  // 0: spectra[node][s][f]; 1 (single dof): sibling-group major,
  // spectra[(node + 7) / 8][f / 4][(node + 7) % 8][f % 4] -- every sibling
  // group's spectra one block, and in it the 8 children's values of 4
  // frequencies 256 contiguous bytes (first children are 1 mod 8)
  int sg = 0;
  // sg == 2: each complex value x is stored as the FP16 pairs
  // {hi(re), hi(im)}, {lo(re), lo(im)} of x * 2^(14 - e), where 2^e >= the
  // FP32 value *bound (k_spectra_bound) -- the operands of the 16-bit
  // tensor-core Hadamard, in the 8 bytes (spectra_sg_index) the FP32 value
  // would take
  const unsigned* bound = nullptr;
  // accumulated spectra in the sibling-group-major layout of
  // spectra_sg_index instead of [node][td][nfc] (written so by the FP16
  // tensor-core Hadamard)
  int effval_sg = 0;
  // sg == 2 and effval_sg: complex slots per dof plane of the
  // sibling-group-major spectra (dof s at s * plane + spectra_sg_index)
  size_t plane = 0;
};
// complex index of (node, compact frequency c) in the sibling-group-major
// layout of nfc frequencies (a multiple of 4)
__host__ __device__ inline size_t spectra_sg_index(int nfc, int node, int c) {
  return (((size_t)((node + 7) >> 3) * (nfc >> 2) + (c >> 2)) * 8 + ((node + 7) & 7)) * 4 + (c & 3);
}

// spectra[node][s][f] (complex, interleaved re/im) of 2^(l*deg) * supeden[node]
template <typename T>
void launch_m2l_forward(const M2LGeom& g, const T* supeden, const int* nodes, int nnodes_work, const int* depth,
                        T* spectra, cudaStream_t st);
// effval[w][t][f] = sum_{s in V(work[w])} Khat[offset] * spectra[s]
template <typename T>
void launch_m2l_hadamard(const M2LGeom& g, const T* khat, const T* spectra, const int* work, int nwork,
                         const int64_t* vptr, const int* vidx, const int* path, T* effval, cudaStream_t st);
// Parent-pair form: effval[child of Q] for the nq target parents Q (first
// child qchd[q], colleague first children coll[q][26], the all-zero block
// zero_node when absent, V-list children mask[q]).  ktiles: operator spectra
// as [td][sd][ceil(nf/32)][343][32] complex, zero-padded; one pass per
// (target dof, source dof).  A mbarrier wait that times out sets bit 0 of
// *status.  Requires m2l_sweep_supported(nf, sd, td) (np = 4, 6, 8; dofs
// 1->1, 4->3, 3->3).
bool m2l_sweep_supported(int nf, int sd, int td);
template <typename T>
void launch_m2l_hadamard_sweep(int nf, int sd, int td, const T* ktiles, const T* spectra, int nq, const int* qchd,
                               const int* coll, const unsigned char* mask, T* effval, int zero_node, int* status,
                               int num_sms, cudaStream_t st);
// The same product with the 2 x 2 x 2 block-Toeplitz factorisation of each
// colleague block (27 instead of 64 complex products per direction).  ttiles:
// [td][sd][ceil(nf/16)][26 directions][14][16][2] complex: for direction d
// and frequency lane l, the 27 transformed values k (padded to 28) stored as
// pairs (k, k+1) at [d][k/2][l][k%2].
template <typename T>
void launch_m2l_hadamard_tz(int nf, int sd, int td, const T* ttiles, const T* spectra, int nq, const int* qchd,
                            const int* coll, const unsigned char* mask, T* effval, int zero_node, int* status,
                            int num_sms, cudaStream_t st);
// The same product for single-dof kernels in FP32 on the tensor cores
// (m2l_tc.cu): tiles of 128 target parents, per frequency a split-TF32 MMA
// with the gathered colleague spectra in TMEM; spectra in the
// sibling-group-major layout.  img: per (chunk of 4
// frequencies, direction) the head and tail images of the 16 x 16 real
// blocks (m2l_tc_images); tile_dirs[t]: the directions present among tile
// t's parents (bit d; never 0).  A wait that times out sets bit 2 of *status.
bool m2l_tc_supported(int nf, int sd, int td);
void m2l_tc_images(int nf, const std::complex<double>* m2l, std::vector<float>* img);
void launch_m2l_hadamard_tc(int nf, const float* img, const float* spectra, int nq, const int* qchd,
                            const int* coll, const unsigned char* mask, const unsigned* tile_dirs, float* effval,
                            int zero_node, int* status, int num_sms, cudaStream_t st);
// The same product on the tensor cores with FP16-pair operands (kind::f16,
// m2l_tc16.cu): spectra written by the forward pass in the sg == 2 layout
// (scaled by the data bound *bound), img per (chunk of 4 frequencies,
// direction) the hi and lo FP16 images of the 16 x 16 real blocks, scaled by
// 1 / inv_sb[chunk] (m2l_tc16_images).  groups: producer warp groups = TMEM A
// stages (2 or 3 groups: 4 or 6 stages).  wait_limit bounds every pipeline
// wait (polls); a time-out sets bit 3 of *status.
// Equivalent kernels with sd x td dofs (1 x 1, Stokes 4 x 3, Navier 3 x 3):
// the images are [chunk][direction][td][sd]; the source spectra and the
// accumulated spectra hold one sibling-group-major plane of `plane` complex
// slots per dof, and a work item is (chunk, target dof, tile) whose steps
// are (direction, source dof).
bool m2l_tc16_supported(int nf, int sd, int td);
void m2l_tc16_images(int nf, int sd, int td, const std::complex<double>* m2l, std::vector<unsigned short>* img,
                     std::vector<float>* inv_sb);
// *bound = max over nodes and source dofs s of 2^((depth + rootlvl) deg[s]) *
// sum_k |supeden[node][k][s]| (FP32 bits)
void launch_spectra_bound(const float* supeden, const int* nodes, int n, const int* depth, int rootlvl,
                          const int* deg, int sd, int nsurf, unsigned* bound, int num_sms, cudaStream_t st);
void launch_m2l_hadamard_tc16(int groups, int nf, int sd, int td, const unsigned short* img,
                              const unsigned* spectra, int nq, const int* qchd, const int* ctab,
                              const unsigned* tile_dirs, float* effval, size_t plane, const unsigned* bound,
                              const float* inv_sb, int wait_limit, int* status, int num_sms, cudaStream_t st);
// colleague tables of the FP16 form: per tile of 128 target parents and
// direction, the sibling group ((first child + 7) / 8) of each row's colleague
// (the all-zero group for an absent one or a padding row), [tile][26][128]
void m2l_tc16_tables(int nq, int zero_node, const int* coll, std::vector<int>* ctab);
// tdncval[node] += extract(inverse(effval[node]))
template <typename T>
void launch_m2l_inverse(const M2LGeom& g, const T* effval, const int* work, int nwork, T* tdncval,
                        cudaStream_t st);

}  // namespace kifmm
