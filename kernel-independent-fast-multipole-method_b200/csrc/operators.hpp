// Translation operators of the KIFMM (host FP64 precompute, once per
// (equivalent kernel, np), cached process-wide like the reference's
// MatMgnt3d::getmmptr cache, fmm3d/matmgnt3d.cpp:438-452).
//
//   surface grids      MatMgnt3d::splposcal, fmm3d/matmgnt3d.cpp:375-398
//   UC2UE, DC2DE       pseudo-inverses, fmm3d/matmgnt3d.cpp:91-123,158-188
//   UE2UC, DE2DC       child/parent matrices, fmm3d/matmgnt3d.cpp:125-156,190-221
//   M2L spectra        FFT of the kernel sampled on the (2np)^3 grid,
//                      fmm3d/matmgnt3d.cpp:296-361 (regposcal :400-420)
//
// The device passes use the pseudo-inverses in factored form (see Operators);
// the per-level homogeneous scalings 2^(+-l*deg) (fmm3d/matmgnt3d.cpp:107-118,
// 141-153) are applied in the epilogue of the V-factor GEMMs.
#pragma once

#include <complex>
#include <memory>
#include <string>
#include <vector>

namespace kifmm {

// Kernel ids of fmm3d/kernel3d.hpp:29-53 handled by FMM3d::setup.
struct KernelDesc {
  int kt = 0;
  int sd = 0, td = 0;
  bool dl = false;  // double layer: needs source normals
  double coefs[2] = {1.0, 0.25};
};

bool kernel_desc(int kt, const double* coefs, int ncoef, KernelDesc* out);
// FMM3d::setup's choice of equivalent-density kernel, fmm3d/fmm3d_setup.cpp:41-54.
bool equivalent_kernel(const KernelDesc& user, KernelDesc* mm);
// Homogeneity degree per source dof, Kernel3d::homsdeg (fmm3d/kernel3d.cpp:103-112).
void homogeneous_degrees(int kt_mm, std::vector<int>* deg);

// Row-major (n_t*td) x (n_s*sd) kernel matrix, Kernel3d::kernel semantics
// (fmm3d/kernel3d.cpp:116-414), including the r < 1e-8 cut-off.
void kernel_matrix(const KernelDesc& k, int nt, const double* trg, int ns, const double* src, const double* nor,
                   double* out);

// Pseudo-inverse V S^-1 U^T with singular values below rel_cut * s_max
// dropped (pinv + SVDRep::construct, common/vecmatop.cpp:124-159,
// common/svdrep.cpp:31-74).  a is m x n row-major; out is n x m row-major.
// Returns false if the one-sided Jacobi SVD did not converge.
bool pseudo_inverse(int m, int n, const double* a, double rel_cut, double* out, int nthreads);
// Same truncated SVD, returned as factors pinv = V * W: V is n x r with
// orthonormal columns, W = Sigma^-1 U^T is r x m (both row-major).
bool pinv_factors(int m, int n, const double* a, double rel_cut, int nthreads, std::vector<double>* V,
                  std::vector<double>* W, int* rank);

struct Operators {
  KernelDesc mm;
  int np = 0;
  int nsurf = 0;          // |UE| = |DE| = |DC| = np^3 - (np-2)^3
  int nuc = 0;            // |UC| = (np+2)^3 - np^3
  int n = 0, nh = 0;      // FFT grid 2np, halved axis n/2+1
  int nfreq = 0;          // n*n*nh
  int nfc = 0;            // independent (Hermitian-canonical) frequencies, 4 np^3 + 4
  std::vector<int> fc2f;  // compact -> full frequency index
  std::vector<int> ff2c;  // full -> compact index c, or -c-1 where the value is conj(compact c)
  std::vector<int> deg;   // per sd
  std::vector<double> ue, uc, de, dc;   // unit grids (3 per point), radii 1, 3, 3, 1
  std::vector<int> surf_ijk;            // (i,j,k) grid index of each np-surface point
  std::vector<std::complex<double>> m2l;  // [343 offsets][td][sd][nfc], scaled by 1/n^3
  // Surface contractions in factored form.  UC2UE = pinv(K(UC <- UE)) =
  // up_V * up_W and DC2DE = pinv(K(DC <- DE)) = dn_V * dn_W, V with orthonormal
  // columns and W = Sigma^-1 U^T.  The pseudo-inverses' entries reach
  // 10^(np+1) times the data; applied as the two well-conditioned factors the
  // products stay accurate in FP32, and the M2M / L2L chains run in the
  // rank-r coordinates y = up_W * check and z = dn_W * check.
  int rank_up = 0, rank_dn = 0;
  std::vector<double> up_W;    // rank_up x (nuc*td)
  std::vector<double> up_V;    // (nsurf*sd) x rank_up
  std::vector<double> m2m_y;   // rank_up x (8*rank_up): block o = up_W * UE2UC_o * up_V
  std::vector<double> dn_W;    // rank_dn x (nsurf*td)
  std::vector<double> dn_V;    // (nsurf*sd) x rank_dn
  std::vector<double> l2l_z;   // (8*rank_dn) x rank_dn: row block o = dn_W * DE2DC_o * dn_V
  // Per-level form (the reference's non-homogeneous branch, _hom == false in
  // fmm3d/matmgnt3d.cpp:93-361): every operator built at this level's box
  // radius R = 2^-level instead of at R = 1, no 2^(+-l deg) scaling (deg all
  // zero), and the two child/parent matrices kept raw so that the level set
  // can chain them with the neighbouring level's factors:
  //   ue2uc_raw[o]  K(2R UC <- R UE + (2 idx_o - 1) R)   children at this level
  //   de2dc_raw[o]  K(R DC / 2 + (idx_o - 1/2) R <- R DE) parent at this level
  int level = -1;  // < 0: the homogeneous (scaled) form at R = 1
  double R = 1.0;
  std::vector<double> ue2uc_raw;  // [8][(nuc*td) x (nsurf*sd)]
  std::vector<double> de2dc_raw;  // [8][(nsurf*td) x (nsurf*sd)]
};

// Builds (or returns the cached) operators; nullptr + err on failure.
std::shared_ptr<const Operators> get_operators(const KernelDesc& mm, int np, int nthreads, std::string* err);

// The per-level operator set for absolute levels lmin..lmax: ops[l - lmin]
// built at R = 2^-l, and the rank-space chains between neighbouring levels
//   m2m_y[l - lmin]  (rank_up(l) x 8 rank_up(l+1)), block o =
//                    up_W(l) * ue2uc_raw(l+1)[o] * up_V(l+1)
//   l2l_z[l - lmin]  (8 rank_dn(l+1) x rank_dn(l)), row block o =
//                    dn_W(l+1) * de2dc_raw(l)[o] * dn_V(l)
// (fmm3d/matmgnt3d.cpp:125-156, 190-221 with R = 2^-l).
struct LevelOperators {
  int lmin = 0, lmax = 0;
  std::vector<std::shared_ptr<const Operators>> ops;
  std::vector<std::vector<double>> m2m_y, l2l_z;
};
std::shared_ptr<const LevelOperators> get_level_operators(const KernelDesc& mm, int np, int lmin, int lmax,
                                                          int nthreads, std::string* err);

// Surface grid of MatMgnt3d::splposcal(np, R): the np^3 lattice on [-R,R]^3
// restricted to its boundary, x outermost and z innermost.
void surface_grid(int np, double R, std::vector<double>* pos, std::vector<int>* ijk);

inline int offset_index(int dx, int dy, int dz) { return (dx + 3) * 49 + (dy + 3) * 7 + (dz + 3); }

}  // namespace kifmm
