// Host FP64 precompute of the KIFMM translation operators; see operators.hpp.
#include "operators.hpp"

#include <algorithm>
#include <barrier>
#include <cmath>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>

namespace kifmm {

bool kernel_desc(int kt, const double* coefs, int ncoef, KernelDesc* out) {
  KernelDesc k;
  k.kt = kt;
  switch (kt) {  // Kernel3d::sdof/tdof, fmm3d/kernel3d.cpp:24-86
    case 111: k.sd = 1; k.td = 1; break;
    case 121: k.sd = 1; k.td = 1; k.dl = true; break;
    case 301: k.sd = 4; k.td = 3; break;
    case 311: k.sd = 3; k.td = 3; break;
    case 312: k.sd = 3; k.td = 1; break;
    case 321: k.sd = 3; k.td = 3; k.dl = true; break;
    case 322: k.sd = 3; k.td = 1; k.dl = true; break;
    case 511: k.sd = 3; k.td = 3; break;
    case 521: k.sd = 3; k.td = 3; k.dl = true; break;
    default: return false;
  }
  int need = (kt == 511 || kt == 521) ? 2 : (kt == 111 || kt == 121) ? 0 : 1;  // iA(_coefs.size()>=..)
  if (ncoef < need) return false;
  for (int i = 0; i < 2 && i < ncoef; i++) k.coefs[i] = coefs[i];
  if (need >= 1 && k.coefs[0] == 0.0) return false;
  *out = k;
  return true;
}

bool equivalent_kernel(const KernelDesc& u, KernelDesc* mm) {
  int kmm;
  switch (u.kt) {  // fmm3d/fmm3d_setup.cpp:41-54
    case 111: case 121: case 312: case 322: kmm = 111; break;
    case 311: case 321: kmm = 301; break;
    case 511: case 521: kmm = 511; break;
    default: return false;
  }
  double c[2] = {u.coefs[0], u.coefs[1]};
  // the pressure kernels use a coefficient-free Laplace kernel (fmm3d_setup.cpp:47,49)
  return kernel_desc(kmm, c, (kmm == 111) ? 0 : 2, mm);
}

void homogeneous_degrees(int kt_mm, std::vector<int>* deg) {
  switch (kt_mm) {  // fmm3d/kernel3d.cpp:103-112
    case 111: *deg = {1}; break;
    case 301: *deg = {1, 1, 1, 2}; break;
    case 511: *deg = {1, 1, 1}; break;
    default: deg->clear();
  }
}

// One (target, source) block, row-major [td][sd]; fmm3d/kernel3d.cpp:116-369.
static void block(const KernelDesc& k, const double* x, const double* n, double* b) {
  double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
  double r = std::sqrt(r2);
  int sd = k.sd, td = k.td;
  if (r < 1e-8) {  // Kernel3d::_mindif
    for (int i = 0; i < sd * td; i++) b[i] = 0.0;
    return;
  }
  double r3 = r2 * r, r5 = r3 * r2;
  double rn = k.dl ? x[0] * n[0] + x[1] * n[1] + x[2] * n[2] : 0.0;
  switch (k.kt) {
    case 111: b[0] = 1.0 / (4.0 * M_PI) / r; break;
    case 121: b[0] = -1.0 / (4.0 * M_PI) / r3 * rn; break;
    case 301: {
      double mu = k.coefs[0];
      double G = (1.0 / mu) / (8.0 * M_PI) / r, H = (1.0 / mu) / (8.0 * M_PI) / r3, A = 1.0 / (4.0 * M_PI) / r3;
      for (int a = 0; a < 3; a++) {
        for (int c = 0; c < 3; c++) b[a * 4 + c] = (a == c ? G : 0.0) + H * x[a] * x[c];
        b[a * 4 + 3] = A * x[a];
      }
      break;
    }
    case 311: {
      double oomu = 1.0 / k.coefs[0];
      double G = 1.0 / (8.0 * M_PI) / r, H = 1.0 / (8.0 * M_PI) / r3;
      for (int a = 0; a < 3; a++)
        for (int c = 0; c < 3; c++) b[a * 3 + c] = oomu * ((a == c ? G : 0.0) + H * x[a] * x[c]);
      break;
    }
    case 312:
      for (int c = 0; c < 3; c++) b[c] = 1.0 / (4.0 * M_PI) * x[c] / r3;
      break;
    case 321: {
      double C = -6.0 / (8.0 * M_PI) / r5;
      for (int a = 0; a < 3; a++)
        for (int c = 0; c < 3; c++) b[a * 3 + c] = C * rn * x[a] * x[c];
      break;
    }
    case 322: {
      double coef = k.coefs[0] / (2.0 * M_PI);
      for (int c = 0; c < 3; c++) b[c] = coef * (n[c] / r3 - 3 * rn * x[c] / r5);
      break;
    }
    case 511: {
      double mu = k.coefs[0], ve = k.coefs[1];
      double sc1 = (3.0 - 4.0 * ve) / (16.0 * M_PI * (1.0 - ve)), sc2 = 1.0 / (16.0 * M_PI * (1.0 - ve));
      double G = sc1 / r, H = sc2 / r3;
      for (int a = 0; a < 3; a++)
        for (int c = 0; c < 3; c++) b[a * 3 + c] = (1.0 / mu) * ((a == c ? G : 0.0) + H * x[a] * x[c]);
      break;
    }
    case 521: {
      double ve = k.coefs[1];
      double A = -(1 - 2.0 * ve) / (8.0 * M_PI * (1.0 - ve)) / r3;
      double B = (1 - 2.0 * ve) / (8.0 * M_PI * (1.0 - ve)) / r3;
      double C = -3.0 / (8.0 * M_PI * (1.0 - ve)) / r5;
      for (int a = 0; a < 3; a++)
        for (int c = 0; c < 3; c++)
          b[a * 3 + c] = A * ((a == c ? rn : 0.0) + n[a] * x[c]) + B * (x[a] * n[c]) + C * rn * x[a] * x[c];
      break;
    }
  }
}

void kernel_matrix(const KernelDesc& k, int nt, const double* trg, int ns, const double* src, const double* nor,
                   double* out) {
  int sd = k.sd, td = k.td;
  size_t ld = (size_t)ns * sd;
  double b[16];
  for (int i = 0; i < nt; i++)
    for (int j = 0; j < ns; j++) {
      double x[3] = {trg[3 * i] - src[3 * j], trg[3 * i + 1] - src[3 * j + 1], trg[3 * i + 2] - src[3 * j + 2]};
      block(k, x, nor ? nor + 3 * (size_t)j : nullptr, b);
      for (int a = 0; a < td; a++)
        for (int c = 0; c < sd; c++) out[((size_t)i * td + a) * ld + (size_t)j * sd + c] = b[a * sd + c];
    }
}

void surface_grid(int np, double R, std::vector<double>* pos, std::vector<int>* ijk) {
  pos->clear();
  if (ijk) ijk->clear();
  double step = 2.0 / (np - 1);
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++)
      for (int k = 0; k < np; k++)
        if (i == 0 || i == np - 1 || j == 0 || j == np - 1 || k == 0 || k == np - 1) {
          pos->push_back(R * (-1.0 + i * step));
          pos->push_back(R * (-1.0 + j * step));
          pos->push_back(R * (-1.0 + k * step));
          if (ijk) {
            ijk->push_back(i);
            ijk->push_back(j);
            ijk->push_back(k);
          }
        }
}

// ---------------------------------------------------------------------------
// One-sided Jacobi SVD (Hestenes) with round-robin parallel pair ordering.
// ---------------------------------------------------------------------------
// On return B V = U with B = tr ? A^T : A (R x C, R >= C); the columns of U
// (column-major, R per column) are orthogonal with norms sigma_c, V (C x C,
// column-major) is orthogonal.
static bool jacobi_svd(int m, int n, const double* a, int nthreads, bool& tr, int& R, int& C, std::vector<double>& U,
                       std::vector<double>& V) {
  tr = m < n;
  R = tr ? n : m;
  C = tr ? m : n;
  U.assign((size_t)R * C, 0.0);
  V.assign((size_t)C * C, 0.0);
  for (int c = 0; c < C; c++)
    for (int r = 0; r < R; r++) U[(size_t)c * R + r] = tr ? a[(size_t)c * n + r] : a[(size_t)r * n + c];
  for (int c = 0; c < C; c++) V[(size_t)c * C + c] = 1.0;
  int P = C + (C & 1);  // players (one dummy when odd)
  std::vector<int> ring(P);
  for (int i = 0; i < P; i++) ring[i] = i;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > P / 2) nthreads = std::max(1, P / 2);
  std::vector<double> offmax(nthreads, 0.0);
  const double tol = 1e-15;
  bool converged = false;
  int sweep = 0;
  std::barrier sync(nthreads);
  std::vector<int> round_pairs(P);
  auto rotate_pair = [&](int p, int q, double* off) {
    if (p >= C || q >= C) return;
    double* up = &U[(size_t)p * R];
    double* uq = &U[(size_t)q * R];
    double al = 0, be = 0, ga = 0;
    for (int r = 0; r < R; r++) {
      al += up[r] * up[r];
      be += uq[r] * uq[r];
      ga += up[r] * uq[r];
    }
    if (al == 0.0 || be == 0.0) return;
    double rel = std::fabs(ga) / std::sqrt(al * be);
    if (rel > *off) *off = rel;
    if (rel <= tol) return;
    double zeta = (be - al) / (2.0 * ga);
    double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
    double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
    for (int r = 0; r < R; r++) {
      double x = up[r], y = uq[r];
      up[r] = c * x - s * y;
      uq[r] = s * x + c * y;
    }
    double* vp = &V[(size_t)p * C];
    double* vq = &V[(size_t)q * C];
    for (int r = 0; r < C; r++) {
      double x = vp[r], y = vq[r];
      vp[r] = c * x - s * y;
      vq[r] = s * x + c * y;
    }
  };
  auto worker = [&](int th) {
    for (int sw = 0; sw < 60; sw++) {
      offmax[th] = 0.0;
      for (int rd = 0; rd < P - 1; rd++) {
        // circle method: player ring[0] fixed, the rest rotate each round
        int npair = P / 2;
        for (int k = th; k < npair; k += nthreads) {
          int p = ring[k], q = ring[P - 1 - k];
          if (p > q) std::swap(p, q);
          rotate_pair(p, q, &offmax[th]);
        }
        sync.arrive_and_wait();
        if (th == 0) {
          int last = ring[P - 1];
          for (int i = P - 1; i > 1; i--) ring[i] = ring[i - 1];
          ring[1] = last;
        }
        sync.arrive_and_wait();
      }
      bool done = true;
      for (double o : offmax)
        if (o > tol) done = false;
      sync.arrive_and_wait();
      if (done) {
        if (th == 0) {
          converged = true;
          sweep = sw;
        }
        return;
      }
    }
  };
  std::vector<std::thread> th;
  for (int i = 1; i < nthreads; i++) th.emplace_back(worker, i);
  worker(0);
  for (auto& x : th) x.join();
  (void)sweep;
  return converged;
}

bool pinv_factors(int m, int n, const double* a, double rel_cut, int nthreads, std::vector<double>* Vout,
                  std::vector<double>* Wout, int* rank) {
  bool tr;
  int R, C;
  std::vector<double> U, V;
  if (!jacobi_svd(m, n, a, nthreads, tr, R, C, U, V)) return false;
  std::vector<double> sig(C);
  double smax = 0.0;
  for (int c = 0; c < C; c++) {
    double s = 0;
    for (int r = 0; r < R; r++) s += U[(size_t)c * R + r] * U[(size_t)c * R + r];
    sig[c] = std::sqrt(s);
    smax = std::max(smax, sig[c]);
  }
  std::vector<int> keep;  // in decreasing singular value order
  for (int c = 0; c < C; c++)
    if (sig[c] >= rel_cut * smax && sig[c] > 0.0) keep.push_back(c);
  std::sort(keep.begin(), keep.end(), [&](int x, int y) { return sig[x] > sig[y]; });
  const int r = (int)keep.size();
  // pinv(A) = sum_c (n-vector p_c)(m-vector q_c)^T with p_c unit length:
  //   not transposed: p_c = V_c,          q_c = U_c / sigma_c^2
  //   transposed:     p_c = U_c / sigma_c, q_c = V_c / sigma_c
  Vout->assign((size_t)n * r, 0.0);
  Wout->assign((size_t)r * m, 0.0);
  for (int k = 0; k < r; k++) {
    int c = keep[k];
    const double* u = &U[(size_t)c * R];
    const double* v = &V[(size_t)c * C];
    double s = sig[c];
    for (int j = 0; j < n; j++) (*Vout)[(size_t)j * r + k] = tr ? u[j] / s : v[j];
    for (int i = 0; i < m; i++) (*Wout)[(size_t)k * m + i] = tr ? v[i] / s : u[i] / (s * s);
  }
  *rank = r;
  return true;
}

bool pseudo_inverse(int m, int n, const double* a, double rel_cut, double* out, int nthreads) {
  bool tr;
  int R, C;
  std::vector<double> U, V;
  if (!jacobi_svd(m, n, a, nthreads, tr, R, C, U, V)) return false;
  // singular values, truncation (common/svdrep.cpp:51-58)
  std::vector<double> sig(C);
  double smax = 0.0;
  for (int c = 0; c < C; c++) {
    double s = 0;
    for (int r = 0; r < R; r++) s += U[(size_t)c * R + r] * U[(size_t)c * R + r];
    sig[c] = std::sqrt(s);
    smax = std::max(smax, sig[c]);
  }
  double cut = rel_cut * smax;
  // B = sum_c (U_c/sig_c) sig_c V_c^T ; pinv(B) = sum_c V_c (1/sig_c) (U_c/sig_c)^T = sum_c V_c U_c^T / sig_c^2
  // out is n x m row-major.
  std::fill(out, out + (size_t)n * m, 0.0);
  for (int c = 0; c < C; c++) {
    if (!(sig[c] >= cut) || sig[c] == 0.0) continue;
    double w = 1.0 / (sig[c] * sig[c]);
    const double* u = &U[(size_t)c * R];
    const double* v = &V[(size_t)c * C];
    if (!tr) {  // pinv(A) (n x m) = V S^-1 U^T : out[j][i] += v[j] u[i] w, j<C=n, i<R=m
      for (int j = 0; j < n; j++) {
        double vj = v[j] * w;
        double* o = out + (size_t)j * m;
        for (int i = 0; i < m; i++) o[i] += vj * u[i];
      }
    } else {  // pinv(A) = U S^-1 V^T : out[j][i] += u[j] v[i] w, j<R=n, i<C=m
      for (int j = 0; j < n; j++) {
        double uj = u[j] * w;
        double* o = out + (size_t)j * m;
        for (int i = 0; i < m; i++) o[i] += uj * v[i];
      }
    }
  }
  return true;
}

// ---------------------------------------------------------------------------
namespace {

void matmul(int M, int K, int N, const double* A, const double* B, double* Cm) {  // row-major
  for (int i = 0; i < M; i++) {
    double* c = Cm + (size_t)i * N;
    for (int j = 0; j < N; j++) c[j] = 0.0;
    for (int k = 0; k < K; k++) {
      double a = A[(size_t)i * K + k];
      const double* b = B + (size_t)k * N;
      for (int j = 0; j < N; j++) c[j] += a * b[j];
    }
  }
}

template <class F>
void parallel_range(int n, int nthreads, F&& f) {
  std::vector<std::thread> th;
  nthreads = std::max(1, std::min(nthreads, n));
  for (int t = 0; t < nthreads; t++)
    th.emplace_back([&, t] {
      for (int i = t; i < n; i += nthreads) f(i);
    });
  for (auto& x : th) x.join();
}

// level < 0: the homogeneous form (R = 1, scaled per level by 2^(+-l deg));
// level >= 0: the per-level form at R = 2^-level (see Operators)
std::shared_ptr<Operators> build_operators(const KernelDesc& mm, int np, int nthreads, std::string* err,
                                           int level = -1) {
  auto op = std::make_shared<Operators>();
  Operators& o = *op;
  o.mm = mm;
  o.np = np;
  o.level = level;
  const double R = level < 0 ? 1.0 : std::ldexp(1.0, -level);
  o.R = R;
  if (level < 0)
    homogeneous_degrees(mm.kt, &o.deg);
  else
    o.deg.assign(mm.sd, 0);
  surface_grid(np, 1.0, &o.ue, &o.surf_ijk);  // MatMgnt3d::setup, fmm3d/matmgnt3d.cpp:51-54
  surface_grid(np + 2, 3.0, &o.uc, nullptr);
  surface_grid(np, 3.0, &o.de, nullptr);
  surface_grid(np, 1.0, &o.dc, nullptr);
  o.nsurf = (int)o.ue.size() / 3;
  o.nuc = (int)o.uc.size() / 3;
  o.n = 2 * np;
  o.nh = np + 1;
  o.nfreq = o.n * o.n * o.nh;
  const int sd = mm.sd, td = mm.td, ns = o.nsurf, nc = o.nuc;
  const double cut = std::pow(0.1, np + 1);  // MatMgnt3d::alt, fmm3d/matmgnt3d.cpp:38-41

  // the grids at this form's radius (R = 1 in the homogeneous form)
  auto scaled = [R](const std::vector<double>& v) {
    std::vector<double> s(v.size());
    for (size_t i = 0; i < v.size(); i++) s[i] = R * v[i];
    return s;
  };
  const std::vector<double> ueR = scaled(o.ue), ucR = scaled(o.uc), deR = scaled(o.de), dcR = scaled(o.dc);
  // UC2UE = pinv(K(UC <- UE)) (fmm3d/matmgnt3d.cpp:96-105)
  std::vector<double> ue2ucm((size_t)nc * td * ns * sd);
  kernel_matrix(mm, nc, ucR.data(), ns, ueR.data(), ueR.data(), ue2ucm.data());
  if (!pinv_factors(nc * td, ns * sd, ue2ucm.data(), cut, nthreads, &o.up_V, &o.up_W, &o.rank_up)) {
    if (err) *err = "UC2UE SVD did not converge";
    return nullptr;
  }
  // DC2DE = pinv(K(DC <- DE)) (fmm3d/matmgnt3d.cpp:163-172)
  std::vector<double> de2dcm((size_t)ns * td * ns * sd);
  kernel_matrix(mm, ns, dcR.data(), ns, deR.data(), deR.data(), de2dcm.data());
  if (!pinv_factors(ns * td, ns * sd, de2dcm.data(), cut, nthreads, &o.dn_V, &o.dn_W, &o.rank_dn)) {
    if (err) *err = "DC2DE SVD did not converge";
    return nullptr;
  }
  // M2M_o = UC2UE * UE2UC_o, UE2UC_o: UE shifted by (2*idx-1), UC scaled x2
  // (fmm3d/matmgnt3d.cpp:131-138).  With UC2UE = up_V * up_W the upward pass
  // runs on y = up_W * (check values): a parent's y is sum_o (up_W UE2UC_o up_V)
  // y_child_o; the child's 2^(-l deg) output and the parent's 2^(+l deg) input
  // scaling cancel exactly.  Same for L2L_o = DC2DE * DE2DC_o, DE2DC_o: DC
  // scaled x0.5 and shifted by (idx-0.5) (:199-203), on z = dn_W * (check values).
  const int K1 = ns * sd;
  const int ru = o.rank_up, rd = o.rank_dn;
  if (level < 0) {
    o.m2m_y.assign((size_t)ru * 8 * ru, 0.0);
    o.l2l_z.assign((size_t)8 * rd * rd, 0.0);
  } else {
    o.ue2uc_raw.assign((size_t)8 * nc * td * K1, 0.0);
    o.de2dc_raw.assign((size_t)8 * ns * td * K1, 0.0);
  }
  parallel_range(8, nthreads, [&](int oct) {
    int idx[3] = {(oct >> 2) & 1, (oct >> 1) & 1, oct & 1};
    std::vector<double> chk(o.uc.size()), den(o.ue.size());
    for (size_t i = 0; i < o.uc.size(); i++) chk[i] = 2.0 * R * o.uc[i];
    for (int j = 0; j < ns; j++)
      for (int d = 0; d < 3; d++) den[3 * j + d] = R * o.ue[3 * j + d] + (2 * idx[d] - 1) * R;
    std::vector<double> ue2uc((size_t)nc * td * K1);
    kernel_matrix(mm, nc, chk.data(), ns, den.data(), den.data(), ue2uc.data());
    std::vector<double> dchk(o.dc.size());
    for (int j = 0; j < ns; j++)
      for (int d = 0; d < 3; d++) dchk[3 * j + d] = 0.5 * R * o.dc[3 * j + d] + (double(idx[d]) - 0.5) * R;
    std::vector<double> de2dc((size_t)ns * td * K1);
    kernel_matrix(mm, ns, dchk.data(), ns, deR.data(), deR.data(), de2dc.data());
    if (level >= 0) {  // chained with the neighbouring levels by get_level_operators
      std::copy(ue2uc.begin(), ue2uc.end(), o.ue2uc_raw.begin() + (size_t)oct * nc * td * K1);
      std::copy(de2dc.begin(), de2dc.end(), o.de2dc_raw.begin() + (size_t)oct * ns * td * K1);
      return;
    }
    std::vector<double> qb((size_t)ru * K1), qy((size_t)ru * ru);
    matmul(ru, nc * td, K1, o.up_W.data(), ue2uc.data(), qb.data());
    matmul(ru, K1, ru, qb.data(), o.up_V.data(), qy.data());
    for (int r = 0; r < ru; r++)
      for (int c = 0; c < ru; c++) o.m2m_y[(size_t)r * 8 * ru + (size_t)oct * ru + c] = qy[(size_t)r * ru + c];
    std::vector<double> rb((size_t)rd * K1), rz((size_t)rd * rd);
    matmul(rd, ns * td, K1, o.dn_W.data(), de2dc.data(), rb.data());
    matmul(rd, K1, rd, rb.data(), o.dn_V.data(), rz.data());
    for (int r = 0; r < rd; r++)
      for (int c = 0; c < rd; c++) o.l2l_z[((size_t)oct * rd + r) * rd + c] = rz[(size_t)r * rd + c];
  });

  // M2L spectra (fmm3d/matmgnt3d.cpp:307-325): kernel sampled at
  // reg(g) - 2*idx with reg(g) = wrap(g)*step, wrap(g) = g < np ? g : g - n,
  // transformed with w = exp(-2 pi i / n); kx halved; scaled by 1/n^3.
  const int n = o.n, nh = o.nh;
  const double step = 2.0 / (np - 1);
  // Hermitian compaction: a real grid's half spectrum (kx < nh) repeats its
  // kx = 0 and kx = n/2 planes as X(kx,-ky,-kz) = conj X(kx,ky,kz); only the
  // canonical member of each pair, (kz,ky) <= (-kz,-ky) mod n, is kept.
  o.ff2c.assign(o.nfreq, 0);
  o.fc2f.clear();
  for (int kz = 0; kz < n; kz++)
    for (int ky = 0; ky < n; ky++)
      for (int kx = 0; kx < nh; kx++) {
        const int f = (kz * n + ky) * nh + kx;
        const int mz = (n - kz) % n, my = (n - ky) % n;
        const bool edge = kx == 0 || 2 * kx == n;
        if (!edge || kz < mz || (kz == mz && ky <= my)) {
          o.ff2c[f] = (int)o.fc2f.size();
          o.fc2f.push_back(f);
        }
      }
  o.nfc = (int)o.fc2f.size();
  for (int kz = 0; kz < n; kz++)
    for (int ky = 0; ky < n; ky++)
      for (int kx : {0, n / 2}) {
        const int f = (kz * n + ky) * nh + kx;
        const int mz = (n - kz) % n, my = (n - ky) % n;
        if (!(kz < mz || (kz == mz && ky <= my))) o.ff2c[f] = -o.ff2c[(mz * n + my) * nh + kx] - 1;
      }
  const int nfc = o.nfc;
  o.m2l.assign((size_t)343 * td * sd * nfc, std::complex<double>(0.0, 0.0));
  std::vector<std::complex<double>> w(n);
  for (int j = 0; j < n; j++) w[j] = std::polar(1.0, -2.0 * M_PI * j / n);
  const double scale = 1.0 / ((double)n * n * n);
  std::vector<int> offs;
  for (int dx = -3; dx <= 3; dx++)
    for (int dy = -3; dy <= 3; dy++)
      for (int dz = -3; dz <= 3; dz++)
        if (std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz))) > 1) offs.push_back(offset_index(dx, dy, dz));
  parallel_range((int)offs.size(), nthreads, [&](int oi) {
    int oidx = offs[oi];
    int dx = oidx / 49 - 3, dy = (oidx / 7) % 7 - 3, dz = oidx % 7 - 3;
    std::vector<double> kg((size_t)n * n * n * td * sd);
    double b[16];
    for (int gz = 0; gz < n; gz++)
      for (int gy = 0; gy < n; gy++)
        for (int gx = 0; gx < n; gx++) {
          // (at R = 2^-level in the per-level form, fmm3d/matmgnt3d.cpp:308-309)
          double x[3] = {R * ((gx < np ? gx : gx - n) * step - 2.0 * dx), R * ((gy < np ? gy : gy - n) * step - 2.0 * dy),
                         R * ((gz < np ? gz : gz - n) * step - 2.0 * dz)};
          block(mm, x, x, b);
          size_t g = ((size_t)gz * n + gy) * n + gx;
          for (int e = 0; e < td * sd; e++) kg[g * td * sd + e] = b[e];
        }
    std::vector<std::complex<double>> A((size_t)n * n * nh), B((size_t)n * n * nh);
    for (int e = 0; e < td * sd; e++) {
      // x pass: A[gz][gy][kx]
      for (int gz = 0; gz < n; gz++)
        for (int gy = 0; gy < n; gy++)
          for (int kx = 0; kx < nh; kx++) {
            std::complex<double> s(0, 0);
            for (int gx = 0; gx < n; gx++) s += kg[(((size_t)gz * n + gy) * n + gx) * td * sd + e] * w[(gx * kx) % n];
            A[((size_t)gz * n + gy) * nh + kx] = s;
          }
      // y pass: B[gz][ky][kx]
      for (int gz = 0; gz < n; gz++)
        for (int ky = 0; ky < n; ky++)
          for (int kx = 0; kx < nh; kx++) {
            std::complex<double> s(0, 0);
            for (int gy = 0; gy < n; gy++) s += A[((size_t)gz * n + gy) * nh + kx] * w[(gy * ky) % n];
            B[((size_t)gz * n + ky) * nh + kx] = s;
          }
      // z pass at the canonical frequencies, f = (kz*n + ky)*nh + kx
      std::complex<double>* dst = &o.m2l[((size_t)oidx * td * sd + e) * nfc];
      for (int c = 0; c < nfc; c++) {
        const int f = o.fc2f[c], kx = f % nh, ky = (f / nh) % n, kz = f / (nh * n);
        std::complex<double> s(0, 0);
        for (int gz = 0; gz < n; gz++) s += B[((size_t)gz * n + ky) * nh + kx] * w[(gz * kz) % n];
        dst[c] = s * scale;
      }
    }
  });
  return op;
}

}  // namespace

namespace {
std::shared_ptr<const Operators> cached_operators(const KernelDesc& mm, int np, int level, int nthreads,
                                                  std::string* err) {
  static std::mutex mu;
  static std::map<std::tuple<int, double, double, int, int>, std::shared_ptr<const Operators>> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_tuple(mm.kt, mm.coefs[0], mm.coefs[1], np, level);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  auto op = build_operators(mm, np, nthreads, err, level);
  if (!op) return nullptr;
  cache[key] = op;
  return op;
}
}  // namespace

std::shared_ptr<const Operators> get_operators(const KernelDesc& mm, int np, int nthreads, std::string* err) {
  return cached_operators(mm, np, -1, nthreads, err);
}

std::shared_ptr<const LevelOperators> get_level_operators(const KernelDesc& mm, int np, int lmin, int lmax,
                                                          int nthreads, std::string* err) {
  auto L = std::make_shared<LevelOperators>();
  L->lmin = lmin;
  L->lmax = lmax;
  for (int l = lmin; l <= lmax; l++) {
    auto o = cached_operators(mm, np, l, nthreads, err);
    if (!o) return nullptr;
    L->ops.push_back(o);
  }
  const int nl = lmax - lmin + 1;
  L->m2m_y.resize(nl);
  L->l2l_z.resize(nl);
  for (int i = 0; i + 1 < nl; i++) {
    const Operators& p = *L->ops[i];      // parent level
    const Operators& c = *L->ops[i + 1];  // child level
    const int K1 = p.nsurf * mm.sd, Kuc = p.nuc * mm.td, Kdc = p.nsurf * mm.td;
    const int rp = p.rank_up, rc = c.rank_up, dp = p.rank_dn, dc = c.rank_dn;
    L->m2m_y[i].assign((size_t)rp * 8 * rc, 0.0);
    L->l2l_z[i].assign((size_t)8 * dc * dp, 0.0);
    parallel_range(8, nthreads, [&](int oct) {
      std::vector<double> qb((size_t)rp * K1), qy((size_t)rp * rc);
      matmul(rp, Kuc, K1, p.up_W.data(), c.ue2uc_raw.data() + (size_t)oct * Kuc * K1, qb.data());
      matmul(rp, K1, rc, qb.data(), c.up_V.data(), qy.data());
      for (int r = 0; r < rp; r++)
        for (int k = 0; k < rc; k++) L->m2m_y[i][(size_t)r * 8 * rc + (size_t)oct * rc + k] = qy[(size_t)r * rc + k];
      std::vector<double> rb((size_t)dc * K1), rz((size_t)dc * dp);
      matmul(dc, Kdc, K1, c.dn_W.data(), p.de2dc_raw.data() + (size_t)oct * Kdc * K1, rb.data());
      matmul(dc, K1, dp, rb.data(), p.dn_V.data(), rz.data());
      for (int r = 0; r < dc; r++)
        for (int k = 0; k < dp; k++) L->l2l_z[i][((size_t)oct * dc + r) * dp + k] = rz[(size_t)r * dp + k];
    });
  }
  return L;
}

}  // namespace kifmm
