// FMM3d::setup / FMM3d::eval on one B200 (fmm3d/fmm3d_setup.cpp:26-140,
// fmm3d/fmm3d_eval.cpp:24-243).  Host code: builds the tree and operators,
// lays the per-level work lists and node data out in HBM once, and then
// enqueues the evaluation passes on one stream:
//
//   load      scatter densities into leaf (Morton) order        eval.cpp:50-64
//   upward    S2M P2P; per level bottom-up: UC2UE on leaves,
//             fused M2M (UC2UE*UE2UC) on parents               eval.cpp:69-92
//   V list    forward spectra, Hadamard accumulate, inverse    eval.cpp:115-150
//   X list    S2L P2P to downward check surfaces               eval.cpp:176-191
//   downward  per level top-down: DC2DE, fused L2L              eval.cpp:195-209
//   leaves    U + W + X direct + M2T + L2T in one P2P pass     eval.cpp:98-111,154-172,210-213
//   save      gather potentials back to the caller's order     eval.cpp:221-235
#include "engine.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <thread>
#include <tuple>

#include "../../include/kifmm.h"
#include "launch.hpp"

namespace kifmm {

namespace {

int host_threads() {
  unsigned n = std::thread::hardware_concurrency();
  return n ? (int)std::min(n, 64u) : 4;
}

struct CudaError {
  cudaError_t e;
  const char* where;
};

#define KCHECK(call)                                      \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) throw CudaError{_e, #call};    \
  } while (0)

// The FP16 operator images of the tensor-core Hadamard on one device, shared
// by every engine whose translation operators are the same object (the
// operator cache hands one object per kernel and np to every engine): the
// images of a multi-dof kernel reach hundreds of MB (Stokes np=6: 217 chunks
// x 26 directions x 12 dof pairs x 4 KB), so instances of a batch keep one
// copy.  Freed with the last engine that holds them.
struct Tc16Images {
  unsigned short* img = nullptr;
  float* inv_sb = nullptr;
  int device = 0;
  ~Tc16Images() {
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    if (img) cudaFree(img);
    if (inv_sb) cudaFree(inv_sb);
    if (cur != device) cudaSetDevice(cur);
  }
};

std::shared_ptr<Tc16Images> tc16_images(const std::shared_ptr<const Operators>& ops, int device, int nf, int sd,
                                        int td) {
  static std::mutex mu;
  static std::map<std::pair<const Operators*, int>, std::pair<std::weak_ptr<const Operators>, std::weak_ptr<Tc16Images>>>
      cache;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_pair(ops.get(), device);
  auto it = cache.find(key);
  if (it != cache.end() && !it->second.first.expired())
    if (auto p = it->second.second.lock()) return p;
  std::vector<unsigned short> im;
  std::vector<float> isb;
  m2l_tc16_images(nf, sd, td, ops->m2l.data(), &im, &isb);
  auto p = std::make_shared<Tc16Images>();
  p->device = device;
  KCHECK(cudaMalloc(&p->img, im.size() * sizeof(unsigned short)));
  KCHECK(cudaMemcpy(p->img, im.data(), im.size() * sizeof(unsigned short), cudaMemcpyHostToDevice));
  KCHECK(cudaMalloc(&p->inv_sb, isb.size() * sizeof(float)));
  KCHECK(cudaMemcpy(p->inv_sb, isb.data(), isb.size() * sizeof(float), cudaMemcpyHostToDevice));
  cache[key] = std::make_pair(std::weak_ptr<const Operators>(ops), std::weak_ptr<Tc16Images>(p));
  return p;
}

}  // namespace

template <typename T>
struct Impl : ImplBase {
  Engine& E;
  const Tree& tr;
  const Operators& op;
  std::vector<void*> allocs;

  template <class U>
  U* dalloc(size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    KCHECK(cudaMalloc(&p, n * sizeof(U)));
    allocs.push_back(p);
    return (U*)p;
  }
  template <class U>
  U* upload(const std::vector<U>& v) {
    U* p = dalloc<U>(v.size());
    if (!v.empty()) KCHECK(cudaMemcpy(p, v.data(), v.size() * sizeof(U), cudaMemcpyHostToDevice));
    return p;
  }
  template <class U>
  T* upload_as_T(const std::vector<U>& v) {
    std::vector<T> t(v.size());
    for (size_t i = 0; i < v.size(); i++) t[i] = (T)v[i];
    return upload(t);
  }

  struct List {
    int* work = nullptr;   // column / CTA node ids
    int* aux = nullptr;    // second index list (GEMM B or C ids)
    int n = 0;
    int64_t* ptr = nullptr;
    int* idx = nullptr;
    int64_t* ptr2 = nullptr;
    int* idx2 = nullptr;
    // GEMM column lists over R density vectors: the node lists repeated
    // with offsets r * nnodes into the [r][node][...] buffers (aux offset
    // too when it holds node ids, copied when it holds levels)
    std::vector<int> hw, ha;
    bool aux_nodes = false;
    int R = 0;
    int *rw = nullptr, *ra = nullptr;
  };

  int sd_u, td_u, sd_m, td_m, nsurf, nuc;
  P2PArgs<T> args;
  // Double-layer kernels in mixed precision: the U-list sums in FP64.  For
  // two sources closer than their leaf's size the double-layer factor r.n is
  // O(|r|^2) and comes out of the FP32 coordinates with an error of the
  // leaf size times 2^-24, which near-coincident pairs turn into a relative
  // error of order one in their term (0.27 at 262,144 points on the
  // (1, .5, .25) ellipsoid, kernel 321).  FP64 coordinates relative to the
  // leaf centre hold it to 2^-53; every other pass keeps the
  // well-separated, FP32-safe evaluations.
  bool near64 = false;
  P2PArgs<double> a64;
  List near_u;
  double *sden64 = nullptr, *tval64 = nullptr;
  M2LGeom geom;
  GemmScale scl;
  // device buffers
  int *d_sperm = nullptr, *d_tperm = nullptr, *d_path = nullptr, *d_depth = nullptr;
  T *sden = nullptr, *tval = nullptr;
  int cap_rhs = 0;
  T *supeden = nullptr, *supcval = nullptr, *tdncval = nullptr, *tdneden = nullptr, *spectra = nullptr,
    *effval = nullptr;
  // A surface operator: row-major M x K in T (SIMT path) and, for FP32 data,
  // the split-TF32 pair for the tensor-core path.
  struct SurfOp {
    const T* a = nullptr;
    TcOperator tc;
    int M = 0, K = 0;
  };
  SurfOp op_upW, op_upV, op_m2my, op_dnW, op_dnV, op_l2lz;  // factored surface operators
  // per-level operators (E.per_level), by depth: the factors of each level and
  // the chains from depth d to d + 1; per-level ranges of the level-ordered
  // lists (s2m, up_all, dn_all, the V-list parents), and the sweep's operator
  // tiles per level
  struct LevelOps {
    SurfOp upW, upV, m2my, dnW, dnV, l2lz;
  };
  std::vector<LevelOps> lv;
  std::vector<int> off_s2m, off_up, off_dn, off_pairs;
  std::vector<T*> ktiles_lv;
  T *ybuf, *zbuf;  // per-node rank-space coordinates of the upward / downward densities
  int ru = 0, rd = 0;  // ranks rounded up to multiples of 8 (zero-padded rows / columns)
  bool use_tc = false;
  T* khat;
  T* ktiles = nullptr;  // [td][sd][ceil(nf/32)][343][32] operator spectra for the parent-pair sweep
  T* ttiles = nullptr;  // [td][sd][ceil(nf/16)][26][27][16] Toeplitz-factored operator
  float* htc_img = nullptr;         // tensor-core Hadamard (split TF32): operator images per (4 frequencies, direction)
  unsigned short* htc16_img = nullptr;  // tensor-core Hadamard (FP16 pairs): the same images, [chunk][dir][td][sd]
  std::shared_ptr<Tc16Images> htc16_shared;  // ... held from the per-device cache
  float* htc16_inv_sb = nullptr;        // ... and the inverse of each chunk's operator scale
  unsigned* d_bound = nullptr;          // ... and the per-eval bound of the spectra (FP32 bits)
  int* htc16_ctab = nullptr;            // ... and its colleague tables [tile][26][128]
  bool htc() const { return htc_img || htc16_img; }
  unsigned* htc_dirs = nullptr;     // tensor-core Hadamard: directions present per tile of 128 parents
  int* h_status = nullptr;  // mapped host word: device-side wait time-outs (bit 0 sweep, bit 1 GEMM, bit 2 TC Hadamard)
  int* d_status = nullptr;
  List s2m, s2l, leaf, m2l, fwd;
  std::vector<List> up_non, dn_par;
  List up_all, dn_all;
  double* gemm_ws = nullptr;
  size_t gemm_ws_len = 0;
  cudaEvent_t ev[9];  // phase boundaries + the two interior V-list kernel boundaries
  bool have_events = false;
  int nlaunch = 0;
  double pt[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};

  Impl(Engine& e) : E(e), tr(e.tree), op(*e.ops) {}
  ~Impl() override {
    for (void* p : allocs) cudaFree(p);
    if (h_status) cudaFreeHost(h_status);
    if (have_events)
      for (auto& x : ev) cudaEventDestroy(x);
  }

  void build() {
    sd_u = E.user.sd;
    td_u = E.user.td;
    sd_m = E.mm.sd;
    td_m = E.mm.td;
    nsurf = op.nsurf;
    nuc = op.nuc;
    const int nn = tr.nnodes;
    // ---- node arrays
    std::vector<int> chd = tr.chd;
    args.nnodes = nn;
    args.ns = E.ns;
    args.nt = E.nt;
    args.nsurf = nsurf;
    args.nuc = nuc;
    args.sbeg = upload(tr.sbeg);
    args.scnt = upload(tr.scnt);
    args.tbeg = upload(tr.tbeg);
    args.tcnt = upload(tr.tcnt);
    d_depth = upload(tr.depth);
    args.depth = d_depth;
    d_path = upload(tr.path);
    args.center = upload(tr.center);
    args.radius = upload(tr.radius);
    d_sperm = upload(tr.sperm);
    d_tperm = upload(tr.tperm);
    // ---- points: coordinates relative to their leaf centre
    std::vector<double> sl[6], tl[3];
    for (auto& v : sl) v.assign(E.ns, 0.0);
    for (auto& v : tl) v.assign(E.nt, 0.0);
    for (int g = 0; g < nn; g++) {
      if (!tr.terminal(g)) continue;
      const double* c = &tr.center[3 * g];
      for (int i = tr.sbeg[g]; i < tr.sbeg[g] + tr.scnt[g]; i++) {
        int p = tr.sperm[i];
        for (int d = 0; d < 3; d++) {
          sl[d][i] = E.srcpos[3 * (size_t)p + d] - c[d];
          sl[3 + d][i] = E.srcnor[3 * (size_t)p + d];
        }
      }
      for (int i = tr.tbeg[g]; i < tr.tbeg[g] + tr.tcnt[g]; i++) {
        int p = tr.tperm[i];
        for (int d = 0; d < 3; d++) tl[d][i] = E.trgpos[3 * (size_t)p + d] - c[d];
      }
    }
    args.sx = upload_as_T(sl[0]);
    args.sy = upload_as_T(sl[1]);
    args.sz = upload_as_T(sl[2]);
    if (E.user.dl) {
      args.snx = upload_as_T(sl[3]);
      args.sny = upload_as_T(sl[4]);
      args.snz = upload_as_T(sl[5]);
    }
    args.tx = upload_as_T(tl[0]);
    args.ty = upload_as_T(tl[1]);
    args.tz = upload_as_T(tl[2]);
    near64 = sizeof(T) == 4 && E.user.dl;
    if (near64) {
      a64.nnodes = nn;
      a64.ns = E.ns;
      a64.nt = E.nt;
      a64.nsurf = nsurf;
      a64.nuc = nuc;
      a64.sbeg = args.sbeg;
      a64.scnt = args.scnt;
      a64.tbeg = args.tbeg;
      a64.tcnt = args.tcnt;
      a64.depth = args.depth;
      a64.center = args.center;
      a64.radius = args.radius;
      a64.sx = upload(sl[0]);
      a64.sy = upload(sl[1]);
      a64.sz = upload(sl[2]);
      a64.snx = upload(sl[3]);
      a64.sny = upload(sl[4]);
      a64.snz = upload(sl[5]);
      a64.tx = upload(tl[0]);
      a64.ty = upload(tl[1]);
      a64.tz = upload(tl[2]);
      a64.l2t_depth = 1 << 30;  // near field only
    }
    // ---- surfaces and operators
    args.ue_unit = upload_as_T(op.ue);
    args.uc_unit = upload_as_T(op.uc);
    args.de_unit = upload_as_T(op.de);
    args.dc_unit = upload_as_T(op.dc);
    build_surface_ops();
    {
      std::vector<T> kh(op.m2l.size() * 2);
      for (size_t i = 0; i < op.m2l.size(); i++) {
        kh[2 * i] = (T)op.m2l[i].real();
        kh[2 * i + 1] = (T)op.m2l[i].imag();
      }
      khat = upload(kh);
      if (m2l_sweep_supported(op.nfc, sd_m, td_m)) {
        // [td][sd][ftile][343][32]; the spectra are [343][td][sd][nf]
        const int nf = op.nfc, ftiles = (nf + 31) / 32, tsd = td_m * sd_m;
        std::vector<T> kt((size_t)tsd * ftiles * 343 * 32 * 2, T(0));
        for (int ts = 0; ts < tsd; ts++)
          for (int ft = 0; ft < ftiles; ft++)
            for (int o = 0; o < 343; o++)
              for (int l = 0; l < 32 && ft * 32 + l < nf; l++) {
                const size_t dst = ((((size_t)ts * ftiles + ft) * 343 + o) * 32 + l) * 2;
                const size_t src = (((size_t)o * tsd + ts) * nf + ft * 32 + l) * 2;
                kt[dst] = kh[src];
                kt[dst + 1] = kh[src + 1];
              }
        if (sizeof(T) == 4 && E.m2l_tc && !E.m2l_tc_tf32 && m2l_tc16_supported(nf, sd_m, td_m)) {
          htc16_shared = tc16_images(E.ops, E.device, nf, sd_m, td_m);
          htc16_img = htc16_shared->img;
          htc16_inv_sb = htc16_shared->inv_sb;
        } else if (sizeof(T) == 4 && E.m2l_tc && m2l_tc_supported(nf, sd_m, td_m)) {
          std::vector<float> im;
          m2l_tc_images(nf, op.m2l.data(), &im);
          htc_img = upload(im);
        } else if (E.m2l_toeplitz) {
          ttiles = upload(toeplitz_tables());
        } else if (E.per_level) {  // one set of operator tiles per level
          for (auto& lo : E.lops->ops) ktiles_lv.push_back(upload(sweep_tiles(*lo)));
          ktiles = ktiles_lv[0];
        } else {
          ktiles = upload(kt);
        }
      }
    }
    KCHECK(cudaHostAlloc((void**)&h_status, sizeof(int), cudaHostAllocMapped));
    *h_status = 0;
    KCHECK(cudaHostGetDevicePointer((void**)&d_status, h_status, 0));
    double kc[3];
    kernel_constants(E.user.kt, E.user.coefs, kc);
    args.ku = KConst<T>{(T)kc[0], (T)kc[1], (T)kc[2]};
    if (near64) a64.ku = KConst<double>{kc[0], kc[1], kc[2]};
    kernel_constants(E.mm.kt, E.mm.coefs, kc);
    args.km = KConst<T>{(T)kc[0], (T)kc[1], (T)kc[2]};
    if (near64) a64.km = KConst<double>{kc[0], kc[1], kc[2]};
    // ---- per-node data: allocated per chunk of density vectors (ensure_chunk)
    S_supe = (size_t)nn * nsurf * sd_m;
    S_supc = (size_t)nn * nuc * td_m;
    S_tdnc = (size_t)nn * nsurf * td_m;
    S_tdne = (size_t)nn * nsurf * sd_m;
    S_y = (size_t)nn * ru;
    S_z = (size_t)nn * rd;

    // ---- work lists
    const int md = tr.maxdepth;
    up_non.resize(md + 1);
    dn_par.resize(md + 1);
    std::vector<int> v_s2m;
    for (int d = 2; d <= md; d++) {
      std::vector<int> un, unc, dp, dpc;
      for (int g = tr.level_beg[d]; g < tr.level_beg[d + 1]; g++) {
        if (!(tr.tag[g] & TAG_SRC)) continue;
        if (tr.terminal(g)) {
          v_s2m.push_back(g);
        } else {
          un.push_back(g);
          unc.push_back(tr.chd[g]);
        }
      }
      if (d >= 3)
        for (int g = tr.level_beg[d - 1]; g < tr.level_beg[d]; g++)
          if ((tr.tag[g] & TAG_TRG) && !tr.terminal(g)) {
            dp.push_back(g);
            dpc.push_back(tr.chd[g]);
          }
      up_non[d] = make_list(un, unc);
      dn_par[d] = make_list(dp, dpc);
      up_non[d].hw = un;
      up_non[d].ha = unc;
      up_non[d].aux_nodes = true;
      dn_par[d].hw = dp;
      dn_par[d].ha = dpc;
      dn_par[d].aux_nodes = true;
    }
    {
      // all-level lists (aux = node depth): source leaves, every upward node,
      // every downward node
      std::vector<int> s2m_lvl, all_up, all_up_lvl, all_dn, all_dn_lvl;
      for (int g : v_s2m) s2m_lvl.push_back(tr.depth[g]);
      for (int d = 2; d <= md; d++)
        for (int g = tr.level_beg[d]; g < tr.level_beg[d + 1]; g++)
          if (tr.tag[g] & TAG_SRC) {
            all_up.push_back(g);
            all_up_lvl.push_back(d);
          }
      for (int d = 2; d <= md; d++)
        for (int g = tr.level_beg[d]; g < tr.level_beg[d + 1]; g++)
          if (tr.tag[g] & TAG_TRG) {
            all_dn.push_back(g);
            all_dn_lvl.push_back(d);
          }
      s2m = make_list(v_s2m, s2m_lvl);
      up_all = make_list(all_up, all_up_lvl);
      dn_all = make_list(all_dn, all_dn_lvl);
      s2m.hw = v_s2m;
      s2m.ha = s2m_lvl;
      up_all.hw = all_up;
      up_all.ha = all_up_lvl;
      dn_all.hw = all_dn;
      dn_all.ha = all_dn_lvl;
      if (E.per_level) {
        off_s2m = level_offsets(s2m_lvl, md);
        off_up = level_offsets(all_up_lvl, md);
        off_dn = level_offsets(all_dn_lvl, md);
      }
      KCHECK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, E.device));
      gemm_ws_len = (size_t)4 << 20;  // split-K slices of the shallow levels (32 MB)
      gemm_ws = dalloc<double>(gemm_ws_len);
    }
    // V list (M2L), forward set
    {
      std::vector<int> work, fwdn;
      std::vector<int64_t> ptr{0};
      std::vector<int> idx;
      std::vector<char> mark(nn, 0);
      const Csr& V = tr.lists[1];
      for (int g = 0; g < nn; g++) {
        int64_t b = V.ptr[g], e = V.ptr[g + 1];
        if (e == b) continue;
        if (e - b > 192) throw CudaError{cudaErrorInvalidValue, "V list longer than 189"};
        work.push_back(g);
        for (int64_t k = b; k < e; k++) {
          idx.push_back(V.idx[k]);
          mark[V.idx[k]] = 1;
        }
        ptr.push_back((int64_t)idx.size());
      }
      for (int g = 0; g < nn; g++)
        if (mark[g]) fwdn.push_back(g);
      m2l = make_list(work, {}, ptr, idx);
      fwd = make_list(fwdn, {});
      S_eff = (size_t)((nn + 15) / 8 * 8) * td_m * op.nfc * 2;  // room for the sibling-group layout
      // nn + 8 blocks: nodes outside every V list keep a zero spectrum, and the
      // 8 blocks from index nn on stand for an absent colleague (parent-pair form)
      // (tensor-core form: sibling-group major, node n in group (n + 7) / 8,
      // the zero block a group of its own: (nn + 15) / 8 groups of 8 nodes)
      // (FP16 form, several source dofs: one such plane per dof)
      S_spec = std::max((size_t)(nn + 8) * sd_m, htc() ? (size_t)(nn + 15) / 8 * 8 * (htc16_img ? sd_m : 1) : 0) *
               op.nfc * 2;
      counters_v = (double)idx.size();
      if (ktiles || ttiles || htc()) build_pairs(work);
      counters_fwd = (double)fwdn.size();
      counters_inv = (double)work.size();
    }
    // X list (S2L when not direct), leaf work (U + direct W/X; M2T W)
    {
      std::vector<int> xw, lw;
      std::vector<int64_t> xptr{0}, nptr{0}, mptr{0}, uptr{0};
      std::vector<int> xidx, nidx, midx, uidx;
      const Csr& U = tr.lists[0];
      const Csr& W = tr.lists[2];
      const Csr& X = tr.lists[3];
      double near_int = 0, surf_int = 0;
      for (int g = 0; g < nn; g++) {
        if (!(tr.tag[g] & TAG_TRG)) continue;
        bool term = tr.terminal(g);
        bool x_direct = term && (int64_t)tr.tcnt[g] * td_u < (int64_t)nsurf * td_m;  // fmm3d_eval.cpp:183
        if (X.ptr[g + 1] > X.ptr[g] && !x_direct) {
          xw.push_back(g);
          for (int64_t k = X.ptr[g]; k < X.ptr[g + 1]; k++) {
            xidx.push_back(X.idx[k]);
            surf_int += (double)nsurf * tr.scnt[X.idx[k]];
          }
          xptr.push_back((int64_t)xidx.size());
        }
        if (!term) continue;
        lw.push_back(g);
        for (int64_t k = U.ptr[g]; k < U.ptr[g + 1]; k++) {
          (near64 ? uidx : nidx).push_back(U.idx[k]);
          near_int += (double)tr.tcnt[g] * tr.scnt[U.idx[k]] * (near64 ? 1 : 0);
        }
        uptr.push_back((int64_t)uidx.size());
        for (int64_t k = W.ptr[g]; k < W.ptr[g + 1]; k++) {
          int w = W.idx[k];
          bool w_direct = tr.terminal(w) && (int64_t)tr.scnt[w] * sd_u < (int64_t)nsurf * sd_m;  // :161
          if (w_direct)
            nidx.push_back(w);
          else
            midx.push_back(w);
        }
        if (x_direct)
          for (int64_t k = X.ptr[g]; k < X.ptr[g + 1]; k++) nidx.push_back(X.idx[k]);
        for (int64_t k = nptr.back(); k < (int64_t)nidx.size(); k++) near_int += (double)tr.tcnt[g] * tr.scnt[nidx[k]];
        surf_int += (double)tr.tcnt[g] * nsurf * ((int64_t)midx.size() - mptr.back() + (tr.depth[g] >= 2 ? 1 : 0));
        nptr.push_back((int64_t)nidx.size());
        mptr.push_back((int64_t)midx.size());
      }
      s2l = make_list(xw, {}, xptr, xidx);
      leaf = make_list(lw, {}, nptr, nidx, mptr, midx);
      if (near64) near_u = make_list(lw, {}, uptr, uidx, std::vector<int64_t>(lw.size() + 1, 0), {});
      for (int g : v_s2m) surf_int += (double)nuc * tr.scnt[g];
      counters_near = near_int;
      counters_surf = surf_int;
    }
    // ---- M2L geometry
    geom.np = op.np;
    geom.n = op.n;
    geom.nh = op.nh;
    geom.nfreq = op.nfreq;
    geom.nfc = op.nfc;
    geom.fc2f = upload(op.fc2f);
    geom.ff2c = upload(op.ff2c);
    geom.nsurf = nsurf;
    geom.surf_ijk = upload(op.surf_ijk);
    geom.sd = sd_m;
    geom.td = td_m;
    for (int s = 0; s < sd_m && s < 4; s++) geom.deg[s] = E.per_level ? 0 : op.deg[s];
    geom.rootlvl = E.rootlvl;
    geom.sg = htc16_img ? 2 : htc_img ? 1 : 0;
    geom.effval_sg = htc16_img ? 1 : 0;
    geom.plane = htc16_img ? (size_t)((nn + 15) / 8 * 8) * op.nfc : 0;
    geom.bound = d_bound;
    scl.sd = sd_m;
    for (int s = 0; s < sd_m && s < 4; s++) scl.deg[s] = E.per_level ? 0 : op.deg[s];
    // GEMM flops per eval
    double gf = 2.0 * ru * (nuc * td_m) * s2m.n + 2.0 * (nsurf * sd_m) * ru * up_all.n +
                2.0 * rd * (nsurf * td_m) * dn_all.n + 2.0 * (nsurf * sd_m) * rd * dn_all.n;
    for (int d = 2; d <= md; d++) {
      gf += 2.0 * ru * (8.0 * ru) * up_non[d].n;
      gf += 2.0 * (8.0 * rd) * rd * dn_par[d].n;
    }
    counters_gemm = gf;
    for (auto& x : ev) KCHECK(cudaEventCreate(&x));
    have_events = true;
    // density vectors per pass: as many as fit 8 GB of per-vector node data,
    // at most 8 (the spectra are one set, reused vector by vector)
    const double per_rhs = (double)sizeof(T) * (S_supe + S_supc + S_tdnc + S_tdne + S_y + S_z);
    max_chunk = (int)std::max(1.0, std::min(8.0, std::floor(8e9 / std::max(per_rhs, 1.0))));
    if (E.per_level) max_chunk = 1;  // the per-level passes run on the single-vector lists
    ensure_rhs(1);
  }

  SurfOp make_op(const std::vector<double>& A, int M, int K) {
    SurfOp o;
    o.M = M;
    o.K = K;
    o.a = upload_as_T(A);
    if constexpr (sizeof(T) == 4) {
      if (use_tc && M % 4 == 0 && K % 4 == 0) {
        std::vector<float> img;
        tc_operator_images(M, K, A.data(), &img, &o.tc);
        o.tc.img = upload(img);
      }
    }
    return o;
  }

  // The factored operators with both ranks rounded up to multiples of 8, so
  // that every rank-space vector starts on a 32-byte boundary; the padding
  // rows and columns are zero, and so are the padded coordinates.
  // zero-padded copy of a row-major r0 x c0 block into R x C
  static std::vector<double> padded(const std::vector<double>& a, int r0, int c0, int R, int C) {
    std::vector<double> o((size_t)R * C, 0.0);
    for (int r = 0; r < r0; r++)
      for (int c = 0; c < c0; c++) o[(size_t)r * C + c] = a[(size_t)r * c0 + c];
    return o;
  }

  // per-level form: every level's factors and chains padded to the largest
  // ranks over the levels
  void build_level_ops() {
    const LevelOperators& L = *E.lops;
    const int nl = (int)L.ops.size();
    int mu = 0, md_ = 0;
    for (auto& o : L.ops) {
      mu = std::max(mu, o->rank_up);
      md_ = std::max(md_, o->rank_dn);
    }
    ru = (mu + 7) / 8 * 8;
    rd = (md_ + 7) / 8 * 8;
    const int K1 = nsurf * sd_m, Kuc = nuc * td_m, Kdc = nsurf * td_m;
    use_tc = sizeof(T) == 4 && E.tensor_cores && K1 % 4 == 0 && Kuc % 4 == 0 && Kdc % 4 == 0;
    lv.resize(nl);
    for (int d = 0; d < nl; d++) {
      const Operators& o = *L.ops[d];
      lv[d].upW = make_op(padded(o.up_W, o.rank_up, Kuc, ru, Kuc), ru, Kuc);
      lv[d].upV = make_op(padded(o.up_V, K1, o.rank_up, K1, ru), K1, ru);
      lv[d].dnW = make_op(padded(o.dn_W, o.rank_dn, Kdc, rd, Kdc), rd, Kdc);
      lv[d].dnV = make_op(padded(o.dn_V, K1, o.rank_dn, K1, rd), K1, rd);
      if (d + 1 < nl) {
        const int rc = L.ops[d + 1]->rank_up, dc = L.ops[d + 1]->rank_dn;
        std::vector<double> m2my((size_t)ru * 8 * ru, 0.0), l2lz((size_t)8 * rd * rd, 0.0);
        for (int r = 0; r < o.rank_up; r++)
          for (int b = 0; b < 8; b++)
            for (int c = 0; c < rc; c++)
              m2my[(size_t)r * 8 * ru + (size_t)b * ru + c] = L.m2m_y[d][(size_t)r * 8 * rc + (size_t)b * rc + c];
        for (int b = 0; b < 8; b++)
          for (int r = 0; r < dc; r++)
            for (int c = 0; c < o.rank_dn; c++)
              l2lz[((size_t)b * rd + r) * rd + c] = L.l2l_z[d][((size_t)b * dc + r) * o.rank_dn + c];
        lv[d].m2my = make_op(m2my, ru, 8 * ru);
        lv[d].l2lz = make_op(l2lz, 8 * rd, rd);
      }
    }
  }

  void build_surface_ops() {
    if (E.per_level) {
      build_level_ops();
      return;
    }
    const int r0u = op.rank_up, r0d = op.rank_dn;
    ru = (r0u + 7) / 8 * 8;
    rd = (r0d + 7) / 8 * 8;
    const int K1 = nsurf * sd_m, Kuc = nuc * td_m, Kdc = nsurf * td_m;
    use_tc = sizeof(T) == 4 && E.tensor_cores && K1 % 4 == 0 && Kuc % 4 == 0 && Kdc % 4 == 0;
    std::vector<double> upW((size_t)ru * Kuc, 0.0), upV((size_t)K1 * ru, 0.0), m2my((size_t)ru * 8 * ru, 0.0);
    std::vector<double> dnW((size_t)rd * Kdc, 0.0), dnV((size_t)K1 * rd, 0.0), l2lz((size_t)8 * rd * rd, 0.0);
    for (int r = 0; r < r0u; r++)
      for (int k = 0; k < Kuc; k++) upW[(size_t)r * Kuc + k] = op.up_W[(size_t)r * Kuc + k];
    for (int i = 0; i < K1; i++)
      for (int r = 0; r < r0u; r++) upV[(size_t)i * ru + r] = op.up_V[(size_t)i * r0u + r];
    for (int r = 0; r < r0u; r++)
      for (int o = 0; o < 8; o++)
        for (int c = 0; c < r0u; c++)
          m2my[(size_t)r * 8 * ru + (size_t)o * ru + c] = op.m2m_y[(size_t)r * 8 * r0u + (size_t)o * r0u + c];
    for (int r = 0; r < r0d; r++)
      for (int k = 0; k < Kdc; k++) dnW[(size_t)r * Kdc + k] = op.dn_W[(size_t)r * Kdc + k];
    for (int i = 0; i < K1; i++)
      for (int r = 0; r < r0d; r++) dnV[(size_t)i * rd + r] = op.dn_V[(size_t)i * r0d + r];
    for (int o = 0; o < 8; o++)
      for (int r = 0; r < r0d; r++)
        for (int c = 0; c < r0d; c++)
          l2lz[((size_t)o * rd + r) * rd + c] = op.l2l_z[((size_t)o * r0d + r) * r0d + c];
    op_upW = make_op(upW, ru, Kuc);
    op_upV = make_op(upV, K1, ru);
    op_m2my = make_op(m2my, ru, 8 * ru);
    op_dnW = make_op(dnW, rd, Kdc);
    op_dnV = make_op(dnV, K1, rd);
    op_l2lz = make_op(l2lz, 8 * rd, rd);
  }

  // operator tiles of the parent-pair sweep, [td][sd][ftile][343][32] complex
  // (the spectra are [343][td][sd][nf])
  std::vector<T> sweep_tiles(const Operators& o) const {
    const int nf = o.nfc, ftiles = (nf + 31) / 32, tsd = td_m * sd_m;
    std::vector<T> kt((size_t)tsd * ftiles * 343 * 32 * 2, T(0));
    for (int ts = 0; ts < tsd; ts++)
      for (int ft = 0; ft < ftiles; ft++)
        for (int oo = 0; oo < 343; oo++)
          for (int l = 0; l < 32 && ft * 32 + l < nf; l++) {
            const size_t dst = ((((size_t)ts * ftiles + ft) * 343 + oo) * 32 + l) * 2;
            const std::complex<double> v = o.m2l[((size_t)oo * tsd + ts) * nf + ft * 32 + l];
            kt[dst] = (T)v.real();
            kt[dst + 1] = (T)v.imag();
          }
    return kt;
  }

  // first index of each depth (and one past the last) in a depth-ordered list
  static std::vector<int> level_offsets(const std::vector<int>& lvl, int md) {
    std::vector<int> off(md + 2, 0);
    for (int d = 0; d <= md + 1; d++)
      off[d] = (int)(std::lower_bound(lvl.begin(), lvl.end(), d) - lvl.begin());
    return off;
  }

  // Transformed operator of the Toeplitz-factored Hadamard: for direction d
  // (components d = (dd/9-1, dd/3%3-1, dd%3-1), dd skipping the centre) and
  // k = (kx, ky, kz) in {A, B, C}^3, T_k = sum over delta in {-1,0,1}^3 of
  // c_kx(dx) c_ky(dy) c_kz(dz) K(2d + delta), with c_A = [delta = 0],
  // c_B = [delta = 1] - [delta = 0], c_C = [delta = -1] - [delta = 0];
  // in FP64 from the operator spectra, rounded once.
  std::vector<T> toeplitz_tables() const {
    const int nf = op.nfc, ft16 = (nf + 15) / 16, tsd = td_m * sd_m;
    std::vector<T> out((size_t)tsd * ft16 * 26 * 28 * 16 * 2, T(0));  // [ts][tile][dir][k/2][16][k%2]
    auto coef = [](int k, int d) -> double {
      if (k == 0) return d == 0 ? 1.0 : 0.0;
      if (k == 1) return (d == 1 ? 1.0 : 0.0) - (d == 0 ? 1.0 : 0.0);
      return (d == -1 ? 1.0 : 0.0) - (d == 0 ? 1.0 : 0.0);
    };
    for (int dir = 0; dir < 26; dir++) {
      const int dd = dir < 13 ? dir : dir + 1;
      const int dv[3] = {dd / 9 - 1, (dd / 3) % 3 - 1, dd % 3 - 1};
      for (int k = 0; k < 27; k++) {
        const int kx = k / 9, ky = (k / 3) % 3, kz = k % 3;
        for (int ts = 0; ts < tsd; ts++)
          for (int f = 0; f < nf; f++) {
            std::complex<double> acc(0.0, 0.0);
            for (int ex = -1; ex <= 1; ex++)
              for (int ey = -1; ey <= 1; ey++)
                for (int ez = -1; ez <= 1; ez++) {
                  const double c = coef(kx, ex) * coef(ky, ey) * coef(kz, ez);
                  if (c == 0.0) continue;
                  const int o = offset_index(2 * dv[0] + ex, 2 * dv[1] + ey, 2 * dv[2] + ez);
                  acc += c * op.m2l[((size_t)o * tsd + ts) * nf + f];
                }
            const size_t dst = ((((((size_t)ts * ft16 + f / 16) * 26 + dir) * 14 + k / 2) * 16 + f % 16) * 2 + k % 2) * 2;
            out[dst] = (T)acc.real();
            out[dst + 1] = (T)acc.imag();
          }
      }
    }
    return out;
  }

  // Parent-pair form of the V list (single-dof equivalent kernels): one work
  // item per target parent Q with its 26 colleague parents' first-child ids.
  int pairs_n = 0, num_sms = 148;
  int *pairs_chd = nullptr, *pairs_coll = nullptr;
  unsigned char* pairs_mask = nullptr;

  void build_pairs(const std::vector<int>& vtargets) {
    const Csr& V = tr.lists[1];
    KCHECK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, E.device));
    // one work item per target parent of a node with a V list
    std::vector<int> qlist;
    std::vector<char> seen(tr.nnodes, 0);
    for (int t : vtargets) {
      int q = tr.par[t];
      if (!seen[q]) {
        seen[q] = 1;
        qlist.push_back(q);
      }
    }
    std::sort(qlist.begin(), qlist.end());
    if (E.per_level) {  // parents by depth (node ids are breadth first)
      std::vector<int> ql;
      for (int q : qlist) ql.push_back(tr.depth[q]);
      off_pairs = level_offsets(ql, tr.maxdepth);
    }
    std::vector<int> qchd, coll(qlist.size() * 26, tr.nnodes);  // absent: the zero block
    std::vector<unsigned char> mask(qlist.size(), 0);
    for (size_t w = 0; w < qlist.size(); w++) {
      int q = qlist[w];
      qchd.push_back(tr.chd[q]);
      for (int i = 0; i < 8; i++) {
        int t = tr.chd[q] + i;
        if (V.ptr[t + 1] == V.ptr[t]) continue;
        mask[w] |= (unsigned char)(1u << i);
        for (int64_t k = V.ptr[t]; k < V.ptr[t + 1]; k++) {
          int p = tr.par[V.idx[k]];
          int dd[3];
          for (int a = 0; a < 3; a++) dd[a] = tr.path[3 * p + a] - tr.path[3 * q + a];
          int d = (dd[0] + 1) * 9 + (dd[1] + 1) * 3 + (dd[2] + 1);
          if (d > 13) d--;  // skip (0,0,0)
          coll[w * 26 + d] = tr.chd[p];
        }
      }
    }
    pairs_chd = upload(qchd);
    pairs_coll = upload(coll);
    pairs_mask = upload(mask);
    pairs_n = (int)qlist.size();
    if (htc()) {  // directions present per tile of 128 target parents (an empty tile keeps one)
      std::vector<unsigned> dirs((pairs_n + 127) / 128, 0u);
      double steps = 0;
      for (int t = 0; t < (int)dirs.size(); t++) {
        for (int w = t * 128; w < std::min(pairs_n, t * 128 + 128); w++)
          for (int d = 0; d < 26; d++)
            if (coll[(size_t)w * 26 + d] != tr.nnodes) dirs[t] |= 1u << d;
        if (!dirs[t]) dirs[t] = 1u;
        steps += __builtin_popcount(dirs[t]);
      }
      // executed MMA work: per (tile, direction, 4 frequencies) 8 MMAs of
      // 128 x 32 x 8 and 8 of 128 x 16 x 8
      counters_tc_had = steps * (op.nfc / 4) * (8.0 * 2 * 128 * 32 * 8 + 8.0 * 2 * 128 * 16 * 8) *
                        (htc16_img ? sd_m * td_m : 1);
      htc_dirs = upload(dirs);
      if (htc16_img) {
        std::vector<int> ct;
        m2l_tc16_tables(pairs_n, tr.nnodes, coll.data(), &ct);
        htc16_ctab = upload(ct);
      }
    }
  }

  double counters_v = 0, counters_fwd = 0, counters_inv = 0, counters_near = 0, counters_surf = 0,
         counters_gemm = 0, counters_tc_had = 0;

  List make_list(const std::vector<int>& work, const std::vector<int>& aux, const std::vector<int64_t>& ptr = {},
                 const std::vector<int>& idx = {}, const std::vector<int64_t>& ptr2 = {},
                 const std::vector<int>& idx2 = {}) {
    List l;
    l.n = (int)work.size();
    l.work = upload(work);
    if (!aux.empty()) l.aux = upload(aux);
    if (!ptr.empty()) {
      l.ptr = upload(ptr);
      l.idx = upload(idx);
    }
    if (!ptr2.empty()) {
      l.ptr2 = upload(ptr2);
      l.idx2 = upload(idx2);
    }
    return l;
  }

  size_t S_supe = 0, S_supc = 0, S_tdnc = 0, S_tdne = 0, S_y = 0, S_z = 0, S_spec = 0, S_eff = 0;
  int cap_chunk = 0, max_chunk = 1;

  void replicate(List& L, int R) {
    if (L.n <= 0 || L.R >= R) return;
    const int nn = tr.nnodes;
    std::vector<int> w((size_t)R * L.n), a;
    if (!L.ha.empty()) a.resize((size_t)R * L.n);
    for (int r = 0; r < R; r++)
      for (int j = 0; j < L.n; j++) {
        w[(size_t)r * L.n + j] = L.hw[j] + r * nn;
        if (!a.empty()) a[(size_t)r * L.n + j] = L.ha[j] + (L.aux_nodes ? r * nn : 0);
      }
    L.rw = upload(w);
    L.ra = a.empty() ? nullptr : upload(a);
    L.R = R;
  }

  // per-vector node data for R density vectors at once, [r][node][...]
  void ensure_chunk(int R) {
    if (R <= cap_chunk) return;
    supeden = dalloc<T>((size_t)R * S_supe);
    KCHECK(cudaMemset(supeden, 0, sizeof(T) * (size_t)R * S_supe));  // empty nodes stay zero
    supcval = dalloc<T>((size_t)R * S_supc);
    tdncval = dalloc<T>((size_t)R * S_tdnc);
    tdneden = dalloc<T>((size_t)R * S_tdne);
    KCHECK(cudaMemset(tdneden, 0, sizeof(T) * (size_t)R * S_tdne));
    // y of a source-free child stays zero; z of a target-free child is written
    // by the L2L chain but never read
    ybuf = dalloc<T>((size_t)R * S_y);
    KCHECK(cudaMemset(ybuf, 0, sizeof(T) * (size_t)R * S_y));
    zbuf = dalloc<T>((size_t)R * S_z);
    KCHECK(cudaMemset(zbuf, 0, sizeof(T) * (size_t)R * S_z));
    if (!spectra && S_spec) {  // one set: the V list runs vector by vector
      spectra = dalloc<T>(S_spec);
      KCHECK(cudaMemset(spectra, 0, sizeof(T) * S_spec));
      effval = dalloc<T>(S_eff);
    }
    if (htc16_img) d_bound = dalloc<unsigned>(R);
    args.supeden = supeden;
    args.supcval = supcval;
    args.tdncval = tdncval;
    args.tdneden = tdneden;
    replicate(s2m, R);
    replicate(up_all, R);
    replicate(dn_all, R);
    for (auto& L : up_non) replicate(L, R);
    for (auto& L : dn_par) replicate(L, R);
    cap_chunk = R;
  }

  void ensure_rhs(int nrhs) {
    ensure_chunk(std::min(nrhs, max_chunk));
    if (nrhs <= cap_rhs) return;
    sden = dalloc<T>((size_t)nrhs * E.ns * sd_u);
    tval = dalloc<T>((size_t)nrhs * E.nt * td_u);
    cap_rhs = nrhs;
    args.sden = sden;
    args.tval = tval;
    if (near64) {
      sden64 = dalloc<double>((size_t)nrhs * E.ns * sd_u);
      tval64 = dalloc<double>((size_t)nrhs * E.nt * td_u);
      a64.sden = sden64;
      a64.tval = tval64;
    }
  }

  // col_lvl set: output rows scaled by 2^(-(depth + rootlvl) * deg)
  void gemm(const SurfOp& A, const T* B, int64_t ldb, const int* bidx, T* C, int64_t ldc, const int* cidx, int ncol,
            bool acc, cudaStream_t st, const int* col_lvl = nullptr) {
    if (ncol <= 0) return;
    GemmScale s = scl;
    s.col_lvl = col_lvl;
    s.lvl_base = E.rootlvl;
    if constexpr (sizeof(T) == 4) {
      if (A.tc.img && ldb % 4 == 0 && ldc % 4 == 0) {
        nlaunch += launch_node_gemm_tc(A.tc, B, ldb, bidx, C, ldc, cidx, ncol, acc, s, gemm_ws, gemm_ws_len, num_sms,
                                       d_status, st);
        return;
      }
    }
    nlaunch += launch_node_gemm<T>(A.M, A.K, A.a, B, ldb, bidx, C, ldc, cidx, ncol, acc, s, gemm_ws, gemm_ws_len,
                                   num_sms, st);
  }

  // a P2P pass for density vector rhs (global index, selects the sorted
  // densities and potentials) on slice r of the per-vector node data
  void p2p(const List& l, int which, int rhs, int r, cudaStream_t st) {
    if (l.n <= 0) return;
    P2PWork w;
    w.work = l.work;
    w.n = l.n;
    w.ptr = l.ptr;
    w.idx = l.idx;
    w.ptr2 = l.ptr2;
    w.idx2 = l.idx2;
    P2PArgs<T> a = args;
    a.supeden = supeden + (size_t)r * S_supe;
    a.supcval = supcval + (size_t)r * S_supc;
    a.tdncval = tdncval + (size_t)r * S_tdnc;
    a.tdneden = tdneden + (size_t)r * S_tdne;
    launch_p2p<T>(E.user.kt, a, w, which, rhs, st);
    nlaunch++;
  }

  // the V list for density vector slice r: forward spectra, Hadamard, inverse
  void vlist(int r, bool prof, cudaStream_t st) {
    T* sup = supeden + (size_t)r * S_supe;
    T* spec = spectra;  // reused by every vector of the chunk, in stream order
    T* eff = effval;
    T* tdc = tdncval + (size_t)r * S_tdnc;
    M2LGeom g = geom;
    if constexpr (sizeof(T) == 4) {
      if (htc16_img) {  // the largest value a spectrum can hold, for the FP16 scale
        g.bound = d_bound + r;
        launch_spectra_bound(sup, fwd.work, fwd.n, d_depth, E.rootlvl, op.deg.data(), sd_m, nsurf, d_bound + r,
                             num_sms, st);
        nlaunch++;
      }
    }
    launch_m2l_forward<T>(g, sup, fwd.work, fwd.n, d_depth, spec, st);
    if (prof) KCHECK(cudaEventRecord(ev[7], st));
    if (pairs_n > 0 && htc16_img) {
      launch_m2l_hadamard_tc16(E.had_groups, op.nfc, sd_m, td_m, htc16_img, reinterpret_cast<const unsigned*>(spec),
                               pairs_n, pairs_chd, htc16_ctab, htc_dirs, reinterpret_cast<float*>(eff), geom.plane,
                               d_bound + r, htc16_inv_sb, E.wait_limit, d_status, num_sms, st);
      KCHECK(cudaGetLastError());
    } else if (pairs_n > 0 && htc_img) {
      launch_m2l_hadamard_tc(op.nfc, htc_img, reinterpret_cast<const float*>(spec), pairs_n, pairs_chd, pairs_coll,
                             pairs_mask, htc_dirs, reinterpret_cast<float*>(eff), tr.nnodes, d_status, num_sms, st);
      KCHECK(cudaGetLastError());
    } else if (pairs_n > 0 && E.per_level) {
      // parents by depth d, their children's V lists with level d + 1's operators
      for (int d = 0; d + 1 < (int)ktiles_lv.size(); d++) {
        const int b = off_pairs[d], n = off_pairs[d + 1] - b;
        if (n > 0)
          launch_m2l_hadamard_sweep<T>(op.nfc, sd_m, td_m, ktiles_lv[d + 1], spec, n, pairs_chd + b,
                                       pairs_coll + (size_t)b * 26, pairs_mask + b, eff, tr.nnodes, d_status, num_sms,
                                       st);
      }
    } else if (pairs_n > 0) {
      if (ttiles)
        launch_m2l_hadamard_tz<T>(op.nfc, sd_m, td_m, ttiles, spec, pairs_n, pairs_chd, pairs_coll, pairs_mask, eff,
                                  tr.nnodes, d_status, num_sms, st);
      else
        launch_m2l_hadamard_sweep<T>(op.nfc, sd_m, td_m, ktiles, spec, pairs_n, pairs_chd, pairs_coll, pairs_mask,
                                     eff, tr.nnodes, d_status, num_sms, st);
    } else {
      launch_m2l_hadamard<T>(g, khat, spec, m2l.work, m2l.n, m2l.ptr, m2l.idx, d_path, eff, st);
    }
    if (prof) KCHECK(cudaEventRecord(ev[8], st));
    launch_m2l_inverse<T>(g, eff, m2l.work, m2l.n, tdc, st);
    nlaunch += 2 + (pairs_n > 0 ? (htc() ? 1 : sd_m * td_m) : 1);
  }

  // Density vectors go through the passes in chunks of up to max_chunk: the
  // point-surface passes and the V list run once per vector, and every
  // surface contraction runs once per chunk over all of its vectors' nodes
  // (the node lists repeated with offsets into [r][node][...] buffers), so
  // the operator is read once for the whole chunk.
  int eval(const double* d_srcden, double* d_trgval, int nrhs, cudaStream_t st) override {
    ensure_rhs(nrhs);
    nlaunch = 0;
    const int md = tr.maxdepth;
    const int K1 = nsurf * sd_m;
    const int chunk = std::max(1, std::min({nrhs, cap_chunk, E.rhs_chunk > 0 ? E.rhs_chunk : cap_chunk}));
    const bool prof = E.profiling && nrhs <= chunk;  // phase events for a single chunk
    if (prof) KCHECK(cudaEventRecord(ev[0], st));
    launch_scatter_den<T>(d_srcden, d_sperm, E.ns, sd_u, nrhs, sden, st);
    nlaunch++;
    if (near64) {
      launch_scatter_den<double>(d_srcden, d_sperm, E.ns, sd_u, nrhs, sden64, st);
      nlaunch++;
    }
    for (int r0 = 0; r0 < nrhs; r0 += chunk) {
      const int R = std::min(chunk, nrhs - r0);
      // upward: S2M per vector, then y = up_W * check on the leaves of every
      // level and vector at once, M2M bottom-up in y coordinates, and every
      // node's density = 2^(-l deg) up_V * y
      for (int r = 0; r < R; r++) p2p(s2m, P2P_S2M, r0 + r, r, st);
      if (E.per_level) {  // each level with its own operators (R = 1 here)
        for (int d = 0; d <= md; d++) {
          const int b = off_s2m[d];
          gemm(lv[d].upW, supcval, (int64_t)nuc * td_m, s2m.rw + b, ybuf, ru, s2m.rw + b, off_s2m[d + 1] - b, false,
               st);
        }
        for (int d = md - 1; d >= 2; d--) {
          const List& P = up_non[d];
          gemm(lv[d].m2my, ybuf, ru, P.ra, ybuf, ru, P.rw, P.n, false, st);
        }
        for (int d = 0; d <= md; d++) {
          const int b = off_up[d];
          gemm(lv[d].upV, ybuf, ru, up_all.rw + b, supeden, K1, up_all.rw + b, off_up[d + 1] - b, false, st);
        }
      } else {
        gemm(op_upW, supcval, (int64_t)nuc * td_m, s2m.rw, ybuf, ru, s2m.rw, R * s2m.n, false, st);
        for (int d = md - 1; d >= 2; d--) {
          const List& P = up_non[d];
          gemm(op_m2my, ybuf, ru, P.ra, ybuf, ru, P.rw, R * P.n, false, st);
        }
        gemm(op_upV, ybuf, ru, up_all.rw, supeden, K1, up_all.rw, R * up_all.n, false, st, up_all.ra);
      }
      if (prof) KCHECK(cudaEventRecord(ev[1], st));
      // V list
      KCHECK(cudaMemsetAsync(tdncval, 0, sizeof(T) * (size_t)R * S_tdnc, st));
      if (m2l.n > 0)
        for (int r = 0; r < R; r++) vlist(r, prof && r == 0, st);
      if (prof) KCHECK(cudaEventRecord(ev[2], st));
      // X list
      for (int r = 0; r < R; r++) p2p(s2l, P2P_S2L, r0 + r, r, st);
      if (prof) KCHECK(cudaEventRecord(ev[3], st));
      // downward: z = dn_W * check on the target nodes of every level and
      // vector at once, L2L top-down in z coordinates into the 8 children,
      // then every node's density = 2^(-l deg) dn_V * z
      if (E.per_level) {
        for (int d = 0; d <= md; d++) {
          const int b = off_dn[d];
          gemm(lv[d].dnW, tdncval, (int64_t)nsurf * td_m, dn_all.rw + b, zbuf, rd, dn_all.rw + b, off_dn[d + 1] - b,
               false, st);
        }
        for (int d = 3; d <= md; d++) {  // parents at depth d - 1
          const List& P = dn_par[d];
          gemm(lv[d - 1].l2lz, zbuf, rd, P.rw, zbuf, rd, P.ra, P.n, true, st);
        }
        for (int d = 0; d <= md; d++) {
          const int b = off_dn[d];
          gemm(lv[d].dnV, zbuf, rd, dn_all.rw + b, tdneden, K1, dn_all.rw + b, off_dn[d + 1] - b, false, st);
        }
      } else {
        gemm(op_dnW, tdncval, (int64_t)nsurf * td_m, dn_all.rw, zbuf, rd, dn_all.rw, R * dn_all.n, false, st);
        for (int d = 3; d <= md; d++) {
          const List& P = dn_par[d];
          gemm(op_l2lz, zbuf, rd, P.rw, zbuf, rd, P.ra, R * P.n, true, st);
        }
        gemm(op_dnV, zbuf, rd, dn_all.rw, tdneden, K1, dn_all.rw, R * dn_all.n, false, st, dn_all.ra);
      }
      if (prof) KCHECK(cudaEventRecord(ev[4], st));
      // leaves
      for (int r = 0; r < R; r++) {
        p2p(leaf, P2P_LEAF, r0 + r, r, st);
        if (near64 && near_u.n > 0) {
          P2PWork w;
          w.work = near_u.work;
          w.n = near_u.n;
          w.ptr = near_u.ptr;
          w.idx = near_u.idx;
          w.ptr2 = near_u.ptr2;
          w.idx2 = near_u.idx2;
          launch_p2p<double>(E.user.kt, a64, w, P2P_LEAF, r0 + r, st);
          nlaunch++;
        }
      }
      if (prof) KCHECK(cudaEventRecord(ev[5], st));
    }
    if constexpr (sizeof(T) == 4) {
      if (near64)
        launch_gather_val_sum(tval, tval64, d_tperm, E.nt, td_u, nrhs, d_trgval, st);
      else
        launch_gather_val<T>(tval, d_tperm, E.nt, td_u, nrhs, d_trgval, st);
    } else {
      launch_gather_val<T>(tval, d_tperm, E.nt, td_u, nrhs, d_trgval, st);
    }
    nlaunch++;
    if (prof) {
      KCHECK(cudaEventRecord(ev[6], st));
      KCHECK(cudaEventSynchronize(ev[6]));
      float ms;
      for (int i = 0; i < 5; i++) {
        KCHECK(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
        pt[i] = ms;
      }
      KCHECK(cudaEventElapsedTime(&ms, ev[0], ev[6]));
      pt[5] = ms;
      if (m2l.n > 0) {
        // ev[1] -> memset -> fwd -> ev[7] -> hadamard -> ev[8] -> inverse (vector 0) ...
        KCHECK(cudaEventElapsedTime(&ms, ev[1], ev[7]));
        pt[6] = ms;
        KCHECK(cudaEventElapsedTime(&ms, ev[7], ev[8]));
        pt[7] = ms;
        KCHECK(cudaEventElapsedTime(&ms, ev[8], ev[2]));
        pt[8] = ms;
      }
    }
    KCHECK(cudaGetLastError());
    return KIFMM_OK;
  }

  void reserve(int nrhs) override { ensure_rhs(nrhs); }
  int take_status() override {
    volatile int* p = h_status;
    int v = *p;
    *p = 0;
    return v;
  }

  void phase_times(double* ms) const override {
    for (int i = 0; i < 9; i++) ms[i] = pt[i];
  }
  int launches() const override { return nlaunch; }
  int max_rhs_chunk() const override { return max_chunk; }
  bool tunable_groups() const override { return htc16_img != nullptr && pairs_n > 0; }
};

// ---------------------------------------------------------------------------
Engine::~Engine() { release_device(); }

void Engine::release_device() {
  impl.reset();
  double** bufs[] = {&d_in, &d_out, &d_spos, &d_snor, &d_sden, &d_tchk, &d_vchk};
  for (double** b : bufs)
    if (*b) {
      cudaFree(*b);
      *b = nullptr;
    }
  d_in_cap = d_out_cap = d_sden_cap = d_tchk_cap = 0;
  if (stream) {
    cudaStreamDestroy(stream);
    stream = nullptr;
  }
}

static bool parse_int(const std::map<std::string, std::string>& o, const std::string& key, int* v, bool* found) {
  auto it = o.find(key);
  *found = it != o.end();
  if (!*found) return true;
  const char* s = it->second.c_str();
  char* end = nullptr;
  long x = std::strtol(s, &end, 10);  // first token, like istringstream >> int
  if (end == s) return false;
  *v = (int)x;
  return true;
}

int Engine::setup() {
  ready = false;
  if (!have_geom) {
    err = "geometry not set (kifmm_set_geometry)";
    return KIFMM_ERR_STATE;
  }
  if (!have_kernel) {
    err = "kernel not set (kifmm_set_kernel)";
    return KIFMM_ERR_STATE;
  }
  // options, FMM3d::setup (fmm3d/fmm3d_setup.cpp:30-31) and Let3d::setup (fmm3d/let3d.cpp:45-48)
  bool f1, f2, f3;
  if (!parse_int(opts, "-" + prefix + "np", &np, &f1) || !parse_int(opts, "-" + prefix + "let3d_ptsmax", &ptsmax, &f2) ||
      !parse_int(opts, "-" + prefix + "let3d_maxlevel", &maxlevel, &f3)) {
    err = "malformed option value";
    return KIFMM_ERR_OPTION;
  }
  if (!f1 || !f2 || !f3) {
    err = "missing required option (-" + prefix + "np, -" + prefix + "let3d_ptsmax, -" + prefix + "let3d_maxlevel)";
    return KIFMM_ERR_OPTION;
  }
  if (np < 2 || np > 8) {
    err = "np must be in [2, 8]";
    return KIFMM_ERR_OPTION;
  }
  if (maxlevel < 1 || maxlevel > 21 || ptsmax < 1) {
    err = "ptsmax must be >= 1 and maxlevel in [1, 21]";
    return KIFMM_ERR_OPTION;
  }
  auto pit = opts.find("-" + prefix + "precision");
  mixed = false;
  if (pit != opts.end()) {
    std::string v = pit->second;
    v.erase(0, v.find_first_not_of(" \t"));
    v = v.substr(0, v.find_first_of(" \t%"));
    if (v == "mixed" || v == "fp32")
      mixed = true;
    else if (v != "fp64") {
      err = "precision must be fp64 or mixed";
      return KIFMM_ERR_OPTION;
    }
  }
  {
    bool found = false;
    int tc = 1;
    if (!parse_int(opts, "-" + prefix + "tensor_cores", &tc, &found)) {
      err = "tensor_cores must be 0 or 1";
      return KIFMM_ERR_OPTION;
    }
    tensor_cores = tc != 0;
    auto fit = opts.find("-" + prefix + "m2l_form");
    // default: in mixed precision the tensor-core form for single-dof kernels
    // (tensor_cores on), else the factored form (as fast as the direct form
    // with ~40 % fewer multiply-adds); the direct form in FP64 (faster there)
    m2l_toeplitz = mixed;
    m2l_tc = mixed && tensor_cores;
    m2l_tc_tf32 = false;
    int wl = 1 << 22;
    if (!parse_int(opts, "-" + prefix + "wait_limit", &wl, &found) || wl < 0) {
      err = "wait_limit must be a non-negative integer";
      return KIFMM_ERR_OPTION;
    }
    wait_limit = wl;
    int hg = 3;
    if (!parse_int(opts, "-" + prefix + "had_groups", &hg, &found) || hg < 2 || hg > 3) {
      err = "had_groups must be 2 or 3";
      return KIFMM_ERR_OPTION;
    }
    had_groups = hg;
    had_groups_set = found;
    int rc = 0;
    if (!parse_int(opts, "-" + prefix + "rhs_chunk", &rc, &found) || rc < 0 || rc > 8) {
      err = "rhs_chunk must be in [0, 8]";
      return KIFMM_ERR_OPTION;
    }
    rhs_chunk = rc;
    rhs_chunk_set = found;
    int at = 0;
    if (!parse_int(opts, "-" + prefix + "autotune", &at, &found) || at < 0 || at > 1) {
      err = "autotune must be 0 or 1";
      return KIFMM_ERR_OPTION;
    }
    autotune = at;
    int ar = 1;
    if (!parse_int(opts, "-" + prefix + "autotune_rhs", &ar, &found) || ar < 1 || ar > 64) {
      err = "autotune_rhs must be in [1, 64]";
      return KIFMM_ERR_OPTION;
    }
    autotune_rhs = ar;
    if (fit != opts.end()) {
      std::string v = fit->second;
      v.erase(0, v.find_first_not_of(" \t"));
      v = v.substr(0, v.find_first_of(" \t%"));
      if (v == "direct") {
        m2l_toeplitz = false;
        m2l_tc = false;
      } else if (v == "toeplitz") {
        m2l_toeplitz = true;
        m2l_tc = false;
      } else if (v == "tensor") {  // where unsupported (FP64, several dofs): the default form
        m2l_tc = true;
      } else if (v == "tensor_tf32") {
        m2l_tc = true;
        m2l_tc_tf32 = true;
      } else {
        err = "m2l_form must be tensor, tensor_tf32, toeplitz or direct";
        return KIFMM_ERR_OPTION;
      }
    }
  }
  if (!equivalent_kernel(user, &mm)) {
    err = "kernel not supported by FMM3d";
    return KIFMM_ERR_KERNEL;
  }
  per_level = false;
  {
    auto oit = opts.find("-" + prefix + "operators");
    if (oit != opts.end()) {
      std::string v = oit->second;
      v.erase(0, v.find_first_not_of(" \t"));
      v = v.substr(0, v.find_first_of(" \t%"));
      if (v == "per_level")
        per_level = true;
      else if (v != "scaled") {
        err = "operators must be scaled or per_level";
        return KIFMM_ERR_OPTION;
      }
    }
    if (per_level) {
      // the per-level operators run with the direct parent-pair V-list form
      auto fit = opts.find("-" + prefix + "m2l_form");
      if (fit != opts.end() && fit->second.find("direct") == std::string::npos) {
        err = "per_level operators use the direct V-list form (-" + prefix + "m2l_form direct)";
        return KIFMM_ERR_OPTION;
      }
      if (np != 4 && np != 6 && np != 8) {
        err = "per_level operators need np = 4, 6 or 8";
        return KIFMM_ERR_OPTION;
      }
      m2l_tc = false;
      m2l_toeplitz = false;
    }
  }
  bool tree_on_device = true;
  {
    auto tit = opts.find("-" + prefix + "tree");
    if (tit != opts.end()) {
      std::string v = tit->second;
      v.erase(0, v.find_first_not_of(" \t"));
      v = v.substr(0, v.find_first_of(" \t%"));
      if (v == "host")
        tree_on_device = false;
      else if (v != "device") {
        err = "tree must be device or host";
        return KIFMM_ERR_OPTION;
      }
    }
  }
  release_device();
  tree_ready = false;
  int ndev = 0;
  const bool have_device = cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0;
  if (!have_device) cudaGetLastError();
  // tree + lists: on the GPU (tree_gpu.cu); the host builder (tree.cpp) on
  // request, or where there is no GPU at all -- setup then stops below with
  // KIFMM_ERR_NO_DEVICE, and only the tree introspection is available
  auto t0 = std::chrono::steady_clock::now();
  tree = Tree();
  tree.ctr[0] = ctr[0];
  tree.ctr[1] = ctr[1];
  tree.ctr[2] = ctr[2];
  tree.rootlvl = rootlvl;
  tree.ptsmax = ptsmax;
  tree.maxlevel = maxlevel;
  int rc = (tree_on_device && have_device) ? build_tree_device(tree, ns, srcpos.data(), nt, trgpos.data(), &err)
                                           : build_tree(tree, ns, srcpos.data(), nt, trgpos.data(), host_threads(), &err);
  if (rc == 3) return KIFMM_ERR_OUT_OF_BOX;
  if (rc == 4) return KIFMM_ERR_CUDA;
  if (rc != 0) return KIFMM_ERR_OPTION;
  tree_ready = true;
  auto t1 = std::chrono::steady_clock::now();
  ops = get_operators(mm, np, host_threads(), &err);
  if (!ops) return KIFMM_ERR_NUMERIC;
  lops.reset();
  if (per_level) {
    lops = get_level_operators(mm, np, rootlvl, rootlvl + std::max(tree.maxdepth, 0), host_threads(), &err);
    if (!lops) return KIFMM_ERR_NUMERIC;
  }
  auto t2 = std::chrono::steady_clock::now();
  setup_ms[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
  setup_ms[1] = std::chrono::duration<double, std::milli>(t2 - t1).count();
  // device stage: there is no CPU fallback
  if (!have_device) {
    err = "no CUDA device";
    return KIFMM_ERR_NO_DEVICE;
  }
  cudaGetDevice(&device);
  try {
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) throw CudaError{cudaGetLastError(), "stream"};
    if (mixed) {
      auto p = std::make_unique<Impl<float>>(*this);
      p->build();
      counters = {p->counters_near, p->counters_v, 0, (double)tree.nnodes, 0, p->counters_gemm, p->counters_fwd,
                  p->counters_inv, p->counters_surf, p->counters_tc_had};
      impl = std::move(p);
    } else {
      auto p = std::make_unique<Impl<double>>(*this);
      p->build();
      counters = {p->counters_near, p->counters_v, 0, (double)tree.nnodes, 0, p->counters_gemm, p->counters_fwd,
                  p->counters_inv, p->counters_surf, p->counters_tc_had};
      impl = std::move(p);
    }
    int nleaf = 0;
    for (int g = 0; g < tree.nnodes; g++) nleaf += tree.terminal(g) && (tree.tag[g] & TAG_TRG);
    counters[4] = nleaf;
    KCHECK(cudaDeviceSynchronize());
  } catch (const CudaError& e) {
    err = std::string(e.where) + ": " + cudaGetErrorString(e.e);
    cudaGetLastError();
    release_device();
    return e.e == cudaErrorMemoryAllocation ? KIFMM_ERR_ALLOC : KIFMM_ERR_CUDA;
  }
  setup_ms[2] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t2).count();
  setup_ms[3] = 0;
  ready = true;
  schedule[0] = had_groups;
  schedule[1] = rhs_chunk;
  for (int i = 2; i < 6; i++) schedule[i] = 0;
  if (autotune) {
    const int rc = autotune_run();
    if (rc != KIFMM_OK) {
      ready = false;
      return rc;
    }
  }
  return KIFMM_OK;
}

// ---------------------------------------------------------------------------
// Setup-time autotuner: the schedule knobs that change no result bit of
// meaning (the FP16 Hadamard's producer groups, and how many density vectors
// one pass of the surface contractions carries) are timed on the engine
// itself, on autotune_rhs synthetic density vectors, one warm-up and two
// timed evals per candidate (CUDA events on the engine stream, the faster of
// the two), and the fastest is kept.  Choices are cached process-wide per
// (kernel, equivalent kernel, np, precision, V-list form, size class of the
// tree = round(2 log2 nodes), vectors), so instances of one batch that share
// these tune once.  A knob given explicitly as an option is not tuned.
namespace {
struct TuneKey {
  int kt, kt_mm, np, mixed, form, size_class, nrhs;
  bool operator<(const TuneKey& o) const {
    return std::tie(kt, kt_mm, np, mixed, form, size_class, nrhs) <
           std::tie(o.kt, o.kt_mm, o.np, o.mixed, o.form, o.size_class, o.nrhs);
  }
};
struct TuneVal {
  int groups, chunk, ncand;
  double ms;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tuned;
}  // namespace

int Engine::autotune_run() {
  const auto t0 = std::chrono::steady_clock::now();
  const int R = autotune_rhs;
  const int form = m2l_tc ? (m2l_tc_tf32 ? 3 : 2) : (m2l_toeplitz ? 1 : 0);
  const TuneKey key{user.kt, mm.kt, np, mixed ? 1 : 0, form,
                    (int)std::lround(2.0 * std::log2((double)std::max(2, tree.nnodes))), R};
  auto finish = [&](const TuneVal& v, bool cached) {
    if (!had_groups_set) had_groups = v.groups;
    if (!rhs_chunk_set) rhs_chunk = v.chunk;
    schedule[0] = had_groups;
    schedule[1] = rhs_chunk;
    schedule[2] = 1;
    schedule[3] = cached ? 1 : 0;
    schedule[4] = v.ncand;
    schedule[5] = v.ms;
    setup_ms[3] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  };
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      finish(it->second, true);
      return KIFMM_OK;
    }
  }
  std::vector<int> groups = {had_groups};
  if (!had_groups_set && impl->tunable_groups()) groups = {2, 3};
  std::vector<int> chunks = {rhs_chunk};
  const int cmax = std::max(1, std::min(R, impl->max_rhs_chunk()));
  if (!rhs_chunk_set && R > 1) {
    chunks.clear();
    for (int c : {1, 2, 4})
      if (c < cmax) chunks.push_back(c);
    chunks.push_back(cmax);
  }
  // synthetic densities in [-1, 1): a fixed linear congruential sequence
  const size_t nin = (size_t)ns * user.sd * R, nout = (size_t)nt * user.td * R;
  std::vector<double> h(nin);
  uint64_t x = 0x9E3779B97F4A7C15ull;
  for (size_t i = 0; i < nin; i++) {
    x = x * 6364136223846793005ull + 1442695040888963407ull;
    h[i] = (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
  double *din = nullptr, *dout = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  TuneVal best{had_groups, rhs_chunk, 0, 1e300};
  int rc = KIFMM_OK;
  try {
    if (cudaMalloc(&din, std::max<size_t>(nin, 1) * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dout, std::max<size_t>(nout, 1) * sizeof(double)) != cudaSuccess)
      throw CudaError{cudaErrorMemoryAllocation, "autotune buffers"};
    KCHECK(cudaMemcpy(din, h.data(), nin * sizeof(double), cudaMemcpyHostToDevice));
    KCHECK(cudaEventCreate(&e0));
    KCHECK(cudaEventCreate(&e1));
    const bool prof = profiling;
    profiling = false;
    for (int g : groups)
      for (int c : chunks) {
        had_groups = g;
        rhs_chunk = c;
        double tbest = 1e300;
        for (int it = 0; it < 3; it++) {
          KCHECK(cudaEventRecord(e0, stream));
          int r = impl->eval(din, dout, R, stream);
          if (r != KIFMM_OK) throw CudaError{cudaErrorUnknown, "autotune eval"};
          KCHECK(cudaEventRecord(e1, stream));
          KCHECK(cudaEventSynchronize(e1));
          float ms = 0;
          KCHECK(cudaEventElapsedTime(&ms, e0, e1));
          if (it > 0) tbest = std::min(tbest, (double)ms);
        }
        best.ncand++;
        if (tbest < best.ms) {
          best.ms = tbest;
          best.groups = g;
          best.chunk = c;
        }
      }
    profiling = prof;
    if (impl->take_status()) {
      err = "a device-side wait timed out while autotuning";
      rc = KIFMM_ERR_CUDA;
    }
  } catch (const CudaError& e) {
    err = std::string("autotune: ") + e.where + ": " + cudaGetErrorString(e.e);
    cudaGetLastError();
    rc = e.e == cudaErrorMemoryAllocation ? KIFMM_ERR_ALLOC : KIFMM_ERR_CUDA;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (din) cudaFree(din);
  if (dout) cudaFree(dout);
  if (rc != KIFMM_OK) return rc;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = best;
  }
  finish(best, false);
  return KIFMM_OK;
}

// ---------------------------------------------------------------------------
// Concatenated instances.  Member trees go side by side: for every depth,
// each member's nodes of that depth as one block in its own breadth-first
// order, every block at depth >= 1 starting at an id that is 1 mod 8 (empty
// padding nodes fill the gaps), so every sibling group stays one aligned
// group of 8 and the forest's ids are breadth first again (depth never
// decreases).  Lists, parents and children are renumbered; point ranges are
// shifted by the member's point offset.  Padding nodes carry no points, no
// tag and no lists, so no pass touches them.
namespace {
void merge_trees(const std::vector<const Tree*>& ts, const std::vector<int>& soff, const std::vector<int>& toff,
                 Tree& t) {
  const int K = (int)ts.size();
  int md = 0;
  for (auto* x : ts) md = std::max(md, x->maxdepth);
  std::vector<std::vector<int>> map(K);
  for (int k = 0; k < K; k++) map[k].assign(ts[k]->nnodes, -1);
  std::vector<int> from_k, from_old;  // per forest node: member and its id there (-1: padding)
  std::vector<int> pad_depth;
  t.level_beg.clear();
  for (int d = 0; d <= md; d++) {
    t.level_beg.push_back((int)from_k.size());
    for (int k = 0; k < K; k++) {
      const Tree& x = *ts[k];
      if (d > x.maxdepth) continue;
      const int lb = x.level_beg[d], le = x.level_beg[d + 1];
      if (le <= lb) continue;
      if (d >= 1)
        while (from_k.size() % 8 != 1) {
          from_k.push_back(-1);
          from_old.push_back(d);
        }
      for (int g = lb; g < le; g++) {
        map[k][g] = (int)from_k.size();
        from_k.push_back(k);
        from_old.push_back(g);
      }
    }
  }
  t.level_beg.push_back((int)from_k.size());
  const int n = (int)from_k.size();
  t.nnodes = n;
  t.maxdepth = md;
  t.ctr[0] = ts[0]->ctr[0];
  t.ctr[1] = ts[0]->ctr[1];
  t.ctr[2] = ts[0]->ctr[2];
  t.rootlvl = ts[0]->rootlvl;
  t.ptsmax = ts[0]->ptsmax;
  t.maxlevel = ts[0]->maxlevel;
  t.depth.assign(n, 0);
  t.par.assign(n, -1);
  t.chd.assign(n, -1);
  t.tag.assign(n, 0);
  t.path.assign(3 * (size_t)n, 0);
  t.sbeg.assign(n, 0);
  t.scnt.assign(n, 0);
  t.tbeg.assign(n, 0);
  t.tcnt.assign(n, 0);
  t.center.assign(3 * (size_t)n, 0.0);
  t.radius.assign(n, 0.0);
  for (int g = 0; g < n; g++) {
    const int k = from_k[g];
    if (k < 0) {
      t.depth[g] = from_old[g];
      continue;
    }
    const Tree& x = *ts[k];
    const int o = from_old[g];
    t.depth[g] = x.depth[o];
    t.par[g] = x.par[o] >= 0 ? map[k][x.par[o]] : -1;
    t.chd[g] = x.chd[o] >= 0 ? map[k][x.chd[o]] : -1;
    t.tag[g] = x.tag[o];
    for (int a = 0; a < 3; a++) {
      t.path[3 * (size_t)g + a] = x.path[3 * (size_t)o + a];
      t.center[3 * (size_t)g + a] = x.center[3 * (size_t)o + a];
    }
    t.sbeg[g] = x.sbeg[o] + soff[k];
    t.scnt[g] = x.scnt[o];
    t.tbeg[g] = x.tbeg[o] + toff[k];
    t.tcnt[g] = x.tcnt[o];
    t.radius[g] = x.radius[o];
  }
  t.sperm.clear();
  t.tperm.clear();
  for (int k = 0; k < K; k++) {
    for (int p : ts[k]->sperm) t.sperm.push_back(p + soff[k]);
    for (int p : ts[k]->tperm) t.tperm.push_back(p + toff[k]);
  }
  for (int w = 0; w < 4; w++) {
    Csr& c = t.lists[w];
    c.ptr.assign(1, 0);
    c.idx.clear();
    for (int g = 0; g < n; g++) {
      const int k = from_k[g];
      if (k >= 0) {
        const Csr& xc = ts[k]->lists[w];
        const int o = from_old[g];
        for (int64_t e = xc.ptr[o]; e < xc.ptr[o + 1]; e++) c.idx.push_back(map[k][xc.idx[e]]);
      }
      c.ptr.push_back((int64_t)c.idx.size());
    }
  }
}
}  // namespace

std::string Engine::forest_key() const {
  if (!ready || per_level || !tree_ready) return std::string();
  // (the schedule knobs -- producer groups, density vectors per pass --
  // change no result, so members may have tuned them differently; the
  // forest takes its first member's)
  char b[320];
  std::snprintf(b, sizeof b, "%d %.17g %.17g %d %d %d %d %d %d %d %d %d", user.kt, user.coefs[0], user.coefs[1], mm.kt,
                np, mixed ? 1 : 0, tensor_cores ? 1 : 0, m2l_toeplitz ? 1 : 0, m2l_tc ? 1 : 0, m2l_tc_tf32 ? 1 : 0,
                rootlvl, wait_limit);
  return std::string(b);
}

int Engine::setup_forest(const std::vector<const Engine*>& ms) {
  ready = false;
  if (ms.empty()) {
    err = "no members";
    return KIFMM_ERR_ARG;
  }
  const Engine& m0 = *ms[0];
  const std::string key = m0.forest_key();
  for (const Engine* m : ms)
    if (key.empty() || m->forest_key() != key) {
      err = "members differ in kernel, np, precision, V-list form or root level";
      return KIFMM_ERR_ARG;
    }
  prefix = m0.prefix;
  opts = m0.opts;
  np = m0.np;
  ptsmax = m0.ptsmax;
  maxlevel = m0.maxlevel;
  mixed = m0.mixed;
  tensor_cores = m0.tensor_cores;
  m2l_toeplitz = m0.m2l_toeplitz;
  m2l_tc = m0.m2l_tc;
  m2l_tc_tf32 = m0.m2l_tc_tf32;
  wait_limit = m0.wait_limit;
  had_groups = m0.had_groups;
  rhs_chunk = m0.rhs_chunk;
  per_level = false;
  user = m0.user;
  mm = m0.mm;
  have_kernel = true;
  rootlvl = m0.rootlvl;
  for (int a = 0; a < 3; a++) ctr[a] = m0.ctr[a];
  ops = m0.ops;
  src_off.clear();
  trg_off.clear();
  ns = nt = 0;
  srcpos.clear();
  srcnor.clear();
  trgpos.clear();
  std::vector<const Tree*> ts;
  for (const Engine* m : ms) {
    src_off.push_back(ns);
    trg_off.push_back(nt);
    ns += m->ns;
    nt += m->nt;
    srcpos.insert(srcpos.end(), m->srcpos.begin(), m->srcpos.end());
    srcnor.insert(srcnor.end(), m->srcnor.begin(), m->srcnor.end());
    trgpos.insert(trgpos.end(), m->trgpos.begin(), m->trgpos.end());
    ts.push_back(&m->tree);
  }
  have_geom = true;
  release_device();
  tree = Tree();
  merge_trees(ts, src_off, trg_off, tree);
  tree_ready = true;
  device = m0.device;
  try {
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) throw CudaError{cudaGetLastError(), "stream"};
    if (mixed) {
      auto p = std::make_unique<Impl<float>>(*this);
      p->build();
      impl = std::move(p);
    } else {
      auto p = std::make_unique<Impl<double>>(*this);
      p->build();
      impl = std::move(p);
    }
    KCHECK(cudaDeviceSynchronize());
  } catch (const CudaError& e) {
    err = std::string(e.where) + ": " + cudaGetErrorString(e.e);
    cudaGetLastError();
    release_device();
    return e.e == cudaErrorMemoryAllocation ? KIFMM_ERR_ALLOC : KIFMM_ERR_CUDA;
  }
  schedule[0] = had_groups;
  schedule[1] = rhs_chunk;
  ready = true;
  return KIFMM_OK;
}

int Engine::eval_device(const double* d_srcden, double* d_trgval, int nrhs, cudaStream_t st, bool sync) {
  if (!ready) {
    err = "eval before a successful setup";
    return KIFMM_ERR_STATE;
  }
  if (nrhs < 1 || (!d_srcden && ns > 0) || (!d_trgval && nt > 0)) {
    err = "bad eval arguments";
    return KIFMM_ERR_ARG;
  }
  // a time-out of an earlier asynchronous eval surfaces at the next call,
  // the way CUDA reports errors of earlier asynchronous launches
  if (!sync && poll_status() != KIFMM_OK) return KIFMM_ERR_CUDA;
  try {
    int rc = impl->eval(d_srcden, d_trgval, nrhs, st);  // st as given: NULL is the legacy default stream
    if (rc != KIFMM_OK) return rc;
    if (sync) {
      KCHECK(cudaStreamSynchronize(st));
      if (impl->take_status()) {
        err = "a device-side wait timed out; results are incomplete";
        return KIFMM_ERR_CUDA;
      }
    }
  } catch (const CudaError& e) {
    err = std::string(e.where) + ": " + cudaGetErrorString(e.e);
    cudaGetLastError();
    return KIFMM_ERR_CUDA;
  }
  return KIFMM_OK;
}

int Engine::poll_status() {
  if (!ready) {
    err = "poll before a successful setup";
    return KIFMM_ERR_STATE;
  }
  const int v = impl->take_status();
  if (v) {
    err = "a device-side wait timed out (status bits " + std::to_string(v) + "); the results of that eval are incomplete";
    return KIFMM_ERR_CUDA;
  }
  return KIFMM_OK;
}

int Engine::reserve(int nrhs) {
  if (!ready) {
    err = "eval before a successful setup";
    return KIFMM_ERR_STATE;
  }
  try {
    impl->reserve(nrhs);
  } catch (const CudaError& e) {
    err = std::string(e.where) + ": " + cudaGetErrorString(e.e);
    return KIFMM_ERR_CUDA;
  }
  return KIFMM_OK;
}

int Engine::enqueue(const double* d_srcden, double* d_trgval, int nrhs, cudaStream_t st) {
  if (!ready) {
    err = "eval before a successful setup";
    return KIFMM_ERR_STATE;
  }
  if (nrhs < 1 || (!d_srcden && ns > 0) || (!d_trgval && nt > 0)) {
    err = "bad eval arguments";
    return KIFMM_ERR_ARG;
  }
  bool prof = profiling;
  profiling = false;  // per-phase event timing synchronises; not inside a capture
  int rc = KIFMM_OK;
  try {
    rc = impl->eval(d_srcden, d_trgval, nrhs, st);
  } catch (const CudaError& e) {
    err = std::string(e.where) + ": " + cudaGetErrorString(e.e);
    rc = KIFMM_ERR_CUDA;
  }
  profiling = prof;
  return rc;
}

int Engine::eval_host(const double* srcden, double* trgval, int nrhs) {
  if (!ready) {
    err = "eval before a successful setup";
    return KIFMM_ERR_STATE;
  }
  if (nrhs < 1 || (!srcden && ns > 0) || (!trgval && nt > 0)) {
    err = "bad eval arguments";
    return KIFMM_ERR_ARG;
  }
  size_t nin = (size_t)nrhs * ns * user.sd, nout = (size_t)nrhs * nt * user.td;
  try {
    if (nin > d_in_cap) {
      if (d_in) cudaFree(d_in);
      d_in = nullptr;
      KCHECK(cudaMalloc(&d_in, std::max<size_t>(nin, 1) * sizeof(double)));
      d_in_cap = nin;
    }
    if (nout > d_out_cap) {
      if (d_out) cudaFree(d_out);
      d_out = nullptr;
      KCHECK(cudaMalloc(&d_out, std::max<size_t>(nout, 1) * sizeof(double)));
      d_out_cap = nout;
    }
    KCHECK(cudaMemcpyAsync(d_in, srcden, nin * sizeof(double), cudaMemcpyHostToDevice, stream));
    int rc = impl->eval(d_in, d_out, nrhs, stream);
    if (rc != KIFMM_OK) return rc;
    KCHECK(cudaMemcpyAsync(trgval, d_out, nout * sizeof(double), cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaStreamSynchronize(stream));
    if (impl->take_status()) {
      err = "a device-side wait timed out; results are incomplete";
      return KIFMM_ERR_CUDA;
    }
  } catch (const CudaError& e) {
    err = std::string(e.where) + ": " + cudaGetErrorString(e.e);
    cudaGetLastError();
    return KIFMM_ERR_CUDA;
  }
  return KIFMM_OK;
}

int Engine::direct(const double* srcden, int ntc, const double* tpos, double* out) {
  if (!ready) {
    err = "direct before a successful setup";
    return KIFMM_ERR_STATE;
  }
  try {
    if (!d_spos) {
      KCHECK(cudaMalloc(&d_spos, std::max<size_t>(1, 3 * (size_t)ns) * sizeof(double)));
      KCHECK(cudaMalloc(&d_snor, std::max<size_t>(1, 3 * (size_t)ns) * sizeof(double)));
      KCHECK(cudaMemcpy(d_spos, srcpos.data(), 3 * (size_t)ns * sizeof(double), cudaMemcpyHostToDevice));
      KCHECK(cudaMemcpy(d_snor, srcnor.data(), 3 * (size_t)ns * sizeof(double), cudaMemcpyHostToDevice));
    }
    size_t nden = (size_t)ns * user.sd;
    if (nden > d_sden_cap || !d_sden) {
      if (d_sden) cudaFree(d_sden);
      d_sden = nullptr;
      KCHECK(cudaMalloc(&d_sden, std::max<size_t>(1, nden) * sizeof(double)));
      d_sden_cap = nden;
    }
    KCHECK(cudaMemcpy(d_sden, srcden, nden * sizeof(double), cudaMemcpyHostToDevice));
    size_t ntp = std::max<size_t>(1, (size_t)ntc);
    if (ntp > d_tchk_cap || !d_tchk) {
      if (d_tchk) cudaFree(d_tchk);
      if (d_vchk) cudaFree(d_vchk);
      d_tchk = d_vchk = nullptr;
      KCHECK(cudaMalloc(&d_tchk, 3 * ntp * sizeof(double)));
      KCHECK(cudaMalloc(&d_vchk, 4 * ntp * sizeof(double)));
      d_tchk_cap = ntp;
    }
    KCHECK(cudaMemcpy(d_tchk, tpos, 3 * (size_t)ntc * sizeof(double), cudaMemcpyHostToDevice));
    double kc[3];
    kernel_constants(user.kt, user.coefs, kc);
    launch_direct(user.kt, d_spos, d_snor, d_sden, ns, d_tchk, ntc, d_vchk, kc, stream);
    KCHECK(cudaGetLastError());
    KCHECK(cudaMemcpyAsync(out, d_vchk, (size_t)ntc * user.td * sizeof(double), cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaStreamSynchronize(stream));
  } catch (const CudaError& e) {
    err = std::string(e.where) + ": " + cudaGetErrorString(e.e);
    cudaGetLastError();
    return KIFMM_ERR_CUDA;
  }
  return KIFMM_OK;
}

int Engine::check(const double* srcden, const double* trgval, int numchk, uint64_t seed, double* relerr) {
  if (!ready) {
    err = "check before a successful setup";
    return KIFMM_ERR_STATE;
  }
  if (numchk < 1 || nt < 1) {
    err = "numchk and the target count must be positive";
    return KIFMM_ERR_ARG;
  }
  // FMM3d::check picks targets uniformly at random (fmm3d/fmm3d_check.cpp:33-36)
  std::mt19937_64 rng(seed);
  std::vector<int> pick(numchk);
  std::vector<double> tp(3 * (size_t)numchk), dv((size_t)numchk * user.td);
  for (int k = 0; k < numchk; k++) {
    pick[k] = (int)(rng() % (uint64_t)nt);
    for (int d = 0; d < 3; d++) tp[3 * k + d] = trgpos[3 * (size_t)pick[k] + d];
  }
  int rc = direct(srcden, numchk, tp.data(), dv.data());
  if (rc != KIFMM_OK) return rc;
  double vn = 0, en = 0;  // :61-69
  for (int k = 0; k < numchk; k++)
    for (int i = 0; i < user.td; i++) {
      double f = trgval[(size_t)pick[k] * user.td + i];
      double dd = dv[(size_t)k * user.td + i] - f;
      vn += f * f;
      en += dd * dd;
    }
  *relerr = std::sqrt(en) / std::sqrt(vn);
  return KIFMM_OK;
}

}  // namespace kifmm
