// The adaptive octree and the U/V/W/X interaction lists of the reference's
// Let3d (fmm3d/let3d.cpp:56-281) built on the GPU, bit for bit the same tree
// and lists as the reference (and as the host builder of tree.cpp):
//
//   keys     every point's Morton key from the reference's FP64 octant test
//            (p >= centre per axis, centre = ll + (2 rad)(path + 0.5) / 2^d,
//            fmm3d/let3d.cpp:99, :309-318), one 3-bit digit per level, x most
//            significant (child index a*4 + b*2 + c, :307); points outside
//            the root box are reported (:73, :155)
//   sort     a stable least-significant-digit radix sort of (key, point id),
//            8 bits per pass: per-tile digit histograms, one exclusive scan,
//            a stable scatter that ranks each tile's elements in order
//            (warp match for the rank inside a warp, shared counters across
//            warps and rounds), so equal keys keep the original point order
//            the reference inserts them in (:117-135)
//   levels   breadth first, one level at a time: a node splits while it holds
//            more than ptsmax sources and its depth is below maxlevel - 1
//            (:86); its 8 children get consecutive ids after every node of
//            the level (the order of Let3d::ndevec), and each child's source
//            and target ranges are found by binary search on the digit of the
//            sorted keys
//   lists    Let3d::calgnext (:214-281) per target node, one thread each:
//            the 6 x 6 x 6 children of the parent's neighbourhood, findgnt
//            (:325-337) from the root, adjacent (:339-352), the descent into
//            adjacent same-level colleagues as an explicit depth-first stack;
//            a counting pass, a scan, a filling pass, then each list sorted
//            in place (the reference keeps std::sets sorted by node id)
//
// The result is copied into the host Tree the rest of setup reads.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "tree.hpp"

namespace kifmm {
namespace {

constexpr int TB = 256;             // threads per block of the sort kernels
constexpr int TILE = TB * 8;        // elements per sort tile
constexpr int MAXLEV = 21;          // maxlevel <= 21
constexpr int STACK = 8 * MAXLEV;   // depth-first descent stack

struct DevErr {
  cudaError_t e;
  const char* where;
};
#define TCHECK(call)                                   \
  do {                                                 \
    cudaError_t _e = (call);                           \
    if (_e != cudaSuccess) throw DevErr{_e, #call};    \
  } while (0)

// ---------------------------------------------------------------------------
// keys
__global__ void k_keys(const double* __restrict__ pos, int n, double llx, double lly, double llz, double rad,
                       double cx, double cy, double cz, int nlev, unsigned long long* __restrict__ key,
                       int* __restrict__ id, int* __restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double p[3] = {pos[3 * (size_t)i], pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2]};
  const double ll[3] = {llx, lly, llz}, c0[3] = {cx, cy, cz};
  for (int a = 0; a < 3; a++)
    if (!(p[a] >= __dsub_rn(c0[a], rad) && p[a] <= __dadd_rn(c0[a], rad))) atomicOr(bad, 1);
  int path[3] = {0, 0, 0};
  unsigned long long k = 0;
  for (int d = 0; d < nlev; d++) {
    const double tmp = (double)(1 << d);
    int dig = 0;
    for (int a = 0; a < 3; a++) {
      // ll + (2 rad)(path + 0.5) / tmp, operation by operation as the reference
      const double c = __dadd_rn(ll[a], __ddiv_rn(__dmul_rn(__dmul_rn(2.0, rad), __dadd_rn((double)path[a], 0.5)), tmp));
      const int b = p[a] >= c;
      path[a] = 2 * path[a] + b;
      dig = (dig << 1) | b;
    }
    k = (k << 3) | (unsigned long long)dig;
  }
  key[i] = k;
  id[i] = i;
}

// ---------------------------------------------------------------------------
// stable LSD radix sort, 8 bits per pass
__global__ void __launch_bounds__(TB) k_hist(const unsigned long long* __restrict__ key, int n, int sh,
                                              int ntiles, int* __restrict__ hist) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int t0 = blockIdx.x * TILE;
  for (int e = t0 + threadIdx.x; e < min(n, t0 + TILE); e += TB) atomicAdd(&h[(key[e] >> sh) & 255], 1);
  __syncthreads();
  hist[threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];  // digit major
}

// exclusive scan of n ints in place, one block (n up to a few million)
__global__ void __launch_bounds__(1024) k_scan_excl(int* __restrict__ a, int n, int* __restrict__ total) {
  __shared__ int part[1024];
  const int per = (n + 1023) / 1024;
  const int b = threadIdx.x * per, e = min(n, b + per);
  int s = 0;
  for (int i = b; i < e; i++) s += a[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = part[threadIdx.x] - s;
  for (int i = b; i < e; i++) {
    const int v = a[i];
    a[i] = run;
    run += v;
  }
  if (threadIdx.x == 1023 && total) *total = part[1023];
}

// 64-bit variant for list offsets
__global__ void __launch_bounds__(1024) k_scan_excl64(const int* __restrict__ cnt, long long* __restrict__ out, int n) {
  __shared__ long long part[1024];
  const int per = (n + 1023) / 1024;
  const int b = threadIdx.x * per, e = min(n, b + per);
  long long s = 0;
  for (int i = b; i < e; i++) s += cnt[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const long long v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  long long run = part[threadIdx.x] - s;
  for (int i = b; i < e; i++) {
    out[i] = run;
    run += cnt[i];
  }
  if (threadIdx.x == 1023) out[n] = part[1023];
}

__global__ void __launch_bounds__(TB) k_scatter(const unsigned long long* __restrict__ key, const int* __restrict__ id,
                                                 int n, int sh, int ntiles, const int* __restrict__ off,
                                                 unsigned long long* __restrict__ key2, int* __restrict__ id2) {
  __shared__ int cnt[TB / 32][256];
  __shared__ int run[256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  run[threadIdx.x] = off[threadIdx.x * ntiles + blockIdx.x];
  const int t0 = blockIdx.x * TILE;
  for (int r = 0; r < TILE / TB; r++) {
    for (int w = 0; w < TB / 32; w++) cnt[w][threadIdx.x] = 0;
    __syncthreads();
    const int e = t0 + r * TB + threadIdx.x;  // round r: elements in order, warp w covers 32 consecutive
    const bool v = e < n;
    const unsigned long long k = v ? key[e] : 0ull;
    const int dig = v ? (int)((k >> sh) & 255) : 256 + lane;  // invalid lanes match nobody
    const unsigned act = __ballot_sync(0xffffffffu, v);
    const unsigned peers = __match_any_sync(0xffffffffu, dig) & act;
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (v && rank == 0) cnt[warp][dig] = __popc(peers);
    __syncthreads();
    {  // per digit: exclusive prefix over the warps, in warp order
      int acc = 0;
      for (int w = 0; w < TB / 32; w++) {
        const int c = cnt[w][threadIdx.x];
        cnt[w][threadIdx.x] = acc;
        acc += c;
      }
      __syncthreads();
      if (v) {
        const int dst = run[dig] + cnt[warp][dig] + rank;
        key2[dst] = k;
        id2[dst] = id[e];
      }
      __syncthreads();
      run[threadIdx.x] += acc;
    }
    __syncthreads();
  }
}

void radix_sort_pairs(unsigned long long*& key, int*& id, unsigned long long*& key2, int*& id2, int* d_hist, int n,
                      int bits, cudaStream_t st) {
  if (n <= 1) return;
  const int ntiles = (n + TILE - 1) / TILE;
  for (int sh = 0; sh < bits; sh += 8) {
    k_hist<<<ntiles, TB, 0, st>>>(key, n, sh, ntiles, d_hist);
    k_scan_excl<<<1, 1024, 0, st>>>(d_hist, 256 * ntiles, nullptr);
    k_scatter<<<ntiles, TB, 0, st>>>(key, id, n, sh, ntiles, d_hist, key2, id2);
    std::swap(key, key2);
    std::swap(id, id2);
  }
}

// ---------------------------------------------------------------------------
// levels
struct DNodes {
  int *par, *chd, *depth, *path, *sbeg, *scnt, *tbeg, *tcnt;
};

__global__ void k_split_flags(DNodes nd, int beg, int end, int ptsmax, int can_split, int* __restrict__ flag) {
  const int k = beg + blockIdx.x * blockDim.x + threadIdx.x;
  if (k < end) flag[k - beg] = (can_split && nd.scnt[k] > ptsmax) ? 1 : 0;
}

// first index in [lo, hi) of sorted keys whose digit at depth d is >= v
__device__ __forceinline__ int digit_lb(const unsigned long long* key, int lo, int hi, int d, int nlev, int v) {
  const int sh = 3 * (nlev - 1 - d);
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if ((int)((key[mid] >> sh) & 7) < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__global__ void k_children(DNodes nd, int beg, int end, const int* __restrict__ flag, const int* __restrict__ pre,
                           const unsigned long long* __restrict__ skey, const unsigned long long* __restrict__ tkey,
                           int nlev) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;  // (node of the level, octant)
  const int k = beg + (w >> 3), o = w & 7;
  if (k >= end || !flag[k - beg]) return;
  const int cb = end + 8 * pre[k - beg];
  if (o == 0) nd.chd[k] = cb;
  const int d = nd.depth[k];
  const int sb = nd.sbeg[k], se = sb + nd.scnt[k], tb = nd.tbeg[k], te = tb + nd.tcnt[k];
  const int s0 = digit_lb(skey, sb, se, d, nlev, o), s1 = digit_lb(skey, sb, se, d, nlev, o + 1);
  const int t0 = digit_lb(tkey, tb, te, d, nlev, o), t1 = digit_lb(tkey, tb, te, d, nlev, o + 1);
  const int c = cb + o;
  nd.par[c] = k;
  nd.chd[c] = -1;
  nd.depth[c] = d + 1;
  nd.path[3 * c] = 2 * nd.path[3 * k] + ((o >> 2) & 1);
  nd.path[3 * c + 1] = 2 * nd.path[3 * k + 1] + ((o >> 1) & 1);
  nd.path[3 * c + 2] = 2 * nd.path[3 * k + 2] + (o & 1);
  nd.sbeg[c] = s0;
  nd.scnt[c] = s1 - s0;
  nd.tbeg[c] = t0;
  nd.tcnt[c] = t1 - t0;
}

__global__ void k_geom(DNodes nd, int nn, double llx, double lly, double llz, double rad, int* __restrict__ tag,
                       double* __restrict__ center, double* __restrict__ radius) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nn) return;
  tag[g] = (nd.scnt[g] > 0 ? TAG_SRC : 0) | (nd.tcnt[g] > 0 ? TAG_TRG : 0);
  const double tmp = (double)(1 << nd.depth[g]);
  const double ll[3] = {llx, lly, llz};
  for (int a = 0; a < 3; a++)
    center[3 * g + a] =
        __dadd_rn(ll[a], __ddiv_rn(__dmul_rn(__dmul_rn(2.0, rad), __dadd_rn((double)nd.path[3 * g + a], 0.5)), tmp));
  radius[g] = __ddiv_rn(rad, tmp);
}

// ---------------------------------------------------------------------------
// lists (Let3d::calgnext)
struct ListOut {
  long long* ptr[4];  // nullptr in the counting pass
  int* idx[4];
  int* cnt[4];        // counting pass: per node
};

__device__ __forceinline__ int findgnt(const DNodes& nd, int wdepth, const int* wpath) {
  int cur = 0;
  int left[3] = {wpath[0], wpath[1], wpath[2]};
  while (nd.depth[cur] < wdepth && nd.chd[cur] != -1) {
    const int dif = wdepth - nd.depth[cur];
    const int tmp = 1 << (dif - 1);
    int ch[3];
    for (int a = 0; a < 3; a++) {
      ch[a] = left[a] / tmp;
      left[a] -= ch[a] * tmp;
    }
    cur = nd.chd[cur] + ch[0] * 4 + ch[1] * 2 + ch[2];
  }
  return cur;
}

__device__ __forceinline__ bool adjacent(const DNodes& nd, int me, int yo) {
  const int md = max(nd.depth[me], nd.depth[yo]);
  const int merad = 1 << (md - nd.depth[me]);
  const int yorad = 1 << (md - nd.depth[yo]);
  const int r = merad + yorad;
  int mx = 0;
  for (int a = 0; a < 3; a++) {
    const int dif = abs((2 * nd.path[3 * me + a] + 1) * merad - (2 * nd.path[3 * yo + a] + 1) * yorad);
    if (dif > r) return false;
    mx = max(mx, dif);
  }
  return mx == r;
}

__device__ __forceinline__ void isort(int* a, int n) {
  for (int i = 1; i < n; i++) {
    const int v = a[i];
    int j = i - 1;
    while (j >= 0 && a[j] > v) {
      a[j + 1] = a[j];
      j--;
    }
    a[j + 1] = v;
  }
}

__device__ __forceinline__ int sort_unique(int* a, int n) {
  isort(a, n);
  int m = 0;
  for (int i = 0; i < n; i++)
    if (m == 0 || a[m - 1] != a[i]) a[m++] = a[i];
  return m;
}

// one thread per target node; fill == false counts, fill == true writes
template <bool FILL>
__global__ void __launch_bounds__(128) k_lists(DNodes nd, const int* __restrict__ tag, int nn, ListOut out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nn) return;
  int n[4] = {0, 0, 0, 0};
  long long base[4] = {0, 0, 0, 0};
  if (FILL)
    for (int l = 0; l < 4; l++) base[l] = out.ptr[l][g];
  auto put = [&](int l, int x) {
    if (!(tag[x] & TAG_SRC)) return;
    if (FILL) out.idx[l][base[l] + n[l]] = x;
    n[l]++;
  };
  if (tag[g] & TAG_TRG) {
    const bool term = nd.chd[g] == -1;
    const int pg = nd.par[g];
    int cu[216], cx[216];  // coarser U and X candidates (duplicates possible)
    int vb[216];           // V (distinct same-level nodes), sorted before they are written
    int ncu = 0, ncx = 0, nvb = 0;
    int stack[STACK];
    if (pg != -1) {
      const int dg = nd.depth[g];
      const int maxidx = 1 << dg;
      for (int i = -2; i < 4; i++)
        for (int j = -2; j < 4; j++)
          for (int k = -2; k < 4; k++) {
            const int tp[3] = {2 * nd.path[3 * pg] + i, 2 * nd.path[3 * pg + 1] + j, 2 * nd.path[3 * pg + 2] + k};
            if (tp[0] < 0 || tp[1] < 0 || tp[2] < 0 || tp[0] >= maxidx || tp[1] >= maxidx || tp[2] >= maxidx)
              continue;
            if (tp[0] == nd.path[3 * g] && tp[1] == nd.path[3 * g + 1] && tp[2] == nd.path[3 * g + 2]) continue;
            const int res = findgnt(nd, dg, tp);
            const bool adj = adjacent(nd, res, g);
            if (nd.depth[res] < dg) {
              if (adj) {
                if (term) cu[ncu++] = res;
              } else {
                cx[ncx++] = res;
              }
            }
            if (nd.depth[res] == dg) {
              if (!adj) {
                vb[nvb++] = res;
              } else if (term) {
                // descent into an adjacent colleague: non-adjacent descendants
                // are W, adjacent leaves U (the reference's breadth-first
                // queue, here depth first; the lists are sorted below)
                int sp = 0;
                stack[sp++] = res;
                while (sp > 0) {
                  const int f = stack[--sp];
                  if (!adjacent(nd, f, g)) {
                    put(2, f);
                  } else if (nd.chd[f] == -1) {
                    put(0, f);
                  } else {
                    for (int c = 7; c >= 0; c--) stack[sp++] = nd.chd[f] + c;
                  }
                }
              }
            }
          }
    }
    if (term) cu[ncu++] = g;
    ncu = sort_unique(cu, ncu);
    ncx = sort_unique(cx, ncx);
    isort(vb, nvb);
    for (int i = 0; i < ncu; i++) put(0, cu[i]);
    for (int i = 0; i < nvb; i++) put(1, vb[i]);
    for (int i = 0; i < ncx; i++) put(3, cx[i]);
  }
  if (!FILL)
    for (int l = 0; l < 4; l++) out.cnt[l][g] = n[l];
}

// each node's list segment sorted in place (ascending node id)
__global__ void k_sort_segments(const long long* __restrict__ ptr, int* __restrict__ idx, int nn) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nn) return;
  const long long b = ptr[g], e = ptr[g + 1];
  for (long long i = b + 1; i < e; i++) {
    const int v = idx[i];
    long long j = i - 1;
    while (j >= b && idx[j] > v) {
      idx[j + 1] = idx[j];
      j--;
    }
    idx[j + 1] = v;
  }
}

template <class T>
T* dnew(size_t n, std::vector<void*>& owned) {
  void* p = nullptr;
  TCHECK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  owned.push_back(p);
  return (T*)p;
}

template <class T>
void d2h(std::vector<T>& v, const T* d, size_t n, cudaStream_t st) {
  v.resize(n);
  if (n) TCHECK(cudaMemcpyAsync(v.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, st));
}

}  // namespace

int build_tree_device(Tree& t, int ns, const double* srcpos, int nt, const double* trgpos, std::string* err) {
  if (t.maxlevel < 1 || t.maxlevel > MAXLEV || t.ptsmax < 0 || ns < 0 || nt < 0) {
    if (err) *err = "bad ptsmax/maxlevel (maxlevel must be in [1,21])";
    return 1;
  }
  std::vector<void*> owned;
  cudaStream_t st = nullptr;
  int rc = 0;
  try {
    TCHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const double rad = t.rad();
    const double ll[3] = {t.ctr[0] - rad, t.ctr[1] - rad, t.ctr[2] - rad};
    const int nlev = t.maxlevel - 1;
    // ---- keys and the sort
    // every key / id buffer holds max(ns, nt): the sort swaps buffers, so the
    // scratch of the second sort may be the first one's input buffer
    const size_t nmax = (size_t)std::max(ns, nt);
    double* d_pos = dnew<double>(3 * nmax, owned);
    unsigned long long* skey = dnew<unsigned long long>(nmax, owned);
    unsigned long long* tkey = dnew<unsigned long long>(nmax, owned);
    unsigned long long* kbuf = dnew<unsigned long long>(nmax, owned);
    int* sid = dnew<int>(nmax, owned);
    int* tid = dnew<int>(nmax, owned);
    int* ibuf = dnew<int>(nmax, owned);
    int* d_bad = dnew<int>(1, owned);
    int* d_hist = dnew<int>(256 * ((size_t)std::max(ns, nt) / TILE + 1), owned);
    TCHECK(cudaMemsetAsync(d_bad, 0, sizeof(int), st));
    auto keys = [&](const double* pos, int n, unsigned long long*& key, int*& id) {
      if (n == 0) return;
      TCHECK(cudaMemcpyAsync(d_pos, pos, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
      k_keys<<<(n + 255) / 256, 256, 0, st>>>(d_pos, n, ll[0], ll[1], ll[2], rad, t.ctr[0], t.ctr[1], t.ctr[2], nlev,
                                              key, id, d_bad);
      radix_sort_pairs(key, id, kbuf, ibuf, d_hist, n, 3 * nlev, st);
    };
    keys(srcpos, ns, skey, sid);
    keys(trgpos, nt, tkey, tid);
    int bad = 0;
    TCHECK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    TCHECK(cudaStreamSynchronize(st));
    if (bad) {
      if (err) *err = "a point lies outside the root box";
      throw 3;
    }
    d2h(t.sperm, sid, ns, st);
    d2h(t.tperm, tid, nt, st);
    // ---- levels
    size_t cap = 1024;
    DNodes nd{};
    auto alloc_nodes = [&](size_t c) {
      DNodes n2{dnew<int>(c, owned), dnew<int>(c, owned), dnew<int>(c, owned), dnew<int>(3 * c, owned),
                dnew<int>(c, owned), dnew<int>(c, owned), dnew<int>(c, owned), dnew<int>(c, owned)};
      return n2;
    };
    nd = alloc_nodes(cap);
    {
      const int root[1] = {-1}, zero[3] = {0, 0, 0};
      TCHECK(cudaMemcpyAsync(nd.par, root, sizeof(int), cudaMemcpyHostToDevice, st));
      TCHECK(cudaMemcpyAsync(nd.chd, root, sizeof(int), cudaMemcpyHostToDevice, st));
      TCHECK(cudaMemcpyAsync(nd.depth, zero, sizeof(int), cudaMemcpyHostToDevice, st));
      TCHECK(cudaMemcpyAsync(nd.path, zero, 3 * sizeof(int), cudaMemcpyHostToDevice, st));
      TCHECK(cudaMemcpyAsync(nd.sbeg, zero, sizeof(int), cudaMemcpyHostToDevice, st));
      TCHECK(cudaMemcpyAsync(nd.scnt, &ns, sizeof(int), cudaMemcpyHostToDevice, st));
      TCHECK(cudaMemcpyAsync(nd.tbeg, zero, sizeof(int), cudaMemcpyHostToDevice, st));
      TCHECK(cudaMemcpyAsync(nd.tcnt, &nt, sizeof(int), cudaMemcpyHostToDevice, st));
    }
    std::vector<int> level_beg{0};
    int beg = 0, end = 1, level = 0;
    int* flag = nullptr;
    size_t flag_cap = 0;
    int* d_total = dnew<int>(1, owned);
    while (beg < end) {
      const int cnt = end - beg;
      if ((size_t)cnt > flag_cap) {
        flag_cap = std::max<size_t>(2 * flag_cap, cnt);
        flag = dnew<int>(flag_cap, owned);
      }
      const int can_split = level < t.maxlevel - 1;
      k_split_flags<<<(cnt + 255) / 256, 256, 0, st>>>(nd, beg, end, t.ptsmax, can_split, flag);
      // prefix of the flags (a copy: the flags are read again)
      int* pre = dnew<int>(cnt, owned);
      TCHECK(cudaMemcpyAsync(pre, flag, cnt * sizeof(int), cudaMemcpyDeviceToDevice, st));
      k_scan_excl<<<1, 1024, 0, st>>>(pre, cnt, d_total);
      int nsplit = 0;
      TCHECK(cudaMemcpyAsync(&nsplit, d_total, sizeof(int), cudaMemcpyDeviceToHost, st));
      TCHECK(cudaStreamSynchronize(st));
      const size_t need = (size_t)end + 8 * (size_t)nsplit;
      if (need > cap) {  // grow the node arrays (copy what exists)
        size_t c2 = cap;
        while (c2 < need) c2 *= 2;
        DNodes n2 = alloc_nodes(c2);
        TCHECK(cudaMemcpyAsync(n2.par, nd.par, end * sizeof(int), cudaMemcpyDeviceToDevice, st));
        TCHECK(cudaMemcpyAsync(n2.chd, nd.chd, end * sizeof(int), cudaMemcpyDeviceToDevice, st));
        TCHECK(cudaMemcpyAsync(n2.depth, nd.depth, end * sizeof(int), cudaMemcpyDeviceToDevice, st));
        TCHECK(cudaMemcpyAsync(n2.path, nd.path, 3 * (size_t)end * sizeof(int), cudaMemcpyDeviceToDevice, st));
        TCHECK(cudaMemcpyAsync(n2.sbeg, nd.sbeg, end * sizeof(int), cudaMemcpyDeviceToDevice, st));
        TCHECK(cudaMemcpyAsync(n2.scnt, nd.scnt, end * sizeof(int), cudaMemcpyDeviceToDevice, st));
        TCHECK(cudaMemcpyAsync(n2.tbeg, nd.tbeg, end * sizeof(int), cudaMemcpyDeviceToDevice, st));
        TCHECK(cudaMemcpyAsync(n2.tcnt, nd.tcnt, end * sizeof(int), cudaMemcpyDeviceToDevice, st));
        nd = n2;
        cap = c2;
      }
      if (nsplit > 0)
        k_children<<<(8 * cnt + 255) / 256, 256, 0, st>>>(nd, beg, end, flag, pre, skey, tkey, nlev);
      level++;
      beg = end;
      end = (int)need;
      level_beg.push_back(beg);
    }
    const int nn = end;
    t.nnodes = nn;
    // ---- geometry, tags
    int* tag = dnew<int>(nn, owned);
    double* center = dnew<double>(3 * (size_t)nn, owned);
    double* radius = dnew<double>(nn, owned);
    k_geom<<<(nn + 255) / 256, 256, 0, st>>>(nd, nn, ll[0], ll[1], ll[2], rad, tag, center, radius);
    // ---- lists: count, scan, fill, sort
    ListOut lo{};
    for (int l = 0; l < 4; l++) lo.cnt[l] = dnew<int>(nn, owned);
    k_lists<false><<<(nn + 127) / 128, 128, 0, st>>>(nd, tag, nn, lo);
    long long* ptr[4];
    for (int l = 0; l < 4; l++) {
      ptr[l] = dnew<long long>((size_t)nn + 1, owned);
      k_scan_excl64<<<1, 1024, 0, st>>>(lo.cnt[l], ptr[l], nn);
    }
    long long tot[4];
    for (int l = 0; l < 4; l++) TCHECK(cudaMemcpyAsync(&tot[l], ptr[l] + nn, sizeof(long long), cudaMemcpyDeviceToHost, st));
    TCHECK(cudaStreamSynchronize(st));
    for (int l = 0; l < 4; l++) {
      lo.ptr[l] = ptr[l];
      lo.idx[l] = dnew<int>((size_t)tot[l], owned);
    }
    k_lists<true><<<(nn + 127) / 128, 128, 0, st>>>(nd, tag, nn, lo);
    // U (descent leaves, then the sorted coarser nodes and the node itself)
    // and W (descent nodes) need sorting; V and X are written sorted
    k_sort_segments<<<(nn + 127) / 128, 128, 0, st>>>(ptr[0], lo.idx[0], nn);
    k_sort_segments<<<(nn + 127) / 128, 128, 0, st>>>(ptr[2], lo.idx[2], nn);
    // ---- back to the host Tree
    d2h(t.par, nd.par, nn, st);
    d2h(t.chd, nd.chd, nn, st);
    d2h(t.depth, nd.depth, nn, st);
    d2h(t.path, nd.path, 3 * (size_t)nn, st);
    d2h(t.sbeg, nd.sbeg, nn, st);
    d2h(t.scnt, nd.scnt, nn, st);
    d2h(t.tbeg, nd.tbeg, nn, st);
    d2h(t.tcnt, nd.tcnt, nn, st);
    d2h(t.tag, tag, nn, st);
    d2h(t.center, center, 3 * (size_t)nn, st);
    d2h(t.radius, radius, nn, st);
    for (int l = 0; l < 4; l++) {
      std::vector<long long> p;
      d2h(p, ptr[l], (size_t)nn + 1, st);
      d2h(t.lists[l].idx, lo.idx[l], (size_t)tot[l], st);
      TCHECK(cudaStreamSynchronize(st));
      t.lists[l].ptr.assign(p.begin(), p.end());
    }
    TCHECK(cudaStreamSynchronize(st));
    t.maxdepth = 0;
    for (int g = 0; g < nn; g++) t.maxdepth = std::max(t.maxdepth, t.depth[g]);
    level_beg.resize(t.maxdepth + 2);
    level_beg[t.maxdepth + 1] = nn;
    t.level_beg = level_beg;
  } catch (const DevErr& e) {
    if (err) *err = std::string(e.where) + ": " + cudaGetErrorString(e.e);
    cudaGetLastError();
    rc = 4;
  } catch (int code) {
    rc = code;
  }
  if (st) cudaStreamSynchronize(st);
  for (void* p : owned) cudaFree(p);
  if (st) cudaStreamDestroy(st);
  return rc;
}

}  // namespace kifmm
