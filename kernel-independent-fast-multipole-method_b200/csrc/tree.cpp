// Host octree + interaction lists; see tree.hpp for how this relates to the
// reference's Let3d (fmm3d/let3d.cpp).
#include "tree.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <thread>

namespace kifmm {

double Tree::rad() const { return std::pow(2.0, -rootlvl); }  // Let3d::rad, fmm3d/let3d.hpp:98

namespace {

// Morton key from the reference's FP64 octant test: at depth d the point is
// compared against the centre of its depth-d ancestor, computed as
// ll + (2 rad)(path + 0.5) / 2^d (fmm3d/let3d.cpp:99, :309-318).  One 3-bit
// digit per level, x most significant (child index a*4+b*2+c, :307).
inline uint64_t point_key(const double* p, const double* ll, double rad, int nlev) {
  int path[3] = {0, 0, 0};
  uint64_t key = 0;
  for (int d = 0; d < nlev; d++) {
    double tmp = (double)(1 << d);
    int dig = 0;
    for (int a = 0; a < 3; a++) {
      double c = ll[a] + (2 * rad) * (path[a] + 0.5) / tmp;
      int b = p[a] >= c;
      path[a] = 2 * path[a] + b;
      dig = (dig << 1) | b;
    }
    key = (key << 3) | (uint64_t)dig;
  }
  return key;
}

template <class F>
void parallel_for(int n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 2048) {
    f(0, n, 0);
    return;
  }
  std::vector<std::thread> th;
  for (int i = 0; i < nthreads; i++) {
    int b = (int)((int64_t)n * i / nthreads), e = (int)((int64_t)n * (i + 1) / nthreads);
    th.emplace_back([&, b, e, i] { f(b, e, i); });
  }
  for (auto& x : th) x.join();
}

// Stable LSD radix sort of (key, id) by key over `bits` low bits.
void radix_sort(std::vector<uint64_t>& key, std::vector<int>& id, int bits) {
  size_t n = key.size();
  std::vector<uint64_t> k2(n);
  std::vector<int> i2(n);
  for (int sh = 0; sh < bits; sh += 8) {
    size_t cnt[257] = {0};
    for (size_t i = 0; i < n; i++) cnt[((key[i] >> sh) & 255) + 1]++;
    for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
    for (size_t i = 0; i < n; i++) {
      size_t dst = cnt[(key[i] >> sh) & 255]++;
      k2[dst] = key[i];
      i2[dst] = id[i];
    }
    key.swap(k2);
    id.swap(i2);
  }
}

struct ListBuilder {
  const Tree& t;
  explicit ListBuilder(const Tree& tr) : t(tr) {}

  int child(int g, int a, int b, int c) const { return t.chd[g] + a * 4 + b * 2 + c; }

  // Let3d::findgnt, fmm3d/let3d.cpp:325-337
  int findgnt(int wdepth, const int* wpath) const {
    int cur = 0;
    int left[3] = {wpath[0], wpath[1], wpath[2]};
    while (t.depth[cur] < wdepth && t.chd[cur] != -1) {
      int dif = wdepth - t.depth[cur];
      int tmp = 1 << (dif - 1);
      int ch[3];
      for (int d = 0; d < 3; d++) {
        ch[d] = left[d] / tmp;
        left[d] -= ch[d] * tmp;
      }
      cur = child(cur, ch[0], ch[1], ch[2]);
    }
    return cur;
  }

  // Let3d::adjacent, fmm3d/let3d.cpp:339-352
  bool adjacent(int me, int yo) const {
    int md = std::max(t.depth[me], t.depth[yo]);
    int merad = 1 << (md - t.depth[me]);
    int yorad = 1 << (md - t.depth[yo]);
    int rad = merad + yorad;
    int mx = 0;
    for (int d = 0; d < 3; d++) {
      int dif = std::abs((2 * t.path[3 * me + d] + 1) * merad - (2 * t.path[3 * yo + d] + 1) * yorad);
      if (dif > rad) return false;
      mx = std::max(mx, dif);
    }
    return mx == rad;
  }

  // Let3d::calgnext, fmm3d/let3d.cpp:214-281.  Appends the sorted, unique,
  // source-only lists of node g to out[0..3].
  void lists(int g, std::vector<int>* out, std::vector<int>& queue) const {
    std::vector<int> U, V, W, X;
    bool term = t.chd[g] == -1;
    if (t.par[g] != -1) {
      int pg = t.par[g];
      int maxidx = 1 << t.depth[g];
      for (int i = -2; i < 4; i++)
        for (int j = -2; j < 4; j++)
          for (int k = -2; k < 4; k++) {
            int tp[3] = {2 * t.path[3 * pg] + i, 2 * t.path[3 * pg + 1] + j, 2 * t.path[3 * pg + 2] + k};
            if (tp[0] < 0 || tp[1] < 0 || tp[2] < 0 || tp[0] >= maxidx || tp[1] >= maxidx || tp[2] >= maxidx)
              continue;
            if (tp[0] == t.path[3 * g] && tp[1] == t.path[3 * g + 1] && tp[2] == t.path[3 * g + 2]) continue;
            int res = findgnt(t.depth[g], tp);
            bool adj = adjacent(res, g);
            if (t.depth[res] < t.depth[g]) {
              if (adj) {
                if (term) U.push_back(res);
              } else {
                X.push_back(res);
              }
            }
            if (t.depth[res] == t.depth[g]) {
              if (!adj) {
                V.push_back(res);
              } else if (term) {
                queue.clear();
                queue.push_back(res);
                for (size_t qh = 0; qh < queue.size(); qh++) {
                  int f = queue[qh];
                  if (!adjacent(f, g)) {
                    W.push_back(f);
                  } else if (t.chd[f] == -1) {
                    U.push_back(f);
                  } else {
                    for (int a = 0; a < 2; a++)
                      for (int b = 0; b < 2; b++)
                        for (int c = 0; c < 2; c++) queue.push_back(child(f, a, b, c));
                  }
                }
              }
            }
          }
    }
    if (term) U.push_back(g);
    std::vector<int>* sets[4] = {&U, &V, &W, &X};
    for (int l = 0; l < 4; l++) {
      std::vector<int>& s = *sets[l];
      std::sort(s.begin(), s.end());
      s.erase(std::unique(s.begin(), s.end()), s.end());
      for (int x : s)
        if (t.tag[x] & TAG_SRC) out[l].push_back(x);
    }
  }
};

bool inside(const double* p, const double* ctr, double rad) {
  for (int d = 0; d < 3; d++)
    if (!(p[d] >= ctr[d] - rad && p[d] <= ctr[d] + rad)) return false;
  return true;
}

}  // namespace

int build_tree(Tree& t, int ns, const double* srcpos, int nt, const double* trgpos, int nthreads, std::string* err) {
  if (t.maxlevel < 1 || t.maxlevel > 21 || t.ptsmax < 0 || ns < 0 || nt < 0) {
    if (err) *err = "bad ptsmax/maxlevel (maxlevel must be in [1,21])";
    return 1;
  }
  if (nthreads < 1) nthreads = 1;
  const double rad = t.rad();
  const double ll[3] = {t.ctr[0] - rad, t.ctr[1] - rad, t.ctr[2] - rad};
  const int nlev = t.maxlevel - 1;  // deepest possible depth (fmm3d/let3d.cpp:86)

  // 1. box check + keys
  std::vector<uint64_t> skey(ns), tkey(nt);
  std::vector<int> bad(nthreads, 0);
  parallel_for(ns, nthreads, [&](int b, int e, int th) {
    for (int i = b; i < e; i++) {
      if (!inside(srcpos + 3 * (size_t)i, t.ctr, rad)) bad[th] = 1;
      skey[i] = point_key(srcpos + 3 * (size_t)i, ll, rad, nlev);
    }
  });
  parallel_for(nt, nthreads, [&](int b, int e, int th) {
    for (int i = b; i < e; i++) {
      if (!inside(trgpos + 3 * (size_t)i, t.ctr, rad)) bad[th] = 1;
      tkey[i] = point_key(trgpos + 3 * (size_t)i, ll, rad, nlev);
    }
  });
  for (int x : bad)
    if (x) {
      if (err) *err = "a point lies outside the root box";
      return 3;
    }
  t.sperm.resize(ns);
  t.tperm.resize(nt);
  for (int i = 0; i < ns; i++) t.sperm[i] = i;
  for (int i = 0; i < nt; i++) t.tperm[i] = i;
  radix_sort(skey, t.sperm, 3 * nlev);
  radix_sort(tkey, t.tperm, 3 * nlev);

  // 2. breadth-first nodes (Let3d::srcdata loop, fmm3d/let3d.cpp:80-112)
  auto clear = [&]() {
    t.depth.clear(); t.par.clear(); t.chd.clear(); t.tag.clear(); t.path.clear();
    t.sbeg.clear(); t.scnt.clear(); t.tbeg.clear(); t.tcnt.clear();
  };
  clear();
  auto add = [&](int par, int p0, int p1, int p2, int dep, int sb, int sc, int tb, int tc) {
    t.par.push_back(par); t.chd.push_back(-1); t.depth.push_back(dep); t.tag.push_back(0);
    t.path.push_back(p0); t.path.push_back(p1); t.path.push_back(p2);
    t.sbeg.push_back(sb); t.scnt.push_back(sc); t.tbeg.push_back(tb); t.tcnt.push_back(tc);
  };
  add(-1, 0, 0, 0, 0, 0, ns, 0, nt);
  t.level_beg.assign(1, 0);
  int level = 0, arrbeg = 0, arrend = 1;
  auto digit = [&](uint64_t k, int d) { return (int)((k >> (3 * (nlev - 1 - d))) & 7); };
  while (arrbeg < arrend) {
    int arrcnt = arrend;
    for (int k = arrbeg; k < arrend; k++) {
      if (t.scnt[k] > t.ptsmax && level < t.maxlevel - 1) {
        t.chd[k] = arrcnt;
        arrcnt += 8;
        int sb = t.sbeg[k], se = sb + t.scnt[k];
        int tb = t.tbeg[k], te = tb + t.tcnt[k];
        int d = t.depth[k];
        for (int o = 0; o < 8; o++) {
          int s0 = (int)(std::lower_bound(skey.begin() + sb, skey.begin() + se, o,
                                          [&](uint64_t a, int v) { return digit(a, d) < v; }) - skey.begin());
          int s1 = (int)(std::lower_bound(skey.begin() + sb, skey.begin() + se, o + 1,
                                          [&](uint64_t a, int v) { return digit(a, d) < v; }) - skey.begin());
          int t0 = (int)(std::lower_bound(tkey.begin() + tb, tkey.begin() + te, o,
                                          [&](uint64_t a, int v) { return digit(a, d) < v; }) - tkey.begin());
          int t1 = (int)(std::lower_bound(tkey.begin() + tb, tkey.begin() + te, o + 1,
                                          [&](uint64_t a, int v) { return digit(a, d) < v; }) - tkey.begin());
          int a = (o >> 2) & 1, b = (o >> 1) & 1, c = o & 1;
          add(k, 2 * t.path[3 * k] + a, 2 * t.path[3 * k + 1] + b, 2 * t.path[3 * k + 2] + c, d + 1, s0, s1 - s0,
              t0, t1 - t0);
        }
      }
    }
    level++;
    arrbeg = arrend;
    arrend = arrcnt;
    t.level_beg.push_back(arrbeg);  // first node of depth `level`
  }
  t.nnodes = (int)t.depth.size();
  t.maxdepth = 0;
  for (int g = 0; g < t.nnodes; g++) t.maxdepth = std::max(t.maxdepth, t.depth[g]);
  // level_beg has one entry per processed level + the end; trim to maxdepth+2 entries
  t.level_beg.resize(t.maxdepth + 2);
  t.level_beg[t.maxdepth + 1] = t.nnodes;

  // 3. tags (fmm3d/let3d.cpp:117-135, :184-200), geometry
  t.center.resize(3 * (size_t)t.nnodes);
  t.radius.resize(t.nnodes);
  for (int g = 0; g < t.nnodes; g++) {
    if (t.scnt[g] > 0) t.tag[g] |= TAG_SRC;
    if (t.tcnt[g] > 0) t.tag[g] |= TAG_TRG;
    double tmp = (double)(1 << t.depth[g]);
    for (int d = 0; d < 3; d++) t.center[3 * g + d] = ll[d] + (2 * rad) * (t.path[3 * g + d] + 0.5) / tmp;
    t.radius[g] = rad / tmp;
  }

  // 4. lists, in parallel over target nodes
  ListBuilder lb(t);
  std::vector<std::vector<int>> part_idx[4], part_cnt[4];
  for (int l = 0; l < 4; l++) {
    part_idx[l].assign(nthreads, {});
    part_cnt[l].assign(nthreads, {});
  }
  std::vector<int> bnds(nthreads + 1);
  for (int i = 0; i <= nthreads; i++) bnds[i] = (int)((int64_t)t.nnodes * i / nthreads);
  auto work = [&](int b, int e, int th) {
    std::vector<int> out[4], queue;
    for (int g = b; g < e; g++) {
      for (int l = 0; l < 4; l++) out[l].clear();
      if (t.tag[g] & TAG_TRG) lb.lists(g, out, queue);
      for (int l = 0; l < 4; l++) {
        part_cnt[l][th].push_back((int)out[l].size());
        part_idx[l][th].insert(part_idx[l][th].end(), out[l].begin(), out[l].end());
      }
    }
  };
  if (nthreads <= 1 || t.nnodes < 256) {
    for (int l = 0; l < 4; l++) { part_idx[l].assign(1, {}); part_cnt[l].assign(1, {}); }
    work(0, t.nnodes, 0);
    bnds = {0, t.nnodes};
  } else {
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; i++) th.emplace_back(work, bnds[i], bnds[i + 1], i);
    for (auto& x : th) x.join();
  }
  for (int l = 0; l < 4; l++) {
    Csr& c = t.lists[l];
    c.ptr.assign(t.nnodes + 1, 0);
    c.idx.clear();
    int g = 0;
    for (size_t p = 0; p < part_cnt[l].size(); p++) {
      for (int cnt : part_cnt[l][p]) {
        c.ptr[g + 1] = c.ptr[g] + cnt;
        g++;
      }
      c.idx.insert(c.idx.end(), part_idx[l][p].begin(), part_idx[l][p].end());
    }
  }
  return 0;
}

}  // namespace kifmm
