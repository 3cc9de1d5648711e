// Point <-> point and point <-> surface evaluation passes.
//
//   k_s2m   S2M  : leaf sources -> its upward check surface      (SE2UC_dgemv, fmm3d/fmm3d.cpp:62-71)
//   k_s2l   S2L  : X-list leaf sources -> downward check surface  (SE2DC_dgemv, fmm3d/fmm3d.cpp:73-82)
//   k_leaf  near : U list + direct W/X (SE2TC_dgemv, fmm3d/fmm3d.cpp:35-60), M2T from W-list
//                  upward equivalent surfaces (UE2TC_dgemv, :114-141) and L2T from the leaf's own
//                  downward equivalent surface (DE2TC_dgemv, :84-112), fused into one pass that
//                  writes each target once.
//   k_direct     : FP64 direct sum (Dense3d::eval, fmm3d/dense3d.cpp:38-57).
//
// One CTA per work node.  Sources are staged through shared memory in tiles
// and every target accumulates in registers; when a node has few targets the
// CTA's threads split the source tile among several groups per target and
// reduce through shared memory at the end.  Positions are stored relative to
// the centre of their leaf and re-centred on the target node's centre while
// staging, so FP32 differences lose no more than the node size's precision.
#include "kernels_common.cuh"
#include "launch.hpp"

namespace kifmm {

namespace {

constexpr int P2P_THREADS = 128;
constexpr int TILE = 256;

template <typename T, int SDMAX>
struct Tile {
  T x[TILE], y[TILE], z[TILE];
  T nx[TILE], ny[TILE], nz[TILE];
  T f[TILE * SDMAX];
};

template <typename T, int TDMAX>
struct Red {
  T v[P2P_THREADS * TDMAX];
};

// Packed source tile: p[j] = (x, y, z, first density component); further
// density components in f (SD-1 per point) and normals in n (double layer).
// A single-dof single-layer interaction then reads one 16-byte (FP32) word.
template <typename T>
struct P4 {
  T x, y, z, w;
};

template <typename T>
struct PTile {
  P4<T> p[TILE];
  T f[TILE * 3];
  T n[TILE * 3];
};

template <typename T, int KT>
__device__ __forceinline__ void accumulate_ptile(const PTile<T>& t, int cnt, int j0, int jstep, T px, T py, T pz,
                                                 T* acc, const KConst<T>& kc) {
  constexpr int SD = KTraits<KT>::SD;
  constexpr bool DL = KTraits<KT>::DL;
  const int rounds = j0 < cnt ? (cnt - j0 + jstep - 1) / jstep : 0;
  if constexpr (KT == 111) {  // sum f / r, times 1/(4 pi) once
    T s1 = T(0);
#pragma unroll 4
    for (int r = 0; r < rounds; r++) {
      const P4<T> s = t.p[j0 + r * jstep];
      const T x = px - s.x, y = py - s.y, z = pz - s.z;
      const T r2 = x * x + y * y + z * z;
      const T ri = (r2 >= T(1e-16)) ? rsqrt_t(r2) : T(0);
      s1 += ri * s.w;
    }
    acc[0] += kc.c0 * s1;
  } else {
#pragma unroll 4
    for (int r = 0; r < rounds; r++) {
      const int j = j0 + r * jstep;
      const P4<T> s = t.p[j];
      T f[SD];
      f[0] = s.w;
#pragma unroll
      for (int k = 1; k < SD; k++) f[k] = t.f[j * (SD - 1) + k - 1];
      T nrm[3];
      if constexpr (DL) {
        nrm[0] = t.n[3 * j];
        nrm[1] = t.n[3 * j + 1];
        nrm[2] = t.n[3 * j + 2];
      }
      keval<KT, T>(px - s.x, py - s.y, pz - s.z, nrm, f, acc, kc);
    }
  }
}

// writes point k of the tile
template <typename T, int SD, bool DL>
__device__ __forceinline__ void put_point(PTile<T>& t, int k, T x, T y, T z, const T* f, const T* nrm) {
  t.p[k] = P4<T>{x, y, z, f[0]};
#pragma unroll
  for (int s = 1; s < SD; s++) t.f[k * (SD - 1) + s - 1] = f[s];
  if constexpr (DL) {
    t.n[3 * k] = nrm[0];
    t.n[3 * k + 1] = nrm[1];
    t.n[3 * k + 2] = nrm[2];
  }
}

__device__ __forceinline__ int group_size(int nt) {
  int g = ((nt + 31) / 32) * 32;
  return g > P2P_THREADS ? P2P_THREADS : (g < 32 ? 32 : g);
}

// Stages points [b, b+cnt) of a source leaf (local coords + shift) into the tile.
template <typename T, int SD, bool DL>
__device__ __forceinline__ void stage_points(Tile<T, 4>& t, const P2PArgs<T>& a, int b, int cnt, T shx, T shy,
                                             T shz, int rhs) {
  for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
    int p = b + j;
    t.x[j] = a.sx[p] + shx;
    t.y[j] = a.sy[p] + shy;
    t.z[j] = a.sz[p] + shz;
    if constexpr (DL) {
      t.nx[j] = a.snx[p];
      t.ny[j] = a.sny[p];
      t.nz[j] = a.snz[p];
    }
#pragma unroll
    for (int s = 0; s < SD; s++) t.f[j * SD + s] = a.sden[(size_t)rhs * a.ns * SD + (size_t)p * SD + s];
  }
}

// Stages `cnt` points of a surface grid (unit * rad + shift) with densities den[k*SD + s].
template <typename T, int SD>
__device__ __forceinline__ void stage_surface(Tile<T, 4>& t, const T* unit, int k0, int cnt, T rad, T shx, T shy,
                                              T shz, const T* den) {
  for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
    int k = k0 + j;
    t.x[j] = unit[3 * k] * rad + shx;
    t.y[j] = unit[3 * k + 1] * rad + shy;
    t.z[j] = unit[3 * k + 2] * rad + shz;
#pragma unroll
    for (int s = 0; s < SD; s++) t.f[j * SD + s] = den[(size_t)k * SD + s];
  }
}

template <typename T, int KT>
__device__ __forceinline__ void accumulate_tile(const Tile<T, 4>& t, int cnt, int j0, int jstep, T px, T py, T pz,
                                                T* acc, const KConst<T>& kc) {
  constexpr int SD = KTraits<KT>::SD;
  for (int j = j0; j < cnt; j += jstep) {
    T nrm[3];
    if constexpr (KTraits<KT>::DL) {
      nrm[0] = t.nx[j];
      nrm[1] = t.ny[j];
      nrm[2] = t.nz[j];
    }
    keval<KT, T>(px - t.x[j], py - t.y[j], pz - t.z[j], nrm, &t.f[j * SD], acc, kc);
  }
}

template <typename T, int TD>
__device__ __forceinline__ void reduce_and_store(Red<T, 4>& red, const T* acc, int G, int nsplit, bool valid,
                                                 T* out, bool add) {
  int slot = threadIdx.x % G, sg = threadIdx.x / G;
  if (sg < nsplit) {
#pragma unroll
    for (int d = 0; d < TD; d++) red.v[(sg * G + slot) * TD + d] = acc[d];
  }
  __syncthreads();
  if (sg == 0 && valid) {
#pragma unroll
    for (int d = 0; d < TD; d++) {
      T s = red.v[slot * TD + d];
      for (int q = 1; q < nsplit; q++) s += red.v[(q * G + slot) * TD + d];
      if (add)
        out[d] += s;
      else
        out[d] = s;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Each thread owns up to S2M_R upward check points (tid, tid + 128, ...), so a
// staged source feeds all of them; the leaf's sources are staged once per tile.
constexpr int S2M_R = 4;  // |UC| <= 488 (np = 8) <= 4 x 128

template <typename T, int KT>
__global__ void __launch_bounds__(P2P_THREADS) k_s2m(P2PArgs<T> a, const int* work, int nwork, int rhs) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  constexpr bool DL = KTraits<KT>::DL;
  __shared__ PTile<T> tile;
  const int g = work[blockIdx.x];
  const T rad = (T)a.radius[g];
  const int nt = a.nuc;
  const int sb = a.sbeg[g], sc = a.scnt[g];
  T px[S2M_R], py[S2M_R], pz[S2M_R], acc[S2M_R][4];
#pragma unroll
  for (int r = 0; r < S2M_R; r++) {
    const int ti = threadIdx.x + r * P2P_THREADS;
    px[r] = py[r] = pz[r] = T(0);
    if (ti < nt) {
      px[r] = a.uc_unit[3 * ti] * rad;
      py[r] = a.uc_unit[3 * ti + 1] * rad;
      pz[r] = a.uc_unit[3 * ti + 2] * rad;
    }
#pragma unroll
    for (int d = 0; d < 4; d++) acc[r][d] = T(0);
  }
  const T* den = a.sden + (size_t)rhs * a.ns * SD;
  for (int c0 = 0; c0 < sc; c0 += TILE) {
    const int cnt = min(TILE, sc - c0);
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      const int p = sb + c0 + j;
      T f[SD], nrm[3] = {T(0), T(0), T(0)};
#pragma unroll
      for (int s = 0; s < SD; s++) f[s] = den[(size_t)p * SD + s];
      if constexpr (DL) {
        nrm[0] = a.snx[p];
        nrm[1] = a.sny[p];
        nrm[2] = a.snz[p];
      }
      put_point<T, SD, DL>(tile, j, a.sx[p], a.sy[p], a.sz[p], f, nrm);
    }
    __syncthreads();
    for (int j = 0; j < cnt; j++) {  // one staged source, every check point of this thread
      const P4<T> sp = tile.p[j];
      T f[SD];
      f[0] = sp.w;
#pragma unroll
      for (int k = 1; k < SD; k++) f[k] = tile.f[j * (SD - 1) + k - 1];
      T nrm[3];
      if constexpr (DL) {
        nrm[0] = tile.n[3 * j];
        nrm[1] = tile.n[3 * j + 1];
        nrm[2] = tile.n[3 * j + 2];
      }
#pragma unroll
      for (int r = 0; r < S2M_R; r++)
        if (threadIdx.x + r * P2P_THREADS < nt) keval<KT, T>(px[r] - sp.x, py[r] - sp.y, pz[r] - sp.z, nrm, f, acc[r], a.ku);
    }
  }
  T* outbase = a.supcval + (size_t)g * a.nuc * TD;
#pragma unroll
  for (int r = 0; r < S2M_R; r++) {
    const int ti = threadIdx.x + r * P2P_THREADS;
    if (ti < nt)
#pragma unroll
      for (int d = 0; d < TD; d++) outbase[(size_t)ti * TD + d] = acc[r][d];
  }
}

template <typename T, int KT>
__global__ void __launch_bounds__(P2P_THREADS) k_s2l(P2PArgs<T> a, const int* work, const int64_t* ptr,
                                                      const int* idx, int nwork, int rhs) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  constexpr bool DL = KTraits<KT>::DL;
  __shared__ Tile<T, 4> tile;
  __shared__ Red<T, 4> red;
  int w = blockIdx.x;
  int g = work[w];
  T rad = (T)a.radius[g];
  double cx = a.center[3 * g], cy = a.center[3 * g + 1], cz = a.center[3 * g + 2];
  int nt = a.nsurf;
  int G = group_size(nt), nsplit = P2P_THREADS / G;
  int slot = threadIdx.x % G, sg = threadIdx.x / G;
  T* outbase = a.tdncval + (size_t)g * a.nsurf * TD;
  for (int tb = 0; tb < nt; tb += G) {
    int ti = tb + slot;
    bool valid = ti < nt && sg < nsplit;
    T px = 0, py = 0, pz = 0;
    if (valid) {
      px = a.dc_unit[3 * ti] * rad;
      py = a.dc_unit[3 * ti + 1] * rad;
      pz = a.dc_unit[3 * ti + 2] * rad;
    }
    T acc[4] = {0, 0, 0, 0};
    for (int64_t e = ptr[w]; e < ptr[w + 1]; e++) {
      int s = idx[e];
      T shx = (T)(a.center[3 * s] - cx), shy = (T)(a.center[3 * s + 1] - cy), shz = (T)(a.center[3 * s + 2] - cz);
      int sb = a.sbeg[s], sc = a.scnt[s];
      for (int c0 = 0; c0 < sc; c0 += TILE) {
        int cnt = min(TILE, sc - c0);
        __syncthreads();
        stage_points<T, SD, DL>(tile, a, sb + c0, cnt, shx, shy, shz, rhs);
        __syncthreads();
        if (valid) accumulate_tile<T, KT>(tile, cnt, sg, nsplit, px, py, pz, acc, a.ku);
      }
    }
    reduce_and_store<T, TD>(red, acc, G, nsplit, ti < nt, outbase + (size_t)ti * TD, true);
  }
}

// Segment table of the sources a CTA stages: a run of point leaves or of
// surface grids, flattened so that one shared-memory tile can span many
// small segments (leaves average a dozen points at ptsmax=64, so staging one
// leaf per barrier pair would leave the CTA mostly waiting).
constexpr int SEGS = 64;

template <typename T>
struct Segs {
  int beg[SEGS];        // first sorted point (point segments) or node id (surface segments)
  int pre[SEGS + 1];    // prefix sums of the segment sizes
  T shx[SEGS], shy[SEGS], shz[SEGS], rad[SEGS];
  const T* unit[SEGS];  // surface grid (surface segments)
  const T* den[SEGS];   // surface densities (surface segments)
};

__device__ __forceinline__ int find_seg(const int* pre, int ns, int k) {
  int lo = 0, hi = ns;  // pre[lo] <= k < pre[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (pre[mid] <= k)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

template <typename T, int KT>
__global__ void __launch_bounds__(P2P_THREADS) k_leaf(P2PArgs<T> a, const int* work, const int64_t* nptr,
                                                       const int* nidx, const int64_t* mptr, const int* midx,
                                                       int nwork, int rhs) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  constexpr bool DL = KTraits<KT>::DL;
  constexpr int MM = KTraits<KT>::MM;
  constexpr int SDM = KTraits<MM>::SD;
  __shared__ PTile<T> tile;
  __shared__ Red<T, 4> red;
  __shared__ Segs<T> seg;
  const int w = blockIdx.x;
  const int g = work[w];
  const double cx = a.center[3 * g], cy = a.center[3 * g + 1], cz = a.center[3 * g + 2];
  const T rad = (T)a.radius[g];
  const int tb0 = a.tbeg[g], nt = a.tcnt[g];
  // thread -> (target slot, source split): every thread of the CTA is busy
  const int G = nt < P2P_THREADS ? (nt > 0 ? nt : 1) : P2P_THREADS;
  const int nsplit = P2P_THREADS / G;
  const int slot = threadIdx.x % G, sg = threadIdx.x / G;
  const bool l2t = a.depth[g] >= 2;
  T* outbase = a.tval + (size_t)rhs * a.nt * TD;
  const T* den = a.sden + (size_t)rhs * a.ns * SD;
  const int64_t nb = nptr[w], ne = nptr[w + 1];
  const int64_t mb = mptr[w], me = mptr[w + 1];
  const int nsurf = a.nsurf;
  const int nsurf_segs = (int)(me - mb) + (l2t ? 1 : 0);
  for (int tb = 0; tb < nt; tb += G) {
    const int ti = tb + slot;
    const bool valid = ti < nt && sg < nsplit;
    T px = 0, py = 0, pz = 0;
    if (valid) {
      px = a.tx[tb0 + ti];
      py = a.ty[tb0 + ti];
      pz = a.tz[tb0 + ti];
    }
    T acc[4] = {0, 0, 0, 0};
    // point sources: U list, direct W and X (user kernel, with normals)
    for (int64_t c0 = nb; c0 < ne; c0 += SEGS) {
      const int nseg = (int)min((int64_t)SEGS, ne - c0);
      __syncthreads();
      if (threadIdx.x < nseg) {
        int s = nidx[c0 + threadIdx.x];
        seg.beg[threadIdx.x] = a.sbeg[s];
        seg.pre[threadIdx.x + 1] = a.scnt[s];
        seg.shx[threadIdx.x] = (T)(a.center[3 * s] - cx);
        seg.shy[threadIdx.x] = (T)(a.center[3 * s + 1] - cy);
        seg.shz[threadIdx.x] = (T)(a.center[3 * s + 2] - cz);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        seg.pre[0] = 0;
        for (int e = 0; e < nseg; e++) seg.pre[e + 1] += seg.pre[e];
      }
      __syncthreads();
      const int total = seg.pre[nseg];
      for (int k0 = 0; k0 < total; k0 += TILE) {
        const int cnt = min(TILE, total - k0);
        // one thread per staged point; its source leaf by bisection of the prefix sums
        for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
          const int k = k0 + j;
          const int e = find_seg(seg.pre, nseg, k);
          const int p = seg.beg[e] + (k - seg.pre[e]);
          T f[SD], nrm[3] = {T(0), T(0), T(0)};
#pragma unroll
          for (int s = 0; s < SD; s++) f[s] = den[(size_t)p * SD + s];
          if constexpr (DL) {
            nrm[0] = a.snx[p];
            nrm[1] = a.sny[p];
            nrm[2] = a.snz[p];
          }
          put_point<T, SD, DL>(tile, j, a.sx[p] + seg.shx[e], a.sy[p] + seg.shy[e], a.sz[p] + seg.shz[e], f, nrm);
        }
        __syncthreads();
        if (valid) accumulate_ptile<T, KT>(tile, cnt, sg, nsplit, px, py, pz, acc, a.ku);
        __syncthreads();
      }
    }
    // surface sources: W-list upward equivalent surfaces (M2T) and the leaf's
    // own downward equivalent surface (L2T), equivalent kernel
    for (int c0 = 0; c0 < nsurf_segs; c0 += SEGS) {
      const int nseg = min(SEGS, nsurf_segs - c0);
      __syncthreads();
      if (threadIdx.x < nseg) {
        int e = c0 + threadIdx.x;
        if (e < (int)(me - mb)) {
          int s = midx[mb + e];
          seg.shx[threadIdx.x] = (T)(a.center[3 * s] - cx);
          seg.shy[threadIdx.x] = (T)(a.center[3 * s + 1] - cy);
          seg.shz[threadIdx.x] = (T)(a.center[3 * s + 2] - cz);
          seg.rad[threadIdx.x] = (T)a.radius[s];
          seg.unit[threadIdx.x] = a.ue_unit;
          seg.den[threadIdx.x] = a.supeden + (size_t)s * nsurf * SDM;
        } else {
          seg.shx[threadIdx.x] = seg.shy[threadIdx.x] = seg.shz[threadIdx.x] = T(0);
          seg.rad[threadIdx.x] = rad;
          seg.unit[threadIdx.x] = a.de_unit;
          seg.den[threadIdx.x] = a.tdneden + (size_t)g * nsurf * SDM;
        }
      }
      __syncthreads();
      const int total = nseg * nsurf;
      for (int k0 = 0; k0 < total; k0 += TILE) {
        const int cnt = min(TILE, total - k0);
        for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
          const int k = k0 + j;
          const int e = k / nsurf, m = k - e * nsurf;
          const T* u = seg.unit[e];
          const T* sd = seg.den[e];
          const T r = seg.rad[e];
          T f[SDM];
#pragma unroll
          for (int s = 0; s < SDM; s++) f[s] = sd[(size_t)m * SDM + s];
          put_point<T, SDM, false>(tile, j, u[3 * m] * r + seg.shx[e], u[3 * m + 1] * r + seg.shy[e],
                                   u[3 * m + 2] * r + seg.shz[e], f, nullptr);
        }
        __syncthreads();
        if (valid) accumulate_ptile<T, MM>(tile, cnt, sg, nsplit, px, py, pz, acc, a.km);
        __syncthreads();
      }
    }
    reduce_and_store<T, TD>(red, acc, G, nsplit, ti < nt, outbase + (size_t)(tb0 + ti) * TD, false);
  }
}

// FP64 direct sum over all sources, absolute coordinates (3 x n interleaved).
template <int KT>
__global__ void __launch_bounds__(P2P_THREADS) k_direct(const double* spos, const double* snor, const double* sden,
                                                         int ns, const double* tpos, int nt, double* out,
                                                         KConst<double> kc) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  __shared__ double sx[TILE], sy[TILE], sz[TILE], nx[TILE], ny[TILE], nz[TILE], f[TILE * 4];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double px = 0, py = 0, pz = 0;
  if (t < nt) {
    px = tpos[3 * t];
    py = tpos[3 * t + 1];
    pz = tpos[3 * t + 2];
  }
  double acc[4] = {0, 0, 0, 0};
  for (int c0 = 0; c0 < ns; c0 += TILE) {
    int cnt = min(TILE, ns - c0);
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      int p = c0 + j;
      sx[j] = spos[3 * p];
      sy[j] = spos[3 * p + 1];
      sz[j] = spos[3 * p + 2];
      nx[j] = snor[3 * p];
      ny[j] = snor[3 * p + 1];
      nz[j] = snor[3 * p + 2];
      for (int s = 0; s < SD; s++) f[j * SD + s] = sden[(size_t)p * SD + s];
    }
    __syncthreads();
    if (t < nt)
      for (int j = 0; j < cnt; j++) {
        double nrm[3] = {nx[j], ny[j], nz[j]};
        keval<KT, double>(px - sx[j], py - sy[j], pz - sz[j], nrm, &f[j * SD], acc, kc);
      }
  }
  if (t < nt)
    for (int d = 0; d < TD; d++) out[(size_t)t * TD + d] = acc[d];
}

// sden_sorted[r][i][s] = srcden[r][perm[i]][s]
template <typename T>
__global__ void k_scatter_den(const double* srcden, const int* perm, int ns, int sd, int nrhs, T* out) {
  size_t n = (size_t)ns * sd * nrhs;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    size_t r = e / ((size_t)ns * sd);
    size_t rem = e % ((size_t)ns * sd);
    int i = (int)(rem / sd), s = (int)(rem % sd);
    out[e] = (T)srcden[r * ns * sd + (size_t)perm[i] * sd + s];
  }
}

// trgval[r][perm[i]][t] = tval[r][i][t]
template <typename T>
__global__ void k_gather_val(const T* tval, const int* perm, int nt, int td, int nrhs, double* trgval) {
  size_t n = (size_t)nt * td * nrhs;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    size_t r = e / ((size_t)nt * td);
    size_t rem = e % ((size_t)nt * td);
    int i = (int)(rem / td), d = (int)(rem % td);
    trgval[r * nt * td + (size_t)perm[i] * td + d] = (double)tval[e];
  }
}

template <typename T, int KT>
void launch_p2p_kt(const P2PArgs<T>& a, const P2PWork& w, int which, int rhs, cudaStream_t st) {
  switch (which) {
    case P2P_S2M:
      if (w.n) k_s2m<T, KT><<<w.n, P2P_THREADS, 0, st>>>(a, w.work, w.n, rhs);
      break;
    case P2P_S2L:
      if (w.n) k_s2l<T, KT><<<w.n, P2P_THREADS, 0, st>>>(a, w.work, w.ptr, w.idx, w.n, rhs);
      break;
    case P2P_LEAF:
      if (w.n) k_leaf<T, KT><<<w.n, P2P_THREADS, 0, st>>>(a, w.work, w.ptr, w.idx, w.ptr2, w.idx2, w.n, rhs);
      break;
  }
}

}  // namespace

template <typename T>
void launch_p2p(int kt, const P2PArgs<T>& a, const P2PWork& w, int which, int rhs, cudaStream_t st) {
  switch (kt) {
    case 111: launch_p2p_kt<T, 111>(a, w, which, rhs, st); break;
    case 121: launch_p2p_kt<T, 121>(a, w, which, rhs, st); break;
    case 311: launch_p2p_kt<T, 311>(a, w, which, rhs, st); break;
    case 312: launch_p2p_kt<T, 312>(a, w, which, rhs, st); break;
    case 321: launch_p2p_kt<T, 321>(a, w, which, rhs, st); break;
    case 322: launch_p2p_kt<T, 322>(a, w, which, rhs, st); break;
    case 511: launch_p2p_kt<T, 511>(a, w, which, rhs, st); break;
    case 521: launch_p2p_kt<T, 521>(a, w, which, rhs, st); break;
  }
}
template void launch_p2p<double>(int, const P2PArgs<double>&, const P2PWork&, int, int, cudaStream_t);
template void launch_p2p<float>(int, const P2PArgs<float>&, const P2PWork&, int, int, cudaStream_t);

void launch_direct(int kt, const double* spos, const double* snor, const double* sden, int ns, const double* tpos,
                   int nt, double* out, const double* kc3, cudaStream_t st) {
  KConst<double> kc{kc3[0], kc3[1], kc3[2]};
  int grid = (nt + P2P_THREADS - 1) / P2P_THREADS;
  if (grid == 0) return;
  switch (kt) {
    case 111: k_direct<111><<<grid, P2P_THREADS, 0, st>>>(spos, snor, sden, ns, tpos, nt, out, kc); break;
    case 121: k_direct<121><<<grid, P2P_THREADS, 0, st>>>(spos, snor, sden, ns, tpos, nt, out, kc); break;
    case 311: k_direct<311><<<grid, P2P_THREADS, 0, st>>>(spos, snor, sden, ns, tpos, nt, out, kc); break;
    case 312: k_direct<312><<<grid, P2P_THREADS, 0, st>>>(spos, snor, sden, ns, tpos, nt, out, kc); break;
    case 321: k_direct<321><<<grid, P2P_THREADS, 0, st>>>(spos, snor, sden, ns, tpos, nt, out, kc); break;
    case 322: k_direct<322><<<grid, P2P_THREADS, 0, st>>>(spos, snor, sden, ns, tpos, nt, out, kc); break;
    case 511: k_direct<511><<<grid, P2P_THREADS, 0, st>>>(spos, snor, sden, ns, tpos, nt, out, kc); break;
    case 521: k_direct<521><<<grid, P2P_THREADS, 0, st>>>(spos, snor, sden, ns, tpos, nt, out, kc); break;
  }
}

template <typename T>
void launch_scatter_den(const double* srcden, const int* perm, int ns, int sd, int nrhs, T* out, cudaStream_t st) {
  size_t n = (size_t)ns * sd * nrhs;
  if (!n) return;
  int grid = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_scatter_den<T><<<grid, 256, 0, st>>>(srcden, perm, ns, sd, nrhs, out);
}
template void launch_scatter_den<double>(const double*, const int*, int, int, int, double*, cudaStream_t);
template void launch_scatter_den<float>(const double*, const int*, int, int, int, float*, cudaStream_t);

template <typename T>
void launch_gather_val(const T* tval, const int* perm, int nt, int td, int nrhs, double* trgval, cudaStream_t st) {
  size_t n = (size_t)nt * td * nrhs;
  if (!n) return;
  int grid = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_gather_val<T><<<grid, 256, 0, st>>>(tval, perm, nt, td, nrhs, trgval);
}
template void launch_gather_val<double>(const double*, const int*, int, int, int, double*, cudaStream_t);
template void launch_gather_val<float>(const float*, const int*, int, int, int, double*, cudaStream_t);

}  // namespace kifmm
