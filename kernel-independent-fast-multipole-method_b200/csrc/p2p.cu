// Point <-> point and point <-> surface evaluation passes.
//
//   k_s2m_warp   S2M  : leaf sources -> its upward check surface      (SE2UC_dgemv, fmm3d/fmm3d.cpp:62-71)
//   k_s2l        S2L  : X-list leaf sources -> downward check surface  (SE2DC_dgemv, fmm3d/fmm3d.cpp:73-82)
//   k_leaf_warp  near : U list + direct W/X (SE2TC_dgemv, fmm3d/fmm3d.cpp:35-60), M2T from W-list
//                       upward equivalent surfaces (UE2TC_dgemv, :114-141) and L2T from the leaf's own
//                       downward equivalent surface (DE2TC_dgemv, :84-112), fused into one pass that
//                       writes each target once.
//   k_direct          : FP64 direct sum (Dense3d::eval, fmm3d/dense3d.cpp:38-57).
//
// S2M and the leaf pass run one warp per leaf (see below); S2L, rare, one CTA
// per node with shared-memory tiles.  Every target accumulates in registers.
// Positions are stored relative to the centre of their leaf and re-centred on
// the target node's centre while staging, so FP32 differences lose no more
// than the node size's precision.
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

// Packed staged source: (x, y, z, first density component); a single-dof
// single-layer interaction then reads one 16-byte (FP32) word.
template <typename T>
struct P4 {
  T x, y, z, w;
};

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

// ---------------------------------------------------------------------------
// Warp-per-leaf forms.  A warp owns one leaf, stages its sources 32 at a time
// in a private slice of shared memory and synchronises with __syncwarp only,
// so the other warps of the SM keep issuing while it waits on its loads.
constexpr int WP_WARPS = 8;  // warps per CTA

template <typename T>
struct WarpSrc {  // one staged batch of 32 sources
  P4<T> p[32];
  T f[32 * 3];
  T n[32 * 3];
};

template <typename T>
struct WarpSrc64 {  // one staged batch of 64 sources
  P4<T> p[64];
  T f[64 * 3];
  T n[64 * 3];
};

// Single-dof Laplace sums in FP32 run on packed f32x2 arithmetic, two
// sources per instruction: the staged batch is then pair-interleaved,
// pair q = sources 2q, 2q + 1 as {x0, x1, y0, y1} {z0, z1, w0, w1}, so one
// pair is two 16-byte shared loads already in packed-register order.
template <typename T>
__device__ __forceinline__ void stage_src(WarpSrc64<T>& w, int j, P4<T> v, bool paired) {
  if (!paired) {
    w.p[j] = v;
    return;
  }
  T* q = reinterpret_cast<T*>(w.p) + 8 * (j >> 1) + (j & 1);
  q[0] = v.x;
  q[2] = v.y;
  q[4] = v.z;
  q[6] = v.w;
}

__device__ __forceinline__ unsigned long long pk2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void upk2(unsigned long long v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// sum over the pairs q = sg, sg + nsplit, ... < npairs of w / |t - s| (the
// 1e-16 cut-off as in keval), for target t = (px, py, pz)
__device__ __forceinline__ float lap_pairs(const WarpSrc64<float>& w, float px, float py, float pz, int sg,
                                           int nsplit, int npairs) {
  const float4* wp = reinterpret_cast<const float4*>(w.p);
  const unsigned long long PX = pk2(px, px), PY = pk2(py, py), PZ = pk2(pz, pz);
  unsigned long long S = pk2(0.f, 0.f);
  const int rounds = sg < npairs ? (npairs - sg + nsplit - 1) / nsplit : 0;
#pragma unroll 8
  for (int r = 0; r < rounds; r++) {
    const int q = sg + r * nsplit;
    const float4 A = wp[2 * q], B = wp[2 * q + 1];
    const unsigned long long X = sub2(PX, pk2(A.x, A.y)), Y = sub2(PY, pk2(A.z, A.w)), Z = sub2(PZ, pk2(B.x, B.y));
    unsigned long long R2 = mul2(X, X);
    R2 = fma2(Y, Y, R2);
    R2 = fma2(Z, Z, R2);
    float r2a, r2b;
    upk2(R2, r2a, r2b);
    const float ria = (r2a >= 1e-16f) ? rsqrt_t(r2a) : 0.f, rib = (r2b >= 1e-16f) ? rsqrt_t(r2b) : 0.f;
    S = fma2(pk2(ria, rib), pk2(B.z, B.w), S);
  }
  float sa, sb;
  upk2(S, sa, sb);
  return sa + sb;
}

// S2M: lane l owns upward check points l, l + 32, ... (R rounds); every
// staged source (a broadcast load) updates all of them.
template <typename T, int KT, int R>
__global__ void __launch_bounds__(32 * WP_WARPS) k_s2m_warp(P2PArgs<T> a, const int* work, int nwork, int rhs) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  constexpr bool DL = KTraits<KT>::DL;
  __shared__ WarpSrc<T> ws[WP_WARPS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSrc<T>& w = ws[warp];
  const T* den = a.sden + (size_t)rhs * a.ns * SD;
  const int nt = a.nuc;
  for (int wi = blockIdx.x * WP_WARPS + warp; wi < nwork; wi += gridDim.x * WP_WARPS) {
    const int g = work[wi];
    const T rad = (T)a.radius[g];
    const int sb = a.sbeg[g], sc = a.scnt[g];
    T px[R], py[R], pz[R], acc[R][TD];
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int ti = lane + 32 * r;
      px[r] = py[r] = pz[r] = T(0);
      if (ti < nt) {
        px[r] = a.uc_unit[3 * ti] * rad;
        py[r] = a.uc_unit[3 * ti + 1] * rad;
        pz[r] = a.uc_unit[3 * ti + 2] * rad;
      }
#pragma unroll
      for (int d = 0; d < TD; d++) acc[r][d] = T(0);
    }
    // FP32 Laplace: packed f32x2 sums over pairs of this lane's check points
    constexpr bool PACKED = KT == 111 && sizeof(T) == 4;
    unsigned long long PX[R / 2 > 0 ? R / 2 : 1], PY[R / 2 > 0 ? R / 2 : 1], PZ[R / 2 > 0 ? R / 2 : 1],
        SP[R / 2 > 0 ? R / 2 : 1];
    float s_last = 0.f;
    if constexpr (PACKED) {
#pragma unroll
      for (int rp = 0; rp < R / 2; rp++) {
        PX[rp] = pk2(px[2 * rp], px[2 * rp + 1]);
        PY[rp] = pk2(py[2 * rp], py[2 * rp + 1]);
        PZ[rp] = pk2(pz[2 * rp], pz[2 * rp + 1]);
        SP[rp] = pk2(0.f, 0.f);
      }
    }
    for (int c0 = 0; c0 < sc; c0 += 32) {
      const int cnt = min(32, sc - c0);
      __syncwarp();
      if (lane < cnt) {
        const int p = sb + c0 + lane;
        T f[SD], nrm[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int s = 0; s < SD; s++) f[s] = den[(size_t)p * SD + s];
        if constexpr (DL) {
          nrm[0] = a.snx[p];
          nrm[1] = a.sny[p];
          nrm[2] = a.snz[p];
        }
        w.p[lane] = P4<T>{a.sx[p], a.sy[p], a.sz[p], f[0]};
#pragma unroll
        for (int s = 1; s < SD; s++) w.f[lane * (SD - 1) + s - 1] = f[s];
        if constexpr (DL) {
          w.n[3 * lane] = nrm[0];
          w.n[3 * lane + 1] = nrm[1];
          w.n[3 * lane + 2] = nrm[2];
        }
      }
      __syncwarp();
      for (int j = 0; j < cnt; j++) {
        const P4<T> sp = w.p[j];
        T f[SD];
        f[0] = sp.w;
#pragma unroll
        for (int k = 1; k < SD; k++) f[k] = w.f[j * (SD - 1) + k - 1];
        T nrm[3];
        if constexpr (DL) {
          nrm[0] = w.n[3 * j];
          nrm[1] = w.n[3 * j + 1];
          nrm[2] = w.n[3 * j + 2];
        }
        if constexpr (PACKED) {
          // check points 2 rp, 2 rp + 1 as one f32x2 pair; an odd last round scalar
          const unsigned long long SX = pk2(sp.x, sp.x), SY = pk2(sp.y, sp.y), SZ = pk2(sp.z, sp.z),
                                   SW = pk2(sp.w, sp.w);
#pragma unroll
          for (int rp = 0; rp < R / 2; rp++) {
            if (64 * rp >= nt) break;
            const unsigned long long X = sub2(PX[rp], SX), Y = sub2(PY[rp], SY), Z = sub2(PZ[rp], SZ);
            unsigned long long R2 = mul2(X, X);
            R2 = fma2(Y, Y, R2);
            R2 = fma2(Z, Z, R2);
            float r2a, r2b;
            upk2(R2, r2a, r2b);
            const float ria = (r2a >= 1e-16f) ? rsqrt_t(r2a) : 0.f, rib = (r2b >= 1e-16f) ? rsqrt_t(r2b) : 0.f;
            SP[rp] = fma2(pk2(ria, rib), SW, SP[rp]);
          }
          if constexpr (R % 2 == 1) {
            if (32 * (R - 1) < nt) {
              const float x = px[R - 1] - sp.x, y = py[R - 1] - sp.y, z = pz[R - 1] - sp.z;
              const float r2 = x * x + y * y + z * z;
              s_last += ((r2 >= 1e-16f) ? rsqrt_t(r2) : 0.f) * sp.w;
            }
          }
        } else {
#pragma unroll
          for (int r = 0; r < R; r++)
            if (32 * r < nt) keval<KT, T>(px[r] - sp.x, py[r] - sp.y, pz[r] - sp.z, nrm, f, acc[r], a.ku);
        }
      }
    }
    if constexpr (PACKED) {  // sum f / r, times 1/(4 pi) once
#pragma unroll
      for (int rp = 0; rp < R / 2; rp++) {
        float sa, sb;
        upk2(SP[rp], sa, sb);
        acc[2 * rp][0] = a.ku.c0 * sa;
        acc[2 * rp + 1][0] = a.ku.c0 * sb;
      }
      if constexpr (R % 2 == 1) acc[R - 1][0] = a.ku.c0 * s_last;
    }
    T* outbase = a.supcval + (size_t)g * nt * TD;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int ti = lane + 32 * r;
      if (ti < nt)
#pragma unroll
        for (int d = 0; d < TD; d++) outbase[(size_t)ti * TD + d] = acc[r][d];
    }
  }
}

// Leaf pass: the leaf's targets in rounds of up to 32; in a round lane =
// (target slot, source split) with G = the power of two >= the round's
// target count (<= 32) slots and 32 / G splits, so a leaf of 33-64 targets
// splits its last round's sources over the lanes its few targets leave;
// splits are summed with warp shuffles.  Sources are staged 32 at a time: point
// sources from the leaf's near list (segments = source leaves, found by
// bisection of the warp's prefix sums), then the W-list upward equivalent
// surfaces and the leaf's own downward equivalent surface.
template <typename T>
struct WarpSegs {
  int beg[32];
  int pre[33];
  T shx[32], shy[32], shz[32], rad[32];
  const T* unit[32];
  const T* den[32];
};

template <typename T, int KT, int NWARP>
__global__ void __launch_bounds__(32 * NWARP) k_leaf_warp(P2PArgs<T> a, const int* work, const int64_t* nptr,
                                                             const int* nidx, const int64_t* mptr, const int* midx,
                                                             int nwork, int rhs) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  constexpr bool DL = KTraits<KT>::DL;
  constexpr int MM = KTraits<KT>::MM;
  constexpr int SDM = KTraits<MM>::SD;
  __shared__ WarpSrc64<T> ws[NWARP];
  __shared__ WarpSegs<T> wg[NWARP];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSrc64<T>& w = ws[warp];
  WarpSegs<T>& sgt = wg[warp];
  // packed FP32 Laplace sums (near field for KT 111, surfaces for MM 111)
  constexpr bool PAIR_NEAR = KT == 111 && sizeof(T) == 4, PAIR_SURF = MM == 111 && sizeof(T) == 4;
  const T* den = a.sden + (size_t)rhs * a.ns * SD;
  T* outbase = a.tval + (size_t)rhs * a.nt * TD;
  const int nsurf = a.nsurf;
  for (int wi = blockIdx.x * NWARP + warp; wi < nwork; wi += gridDim.x * NWARP) {
    const int g = work[wi];
    const double cx = a.center[3 * g], cy = a.center[3 * g + 1], cz = a.center[3 * g + 2];
    const T rad = (T)a.radius[g];
    const int tb0 = a.tbeg[g], nt = a.tcnt[g];
    const bool l2t = a.depth[g] >= a.l2t_depth;
    const int64_t nb = nptr[wi], ne = nptr[wi + 1];
    const int64_t mb = mptr[wi], me = mptr[wi + 1];
    const int nsurf_segs = (int)(me - mb) + (l2t ? 1 : 0);
    for (int tb = 0, G = 32; tb < nt; tb += G) {
      G = 1;
      while (G < nt - tb && G < 32) G <<= 1;
      const int nsplit = 32 / G, slot = lane % G, sg = lane / G;
      const int ti = tb + slot;
      const bool valid = ti < nt;
      T px = 0, py = 0, pz = 0;
      if (valid) {
        px = a.tx[tb0 + ti];
        py = a.ty[tb0 + ti];
        pz = a.tz[tb0 + ti];
      }
      T acc[4] = {0, 0, 0, 0};
      // point sources, up to 32 source leaves per batch
      for (int64_t c0 = nb; c0 < ne; c0 += 32) {
        const int nseg = (int)min((int64_t)32, ne - c0);
        __syncwarp();
        int cntl = 0;
        if (lane < nseg) {
          const int s = nidx[c0 + lane];
          sgt.beg[lane] = a.sbeg[s];
          cntl = a.scnt[s];
          sgt.shx[lane] = (T)(a.center[3 * s] - cx);
          sgt.shy[lane] = (T)(a.center[3 * s + 1] - cy);
          sgt.shz[lane] = (T)(a.center[3 * s + 2] - cz);
        }
        // inclusive scan of the segment sizes
        int incl = cntl;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        sgt.pre[lane + 1] = incl;
        if (lane == 0) sgt.pre[0] = 0;
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        __syncwarp();
        for (int k0 = 0; k0 < total; k0 += 64) {
          const int cnt = min(64, total - k0);
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int jl = lane + 32 * h;
            if (jl >= cnt) {
              // an odd batch's last pair: a zero-weight partner
              if (PAIR_NEAR && jl == cnt && (cnt & 1)) stage_src(w, jl, P4<T>{T(0), T(0), T(0), T(0)}, true);
              break;
            }
            const int k = k0 + jl;
            int lo = 0, hi = nseg;  // pre[lo] <= k < pre[hi]
            while (hi - lo > 1) {
              const int mid = (lo + hi) >> 1;
              if (sgt.pre[mid] <= k)
                lo = mid;
              else
                hi = mid;
            }
            const int p = sgt.beg[lo] + (k - sgt.pre[lo]);
            T f[SD];
#pragma unroll
            for (int s = 0; s < SD; s++) f[s] = den[(size_t)p * SD + s];
            stage_src(w, jl, P4<T>{a.sx[p] + sgt.shx[lo], a.sy[p] + sgt.shy[lo], a.sz[p] + sgt.shz[lo], f[0]},
                      PAIR_NEAR);
#pragma unroll
            for (int s = 1; s < SD; s++) w.f[jl * (SD - 1) + s - 1] = f[s];
            if constexpr (DL) {
              w.n[3 * jl] = a.snx[p];
              w.n[3 * jl + 1] = a.sny[p];
              w.n[3 * jl + 2] = a.snz[p];
            }
          }
          __syncwarp();
          if (valid) {
            const int rounds = sg < cnt ? (cnt - sg + nsplit - 1) / nsplit : 0;
            if constexpr (PAIR_NEAR) {  // sum f / r on source pairs, times 1/(4 pi) once
              acc[0] += a.ku.c0 * lap_pairs(w, px, py, pz, sg, nsplit, (cnt + 1) >> 1);
            } else if constexpr (KT == 111) {  // FP64: sum f / r, times 1/(4 pi) once
              T s1 = T(0);
#pragma unroll 4
              for (int r = 0; r < rounds; r++) {
                const P4<T> s = w.p[sg + r * nsplit];
                const T x = px - s.x, y = py - s.y, z = pz - s.z;
                const T r2 = x * x + y * y + z * z;
                const T ri = (r2 >= T(1e-16)) ? rsqrt_t(r2) : T(0);
                s1 += ri * s.w;
              }
              acc[0] += a.ku.c0 * s1;
            } else {
#pragma unroll 4
              for (int r = 0; r < rounds; r++) {
                const int j = sg + r * nsplit;
                const P4<T> s = w.p[j];
                T f[SD];
                f[0] = s.w;
#pragma unroll
                for (int k = 1; k < SD; k++) f[k] = w.f[j * (SD - 1) + k - 1];
                T nrm[3];
                if constexpr (DL) {
                  nrm[0] = w.n[3 * j];
                  nrm[1] = w.n[3 * j + 1];
                  nrm[2] = w.n[3 * j + 2];
                }
                keval<KT, T>(px - s.x, py - s.y, pz - s.z, nrm, f, acc, a.ku);
              }
            }
          }
          __syncwarp();
        }
      }
      // surface sources: W-list upward equivalent surfaces and the leaf's own
      // downward equivalent surface, equivalent kernel
      for (int c0 = 0; c0 < nsurf_segs; c0 += 32) {
        const int nseg = min(32, nsurf_segs - c0);
        __syncwarp();
        if (lane < nseg) {
          const int e = c0 + lane;
          if (e < (int)(me - mb)) {
            const int s = midx[mb + e];
            sgt.shx[lane] = (T)(a.center[3 * s] - cx);
            sgt.shy[lane] = (T)(a.center[3 * s + 1] - cy);
            sgt.shz[lane] = (T)(a.center[3 * s + 2] - cz);
            sgt.rad[lane] = (T)a.radius[s];
            sgt.unit[lane] = a.ue_unit;
            sgt.den[lane] = a.supeden + (size_t)s * nsurf * SDM;
          } else {
            sgt.shx[lane] = sgt.shy[lane] = sgt.shz[lane] = T(0);
            sgt.rad[lane] = rad;
            sgt.unit[lane] = a.de_unit;
            sgt.den[lane] = a.tdneden + (size_t)g * nsurf * SDM;
          }
        }
        __syncwarp();
        const int total = nseg * nsurf;
        for (int k0 = 0; k0 < total; k0 += 64) {
          const int cnt = min(64, total - k0);
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int jl = lane + 32 * h;
            if (jl >= cnt) {
              if (PAIR_SURF && jl == cnt && (cnt & 1)) stage_src(w, jl, P4<T>{T(0), T(0), T(0), T(0)}, true);
              break;
            }
            const int k = k0 + jl;
            const int e = k / nsurf, m = k - e * nsurf;
            const T* u = sgt.unit[e];
            const T* sd = sgt.den[e];
            const T r = sgt.rad[e];
            stage_src(w, jl,
                      P4<T>{u[3 * m] * r + sgt.shx[e], u[3 * m + 1] * r + sgt.shy[e], u[3 * m + 2] * r + sgt.shz[e],
                            sd[(size_t)m * SDM]},
                      PAIR_SURF);
#pragma unroll
            for (int s = 1; s < SDM; s++) w.f[jl * (SDM - 1) + s - 1] = sd[(size_t)m * SDM + s];
          }
          __syncwarp();
          if (valid) {
            const int rounds = sg < cnt ? (cnt - sg + nsplit - 1) / nsplit : 0;
            if constexpr (PAIR_SURF) {
              acc[0] += a.km.c0 * lap_pairs(w, px, py, pz, sg, nsplit, (cnt + 1) >> 1);
            } else if constexpr (MM == 111) {
              T s1 = T(0);
#pragma unroll 4
              for (int r = 0; r < rounds; r++) {
                const P4<T> s = w.p[sg + r * nsplit];
                const T x = px - s.x, y = py - s.y, z = pz - s.z;
                const T r2 = x * x + y * y + z * z;
                const T ri = (r2 >= T(1e-16)) ? rsqrt_t(r2) : T(0);
                s1 += ri * s.w;
              }
              acc[0] += a.km.c0 * s1;
            } else {
#pragma unroll 4
              for (int r = 0; r < rounds; r++) {
                const int j = sg + r * nsplit;
                const P4<T> s = w.p[j];
                T f[SDM];
                f[0] = s.w;
#pragma unroll
                for (int k = 1; k < SDM; k++) f[k] = w.f[j * (SDM - 1) + k - 1];
                T nrm[3];
                keval<MM, T>(px - s.x, py - s.y, pz - s.z, nrm, f, acc, a.km);
              }
            }
          }
          __syncwarp();
        }
      }
      // sum the splits (lanes slot, slot + G, ...)
#pragma unroll
      for (int d = 0; d < TD; d++)
        for (int o = G; o < 32; o <<= 1) acc[d] += __shfl_xor_sync(0xffffffffu, acc[d], o);
      if (valid && sg == 0)
#pragma unroll
        for (int d = 0; d < TD; d++) outbase[(size_t)(tb0 + ti) * TD + d] = acc[d];
    }
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

// trgval[r][perm[i]][t] = tval[r][i][t] + near[r][i][t]: the FP32 passes'
// potentials plus an FP64 near-field sum
__global__ void k_gather_val_sum(const float* tval, const double* near, const int* perm, int nt, int td, int nrhs,
                                 double* trgval) {
  size_t n = (size_t)nt * td * nrhs;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    size_t r = e / ((size_t)nt * td);
    size_t rem = e % ((size_t)nt * td);
    int i = (int)(rem / td), d = (int)(rem % td);
    trgval[r * nt * td + (size_t)perm[i] * td + d] = (double)tval[e] + near[e];
  }
}

template <typename T, int KT>
void launch_p2p_kt(const P2PArgs<T>& a, const P2PWork& w, int which, int rhs, cudaStream_t st) {
  switch (which) {
    case P2P_S2M:
      if (w.n) {
        const int grid = std::min((w.n + WP_WARPS - 1) / WP_WARPS, 148 * 32);
        if (a.nuc <= 160)
          k_s2m_warp<T, KT, 5><<<grid, 32 * WP_WARPS, 0, st>>>(a, w.work, w.n, rhs);
        else if (a.nuc <= 320)
          k_s2m_warp<T, KT, 10><<<grid, 32 * WP_WARPS, 0, st>>>(a, w.work, w.n, rhs);
        else  // |UC| <= 488 for np <= 8
          k_s2m_warp<T, KT, 16><<<grid, 32 * WP_WARPS, 0, st>>>(a, w.work, w.n, rhs);
      }
      break;
    case P2P_S2L:
      if (w.n) k_s2l<T, KT><<<w.n, P2P_THREADS, 0, st>>>(a, w.work, w.ptr, w.idx, w.n, rhs);
      break;
    case P2P_LEAF:
      if (w.n) {
        constexpr int nw = sizeof(T) == 4 ? 8 : 4;  // static shared memory: 64 staged sources per warp
        const int grid = std::min((w.n + nw - 1) / nw, 148 * 32);
        k_leaf_warp<T, KT, nw><<<grid, 32 * nw, 0, st>>>(a, w.work, w.ptr, w.idx, w.ptr2, w.idx2, w.n, rhs);
      }
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

void launch_gather_val_sum(const float* tval, const double* near, const int* perm, int nt, int td, int nrhs,
                           double* trgval, cudaStream_t st) {
  size_t n = (size_t)nt * td * nrhs;
  if (!n) return;
  int grid = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_gather_val_sum<<<grid, 256, 0, st>>>(tval, near, perm, nt, td, nrhs, trgval);
}
template void launch_gather_val<float>(const float*, const int*, int, int, int, double*, cudaStream_t);

}  // namespace kifmm
