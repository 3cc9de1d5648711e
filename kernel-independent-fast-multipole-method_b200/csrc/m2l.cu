// FFT-accelerated M2L (V list), the reference's dominant phase
// (fmm3d/fmm3d_eval.cpp:115-150; MatMgnt3d::plnden2effden, UE2DC_dgemv,
// effval2plnval, fmm3d/matmgnt3d.cpp:223-361).
//
// The surface density of a node is a sparse (2np)^3 grid: only the np^3
// corner block holds data, and only on its boundary.  Instead of a general
// FFT library the transforms are pruned separable DFTs done in shared
// memory, one CTA per node:
//   forward : x pass (np^2 lines, np inputs -> np+1 outputs), y pass, z pass
//   inverse : z and y passes evaluated only at the np outputs the surface
//             needs, then the Hermitian half-line c2r along x at the surface
//             points only.
// The kernel spectra are computed once on the host (operators.cpp) with the
// same sign convention w = exp(-2 pi i / n) and already carry 1/n^3.
// Spectra are stored Hermitian-compacted: of the kx = 0 and kx = n/2 planes,
// which a real grid's half spectrum repeats as X(kx,-ky,-kz) = conj X(kx,ky,kz),
// only the canonical half is kept (4 np^3 + 4 values instead of 4 np^2 (np+1);
// 868 of 1008 at np = 6).  The products K X keep the symmetry, so the
// forward pass computes, the Hadamard pass multiplies and the inverse pass
// reads back (conjugating the mirrored half) only the independent values.
// Density and potential grids use indices [0, np) per axis; the reference's
// np/2 shift (matmgnt3d.cpp:256) cancels between embedding and extraction.
#include <cuda_fp16.h>

#include <algorithm>

#include "launch.hpp"

namespace kifmm {
namespace {

constexpr int FFT_THREADS = 256;

template <typename T>
struct Cpx {
  T re, im;
};

// ---------------------------------------------------------------------------
// Warp-per-node transforms.  One warp carries one node through all passes
// with only warp-level synchronisation, so a CTA keeps up to 8 nodes in
// flight and never waits on a CTA-wide barrier between passes.  Shared
// memory: the CTA's twiddle-product table W2[n*n], then one region per warp.
template <typename T>
__device__ __forceinline__ void fill_w2(Cpx<T>* W2, int n) {
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int m = ((e / n) * (e % n)) % n;
    double s, c;
    sincospi(-2.0 * (double)m / (double)n, &s, &c);
    W2[e].re = (T)c;
    W2[e].im = (T)s;
  }
}

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

template <typename T>
__host__ __device__ inline size_t fwd_warp_bytes(int np, int n, int nh) {
  return align16(sizeof(T) * np * np * np) + align16(sizeof(Cpx<T>) * np * np * nh) +
         align16(sizeof(Cpx<T>) * np * n * nh);
}

// register-blocked forward: A (np x np x nh) and Bm (np x n x nh) per warp; the
// density grid (np^3) shares Bm's space, being dead before the y pass writes Bm
template <typename T>
__host__ __device__ inline size_t fwd_rb_warp_bytes(int np, int n, int nh) {
  return align16(sizeof(Cpx<T>) * np * np * nh) + align16(sizeof(Cpx<T>) * np * n * nh);
}

// register-blocked inverse: Bm (np x n x nh) and A (np x np x nh) per warp
template <typename T>
__host__ __device__ inline size_t inv_rb_warp_bytes(int np, int n, int nh) {
  return align16(sizeof(Cpx<T>) * np * n * nh) + align16(sizeof(Cpx<T>) * np * np * nh);
}

// the staged accumulated spectrum of one node (sibling-group-major FP32 form)
template <typename T>
__host__ __device__ inline size_t inv_rb_stage_bytes(int np) {
  return align16(sizeof(Cpx<T>) * (4 * np * np * np + 4));
}

template <typename T>
__host__ __device__ inline size_t inv_warp_bytes(int np, int n, int nh) {
  return align16(sizeof(Cpx<T>) * n * n * nh) + align16(sizeof(Cpx<T>) * np * n * nh) +
         align16(sizeof(Cpx<T>) * np * np * nh);
}

template <typename T, int NP>
__global__ void __launch_bounds__(256) k_m2l_fwd_warp(M2LGeom g, const T* __restrict__ supeden,
                                                      const int* __restrict__ nodes, int nwork,
                                                      const int* __restrict__ depth, T* __restrict__ spectra) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // NP > 0: compile-time sizes (constant divisors, unrolled sums); NP = 0: any np
  const int np = NP > 0 ? NP : g.np, n = NP > 0 ? 2 * NP : g.n, nh = NP > 0 ? NP + 1 : g.nh;
  const int nfc = NP > 0 ? 4 * NP * NP * NP + 4 : g.nfc;
  const int nsurf = NP > 0 ? NP * NP * NP - (NP - 2) * (NP - 2) * (NP - 2) : g.nsurf;
  Cpx<T>* W2 = reinterpret_cast<Cpx<T>*>(smem_raw);
  fill_w2(W2, n);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpc = blockDim.x >> 5;
  unsigned char* mine = smem_raw + align16(sizeof(Cpx<T>) * n * n) + (size_t)warp * fwd_warp_bytes<T>(np, n, nh);
  T* xg = reinterpret_cast<T*>(mine);
  Cpx<T>* A = reinterpret_cast<Cpx<T>*>(mine + align16(sizeof(T) * np * np * np));
  Cpx<T>* Bm = reinterpret_cast<Cpx<T>*>(reinterpret_cast<unsigned char*>(A) + align16(sizeof(Cpx<T>) * np * np * nh));
  for (int wi = blockIdx.x * wpc + warp; wi < nwork; wi += gridDim.x * wpc) {
    const int node = nodes[wi];
    const int lvl = depth[node] + g.rootlvl;
    const T* den = supeden + (size_t)node * nsurf * g.sd;
    for (int s = 0; s < g.sd; s++) {
      const T scale = (T)ldexp(1.0, lvl * g.deg[s]);  // plnden2effden scaling, matmgnt3d.cpp:228-235
      for (int e = lane; e < np * np * np; e += 32) xg[e] = T(0);
      __syncwarp();
      for (int k = lane; k < nsurf; k += 32) {
        int i = g.surf_ijk[3 * k], j = g.surf_ijk[3 * k + 1], kk = g.surf_ijk[3 * k + 2];
        xg[(i * np + j) * np + kk] = den[(size_t)k * g.sd + s] * scale;
      }
      __syncwarp();
      for (int e = lane; e < np * np * nh; e += 32) {  // x pass
        int kx = e % nh, j = (e / nh) % np, k = e / (nh * np);
        T re = 0, im = 0;
#pragma unroll
        for (int i = 0; i < np; i++) {
          T v = xg[(i * np + j) * np + k];
          Cpx<T> t = W2[i * n + kx];
          re += v * t.re;
          im += v * t.im;
        }
        A[e].re = re;
        A[e].im = im;
      }
      __syncwarp();
      for (int e = lane; e < np * n * nh; e += 32) {  // y pass
        int kx = e % nh, ky = (e / nh) % n, k = e / (nh * n);
        T re = 0, im = 0;
#pragma unroll
        for (int j = 0; j < np; j++) {
          Cpx<T> a = A[(k * np + j) * nh + kx];
          Cpx<T> t = W2[j * n + ky];
          re = fmt(-a.im, t.im, fmt(a.re, t.re, re));
          im = fmt(a.im, t.re, fmt(a.re, t.im, im));
        }
        Bm[e].re = re;
        Bm[e].im = im;
      }
      __syncwarp();
      Cpx<T>* out = reinterpret_cast<Cpx<T>*>(spectra + ((size_t)node * g.sd + s) * nfc * 2);
      for (int c = lane; c < nfc; c += 32) {  // z pass, at the canonical frequencies only
        const int e = g.fc2f[c];
        int kxy = e % (n * nh), kz = e / (n * nh);
        Cpx<T> r;
        r.re = r.im = T(0);
#pragma unroll
        for (int k = 0; k < np; k++) {
          Cpx<T> b = Bm[k * n * nh + kxy];
          Cpx<T> t = W2[k * n + kz];
          r.re = fmt(-b.im, t.im, fmt(b.re, t.re, r.re));
          r.im = fmt(b.im, t.re, fmt(b.re, t.im, r.im));
        }
        if (g.sg)
          reinterpret_cast<Cpx<T>*>(spectra)[spectra_sg_index(nfc, node, c)] = r;
        else
          out[c] = r;
      }
      __syncwarp();
    }
  }
}

template <typename T, int NP>
__global__ void __launch_bounds__(256) k_m2l_inv_warp(M2LGeom g, const T* __restrict__ effval,
                                                      const int* __restrict__ work, int nwork,
                                                      T* __restrict__ tdncval) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // NP > 0: compile-time sizes (constant divisors, unrolled sums); NP = 0: any np
  const int np = NP > 0 ? NP : g.np, n = NP > 0 ? 2 * NP : g.n, nh = NP > 0 ? NP + 1 : g.nh;
  const int nf = NP > 0 ? 4 * NP * NP * (NP + 1) : g.nfreq;
  const int nfc = NP > 0 ? 4 * NP * NP * NP + 4 : g.nfc;
  const int nsurf = NP > 0 ? NP * NP * NP - (NP - 2) * (NP - 2) * (NP - 2) : g.nsurf;
  Cpx<T>* W2 = reinterpret_cast<Cpx<T>*>(smem_raw);
  fill_w2(W2, n);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpc = blockDim.x >> 5;
  unsigned char* mine = smem_raw + align16(sizeof(Cpx<T>) * n * n) + (size_t)warp * inv_warp_bytes<T>(np, n, nh);
  Cpx<T>* Y = reinterpret_cast<Cpx<T>*>(mine);
  Cpx<T>* Bm = reinterpret_cast<Cpx<T>*>(mine + align16(sizeof(Cpx<T>) * n * n * nh));
  Cpx<T>* A = reinterpret_cast<Cpx<T>*>(reinterpret_cast<unsigned char*>(Bm) + align16(sizeof(Cpx<T>) * np * n * nh));
  for (int wi = blockIdx.x * wpc + warp; wi < nwork; wi += gridDim.x * wpc) {
    const int node = work[wi];
    T* dst = tdncval + (size_t)node * nsurf * g.td;
    for (int t = 0; t < g.td; t++) {
      const Cpx<T>* src = reinterpret_cast<const Cpx<T>*>(effval + ((size_t)node * g.td + t) * nfc * 2);
      for (int e = lane; e < nf; e += 32) {  // full half spectrum from the canonical values
        const int m = g.ff2c[e];
        Cpx<T> v = src[m >= 0 ? m : -m - 1];
        if (m < 0) v.im = -v.im;
        Y[e] = v;
      }
      __syncwarp();
      for (int e = lane; e < np * n * nh; e += 32) {  // z pass (inverse), k < np
        int kxy = e % (n * nh), k = e / (n * nh);
        T re = 0, im = 0;
#pragma unroll
        for (int kz = 0; kz < n; kz++) {
          Cpx<T> y = Y[kz * n * nh + kxy];
          Cpx<T> c = W2[k * n + kz];
          re = fmt(y.im, c.im, fmt(y.re, c.re, re));
          im = fmt(-y.re, c.im, fmt(y.im, c.re, im));
        }
        Bm[e].re = re;
        Bm[e].im = im;
      }
      __syncwarp();
      for (int e = lane; e < np * np * nh; e += 32) {  // y pass (inverse), j < np
        int kx = e % nh, j = (e / nh) % np, k = e / (nh * np);
        T re = 0, im = 0;
#pragma unroll
        for (int ky = 0; ky < n; ky++) {
          Cpx<T> b = Bm[(k * n + ky) * nh + kx];
          Cpx<T> c = W2[j * n + ky];
          re = fmt(b.im, c.im, fmt(b.re, c.re, re));
          im = fmt(-b.re, c.im, fmt(b.im, c.re, im));
        }
        A[e].re = re;
        A[e].im = im;
      }
      __syncwarp();
      for (int m = lane; m < nsurf; m += 32) {  // c2r along x at the surface points
        int i = g.surf_ijk[3 * m], j = g.surf_ijk[3 * m + 1], k = g.surf_ijk[3 * m + 2];
        const Cpx<T>* a = &A[(k * np + j) * nh];
        T v = a[0].re + ((i & 1) ? -a[nh - 1].re : a[nh - 1].re);
        T acc = 0;
#pragma unroll
        for (int kx = 1; kx < nh - 1; kx++) {
          Cpx<T> c = W2[i * n + kx];
          acc = fmt(a[kx].im, c.im, fmt(a[kx].re, c.re, acc));
        }
        dst[(size_t)m * g.td + t] += v + T(2) * acc;
      }
      __syncwarp();
    }
  }
}

// effval[w][t][f] = sum_{s in V} sum_sd Khat[off][t][sd][f] * X[s][sd][f]   (cptwvv, matmgnt3d.cpp:343-360)
template <typename T, int SD, int TD>
__global__ void __launch_bounds__(FFT_THREADS) k_m2l_had(M2LGeom g, const T* __restrict__ khat,
                                                          const T* __restrict__ spectra, const int* __restrict__ work,
                                                          const int64_t* __restrict__ vptr,
                                                          const int* __restrict__ vidx, const int* __restrict__ path,
                                                          T* __restrict__ effval) {
  // A V list holds at most 6^3 - 3^3 = 189 nodes (fmm3d/let3d.cpp:228-247);
  // the host checks this bound before launching.
  constexpr int VMAX = 192;
  __shared__ int vs[VMAX], vo[VMAX];
  const int wi = blockIdx.x;
  const int t = work[wi];
  const int nf = g.nfc;  // canonical frequencies only
  const int64_t b = vptr[wi];
  const int cnt = (int)(vptr[wi + 1] - b);
  const int tp0 = path[3 * t], tp1 = path[3 * t + 1], tp2 = path[3 * t + 2];
  T* out = effval + (size_t)t * TD * nf * 2;
  for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
    int s = vidx[b + q];
    vs[q] = s;
    vo[q] = (path[3 * s] - tp0 + 3) * 49 + (path[3 * s + 1] - tp1 + 3) * 7 + (path[3 * s + 2] - tp2 + 3);
  }
  __syncthreads();
  for (int f = threadIdx.x; f < nf; f += blockDim.x) {
    T ar[TD], ai[TD];
#pragma unroll
    for (int d = 0; d < TD; d++) ar[d] = ai[d] = T(0);
    {
      for (int q = 0; q < cnt; q++) {
        const T* X = spectra + (size_t)vs[q] * SD * nf * 2;
        const T* K = khat + (size_t)vo[q] * TD * SD * nf * 2;
        T xr[SD], xi[SD];
#pragma unroll
        for (int s = 0; s < SD; s++) {
          xr[s] = X[((size_t)s * nf + f) * 2];
          xi[s] = X[((size_t)s * nf + f) * 2 + 1];
        }
#pragma unroll
        for (int d = 0; d < TD; d++)
#pragma unroll
          for (int s = 0; s < SD; s++) {
            T kr = K[(((size_t)d * SD + s) * nf + f) * 2];
            T ki = K[(((size_t)d * SD + s) * nf + f) * 2 + 1];
            ar[d] = fmt(-ki, xi[s], fmt(kr, xr[s], ar[d]));
            ai[d] = fmt(ki, xr[s], fmt(kr, xi[s], ai[d]));
          }
      }
    }
#pragma unroll
    for (int d = 0; d < TD; d++) {
      out[((size_t)d * nf + f) * 2] = ar[d];
      out[((size_t)d * nf + f) * 2 + 1] = ai[d];
    }
  }
}

// ---------------------------------------------------------------------------
// Register-blocked transforms for np = 4, 6, 8.  Each lane owns one line of a
// pass, keeps that line's np (or n) inputs in registers and produces every
// output of the line, so a shared-memory value feeds a whole row of complex
// multiply-adds instead of one.  The twiddle factors are compile-time
// constants (tw_re / tw_im below), folded into the multiply-adds.

// cos and sin on |r| <= pi/4 by their Taylor series (10 terms: below 1e-20)
__host__ __device__ constexpr double taylor_sin(double r) {
  double r2 = r * r, t = r, s = r;
  for (int k = 1; k <= 10; k++) {
    t *= -r2 / ((2.0 * k) * (2.0 * k + 1.0));
    s += t;
  }
  return s;
}
__host__ __device__ constexpr double taylor_cos(double r) {
  double r2 = r * r, t = 1.0, s = 1.0;
  for (int k = 1; k <= 10; k++) {
    t *= -r2 / ((2.0 * k - 1.0) * (2.0 * k));
    s += t;
  }
  return s;
}
// w^m = exp(-2 pi i m / n): the angle 2 pi m / n is split into q quarter turns
// plus a remainder r, |r| <= pi/4, both exact in m and n
__host__ __device__ constexpr double tw_re(int m, int n) {
  m %= n;
  const int q = (8 * m + n) / (2 * n);
  const double r = 1.5707963267948966 * (double)(4 * m - q * n) / (double)n;
  const int o = q & 3;
  return o == 0 ? taylor_cos(r) : o == 1 ? -taylor_sin(r) : o == 2 ? -taylor_cos(r) : taylor_sin(r);
}
__host__ __device__ constexpr double tw_im(int m, int n) {
  m %= n;
  const int q = (8 * m + n) / (2 * n);
  const double r = 1.5707963267948966 * (double)(4 * m - q * n) / (double)n;
  const int o = q & 3;
  const double s = o == 0 ? taylor_sin(r) : o == 1 ? taylor_cos(r) : o == 2 ? -taylor_sin(r) : -taylor_cos(r);
  return -s;
}

// twiddle tables for n = 8, 12, 16, statically initialised from tw_re / tw_im;
// indexed with compile-time offsets they are constant-bank operands
#define KIFMM_TW16(F, n)                                                                                         \
  {F(0, n), F(1, n), F(2, n), F(3, n), F(4, n), F(5, n), F(6, n), F(7, n), F(8, n), F(9, n), F(10, n), F(11, n), \
   F(12, n), F(13, n), F(14, n), F(15, n)}
#define KIFMM_TWSET(F) {KIFMM_TW16(F, 8), KIFMM_TW16(F, 12), KIFMM_TW16(F, 16)}
#define KIFMM_FRE(m, n) (float)tw_re(m, n)
#define KIFMM_FIM(m, n) (float)tw_im(m, n)
#define KIFMM_DRE(m, n) tw_re(m, n)
#define KIFMM_DIM(m, n) tw_im(m, n)
__constant__ float c_twf_re[3][16] = KIFMM_TWSET(KIFMM_FRE);
__constant__ float c_twf_im[3][16] = KIFMM_TWSET(KIFMM_FIM);
__constant__ double c_twd_re[3][16] = KIFMM_TWSET(KIFMM_DRE);
__constant__ double c_twd_im[3][16] = KIFMM_TWSET(KIFMM_DIM);
#undef KIFMM_FRE
#undef KIFMM_FIM
#undef KIFMM_DRE
#undef KIFMM_DIM
#undef KIFMM_TWSET
#undef KIFMM_TW16

template <typename T, int N>
__device__ __forceinline__ T twr(int m) {
  constexpr int t = N == 8 ? 0 : N == 12 ? 1 : 2;
  if constexpr (sizeof(T) == 4)
    return c_twf_re[t][m % N];
  else
    return c_twd_re[t][m % N];
}
template <typename T, int N>
__device__ __forceinline__ T twi(int m) {
  constexpr int t = N == 8 ? 0 : N == 12 ? 1 : 2;
  if constexpr (sizeof(T) == 4)
    return c_twf_im[t][m % N];
  else
    return c_twd_im[t][m % N];
}

// scale 2^(14 - e) of the FP16-pair spectra, 2^e >= the bound (1 without one)
__device__ __forceinline__ float spectra_scale16(const unsigned* bound) {
  const float b = bound ? __uint_as_float(*bound) : 0.f;
  if (!(b > 0.f)) return 1.f;
  int e;
  frexpf(b, &e);
  return ldexpf(1.f, 14 - e);
}

// x * s as {hi(re), hi(im)}, {lo(re), lo(im)}: FP16 rounded to nearest,
// lo = the FP16 rounding of what hi leaves over
__device__ __forceinline__ uint2 f16_pairs(float re, float im, float s) {
  const float xr = re * s, xi = im * s;
  const __half2 hi = __floats2half2_rn(xr, xi);
  const float2 hf = __half22float2(hi);
  const __half2 lo = __floats2half2_rn(xr - hf.x, xi - hf.y);
  return make_uint2(*reinterpret_cast<const unsigned*>(&hi), *reinterpret_cast<const unsigned*>(&lo));
}

template <typename T, int NP>
__global__ void __launch_bounds__(256) k_m2l_fwd_rb(M2LGeom g, const T* __restrict__ supeden,
                                                    const int* __restrict__ nodes, int nwork,
                                                    const int* __restrict__ depth, T* __restrict__ spectra) {
  constexpr int N = 2 * NP, NH = NP + 1, NFC = 4 * NP * NP * NP + 4;
  constexpr int NSURF = NP * NP * NP - (NP - 2) * (NP - 2) * (NP - 2);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpc = blockDim.x >> 5;
  int* c_of = reinterpret_cast<int*>(smem_raw);  // full -> compact frequency index (< 0: not stored)
  for (int e = threadIdx.x; e < N * N * NH; e += blockDim.x) c_of[e] = g.ff2c[e];
  unsigned char* mine = smem_raw + align16(sizeof(int) * N * N * NH) + (size_t)warp * fwd_rb_warp_bytes<T>(NP, N, NH);
  Cpx<T>* A = reinterpret_cast<Cpx<T>*>(mine);
  Cpx<T>* Bm = reinterpret_cast<Cpx<T>*>(mine + align16(sizeof(Cpx<T>) * NP * NP * NH));
  // the density grid lives in Bm's space: read only by the x pass, which a
  // __syncwarp separates from the y pass's first write of Bm
  T* xg = reinterpret_cast<T*>(Bm);
  static_assert(sizeof(T) * NP * NP * NP <= sizeof(Cpx<T>) * NP * N * NH, "density grid fits in Bm");
  const float s16 = g.sg == 2 ? spectra_scale16(g.bound) : 1.f;
  __syncthreads();
  for (int wi = blockIdx.x * wpc + warp; wi < nwork; wi += gridDim.x * wpc) {
    const int node = nodes[wi];
    const int lvl = depth[node] + g.rootlvl;
    const T* den = supeden + (size_t)node * NSURF * g.sd;
    for (int s = 0; s < g.sd; s++) {
      const T scale = (T)ldexp(1.0, lvl * g.deg[s]);  // plnden2effden scaling, matmgnt3d.cpp:228-235
      for (int e = lane; e < NP * NP * NP; e += 32) xg[e] = T(0);
      __syncwarp();
      for (int k = lane; k < NSURF; k += 32) {
        const int i = g.surf_ijk[3 * k], j = g.surf_ijk[3 * k + 1], kk = g.surf_ijk[3 * k + 2];
        xg[(i * NP + j) * NP + kk] = den[(size_t)k * g.sd + s] * scale;
      }
      __syncwarp();
      // x pass, lines (j, k): A[k][j][kx] = sum_i xg[i][j][k] w^(i kx)
      for (int line = lane; line < NP * NP; line += 32) {
        const int j = line % NP, k = line / NP;
        T v[NP];
#pragma unroll
        for (int i = 0; i < NP; i++) v[i] = xg[(i * NP + j) * NP + k];
#pragma unroll
        for (int kx = 0; kx < NH; kx++) {
          T re = 0, im = 0;
#pragma unroll
          for (int i = 0; i < NP; i++) {
            re += v[i] * twr<T, N>(i * kx);
            im += v[i] * twi<T, N>(i * kx);
          }
          A[(k * NP + j) * NH + kx] = Cpx<T>{re, im};
        }
      }
      __syncwarp();
      // y pass, lines (k, kx): Bm[k][ky][kx] = sum_j A[k][j][kx] w^(j ky)
      for (int line = lane; line < NP * NH; line += 32) {
        const int kx = line % NH, k = line / NH;
        Cpx<T> a[NP];
#pragma unroll
        for (int j = 0; j < NP; j++) a[j] = A[(k * NP + j) * NH + kx];
#pragma unroll
        for (int ky = 0; ky < N; ky++) {
          T re = 0, im = 0;
#pragma unroll
          for (int j = 0; j < NP; j++) {
            const T c = twr<T, N>(j * ky), d = twi<T, N>(j * ky);
            re = fmt(-a[j].im, d, fmt(a[j].re, c, re));
            im = fmt(a[j].im, c, fmt(a[j].re, d, im));
          }
          Bm[(k * N + ky) * NH + kx] = Cpx<T>{re, im};
        }
      }
      __syncwarp();
      // z pass, lines (ky, kx): spectrum[kz][ky][kx] = sum_k Bm[k][ky][kx] w^(k kz), canonical only
      Cpx<T>* out = reinterpret_cast<Cpx<T>*>(spectra + ((size_t)node * g.sd + s) * NFC * 2);
      for (int line = lane; line < N * NH; line += 32) {
        const int kx = line % NH, ky = line / NH;
        Cpx<T> b[NP];
#pragma unroll
        for (int k = 0; k < NP; k++) b[k] = Bm[(k * N + ky) * NH + kx];
#pragma unroll
        for (int kz = 0; kz < N; kz++) {
          const int c = c_of[(kz * N + ky) * NH + kx];
          if (c < 0) continue;
          T re = 0, im = 0;
#pragma unroll
          for (int k = 0; k < NP; k++) {
            const T cr = twr<T, N>(k * kz), ci = twi<T, N>(k * kz);
            re = fmt(-b[k].im, ci, fmt(b[k].re, cr, re));
            im = fmt(b[k].im, cr, fmt(b[k].re, ci, im));
          }
          if constexpr (sizeof(T) == 4) {
            if (g.sg == 2) {
              reinterpret_cast<uint2*>(spectra)[s * g.plane + spectra_sg_index(NFC, node, c)] =
                  f16_pairs(re, im, s16);
              continue;
            }
          }
          if (g.sg)
            reinterpret_cast<Cpx<T>*>(spectra)[spectra_sg_index(NFC, node, c)] = Cpx<T>{re, im};
          else
            out[c] = Cpx<T>{re, im};
        }
      }
      __syncwarp();
    }
  }
}

template <typename T, int NP>
__global__ void __launch_bounds__(256) k_m2l_inv_rb(M2LGeom g, const T* __restrict__ effval,
                                                    const int* __restrict__ work, int nwork,
                                                    T* __restrict__ tdncval) {
  constexpr int N = 2 * NP, NH = NP + 1, NFC = 4 * NP * NP * NP + 4;
  constexpr int NSURF = NP * NP * NP - (NP - 2) * (NP - 2) * (NP - 2);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpc = blockDim.x >> 5;
  int* c_of = reinterpret_cast<int*>(smem_raw);                      // full -> compact (< 0: conj of -c-1)
  int* m_of = c_of + N * N * NH;                                     // grid point (i,j,k) -> surface index or -1
  for (int e = threadIdx.x; e < N * N * NH; e += blockDim.x) c_of[e] = g.ff2c[e];
  for (int e = threadIdx.x; e < NP * NP * NP; e += blockDim.x) m_of[e] = -1;
  __syncthreads();
  for (int m = threadIdx.x; m < NSURF; m += blockDim.x)
    m_of[(g.surf_ijk[3 * m] * NP + g.surf_ijk[3 * m + 1]) * NP + g.surf_ijk[3 * m + 2]] = m;
  // the sibling-group-major FP32 form stages each node's spectrum first
  constexpr bool kStage = sizeof(T) == 4;
  const bool stage_sg = kStage && g.effval_sg;
  const size_t per_warp = inv_rb_warp_bytes<T>(NP, N, NH) + (stage_sg ? inv_rb_stage_bytes<T>(NP) : 0);
  unsigned char* mine = smem_raw + align16(sizeof(int) * (N * N * NH + NP * NP * NP)) + (size_t)warp * per_warp;
  Cpx<T>* Bm = reinterpret_cast<Cpx<T>*>(mine);
  Cpx<T>* A = reinterpret_cast<Cpx<T>*>(mine + align16(sizeof(Cpx<T>) * NP * N * NH));
  Cpx<T>* stage = reinterpret_cast<Cpx<T>*>(mine + inv_rb_warp_bytes<T>(NP, N, NH));
  __syncthreads();
  for (int wi = blockIdx.x * wpc + warp; wi < nwork; wi += gridDim.x * wpc) {
    const int node = work[wi];
    T* dst = tdncval + (size_t)node * NSURF * g.td;
    for (int t = 0; t < g.td; t++) {
      const Cpx<T>* src = reinterpret_cast<const Cpx<T>*>(effval + ((size_t)node * g.td + t) * NFC * 2);
      // sibling-group-major accumulated spectra: value c of dof t at
      // t * plane + spectra_sg_index; the node's 4 values of each chunk of 4
      // frequencies (32 bytes at a 256-byte stride) are copied into the
      // warp's stage all at once, so the warp waits for memory once per node
      // (the stage was last read by the previous z pass, which ends in a
      // __syncwarp)
      const Cpx<T>* srcg = reinterpret_cast<const Cpx<T>*>(effval) + t * g.plane + spectra_sg_index(NFC, node, 0);
      if constexpr (kStage) {
        if (stage_sg) {
          for (int b = lane; b < NFC / 4; b += 32) {
            const unsigned d0 = (unsigned)__cvta_generic_to_shared(stage + 4 * b);
            const Cpx<T>* s0 = srcg + 32 * b;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d0), "l"(s0) : "memory");
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d0 + 16), "l"(s0 + 2) : "memory");
          }
          asm volatile("cp.async.wait_all;" ::: "memory");
          __syncwarp();
        }
      }
      // z pass (inverse), lines (ky, kx): Bm[k][ky][kx] = sum_kz Y[kz][ky][kx] w^(-k kz), k < np
      for (int line = lane; line < N * NH; line += 32) {
        const int kx = line % NH, ky = line / NH;
        Cpx<T> y[N];
#pragma unroll
        for (int kz = 0; kz < N; kz++) {
          const int c = c_of[(kz * N + ky) * NH + kx];
          const int ca = c >= 0 ? c : -c - 1;
          Cpx<T> v = stage_sg ? stage[ca] : g.effval_sg ? srcg[(ca >> 2) * 32 + (ca & 3)] : src[ca];
          if (c < 0) v.im = -v.im;
          y[kz] = v;
        }
#pragma unroll
        for (int k = 0; k < NP; k++) {
          T re = 0, im = 0;
#pragma unroll
          for (int kz = 0; kz < N; kz++) {
            const T cr = twr<T, N>(k * kz), ci = twi<T, N>(k * kz);
            re = fmt(y[kz].im, ci, fmt(y[kz].re, cr, re));
            im = fmt(-y[kz].re, ci, fmt(y[kz].im, cr, im));
          }
          Bm[(k * N + ky) * NH + kx] = Cpx<T>{re, im};
        }
      }
      __syncwarp();
      // y pass (inverse), lines (k, kx): A[k][j][kx] = sum_ky Bm[k][ky][kx] w^(-j ky), j < np
      for (int line = lane; line < NP * NH; line += 32) {
        const int kx = line % NH, k = line / NH;
        Cpx<T> b[N];
#pragma unroll
        for (int ky = 0; ky < N; ky++) b[ky] = Bm[(k * N + ky) * NH + kx];
#pragma unroll
        for (int j = 0; j < NP; j++) {
          T re = 0, im = 0;
#pragma unroll
          for (int ky = 0; ky < N; ky++) {
            const T cr = twr<T, N>(j * ky), ci = twi<T, N>(j * ky);
            re = fmt(b[ky].im, ci, fmt(b[ky].re, cr, re));
            im = fmt(-b[ky].re, ci, fmt(b[ky].im, cr, im));
          }
          A[(k * NP + j) * NH + kx] = Cpx<T>{re, im};
        }
      }
      __syncwarp();
      // c2r along x, lines (j, k): x_i = Re(a_0) + (-1)^i Re(a_{n/2}) + 2 sum_{0<kx<n/2} Re(a_kx w^(-i kx)),
      // kept at the surface points only
      for (int line = lane; line < NP * NP; line += 32) {
        const int j = line % NP, k = line / NP;
        Cpx<T> a[NH];
#pragma unroll
        for (int kx = 0; kx < NH; kx++) a[kx] = A[(k * NP + j) * NH + kx];
#pragma unroll
        for (int i = 0; i < NP; i++) {
          const int m = m_of[(i * NP + j) * NP + k];
          if (m < 0) continue;
          T acc = 0;
#pragma unroll
          for (int kx = 1; kx < NH - 1; kx++)
            acc = fmt(a[kx].im, twi<T, N>(i * kx), fmt(a[kx].re, twr<T, N>(i * kx), acc));
          const T v = a[0].re + ((i & 1) ? -a[NH - 1].re : a[NH - 1].re);
          dst[(size_t)m * g.td + t] += v + T(2) * acc;
        }
      }
      __syncwarp();
    }
  }
}

}  // namespace

template <typename T>
void launch_m2l_forward(const M2LGeom& g, const T* supeden, const int* nodes, int nn, const int* depth, T* spectra,
                        cudaStream_t st) {
  if (nn <= 0) return;
  // warp per node; as many warps per CTA (<= 8) as fit in ~200 KB of shared memory
  const size_t per_warp = fwd_warp_bytes<T>(g.np, g.n, g.nh);
  const size_t head = align16(sizeof(Cpx<T>) * g.n * g.n);
  int wpc = (int)std::max<size_t>(1, std::min<size_t>(8, (200 * 1024 - head) / per_warp));
  size_t smem = head + per_warp * wpc;
  int grid = std::max(1, std::min((nn + wpc - 1) / wpc, 148 * 8));
  if (g.np == 4 || g.np == 6 || g.np == 8) {
    const size_t head_rb = align16(sizeof(int) * g.n * g.n * g.nh);
    const size_t per_rb = fwd_rb_warp_bytes<T>(g.np, g.n, g.nh);
    const int w = (int)std::max<size_t>(1, std::min<size_t>(8, (200 * 1024 - head_rb) / per_rb));
    const size_t sm = head_rb + per_rb * w;
    const int gr = std::max(1, std::min((nn + w - 1) / w, 148 * 8));
    auto kern = g.np == 6 ? k_m2l_fwd_rb<T, 6> : g.np == 4 ? k_m2l_fwd_rb<T, 4> : k_m2l_fwd_rb<T, 8>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    kern<<<gr, 32 * w, sm, st>>>(g, supeden, nodes, nn, depth, spectra);
    return;
  }
  cudaFuncSetAttribute(k_m2l_fwd_warp<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_m2l_fwd_warp<T, 0><<<grid, 32 * wpc, smem, st>>>(g, supeden, nodes, nn, depth, spectra);
}

template <typename T>
void launch_m2l_hadamard(const M2LGeom& g, const T* khat, const T* spectra, const int* work, int nwork,
                         const int64_t* vptr, const int* vidx, const int* path, T* effval, cudaStream_t st) {
  if (nwork <= 0) return;
  if (g.sd == 1 && g.td == 1)
    k_m2l_had<T, 1, 1><<<nwork, FFT_THREADS, 0, st>>>(g, khat, spectra, work, vptr, vidx, path, effval);
  else if (g.sd == 4 && g.td == 3)
    k_m2l_had<T, 4, 3><<<nwork, FFT_THREADS, 0, st>>>(g, khat, spectra, work, vptr, vidx, path, effval);
  else if (g.sd == 3 && g.td == 3)
    k_m2l_had<T, 3, 3><<<nwork, FFT_THREADS, 0, st>>>(g, khat, spectra, work, vptr, vidx, path, effval);
}

template <typename T>
void launch_m2l_inverse(const M2LGeom& g, const T* effval, const int* work, int nwork, T* tdncval, cudaStream_t st) {
  if (nwork <= 0) return;
  const size_t per_warp = inv_warp_bytes<T>(g.np, g.n, g.nh);
  const size_t head = align16(sizeof(Cpx<T>) * g.n * g.n);
  int wpc = (int)std::max<size_t>(1, std::min<size_t>(8, (200 * 1024 - head) / per_warp));
  size_t smem = head + per_warp * wpc;
  int grid = std::max(1, std::min((nwork + wpc - 1) / wpc, 148 * 8));
  if (g.np == 4 || g.np == 6 || g.np == 8) {
    const size_t per_rb =
        inv_rb_warp_bytes<T>(g.np, g.n, g.nh) + (sizeof(T) == 4 && g.effval_sg ? inv_rb_stage_bytes<T>(g.np) : 0);
    const size_t head_rb = align16(sizeof(int) * (g.n * g.n * g.nh + g.np * g.np * g.np));
    const int w = (int)std::max<size_t>(1, std::min<size_t>(8, (200 * 1024 - head_rb) / per_rb));
    const size_t sm = head_rb + per_rb * w;
    const int gr = std::max(1, std::min((nwork + w - 1) / w, 148 * 8));
    auto kern = g.np == 6 ? k_m2l_inv_rb<T, 6> : g.np == 4 ? k_m2l_inv_rb<T, 4> : k_m2l_inv_rb<T, 8>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    kern<<<gr, 32 * w, sm, st>>>(g, effval, work, nwork, tdncval);
    return;
  }
  cudaFuncSetAttribute(k_m2l_inv_warp<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_m2l_inv_warp<T, 0><<<grid, 32 * wpc, smem, st>>>(g, effval, work, nwork, tdncval);
}

// ---------------------------------------------------------------------------
// Hadamard accumulation in parent-pair form (single-dof equivalent kernel).
//
// The V list of a node t is the set of children c of the 26 colleagues P of
// t's parent Q that are not adjacent to t (fmm3d/let3d.cpp:228-247), and the
// translation from c to t depends only on the offset 2*(P-Q) + oct(c) -
// oct(t), one of 316 values.  So per frequency the whole pass is, for every
// target parent Q, Y[Q's 8 children] += sum_dir M_dir * X[P_dir's 8 children]
// with 8x8 blocks drawn from the same 316 operator values.
//
// Persistent sweep: each CTA owns a contiguous slice of target parents (Morton
// order, so neighbouring parents share colleagues) and sweeps the frequency
// tiles in order.  All CTAs therefore work on about the same tile at the same
// time and its source spectra (nodes x 32 freq x 8 B, ~93 MB at 4M points)
// stay in L2 for their 26-fold reuse.  The next colleague's 8 child spectra
// are loaded into registers while the current colleague is multiplied.
//
// The operator tile of a frequency tile (all 343 offsets x 32 frequencies,
// zero for |o| <= 1, stored contiguously per tile) is staged into shared
// memory by one bulk asynchronous copy completing on an mbarrier; with two
// buffers (FP32) the next tile's copy runs under the current tile's work.
// NF (frequencies per node) is a template argument, so the 8 child spectra
// of a colleague are 8 loads at immediate offsets from one address.  Absent
// colleagues point at an all-zero spectrum block (zero_node), so the loads
// need no predicate.  Every mbarrier wait is bounded: on time-out the kernel
// sets bit 0 of *status and returns.
namespace {

__device__ __constant__ short c_dir_base[26] = {57,  59,  61,  71,  73,  75,  85,  87,  89,  155, 157, 159, 169,
                                               173, 183, 185, 187, 253, 255, 257, 267, 269, 271, 281, 283, 285};

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity) {
  for (int it = 0; it < (1 << 22); it++) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// The work of one frequency tile for one warp: claim QPT target parents at a
// time from *claim until the CTA's slice [.., qend) is exhausted.
// SD / TD: dofs per node of the source / target spectra; this pass reads
// source component sc and adds into target component tc (first sc writes).
template <typename T, int NF, int QPT, int SD, int TD>
__device__ __forceinline__ void sweep_tile(const Cpx<T>* __restrict__ Ks, const Cpx<T>* __restrict__ spectra,
                                           int* claim, int qend, int f, const int* __restrict__ qchd,
                                           const int* __restrict__ coll, const unsigned char* __restrict__ mask,
                                           Cpx<T>* __restrict__ effval, int zero_node, int sc, int tc, bool acc) {
  constexpr int XS = SD * NF;  // source child stride
  const int lane = threadIdx.x & 31;
  const int fl = min(f, NF - 1);  // lanes past NF load a valid spectrum and store nothing
  while (true) {
    int q0 = 0;
    if (lane == 0) q0 = atomicAdd(claim, QPT);
    q0 = __shfl_sync(0xffffffffu, q0, 0);
    if (q0 >= qend) break;
    T ar[QPT][8], ai[QPT][8];
#pragma unroll
    for (int q = 0; q < QPT; q++)
#pragma unroll
      for (int i = 0; i < 8; i++) ar[q][i] = ai[q][i] = T(0);
    const int* cq[QPT];
#pragma unroll
    for (int q = 0; q < QPT; q++) cq[q] = coll + (size_t)min(q0 + q, qend - 1) * 26;
    // two register sets of colleague child spectra, alternating over the 26
    // directions: set B is loaded while set A is multiplied and vice versa
    int nbA[QPT], nbB[QPT];
    T axr[QPT][8], axi[QPT][8], bxr[QPT][8], bxi[QPT][8];
    auto load = [&](int dir, int* nb, T (*xr)[8], T (*xi)[8]) {
#pragma unroll
      for (int q = 0; q < QPT; q++) {
        nb[q] = (q0 + q < qend) ? cq[q][dir] : zero_node;
        const Cpx<T>* X = spectra + ((size_t)nb[q] * SD + sc) * NF + fl;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const Cpx<T> x = X[j * XS];
          xr[q][j] = x.re;
          xi[q][j] = x.im;
        }
      }
    };
    auto mult = [&](int dir, const int* nb, T (*xr)[8], T (*xi)[8]) {
      bool any = false;
#pragma unroll
      for (int q = 0; q < QPT; q++) any |= nb[q] != zero_node;
      if (!any) return;
      // offset of child j of P from child i of Q: 2*dir + oct(j) - oct(i); the
      // adjacent pairs (|offset| <= 1) read the zero rows of the tile
      const Cpx<T>* Kd = Ks + c_dir_base[dir] * 32 + lane;
#pragma unroll
      for (int j = 0; j < 8; j++) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int cij = (((j >> 2) & 1) - ((i >> 2) & 1)) * 49 + (((j >> 1) & 1) - ((i >> 1) & 1)) * 7 +
                          ((j & 1) - (i & 1));
          const Cpx<T> k = Kd[cij * 32];
#pragma unroll
          for (int q = 0; q < QPT; q++) {
            ar[q][i] = fmt(-k.im, xi[q][j], fmt(k.re, xr[q][j], ar[q][i]));
            ai[q][i] = fmt(k.im, xr[q][j], fmt(k.re, xi[q][j], ai[q][i]));
          }
        }
      }
    };
    load(0, nbA, axr, axi);
    for (int dir = 0; dir < 26; dir += 2) {
      load(dir + 1, nbB, bxr, bxi);
      mult(dir, nbA, axr, axi);
      if (dir + 2 < 26) load(dir + 2, nbA, axr, axi);
      mult(dir + 1, nbB, bxr, bxi);
    }
    if (f < NF) {
#pragma unroll
      for (int q = 0; q < QPT; q++) {
        if (q0 + q >= qend) continue;
        const int c0 = qchd[q0 + q];
        const unsigned m = mask[q0 + q];
#pragma unroll
        for (int i = 0; i < 8; i++) {
          if (!((m >> i) & 1)) continue;
          Cpx<T>* py = effval + ((size_t)(c0 + i) * TD + tc) * NF + f;
          Cpx<T> y;
          y.re = ar[q][i];
          y.im = ai[q][i];
          if (acc) {
            const Cpx<T> o = *py;
            y.re += o.re;
            y.im += o.im;
          }
          *py = y;
        }
      }
    }
  }
}

// NBUF = 2 (FP32): no CTA-wide barrier inside the sweep.  Each warp walks the
// frequency tiles on its own; the last warp to finish a tile (a shared
// counter) resets that buffer's claim counter and issues the copy of the tile
// two ahead into it, so warps drift apart by at most one tile.  The copy's
// mbarrier arrive releases the reset to the warps that wait on that buffer.
// NBUF = 1 (FP64, one 176 KB tile): the tile is reloaded between two CTA
// barriers.
template <typename T, int NF, int QPT, int NTHR, int NBUF, int SD, int TD>
__global__ void __launch_bounds__(NTHR) k_m2l_had_sweep(const Cpx<T>* __restrict__ ktiles,
                                                       const Cpx<T>* __restrict__ spectra, int nq,
                                                       const int* __restrict__ qchd, const int* __restrict__ coll,
                                                       const unsigned char* __restrict__ mask,
                                                       Cpx<T>* __restrict__ effval, int zero_node, int sc, int tc,
                                                       int acc, int* __restrict__ status) {
  constexpr int TILE = 343 * 32;
  constexpr unsigned TILE_BYTES = TILE * sizeof(Cpx<T>);
  constexpr int FTILES = (NF + 31) / 32;
  constexpr int NW = NTHR / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cpx<T>* Kbuf = reinterpret_cast<Cpx<T>*>(smem_raw);  // NBUF x [343][32]
  __shared__ __align__(8) unsigned long long bars[NBUF];
  __shared__ int claim[NBUF], done_cnt[NBUF];
  const int lane = threadIdx.x & 31;
  const int per_cta = (nq + gridDim.x - 1) / gridDim.x;
  const int qbeg = blockIdx.x * per_cta;
  const int qend = min(nq, qbeg + per_cta);
  if (threadIdx.x == 0) {
    for (int b = 0; b < NBUF; b++) {
      mbar_init(smem_addr(&bars[b]), 1);
      claim[b] = qbeg;
      done_cnt[b] = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (NBUF == 2) {
      bulk_load(smem_addr(Kbuf), ktiles, TILE_BYTES, smem_addr(&bars[0]));
      if (FTILES > 1) bulk_load(smem_addr(Kbuf + TILE), ktiles + TILE, TILE_BYTES, smem_addr(&bars[1]));
    }
  }
  __syncthreads();
  if constexpr (NBUF == 2) {
    for (int ft = 0; ft < FTILES; ft++) {
      const int b = ft & 1;
      const bool ok = mbar_wait_bounded(smem_addr(&bars[b]), (ft >> 1) & 1);
      if (!ok) {  // the warp stops; the others then time out on the tiles it never releases
        if (lane == 0) atomicOr(status, 1);
        return;
      }
      sweep_tile<T, NF, QPT, SD, TD>(Kbuf + (size_t)b * TILE, spectra, &claim[b], qend, ft * 32 + lane, qchd, coll,
                                     mask, effval, zero_node, sc, tc, acc != 0);
      if (lane == 0) {
        if (atomicAdd(&done_cnt[b], 1) == NW - 1) {  // the last warp out of tile ft
          done_cnt[b] = 0;
          claim[b] = qbeg;
          if (ft + 2 < FTILES)
            bulk_load(smem_addr(Kbuf + (size_t)b * TILE), ktiles + (size_t)(ft + 2) * TILE, TILE_BYTES,
                      smem_addr(&bars[b]));
        }
      }
      __syncwarp();
    }
  } else {
    for (int ft = 0; ft < FTILES; ft++) {
      if (threadIdx.x == 0) {
        claim[0] = qbeg;
        bulk_load(smem_addr(Kbuf), ktiles + (size_t)ft * TILE, TILE_BYTES, smem_addr(&bars[0]));
      }
      __syncthreads();
      const bool ok = mbar_wait_bounded(smem_addr(&bars[0]), ft & 1);
      if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(status, 1);
        return;
      }
      sweep_tile<T, NF, QPT, SD, TD>(Kbuf, spectra, &claim[0], qend, ft * 32 + lane, qchd, coll, mask, effval,
                                     zero_node, sc, tc, acc != 0);
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// Toeplitz-factored parent-pair Hadamard.  For one colleague direction d the
// child-to-child block is M[i][j] = K(2d + oct(j) - oct(i)): along each axis a
// 2 x 2 Toeplitz matrix [[t0, t1], [t-1, t0]], whose product needs three
// multiplications instead of four:
//   y0 = A + B, y1 = A + C,  A = t0 (x0 + x1), B = (t1 - t0) x1, C = (t-1 - t0) x0.
// Over the three axes that is 27 products U_k T_k instead of 64.  The input
// combinations U_k (x0 + x1, x1, x0 per axis) do not depend on d and the output
// combination is linear, so each lane accumulates sum_d T_k(d) U_k(d) for all
// 27 k and applies the output combination once per target parent.  Per
// frequency and direction: 27 complex multiply-adds and 19 complex adds in
// place of 64 complex multiply-adds.  The transformed operator T[d][k] (26 x 27
// values per frequency, products of the differences above, formed in FP64 on
// the host) is staged per tile of 16 frequencies; a warp carries two target
// parents, one per half-warp, on the same 16 frequencies.
constexpr int TZ_F = 16;          // frequencies per tile
constexpr int TZ_ROWS = 26 * 28;  // transformed operator values per frequency (27 per direction, padded to 28)

// two consecutive transformed operator values of one frequency: layout
// [dir][k/2][16][2] lets one 16-byte shared load (FP32) fetch both
template <typename T>
struct __align__(4 * sizeof(T)) Cpx2 {
  Cpx<T> a, b;
};

template <typename T>
__device__ __forceinline__ void cadd(Cpx<T>& r, const Cpx<T>& a, const Cpx<T>& b) {
  r.re = a.re + b.re;
  r.im = a.im + b.im;
}

template <typename T, int NF, int SD, int TD>
__device__ __forceinline__ void tz_tile(const Cpx<T>* __restrict__ Ts, const Cpx<T>* __restrict__ spectra,
                                        int* claim, int qend, int f, const int* __restrict__ qchd,
                                        const int* __restrict__ coll, const unsigned char* __restrict__ mask,
                                        Cpx<T>* __restrict__ effval, int zero_node, int sc, int tc, bool acc_out) {
  constexpr int XS = SD * NF;  // source child stride
  const int lane = threadIdx.x & 31, hl = lane & 15, hw = lane >> 4;
  const int fl = min(f, NF - 1);  // lanes past NF load a valid spectrum and store nothing
  while (true) {
    int q0 = 0;
    if (lane == 0) q0 = atomicAdd(claim, 2);
    q0 = __shfl_sync(0xffffffffu, q0, 0);
    if (q0 >= qend) break;
    const int q = q0 + hw;  // this half-warp's target parent
    const bool qv = q < qend;
    const int* cq = coll + (size_t)min(q, qend - 1) * 26;
    Cpx<T> acc[27];
#pragma unroll
    for (int k = 0; k < 27; k++) acc[k].re = acc[k].im = T(0);
    Cpx<T> xa[8], xb[8];
    int nba, nbb;
    auto load = [&](int dir, Cpx<T>* x, int& nb) {
      nb = qv ? cq[dir] : zero_node;
      const Cpx<T>* X = spectra + ((size_t)nb * SD + sc) * NF + fl;
#pragma unroll
      for (int j = 0; j < 8; j++) x[j] = X[j * XS];
    };
    auto mult = [&](int dir, const Cpx<T>* x, int nb) {
      if (!__any_sync(0xffffffffu, nb != zero_node)) return;
      const Cpx2<T>* Td = reinterpret_cast<const Cpx2<T>*>(Ts) + (size_t)dir * 14 * TZ_F + hl;
      Cpx2<T> tp;
      // child j = (jx, jy, jz) bits (2, 1, 0); per axis the combinations
      // A = x(0) + x(1), B = x(1), C = x(0)
#pragma unroll
      for (int kx = 0; kx < 3; kx++) {
        Cpx<T> v[4];  // [jy][jz]
#pragma unroll
        for (int e = 0; e < 4; e++) {
          if (kx == 0) cadd(v[e], x[e], x[4 + e]);
          else v[e] = kx == 1 ? x[4 + e] : x[e];
        }
#pragma unroll
        for (int ky = 0; ky < 3; ky++) {
          Cpx<T> w[2];  // [jz]
#pragma unroll
          for (int e = 0; e < 2; e++) {
            if (ky == 0) cadd(w[e], v[e], v[2 + e]);
            else w[e] = ky == 1 ? v[2 + e] : v[e];
          }
#pragma unroll
          for (int kz = 0; kz < 3; kz++) {
            Cpx<T> u;
            if (kz == 0) cadd(u, w[0], w[1]);
            else u = kz == 1 ? w[1] : w[0];
            const int k = (kx * 3 + ky) * 3 + kz;
            if ((k & 1) == 0) tp = Td[(k >> 1) * TZ_F];
            const Cpx<T> t = (k & 1) ? tp.b : tp.a;
            acc[k].re = fmt(-t.im, u.im, fmt(t.re, u.re, acc[k].re));
            acc[k].im = fmt(t.im, u.re, fmt(t.re, u.im, acc[k].im));
          }
        }
      }
    };
    load(0, xa, nba);
    for (int dir = 0; dir < 26; dir += 2) {
      load(dir + 1, xb, nbb);
      mult(dir, xa, nba);
      if (dir + 2 < 26) load(dir + 2, xa, nba);
      mult(dir + 1, xb, nbb);
    }
    if (!qv || f >= NF) continue;
    // output combination per axis: y(0) = A + B, y(1) = A + C
    Cpx<T> r[18];  // [kx][ky][iz]
#pragma unroll
    for (int g = 0; g < 9; g++) {
      cadd(r[2 * g], acc[3 * g], acc[3 * g + 1]);
      cadd(r[2 * g + 1], acc[3 * g], acc[3 * g + 2]);
    }
    Cpx<T> s4[12];  // [kx][iy][iz]
#pragma unroll
    for (int kx = 0; kx < 3; kx++)
#pragma unroll
      for (int iz = 0; iz < 2; iz++) {
        const Cpx<T> a0 = r[(kx * 3 + 0) * 2 + iz], b0 = r[(kx * 3 + 1) * 2 + iz], c0 = r[(kx * 3 + 2) * 2 + iz];
        cadd(s4[(kx * 2 + 0) * 2 + iz], a0, b0);
        cadd(s4[(kx * 2 + 1) * 2 + iz], a0, c0);
      }
    const int c0 = qchd[q];
    const unsigned m = mask[q];
#pragma unroll
    for (int e = 0; e < 4; e++) {  // (iy, iz)
      Cpx<T> y[2];
      cadd(y[0], s4[0 * 4 + e], s4[1 * 4 + e]);
      cadd(y[1], s4[0 * 4 + e], s4[2 * 4 + e]);
#pragma unroll
      for (int ix = 0; ix < 2; ix++) {
        const int i = ix * 4 + e;
        if (!((m >> i) & 1)) continue;
        Cpx<T>* py = effval + ((size_t)(c0 + i) * TD + tc) * NF + f;
        Cpx<T> v = y[ix];
        if (acc_out) {
          const Cpx<T> o = *py;
          v.re += o.re;
          v.im += o.im;
        }
        *py = v;
      }
    }
  }
}

template <typename T, int NF, int NTHR, int NBUF, int SD, int TD>
__global__ void __launch_bounds__(NTHR) k_m2l_had_tz(const Cpx<T>* __restrict__ ttiles,
                                                    const Cpx<T>* __restrict__ spectra, int nq,
                                                    const int* __restrict__ qchd, const int* __restrict__ coll,
                                                    const unsigned char* __restrict__ mask,
                                                    Cpx<T>* __restrict__ effval, int zero_node, int sc, int tc, int acc,
                                                    int* __restrict__ status) {
  constexpr int TILE = TZ_ROWS * TZ_F;
  constexpr unsigned TILE_BYTES = TILE * sizeof(Cpx<T>);
  constexpr int FTILES = (NF + TZ_F - 1) / TZ_F;
  constexpr int NW = NTHR / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cpx<T>* Tbuf = reinterpret_cast<Cpx<T>*>(smem_raw);  // NBUF x [26][27][16]
  __shared__ __align__(8) unsigned long long bars[NBUF];
  __shared__ int claim[NBUF], done_cnt[NBUF];
  const int lane = threadIdx.x & 31;
  const int per_cta = (nq + gridDim.x - 1) / gridDim.x;
  const int qbeg = blockIdx.x * per_cta;
  const int qend = min(nq, qbeg + per_cta);
  if (threadIdx.x == 0) {
    for (int b = 0; b < NBUF; b++) {
      mbar_init(smem_addr(&bars[b]), 1);
      claim[b] = qbeg;
      done_cnt[b] = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (NBUF == 2) {
      bulk_load(smem_addr(Tbuf), ttiles, TILE_BYTES, smem_addr(&bars[0]));
      if (FTILES > 1) bulk_load(smem_addr(Tbuf + TILE), ttiles + TILE, TILE_BYTES, smem_addr(&bars[1]));
    }
  }
  __syncthreads();
  if constexpr (NBUF == 2) {
    for (int ft = 0; ft < FTILES; ft++) {
      const int b = ft & 1;
      const bool ok = mbar_wait_bounded(smem_addr(&bars[b]), (ft >> 1) & 1);
      if (!ok) {
        if (lane == 0) atomicOr(status, 1);
        return;
      }
      tz_tile<T, NF, SD, TD>(Tbuf + (size_t)b * TILE, spectra, &claim[b], qend, ft * TZ_F + (lane & 15), qchd, coll,
                             mask, effval, zero_node, sc, tc, acc != 0);
      if (lane == 0) {
        if (atomicAdd(&done_cnt[b], 1) == NW - 1) {  // the last warp out of tile ft
          done_cnt[b] = 0;
          claim[b] = qbeg;
          if (ft + 2 < FTILES)
            bulk_load(smem_addr(Tbuf + (size_t)b * TILE), ttiles + (size_t)(ft + 2) * TILE, TILE_BYTES,
                      smem_addr(&bars[b]));
        }
      }
      __syncwarp();
    }
  } else {
    for (int ft = 0; ft < FTILES; ft++) {
      if (threadIdx.x == 0) {
        claim[0] = qbeg;
        bulk_load(smem_addr(Tbuf), ttiles + (size_t)ft * TILE, TILE_BYTES, smem_addr(&bars[0]));
      }
      __syncthreads();
      const bool ok = mbar_wait_bounded(smem_addr(&bars[0]), ft & 1);
      if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(status, 1);
        return;
      }
      tz_tile<T, NF, SD, TD>(Tbuf, spectra, &claim[0], qend, ft * TZ_F + (lane & 15), qchd, coll, mask, effval,
                             zero_node, sc, tc, acc != 0);
      __syncthreads();
    }
  }
}

template <typename T, int NF, int SD, int TD>
void tz_launch(const T* ttiles, const T* spectra, int nq, const int* qchd, const int* coll, const unsigned char* mask,
               T* effval, int zero_node, int* status, int num_sms, cudaStream_t st) {
  constexpr int NTHR = sizeof(T) == 4 ? 512 : 256;
  constexpr int NBUF = sizeof(T) == 4 ? 2 : 1;
  const size_t smem = (size_t)NBUF * TZ_ROWS * TZ_F * sizeof(Cpx<T>);
  auto kern = k_m2l_had_tz<T, NF, NTHR, NBUF, SD, TD>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int grid = std::max(1, std::min(num_sms, nq / 32));
  const size_t tiles = (size_t)((NF + TZ_F - 1) / TZ_F) * TZ_ROWS * TZ_F;  // Cpx per (t, s) table
  for (int t = 0; t < TD; t++)
    for (int s = 0; s < SD; s++)
      kern<<<grid, NTHR, smem, st>>>(reinterpret_cast<const Cpx<T>*>(ttiles) + (size_t)(t * SD + s) * tiles,
                                     reinterpret_cast<const Cpx<T>*>(spectra), nq, qchd, coll, mask,
                                     reinterpret_cast<Cpx<T>*>(effval), zero_node, s, t, s > 0 ? 1 : 0, status);
}

template <typename T, int NF>
void tz_dofs(int sd, int td, const T* ttiles, const T* spectra, int nq, const int* qchd, const int* coll,
             const unsigned char* mask, T* effval, int zero_node, int* status, int num_sms, cudaStream_t st) {
  if (sd == 1 && td == 1)
    tz_launch<T, NF, 1, 1>(ttiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
  else if (sd == 4 && td == 3)
    tz_launch<T, NF, 4, 3>(ttiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
  else if (sd == 3 && td == 3)
    tz_launch<T, NF, 3, 3>(ttiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
}

template <typename T, int NF, int SD, int TD>
void sweep_launch(const T* ktiles, const T* spectra, int nq, const int* qchd, const int* coll,
                  const unsigned char* mask, T* effval, int zero_node, int* status, int num_sms, cudaStream_t st) {
  constexpr int QPT = 2;
  // one CTA per SM: 16 warps (FP32, operator tile double-buffered) or 8 warps
  // (FP64: twice the registers, one 176 KB tile)
  constexpr int NTHR = sizeof(T) == 4 ? 512 : 256;
  constexpr int NBUF = sizeof(T) == 4 ? 2 : 1;
  const size_t smem = (size_t)NBUF * 343 * 32 * sizeof(Cpx<T>);
  auto kern = k_m2l_had_sweep<T, NF, QPT, NTHR, NBUF, SD, TD>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  // at least 32 target parents per CTA: each CTA streams every operator tile
  // (28 x 88 KB at np = 6), which a handful of parents would not amortise
  const int grid = std::max(1, std::min(num_sms, nq / 32));
  const size_t tiles = (size_t)((NF + 31) / 32) * 343 * 32;  // Cpx per (t, s) operator table
  // one pass per (target dof, source dof); the first source dof writes
  for (int t = 0; t < TD; t++)
    for (int s = 0; s < SD; s++)
      kern<<<grid, NTHR, smem, st>>>(reinterpret_cast<const Cpx<T>*>(ktiles) + (size_t)(t * SD + s) * tiles,
                                     reinterpret_cast<const Cpx<T>*>(spectra), nq, qchd, coll, mask,
                                     reinterpret_cast<Cpx<T>*>(effval), zero_node, s, t, s > 0 ? 1 : 0, status);
}

template <typename T, int NF>
void sweep_dofs(int sd, int td, const T* ktiles, const T* spectra, int nq, const int* qchd, const int* coll,
                const unsigned char* mask, T* effval, int zero_node, int* status, int num_sms, cudaStream_t st) {
  if (sd == 1 && td == 1)
    sweep_launch<T, NF, 1, 1>(ktiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
  else if (sd == 4 && td == 3)
    sweep_launch<T, NF, 4, 3>(ktiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
  else if (sd == 3 && td == 3)
    sweep_launch<T, NF, 3, 3>(ktiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
}

}  // namespace

bool m2l_sweep_supported(int nf, int sd, int td) {
  return (nf == 260 || nf == 868 || nf == 2052) &&
         ((sd == 1 && td == 1) || (sd == 4 && td == 3) || (sd == 3 && td == 3));
}

template <typename T>
void launch_m2l_hadamard_sweep(int nf, int sd, int td, const T* ktiles, const T* spectra, int nq, const int* qchd,
                               const int* coll, const unsigned char* mask, T* effval, int zero_node, int* status,
                               int num_sms, cudaStream_t st) {
  if (nq <= 0) return;
  if (nf == 868)
    sweep_dofs<T, 868>(sd, td, ktiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
  else if (nf == 260)
    sweep_dofs<T, 260>(sd, td, ktiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
  else if (nf == 2052)
    sweep_dofs<T, 2052>(sd, td, ktiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
}

template <typename T>
void launch_m2l_hadamard_tz(int nf, int sd, int td, const T* ttiles, const T* spectra, int nq, const int* qchd,
                            const int* coll, const unsigned char* mask, T* effval, int zero_node, int* status,
                            int num_sms, cudaStream_t st) {
  if (nq <= 0) return;
  if (nf == 868)
    tz_dofs<T, 868>(sd, td, ttiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
  else if (nf == 260)
    tz_dofs<T, 260>(sd, td, ttiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
  else if (nf == 2052)
    tz_dofs<T, 2052>(sd, td, ttiles, spectra, nq, qchd, coll, mask, effval, zero_node, status, num_sms, st);
}

#define KIFMM_INST(T)                                                                                             \
  template void launch_m2l_hadamard_sweep<T>(int, int, int, const T*, const T*, int, const int*, const int*,     \
                                             const unsigned char*, T*, int, int*, int, cudaStream_t);              \
  template void launch_m2l_hadamard_tz<T>(int, int, int, const T*, const T*, int, const int*, const int*,        \
                                          const unsigned char*, T*, int, int*, int, cudaStream_t);                 \
  template void launch_m2l_forward<T>(const M2LGeom&, const T*, const int*, int, const int*, T*, cudaStream_t);  \
  template void launch_m2l_hadamard<T>(const M2LGeom&, const T*, const T*, const int*, int, const int64_t*,     \
                                       const int*, const int*, T*, cudaStream_t);                                \
  template void launch_m2l_inverse<T>(const M2LGeom&, const T*, const int*, int, T*, cudaStream_t);
KIFMM_INST(double)
KIFMM_INST(float)
#undef KIFMM_INST

}  // namespace kifmm
