// Device-side kernel library shared by every pass.
//
// keval<KT,T>() adds one source's contribution to one target's potential
// without forming the interaction matrix; it is the fused form of
// Kernel3d::kernel + dgemv (fmm3d/kernel3d.cpp:116-414 and
// common/vecmatop.cpp:97-113) used by SE2TC/SE2UC/SE2DC/DE2TC/UE2TC
// (fmm3d/fmm3d.cpp:35-141).  x = target - source, as in the reference.
// The singular cut-off r < 1e-8 -> 0 (fmm3d/kernel3d.cpp:21) becomes
// 1/r := 0 for r^2 < 1e-16, which zeroes every term of every kernel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace kifmm {

constexpr int KT_LAP_S = 111, KT_LAP_D = 121, KT_STK_F = 301, KT_STK_S = 311, KT_STK_SP = 312, KT_STK_D = 321,
              KT_STK_DP = 322, KT_NAV_S = 511, KT_NAV_D = 521;

template <int KT> struct KTraits;
template <> struct KTraits<111> { static constexpr int SD = 1, TD = 1; static constexpr bool DL = false; static constexpr int MM = 111; };
template <> struct KTraits<121> { static constexpr int SD = 1, TD = 1; static constexpr bool DL = true;  static constexpr int MM = 111; };
template <> struct KTraits<301> { static constexpr int SD = 4, TD = 3; static constexpr bool DL = false; static constexpr int MM = 301; };
template <> struct KTraits<311> { static constexpr int SD = 3, TD = 3; static constexpr bool DL = false; static constexpr int MM = 301; };
template <> struct KTraits<312> { static constexpr int SD = 3, TD = 1; static constexpr bool DL = false; static constexpr int MM = 111; };
template <> struct KTraits<321> { static constexpr int SD = 3, TD = 3; static constexpr bool DL = true;  static constexpr int MM = 301; };
template <> struct KTraits<322> { static constexpr int SD = 3, TD = 1; static constexpr bool DL = true;  static constexpr int MM = 111; };
template <> struct KTraits<511> { static constexpr int SD = 3, TD = 3; static constexpr bool DL = false; static constexpr int MM = 511; };
template <> struct KTraits<521> { static constexpr int SD = 3, TD = 3; static constexpr bool DL = true;  static constexpr int MM = 511; };

// Kernel constants, precomputed on the host in FP64 and rounded to T.
template <typename T>
struct KConst {
  T c0, c1, c2;
};

#ifdef __CUDACC__
// explicit fused multiply-add a*b + c: `u += p*q + r*s` written with two of
// these is two instructions, where the expression form leaves an unfused
// product and a separate add
__device__ __forceinline__ float fmt(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmt(double a, double b, double c) { return __fma_rn(a, b, c); }

// FP32: the hardware approximation with denormal inputs flushed (every caller
// has r^2 >= 1e-16), which drops the denormal rescaling steps of rsqrtf
__device__ __forceinline__ float rsqrt_t(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }

template <int KT, typename T>
__device__ __forceinline__ void keval(T x, T y, T z, const T* nrm, const T* f, T* u, const KConst<T>& k) {
  T r2 = x * x + y * y + z * z;
  T ri = (r2 >= T(1e-16)) ? rsqrt_t(r2) : T(0);
  if constexpr (KT == 111) {  // 1/(4 pi r)
    u[0] += k.c0 * ri * f[0];
  } else if constexpr (KT == 121) {  // -(r.n)/(4 pi r^3)
    T rn = x * nrm[0] + y * nrm[1] + z * nrm[2];
    u[0] += k.c0 * ri * ri * ri * rn * f[0];
  } else if constexpr (KT == 301) {  // Stokeslet + r/(4 pi r^3) column
    T ri3 = ri * ri * ri;
    T xf = x * f[0] + y * f[1] + z * f[2];
    T g1 = k.c0 * ri, g3 = k.c0 * ri3 * xf, a3 = k.c1 * ri3 * f[3];
    const T g = g3 + a3;
    u[0] = fmt(g, x, fmt(g1, f[0], u[0]));
    u[1] = fmt(g, y, fmt(g1, f[1], u[1]));
    u[2] = fmt(g, z, fmt(g1, f[2], u[2]));
  } else if constexpr (KT == 311) {  // (delta/r + r r^T / r^3) / (8 pi mu)
    T xf = x * f[0] + y * f[1] + z * f[2];
    T g1 = k.c0 * ri, g3 = k.c0 * ri * ri * ri * xf;
    u[0] = fmt(g3, x, fmt(g1, f[0], u[0]));
    u[1] = fmt(g3, y, fmt(g1, f[1], u[1]));
    u[2] = fmt(g3, z, fmt(g1, f[2], u[2]));
  } else if constexpr (KT == 312) {  // (r.f) / (4 pi r^3)
    T xf = x * f[0] + y * f[1] + z * f[2];
    u[0] += k.c0 * ri * ri * ri * xf;
  } else if constexpr (KT == 321) {  // -6/(8 pi) (r.n) r r^T / r^5
    T xf = x * f[0] + y * f[1] + z * f[2];
    T rn = x * nrm[0] + y * nrm[1] + z * nrm[2];
    T ri2 = ri * ri;
    T c = k.c0 * ri2 * ri2 * ri * rn * xf;
    u[0] += c * x;
    u[1] += c * y;
    u[2] += c * z;
  } else if constexpr (KT == 322) {  // mu/(2 pi) (n.f/r^3 - 3 (r.n)(r.f)/r^5)
    T xf = x * f[0] + y * f[1] + z * f[2];
    T nf = nrm[0] * f[0] + nrm[1] * f[1] + nrm[2] * f[2];
    T rn = x * nrm[0] + y * nrm[1] + z * nrm[2];
    T ri2 = ri * ri, ri3 = ri2 * ri;
    u[0] += k.c0 * (ri3 * nf - T(3) * ri3 * ri2 * rn * xf);
  } else if constexpr (KT == 511) {  // Kelvin solution
    T xf = x * f[0] + y * f[1] + z * f[2];
    T g1 = k.c0 * ri, g3 = k.c1 * ri * ri * ri * xf;
    u[0] = fmt(g3, x, fmt(g1, f[0], u[0]));
    u[1] = fmt(g3, y, fmt(g1, f[1], u[1]));
    u[2] = fmt(g3, z, fmt(g1, f[2], u[2]));
  } else if constexpr (KT == 521) {  // Navier double layer
    T xf = x * f[0] + y * f[1] + z * f[2];
    T nf = nrm[0] * f[0] + nrm[1] * f[1] + nrm[2] * f[2];
    T rn = x * nrm[0] + y * nrm[1] + z * nrm[2];
    T ri2 = ri * ri, ri3 = ri2 * ri;
    T A = k.c0 * ri3, B = k.c1 * ri3, C = k.c2 * ri3 * ri2;
    T s0 = A * rn, s1 = A * xf, s2 = B * nf + C * rn * xf;
    u[0] = fmt(s2, x, fmt(s1, nrm[0], fmt(s0, f[0], u[0])));
    u[1] = fmt(s2, y, fmt(s1, nrm[1], fmt(s0, f[1], u[1])));
    u[2] = fmt(s2, z, fmt(s1, nrm[2], fmt(s0, f[2], u[2])));
  }
}

#endif  // __CUDACC__

// Host-side constants for keval (FP64; converted to T by the caller).
inline void kernel_constants(int kt, const double* coefs, double* c) {
  const double pi = 3.14159265358979323846;
  c[0] = c[1] = c[2] = 0.0;
  double mu = coefs[0], ve = coefs[1];
  switch (kt) {
    case 111: c[0] = 1.0 / (4.0 * pi); break;
    case 121: c[0] = -1.0 / (4.0 * pi); break;
    case 301: c[0] = 1.0 / mu / (8.0 * pi); c[1] = 1.0 / (4.0 * pi); break;
    case 311: c[0] = 1.0 / mu / (8.0 * pi); break;
    case 312: c[0] = 1.0 / (4.0 * pi); break;
    case 321: c[0] = -6.0 / (8.0 * pi); break;
    case 322: c[0] = mu / (2.0 * pi); break;
    case 511: c[0] = (3.0 - 4.0 * ve) / (16.0 * pi * (1.0 - ve)) / mu; c[1] = 1.0 / (16.0 * pi * (1.0 - ve)) / mu; break;
    case 521:
      c[0] = -(1 - 2.0 * ve) / (8.0 * pi * (1.0 - ve));
      c[1] = (1 - 2.0 * ve) / (8.0 * pi * (1.0 - ve));
      c[2] = -3.0 / (8.0 * pi * (1.0 - ve));
      break;
  }
}

// Flop count per interaction (FMA = 2, rsqrt = 1), used for roofline accounting.
inline double kernel_flops(int kt) {
  switch (kt) {
    case 111: return 11; case 121: return 19; case 301: return 36; case 311: return 29; case 312: return 17;
    case 321: return 30; case 322: return 27; case 511: return 29; case 521: return 55;
  }
  return 0;
}

}  // namespace kifmm
