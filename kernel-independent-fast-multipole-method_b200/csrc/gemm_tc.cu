// Node GEMM on the 5th-generation tensor cores (tcgen05, kind::tf32) for the
// FP32 surface contractions of the mixed-precision engine (see gemm.cu for
// the operators and the reference lines they replace).
//
//   D[node][out] = sum_k data[node][k] * op[out][k]
//
// One CTA (one per SM) computes a tile of 128 nodes (the MMA's M, one node
// per TMEM lane) by up to 160 operator rows (the MMA's N).  K advances in
// chunks of 32: the CTA's threads gather the 128 node columns (each a
// contiguous K-vector) with 16-byte loads, split every value into a TF32 head
// and a TF32 tail and store both into shared memory in the no-swizzle K-major
// core-matrix layout; the operator chunk (split once on the host) arrives by
// cp.async.  One thread then issues, per K-step of 8,
//   D += A_hi B_hi,  D += A_hi B_lo,  D += A_lo B_hi
// into a fresh TMEM accumulator per chunk and commits them to an mbarrier.
// Two accumulators alternate: while the MMAs of chunk c run, the threads
// drain chunk c-1's accumulator (tcgen05.ld) into FP32 register sums and
// load chunk c+1's node columns.  The epilogue applies the homogeneous level
// scaling of the node and stores (or adds) 16-byte vectors.
//
// Precision: each product carries head*head exactly and the two cross terms
// to TF32 accuracy (tail*tail, 2^-22 relative, is dropped).  The tensor core
// adds the products of one MMA to its accumulator with a single alignment
// whose rounding error grows with every MMA folded into the same
// accumulator; letting only 12 MMAs meet in TMEM and summing the chunks in
// FP32 registers keeps the contractions -- which cancel strongly in the
// Sigma^-1 U^T factors -- in the error class of FP32 FMA accumulation.
#include <algorithm>
#include <cstring>

#include "launch.hpp"

namespace kifmm {
namespace {

constexpr int TC_M = 128;       // nodes per tile (MMA M, TMEM lanes)
constexpr int TC_KC = 32;       // K per chunk (8 core matrices of 4 TF32)
constexpr int TC_NMAX = 160;    // operator rows per tile (MMA N)
constexpr int TC_HALF = TC_NMAX / 2;  // columns drained per thread
constexpr int TC_THREADS = 256;
constexpr int TC_TMEM_COLS = 512;     // two accumulators of up to 160 columns
constexpr unsigned A_BYTES = TC_M * TC_KC * 4;        // 16 KB per head / tail
constexpr unsigned B_BYTES = TC_NMAX * TC_KC * 4;     // 20 KB per head / tail
// 72 KB of operands, padded so that only one CTA fits on an SM: it owns all
// 512 TMEM columns
constexpr unsigned TC_SMEM = 120 * 1024;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// byte offset of (row, 4-element column group q) in a [rows][32] K-major
// no-swizzle tile: core matrices of 8 rows x 16 B, 8 along K (LBO = 128 B),
// row groups 1024 B apart (SBO)
__device__ __forceinline__ unsigned core_off(int row, int q) {
  return (unsigned)(((row >> 3) * 8 + q) * 128 + (row & 7) * 16);
}

__device__ __forceinline__ uint64_t smem_desc(unsigned addr) {
  const uint64_t lbo = 128, sbo = 1024;
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((lbo >> 4) << 16) | ((sbo >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ float tf32_round(float x) {
  unsigned u = __float_as_uint(x);
  u = (u + 0x1000u) & 0xFFFFE000u;
  return __uint_as_float(u);
}

__device__ __forceinline__ void split4(float4 v, float4& hi, float4& lo) {
  hi.x = tf32_round(v.x);
  hi.y = tf32_round(v.y);
  hi.z = tf32_round(v.z);
  hi.w = tf32_round(v.w);
  lo.x = tf32_round(v.x - hi.x);
  lo.y = tf32_round(v.y - hi.y);
  lo.z = tf32_round(v.z - hi.z);
  lo.w = tf32_round(v.w - hi.w);
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
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

__device__ __forceinline__ void cp_async16(unsigned dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

__device__ __forceinline__ void mma_tf32(unsigned d, uint64_t a, uint64_t b, unsigned idesc, int acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

// instruction descriptor, kind::tf32: D F32, A and B TF32, both K-major
__device__ __forceinline__ unsigned idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(n >> 3) << 17) | ((unsigned)(TC_M >> 4) << 24);
}

// adds 8 consecutive TMEM columns of this thread's lane to s[0..7]
__device__ __forceinline__ void tmem_ld8_add(unsigned taddr, float* s) {
  unsigned r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) s[i] += __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_node_gemm_tc(TcOperator A, const float* __restrict__ B,
                                                               int64_t ldb, const int* __restrict__ bidx,
                                                               float* __restrict__ C, int64_t ldc,
                                                               const int* __restrict__ cidx, int ncol, int accumulate,
                                                               GemmScale sc, int ntile, int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) unsigned long long bar;
  __shared__ unsigned tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char* a_hi = smem;
  unsigned char* a_lo = smem + A_BYTES;
  unsigned char* b_hi = smem + 2 * A_BYTES;
  unsigned char* b_lo = smem + 2 * A_BYTES + B_BYTES;
  const int n0 = blockIdx.y * ntile;
  const int nn = min(ntile, A.Np - n0);  // rows of this tile (multiple of 16, <= 160)
  const int half = nn / 2;               // columns per draining thread (multiple of 8)
  const int col0 = blockIdx.x * TC_M;
  const int nk = A.Kp / TC_KC;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(smem_u32(&bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_base;

  // loading: row (tid & 127) of the tile, column groups 4*(tid >> 7) .. +4
  const int lrow = tid & (TC_M - 1), lq0 = (tid >> 7) * 4;
  const int lj = col0 + lrow;
  const float* bcol = (lj < ncol) ? B + (int64_t)bidx[lj] * ldb : nullptr;
  float4 cur[4];
  auto load_chunk = [&](int kc) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int k = kc * TC_KC + 4 * (lq0 + q);
      cur[q] = (bcol && k < A.K) ? *reinterpret_cast<const float4*>(bcol + k) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  // draining: TMEM lanes 32*(warp & 3) + lane, columns (warp >> 2) * half .. +half
  const unsigned lane_addr = ((unsigned)((warp & 3) * 32) << 16) + (unsigned)((warp >> 2) * half);
  float sum[TC_HALF];
#pragma unroll
  for (int i = 0; i < TC_HALF; i++) sum[i] = 0.f;
  auto drain = [&](int buf) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned base = tmem + lane_addr + (unsigned)(buf * TC_NMAX);
#pragma unroll
    for (int c = 0; c < TC_HALF / 8; c++)
      if (c * 8 < half) tmem_ld8_add(base + c * 8, &sum[c * 8]);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  };

  load_chunk(0);
  const unsigned idesc = idesc_tf32(nn);
  bool ok = true;
  for (int kc = 0; kc < nk; kc++) {
    // operator chunk: rows n0..n0+nn, columns kc*32..+32, head and tail
    for (int e = tid; e < nn * 8; e += TC_THREADS) {
      const int r = e >> 3, q = e & 7;
      const size_t g = (size_t)(n0 + r) * A.Kp + (size_t)kc * TC_KC + 4 * q;
      cp_async16(smem_u32(b_hi + core_off(r, q)), A.hi + g);
      cp_async16(smem_u32(b_lo + core_off(r, q)), A.lo + g);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 4; q++) {
      float4 h, l;
      split4(cur[q], h, l);
      *reinterpret_cast<float4*>(a_hi + core_off(lrow, lq0 + q)) = h;
      *reinterpret_cast<float4*>(a_lo + core_off(lrow, lq0 + q)) = l;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned d = tmem + (unsigned)((kc & 1) * TC_NMAX);
#pragma unroll
      for (int s = 0; s < TC_KC / 8; s++) {
        const unsigned off = s * 256;  // two core matrices along K per MMA
        const uint64_t ah = smem_desc(smem_u32(a_hi) + off), al = smem_desc(smem_u32(a_lo) + off);
        const uint64_t bh = smem_desc(smem_u32(b_hi) + off), bl = smem_desc(smem_u32(b_lo) + off);
        mma_tf32(d, ah, bh, idesc, s != 0);  // a fresh accumulator per chunk
        mma_tf32(d, ah, bl, idesc, 1);
        mma_tf32(d, al, bh, idesc, 1);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bar))
                   : "memory");
    }
    if (kc > 0) drain((kc - 1) & 1);       // the previous chunk, under this chunk's MMAs
    if (kc + 1 < nk) load_chunk(kc + 1);  // in flight while the MMAs run
    const bool done = mbar_wait_bounded(smem_u32(&bar), kc & 1);
    if (__syncthreads_or(!done)) {
      ok = false;
      break;
    }
  }
  if (ok) {
    drain((nk - 1) & 1);
    // lane of this thread = node row (warp & 3) * 32 + lane; columns of its half
    const int j = col0 + (warp & 3) * 32 + lane;
    if (j < ncol) {
      float* crow = C + (int64_t)cidx[j] * ldc;
      const int lvl = sc.col_lvl ? sc.col_lvl[j] + sc.lvl_base : 0;
      const int nb = n0 + (warp >> 2) * half;
#pragma unroll
      for (int i = 0; i < TC_HALF; i += 4) {
        const int n = nb + i;
        if (i >= half || n >= A.M) break;
        float4 o = make_float4(sum[i], sum[i + 1], sum[i + 2], sum[i + 3]);
        if (sc.col_lvl) {
          o.x = ldexpf(o.x, -lvl * sc.deg[(n + 0) % sc.sd]);
          o.y = ldexpf(o.y, -lvl * sc.deg[(n + 1) % sc.sd]);
          o.z = ldexpf(o.z, -lvl * sc.deg[(n + 2) % sc.sd]);
          o.w = ldexpf(o.w, -lvl * sc.deg[(n + 3) % sc.sd]);
        }
        float4* p = reinterpret_cast<float4*>(crow + n);
        if (accumulate) {
          const float4 c = *p;
          o.x += c.x;
          o.y += c.y;
          o.z += c.z;
          o.w += c.w;
        }
        *p = o;
      }
    }
  } else if (tid == 0) {
    atomicOr(status, 2);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
  }
}

inline float tf32_round_host(float x) {
  unsigned u;
  std::memcpy(&u, &x, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  std::memcpy(&x, &u, 4);
  return x;
}

}  // namespace

void split_tf32(int M, int K, const double* A, std::vector<float>* hi, std::vector<float>* lo, int* Np, int* Kp) {
  *Np = (M + 15) / 16 * 16;
  *Kp = (K + TC_KC - 1) / TC_KC * TC_KC;
  hi->assign((size_t)*Np * *Kp, 0.f);
  lo->assign((size_t)*Np * *Kp, 0.f);
  for (int r = 0; r < M; r++)
    for (int k = 0; k < K; k++) {
      const double a = A[(size_t)r * K + k];
      const float h = tf32_round_host((float)a);
      (*hi)[(size_t)r * *Kp + k] = h;
      (*lo)[(size_t)r * *Kp + k] = tf32_round_host((float)(a - (double)h));
    }
}

int launch_node_gemm_tc(const TcOperator& A, const float* B, int64_t ldb, const int* bidx, float* C, int64_t ldc,
                        const int* cidx, int ncol, bool accumulate, const GemmScale& sc, int* status,
                        cudaStream_t st) {
  if (ncol <= 0 || A.M <= 0 || A.K <= 0) return 0;
  // balanced N tiles of at most 160 rows, multiples of 16
  const int nt_count = (A.Np + TC_NMAX - 1) / TC_NMAX;
  const int ntile = ((A.Np + nt_count - 1) / nt_count + 15) / 16 * 16;
  dim3 grid((ncol + TC_M - 1) / TC_M, (A.Np + ntile - 1) / ntile);
  cudaFuncSetAttribute(k_node_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
  k_node_gemm_tc<<<grid, TC_THREADS, TC_SMEM, st>>>(A, B, ldb, bidx, C, ldc, cidx, ncol, accumulate ? 1 : 0, sc,
                                                     ntile, status);
  return 1;
}

}  // namespace kifmm
