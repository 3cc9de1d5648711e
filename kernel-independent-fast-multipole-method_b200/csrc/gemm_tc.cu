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
constexpr unsigned A_STAGE = 2 * A_BYTES, B_STAGE = 2 * B_BYTES;
// node tiles double-buffered, operator chunks triple-buffered: 184 KB, so one
// CTA per SM, which owns all 512 TMEM columns
constexpr unsigned TC_SMEM = 2 * A_STAGE + 3 * B_STAGE;

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

// starts loading 8 consecutive TMEM columns of this thread's lane into r[0..7];
// the values are valid after tcgen05.wait::ld
__device__ __forceinline__ void tmem_ld8(unsigned taddr, unsigned* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

// 2^e as a float (e in the normal range), else ldexpf
__device__ __forceinline__ float pow2f(int e) {
  return (e >= -126 && e <= 127) ? __int_as_float((e + 127) << 23) : ldexpf(1.0f, e);
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_node_gemm_tc(TcOperator A, const float* __restrict__ B,
                                                               int64_t ldb, const int* __restrict__ bidx,
                                                               float* __restrict__ C, int64_t ldc,
                                                               const int* __restrict__ cidx, int ncol, int accumulate,
                                                               GemmScale sc, int ntile, int kper,
                                                               double* __restrict__ partial, int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ unsigned tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n0 = blockIdx.y * ntile;
  const int nn = min(ntile, A.Np - n0);  // rows of this tile (multiple of 16, <= 160)
  const int half = nn / 2;               // columns per draining thread (multiple of 8)
  const int col0 = blockIdx.x * TC_M;
  // this CTA's K chunks (split K: blockIdx.z)
  const int kb = blockIdx.z * kper, ke = min(A.Kp / TC_KC, kb + kper);
  const int nk = ke - kb;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(smem_u32(&bar[0]), 1);
    mbar_init(smem_u32(&bar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_base;

  auto a_stage = [&](int i) { return smem + (i & 1) * A_STAGE; };
  auto b_stage = [&](int i) { return smem + 2 * A_STAGE + (i % 3) * B_STAGE; };
  // operator chunk i (local) -> its B stage, head and tail; one cp.async group
  auto issue_op = [&](int i) {
    if (i < nk) {
      unsigned char* bh = b_stage(i);
      for (int e = tid; e < nn * 8; e += TC_THREADS) {
        const int r = e >> 3, q = e & 7;
        const size_t g = (size_t)(n0 + r) * A.Kp + (size_t)(kb + i) * TC_KC + 4 * q;
        cp_async16(smem_u32(bh + core_off(r, q)), A.hi + g);
        cp_async16(smem_u32(bh + B_BYTES + core_off(r, q)), A.lo + g);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // node data: row (tid & 127) of the tile, column groups 4*(tid >> 7) .. +4
  const int lrow = tid & (TC_M - 1), lq0 = (tid >> 7) * 4;
  const int lj = col0 + lrow;
  const float* bcol = (lj < ncol) ? B + (int64_t)bidx[lj] * ldb : nullptr;
  auto load_chunk = [&](int i, float4* cur) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int k = (kb + i) * TC_KC + 4 * (lq0 + q);
      cur[q] = (bcol && i < nk && k < A.K) ? *reinterpret_cast<const float4*>(bcol + k)
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  // draining: TMEM lanes 32*(warp & 3) + lane, columns (warp >> 2) * half .. +half
  const unsigned lane_addr = ((unsigned)((warp & 3) * 32) << 16) + (unsigned)((warp >> 2) * half);
  float sum[TC_HALF];
#pragma unroll
  for (int i = 0; i < TC_HALF; i++) sum[i] = 0.f;
  // a drain issues its loads in two groups of up to 40 columns, one wait per
  // group; the empty asm statements pin every use of the loaded registers
  // behind that wait
  auto drain = [&](int buf) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned base = tmem + lane_addr + (unsigned)(buf * TC_NMAX);
#pragma unroll
    for (int g = 0; g < 2; g++) {
      constexpr int GW = TC_HALF / 2;  // 40 columns
      unsigned raw[GW];
#pragma unroll
      for (int c = 0; c < GW / 8; c++)
        if (g * GW + c * 8 < half) tmem_ld8(base + g * GW + c * 8, &raw[c * 8]);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int i = 0; i < GW; i++) {
        if (g * GW + i < half) {
          asm volatile("" : "+r"(raw[i]));
          sum[g * GW + i] += __uint_as_float(raw[i]);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  };

  const unsigned idesc = idesc_tf32(nn);
  bool ok = true;
  float4 cur0[4], cur1[4];
  issue_op(0);
  issue_op(1);
  load_chunk(0, cur0);
  load_chunk(1, cur1);
  // one pipeline step on local chunk i, whose node data is in cur (refilled with chunk i + 2)
  auto step = [&](int i, float4* cur) {
    unsigned char* as = a_stage(i);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      float4 h, l;
      split4(cur[q], h, l);
      *reinterpret_cast<float4*>(as + core_off(lrow, lq0 + q)) = h;
      *reinterpret_cast<float4*>(as + A_BYTES + core_off(lrow, lq0 + q)) = l;
    }
    asm volatile("cp.async.wait_group 1;" ::: "memory");  // chunk i's operator (only i + 1 may be pending)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned d = tmem + (unsigned)((i & 1) * TC_NMAX);
      const unsigned ah0 = smem_u32(as), al0 = ah0 + A_BYTES;
      const unsigned bh0 = smem_u32(b_stage(i)), bl0 = bh0 + B_BYTES;
#pragma unroll
      for (int s = 0; s < TC_KC / 8; s++) {
        const unsigned off = s * 256;  // two core matrices along K per MMA
        const uint64_t ah = smem_desc(ah0 + off), al = smem_desc(al0 + off);
        const uint64_t bh = smem_desc(bh0 + off), bl = smem_desc(bl0 + off);
        mma_tf32(d, ah, bh, idesc, s != 0);  // a fresh accumulator per chunk
        mma_tf32(d, ah, bl, idesc, 1);
        mma_tf32(d, al, bh, idesc, 1);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bar[i & 1]))
                   : "memory");
    }
    load_chunk(i + 2, cur);  // in flight for two steps
    if (i > 0) {
      // chunk i-1's MMAs: their A / B stages and accumulator become free
      const bool done = mbar_wait_bounded(smem_u32(&bar[(i - 1) & 1]), ((i - 1) >> 1) & 1);
      if (__syncthreads_or(!done)) return false;
      drain((i - 1) & 1);
    }
    issue_op(i + 2);  // into the stage chunk i-1 used
    return true;
  };
  for (int i = 0; i < nk && ok; i += 2) {
    ok = step(i, cur0);
    if (ok && i + 1 < nk) ok = step(i + 1, cur1);
  }
  if (ok && nk > 0) {
    const bool done = mbar_wait_bounded(smem_u32(&bar[(nk - 1) & 1]), ((nk - 1) >> 1) & 1);
    ok = !__syncthreads_or(!done);
    if (ok) drain((nk - 1) & 1);
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (ok) {
    // lane of this thread = node row (warp & 3) * 32 + lane; columns of its half
    const int j = col0 + (warp & 3) * 32 + lane;
    const int nb = n0 + (warp >> 2) * half;
    if (j < ncol && partial) {  // split K: raw sums, scaled and added by the reduce
      double* pr = partial + ((size_t)blockIdx.z * ncol + j) * A.M;
#pragma unroll
      for (int i = 0; i < TC_HALF; i++)
        if (i < half && nb + i < A.M) pr[nb + i] = (double)sum[i];
    } else if (j < ncol) {
      float* crow = C + (int64_t)cidx[j] * ldc;
      const int lvl = sc.col_lvl ? sc.col_lvl[j] + sc.lvl_base : 0;
      float f4[4];  // scale of output n: f4[n % sd], sd <= 4
#pragma unroll
      for (int d = 0; d < 4; d++) f4[d] = sc.col_lvl ? pow2f(-lvl * sc.deg[d < sc.sd ? d : 0]) : 1.0f;
#pragma unroll
      for (int i = 0; i < TC_HALF; i += 4) {
        const int n = nb + i;
        if (i >= half || n >= A.M) break;
        float4 o = make_float4(sum[i], sum[i + 1], sum[i + 2], sum[i + 3]);
        if (sc.col_lvl) {
          o.x *= f4[(n + 0) % sc.sd];
          o.y *= f4[(n + 1) % sc.sd];
          o.z *= f4[(n + 2) % sc.sd];
          o.w *= f4[(n + 3) % sc.sd];
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
                        const int* cidx, int ncol, bool accumulate, const GemmScale& sc, double* ws, size_t ws_len,
                        int num_sms, int* status, cudaStream_t st) {
  if (ncol <= 0 || A.M <= 0 || A.K <= 0) return 0;
  // balanced N tiles of at most 160 rows, multiples of 16
  const int nt_count = (A.Np + TC_NMAX - 1) / TC_NMAX;
  const int ntile = ((A.Np + nt_count - 1) / nt_count + 15) / 16 * 16;
  const int gx = (ncol + TC_M - 1) / TC_M, gy = (A.Np + ntile - 1) / ntile;
  const int nk = A.Kp / TC_KC;
  // few tiles (the shallow tree levels): split K so that every SM has work
  int splits = 1;
  if (ws && gx * gy < num_sms && nk >= 4) {
    splits = std::min({(2 * num_sms) / (gx * gy), nk / 2, 16});
    while (splits > 1 && (size_t)splits * ncol * A.M > ws_len) splits--;
    splits = std::max(splits, 1);
  }
  const int kper = (nk + splits - 1) / splits;
  splits = (nk + kper - 1) / kper;
  dim3 grid(gx, gy, splits);
  cudaFuncSetAttribute(k_node_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
  k_node_gemm_tc<<<grid, TC_THREADS, TC_SMEM, st>>>(A, B, ldb, bidx, C, ldc, cidx, ncol, accumulate ? 1 : 0, sc, ntile,
                                                     kper, splits > 1 ? ws : nullptr, status);
  if (splits > 1) launch_node_gemm_reduce_f(A.M, ncol, splits, ws, C, ldc, cidx, accumulate, sc, num_sms, st);
  return splits > 1 ? 2 : 1;
}

}  // namespace kifmm
