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
// core-matrix layout; the operator chunk (split and laid out once on the
// host) arrives as one bulk asynchronous copy on an mbarrier.  One thread
// then issues, per K-step of 8,
//   D += A_hi B_hi,  D += A_hi B_lo,  D += A_lo B_hi
// into a fresh TMEM accumulator per chunk and commits them to an mbarrier.
// Two accumulators alternate: while the MMAs of chunk c run, the threads
// drain chunk c-1's accumulator (tcgen05.ld) into FP32 register sums and
// load chunk c+2's node columns.  The epilogue stages the 128 x N tile in
// shared memory, then writes whole output rows with coalesced 16-byte
// stores, applying the homogeneous level scaling of each node.
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
constexpr int IMG_FLOATS = 2 * TC_NMAX * TC_KC;  // one operator chunk image: head + tail
constexpr int OUT_LD = TC_NMAX + 4;               // staged output row stride (floats)
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

__device__ __forceinline__ void bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_node_gemm_tc(TcOperator A, const float* __restrict__ B,
                                                               int64_t ldb, const int* __restrict__ bidx,
                                                               float* __restrict__ C, int64_t ldc,
                                                               const int* __restrict__ cidx, int ncol, int accumulate,
                                                               GemmScale sc, int kper, double* __restrict__ partial,
                                                               int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) unsigned long long bar[2];  // MMA completion, per accumulator
  __shared__ __align__(8) unsigned long long opb[3];  // operator chunk arrival, per B stage
  __shared__ unsigned tmem_base;
  __shared__ int op_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n0 = blockIdx.y * A.ntile;
  const int nn = min(A.ntile, A.Np - n0);  // rows of this tile (multiple of 16, <= 160)
  const int half = nn / 2;                 // columns per draining thread (multiple of 8)
  const int col0 = blockIdx.x * TC_M;
  const int nkt = A.Kp / TC_KC;
  // this CTA's K chunks (split K: blockIdx.z)
  const int kb = blockIdx.z * kper, ke = min(nkt, kb + kper);
  const int nk = ke - kb;
  const float* img = A.img + ((size_t)blockIdx.y * nkt + kb) * IMG_FLOATS;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int b = 0; b < 2; b++) mbar_init(smem_u32(&bar[b]), 1);
    for (int b = 0; b < 3; b++) mbar_init(smem_u32(&opb[b]), 1);
    op_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_base;

  auto a_stage = [&](int i) { return smem + (i & 1) * A_STAGE; };
  auto b_stage = [&](int i) { return smem + 2 * A_STAGE + (i % 3) * B_STAGE; };
  // operator chunk i (local): one bulk copy of its head + tail image
  auto issue_op = [&](int i) {
    if (tid == 0 && i < nk)
      bulk_load(smem_u32(b_stage(i)), img + (size_t)i * IMG_FLOATS, IMG_FLOATS * 4, smem_u32(&opb[i % 3]));
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
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      if (!mbar_wait_bounded(smem_u32(&opb[i % 3]), (i / 3) & 1)) op_fail = 1;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned d = tmem + (unsigned)((i & 1) * TC_NMAX);
      const unsigned ah0 = smem_u32(as), al0 = ah0 + A_BYTES;
      const unsigned bh0 = smem_u32(b_stage(i)), bl0 = bh0 + B_BYTES;
      if (!op_fail) {
#pragma unroll
        for (int s = 0; s < TC_KC / 8; s++) {
          const unsigned off = s * 256;  // two core matrices along K per MMA
          const uint64_t ah = smem_desc(ah0 + off), al = smem_desc(al0 + off);
          const uint64_t bh = smem_desc(bh0 + off), bl = smem_desc(bl0 + off);
          mma_tf32(d, ah, bh, idesc, s != 0);  // a fresh accumulator per chunk
          mma_tf32(d, ah, bl, idesc, 1);
          mma_tf32(d, al, bh, idesc, 1);
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bar[i & 1]))
                   : "memory");
    }
    load_chunk(i + 2, cur);  // in flight for two steps
    if (i > 0) {
      // chunk i-1's MMAs: their A / B stages and accumulator become free
      const bool done = mbar_wait_bounded(smem_u32(&bar[(i - 1) & 1]), ((i - 1) >> 1) & 1);
      if (__syncthreads_or(!done || op_fail)) return false;
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
    ok = !__syncthreads_or(!done || op_fail);
    if (ok) drain((nk - 1) & 1);
  }
  if (ok) {
    // stage the tile: row (warp & 3) * 32 + lane, columns of this thread's half
    __syncthreads();  // every MMA has completed: the operand stages are free
    float* out = reinterpret_cast<float*>(smem);
    {
      float* orow = out + ((warp & 3) * 32 + lane) * OUT_LD + (warp >> 2) * half;
#pragma unroll
      for (int i = 0; i < TC_HALF; i += 4)
        if (i < half) *reinterpret_cast<float4*>(orow + i) = make_float4(sum[i], sum[i + 1], sum[i + 2], sum[i + 3]);
    }
    __syncthreads();
    const int nv = min(nn, A.M - n0);  // valid output rows of this N tile (multiple of 4)
    const int nv4 = nv / 4;
    const int rows = min(TC_M, ncol - col0);
    if (partial) {  // split K: raw sums, scaled and added by the reduce
      for (int e = tid; e < rows * nv; e += TC_THREADS) {
        const int r = e / nv, c = e - r * nv;
        partial[((size_t)blockIdx.z * ncol + col0 + r) * A.M + n0 + c] = (double)out[r * OUT_LD + c];
      }
    } else {
      for (int e = tid; e < rows * nv4; e += TC_THREADS) {
        const int r = e / nv4, c = e - r * nv4;
        const int j = col0 + r, n = n0 + 4 * c;
        float4 o = *reinterpret_cast<const float4*>(out + r * OUT_LD + 4 * c);
        if (sc.col_lvl) {
          const int lvl = sc.col_lvl[j] + sc.lvl_base;
          o.x *= pow2f(-lvl * sc.deg[(n + 0) % sc.sd]);
          o.y *= pow2f(-lvl * sc.deg[(n + 1) % sc.sd]);
          o.z *= pow2f(-lvl * sc.deg[(n + 2) % sc.sd]);
          o.w *= pow2f(-lvl * sc.deg[(n + 3) % sc.sd]);
        }
        float4* p = reinterpret_cast<float4*>(C + (int64_t)cidx[j] * ldc + n);
        if (accumulate) {
          const float4 c4 = *p;
          o.x += c4.x;
          o.y += c4.y;
          o.z += c4.z;
          o.w += c4.w;
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

void tc_operator_images(int M, int K, const double* A, std::vector<float>* img, TcOperator* d) {
  d->M = M;
  d->K = K;
  d->Np = (M + 15) / 16 * 16;
  d->Kp = (K + TC_KC - 1) / TC_KC * TC_KC;
  // balanced N tiles of at most 160 rows, multiples of 16
  const int nt_count = (d->Np + TC_NMAX - 1) / TC_NMAX;
  d->ntile = ((d->Np + nt_count - 1) / nt_count + 15) / 16 * 16;
  d->ntiles = (d->Np + d->ntile - 1) / d->ntile;
  const int nkt = d->Kp / TC_KC;
  img->assign((size_t)d->ntiles * nkt * IMG_FLOATS, 0.f);
  for (int y = 0; y < d->ntiles; y++)
    for (int c = 0; c < nkt; c++) {
      float* base = img->data() + ((size_t)y * nkt + c) * IMG_FLOATS;
      for (int r = 0; r < d->ntile; r++) {
        const int n = y * d->ntile + r;
        if (n >= M) break;
        for (int k = 0; k < TC_KC; k++) {
          const int kk = c * TC_KC + k;
          if (kk >= K) break;
          const double a = A[(size_t)n * K + kk];
          const float h = tf32_round_host((float)a);
          const float l = tf32_round_host((float)(a - (double)h));
          const size_t off = (size_t)(((r >> 3) * 8 + (k >> 2)) * 32 + (r & 7) * 4 + (k & 3));
          base[off] = h;
          base[TC_NMAX * TC_KC + off] = l;
        }
      }
    }
}

int launch_node_gemm_tc(const TcOperator& A, const float* B, int64_t ldb, const int* bidx, float* C, int64_t ldc,
                        const int* cidx, int ncol, bool accumulate, const GemmScale& sc, double* ws, size_t ws_len,
                        int num_sms, int* status, cudaStream_t st) {
  if (ncol <= 0 || A.M <= 0 || A.K <= 0) return 0;
  const int gx = (ncol + TC_M - 1) / TC_M, gy = A.ntiles;
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
  k_node_gemm_tc<<<grid, TC_THREADS, TC_SMEM, st>>>(A, B, ldb, bidx, C, ldc, cidx, ncol, accumulate ? 1 : 0, sc, kper,
                                                     splits > 1 ? ws : nullptr, status);
  if (splits > 1) launch_node_gemm_reduce_f(A.M, ncol, splits, ws, C, ldc, cidx, accumulate, sc, num_sms, st);
  return splits > 1 ? 2 : 1;
}

}  // namespace kifmm
