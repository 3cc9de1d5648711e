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
constexpr int TC_TMEM_COLS = 512;     // two accumulators of up to 160 columns
constexpr unsigned A_BYTES = TC_M * TC_KC * 4;        // 16 KB per head / tail
constexpr unsigned B_BYTES = TC_NMAX * TC_KC * 4;     // 20 KB per head / tail
constexpr unsigned A_STAGE = 2 * A_BYTES, B_STAGE = 2 * B_BYTES;
constexpr int IMG_FLOATS = 2 * TC_NMAX * TC_KC;  // one operator chunk image: head + tail
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

// whole warp executes, one elected lane issues (a converged warp issues MMAs
// about three times faster than one thread of a diverged warp)
__device__ __forceinline__ void mma_tf32(unsigned d, uint64_t a, uint64_t b, unsigned idesc, int acc) {
  asm volatile(
      "{\n .reg .pred p, e;\n setp.ne.b32 p, %4, 0;\n elect.sync _|e, 0xffffffff;\n"
      " @e tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void commit_elect(unsigned bar) {
  asm volatile(
      "{\n .reg .pred e;\n elect.sync _|e, 0xffffffff;\n"
      " @e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n}\n" ::"r"(bar)
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

// Work items are (node tile, N tile, K split); the grid is persistent (at
// most one CTA per SM, each looping over items blockIdx.x, + gridDim.x, ...).
// Warp-specialised: warps 0-7 stage node data (A stages, two) and drain the
// accumulators (two), warp 8 issues the MMAs and the operator bulk copies (B
// stages, three).  They hand over through mbarriers:
//   afull[s]   (256 arrivals)  A stage s staged            worker -> MMA warp
//   bfull[s]   (bytes)         operator chunk landed        copy   -> MMA warp
//   accfull[b] (commit)        chunk's MMAs complete        MMA    -> workers
//   accempty[b] (256 arrivals) accumulator b drained        worker -> MMA warp
// The chunk stream runs straight across item boundaries; an item's stores
// overlap the next item's MMAs.
constexpr int TC_WORKERS = 256;
constexpr int TC_ALL = TC_WORKERS + 32;

__global__ void __launch_bounds__(TC_ALL, 1) k_node_gemm_tc(TcOperator A, const float* __restrict__ B, int64_t ldb,
                                                           const int* __restrict__ bidx, float* __restrict__ C,
                                                           int64_t ldc, const int* __restrict__ cidx, int ncol,
                                                           int accumulate, GemmScale sc, int kper, int nitems,
                                                           double* __restrict__ partial, int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) unsigned long long afull[2], bfull[3], accfull[2], accempty[2];
  __shared__ unsigned tmem_base;
  __shared__ int fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gx = (ncol + TC_M - 1) / TC_M, gy = A.ntiles;
  const int nkt = A.Kp / TC_KC;
  if ((int)blockIdx.x >= nitems) return;
  const int my_items = (nitems - 1 - (int)blockIdx.x) / (int)gridDim.x + 1;
  auto item_of = [&](int li, int& x, int& y, int& z) {
    const int it = blockIdx.x + li * gridDim.x;
    x = it % gx;
    y = (it / gx) % gy;
    z = it / (gx * gy);
  };
  int x0, y0, z0;
  item_of(0, x0, y0, z0);
  // every item of one launch has the same chunk count except a shorter last K
  // split, which only split launches (one item per CTA) have
  const int nk = min(nkt, (z0 + 1) * kper) - z0 * kper;
  const int total = my_items * nk;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int b = 0; b < 2; b++) {
      mbar_init(smem_u32(&afull[b]), TC_WORKERS);
      mbar_init(smem_u32(&accfull[b]), 1);
      mbar_init(smem_u32(&accempty[b]), TC_WORKERS);
    }
    for (int b = 0; b < 3; b++) mbar_init(smem_u32(&bfull[b]), 1);
    fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_base;
  auto a_stage = [&](int g) { return smem + (g & 1) * A_STAGE; };
  auto b_stage = [&](int g) { return smem + 2 * A_STAGE + (g % 3) * B_STAGE; };
  auto half_of = [&](int g) {
    int x, y, z;
    item_of(g / nk, x, y, z);
    return min(A.ntile, A.Np - y * A.ntile) / 2;
  };
  volatile int* vfail = &fail;
  auto wait = [&](unsigned long long* bar, int parity) {
    if (*vfail) return false;
    if (mbar_wait_bounded(smem_u32(bar), parity)) return true;
    *vfail = 1;
    return false;
  };

  if (warp == TC_WORKERS / 32) {
    // ---- MMA warp: the whole warp runs the loop (warp-uniform waits), one
    // elected lane issues the MMAs and commits, lane 0 the operator copies
    auto wait_w = [&](unsigned long long* bar, int parity) { return __all_sync(0xffffffffu, wait(bar, parity)); };
    {
      auto issue_op = [&](int g) {
        if (g >= total || lane != 0) return;
        int x, y, z;
        item_of(g / nk, x, y, z);
        const float* img = A.img + ((size_t)y * nkt + z * kper + g % nk) * IMG_FLOATS;
        bulk_load(smem_u32(b_stage(g)), img, IMG_FLOATS * 4, smem_u32(&bfull[g % 3]));
      };
      issue_op(0);
      issue_op(1);
      issue_op(2);
      for (int g = 0; g < total; g++) {
        if (!wait_w(&afull[g & 1], (g >> 1) & 1)) break;
        if (!wait_w(&bfull[g % 3], (g / 3) & 1)) break;
        if (g >= 2 && !wait_w(&accempty[g & 1], ((g - 2) >> 1) & 1)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned d = tmem + (unsigned)((g & 1) * TC_NMAX);
        const unsigned ah0 = smem_u32(a_stage(g)), al0 = ah0 + A_BYTES;
        const unsigned bh0 = smem_u32(b_stage(g)), bl0 = bh0 + B_BYTES;
        const unsigned idesc = idesc_tf32(2 * half_of(g));
#pragma unroll
        for (int s = 0; s < TC_KC / 8; s++) {
          const unsigned off = s * 256;  // two core matrices along K per MMA
          const uint64_t ah = smem_desc(ah0 + off), al = smem_desc(al0 + off);
          const uint64_t bh = smem_desc(bh0 + off), bl = smem_desc(bl0 + off);
          mma_tf32(d, ah, bh, idesc, s != 0);  // a fresh accumulator per chunk
          mma_tf32(d, ah, bl, idesc, 1);
          mma_tf32(d, al, bh, idesc, 1);
        }
        commit_elect(smem_u32(&accfull[g & 1]));
        // chunk g-1's MMAs complete -> its operator stage takes chunk g + 2
        if (g >= 1) {
          if (!wait_w(&accfull[(g - 1) & 1], ((g - 1) >> 1) & 1)) break;
          issue_op(g + 2);
        }
      }
    }
  } else {
    // ---- worker warps: stage node data, drain accumulators, store
    const int lrow = tid & (TC_M - 1), lq0 = (tid >> 7) * 4;
    // node column of this thread's row in item li (-1: past the last node)
    auto item_col = [&](int li) {
      int x, y, z;
      item_of(li, x, y, z);
      const int lj = x * TC_M + lrow;
      return lj < ncol ? bidx[lj] : -1;
    };
    // load_chunk is called with g = 0, 1, 2, ...: the next item's node index is
    // fetched one item ahead, so the data loads never wait on it
    int li_cur = -1, idx_next = my_items > 0 ? item_col(0) : -1;
    const float* bcol = nullptr;
    auto load_chunk = [&](int g, float4* cur) {
      int k0 = 0;
      bool have = false;
      if (g < total) {
        const int li = g / nk;
        if (li != li_cur) {
          bcol = idx_next >= 0 ? B + (int64_t)idx_next * ldb : nullptr;
          li_cur = li;
          idx_next = li + 1 < my_items ? item_col(li + 1) : -1;
        }
        int x, y, z;
        item_of(li, x, y, z);
        k0 = (z * kper + g % nk) * TC_KC;
        have = bcol != nullptr;
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int k = k0 + 4 * (lq0 + q);
        cur[q] = (have && k < A.K) ? *reinterpret_cast<const float4*>(bcol + k) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    };
    auto produce = [&](int g, const float4* cur) {
      unsigned char* as = a_stage(g);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        float4 h, l;
        split4(cur[q], h, l);
        *reinterpret_cast<float4*>(as + core_off(lrow, lq0 + q)) = h;
        *reinterpret_cast<float4*>(as + A_BYTES + core_off(lrow, lq0 + q)) = l;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&afull[g & 1])) : "memory");
    };
    float sum[TC_HALF];
#pragma unroll
    for (int i = 0; i < TC_HALF; i++) sum[i] = 0.f;
    // drain chunk g's accumulator: TMEM lanes 32*(warp & 3) + lane, columns
    // (warp >> 2) * half .. +half; two groups of up to 40 columns, one wait
    // per group, uses pinned behind the wait by empty asm statements
    auto drain = [&](int g, int half) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned base =
          tmem + ((unsigned)((warp & 3) * 32) << 16) + (unsigned)((warp >> 2) * half + (g & 1) * TC_NMAX);
#pragma unroll
      for (int gr = 0; gr < 2; gr++) {
        constexpr int GW = TC_HALF / 2;  // 40 columns
        unsigned raw[GW];
#pragma unroll
        for (int c = 0; c < GW / 8; c++)
          if (gr * GW + c * 8 < half) tmem_ld8(base + gr * GW + c * 8, &raw[c * 8]);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int i = 0; i < GW; i++) {
          if (gr * GW + i < half) {
            asm volatile("" : "+r"(raw[i]));
            sum[gr * GW + i] += __uint_as_float(raw[i]);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&accempty[g & 1])) : "memory");
    };
    // store item li's tile from the sums (row (warp & 3) * 32 + lane, this thread's half)
    auto epilogue = [&](int li) {
      int x, y, z;
      item_of(li, x, y, z);
      const int n0 = y * A.ntile, nn = min(A.ntile, A.Np - n0), half = nn / 2;
      const int j = x * TC_M + (warp & 3) * 32 + lane;
      const int nb = n0 + (warp >> 2) * half;
      if (j < ncol && partial) {  // split K: raw sums, scaled and added by the reduce
        double* pr = partial + ((size_t)z * ncol + j) * A.M;
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
            const float4 c4 = *p;
            o.x += c4.x;
            o.y += c4.y;
            o.z += c4.z;
            o.w += c4.w;
          }
          *p = o;
        }
      }
#pragma unroll
      for (int i = 0; i < TC_HALF; i++) sum[i] = 0.f;
    };
    float4 cur[4];
    load_chunk(0, cur);
    if (total > 0) produce(0, cur);
    load_chunk(1, cur);
    if (total > 1) produce(1, cur);
    load_chunk(2, cur);
    // chunk g: wait for its MMAs, hand the freed A stage chunk g + 2 (its data
    // in cur, then refilled with chunk g + 3), drain, store at an item's end
    for (int g = 0; g < total; g++) {
      if (!wait(&accfull[g & 1], (g >> 1) & 1)) break;
      if (g + 2 < total) produce(g + 2, cur);
      load_chunk(g + 3, cur);
      drain(g, half_of(g));
      if (g % nk == nk - 1) epilogue(g / nk);
    }
  }
  __syncthreads();
  if (*vfail && tid == 0) atomicOr(status, 2);
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
  const int nitems = gx * gy * splits;
  // split launches: one item per CTA (the last split may be shorter);
  // otherwise persistent, at most one CTA per SM
  const int grid = splits > 1 ? nitems : std::min(nitems, num_sms);
  cudaFuncSetAttribute(k_node_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
  k_node_gemm_tc<<<grid, TC_ALL, TC_SMEM, st>>>(A, B, ldb, bidx, C, ldc, cidx, ncol, accumulate ? 1 : 0, sc, kper,
                                                 nitems, splits > 1 ? ws : nullptr, status);
  if (splits > 1) launch_node_gemm_reduce_f(A.M, ncol, splits, ws, C, ldc, cidx, accumulate, sc, num_sms, st);
  return splits > 1 ? 2 : 1;
}

}  // namespace kifmm
