// V-list Hadamard accumulate on the 5th-generation tensor cores (tcgen05,
// kind::tf32) for single-dof equivalent kernels in mixed precision: the
// frequency-domain product of the reference's M2L (fmm3d/fmm3d_eval.cpp:
// 115-150, MatMgnt3d::UE2DC_dgemv fmm3d/matmgnt3d.cpp:272-290), in the
// parent-pair form of the V list.
//
// For target parent Q, colleague direction d (P = Q + d) and frequency f the
// V-list products of Q's 8 children with P's 8 children are one 8 x 8
// complex block, M[i][j] = K(2d + oct(j) - oct(i)) (zero for adjacent child
// pairs, which are not V-list pairs), applied to P's 8 child spectra.  In
// real arithmetic (rows 2i + re/im, columns 2j + re/im) that is a 16 x 16
// block B_d(f), and for a tile of 128 target parents
//   D(f)[128 x 16] = sum_d A_d(f)[128 x 16] B_d(f)^T,
// A_d(f) row q = the 8 child spectra of q's colleague in direction d.
//
// The rows of A_d differ per direction (a gather: every colleague's spectra
// serve up to 26 target parents), so they go to the tensor core through
// TMEM, not shared memory: producer warps load each row's 8 x 4 complex
// values, split them into a TF32 head and tail and write both into TMEM with
// tcgen05.st, where the MMA reads A directly (an MMA with A in shared memory
// at N = 16 is bound by the shared-memory reads of A, one with A in TMEM by
// the tensor core).  The spectra are stored sibling-group major (written so
// by the forward transform), so a colleague's 8 children x 4 frequencies
// are 256 contiguous bytes; four
// adjacent threads load children 4 kh .. 4 kh + 3 of one row with 32-byte
// loads (one 128-byte line per row per load instruction) and write them with
// the 16x256b TMEM shape, whose four adjacent threads fill one lane's 8
// columns.  The
// operator images (head and tail, laid out once on the host) arrive per
// (frequency chunk, direction) as one bulk asynchronous copy.  Per frequency
// and K-half of 8, two MMAs:
//   D[0:32)  += A_hi [B_hi | B_lo]^T    (N = 32)
//   D[0:16)  += A_lo B_hi^T             (N = 16)
// and the drain adds D[16:32) to D[0:16): head*head exact, both cross terms
// to TF32 accuracy, tail*tail (2^-22 relative) dropped.
//
// Work items are (frequency chunk of 4, tile of 128 target parents), chunk
// major, over a persistent grid; inside an item the steps are the tile's
// present colleague directions.  Warp roles, handing over through mbarriers:
//   warps 0-11  producers, three groups of four (one warp per TMEM lane
//               quarter); group g owns A stage g and fills it for every step
//               s = g mod 3, so each group waits on its stage's phases in
//               order (a group that skipped a phase of a shared stage could
//               match the parity of a phase two behind); the group also
//               issues the step's operator copy (operator stage s mod 6) and
//               arrives on afull only once it has landed.  A group walks its
//               own steps only (s to s + 3 directly): every instruction it
//               spends between two of its steps lengthens the round trip of
//               its A stage, which with three stages sets the step rate
//   warps 12-15 MMA warps: warp 12 + f issues frequency f's 4 MMAs of every
//               step (its own accumulator columns; one elected lane) and
//               commits; at an item's end it drains TMEM lane quarter
//               (12 + f) mod 4, all four frequencies, into effval
//   bfull[6]   (bytes)         operator images landed           copy -> producers
//   afull[3]   (128 arrivals)  A stage written, images landed   producers -> MMA
//   aempty[3]  (4 commits)     step's MMAs done: A stage and the operator
//                              stage of step - 3 free           MMA -> producers
//   accfull    (4 commits)     item's MMAs done                 MMA -> drain
//   accempty   (128 arrivals)  accumulator read out             drain -> MMA
// Every wait is bounded; a time-out sets bit 2 of *status and ends the CTA.
#include <algorithm>
#include <complex>
#include <cstring>
#include <vector>

#include "launch.hpp"

namespace kifmm {
namespace {

constexpr int HT_M = 128;           // target parents per tile (MMA M, TMEM lanes)
constexpr int HT_F = 4;             // frequencies per item
constexpr int HT_ASTAGES = 3;       // A stages in TMEM, one per producer group
constexpr int HT_MMA_WARP = HT_ASTAGES * 4;
constexpr int HT_THREADS = (HT_MMA_WARP + 4) * 32;
constexpr int HT_NB = 6;                         // operator image stages (step mod 6)
constexpr int HT_IMG_FLOATS = HT_F * 512;        // per (chunk, direction): F x [32 rows x 16 K]
constexpr unsigned HT_IMG_BYTES = HT_IMG_FLOATS * 4;
constexpr unsigned HT_COLS = 512;                // accumulator 0-127, A stages 128-511
constexpr unsigned HT_ACOL0 = HT_F * 32;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

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

__device__ __forceinline__ void bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// no-swizzle K-major descriptor of an operator image block: K-adjacent core
// matrices 512 B apart (LBO), N-adjacent 128 B apart (SBO)
__device__ __forceinline__ uint64_t img_desc(unsigned addr) {
  const uint64_t lbo = 512, sbo = 128;
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((lbo >> 4) << 16) | ((sbo >> 4) << 32) | (1ull << 46);
}

// kind::tf32, D F32, A and B TF32 K-major, M = 128
template <int N>
__device__ __forceinline__ constexpr unsigned idesc_tf32() {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(HT_M >> 4) << 24);
}

// one frequency's 4 MMAs of a step in one block, issued by one elected
// lane of the converged warp: for K-half kh (A columns a + 8 kh head, + 16
// tail; operator block at descriptor b + 1024 kh bytes)
//   D[d, +32) (+)= A_hi [B_hi | B_lo]^T,  D[d, +16) += A_lo B_hi^T
// the first product overwrites D when acc == 0
__device__ __forceinline__ void mma_freq(unsigned d, unsigned a, uint64_t b, int acc) {
  asm volatile(
      "{\n"
      " .reg .pred e, p, t;\n"
      " .reg .b32 a;\n"
      " .reg .b64 b;\n"
      " setp.ne.b32 p, %3, 0;\n"
      " setp.eq.b32 t, %3, %3;\n"
      " elect.sync _|e, 0xffffffff;\n"
      " add.u64 b, %2, 0;\n"
      " add.u32 a, %1, 0;\n"
      " @e tcgen05.mma.cta_group::1.kind::tf32 [%0], [a], b, %4, p;\n"
      " add.u32 a, %1, 16;\n"
      " @e tcgen05.mma.cta_group::1.kind::tf32 [%0], [a], b, %5, t;\n"
      " add.u64 b, %2, 64;\n"
      " add.u32 a, %1, 8;\n"
      " @e tcgen05.mma.cta_group::1.kind::tf32 [%0], [a], b, %4, t;\n"
      " add.u32 a, %1, 24;\n"
      " @e tcgen05.mma.cta_group::1.kind::tf32 [%0], [a], b, %5, t;\n"
      "}\n" ::"r"(d),
      "r"(a), "l"(b), "r"(acc), "r"(idesc_tf32<32>()), "r"(idesc_tf32<16>())
      : "memory");
}

// non-blocking test of an mbarrier phase
__device__ __forceinline__ bool mbar_test(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void commit_elect(unsigned bar) {
  asm volatile(
      "{\n .reg .pred e;\n elect.sync _|e, 0xffffffff;\n"
      " @e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n}\n" ::"r"(bar)
      : "memory");
}

// 16 TMEM lanes x 32 columns: registers 4 i .. 4 i + 3 go to column block i
// (8 columns); thread t's registers 4 i, 4 i + 1 to lane t / 4, columns
// 8 i + 2 (t % 4) + {0, 1}, registers 4 i + 2, 4 i + 3 to lane t / 4 + 8
__device__ __forceinline__ void tmem_st16x256_x4(unsigned taddr, const unsigned* r) {
  asm volatile(
      "tcgen05.st.sync.aligned.16x256b.x4.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}

// one 32-byte read-only load
__device__ __forceinline__ void ld32B(const float* p, float* r) {
  asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7])
               : "l"(p));
}

__device__ __forceinline__ void tmem_ld32(unsigned taddr, unsigned* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}

// TF32 heads (the leading 10 mantissa bits) of a complex value and the exact
// FP32 remainders; the tensor core reads the remainders' leading 10 mantissa
// bits (relative error of a split value below 2^-20)
__device__ __forceinline__ void split_hl2(float re, float im, unsigned* hi, unsigned* lo) {
  hi[0] = __float_as_uint(re) & 0xFFFFE000u;
  hi[1] = __float_as_uint(im) & 0xFFFFE000u;
  lo[0] = __float_as_uint(re - __uint_as_float(hi[0]));
  lo[1] = __float_as_uint(im - __uint_as_float(hi[1]));
}

// The step sequence of one CTA: (item, direction) over its items in order,
// directions the item's tile has.  Every role walks the same sequence.
struct StepIter {
  int li, d, tile, fc;
  unsigned dm;
};

template <int NF>
__global__ void __launch_bounds__(HT_THREADS, 1)
    k_m2l_had_tc(const float* __restrict__ img, const float* __restrict__ spectra, int nq, int ntiles,
                 const int* __restrict__ qchd, const int* __restrict__ coll, const unsigned char* __restrict__ mask,
                 const unsigned* __restrict__ tile_dirs, float* __restrict__ effval, int zero_node, int nitems,
                 int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem[];  // HT_NB operator stages
  __shared__ __align__(8) unsigned long long bfull[HT_NB], afull[HT_ASTAGES], aempty[HT_ASTAGES], accfull, accempty,
      lastbar;
  __shared__ unsigned tmem_base;
  __shared__ int fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if ((int)blockIdx.x >= nitems) return;
  const int my_items = (nitems - 1 - (int)blockIdx.x) / (int)gridDim.x + 1;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(HT_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int b = 0; b < HT_ASTAGES; b++) {
      mbar_init(smem_u32(&afull[b]), 128);
      mbar_init(smem_u32(&aempty[b]), HT_F);
    }
    for (int b = 0; b < HT_NB; b++) mbar_init(smem_u32(&bfull[b]), 1);
    mbar_init(smem_u32(&accfull), HT_F);
    mbar_init(smem_u32(&accempty), 128);
    mbar_init(smem_u32(&lastbar), HT_F);
    fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_base;
  volatile int* vfail = &fail;
  // warp-uniform bounded wait (the tcgen05 .sync.aligned operations after it
  // need the whole warp): false for every lane once any wait has timed out
  auto wait = [&](unsigned long long* bar, int parity) {
    const bool ok = mbar_wait_bounded(smem_u32(bar), parity);
    if (__all_sync(0xffffffffu, ok)) return true;
    *vfail = 1;
    return false;
  };
  // item li -> (tile, frequency chunk), chunk major over the grid
  auto start = [&](StepIter& it, int li) {
    it.li = li;
    it.d = -1;
    if (li < my_items) {
      const int i = blockIdx.x + li * gridDim.x;
      it.fc = i / ntiles;
      it.tile = i - it.fc * ntiles;
      it.dm = tile_dirs[it.tile];
    }
  };
  // advance to the next step; false past the last item
  auto next = [&](StepIter& it) {
    while (it.li < my_items) {
      const unsigned rest = it.d >= 25 ? 0u : (it.dm >> (it.d + 1));
      if (rest) {
        it.d += __ffs(rest);
        return true;
      }
      start(it, it.li + 1);
    }
    return false;
  };
  // advance three steps: inside an item, the third set bit of the direction
  // mask above d (two bit clears and one find-first-set); across an item's
  // end, three single steps
  auto next3 = [&](StepIter& it) {
    if (it.d < 25) {
      unsigned r = it.dm >> (it.d + 1);
      r &= r - 1u;
      r &= r - 1u;
      if (r) {
        it.d += __ffs(r);
        return true;
      }
    }
    bool o = next(it);
    if (o) o = next(it);
    if (o) o = next(it);
    return o;
  };

  // drain item li from TMEM lane quarter (warp & 3) into effval: wait for the
  // item's MMAs, read the four frequencies' accumulators, release them,
  // store the rows' V-list children
  auto drain = [&](int li) {
    StepIter it;
    start(it, li);
    if (!wait(&accfull, li & 1)) return false;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = (warp & 3) * 32 + lane;
    const unsigned lane_off = (unsigned)((warp & 3) * 32) << 16;
    const int q = it.tile * HT_M + row;
    const bool qv = q < nq;
    const int c0 = qv ? qchd[q] : 0;
    const unsigned m = qv ? mask[q] : 0u;
    // frequency f: head*head + tail*head in columns f*32 + 0-15, head*tail in
    // f*32 + 16-31; two frequencies at a time, the accumulator released after
    // the last read
#pragma unroll
    for (int fp = 0; fp < 2; fp++) {
      float y[2][16];
#pragma unroll
      for (int e = 0; e < 2; e++) {
        unsigned r[32];
        tmem_ld32(tmem + lane_off + (2 * fp + e) * 32, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int n = 0; n < 16; n++) y[e][n] = __uint_as_float(r[n]) + __uint_as_float(r[16 + n]);
      }
      if (fp == 1) {
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&accempty)) : "memory");
      }
      float4* dst = reinterpret_cast<float4*>(effval) + ((size_t)c0 * NF + it.fc * HT_F + 2 * fp) / 2;
#pragma unroll
      for (int i = 0; i < 8; i++)
        if ((m >> i) & 1)
          dst[(size_t)i * (NF / 2)] = make_float4(y[0][2 * i], y[0][2 * i + 1], y[1][2 * i], y[1][2 * i + 1]);
    }
    return true;
  };

  if (warp < HT_MMA_WARP) {
    // ---- producers: warp (grp, quarter) writes TMEM lanes 32 * quarter ..
    // + 31 in two halves of 16; thread t carries rows t / 4 and t / 4 + 8 of
    // each half and child 4 kh + t % 4 of each row's colleague
    const int grp = warp >> 2, qd = warp & 3, c = lane & 3;
    // colleague first children of this thread's rows 32 qd + 16 h + 8 ab + t / 4
    auto load_nb = [&](const StepIter& x, int* nb) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int q = x.tile * HT_M + qd * 32 + 16 * (k >> 1) + 8 * (k & 1) + (lane >> 2);
        nb[k] = q < nq ? __ldg(coll + (size_t)q * 26 + x.d) : zero_node;
      }
    };
    // the group walks its own steps only, s = grp, grp + 3, ...: from step s
    // it goes to s + 3 directly, and fetches the colleague indices of s + 3
    // as soon as step s's spectra loads are issued, a whole round of the
    // three groups before they are used
    StepIter it;
    start(it, 0);
    bool ok = true;
    for (int k = 0; k <= grp && ok; k++) ok = next(it);
    int s = grp, pend = -1;  // pend: step of an operator copy not yet seen landed
    int nb[4];               // colleague first children of this thread's rows at step s
    if (ok) load_nb(it, nb);
    while (ok) {
      // the step's operator images into stage s mod 6, last read by step
      // s - 6, whose MMAs completed before this group's stage wait of step
      // s - 3 (stages s mod 6 and s + 3 mod 6 belong to this group alone)
      if (qd == 0 && lane == 0) {
        bulk_load(smem_u32(smem + (size_t)(s % HT_NB) * HT_IMG_BYTES),
                  img + ((size_t)it.fc * 26 + it.d) * HT_IMG_FLOATS, HT_IMG_BYTES, smem_u32(&bfull[s % HT_NB]));
      }
      if (qd == 0) pend = s;
      // v[h][ab][kh]: 4 complex (frequencies f0 .. f0 + 3) of child 4 kh + c
      // of the colleague of row 32 qd + 16 h + 8 ab + t / 4
      float v[2][2][2][8];
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int ab = 0; ab < 2; ab++) {
          // the colleague's block of this chunk: 8 children x 4 frequencies
          const float* row = spectra + (((size_t)((nb[2 * h + ab] + 7) >> 3) * (NF / HT_F) + it.fc) * 8 + c) * 8;
          ld32B(row, v[h][ab][0]);
          ld32B(row + 32, v[h][ab][1]);
        }
      // the group's next step and its colleague indices (nb is free once the
      // loads above are issued)
      StepIter nx = it;
      const bool okn = next3(nx);
      if (okn) load_nb(nx, nb);
      if (s >= HT_ASTAGES && !wait(&aempty[grp], ((s / HT_ASTAGES) + 1) & 1)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned abase = tmem + HT_ACOL0 + (unsigned)grp * (HT_F * 32);
      // frequency f: column blocks f*32 + {head kh 0, head kh 1, tail kh 0,
      // tail kh 1}; block column 2 (t % 4) + (re, im) = child 4 kh + t % 4
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int f = 0; f < HT_F; f++) {
          unsigned r[16];
#pragma unroll
          for (int kh = 0; kh < 2; kh++)
#pragma unroll
            for (int ab = 0; ab < 2; ab++)
              split_hl2(v[h][ab][kh][2 * f], v[h][ab][kh][2 * f + 1], &r[4 * kh + 2 * ab], &r[8 + 4 * kh + 2 * ab]);
          tmem_st16x256_x4(abase + ((unsigned)(qd * 32 + 16 * h) << 16) + f * 32, r);
        }
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      if (qd == 0) {
        if (!wait(&bfull[s % HT_NB], (s / HT_NB) & 1)) break;
        pend = -1;
      }
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&afull[grp])) : "memory");
      it = nx;
      ok = okn;
      s += HT_ASTAGES;
    }
    // after a time-out: the copy this warp issued last has landed before the CTA ends
    if (pend >= 0) mbar_wait_bounded(smem_u32(&bfull[pend % HT_NB]), (pend / HT_NB) & 1);
  } else {
    // ---- MMA warps: warp HT_MMA_WARP + f, frequency f.  The next step's
    // afull is tested (without blocking) before this step's MMAs go out, so
    // the test's latency hides behind them.  The warps go item by item: an
    // item's step count is the population count of its tile's direction mask
    // (loaded one item ahead), so a step costs no walk of the mask
    const int f = warp - HT_MMA_WARP;
    auto tile_of = [&](int li) {
      const int i = blockIdx.x + li * gridDim.x;
      return i - (i / ntiles) * ntiles;
    };
    int s = 0;
    bool ready = false;  // afull of step s seen complete
    bool failed = false;
    unsigned dm_next = __ldg(tile_dirs + tile_of(0));
    for (int li = 0; li < my_items; li++) {
      const unsigned dm = dm_next;
      if (li + 1 < my_items) dm_next = __ldg(tile_dirs + tile_of(li + 1));
      const int nst = __popc(dm);
      for (int k = 0; k < nst; k++) {
        const int stg = s % HT_ASTAGES;
        if (!__all_sync(0xffffffffu, ready) && !wait(&afull[stg], (s / HT_ASTAGES) & 1)) {
          failed = true;
          break;
        }
        if (k == 0 && li >= 1 && !wait(&accempty, (li - 1) & 1)) {
          failed = true;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int s1 = s + 1;
        ready = mbar_test(smem_u32(&afull[s1 % HT_ASTAGES]), (s1 / HT_ASTAGES) & 1);
        mma_freq(tmem + f * 32, tmem + HT_ACOL0 + (unsigned)stg * (HT_F * 32) + f * 32,
                 img_desc(smem_u32(smem + (size_t)(s % HT_NB) * HT_IMG_BYTES + f * 2048)), k == 0 ? 0 : 1);
        commit_elect(smem_u32(&aempty[stg]));
        s++;
      }
      if (failed) break;
      commit_elect(smem_u32(&accfull));
      if (!drain(li)) break;  // lane quarter warp mod 4 of the item just finished
    }
    // before the CTA ends every MMA issued has completed (only a time-out
    // leaves any outstanding)
    commit_elect(smem_u32(&lastbar));
    mbar_wait_bounded(smem_u32(&lastbar), 0);
  }
  __syncthreads();
  if (*vfail && tid == 0) atomicOr(status, 4);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(HT_COLS) : "memory");
  }
}

template <int NF>
void had_tc_launch(const float* img, const float* spectra, int nq, const int* qchd, const int* coll,
                   const unsigned char* mask, const unsigned* tile_dirs, float* effval, int zero_node, int* status,
                   int num_sms, cudaStream_t st) {
  const int ntiles = (nq + HT_M - 1) / HT_M;
  const int nitems = ntiles * (NF / HT_F);
  if (nitems == 0) return;
  const size_t smem = (size_t)HT_NB * HT_IMG_BYTES;
  auto kern = k_m2l_had_tc<NF>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int grid = std::min(num_sms, nitems);
  kern<<<grid, HT_THREADS, smem, st>>>(img, spectra, nq, ntiles, qchd, coll, mask, tile_dirs, effval, zero_node,
                                       nitems, status);
}

inline float tf32_round_host(float x) {
  unsigned u;
  std::memcpy(&u, &x, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  std::memcpy(&x, &u, 4);
  return x;
}

}  // namespace

bool m2l_tc_supported(int nf, int sd, int td) {
  return sd == 1 && td == 1 && (nf == 260 || nf == 868 || nf == 2052);
}

void m2l_tc_images(int nf, const std::complex<double>* m2l, std::vector<float>* img) {
  const int nch = nf / HT_F;
  img->assign((size_t)nch * 26 * HT_IMG_FLOATS, 0.f);
  for (int dir = 0; dir < 26; dir++) {
    const int dd = dir < 13 ? dir : dir + 1;
    const int dv[3] = {dd / 9 - 1, (dd / 3) % 3 - 1, dd % 3 - 1};
    for (int i = 0; i < 8; i++)      // target child
      for (int j = 0; j < 8; j++) {  // source child
        const int o[3] = {2 * dv[0] + ((j >> 2) & 1) - ((i >> 2) & 1), 2 * dv[1] + ((j >> 1) & 1) - ((i >> 1) & 1),
                          2 * dv[2] + (j & 1) - (i & 1)};
        if (std::max(std::abs(o[0]), std::max(std::abs(o[1]), std::abs(o[2]))) <= 1) continue;  // adjacent
        const int oi = (o[0] + 3) * 49 + (o[1] + 3) * 7 + (o[2] + 3);
        for (int f = 0; f < nf; f++) {
          const std::complex<double> t = m2l[(size_t)oi * nf + f];
          // rows 2i + (re, im), columns 2j + (re, im): [[re, -im], [im, re]]
          const double b[2][2] = {{t.real(), -t.imag()}, {t.imag(), t.real()}};
          float* blk = img->data() + ((size_t)(f / HT_F) * 26 + dir) * HT_IMG_FLOATS + (f % HT_F) * 512;
          for (int a = 0; a < 2; a++)
            for (int c = 0; c < 2; c++) {
              const int n = 2 * i + a, k = 2 * j + c;
              const float hi = tf32_round_host((float)b[a][c]);
              const float lo = tf32_round_host((float)(b[a][c] - (double)hi));
              // image offset of (row, k): K-adjacent core matrices 512 B apart,
              // row groups of 8 128 B apart; rows 16-31 hold the tails
              auto at = [&](int row) { return (k / 4) * 128 + (row / 8) * 32 + (row % 8) * 4 + (k % 4); };
              blk[at(n)] = hi;
              blk[at(16 + n)] = lo;
            }
        }
      }
  }
}

void launch_m2l_hadamard_tc(int nf, const float* img, const float* spectra, int nq, const int* qchd,
                            const int* coll, const unsigned char* mask, const unsigned* tile_dirs, float* effval,
                            int zero_node, int* status, int num_sms, cudaStream_t st) {
  if (nf == 868)
    had_tc_launch<868>(img, spectra, nq, qchd, coll, mask, tile_dirs, effval, zero_node, status, num_sms, st);
  else if (nf == 260)
    had_tc_launch<260>(img, spectra, nq, qchd, coll, mask, tile_dirs, effval, zero_node, status, num_sms, st);
  else if (nf == 2052)
    had_tc_launch<2052>(img, spectra, nq, qchd, coll, mask, tile_dirs, effval, zero_node, status, num_sms,
                        st);
}

}  // namespace kifmm
