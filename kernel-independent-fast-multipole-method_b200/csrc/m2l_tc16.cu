// V-list Hadamard accumulate on the 5th-generation tensor cores with 16-bit
// operands (tcgen05, kind::f16) for single-dof equivalent kernels in mixed
// precision: the frequency-domain product of the reference's M2L
// (fmm3d/fmm3d_eval.cpp:115-150, MatMgnt3d::UE2DC_dgemv
// fmm3d/matmgnt3d.cpp:272-290), in the parent-pair form of the V list.
//
// For target parent Q, colleague direction d (P = Q + d) and frequency f the
// V-list products of Q's 8 children with P's 8 children are one 8 x 8
// complex block, M[i][j] = K(2d + oct(j) - oct(i)) (zero for adjacent child
// pairs), applied to P's 8 child spectra; in real arithmetic a 16 x 16
// block B_d(f), and for a tile of 128 target parents
//   D(f)[128 x 16] = sum_d A_d(f)[128 x 16] B_d(f)^T,
// A_d(f) row q = the 8 child spectra of q's colleague in direction d.
//
// Operands are FP16 pairs: every spectrum value x (scaled by a power of two
// s_A) is stored as hi = fp16(x s_A) and lo = fp16(x s_A - hi), both rounded
// to nearest, so hi + lo carries x to 2^-22; the operator images likewise
// with a per-chunk power-of-two scale s_B.  Per frequency two MMAs
//   D[0:32)  += A_hi [B_hi | B_lo]^T    (N = 32)
//   D[0:16)  += A_lo B_hi^T             (N = 16)
// and the drain adds D[16:32) to D[0:16) and multiplies by 1/(s_A s_B):
// head*head, both cross terms, lo*lo (2^-22 relative) dropped, the products
// exact in the FP32 accumulator.  s_A = 2^(14 - e) with 2^e >= the largest
// |x| any spectrum can hold (the L1 norm of a node's scaled density grid,
// reduced over the nodes by k_spectra_bound before the forward transform), so
// |hi| <= 2^14 never overflows FP16; values more than 2^28 below the bound
// lose precision, i.e. none that matter against the accumulated sum.
//
// The forward transform writes the pairs already split, in the 8 bytes an
// FP32 complex value takes in the sibling-group-major layout (the 8 children
// of a colleague x 4 frequencies x {hi, lo} x {re, im} = 256 contiguous
// bytes, 32 per child), so a producer only moves bytes: four adjacent
// threads read one row's 128-byte line (children 0-3, then 4-7) with 32-byte
// loads, and the K order of the A rows (column 2c + e of a column block =
// child c + 4e, the operator images permuted to match) lets thread c write
// what it loaded with 16x256b TMEM stores.  Against the TF32 form this halves
// the TMEM bytes per step (32 KB), the A stage (64 columns, so six stages fit
// beside the 128-column accumulator instead of three) and the operator
// images (4 KB per step), removes the producers' split arithmetic, and runs
// the MMAs at the 16-bit rate.
//
// Work items are (frequency chunk of 4, tile of 128 target parents), chunk
// major over a persistent grid; inside an item the steps are the tile's
// present colleague directions.  Warp roles, handing over through mbarriers:
//   warps 0 .. 4G-1  producers, G groups of four (one warp per TMEM lane
//               quarter); group g fills the steps s = g mod G, step s into A
//               stage s mod 2G, so a group's stage wait looks two of its own
//               steps back.  Per step a producer thread issues all eight of
//               its 32-byte loads at once (the step waits for memory once),
//               reads the colleague groups of its rows at the group's next
//               step from the tile-major colleague table (m2l_tc16_tables)
//               right after them, and issues the step's operator-image copy
//               (image stage s mod 3G) before waiting for its A stage.
//   warps 4G .. 4G+3  MMA warps: warp 4G + f issues frequency f's 2 MMAs of
//               every step (own accumulator columns, one elected lane) and
//               commits; at an item's end each drains TMEM lane quarter
//               (warp mod 4), all four frequencies, into the
//               sibling-group-major accumulated spectra with 32-byte stores
//               (a target parent's 8 children x 4 frequencies are one block)
//   bfull[3G]  (bytes)         operator images landed           copy -> producers
//   afull[2G]  (128 arrivals)  A stage written, images landed   producers -> MMA
//   aempty[2G] (4 commits)     step's MMAs done                 MMA -> producers
//   accfull    (4 commits)     item's MMAs done                 MMA -> drain
//   accempty   (128 arrivals)  accumulator read out             drain -> MMA
// Every pipeline wait is bounded by wait_limit polls; a time-out sets bit 3
// of *status and ends the CTA after its copies landed and its MMAs completed
// (those two final waits use a fixed, long bound).
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "launch.hpp"

namespace kifmm {
namespace {

constexpr int H16_M = 128;                       // target parents per tile (MMA M, TMEM lanes)
// G producer groups (2 or 3), 2 G A stages, MMA warps from warp 4 G on,
// 3 G operator image stages
constexpr int h16_threads(int G) { return (4 * G + 4) * 32; }
constexpr unsigned H16_COLS = 512;
constexpr int H16_LONG_WAIT = 1 << 22;           // polls of the end-of-CTA waits
// Per target-dof count TD (1, or 3 for Stokes and Navier): FI frequencies
// per item, every target dof's accumulator resident in TMEM (TD x FI x 32
// columns from column 0), A stages of FI x 16 columns after them, operator
// images of TD x FI x 1 KB per step (all target dofs of one source dof and
// direction)
template <int TD>
struct H16Shape {
  static constexpr int FI = TD == 1 ? 4 : 2;
  // source dofs per step: a multi-dof step carries a pair (the A stage then
  // holds 2 dofs x 2 frequencies, the bytes of one single-dof step), and its
  // accumulators are 16 columns (the head*tail product is a third N = 16
  // MMA instead of the upper half of an N = 32 one)
  static constexpr int SPS = TD == 1 ? 1 : 2;
  static constexpr unsigned ACC = TD == 1 ? 32 : 16;
  static constexpr unsigned ACOL0 = TD * FI * ACC;
  static constexpr unsigned ACOLS = SPS * FI * 16;
  static constexpr unsigned IMGB = SPS * TD * FI * 1024;
};
// steps per colleague direction: the source-dof pairs
constexpr int h16_dof_steps(int SD, int TD) { return TD == 1 ? SD : (SD + 1) / 2; }

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity, int limit) {
  for (int it = 0; it < limit; it++) {
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

__device__ __forceinline__ void bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// no-swizzle K-major descriptor of one frequency's operator image (32 rows x
// 16 K of fp16): the two K-adjacent core matrices 512 B apart (LBO), row
// groups of 8 128 B apart (SBO)
__device__ __forceinline__ uint64_t img_desc16(unsigned addr) {
  const uint64_t lbo = 512, sbo = 128;
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((lbo >> 4) << 16) | ((sbo >> 4) << 32) | (1ull << 46);
}

// kind::f16, D F32, A and B FP16, both K-major, M = 128
template <int N>
__device__ __forceinline__ constexpr unsigned idesc_f16() {
  return (1u << 4) | ((unsigned)(N >> 3) << 17) | ((unsigned)(H16_M >> 4) << 24);
}

// one frequency's 2 MMAs of a step, issued by one elected lane of the
// converged warp: D[d, +32) (+)= A_hi [B_hi | B_lo]^T, D[d, +16) += A_lo B_hi^T
// (A_lo 8 columns after A_hi); the first product overwrites D when acc == 0
__device__ __forceinline__ void mma_freq16(unsigned d, unsigned a, uint64_t b, int acc) {
  asm volatile(
      "{\n"
      " .reg .pred e, p, t;\n"
      " .reg .b32 a;\n"
      " setp.ne.b32 p, %3, 0;\n"
      " setp.eq.b32 t, %3, %3;\n"
      " elect.sync _|e, 0xffffffff;\n"
      " @e tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %4, p;\n"
      " add.u32 a, %1, 8;\n"
      " @e tcgen05.mma.cta_group::1.kind::f16 [%0], [a], %2, %5, t;\n"
      "}\n" ::"r"(d),
      "r"(a), "l"(b), "r"(acc), "r"(idesc_f16<32>()), "r"(idesc_f16<16>())
      : "memory");
}

// one (target dof, frequency, source dof) block product of a multi-dof step
// into its N = 16 accumulator: D (+)= A_hi B_hi^T + A_lo B_hi^T + A_hi B_lo^T
// (A_lo 8 columns after A_hi, B_lo the image's rows 16-31)
__device__ __forceinline__ void mma3_16(unsigned d, unsigned a, uint64_t bhi, uint64_t blo, int acc) {
  asm volatile(
      "{\n"
      " .reg .pred e, p, t;\n"
      " .reg .b32 a;\n"
      " setp.ne.b32 p, %4, 0;\n"
      " setp.eq.b32 t, %4, %4;\n"
      " elect.sync _|e, 0xffffffff;\n"
      " @e tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %5, p;\n"
      " add.u32 a, %1, 8;\n"
      " @e tcgen05.mma.cta_group::1.kind::f16 [%0], [a], %2, %5, t;\n"
      " @e tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %3, %5, t;\n"
      "}\n" ::"r"(d),
      "r"(a), "l"(bhi), "l"(blo), "r"(acc), "r"(idesc_f16<16>())
      : "memory");
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
__device__ __forceinline__ void ld32B(const unsigned* p, unsigned* r) {
  asm volatile("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "l"(p));
}

// one 16-byte read-only load
__device__ __forceinline__ void ld16B(const unsigned* p, unsigned* r) {
  asm volatile("ld.global.nc.v4.b32 {%0,%1,%2,%3}, [%4];" : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "l"(p));
}

// one 32-byte store
__device__ __forceinline__ void st32B(float* p, float a, float b, float c, float d, float e, float f, float g, float h) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d), "f"(e),
               "f"(f), "f"(g), "f"(h)
               : "memory");
}

// 16 consecutive columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(unsigned taddr, unsigned* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// 2^(e - 14) for the data bound b <= 2^e (b > 0), the inverse of the data scale
__device__ __forceinline__ float inv_data_scale(float b) {
  if (!(b > 0.f)) return 1.f;
  int e;
  frexpf(b, &e);
  return ldexpf(1.f, e - 14);
}

constexpr int H16_NBI = 9;  // room for the operator image stages (G + 2 G for G <= 3)

// dynamic shared memory: image stages, then the CTA's item direction masks
constexpr size_t h16_smem(unsigned imgb, int max_items) { return (size_t)H16_NBI * imgb + 4 * (size_t)max_items; }

// one step forward in a CTA's step sequence (items li in grid-stride order,
// the directions d of each item's mask dm, and for each direction the SD
// source dofs sx); false past the last item
template <int SD>
__device__ __forceinline__ bool h16_step(int& li, int& d, int& sx, int& fc, int& tile, unsigned& dm,
                                         const unsigned* dirs, int my_items, int ntiles) {
  if (SD > 1 && sx + 1 < SD) {
    sx++;
    return true;
  }
  sx = 0;
  const unsigned rest = d >= 25 ? 0u : (dm >> (d + 1));
  if (rest) {
    d += __ffs(rest);
    return true;
  }
  if (++li >= my_items) return false;
  tile += gridDim.x;
  while (tile >= ntiles) {
    tile -= ntiles;
    fc++;
  }
  dm = dirs[li];
  d = __ffs(dm) - 1;
  return true;
}

// G steps forward: inside an item (one source dof) the G-th set bit of the
// mask above d, across an item's end single steps; single steps throughout
// for several source dofs
template <int G, int SD>
__device__ __forceinline__ bool h16_stepG(int& li, int& d, int& sx, int& fc, int& tile, unsigned& dm,
                                          const unsigned* dirs, int my_items, int ntiles) {
  if (SD == 1 && d < 25) {
    unsigned r = dm >> (d + 1);
#pragma unroll
    for (int k = 0; k < G - 1; k++) r &= r - 1u;
    if (r) {
      d += __ffs(r);
      return true;
    }
  }
  bool ok = true;
#pragma unroll 1
  for (int k = 0; k < G && ok; k++) ok = h16_step<SD>(li, d, sx, fc, tile, dm, dirs, my_items, ntiles);
  return ok;
}

template <int NF, int H16_G, int SD, int TD>
__global__ void __launch_bounds__(h16_threads(H16_G), 1)
    k_m2l_had_tc16(const unsigned char* __restrict__ img, const unsigned* __restrict__ spectra, int nq, int ntiles,
                   const int* __restrict__ qchd, const int* __restrict__ ctab, const unsigned* __restrict__ tile_dirs,
                   float* __restrict__ effval, int nitems, size_t plane, const unsigned* __restrict__ bound,
                   const float* __restrict__ inv_sb, int wait_limit, int* __restrict__ status) {
  constexpr int H16_MMA_WARP = H16_G * 4;  // first of the 4 MMA warps
  constexpr int H16_S = 2 * H16_G;         // A stages: step s uses stage s mod S
  constexpr int H16_NB = H16_G + H16_S;    // operator image stages: step s uses s mod NB
  constexpr int FI = H16Shape<TD>::FI;
  constexpr unsigned ACOL0 = H16Shape<TD>::ACOL0, ACOLS = H16Shape<TD>::ACOLS, IMGB = H16Shape<TD>::IMGB;
  constexpr int SDS = h16_dof_steps(SD, TD);  // steps per direction (source dofs or their pairs)
  static_assert(ACOL0 + H16_S * ACOLS <= H16_COLS, "A stages fit in TMEM");
  static_assert(H16_NB <= H16_NBI, "image stages");
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* imgs = smem;                                       // [NB][IMGB]
  unsigned* dirs = reinterpret_cast<unsigned*>(smem + (size_t)H16_NBI * IMGB);
  __shared__ __align__(8) unsigned long long afull[H16_S], aempty[H16_S], bfull[H16_NB], accfull, accempty, lastbar;
  __shared__ unsigned tmem_base;
  __shared__ int fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if ((int)blockIdx.x >= nitems) return;
  const int my_items = (nitems - 1 - (int)blockIdx.x) / (int)gridDim.x + 1;
  auto tile_of = [&](int li) {
    const int i = blockIdx.x + li * gridDim.x;
    return i - (i / ntiles) * ntiles;
  };

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(H16_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int b = 0; b < H16_S; b++) {
      mbar_init(smem_u32(&afull[b]), 128);
      mbar_init(smem_u32(&aempty[b]), 4);
    }
    for (int b = 0; b < H16_NB; b++) mbar_init(smem_u32(&bfull[b]), 1);
    mbar_init(smem_u32(&accfull), 4);
    mbar_init(smem_u32(&accempty), 128);
    mbar_init(smem_u32(&lastbar), 4);
    fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int li = tid; li < my_items; li += blockDim.x) dirs[li] = __ldg(tile_dirs + tile_of(li));
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_base;
  volatile int* vfail = &fail;
  // warp-uniform bounded wait (the tcgen05 .sync.aligned operations after it
  // need the whole warp): false for every lane once any wait has timed out
  auto wait = [&](unsigned long long* bar, int parity) {
    const bool ok = mbar_wait_bounded(smem_u32(bar), parity, wait_limit);
    if (__all_sync(0xffffffffu, ok)) return true;
    *vfail = 1;
    return false;
  };

  if (warp < H16_MMA_WARP) {
    // ---- producers: warp (grp, quarter qd) writes TMEM lanes 32 qd .. + 31
    // in two halves h of 16; thread t carries rows t / 4 and t / 4 + 8 (ab)
    // of each half and children c, c + 4 (c = t % 4) of each row's colleague
    const int grp = warp >> 2, qd = warp & 3, c = lane & 3;
    const int rbase = qd * 32 + (lane >> 2);
    const unsigned abase = tmem + ACOL0 + ((unsigned)(qd * 32) << 16);
    // the group's steps s = grp, grp + G, ...: item li, direction d, source
    // dof sx; the item's chunk fc (of FI frequencies) and tile advance by
    // grid strides
    int li = 0, d = -1, sx = SD - 1, fc = blockIdx.x / ntiles, tile = blockIdx.x - fc * ntiles;
    unsigned dm = dirs[0];
    bool ok = true;
    for (int k = 0; k <= grp && ok; k++) ok = h16_step<SDS>(li, d, sx, fc, tile, dm, dirs, my_items, ntiles);
    // the colleague groups of this thread's 4 rows at the group's next step,
    // loaded one group step ahead of their use
    int g0 = 0, g1 = 0, g2 = 0, g3 = 0;
#define H16_LOAD_G()                                                  \
  {                                                                   \
    const int* tb = ctab + ((size_t)tile * 26 + d) * H16_M + rbase;   \
    g0 = __ldg(tb);                                                   \
    g1 = __ldg(tb + 8);                                               \
    g2 = __ldg(tb + 16);                                              \
    g3 = __ldg(tb + 24);                                              \
  }
    if (ok) H16_LOAD_G()
    // x[h][ab][e][w] = word w (frequency w / 2 of the chunk, {hi, lo} =
    // w % 2) of child c + 4 e of the colleague of row (h, ab); a child's 4
    // frequencies of a 256-byte block are 8 words, FI = 2 takes half of them
    unsigned x[2][2][2][8];
    // the loads of half h of the step at the iterator's position (its
    // colleague groups in g0 .. g3)
#define H16_LOAD_HALF(h)                                                                                  \
  {                                                                                                       \
    if constexpr (TD == 1) {                                                                              \
      const size_t sbase = (size_t)fc * 64 + 8 * c;                                                       \
      _Pragma("unroll") for (int ab = 0; ab < 2; ab++) {                                                  \
        const int gk = (h) == 0 ? (ab == 0 ? g0 : g1) : (ab == 0 ? g2 : g3);                              \
        const unsigned* src = spectra + sbase + (size_t)gk * (NF / 4) * 64;                               \
        ld32B(src, x[h][ab][0]);                                                                          \
        ld32B(src + 32, x[h][ab][1]);                                                                     \
      }                                                                                                   \
    } else {                                                                                              \
      /* source dofs 2 sx and 2 sx + 1 (zero past the last): words 0-3 and 4-7 */                         \
      const size_t sbase = (size_t)(2 * sx) * plane * 2 + (size_t)(fc >> 1) * 64 + 8 * c + (fc & 1) * 4;  \
      const bool two = 2 * sx + 1 < SD;                                                                   \
      _Pragma("unroll") for (int ab = 0; ab < 2; ab++) {                                                  \
        const int gk = (h) == 0 ? (ab == 0 ? g0 : g1) : (ab == 0 ? g2 : g3);                              \
        const unsigned* src = spectra + sbase + (size_t)gk * (NF / 4) * 64;                               \
        ld16B(src, x[h][ab][0]);                                                                          \
        ld16B(src + 32, x[h][ab][1]);                                                                     \
        if (two) {                                                                                        \
          ld16B(src + plane * 2, x[h][ab][0] + 4);                                                        \
          ld16B(src + plane * 2 + 32, x[h][ab][1] + 4);                                                   \
        } else {                                                                                          \
          _Pragma("unroll") for (int q = 4; q < 8; q++) x[h][ab][0][q] = x[h][ab][1][q] = 0u;             \
        }                                                                                                 \
      }                                                                                                   \
    }                                                                                                     \
  }
    if (ok) {
      H16_LOAD_HALF(0)
      H16_LOAD_HALF(1)
    }
    int s = grp, pend = -1;  // pend: step of an operator copy not yet seen landed
    while (ok) {
      // the step's operator images into stage s mod NB, last read by step
      // s - NB; this group's stage wait of step s - G saw the MMAs of step
      // s - G - S complete, and NB = G + S
      // images [chunk][direction][source dof][target dof][frequency]
      if (qd == 0 && lane == 0)
        bulk_load(smem_u32(imgs + (size_t)(s % H16_NB) * IMGB), img + (((size_t)fc * 26 + d) * SDS + sx) * IMGB, IMGB,
                  smem_u32(&bfull[s % H16_NB]));
      if (qd == 0) pend = s;
      const int stg = s % H16_S, sb = s % H16_NB, sbp = (s / H16_NB) & 1;
      // the iterator moves to the group's next step and its colleague groups
      // are requested; the step's own data is already in x
      const bool nxt = h16_stepG<H16_G, SDS>(li, d, sx, fc, tile, dm, dirs, my_items, ntiles);
      if (nxt) H16_LOAD_G()
      if (s >= H16_S && !wait(&aempty[stg], ((s / H16_S) + 1) & 1)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // column block b = 2 f + {hi, lo} (f over the frequencies, or over the
      // pair's dofs x frequencies); in every block column 2c + e holds
      // child c + 4e; one store per half h and 4 column blocks L.  Each
      // half's registers take the next step's loads as soon as its stores
      // are issued, so those loads are in flight through this step's store
      // wait, image wait and arrive
#pragma unroll
      for (int h = 0; h < 2; h++) {
#pragma unroll
        for (int L = 0; L < 2; L++) {
          unsigned r[16];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            r[4 * i + 0] = x[h][0][0][4 * L + i];
            r[4 * i + 1] = x[h][0][1][4 * L + i];
            r[4 * i + 2] = x[h][1][0][4 * L + i];
            r[4 * i + 3] = x[h][1][1][4 * L + i];
          }
          tmem_st16x256_x4(abase + (unsigned)stg * ACOLS + ((unsigned)(16 * h) << 16) + 32 * L, r);
        }
        if (nxt) {
          if (h == 0)
            H16_LOAD_HALF(0)
          else
            H16_LOAD_HALF(1)
        }
      }
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      if (qd == 0) {
        if (!wait(&bfull[sb], sbp)) break;
        pend = -1;
      }
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&afull[stg])) : "memory");
      s += H16_G;
      ok = nxt;
    }
#undef H16_LOAD_HALF
#undef H16_LOAD_G
    // after a time-out: the copy this warp issued last has landed before the CTA ends
    if (pend >= 0) mbar_wait_bounded(smem_u32(&bfull[pend % H16_NB]), (pend / H16_NB) & 1, H16_LONG_WAIT);
  } else {
    // ---- MMA warps: warp H16_MMA_WARP + w issues the 2 MMAs of every
    // step for the accumulators kk = t FI + f = w, w + 4, ... (target dof t,
    // frequency f; own accumulator columns, one elected lane) and commits;
    // the next step's afull is tested without blocking before this step's
    // MMAs go out.  At an item's end each drains TMEM lane quarter
    // (warp mod 4), every accumulator, into effval.
    const int w = warp - H16_MMA_WARP;
    const float inv_sa = inv_data_scale(__uint_as_float(*bound));
    int s = 0;
    bool ready = false, failed = false;
    for (int li = 0; li < my_items; li++) {
      const int nst = __popc(dirs[li]) * SDS;
      for (int k = 0; k < nst; k++) {
        const int stg = s % H16_S;
        if (!__all_sync(0xffffffffu, ready) && !wait(&afull[stg], (s / H16_S) & 1)) {
          failed = true;
          break;
        }
        if (k == 0 && li >= 1 && !wait(&accempty, (li - 1) & 1)) {
          failed = true;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int s1 = s + 1;
        ready = mbar_test(smem_u32(&afull[s1 % H16_S]), (s1 / H16_S) & 1);
        // A_hi of frequency f: column block 2 f, A_lo block 2 f + 1
        if constexpr (TD == 1) {
#pragma unroll
          for (int kk = w; kk < FI; kk += 4)
            mma_freq16(tmem + kk * 32, tmem + ACOL0 + 16 * kk + (unsigned)stg * ACOLS,
                       img_desc16(smem_u32(imgs + (size_t)(s % H16_NB) * IMGB + kk * 1024)), k == 0 ? 0 : 1);
        } else {
          // accumulator kk = t FI + f; the pair's dof L = 0, 1 (the second
          // only where it exists): A blocks 2 (L FI + f) + {hi, lo}, images
          // [L][t][f]
          const int sp = k % SDS;
          const unsigned ib = smem_u32(imgs + (size_t)(s % H16_NB) * IMGB);
#pragma unroll
          for (int kk = w; kk < TD * FI; kk += 4) {
#pragma unroll
            for (int L = 0; L < 2; L++) {
              if (L == 1 && 2 * sp + 1 >= SD) break;
              const unsigned b = ib + (unsigned)((L * TD + kk / FI) * FI + kk % FI) * 1024u;
              mma3_16(tmem + kk * 16, tmem + ACOL0 + 16 * (L * FI + kk % FI) + (unsigned)stg * ACOLS,
                      img_desc16(b), img_desc16(b + 256), (k == 0 && L == 0) ? 0 : 1);
            }
          }
        }
        commit_elect(smem_u32(&aempty[stg]));
        s++;
      }
      if (failed) break;
      commit_elect(smem_u32(&accfull));
      // drain item li from TMEM lane quarter (warp & 3) into effval
      if (!wait(&accfull, li & 1)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int i = blockIdx.x + li * gridDim.x;
      const int fc = i / ntiles, tile = i - fc * ntiles;
      const int fc4 = FI == 4 ? fc : fc >> 1;  // the 4-frequency block
      const int row = (warp & 3) * 32 + lane;
      const unsigned lane_off = (unsigned)((warp & 3) * 32) << 16;
      const int q = tile * H16_M + row;
      const float scl = inv_sa * __ldg(inv_sb + fc4);
      const size_t gblk = q < nq ? ((size_t)((qchd[q] + 7) >> 3) * (NF / 4) + fc4) * 64 : 0;
#pragma unroll 1
      for (int t = 0; t < TD; t++) {
        // frequency f2: head*head + tail*head in columns 32 kk + 0-15,
        // head*tail in 32 kk + 16-31; y[f2][2 i + (re, im)] of child i
        float y[FI][16];
#pragma unroll
        for (int f2 = 0; f2 < FI; f2++) {
          unsigned r[16];
          const unsigned col = (unsigned)(t * FI + f2) * H16Shape<TD>::ACC;
          tmem_ld16(tmem + lane_off + col, r);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int n = 0; n < 16; n++) y[f2][n] = __uint_as_float(r[n]);
          if constexpr (TD == 1) {  // + the head*tail half
            tmem_ld16(tmem + lane_off + col + 16, r);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int n = 0; n < 16; n++) y[f2][n] += __uint_as_float(r[n]);
          }
#pragma unroll
          for (int n = 0; n < 16; n++) y[f2][n] *= scl;
        }
        if (t == TD - 1) {
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&accempty)) : "memory");
        }
        // the row's 8 children x 4 frequencies are one 256-byte block of the
        // sibling-group-major accumulated spectra of dof t (all 8 children;
        // the inverse pass reads only the V-list targets among them); FI = 2
        // writes half of each child's 32 bytes
        if (q < nq) {
          float* dst = effval + (TD == 1 ? 0 : (size_t)t * plane * 2) + gblk;
          if constexpr (FI == 4) {
#pragma unroll
            for (int ch = 0; ch < 8; ch++)
              st32B(dst + 8 * ch, y[0][2 * ch], y[0][2 * ch + 1], y[1][2 * ch], y[1][2 * ch + 1], y[2][2 * ch],
                    y[2][2 * ch + 1], y[3][2 * ch], y[3][2 * ch + 1]);
          } else {
#pragma unroll
            for (int ch = 0; ch < 8; ch++)
              *reinterpret_cast<float4*>(dst + 8 * ch + (fc & 1) * 4) =
                  make_float4(y[0][2 * ch], y[0][2 * ch + 1], y[1][2 * ch], y[1][2 * ch + 1]);
          }
        }
      }
    }
    // before the CTA ends every MMA issued has completed (only a time-out
    // leaves any outstanding)
    commit_elect(smem_u32(&lastbar));
    mbar_wait_bounded(smem_u32(&lastbar), 0, H16_LONG_WAIT);
  }
  __syncthreads();
  if (*vfail && tid == 0) atomicOr(status, 8);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(H16_COLS) : "memory");
  }
}

// bound = max over the nodes and source dofs s of 2^(lvl deg[s]) * sum_k
// |supeden[node][k][s]|, as FP32 bits (non-negative floats order like their
// bit patterns)
__global__ void __launch_bounds__(256) k_spectra_bound(const float* __restrict__ supeden, const int* __restrict__ nodes,
                                                       int n, const int* __restrict__ depth, int rootlvl, int4 deg,
                                                       int sd, int nsurf, unsigned* __restrict__ bound) {
  float best = 0.f;
  const int lane = threadIdx.x & 31;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += (gridDim.x * blockDim.x) >> 5) {
    const int node = nodes[w];
    const float* u = supeden + (size_t)node * nsurf * sd;
    for (int sx = 0; sx < sd; sx++) {
      float s = 0.f;
      for (int k = lane; k < nsurf; k += 32) s += fabsf(u[(size_t)k * sd + sx]);
#pragma unroll
      for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      const int dg = sx == 0 ? deg.x : sx == 1 ? deg.y : sx == 2 ? deg.z : deg.w;
      best = fmaxf(best, ldexpf(s, (depth[node] + rootlvl) * dg));
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
  __shared__ float red[8];
  if (lane == 0) red[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    float b = 0.f;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) b = fmaxf(b, red[k]);
    // a little headroom for the rounding of the FP32 transform
    atomicMax(bound, __float_as_uint(b * 1.0001f));
  }
}

template <int NF, int G, int SD, int TD>
void had_tc16_launch_g(const unsigned char* img, const unsigned* spectra, int nq, const int* qchd, const int* ctab,
                       const unsigned* tile_dirs, float* effval, size_t plane, const unsigned* bound,
                       const float* inv_sb, int wait_limit, int* status, int num_sms, cudaStream_t st) {
  const int ntiles = (nq + H16_M - 1) / H16_M;
  const int nitems = ntiles * (NF / H16Shape<TD>::FI);
  if (nitems == 0) return;
  const int grid = std::min(num_sms, nitems);
  const size_t smem = h16_smem(H16Shape<TD>::IMGB, (nitems + grid - 1) / grid);
  auto kern = k_m2l_had_tc16<NF, G, SD, TD>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<grid, h16_threads(G), smem, st>>>(img, spectra, nq, ntiles, qchd, ctab, tile_dirs, effval, nitems, plane,
                                           bound, inv_sb, wait_limit, status);
}

template <int NF, int SD, int TD>
void had_tc16_launch(int groups, const unsigned char* img, const unsigned* spectra, int nq, const int* qchd,
                     const int* ctab, const unsigned* tile_dirs, float* effval, size_t plane, const unsigned* bound,
                     const float* inv_sb, int wait_limit, int* status, int num_sms, cudaStream_t st) {
  if (groups == 2)
    had_tc16_launch_g<NF, 2, SD, TD>(img, spectra, nq, qchd, ctab, tile_dirs, effval, plane, bound, inv_sb,
                                     wait_limit, status, num_sms, st);
  else
    had_tc16_launch_g<NF, 3, SD, TD>(img, spectra, nq, qchd, ctab, tile_dirs, effval, plane, bound, inv_sb,
                                     wait_limit, status, num_sms, st);
}

template <int NF>
void had_tc16_dofs(int groups, int sd, int td, const unsigned char* img, const unsigned* spectra, int nq,
                   const int* qchd, const int* ctab, const unsigned* tile_dirs, float* effval, size_t plane,
                   const unsigned* bound, const float* inv_sb, int wait_limit, int* status, int num_sms,
                   cudaStream_t st) {
  if (sd == 1 && td == 1)
    had_tc16_launch<NF, 1, 1>(groups, img, spectra, nq, qchd, ctab, tile_dirs, effval, plane, bound, inv_sb,
                              wait_limit, status, num_sms, st);
  else if (sd == 4 && td == 3)
    had_tc16_launch<NF, 4, 3>(groups, img, spectra, nq, qchd, ctab, tile_dirs, effval, plane, bound, inv_sb,
                              wait_limit, status, num_sms, st);
  else if (sd == 3 && td == 3)
    had_tc16_launch<NF, 3, 3>(groups, img, spectra, nq, qchd, ctab, tile_dirs, effval, plane, bound, inv_sb,
                              wait_limit, status, num_sms, st);
}

}  // namespace

bool m2l_tc16_supported(int nf, int sd, int td) {
  const bool dofs = (sd == 1 && td == 1) || (sd == 4 && td == 3) || (sd == 3 && td == 3);
  return dofs && (nf == 260 || nf == 868 || nf == 2052);
}

void m2l_tc16_images(int nf, int sd, int td, const std::complex<double>* m2l, std::vector<unsigned short>* img,
                     std::vector<float>* inv_sb) {
  const int fi = td == 1 ? 4 : 2;  // frequencies per work item (H16Shape)
  // source-dof slots per direction: the dofs, rounded up to whole pairs for
  // several dofs (a padding slot stays zero)
  const int sds = td == 1 ? sd : (sd + 1) / 2 * 2;
  const int nch = nf / 4, ncf = nf / fi, nts = sd * td;
  img->assign((size_t)nf * 26 * sds * td * 512, 0);  // [chunk of fi][dir][s][t][fi] x 512 fp16
  inv_sb->assign(nch, 1.f);
  for (int fc = 0; fc < nch; fc++) {
    // the scale of each block of 4 frequencies (all dof pairs): 2^(14 - e)
    // with every |entry| <= 2^e
    double mx = 0;
    for (size_t o = 0; o < (size_t)343 * nts; o++)
      for (int f = fc * 4; f < fc * 4 + 4; f++) {
        const std::complex<double> t = m2l[o * nf + f];
        mx = std::max(mx, std::max(std::abs(t.real()), std::abs(t.imag())));
      }
    int e = 0;
    if (mx > 0) std::frexp(mx, &e);
    const double sb = std::ldexp(1.0, 14 - e);
    (*inv_sb)[fc] = (float)std::ldexp(1.0, e - 14);
    for (int dir = 0; dir < 26; dir++) {
      const int dd = dir < 13 ? dir : dir + 1;
      const int dv[3] = {dd / 9 - 1, (dd / 3) % 3 - 1, dd % 3 - 1};
      for (int i = 0; i < 8; i++)      // target child
        for (int j = 0; j < 8; j++) {  // source child
          const int o[3] = {2 * dv[0] + ((j >> 2) & 1) - ((i >> 2) & 1), 2 * dv[1] + ((j >> 1) & 1) - ((i >> 1) & 1),
                            2 * dv[2] + (j & 1) - (i & 1)};
          if (std::max(std::abs(o[0]), std::max(std::abs(o[1]), std::abs(o[2]))) <= 1) continue;  // adjacent
          const int oi = (o[0] + 3) * 49 + (o[1] + 3) * 7 + (o[2] + 3);
          for (int t = 0; t < td; t++)
            for (int sx = 0; sx < sd; sx++)
              for (int f = fc * 4; f < fc * 4 + 4; f++) {  // operator [343][td][sd][nf]
                const std::complex<double> v = m2l[((size_t)oi * nts + t * sd + sx) * nf + f] * sb;
                // rows 2i + (re, im), columns 2j + (re, im): [[re, -im], [im, re]]
                const double b[2][2] = {{v.real(), -v.imag()}, {v.imag(), v.real()}};
                const int cf = f / fi, fl = f % fi;
                unsigned short* blk =
                    img->data() + (((((size_t)cf * 26 + dir) * sds + sx) * td + t) * fi + fl) * 512;
                for (int a = 0; a < 2; a++)
                  for (int cc = 0; cc < 2; cc++) {
                    // K order of the A rows: column 2 c + e of a block = child c + 4 e
                    const int n = 2 * i + a, k = 2 * (2 * (j & 3) + (j >> 2)) + cc;
                    const __half hi = __float2half_rn((float)b[a][cc]);
                    const __half lo = __float2half_rn((float)(b[a][cc] - (double)__half2float(hi)));
                    // (row, k): K-adjacent core matrices 512 B apart, row groups
                    // of 8 128 B apart, rows 16 B apart; rows 16-31 hold the tails
                    auto at = [&](int row) { return (k / 8) * 256 + (row / 8) * 64 + (row % 8) * 8 + (k % 8); };
                    blk[at(n)] = __half_as_ushort(hi);
                    blk[at(16 + n)] = __half_as_ushort(lo);
                  }
              }
        }
    }
  }
  (void)ncf;
}

void launch_spectra_bound(const float* supeden, const int* nodes, int n, const int* depth, int rootlvl,
                          const int* deg, int sd, int nsurf, unsigned* bound, int num_sms, cudaStream_t st) {
  cudaMemsetAsync(bound, 0, sizeof(unsigned), st);
  if (n <= 0) return;
  const int grid = std::max(1, std::min(num_sms * 4, (n + 7) / 8));
  const int4 dg = make_int4(deg[0], sd > 1 ? deg[1] : 0, sd > 2 ? deg[2] : 0, sd > 3 ? deg[3] : 0);
  k_spectra_bound<<<grid, 256, 0, st>>>(supeden, nodes, n, depth, rootlvl, dg, sd, nsurf, bound);
}

void launch_m2l_hadamard_tc16(int groups, int nf, int sd, int td, const unsigned short* img,
                              const unsigned* spectra, int nq, const int* qchd, const int* ctab,
                              const unsigned* tile_dirs, float* effval, size_t plane, const unsigned* bound,
                              const float* inv_sb, int wait_limit, int* status, int num_sms, cudaStream_t st) {
  const unsigned char* im = reinterpret_cast<const unsigned char*>(img);
  if (nf == 868)
    had_tc16_dofs<868>(groups, sd, td, im, spectra, nq, qchd, ctab, tile_dirs, effval, plane, bound, inv_sb,
                       wait_limit, status, num_sms, st);
  else if (nf == 260)
    had_tc16_dofs<260>(groups, sd, td, im, spectra, nq, qchd, ctab, tile_dirs, effval, plane, bound, inv_sb,
                       wait_limit, status, num_sms, st);
  else if (nf == 2052)
    had_tc16_dofs<2052>(groups, sd, td, im, spectra, nq, qchd, ctab, tile_dirs, effval, plane, bound, inv_sb,
                        wait_limit, status, num_sms, st);
}

void m2l_tc16_tables(int nq, int zero_node, const int* coll, std::vector<int>* ctab) {
  const int ntiles = (nq + H16_M - 1) / H16_M;
  ctab->assign((size_t)ntiles * 26 * H16_M, (zero_node + 7) >> 3);
  for (int q = 0; q < nq; q++)
    for (int d = 0; d < 26; d++)
      (*ctab)[((size_t)(q / H16_M) * 26 + d) * H16_M + q % H16_M] = (coll[(size_t)q * 26 + d] + 7) >> 3;
}

}  // namespace kifmm
