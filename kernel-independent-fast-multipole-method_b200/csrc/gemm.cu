// Batched node GEMM for the surface translations:
//   upward   UC2UE on leaves, and fused M2M = UC2UE*[UE2UC_o] on the 8-child block
//            (MatMgnt3d::UC2UE_dgemv / UE2UC_dgemv, fmm3d/matmgnt3d.cpp:91-156)
//   downward DC2DE, and fused L2L = [DC2DE*DE2DC_o] into the 8-child block
//            (MatMgnt3d::DC2DE_dgemv / DE2DC_dgemv, fmm3d/matmgnt3d.cpp:158-221)
// Each column is one tree node; all nodes of one level share the operator,
// so the reference's per-node DGEMVs become one GEMM per level.  The
// homogeneous level scalings 2^(-l*deg) / 2^(+l*deg) are applied in the
// epilogue / while staging B.  Columns are gathered from and scattered to
// node-indexed storage through index lists.
//
// Every operator here contains a pseudo-inverse whose entries reach
// 10^(np+1) times the data (cut-off 0.1^(np+1), fmm3d/matmgnt3d.cpp:38-41);
// the dot products cancel accordingly.  The operators therefore stay FP64
// and the products accumulate in FP64 for both data types: an FP32 node
// vector is widened on load and rounded once on store.
#include "launch.hpp"

namespace kifmm {
namespace {

constexpr int BM = 64, BN = 64, BK = 8, NTH = 256;

__device__ __forceinline__ double pow2i(int e) { return ldexp(1.0, e); }

template <typename T>
__global__ void __launch_bounds__(NTH) k_node_gemm(int M, int K, const double* __restrict__ A,
                                                   const T* __restrict__ B, int64_t ldb, const int* __restrict__ bidx,
                                                   T* __restrict__ C, int64_t ldc, const int* __restrict__ cidx,
                                                   int ncol, int accumulate, GemmScale sc) {
  __shared__ double As[BK][BM + 1];
  __shared__ double Bs[BK][BN + 1];
  __shared__ int64_t bcol[BN], ccol[BN];
  const int tid = threadIdx.x;
  const int m0 = blockIdx.y * BM;
  const int n0 = blockIdx.x * BN;
  if (tid < BN) {
    int j = n0 + tid;
    bcol[tid] = (j < ncol) ? (int64_t)bidx[j] * ldb : -1;
    ccol[tid] = (j < ncol) ? (int64_t)cidx[j] * ldc : -1;
  }
  const int tx = tid % 16, ty = tid / 16;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
  __syncthreads();
  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int e = tid; e < BM * BK; e += NTH) {
      int r = e / BK, c = e % BK;
      int gr = m0 + r, gc = k0 + c;
      As[c][r] = (gr < M && gc < K) ? A[(size_t)gr * K + gc] : 0.0;
    }
    for (int e = tid; e < BN * BK; e += NTH) {
      int j = e / BK, c = e % BK;
      int gc = k0 + c;
      double v = 0.0;
      if (bcol[j] >= 0 && gc < K) {
        v = (double)B[bcol[j] + gc];
        if (sc.in_on) v *= pow2i(sc.in_lvl * sc.deg[gc % sc.sd]);
      }
      Bs[c][j] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    int r = m0 + ty + 16 * i;
    if (r >= M) continue;
    double rs = sc.out_on ? pow2i(-sc.out_lvl * sc.deg[r % sc.sd]) : 1.0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      int jj = tx + 16 * j;
      if (ccol[jj] < 0) continue;
      T* p = C + ccol[jj] + r;
      double v = acc[i][j] * rs;
      if (accumulate) v += (double)*p;
      *p = (T)v;
    }
  }
}

}  // namespace

template <typename T>
void launch_node_gemm(int M, int K, const double* A, const T* B, int64_t ldb, const int* bidx, T* C, int64_t ldc,
                      const int* cidx, int ncol, bool accumulate, const GemmScale& sc, cudaStream_t st) {
  if (ncol <= 0 || M <= 0 || K <= 0) return;
  dim3 grid((ncol + BN - 1) / BN, (M + BM - 1) / BM);
  k_node_gemm<T><<<grid, NTH, 0, st>>>(M, K, A, B, ldb, bidx, C, ldc, cidx, ncol, accumulate ? 1 : 0, sc);
}

template void launch_node_gemm<double>(int, int, const double*, const double*, int64_t, const int*, double*, int64_t,
                                       const int*, int, bool, const GemmScale&, cudaStream_t);
template void launch_node_gemm<float>(int, int, const double*, const float*, int64_t, const int*, float*, int64_t,
                                      const int*, int, bool, const GemmScale&, cudaStream_t);

}  // namespace kifmm
