// Batched node GEMM for the surface translations, with the pseudo-inverses
// in factored form (UC2UE = up_V * up_W, DC2DE = dn_V * dn_W):
//   upward   y = up_W * check on the leaves, y_parent = [up_W UE2UC_o up_V]_o *
//            y_children, equivalent density = 2^(-l deg) up_V * y
//            (MatMgnt3d::UC2UE_dgemv / UE2UC_dgemv, fmm3d/matmgnt3d.cpp:91-156)
//   downward z = dn_W * check, z_children += [dn_W DE2DC_o dn_V]_o * z_parent,
//            equivalent density = 2^(-l deg) dn_V * z
//            (MatMgnt3d::DC2DE_dgemv / DE2DC_dgemv, fmm3d/matmgnt3d.cpp:158-221)
// Each column is one tree node; nodes sharing an operator become one GEMM
// (the reference does one DGEMV per node).  Columns are gathered from and
// scattered to node-indexed storage through index lists; the level scaling
// is applied per column in the epilogue.  A launch with few columns (the
// shallow levels) splits K over several CTAs into an FP64 workspace and a
// second kernel adds the slices, so a K = 8r sweep does not run serially on a
// handful of SMs.
//
// The pseudo-inverses' entries reach 10^(np+1) times the data (cut-off
// 0.1^(np+1), fmm3d/matmgnt3d.cpp:38-41), so a fused FP32 product would lose
// everything to cancellation.  Each factor is well conditioned (V has
// orthonormal columns; W = Sigma^-1 U^T scales each row by its own 1/sigma,
// and rounding errors stay in that row's direction, whose far field is
// damped by the same sigma), so the products run in the data type.
#include <algorithm>

#include "launch.hpp"

namespace kifmm {
namespace {

constexpr int BM = 64, BN = 64, BK = 8, NTH = 256;

__device__ __forceinline__ double pow2i(int e) { return ldexp(1.0, e); }

__device__ __forceinline__ double row_scale(const GemmScale& sc, int j, int r) {
  if (!sc.col_lvl) return 1.0;
  return pow2i(-(sc.col_lvl[j] + sc.lvl_base) * sc.deg[r % sc.sd]);
}

// partial != nullptr: write the unscaled K-slice sums to partial[z][j][r].
template <typename T>
__global__ void __launch_bounds__(NTH) k_node_gemm(int M, int K, int kchunk, const T* __restrict__ A,
                                                   const T* __restrict__ B, int64_t ldb, const int* __restrict__ bidx,
                                                   T* __restrict__ C, int64_t ldc, const int* __restrict__ cidx,
                                                   int ncol, int accumulate, GemmScale sc,
                                                   double* __restrict__ partial) {
  __shared__ T As[BK][BM + 1];
  __shared__ T Bs[BK][BN + 1];
  __shared__ int64_t bcol[BN], ccol[BN];
  const int tid = threadIdx.x;
  const int m0 = blockIdx.y * BM;
  const int n0 = blockIdx.x * BN;
  const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  if (tid < BN) {
    int j = n0 + tid;
    bcol[tid] = (j < ncol) ? (int64_t)bidx[j] * ldb : -1;
    ccol[tid] = (j < ncol) ? (int64_t)cidx[j] * ldc : -1;
  }
  const int tx = tid % 16, ty = tid / 16;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = T(0);
  __syncthreads();
  for (int k0 = kb; k0 < ke; k0 += BK) {
    for (int e = tid; e < BM * BK; e += NTH) {
      int r = e / BK, c = e % BK;
      int gr = m0 + r, gc = k0 + c;
      As[c][r] = (gr < M && gc < ke) ? A[(size_t)gr * K + gc] : T(0);
    }
    for (int e = tid; e < BN * BK; e += NTH) {
      int j = e / BK, c = e % BK;
      int gc = k0 + c;
      T v = T(0);
      if (bcol[j] >= 0 && gc < ke) v = B[bcol[j] + gc];
      Bs[c][j] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      T a[4], b[4];
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
#pragma unroll
    for (int j = 0; j < 4; j++) {
      int jj = tx + 16 * j;
      int col = n0 + jj;
      if (ccol[jj] < 0) continue;
      if (partial) {
        partial[((size_t)blockIdx.z * ncol + col) * M + r] = (double)acc[i][j];
        continue;
      }
      T* p = C + ccol[jj] + r;
      double v = (double)acc[i][j] * row_scale(sc, col, r);
      if (accumulate) v += (double)*p;
      *p = (T)v;
    }
  }
}

template <typename T>
__global__ void k_node_gemm_reduce(int M, int ncol, int nslice, const double* __restrict__ partial,
                                   T* __restrict__ C, int64_t ldc, const int* __restrict__ cidx, int accumulate,
                                   GemmScale sc) {
  const size_t n = (size_t)ncol * M;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    int col = (int)(e / M), r = (int)(e % M);
    double s = 0.0;
    for (int z = 0; z < nslice; z++) s += partial[(size_t)z * n + e];
    T* p = C + (int64_t)cidx[col] * ldc + r;
    double v = s * row_scale(sc, col, r);
    if (accumulate) v += (double)*p;
    *p = (T)v;
  }
}

}  // namespace

template <typename T>
int launch_node_gemm(int M, int K, const T* A, const T* B, int64_t ldb, const int* bidx, T* C, int64_t ldc,
                      const int* cidx, int ncol, bool accumulate, const GemmScale& sc, double* ws, size_t ws_len,
                      int num_sms, cudaStream_t st) {
  if (ncol <= 0 || M <= 0 || K <= 0) return 0;
  const int tiles = ((ncol + BN - 1) / BN) * ((M + BM - 1) / BM);
  int ks = 1;
  if (ws && K >= 32 * BK && tiles < 2 * num_sms) {
    ks = std::min(std::max(1, (2 * num_sms) / tiles), K / (16 * BK));
    ks = std::min(ks, 16);
    while (ks > 1 && (size_t)ks * ncol * M > ws_len) ks--;
  }
  int kchunk = ((K + ks - 1) / ks + BK - 1) / BK * BK;
  ks = (K + kchunk - 1) / kchunk;
  dim3 grid((ncol + BN - 1) / BN, (M + BM - 1) / BM, ks);
  k_node_gemm<T><<<grid, NTH, 0, st>>>(M, K, kchunk, A, B, ldb, bidx, C, ldc, cidx, ncol, accumulate ? 1 : 0, sc,
                                       ks > 1 ? ws : nullptr);
  if (ks > 1) {
    size_t n = (size_t)ncol * M;
    int g = (int)std::min<size_t>((n + 255) / 256, (size_t)num_sms * 8);
    k_node_gemm_reduce<T><<<g, 256, 0, st>>>(M, ncol, ks, ws, C, ldc, cidx, accumulate ? 1 : 0, sc);
  }
  return ks > 1 ? 2 : 1;
}

void launch_node_gemm_reduce_f(int M, int ncol, int nslice, const double* partial, float* C, int64_t ldc,
                               const int* cidx, bool accumulate, const GemmScale& sc, int num_sms, cudaStream_t st) {
  const size_t n = (size_t)ncol * M;
  if (!n) return;
  int g = (int)std::min<size_t>((n + 255) / 256, (size_t)num_sms * 8);
  k_node_gemm_reduce<float><<<g, 256, 0, st>>>(M, ncol, nslice, partial, C, ldc, cidx, accumulate ? 1 : 0, sc);
}

template int launch_node_gemm<double>(int, int, const double*, const double*, int64_t, const int*, double*,
                                               int64_t, const int*, int, bool, const GemmScale&, double*, size_t, int,
                                               cudaStream_t);
template int launch_node_gemm<float>(int, int, const float*, const float*, int64_t, const int*, float*, int64_t,
                                            const int*, int, bool, const GemmScale&, double*, size_t, int,
                                            cudaStream_t);

}  // namespace kifmm
