// kifmm_direct_noalloc: the FP64 direct sum (the engine's Dense3d path)
// for callers that must not allocate device memory.
//
// Who needs it: a process whose device memory is owned by someone else --
// a serving runtime or framework that reserved the GPU's memory up front
// through its own caching allocator, or a plug-in host that forbids device
// allocations after start-up -- cannot call cudaMalloc between its own
// steps: the call fails once the budget is taken, bypasses the owner's
// accounting, and synchronises the device in the middle of a stream of
// work.  Such a caller allocates its inputs and outputs itself and needs
// an entry point that allocates nothing else.
//
// How: the sources are split into chunks evaluated by different CTAs (so a
// small target set still fills the GPU); each chunk's partial potentials go
// to a fixed scratch array in device global memory, declared below at file
// scope, and a second kernel adds the chunks up into the caller's output.
// The scratch holds KIFMM_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB) on every
// GPU that loads this library, for the life of the process.  A call needs
// nchunk * nt * tdof of them; nt * tdof above the capacity is rejected with
// KIFMM_ERR_CAPACITY before any launch.  Every slot a call reads was written
// earlier in the same call, so nothing needs clearing between calls; the
// array keeps the last call's partial sums.  All calls share the one array:
// two calls whose kernels overlap on the GPU (different streams, or
// different host threads) race on it and must be serialised by the caller.
//
// The array's device address is looked up with cudaGetSymbolAddress on
// every call, with the caller's device current (host code cannot use the
// symbol itself: on the host it names a stand-in, not device memory); the
// lookup allocates nothing and stays right after a cudaDeviceReset, which
// reloads the module and may move the array.  The first call on a device
// loads the module there and should come before any stream capture.
#include <algorithm>

#include "../../include/kifmm.h"
#include "kernels_common.cuh"

namespace kifmm {
namespace {

static __device__ __align__(256) double g_noalloc_scratch[KIFMM_NOALLOC_SCRATCH_DOUBLES];

constexpr int NA_THREADS = 128;
constexpr int NA_TILE = 128;
constexpr int NA_MAXCHUNK = 64;

// partial[c][t][d] = sum over sources of chunk c of K(trg_t - src) den
template <int KT>
__global__ void __launch_bounds__(NA_THREADS) k_direct_partial(const double* __restrict__ spos,
                                                               const double* __restrict__ snor,
                                                               const double* __restrict__ sden, int ns, int chunk,
                                                               const double* __restrict__ tpos, int nt,
                                                               double* __restrict__ partial, KConst<double> kc) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  __shared__ double sx[NA_TILE], sy[NA_TILE], sz[NA_TILE], nx[NA_TILE], ny[NA_TILE], nz[NA_TILE], f[NA_TILE * 4];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int s0 = blockIdx.y * chunk;
  const int s1 = min(ns, s0 + chunk);
  double px = 0, py = 0, pz = 0;
  if (t < nt) {
    px = tpos[3 * (size_t)t];
    py = tpos[3 * (size_t)t + 1];
    pz = tpos[3 * (size_t)t + 2];
  }
  double acc[4] = {0, 0, 0, 0};
  for (int c0 = s0; c0 < s1; c0 += NA_TILE) {
    const int cnt = min(NA_TILE, s1 - c0);
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      const size_t p = (size_t)(c0 + j);
      sx[j] = spos[3 * p];
      sy[j] = spos[3 * p + 1];
      sz[j] = spos[3 * p + 2];
      nx[j] = snor[3 * p];
      ny[j] = snor[3 * p + 1];
      nz[j] = snor[3 * p + 2];
      for (int s = 0; s < SD; s++) f[j * SD + s] = sden[p * SD + s];
    }
    __syncthreads();
    if (t < nt)
      for (int j = 0; j < cnt; j++) {
        double nrm[3] = {nx[j], ny[j], nz[j]};
        keval<KT, double>(px - sx[j], py - sy[j], pz - sz[j], nrm, &f[j * SD], acc, kc);
      }
  }
  if (t < nt)
    for (int d = 0; d < TD; d++) partial[((size_t)blockIdx.y * nt + t) * TD + d] = acc[d];
}

__global__ void k_direct_reduce(const double* __restrict__ partial, int nchunk, int n, double* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < nchunk; c++) s += partial[(size_t)c * n + e];
    out[e] = s;
  }
}

template <int KT>
void launch_partial(dim3 grid, cudaStream_t st, const double* spos, const double* snor, const double* sden, int ns,
                    int chunk, const double* tpos, int nt, double* partial, const KConst<double>& kc) {
  k_direct_partial<KT><<<grid, NA_THREADS, 0, st>>>(spos, snor, sden, ns, chunk, tpos, nt, partial, kc);
}

}  // namespace
}  // namespace kifmm

extern "C" kifmm_status kifmm_direct_noalloc(int kt, int ncoef, const double* coefs, int ns, const double* d_srcpos,
                                             const double* d_srcnor, const double* d_srcden, int nt,
                                             const double* d_trgpos, double* d_trgval, void* stream) {
  using namespace kifmm;
  int td = 0;
  switch (kt) {
    case 111: case 121: case 312: case 322: td = 1; break;
    case 311: case 321: case 511: case 521: td = 3; break;
    default: return KIFMM_ERR_KERNEL;
  }
  int need = (kt == 511 || kt == 521) ? 2 : (kt == 111 || kt == 121) ? 0 : 1;
  if (ncoef < need || (ncoef > 0 && !coefs)) return KIFMM_ERR_KERNEL;
  if (ns < 0 || nt < 0) return KIFMM_ERR_ARG;
  if (nt == 0) return KIFMM_OK;
  if (!d_trgpos || !d_trgval || (ns > 0 && (!d_srcpos || !d_srcnor || !d_srcden))) return KIFMM_ERR_ARG;
  const size_t per_chunk = (size_t)nt * td;
  if (per_chunk > (size_t)KIFMM_NOALLOC_SCRATCH_DOUBLES) return KIFMM_ERR_CAPACITY;
  // an error left by the caller's earlier work is reported as such (and
  // left pending), not taken for a failure of this call's launches
  if (cudaPeekAtLastError() != cudaSuccess) return KIFMM_ERR_CUDA;
  int dev = 0, num_sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return KIFMM_ERR_NO_DEVICE;
  }
  // the scratch array's address on the current device (every call)
  double* scratch = nullptr;
  {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return KIFMM_ERR_CUDA;
    }
    scratch = (double*)p;
  }
  cudaStream_t st = (cudaStream_t)stream;
  double kcd[3], cf[2] = {1.0, 0.25};
  for (int i = 0; i < ncoef && i < 2; i++) cf[i] = coefs[i];
  kernel_constants(kt, cf, kcd);
  KConst<double> kc{kcd[0], kcd[1], kcd[2]};
  // chunks of sources: enough CTAs to fill the GPU, within the scratch capacity
  const int tblocks = (nt + NA_THREADS - 1) / NA_THREADS;
  int nchunk = (int)std::min<size_t>((size_t)NA_MAXCHUNK, (size_t)KIFMM_NOALLOC_SCRATCH_DOUBLES / per_chunk);
  nchunk = std::max(1, std::min(nchunk, std::max(1, 4 * num_sms / tblocks)));
  nchunk = std::max(1, std::min(nchunk, std::max(1, ns / NA_TILE)));
  const int chunk = ns > 0 ? (ns + nchunk - 1) / nchunk : 0;
  dim3 grid(tblocks, nchunk);
  switch (kt) {
    case 111: launch_partial<111>(grid, st, d_srcpos, d_srcnor, d_srcden, ns, chunk, d_trgpos, nt, scratch, kc); break;
    case 121: launch_partial<121>(grid, st, d_srcpos, d_srcnor, d_srcden, ns, chunk, d_trgpos, nt, scratch, kc); break;
    case 311: launch_partial<311>(grid, st, d_srcpos, d_srcnor, d_srcden, ns, chunk, d_trgpos, nt, scratch, kc); break;
    case 312: launch_partial<312>(grid, st, d_srcpos, d_srcnor, d_srcden, ns, chunk, d_trgpos, nt, scratch, kc); break;
    case 321: launch_partial<321>(grid, st, d_srcpos, d_srcnor, d_srcden, ns, chunk, d_trgpos, nt, scratch, kc); break;
    case 322: launch_partial<322>(grid, st, d_srcpos, d_srcnor, d_srcden, ns, chunk, d_trgpos, nt, scratch, kc); break;
    case 511: launch_partial<511>(grid, st, d_srcpos, d_srcnor, d_srcden, ns, chunk, d_trgpos, nt, scratch, kc); break;
    case 521: launch_partial<521>(grid, st, d_srcpos, d_srcnor, d_srcden, ns, chunk, d_trgpos, nt, scratch, kc); break;
  }
  const int n = (int)per_chunk;
  k_direct_reduce<<<std::max(1, std::min((n + 255) / 256, num_sms * 8)), 256, 0, st>>>(scratch, nchunk, n, d_trgval);
  if (cudaGetLastError() != cudaSuccess) return KIFMM_ERR_CUDA;
  return KIFMM_OK;
}
