// Batched evaluation: many independent FMM instances (each its own FMM3d
// handle, any kernel and size) and several density vectors per instance in
// one CUDA graph.  The reference evaluates one instance at a time on one CPU
// thread (fmm3d/tt.cpp:97-101); here every instance's passes are enqueued on
// its own stream between a fork and a join event, the whole fan-out is
// captured once per (nrhs, buffer set), and later calls replay the graph, so
// small instances overlap on the GPU and the per-kernel launch cost is paid
// once per capture instead of on every call.
#include <cstring>
#include <vector>

#include "../../include/kifmm.h"
#include "engine.hpp"

struct kifmm_batch_s {
  std::vector<kifmm_handle> hs;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> done;
  cudaEvent_t fork = nullptr;
  cudaStream_t cap = nullptr;
  cudaGraphExec_t exec = nullptr;
  int key_nrhs = 0;
  std::vector<const void*> key_ptrs;
  std::string err;
  int replays = 0;
};

namespace {

void release_graph(kifmm_batch b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
}

}  // namespace

extern "C" {

kifmm_status kifmm_batch_create(int n, const kifmm_handle* hs, kifmm_batch* out) {
  if (n < 1 || !hs || !out) return KIFMM_ERR_ARG;
  for (int i = 0; i < n; i++)
    if (!hs[i] || !hs[i]->e.ready) return KIFMM_ERR_STATE;
  kifmm_batch b = new (std::nothrow) kifmm_batch_s;
  if (!b) return KIFMM_ERR_ALLOC;
  b->hs.assign(hs, hs + n);
  b->streams.resize(n, nullptr);
  b->done.resize(n, nullptr);
  bool ok = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; ok && i < n; i++)
    ok = cudaStreamCreateWithFlags(&b->streams[i], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&b->done[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    kifmm_batch_destroy(b);
    return KIFMM_ERR_CUDA;
  }
  *out = b;
  return KIFMM_OK;
}

kifmm_status kifmm_batch_destroy(kifmm_batch b) {
  if (!b) return KIFMM_ERR_ARG;
  release_graph(b);
  for (auto s : b->streams)
    if (s) cudaStreamDestroy(s);
  for (auto e : b->done)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
  return KIFMM_OK;
}

kifmm_status kifmm_batch_eval_device(kifmm_batch b, int nrhs, const double* const* d_srcden,
                                     double* const* d_trgval, void* stream, int sync) {
  if (!b || nrhs < 1 || !d_srcden || !d_trgval) return KIFMM_ERR_ARG;
  const int n = (int)b->hs.size();
  std::vector<const void*> key;
  for (int i = 0; i < n; i++) {
    key.push_back(d_srcden[i]);
    key.push_back(d_trgval[i]);
  }
  if (!b->exec || b->key_nrhs != nrhs || b->key_ptrs != key) {
    release_graph(b);
    for (int i = 0; i < n; i++) {
      int rc = b->hs[i]->e.reserve(nrhs);
      if (rc != KIFMM_OK) {
        b->err = "instance " + std::to_string(i) + ": " + b->hs[i]->e.err;
        return (kifmm_status)rc;
      }
    }
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      b->err = "stream capture could not begin";
      return KIFMM_ERR_CUDA;
    }
    int rc = KIFMM_OK;
    cudaEventRecord(b->fork, b->cap);
    for (int i = 0; i < n && rc == KIFMM_OK; i++) {
      cudaStreamWaitEvent(b->streams[i], b->fork, 0);
      rc = b->hs[i]->e.enqueue(d_srcden[i], d_trgval[i], nrhs, b->streams[i]);
      if (rc != KIFMM_OK) b->err = "instance " + std::to_string(i) + ": " + b->hs[i]->e.err;
      cudaEventRecord(b->done[i], b->streams[i]);
      cudaStreamWaitEvent(b->cap, b->done[i], 0);
    }
    cudaError_t ce = cudaStreamEndCapture(b->cap, &graph);
    if (rc == KIFMM_OK && ce != cudaSuccess) {
      b->err = std::string("capture failed: ") + cudaGetErrorString(ce);
      rc = KIFMM_ERR_CUDA;
    }
    if (rc == KIFMM_OK && cudaGraphInstantiate(&b->exec, graph, 0) != cudaSuccess) {
      b->err = "graph instantiation failed";
      rc = KIFMM_ERR_CUDA;
      b->exec = nullptr;
    }
    if (graph) cudaGraphDestroy(graph);
    if (rc != KIFMM_OK) {
      cudaGetLastError();
      release_graph(b);
      return (kifmm_status)rc;
    }
    b->key_nrhs = nrhs;
    b->key_ptrs = key;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaGraphLaunch(b->exec, st) != cudaSuccess) {
    cudaGetLastError();
    b->err = "graph launch failed";
    return KIFMM_ERR_CUDA;
  }
  b->replays++;
  if (sync && cudaStreamSynchronize(st) != cudaSuccess) {
    b->err = cudaGetErrorString(cudaGetLastError());
    return KIFMM_ERR_CUDA;
  }
  if (sync) return kifmm_batch_poll_status(b);
  return KIFMM_OK;
}

kifmm_status kifmm_batch_poll_status(kifmm_batch b) {
  if (!b) return KIFMM_ERR_ARG;
  kifmm_status rc = KIFMM_OK;
  for (size_t i = 0; i < b->hs.size(); i++)
    if (b->hs[i]->e.poll_status() != KIFMM_OK) {
      b->err = "instance " + std::to_string(i) + ": " + b->hs[i]->e.err;
      rc = KIFMM_ERR_CUDA;
    }
  return rc;
}

const char* kifmm_batch_last_error(kifmm_batch b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"
