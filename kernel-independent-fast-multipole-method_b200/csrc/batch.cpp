// Batched evaluation: many independent FMM instances (each its own FMM3d
// handle, any kernel and size) and several density vectors per instance in
// one CUDA graph.  The reference evaluates one instance at a time on one CPU
// thread (fmm3d/tt.cpp:97-101).
//
// Instances that share kernel, np, precision, V-list form and root level
// (Engine::forest_key) are concatenated into one forest engine: their trees
// side by side, their points one after another, so every pass of the eval is
// ONE launch over the work queues of all of them (leaf lists, V-list parent
// pairs, surface-contraction columns) instead of one launch per instance.
// The instances' density vectors are copied into the forest's buffers and
// its potentials back out (one 2-D device copy per instance and direction).
// Every unit -- a forest, or an instance that shares its key with no other
// -- is enqueued on its own stream between a fork and a join event, the
// whole fan-out is captured once per (nrhs, buffer set), and later calls
// replay the graph.
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/kifmm.h"
#include "engine.hpp"

namespace {

struct Unit {
  std::vector<int> members;                // instance indices (one for a single instance)
  std::unique_ptr<kifmm::Engine> forest;   // the concatenated engine, or null
  double* d_in = nullptr;                  // forest density vectors [rhs][point][sdof]
  double* d_out = nullptr;                 // forest potentials [rhs][point][tdof]
  size_t cap_in = 0, cap_out = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
};

}  // namespace

struct kifmm_batch_s {
  std::vector<kifmm_handle> hs;
  std::vector<Unit> units;
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

void release_unit(Unit& u) {
  if (u.d_in) cudaFree(u.d_in);
  if (u.d_out) cudaFree(u.d_out);
  u.d_in = u.d_out = nullptr;
  u.cap_in = u.cap_out = 0;
  if (u.stream) cudaStreamDestroy(u.stream);
  if (u.done) cudaEventDestroy(u.done);
  u.stream = nullptr;
  u.done = nullptr;
  u.forest.reset();
}

std::string members_str(const Unit& u) {
  if (u.members.size() == 1) return "instance " + std::to_string(u.members[0]);
  std::string s = "instances";
  for (int i : u.members) s += " " + std::to_string(i);
  return s;
}

}  // namespace

extern "C" {

kifmm_status kifmm_batch_create_opts(int n, const kifmm_handle* hs, int concatenate, kifmm_batch* out) {
  if (n < 1 || !hs || !out) return KIFMM_ERR_ARG;
  for (int i = 0; i < n; i++)
    if (!hs[i] || !hs[i]->e.ready) return KIFMM_ERR_STATE;
  kifmm_batch b = new (std::nothrow) kifmm_batch_s;
  if (!b) return KIFMM_ERR_ALLOC;
  b->hs.assign(hs, hs + n);
  // units: instances grouped by forest key (in order of first appearance)
  std::vector<std::vector<int>> groups;
  std::map<std::string, int> by_key;
  for (int i = 0; i < n; i++) {
    const std::string k = concatenate ? hs[i]->e.forest_key() : std::string();
    if (k.empty()) {
      groups.push_back({i});
      continue;
    }
    auto it = by_key.find(k);
    if (it == by_key.end()) {
      by_key[k] = (int)groups.size();
      groups.push_back({i});
    } else {
      groups[it->second].push_back(i);
    }
  }
  b->units.resize(groups.size());
  kifmm_status rc = KIFMM_OK;
  for (size_t u = 0; u < groups.size() && rc == KIFMM_OK; u++) {
    Unit& U = b->units[u];
    U.members = groups[u];
    if (U.members.size() > 1) {
      std::vector<const kifmm::Engine*> ms;
      for (int i : U.members) ms.push_back(&hs[i]->e);
      U.forest = std::make_unique<kifmm::Engine>();
      const int r = U.forest->setup_forest(ms);
      if (r != KIFMM_OK) {
        b->err = members_str(U) + " concatenated: " + U.forest->err;
        rc = (kifmm_status)r;
      }
    }
  }
  bool ok = rc == KIFMM_OK && cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess;
  for (size_t u = 0; ok && u < b->units.size(); u++)
    ok = cudaStreamCreateWithFlags(&b->units[u].stream, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&b->units[u].done, cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    kifmm_batch_destroy(b);
    return rc != KIFMM_OK ? rc : KIFMM_ERR_CUDA;
  }
  *out = b;
  return KIFMM_OK;
}

kifmm_status kifmm_batch_create(int n, const kifmm_handle* hs, kifmm_batch* out) {
  return kifmm_batch_create_opts(n, hs, 1, out);
}

kifmm_status kifmm_batch_destroy(kifmm_batch b) {
  if (!b) return KIFMM_ERR_ARG;
  release_graph(b);
  for (auto& u : b->units) release_unit(u);
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
    // every allocation before the capture begins
    for (auto& u : b->units) {
      if (!u.forest) {
        const int i = u.members[0];
        int rc = b->hs[i]->e.reserve(nrhs);
        if (rc != KIFMM_OK) {
          b->err = "instance " + std::to_string(i) + ": " + b->hs[i]->e.err;
          return (kifmm_status)rc;
        }
        continue;
      }
      kifmm::Engine& F = *u.forest;
      int rc = F.reserve(nrhs);
      if (rc != KIFMM_OK) {
        b->err = members_str(u) + ": " + F.err;
        return (kifmm_status)rc;
      }
      const size_t nin = (size_t)nrhs * F.ns * F.user.sd, nout = (size_t)nrhs * F.nt * F.user.td;
      if (nin > u.cap_in) {
        if (u.d_in) cudaFree(u.d_in);
        u.d_in = nullptr;
        u.cap_in = 0;
        if (cudaMalloc(&u.d_in, std::max<size_t>(nin, 1) * sizeof(double)) != cudaSuccess) {
          cudaGetLastError();
          b->err = members_str(u) + ": forest buffers";
          return KIFMM_ERR_ALLOC;
        }
        u.cap_in = nin;
      }
      if (nout > u.cap_out) {
        if (u.d_out) cudaFree(u.d_out);
        u.d_out = nullptr;
        u.cap_out = 0;
        if (cudaMalloc(&u.d_out, std::max<size_t>(nout, 1) * sizeof(double)) != cudaSuccess) {
          cudaGetLastError();
          b->err = members_str(u) + ": forest buffers";
          return KIFMM_ERR_ALLOC;
        }
        u.cap_out = nout;
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
    for (size_t ui = 0; ui < b->units.size() && rc == KIFMM_OK; ui++) {
      Unit& u = b->units[ui];
      cudaStreamWaitEvent(u.stream, b->fork, 0);
      if (!u.forest) {
        const int i = u.members[0];
        rc = b->hs[i]->e.enqueue(d_srcden[i], d_trgval[i], nrhs, u.stream);
        if (rc != KIFMM_OK) b->err = "instance " + std::to_string(i) + ": " + b->hs[i]->e.err;
      } else {
        kifmm::Engine& F = *u.forest;
        const int sd = F.user.sd, td = F.user.td;
        for (size_t k = 0; k < u.members.size() && rc == KIFMM_OK; k++) {
          const int i = u.members[k];
          const size_t w = (size_t)b->hs[i]->e.ns * sd * sizeof(double);
          if (w && cudaMemcpy2DAsync(u.d_in + (size_t)F.src_off[k] * sd, (size_t)F.ns * sd * sizeof(double),
                                     d_srcden[i], w, w, nrhs, cudaMemcpyDeviceToDevice, u.stream) != cudaSuccess) {
            b->err = "instance " + std::to_string(i) + ": copy into the forest buffers";
            rc = KIFMM_ERR_CUDA;
          }
        }
        if (rc == KIFMM_OK) {
          rc = F.enqueue(u.d_in, u.d_out, nrhs, u.stream);
          if (rc != KIFMM_OK) b->err = members_str(u) + ": " + F.err;
        }
        for (size_t k = 0; k < u.members.size() && rc == KIFMM_OK; k++) {
          const int i = u.members[k];
          const size_t w = (size_t)b->hs[i]->e.nt * td * sizeof(double);
          if (w && cudaMemcpy2DAsync(d_trgval[i], w, u.d_out + (size_t)F.trg_off[k] * td,
                                     (size_t)F.nt * td * sizeof(double), w, nrhs, cudaMemcpyDeviceToDevice,
                                     u.stream) != cudaSuccess) {
            b->err = "instance " + std::to_string(i) + ": copy out of the forest buffers";
            rc = KIFMM_ERR_CUDA;
          }
        }
      }
      cudaEventRecord(u.done, u.stream);
      cudaStreamWaitEvent(b->cap, u.done, 0);
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
  for (auto& u : b->units) {
    kifmm::Engine& e = u.forest ? *u.forest : b->hs[u.members[0]]->e;
    if (e.poll_status() != KIFMM_OK) {
      b->err = members_str(u) + ": " + e.err;
      rc = KIFMM_ERR_CUDA;
    }
  }
  return rc;
}

kifmm_status kifmm_batch_info(kifmm_batch b, int* nunits, int* nforests, int* launches) {
  if (!b || !nunits || !nforests || !launches) return KIFMM_ERR_ARG;
  *nunits = (int)b->units.size();
  *nforests = 0;
  *launches = 0;
  for (auto& u : b->units) {
    if (u.forest) ++*nforests;
    const kifmm::Engine& e = u.forest ? *u.forest : b->hs[u.members[0]]->e;
    if (b->exec && e.impl) *launches += e.impl->launches();
  }
  return KIFMM_OK;
}

const char* kifmm_batch_last_error(kifmm_batch b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"
