// Several systems (handles) stepped together: their Taylor steps are captured
// once into a CUDA graph, each system on its own stream forked from the batch
// stream, and the graph is replayed for every later call with the same time
// steps and step count.  Systems of uneven size run side by side, so small
// systems fill the GPU while a large one runs, and a whole multi-step advance
// of every system costs one graph launch on the host.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "sgpu_internal.cuh"

using sgpu::System;

struct sgpu_batch {
  std::vector<System*> sys;
  cudaStream_t st = nullptr;          // capture / launch stream
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // what the captured graph was built for
  std::vector<double> key_dt;
  std::vector<unsigned long long> key_gen;
  int key_steps = 0;
  std::vector<unsigned long long> launches_per_replay;  // per system
};

namespace {

int bfail(int code, const std::string& msg) {
  sgpu::set_last_error(msg);
  return code;
}

int bcuda(cudaError_t e, const char* what) {
  return bfail(SGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

void drop_graph(sgpu_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// Captures nsteps Taylor steps of every system.  The first step of each system
// gathers its projections from the orbitals, so the graph does not depend on
// what the sphere-value buffer held before a replay.
int capture(sgpu_batch* b, const double* dt, int nsteps) {
  drop_graph(b);
  cudaError_t e;
  for (System* s : b->sys) {
    if ((e = sgpu::prepare_pass(*s)) != cudaSuccess) return bcuda(e, "sgpu_batch_step: prepare");
    if ((e = sgpu::prepare_kb(*s)) != cudaSuccess) return bcuda(e, "sgpu_batch_step: prepare");
    if ((e = sgpu::prepare_resident(*s)) != cudaSuccess) return bcuda(e, "sgpu_batch_step: prepare");
  }
  std::vector<unsigned long long> before(b->sys.size());
  for (size_t i = 0; i < b->sys.size(); ++i) before[i] = b->sys[i]->launches;
  if ((e = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return bcuda(e, "sgpu_batch_step: begin capture");
  cudaError_t err = cudaEventRecord(b->fork, b->st);
  for (size_t i = 0; i < b->sys.size() && err == cudaSuccess; ++i) err = cudaStreamWaitEvent(b->sys[i]->stream, b->fork, 0);
  for (int n = 0; n < nsteps && err == cudaSuccess; ++n)
    for (size_t i = 0; i < b->sys.size() && err == cudaSuccess; ++i)
      err = sgpu::enqueue_taylor_step(*b->sys[i], dt[i], n == 0);
  for (size_t i = 0; i < b->sys.size() && err == cudaSuccess; ++i) {
    err = cudaEventRecord(b->join[i], b->sys[i]->stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(b->st, b->join[i], 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(b->st, &g);
  if (err == cudaSuccess) err = ee;
  if (err != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return bcuda(err, "sgpu_batch_step: capture");
  }
  b->graph = g;
  if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess) {
    drop_graph(b);
    return bcuda(e, "sgpu_batch_step: instantiate");
  }
  b->launches_per_replay.resize(b->sys.size());
  for (size_t i = 0; i < b->sys.size(); ++i) {
    System* s = b->sys[i];
    b->launches_per_replay[i] = s->launches - before[i];
    s->launches = before[i];  // capturing launched nothing
  }
  b->key_dt.assign(dt, dt + b->sys.size());
  b->key_steps = nsteps;
  b->key_gen.resize(b->sys.size());
  for (size_t i = 0; i < b->sys.size(); ++i) b->key_gen[i] = b->sys[i]->gen;
  return 0;
}

}  // namespace

extern "C" {

int sgpu_batch_create(const sgpu_handle* hs, int n, sgpu_batch_handle* out) {
  if (!hs || !out || n < 1 || n > 64) return bfail(SGPU_ERR_ARG, "sgpu_batch_create: need 1..64 handles");
  *out = nullptr;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return bcuda(e, "cudaGetDevice");
  for (int i = 0; i < n; ++i) {
    if (!hs[i]) return bfail(SGPU_ERR_ARG, "sgpu_batch_create: null handle");
    if (hs[i]->dev != dev) return bfail(SGPU_ERR_ARG, "sgpu_batch_create: every handle must live on the current device");
    for (int j = 0; j < i; ++j)
      if (hs[j] == hs[i]) return bfail(SGPU_ERR_ARG, "sgpu_batch_create: a handle appears twice");
  }
  sgpu_batch* b = new sgpu_batch();
  for (int i = 0; i < n; ++i) b->sys.push_back(hs[i]);
  b->join.assign(n, nullptr);
  e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
  for (int i = 0; i < n && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    sgpu_batch_destroy(b);
    return bcuda(e, "sgpu_batch_create");
  }
  *out = b;
  return 0;
}

int sgpu_batch_step(sgpu_batch_handle b, const double* dt, int nsteps) {
  if (!b || !dt || nsteps < 1 || nsteps > 4096) return bfail(SGPU_ERR_ARG, "sgpu_batch_step: bad argument");
  for (System* s : b->sys)
    if (!s->have_state || !s->have_vloc || !s->have_proj)
      return bfail(SGPU_ERR_STATE, "sgpu_batch_step: every system needs state, Vloc and projectors");
  for (System* s : b->sys) {  // a flag_current step's stencil sums still read the orbitals
    cudaError_t e = s->aux_join();
    if (e != cudaSuccess) return bcuda(e, "sgpu_batch_step: join");
  }
  bool stale = !b->exec || b->key_steps != nsteps;
  for (size_t i = 0; i < b->sys.size() && !stale; ++i)
    stale = b->key_dt[i] != dt[i] || b->key_gen[i] != b->sys[i]->gen;
  if (stale) {
    // work already queued on the systems' streams precedes the capture
    for (System* s : b->sys) {
      cudaError_t e = cudaStreamSynchronize(s->stream);
      if (e != cudaSuccess) return bcuda(e, "sgpu_batch_step: synchronize");
    }
    if (int rc = capture(b, dt, nsteps)) return rc;
  }
  cudaError_t e = cudaSuccess;
  // order the replay after each system's queued work, and later work after it
  for (size_t i = 0; i < b->sys.size() && e == cudaSuccess; ++i) {
    e = cudaEventRecord(b->join[i], b->sys[i]->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->st, b->join[i], 0);
  }
  if (e == cudaSuccess) e = cudaGraphLaunch(b->exec, b->st);
  if (e == cudaSuccess) e = cudaEventRecord(b->done, b->st);
  for (size_t i = 0; i < b->sys.size() && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(b->sys[i]->stream, b->done, 0);
  if (e != cudaSuccess) return bcuda(e, "sgpu_batch_step: launch");
  for (size_t i = 0; i < b->sys.size(); ++i) {
    b->sys[i]->launches += b->launches_per_replay[i];
    b->sys[i]->S_valid = b->sys[i]->nsp > 0;
    b->sys[i]->cur_valid = false;
  }
  return 0;
}

void* sgpu_batch_stream(sgpu_batch_handle b) { return b ? (void*)b->st : nullptr; }

int sgpu_batch_destroy(sgpu_batch_handle b) {
  if (!b) return 0;
  if (b->st) cudaStreamSynchronize(b->st);
  drop_graph(b);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->done) cudaEventDestroy(b->done);
  for (cudaEvent_t ev : b->join)
    if (ev) cudaEventDestroy(ev);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return 0;
}

}  // extern "C"
