// chns_ensemble.cu -- many independent runs advanced by one CUDA graph per step.
//
// Ensembles whose members are all ternary FP32 runs at 256^2..1024^2 (the
// batched-run configuration) can also step as ONE persistent kernel
// (chns_persist.cu, chns_ensemble_persistent), captured in the step graph; the
// graph of per-member branches described below is the default.
//
// Each member is an ordinary context.  The ensemble step graph is captured once:
// a fork event on the ensemble stream, then on every member's stream the two
// ETD2RK stages of that member, then a join.  Replaying it runs the members'
// kernels as parallel graph branches, so members whose grids are too small to
// fill 148 SMs alone (256^2 - 1024^2) share the GPU.  The kernels and their
// arguments are those of chns_step, so every member's state evolves exactly as
// it would alone.
#include <cuda_runtime.h>
#include <stdlib.h>

#include <new>
#include <vector>

#include "chns_internal.h"

struct chns_ensemble {
  std::vector<chns_ctx*> m;
  cudaStream_t stream;
  cudaEvent_t fork;
  std::vector<cudaEvent_t> ev;  // one per member
  cudaGraphExec_t graph;
  bool graph_ok, graph_tried;
  chns_persist* persist;  // the one-kernel step when the members allow it (else null)
  bool use_persist;
};

namespace {

#define EK(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return CHNS_ERR_CUDA;  \
  } while (0)

void release(chns_ensemble* e) {
  if (!e) return;
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->persist) chns_persist_destroy(e->persist);
  for (cudaEvent_t v : e->ev)
    if (v) cudaEventDestroy(v);
  if (e->fork) cudaEventDestroy(e->fork);
  for (chns_ctx* c : e->m)
    if (c) chns_destroy(c);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

// the members' stages on their own streams, forked from and joined to e->stream
int enqueue(chns_ensemble* e) {
  if (e->use_persist) return chns_persist_step(e->persist, e->stream);
  EK(cudaEventRecord(e->fork, e->stream));
  for (size_t i = 0; i < e->m.size(); i++) {
    chns_ctx* c = e->m[i];
    EK(cudaStreamWaitEvent(c->stream, e->fork, 0));
    const int n1 = c->L->stage(c, 1);
    const int n2 = c->L->stage(c, 2);
    c->launches_per_step = n1 + n2;
    EK(cudaEventRecord(e->ev[i], c->stream));
    EK(cudaStreamWaitEvent(e->stream, e->ev[i], 0));
  }
  return CHNS_OK;
}

int build_graph(chns_ensemble* e) {
  cudaGraph_t g = nullptr;
  EK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = enqueue(e);
  const cudaError_t ec = cudaStreamEndCapture(e->stream, &g);
  if (rc != CHNS_OK || ec != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return CHNS_ERR_CUDA;
  }
  const cudaError_t ei = cudaGraphInstantiate(&e->graph, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    e->graph = nullptr;
    cudaGetLastError();
    return CHNS_ERR_CUDA;
  }
  e->graph_ok = true;
  return CHNS_OK;
}

}  // namespace

extern "C" {

int chns_ensemble_create(const chns_params* members, int count, chns_ensemble** out) {
  if (!members || count < 1 || !out) return CHNS_ERR_ARG;
  *out = nullptr;
  chns_ensemble* e = new (std::nothrow) chns_ensemble();
  if (!e) return CHNS_ERR_NOMEM;
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) {
    release(e);
    return CHNS_ERR_CUDA;
  }
  e->m.assign(count, nullptr);
  e->ev.assign(count, nullptr);
  for (int i = 0; i < count; i++) {
    const int rc = chns_create(&members[i], &e->m[i]);
    if (rc != CHNS_OK) {
      release(e);
      return rc;
    }
    // P1's two CTAs per row fill the GPU for a lone small grid; in an ensemble the
    // members' branches fill it, and one CTA per row was 1.7% faster on the
    // 64-member ternary ensemble (unless chns_tune_override chose the split)
    if (chns_tune_value(CHNS_TUNE_P1_SPLIT) < 0) e->m[i]->p1_split = false;
    if (cudaEventCreateWithFlags(&e->ev[i], cudaEventDisableTiming) != cudaSuccess) {
      release(e);
      return CHNS_ERR_CUDA;
    }
  }
  // members that allow it can step as one persistent kernel (chns_ensemble_persistent);
  // the graph stays the default: on the batched-run ensemble it measured faster
  if (chns_persist_create(e->m.data(), count, &e->persist) != CHNS_OK) e->persist = nullptr;
  *out = e;
  return CHNS_OK;
}

int chns_ensemble_destroy(chns_ensemble* e) {
  if (!e) return CHNS_ERR_ARG;
  release(e);
  return CHNS_OK;
}

chns_ctx* chns_ensemble_member(chns_ensemble* e, int i) {
  if (!e || i < 0 || i >= (int)e->m.size()) return nullptr;
  return e->m[i];
}

int chns_ensemble_size(const chns_ensemble* e) { return e ? (int)e->m.size() : 0; }

int chns_ensemble_step(chns_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return CHNS_ERR_ARG;
  if (nsteps == 0) return CHNS_OK;
  // the ensemble stream waits for earlier work on every member stream
  for (size_t i = 0; i < e->m.size(); i++) {
    EK(cudaEventRecord(e->ev[i], e->m[i]->stream));
    EK(cudaStreamWaitEvent(e->stream, e->ev[i], 0));
  }
  if (!e->graph_ok && !e->graph_tried) {
    e->graph_tried = true;
    if (build_graph(e) != CHNS_OK) e->graph_ok = false;
  }
  for (int s = 0; s < nsteps; s++) {
    if (e->graph_ok) {
      EK(cudaGraphLaunch(e->graph, e->stream));
    } else {
      const int rc = enqueue(e);
      if (rc != CHNS_OK) return rc;
    }
  }
  // later work on member streams waits for the ensemble
  EK(cudaEventRecord(e->fork, e->stream));
  for (chns_ctx* c : e->m) EK(cudaStreamWaitEvent(c->stream, e->fork, 0));
  EK(cudaGetLastError());
  return CHNS_OK;
}

int chns_ensemble_synchronize(chns_ensemble* e) {
  if (!e) return CHNS_ERR_ARG;
  EK(cudaStreamSynchronize(e->stream));
  if (e->persist) {
    const int rc = chns_persist_check(e->persist, e->stream);
    if (rc != CHNS_OK) return rc;
  }
  for (chns_ctx* c : e->m) {
    const int rc = chns_synchronize(c);
    if (rc != CHNS_OK) return rc;
  }
  return CHNS_OK;
}

int chns_ensemble_persistent(chns_ensemble* e, int enable) {
  if (!e) return CHNS_ERR_ARG;
  if (enable == 0 || enable == 1) {
    if (enable && !e->persist) return CHNS_ERR_UNSUPPORTED;
    if ((bool)enable != e->use_persist) {
      // the captured step belongs to the other mode: capture again on the next step
      if (e->stream) cudaStreamSynchronize(e->stream);
      if (e->graph) cudaGraphExecDestroy(e->graph);
      e->graph = nullptr;
      e->graph_ok = e->graph_tried = false;
      e->use_persist = enable != 0;
    }
  }
  return e->use_persist ? 1 : 0;
}

}  // extern "C"
