// CUDA graphs of the Hamiltonian application: one H*psi call (fixed buffers
// and band count) captured on a private stream and replayed with a single
// cudaGraphLaunch, for callers that apply H to the same block many times
// (iterative eigensolvers, time stepping, serving loops).  Capture runs one
// warm-up call first so that no allocation, attribute set-up or library
// workspace creation happens inside the capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "common.hpp"

struct pw_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  size_t nodes = 0;
};

using namespace pwb;

extern "C" {

int pw_graph_capture_hpsi(pw_ctx* ctx, const void* psi, int ld, void* hpsi, int ldh, int nband, int accumulate,
                          pw_graph** out) {
  PWB_CHECK(ctx && out && nband > 0 && psi && hpsi, PW_EINVAL, "bad arguments");
  PWB_CHECK(!ctx->prof_on, PW_EINVAL, "per-kernel profiling is on (pw_profile); graphs need it off");
  PWB_CUDA(cudaSetDevice(ctx->device));
  // warm-up outside the capture: scratch, kernel attributes, library handles
  int rc = pw_hpsi(ctx, psi, ld, hpsi, ldh, nband, accumulate, nullptr);
  if (rc) return rc;
  PWB_CUDA(cudaDeviceSynchronize());
  cudaStream_t st;
  PWB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  const bool chk = ctx->check_errors;
  ctx->check_errors = false;   // the error-flag read synchronises; not allowed while capturing
  pw_graph* g = new pw_graph();
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = pw_hpsi(ctx, psi, ld, hpsi, ldh, nband, accumulate, st);
    cudaError_t e2 = cudaStreamEndCapture(st, &g->graph);
    if (!rc && e2 != cudaSuccess) e = e2;
  }
  ctx->check_errors = chk;
  if (e == cudaSuccess && !rc) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e == cudaSuccess && !rc) e = cudaGraphGetNodes(g->graph, nullptr, &g->nodes);
  cudaStreamDestroy(st);
  if (rc || e != cudaSuccess) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    if (!rc) {
      set_error(std::string("graph capture failed: ") + cudaGetErrorString(e));
      rc = PW_ECUDA;
    }
    cudaGetLastError();
    return rc;
  }
  *out = g;
  return PW_OK;
}

// independent contexts (cells) on a pool of forked streams
static int batch_enqueue(int ncell, pw_ctx* const* ctxs, const void* const* psi, const int* ld, void* const* out,
                         const int* ldo, const int* nband, cudaStream_t st) {
  constexpr int kPool = 16;
  static cudaStream_t pool[kPool] = {nullptr};
  static cudaEvent_t done[kPool] = {nullptr};
  static cudaEvent_t fork = nullptr;
  if (!fork) {
    PWB_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    for (int i = 0; i < kPool; ++i) {
      PWB_CUDA(cudaStreamCreateWithFlags(&pool[i], cudaStreamNonBlocking));
      PWB_CUDA(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
    }
  }
  const int nuse = std::min(ncell, kPool);
  PWB_CUDA(cudaEventRecord(fork, st));
  for (int i = 0; i < nuse; ++i) PWB_CUDA(cudaStreamWaitEvent(pool[i], fork, 0));
  for (int c = 0; c < ncell; ++c) {
    int rc = pw_hpsi(ctxs[c], psi[c], ld[c], out[c], ldo[c], nband[c], 0, pool[c % kPool]);
    if (rc) return rc;
  }
  for (int i = 0; i < nuse; ++i) {
    PWB_CUDA(cudaEventRecord(done[i], pool[i]));
    PWB_CUDA(cudaStreamWaitEvent(st, done[i], 0));
  }
  return PW_OK;
}

static int batch_check(int ncell, pw_ctx* const* ctxs, const void* const* psi, const int* ld, void* const* out,
                       const int* ldo, const int* nband) {
  PWB_CHECK(ncell > 0 && ctxs && psi && ld && out && ldo && nband, PW_EINVAL, "null argument");
  for (int c = 0; c < ncell; ++c) {
    PWB_CHECK(ctxs[c] && psi[c] && out[c] && nband[c] > 0, PW_EINVAL, "bad cell entry");
    PWB_CHECK(ctxs[c]->device == ctxs[0]->device, PW_EINVAL, "cells of one batch share a device");
    PWB_CHECK(!ctxs[c]->prof_on, PW_EINVAL, "per-kernel profiling is on (pw_profile)");
    for (int d = 0; d < c; ++d) PWB_CHECK(ctxs[d] != ctxs[c], PW_EINVAL, "a context appears twice in one batch");
  }
  return PW_OK;
}

int pw_hpsi_batch(int ncell, pw_ctx* const* ctxs, const void* const* psi, const int* ld, void* const* out,
                  const int* ldo, const int* nband, void* stream) {
  int rc = batch_check(ncell, ctxs, psi, ld, out, ldo, nband);
  if (rc) return rc;
  PWB_CUDA(cudaSetDevice(ctxs[0]->device));
  return batch_enqueue(ncell, ctxs, psi, ld, out, ldo, nband, (cudaStream_t)stream);
}

int pw_graph_capture_batch(int ncell, pw_ctx* const* ctxs, const void* const* psi, const int* ld, void* const* out,
                           const int* ldo, const int* nband, pw_graph** graph) {
  int rc = batch_check(ncell, ctxs, psi, ld, out, ldo, nband);
  if (rc) return rc;
  PWB_CHECK(graph, PW_EINVAL, "null argument");
  PWB_CUDA(cudaSetDevice(ctxs[0]->device));
  // warm-up outside the capture (scratch, attributes, library handles)
  if ((rc = batch_enqueue(ncell, ctxs, psi, ld, out, ldo, nband, nullptr))) return rc;
  PWB_CUDA(cudaDeviceSynchronize());
  std::vector<char> chk(ncell);
  for (int c = 0; c < ncell; ++c) {
    chk[c] = ctxs[c]->check_errors;
    ctxs[c]->check_errors = false;
  }
  cudaStream_t st;
  PWB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  pw_graph* g = new pw_graph();
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = batch_enqueue(ncell, ctxs, psi, ld, out, ldo, nband, st);
    cudaError_t e2 = cudaStreamEndCapture(st, &g->graph);
    if (!rc && e2 != cudaSuccess) e = e2;
  }
  for (int c = 0; c < ncell; ++c) ctxs[c]->check_errors = chk[c];
  if (e == cudaSuccess && !rc) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e == cudaSuccess && !rc) e = cudaGraphGetNodes(g->graph, nullptr, &g->nodes);
  cudaStreamDestroy(st);
  if (rc || e != cudaSuccess) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    if (!rc) {
      set_error(std::string("graph capture failed: ") + cudaGetErrorString(e));
      rc = PW_ECUDA;
    }
    cudaGetLastError();
    return rc;
  }
  *graph = g;
  return PW_OK;
}

int pw_graph_launch(pw_graph* g, void* stream) {
  PWB_CHECK(g && g->exec, PW_EINVAL, "null graph");
  PWB_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  return PW_OK;
}

int pw_graph_nodes(const pw_graph* g, long* nodes) {
  PWB_CHECK(g && nodes, PW_EINVAL, "null argument");
  *nodes = (long)g->nodes;
  return PW_OK;
}

int pw_graph_destroy(pw_graph* g) {
  if (!g) return PW_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return PW_OK;
}

}  // extern "C"
