// CUDA graphs of the Hamiltonian application: one H*psi call (fixed buffers
// and band count) captured on a private stream and replayed with a single
// cudaGraphLaunch, for callers that apply H to the same block many times
// (iterative eigensolvers, time stepping, serving loops).  Capture runs one
// warm-up call first so that no allocation, attribute set-up or library
// workspace creation happens inside the capture.
#include <cuda_runtime.h>

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
