// Grid dispatch of the H*psi pipeline and the allocation-free Teter entry.
// The pipeline kernels and their per-grid Plan live in pipeline.cuh; each
// grid of grids.inc is compiled from grid_instance.cu and registers its entry
// points here when the library is loaded.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "common.hpp"
#include "grid_registry.hpp"

namespace pwb {

static std::vector<GridEntry>& registry() {
  static std::vector<GridEntry> r;
  return r;
}

void register_grid(const GridEntry& e) { registry().push_back(e); }

const GridEntry* find_grid(const int n[3]) {
  for (const auto& g : registry())
    if (g.n0 == n[0] && g.n1 == n[1] && g.n2 == n[2]) return &g;
  return nullptr;
}

int grid_chunk_rows(const int n[3], int prec) {
  const GridEntry* g = find_grid(n);
  return g ? g->cr[prec == PW_F32 ? 1 : 0]() : -1;
}

int gs_teter(pw_ctx* c, const void* r, int ld, void* out, int ldo, int nband, int band0, int npair, int acc,
             cudaStream_t st);

// entry points of the real-space (dual-grid) path that have no sphere-cut form here
static bool gs_refuse(const pw_ctx* c, const char* what) {
  if (!c->gs) return false;
  set_error(std::string(what) + " is not available on a G-space (sphere-cut) context");
  return true;
}

int run_hpsi(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int nband, int band0, int npair, int acc,
             cudaStream_t st) {
  const GridEntry* g = find_grid(c->n);
  if (!g) { set_error("grid not built into this library"); return PW_EUNSUPPORTED; }
  if (c->gs) return g->hpsigs[c->prec == PW_F32 ? 1 : 0](c, psi, ld, out, ldo, nband, band0, npair, acc, st);
  return g->hpsi[c->prec == PW_F32 ? 1 : 0](c, psi, ld, out, ldo, nband, band0, npair, acc, st);
}

int run_build_q(pw_ctx* c, const int* d_idx, const double* d_beta, const long* d_pio, const long* d_pbo,
                const int* d_pnp, int nproj, cudaStream_t st, int deriv, void* out) {
  const GridEntry* g = find_grid(c->n);
  if (!g) { set_error("grid not built into this library"); return PW_EUNSUPPORTED; }
  if (gs_refuse(c, "the real-space projector build")) return PW_EUNSUPPORTED;
  return g->bq[c->prec == PW_F32 ? 1 : 0](c, d_idx, d_beta, d_pio, d_pbo, d_pnp, nproj, st, deriv, out);
}

int run_density(pw_ctx* c, const void* psi, int ld, int nband, int band0, int npair, const double* w, double* rho,
                cudaStream_t st) {
  const GridEntry* g = find_grid(c->n);
  if (!g) { set_error("grid not built into this library"); return PW_EUNSUPPORTED; }
  if (c->gs) return g->densgs[c->prec == PW_F32 ? 1 : 0](c, psi, ld, nband, band0, npair, w, rho, st);
  return g->dens[c->prec == PW_F32 ? 1 : 0](c, psi, ld, nband, band0, npair, w, rho, st);
}

int run_exx(pw_ctx* c, const void* psi, int ld, int nb, void* out, int ldo, int acc, cudaStream_t st) {
  const GridEntry* g = find_grid(c->n);
  if (!g) { set_error("grid not built into this library"); return PW_EUNSUPPORTED; }
  if (c->gs) return gs_exx_apply(c, psi, ld, nb, out, ldo, acc, st);
  return g->exx[c->prec == PW_F32 ? 1 : 0](c, psi, ld, nb, out, ldo, acc, st);
}

int run_hpsi_k(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int band0, int nb, int acc, cudaStream_t st) {
  const GridEntry* g = find_grid(c->n);
  if (!g) { set_error("grid not built into this library"); return PW_EUNSUPPORTED; }
  if (gs_refuse(c, "the k-point H*psi")) return PW_EUNSUPPORTED;
  return g->hpsik[c->prec == PW_F32 ? 1 : 0](c, psi, ld, out, ldo, band0, nb, acc, st);
}

int run_hpsi_kbatch(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int f0, int nf, int acc, cudaStream_t st,
                    int fpk, const void* ekin_all, const void* qk_all) {
  const GridEntry* g = find_grid(c->n);
  if (!g) { set_error("grid not built into this library"); return PW_EUNSUPPORTED; }
  if (gs_refuse(c, "the k-point batch")) return PW_EUNSUPPORTED;
  return g->hpsikb[c->prec == PW_F32 ? 1 : 0](c, psi, ld, out, ldo, f0, nf, acc, st, fpk, ekin_all, qk_all);
}

int run_build_q_k(pw_ctx* c, const int* d_idx, const double* d_beta, const double* d_disp, const long* d_pio,
                  const long* d_pbo, const int* d_pnp, int nproj, const double* kv, void* out, cudaStream_t st) {
  const GridEntry* g = find_grid(c->n);
  if (!g) { set_error("grid not built into this library"); return PW_EUNSUPPORTED; }
  if (gs_refuse(c, "the k-point projector build")) return PW_EUNSUPPORTED;
  return g->bqk[c->prec == PW_F32 ? 1 : 0](c, d_idx, d_beta, d_disp, d_pio, d_pbo, d_pnp, nproj, kv, out, st);
}

int run_ace(pw_ctx* c, const void* psi, int ld, int nb, void* out, int ldo, cudaStream_t st) {
  const GridEntry* g = find_grid(c->n);
  if (!g) { set_error("grid not built into this library"); return PW_EUNSUPPORTED; }
  return g->ace[c->prec == PW_F32 ? 1 : 0](c, psi, ld, nb, out, ldo, 1, st);
}

int run_teter(pw_ctx* c, const void* r, int ld, void* out, int ldo, int nband, int band0, int npair, int acc,
              cudaStream_t st) {
  const GridEntry* g = find_grid(c->n);
  if (!g) { set_error("grid not built into this library"); return PW_EUNSUPPORTED; }
  if (c->gs) return gs_teter(c, r, ld, out, ldo, nband, band0, npair, acc, st);
  return g->teter[c->prec == PW_F32 ? 1 : 0](c, r, ld, out, ldo, nband, band0, npair, acc, st);
}

}  // namespace pwb

// ---------------------------------------------------------------------------
// Allocation-free Teter preconditioner.
//
// Some callers cannot call cudaMalloc at the point where they need the
// preconditioner: code running while a CUDA stream is being captured into a
// graph, real-time or embedded hosts that forbid device allocation after
// start-up, and allocator-owning frameworks (a host code with its own memory
// pool) that must not see device memory change underneath them.  For them the
// entry point pw_teter_precond_noalloc below takes its working memory from one
// fixed array in this file instead of the context's scratch.
// ---------------------------------------------------------------------------
#define PWB_NOALLOC_SCRATCH_BYTES (16u << 20)    // 16 MiB per GPU that loads the library

static __device__ __align__(256) unsigned char g_noalloc_scratch[PWB_NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_noalloc_mu;
// Device address of g_noalloc_scratch per device ordinal, taken once and kept
// for the life of the process.  A cudaDeviceReset (or anything else that
// replaces the device's primary context) invalidates it: calls after such a
// reset are not supported.
void* g_noalloc_addr[64] = {nullptr};
}  // namespace

extern "C" int pw_teter_precond_noalloc(pw_ctx* ctx, const void* r, int ld, void* w, int ldw, int nband,
                                        int accumulate, void* stream) {
  using namespace pwb;
  PWB_CHECK(ctx && (nband == 0 || (r && w)), PW_EINVAL, "null argument");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot && ldw >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CHECK(ctx->device >= 0 && ctx->device < 64, PW_EINVAL, "device ordinal out of range");
  if (nband == 0) return PW_OK;
  // one band pair needs ntot complex values of the context's precision
  const size_t pair_bytes = (size_t)ctx->ntot * 2 * ctx->esz;
  PWB_CHECK(pair_bytes <= PWB_NOALLOC_SCRATCH_BYTES, PW_EINVAL,
            "pw_teter_precond_noalloc: one band pair needs " + std::to_string(pair_bytes) +
                " bytes of scratch, more than the fixed 16 MiB array; use pw_teter_precond");
  PWB_CUDA(cudaSetDevice(ctx->device));
  void* scratch;
  {
    // host code may not use g_noalloc_scratch as a pointer (it names a host-side
    // stand-in); fetch the device address once per device
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[ctx->device]) {
      void* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr) {
        cudaGetLastError();     // clear it: a later, unrelated check must not report this failure as its own
        set_error(std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") + cudaGetErrorString(e));
        return PW_ECUDA;
      }
      g_noalloc_addr[ctx->device] = ptr;
    }
    scratch = g_noalloc_addr[ctx->device];
  }
  const GridEntry* g = find_grid(ctx->n);
  PWB_CHECK(g, PW_EUNSUPPORTED, "grid not built into this library");
  // sphere-cut contexts: the preconditioner is a diagonal product that needs no scratch
  if (ctx->gs) return gs_teter(ctx, r, ld, w, ldw, nband, 0, (nband + 1) / 2, accumulate, (cudaStream_t)stream);
  const int max_pairs = (int)(PWB_NOALLOC_SCRATCH_BYTES / pair_bytes);
  cudaStream_t st = (cudaStream_t)stream;
  for (int b0 = 0; b0 < nband; b0 += 2 * max_pairs) {
    const int npair = std::min(max_pairs, (nband - b0 + 1) / 2);
    int rc = g->teter_scratch[ctx->prec == PW_F32 ? 1 : 0](ctx, r, ld, w, ldw, nband, b0, npair, accumulate, st,
                                                           scratch);
    if (rc) return rc;
  }
  return PW_OK;
}
