// Context set-up: Fourier tables, potential, projector tables, scratch, and
// the C ABI for the H*psi / Teter entry points.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include <cublas_v2.h>

#include "common.hpp"
#include "fft.cuh"
#include "gemm.hpp"
#include "grid_registry.hpp"

namespace pwb {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }

int DevBuf::alloc(size_t nbytes) {
  if (nbytes <= bytes && p) return PW_OK;
  release();
  if (nbytes == 0) return PW_OK;
  cudaError_t e = cudaMalloc(&p, nbytes);
  if (e != cudaSuccess) {
    p = nullptr;
    set_error(std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    return PW_ENOMEM;
  }
  bytes = nbytes;
  return PW_OK;
}
void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

// defined in hpsi.cu
int grid_chunk_rows(const int n[3], int prec);
int run_hpsi(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int nband, int band0, int npair, int acc,
             cudaStream_t st);
int run_teter(pw_ctx* c, const void* r, int ld, void* out, int ldo, int nband, int band0, int npair, int acc,
              cudaStream_t st);
int run_build_q(pw_ctx* c, const int* d_idx, const double* d_beta, const long* d_pio, const long* d_pbo,
                const int* d_pnp, int nproj, cudaStream_t st, int deriv = 0, void* out = nullptr);

// upload a double host vector as the context's precision
int upload_real(pw_ctx* c, DevBuf& dst, const double* src, size_t n) {
  int rc = dst.alloc(n * c->esz);
  if (rc) return rc;
  if (c->prec == PW_F64) {
    PWB_CUDA(cudaMemcpy(dst.p, src, n * 8, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> tmp(n);
    for (size_t i = 0; i < n; ++i) tmp[i] = (float)src[i];
    PWB_CUDA(cudaMemcpy(dst.p, tmp.data(), n * 4, cudaMemcpyHostToDevice));
  }
  return PW_OK;
}

// the fine-plane kernel's permuted copy of vtot, rebuilt after every write of
// vtot (on the legacy stream, finished before returning, so that streams and
// graph replays that read it afterwards see the new potential)
int refresh_vperm(pw_ctx* c) {
  const GridEntry* g = find_grid(c->n);
  if (!g || !c->vtot.p) return PW_OK;
  int rc = g->vperm[c->prec == PW_F32 ? 1 : 0](c, nullptr);
  if (rc) return rc;
  PWB_CUDA(cudaStreamSynchronize(nullptr));
  return PW_OK;
}

int upload_twiddles(pw_ctx* c, int slot, int n) {
  std::vector<double> t(2 * n);
  for (int m = 0; m < n; ++m) {
    // exact values at the quarter points, cos/sin of 2*pi*m/n elsewhere
    const double a = 2.0 * M_PI * (double)m / (double)n;
    double cs = std::cos(a), sn = std::sin(a);
    if (4 * m == n) { cs = 0; sn = 1; }
    if (2 * m == n) { cs = -1; sn = 0; }
    if (4 * m == 3 * n) { cs = 0; sn = -1; }
    t[2 * m] = cs;
    t[2 * m + 1] = -sn;
  }
  return upload_real(c, c->tw[slot], t.data(), 2 * (size_t)n);
}

// After ctx->q (T [nproj][ntot]) is filled: the split-BF16 copies of Q and Q^T
// that the FP32 tensor-core projector GEMMs read
int install_dense_q(pw_ctx* ctx, int nproj) {
  int rc;
  ++ctx->q_version;
  if (ctx->prec == PW_F32) {
    const int npp = (nproj + 7) / 8 * 8;
    ctx->nproj_pad = npp;
    const size_t nt = ctx->ntot;
    const size_t ntp = (nt + 7) / 8 * 8;   // bf16 row stride of Q (16-byte TMA rows)
    if ((rc = ctx->q_bf.alloc((size_t)2 * nproj * ntp * 2)) || (rc = ctx->qt_bf.alloc((size_t)2 * nt * npp * 2)))
      return rc;
    PWB_CUDA(cudaMemset(ctx->qt_bf.p, 0, (size_t)2 * nt * npp * 2));
    char* qb = (char*)ctx->q_bf.p;
    char* qtb = (char*)ctx->qt_bf.p;
    if ((rc = split_bf16((const float*)ctx->q.p, nt, (int)nt, nproj, qb, qb + (size_t)nproj * ntp * 2, ntp, 1.0f,
                         nullptr)))
      return rc;
    if ((rc = split_bf16_t((const float*)ctx->q.p, nt, (int)nt, nproj, qtb, qtb + nt * npp * 2, npp, nullptr)))
      return rc;
    PWB_CUDA(cudaDeviceSynchronize());
  }
  return PW_OK;
}

// In-place P X for nb columns: the Teter pipeline with the 0/1 filter mask as
// its table (forward transform, mask, inverse transform; the normalisations of
// the pair pipeline cancel like FFTWExecute's vol/N and 1/vol).
int wfn_filter_pass(pw_ctx* c, void* X, int ld, int nb, cudaStream_t st) {
  const void* saved = c->teter_tab;
  c->teter_tab = c->wmask.p;
  int rc = PW_OK;
  const int cap = c->pair_cap;
  for (int b0 = 0; b0 < nb && !rc; b0 += 2 * cap) {
    const int npair = std::min(cap, (nb - b0 + 1) / 2);
    rc = run_teter(c, X, ld, X, ld, nb, b0, npair, 0, st);
  }
  c->teter_tab = saved;
  return rc;
}

// rows (T [n][ntot]) -> P rows, and for FP32 contexts the split-BF16 transpose
// the accumulating projector GEMM reads (npad padded columns)
static int filtered_copy(pw_ctx* c, const DevBuf& src, int n, int npad, DevBuf& dst, DevBuf& dst_t_bf) {
  const size_t nt = c->ntot;
  int rc;
  if ((rc = dst.alloc((size_t)n * nt * c->esz))) return rc;
  PWB_CUDA(cudaMemcpy(dst.p, src.p, (size_t)n * nt * c->esz, cudaMemcpyDeviceToDevice));
  if ((rc = wfn_filter_pass(c, dst.p, (int)nt, n, nullptr))) return rc;
  if (c->prec == PW_F32) {
    if ((rc = dst_t_bf.alloc((size_t)2 * nt * npad * 2))) return rc;
    PWB_CUDA(cudaMemset(dst_t_bf.p, 0, (size_t)2 * nt * npad * 2));
    char* bt = (char*)dst_t_bf.p;
    if ((rc = split_bf16_t((const float*)dst.p, nt, (int)nt, n, bt, bt + nt * npad * 2, npad, nullptr))) return rc;
  }
  PWB_CUDA(cudaDeviceSynchronize());
  return PW_OK;
}

// The filtered store-side copies P Q and P xi, made again whenever the
// projectors, the ACE vectors or the cut-off changed since the last copy.
int prepare_wfn_filter(pw_ctx* c) {
  int rc;
  if (c->nproj > 0 && c->nl_mode == PW_NL_DENSE && (c->qf_version != c->q_version || c->qf_ecut != c->wfn_ecut)) {
    if ((rc = filtered_copy(c, c->q, c->nproj, c->nproj_pad, c->qf, c->qtf_bf))) return rc;
    c->qf_version = c->q_version;
    c->qf_ecut = c->wfn_ecut;
  }
  if (c->ace_n > 0 && (c->acef_version != c->ace_version || c->acef_ecut != c->wfn_ecut)) {
    if ((rc = filtered_copy(c, c->ace_xi, c->ace_n, c->ace_npad, c->acef_xi, c->acef_t_bf))) return rc;
    c->acef_version = c->ace_version;
    c->acef_ecut = c->wfn_ecut;
  }
  return PW_OK;
}

int ensure_scratch(pw_ctx* c, int npair) {
  if (npair <= c->pair_cap && c->s_ad.p) return PW_OK;
  const size_t cs = 2 * c->esz;   // complex element
  const size_t nb = (size_t)c->nf[2] * (c->n[1] + 1) * (c->n[0] + 1);
  int rc;
  if ((rc = c->s_ad.alloc((size_t)npair * c->ntot * cs))) return rc;
  if ((rc = c->s_k.alloc((size_t)npair * c->ntot * cs))) return rc;
  if ((rc = c->s_bc.alloc((size_t)npair * nb * cs))) return rc;
  const size_t nslot = std::max(1, c->nl.nslot), nat = std::max(1, c->nl.natom), np = std::max(1, c->nl.npmax);
  if ((rc = c->s_wp.alloc((size_t)npair * nslot * np * cs))) return rc;
  if ((rc = c->s_w.alloc((size_t)npair * nat * np * cs))) return rc;
  if ((rc = c->s_wq.alloc((size_t)std::max(1, c->nproj) * 2 * npair * c->esz))) return rc;
  c->pair_cap = npair;
  return PW_OK;
}

}  // namespace pwb

using namespace pwb;

extern "C" {

const char* pw_last_error(void) { return g_err.c_str(); }
const char* pw_version(void) { return "pwdft_b200 0.1 (sm_100a)"; }

int pw_ctx_create(const double length[3], const int numGrid[3], const int numGridFine[3], int precision, int device,
                  pw_ctx** out) {
  PWB_CHECK(out && length && numGrid && numGridFine, PW_EINVAL, "null argument");
  *out = nullptr;
  PWB_CHECK(precision == PW_F64 || precision == PW_F32, PW_EINVAL, "precision must be PW_F64 or PW_F32");
  for (int d = 0; d < 3; ++d) {
    PWB_CHECK(length[d] > 0, PW_EINVAL, "cell length must be positive");
    PWB_CHECK(numGrid[d] > 0 && numGrid[d] % 2 == 0, PW_EINVAL, "coarse grid sizes must be even");
    PWB_CHECK(numGridFine[d] == 2 * numGrid[d], PW_EUNSUPPORTED,
              "this path needs numGridFine = 2*numGrid (Density_Grid_Factor 2)");
    PWB_CHECK(fft_len_supported(numGrid[d]) && fft_len_supported(numGridFine[d]), PW_EUNSUPPORTED,
              "FFT length not supported");
  }
  PWB_CHECK(find_grid(numGrid) != nullptr, PW_EUNSUPPORTED, "grid not instantiated in this build");
  PWB_CUDA(cudaSetDevice(device));
  pw_ctx* c = new pw_ctx();
  c->prec = precision;
  // the projector GEMMs beside the FFT chain: on in FP32 (Si64 sweep 0.839 ->
  // 0.823 ms), off in FP64, where the FP64 GEMMs and FFTs contend (2.169 ->
  // 2.200 ms)
  c->nl_overlap = precision == PW_F32 ? 1 : 0;
  c->esz = precision == PW_F64 ? 8 : 4;
  c->device = device;
  for (int d = 0; d < 3; ++d) {
    c->L[d] = length[d];
    c->n[d] = numGrid[d];
    c->nf[d] = numGridFine[d];
  }
  c->vol = length[0] * length[1] * length[2];
  c->ntot = (long)numGrid[0] * numGrid[1] * numGrid[2];
  c->ntotf = (long)numGridFine[0] * numGridFine[1] * numGridFine[2];
  // |G|^2/2 and Teter on the full coarse spectrum, KGrid with Nyquist at +n/2
  // (src/SCF/fourier.cpp:124-133, src/SCF/hamiltonian.cpp:2651-2663)
  std::vector<double> ek(c->ntot), te(c->ntot);
  const int n0 = c->n[0], n1 = c->n[1], n2 = c->n[2];
  for (int k = 0; k < n2; ++k)
    for (int j = 0; j < n1; ++j)
      for (int i = 0; i < n0; ++i) {
        const double m0 = i <= n0 / 2 ? i : i - n0, m1 = j <= n1 / 2 ? j : j - n1, m2 = k <= n2 / 2 ? k : k - n2;
        const double g0 = 2 * M_PI / c->L[0] * m0, g1 = 2 * M_PI / c->L[1] * m1, g2 = 2 * M_PI / c->L[2] * m2;
        const double e = (g0 * g0 + g1 * g1 + g2 * g2) / 2;
        const long idx = i + (long)n0 * (j + (long)n1 * k);
        ek[idx] = e;
        const double a = e * 2.0;
        const double b = 27.0 + a * (18.0 + a * (12.0 + a * 8.0));
        te[idx] = b / (b + 16.0 * std::pow(a, 4.0));
      }
  int rc;
  if ((rc = upload_real(c, c->ekin, ek.data(), ek.size())) ||
      (rc = upload_real(c, c->teter, te.data(), te.size()))) {
    delete c;
    return rc;
  }
  const int lens[6] = {n0, n1, n2, c->nf[0], c->nf[1], c->nf[2]};
  for (int s = 0; s < 6; ++s)
    if ((rc = upload_twiddles(c, s, lens[s]))) { delete c; return rc; }
  c->nl.cr = grid_chunk_rows(c->n, c->prec);
  if ((rc = ensure_scratch(c, 32))) { delete c; return rc; }
  {
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) { delete c; set_error("cublasCreate failed"); return PW_ECUDA; }
    cublasSetMathMode(h, CUBLAS_DEFAULT_MATH);
    c->blas = h;
  }
  *out = c;
  return PW_OK;
}

int pw_ctx_destroy(pw_ctx* ctx) {
  if (!ctx) return PW_OK;
  cudaSetDevice(ctx->device);
  for (auto& r : ctx->prof) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  for (auto e : ctx->ev_pool) cudaEventDestroy(e);
  if (ctx->blas) cublasDestroy((cublasHandle_t)ctx->blas);
  for (cudaStream_t st : ctx->io_st)
    if (st) cudaStreamDestroy(st);
  if (ctx->nl_st) cudaStreamDestroy(ctx->nl_st);
  if (ctx->nl_fork) cudaEventDestroy(ctx->nl_fork);
  if (ctx->nl_join) cudaEventDestroy(ctx->nl_join);
  if (ctx->scf_cache_free) ctx->scf_cache_free(ctx->scf_cache);
  if (ctx->twin) pw_ctx_destroy(ctx->twin);
  delete ctx;
  return PW_OK;
}

int pw_profile(pw_ctx* ctx, int enable) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  PWB_CUDA(cudaSetDevice(ctx->device));
  PWB_CUDA(cudaDeviceSynchronize());
  for (auto& r : ctx->prof) { ctx->ev_pool.push_back(r.a); ctx->ev_pool.push_back(r.b); }
  ctx->prof.clear();
  ctx->prof_on = enable != 0;
  return PW_OK;
}

int pw_profile_read(pw_ctx* ctx, int kind, double* total_ms, long* count) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  PWB_CUDA(cudaSetDevice(ctx->device));
  double t = 0;
  long n = 0;
  for (auto& r : ctx->prof) {
    if (r.kind != kind) continue;
    PWB_CUDA(cudaEventSynchronize(r.b));
    float ms = 0;
    PWB_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    t += ms;
    ++n;
  }
  if (total_ms) *total_ms = t;
  if (count) *count = n;
  return PW_OK;
}

int pw_ctx_sizes(const pw_ctx* ctx, long* ntot, long* ntotFine) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  if (ntot) *ntot = ctx->ntot;
  if (ntotFine) *ntotFine = ctx->ntotf;
  return PW_OK;
}

int pw_set_vtot(pw_ctx* ctx, const double* vtot) {
  PWB_CHECK(ctx && vtot, PW_EINVAL, "null argument");
  PWB_CUDA(cudaSetDevice(ctx->device));
  int rc = upload_real(ctx, ctx->vtot, vtot, ctx->ntotf);
  if (rc || (rc = refresh_vperm(ctx))) return rc;
  ctx->h_vtot.assign(vtot, vtot + ctx->ntotf);
  ctx->have_vtot = true;
  return PW_OK;
}

int pw_set_nonlocal_mode(pw_ctx* ctx, int mode) {
  PWB_CHECK(ctx && (mode == PW_NL_DENSE || mode == PW_NL_REALSPACE), PW_EINVAL, "bad nonlocal mode");
  PWB_CHECK(!ctx->have_nl || mode == ctx->nl_mode, PW_EINVAL, "set the nonlocal mode before the projectors");
  ctx->nl_mode = mode;
  return PW_OK;
}

int pw_set_gemm_mode(pw_ctx* ctx, int mode, int terms) {
  PWB_CHECK(ctx && mode == 0 && (terms == 3 || terms == 4), PW_EINVAL, "bad GEMM mode");
  ctx->gemm_terms = terms;
  return PW_OK;
}

int pw_set_check_errors(pw_ctx* ctx, int enable) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  ctx->check_errors = enable != 0;
  return PW_OK;
}

int pw_set_band_batch(pw_ctx* ctx, int nband_batch) {
  PWB_CHECK(ctx && nband_batch > 0, PW_EINVAL, "bad band batch");
  PWB_CUDA(cudaSetDevice(ctx->device));
  ctx->pair_cap = 0;
  return ensure_scratch(ctx, (nband_batch + 1) / 2);
}

int pw_set_nonlocal(pw_ctx* ctx, int natom, const int* atom_npts, const int* atom_nproj, const int* idx,
                    const double* beta, const double* weight) {
  PWB_CHECK(ctx && natom >= 0, PW_EINVAL, "bad arguments");
  PWB_CHECK(!ctx->gs, PW_EUNSUPPORTED, "real-space projector sets do not apply to a G-space context (pw_gs_set_projectors)");
  PWB_CUDA(cudaSetDevice(ctx->device));
  NonlocalDev& nl = ctx->nl;
  const int NXF = ctx->nf[0], NYF = ctx->nf[1], NZF = ctx->nf[2];
  const int cr = nl.cr;
  PWB_CHECK(cr > 0 && NYF % cr == 0, PW_EINVAL, "bad chunk rows");
  const int nchunk = NYF / cr;
  const int ntile = NZF * nchunk;
  int npmax = 0;
  long nent = 0;
  for (int a = 0; a < natom; ++a) {
    PWB_CHECK(atom_npts[a] >= 0 && atom_nproj[a] >= 0, PW_EINVAL, "negative sizes");
    npmax = std::max(npmax, atom_nproj[a]);
    nent += atom_npts[a];
  }
  PWB_CHECK(npmax <= 8, PW_EUNSUPPORTED, "at most 8 projectors per atom are supported");
  PWB_CHECK(nent < (1L << 31), PW_EUNSUPPORTED, "too many projector points");
  ctx->h_nl.clear();   // analytic derivative columns stay only for sets built by pw_set_atoms
  {
    // host copy of the flattened sets: projector l of atom a has its points at
    // idx[pio[l] ..] and values at beta[pbo[l] ..], pnp[l] of them, weight gamma_l
    long off = 0, boff = 0, woff = 0;
    ctx->h_pio.clear(); ctx->h_pbo.clear(); ctx->h_pnp.clear(); ctx->h_patom.clear(); ctx->h_pgamma.clear();
    for (int a = 0; a < natom; ++a) {
      for (int q = 0; q < atom_nproj[a]; ++q) {
        ctx->h_pio.push_back(off);
        ctx->h_pbo.push_back(boff + (long)q * atom_npts[a]);
        ctx->h_pnp.push_back(atom_npts[a]);
        ctx->h_patom.push_back(a);
        ctx->h_pgamma.push_back(weight[woff + q]);
      }
      off += atom_npts[a];
      boff += (long)atom_nproj[a] * atom_npts[a];
      woff += atom_nproj[a];
    }
    ctx->h_nl_idx.assign(idx, idx + off);
    ctx->h_nl_beta.assign(beta, beta + boff);
  }
  if (ctx->nl_mode == PW_NL_DENSE) {
    // per-projector offsets into idx / beta, weights gamma_l * vol / ntot
    std::vector<long> pio, pbo;
    std::vector<int> pnp;
    std::vector<double> qd;
    long off = 0, boff = 0, woff = 0;
    for (int a = 0; a < natom; ++a) {
      for (int q = 0; q < atom_nproj[a]; ++q) {
        pio.push_back(off);
        pbo.push_back(boff + (long)q * atom_npts[a]);
        pnp.push_back(atom_npts[a]);
        qd.push_back(weight[woff + q] * ctx->vol / (double)ctx->ntot);
      }
      for (int i = 0; i < atom_npts[a]; ++i) {
        const int g = idx[off + i];
        PWB_CHECK(g >= 0 && g < ctx->ntotf, PW_EINVAL, "projector index outside the fine grid");
      }
      off += atom_npts[a];
      boff += (long)atom_nproj[a] * atom_npts[a];
      woff += atom_nproj[a];
    }
    const int nproj = (int)pnp.size();
    ctx->nproj = nproj;
    ctx->have_nl = false;
    int rc;
    if (nproj > 0) {
      DevBuf d_idx, d_beta, d_pio, d_pbo, d_pnp;
      if ((rc = d_idx.alloc(std::max<long>(off, 1) * 4)) || (rc = d_beta.alloc(std::max<long>(boff, 1) * 8)) ||
          (rc = d_pio.alloc(nproj * 8)) || (rc = d_pbo.alloc(nproj * 8)) || (rc = d_pnp.alloc(nproj * 4)))
        return rc;
      if (off) PWB_CUDA(cudaMemcpy(d_idx.p, idx, off * 4, cudaMemcpyHostToDevice));
      if (boff) PWB_CUDA(cudaMemcpy(d_beta.p, beta, boff * 8, cudaMemcpyHostToDevice));
      PWB_CUDA(cudaMemcpy(d_pio.p, pio.data(), nproj * 8, cudaMemcpyHostToDevice));
      PWB_CUDA(cudaMemcpy(d_pbo.p, pbo.data(), nproj * 8, cudaMemcpyHostToDevice));
      PWB_CUDA(cudaMemcpy(d_pnp.p, pnp.data(), nproj * 4, cudaMemcpyHostToDevice));
      if ((rc = ctx->q.alloc((size_t)nproj * ctx->ntot * ctx->esz))) return rc;
      if ((rc = upload_real(ctx, ctx->qd, qd.data(), nproj))) return rc;
      const int cap = std::max(ctx->pair_cap, 1);
      ctx->pair_cap = 0;
      if ((rc = ensure_scratch(ctx, cap))) return rc;
      rc = run_build_q(ctx, (const int*)d_idx.p, (const double*)d_beta.p, (const long*)d_pio.p,
                       (const long*)d_pbo.p, (const int*)d_pnp.p, nproj, nullptr);
      if (rc) return rc;
      if ((rc = install_dense_q(ctx, nproj))) return rc;
    }
    nl.natom = natom;
    nl.npmax = npmax;
    ctx->have_nl = nproj > 0;
    return PW_OK;
  }
  // bucket entries by tile, stable in (atom, point order)
  std::vector<int> tile_count(ntile + 1, 0);
  {
    long off = 0;
    for (int a = 0; a < natom; ++a) {
      for (int i = 0; i < atom_npts[a]; ++i) {
        const int g = idx[off + i];
        PWB_CHECK(g >= 0 && g < ctx->ntotf, PW_EINVAL, "projector index outside the fine grid");
        const int z = g / (NXF * NYF), y = (g / NXF) % NYF;
        tile_count[z * nchunk + y / cr + 1]++;
      }
      off += atom_npts[a];
    }
  }
  for (int t = 0; t < ntile; ++t) tile_count[t + 1] += tile_count[t];
  std::vector<int> e_xy(nent), e_atom(nent);
  std::vector<double> e_beta((size_t)std::max(npmax, 1) * nent, 0.0);
  {
    std::vector<int> fill(tile_count.begin(), tile_count.end() - 1);
    long off = 0, boff = 0;
    for (int a = 0; a < natom; ++a) {
      const int np = atom_npts[a];
      for (int i = 0; i < np; ++i) {
        const int g = idx[off + i];
        const int z = g / (NXF * NYF), y = (g / NXF) % NYF, x = g % NXF;
        const int e = fill[z * nchunk + y / cr]++;
        e_xy[e] = y * NXF + x;
        e_atom[e] = a;
        for (int q = 0; q < atom_nproj[a]; ++q) e_beta[(size_t)q * nent + e] = beta[boff + (long)q * np + i];
      }
      off += np;
      boff += (long)atom_nproj[a] * np;
    }
  }
  // slots: runs of equal atom inside a tile
  std::vector<int> tile_slot(ntile + 1, 0), slot_atom, slot_ent;
  for (int t = 0; t < ntile; ++t) {
    tile_slot[t] = (int)slot_atom.size();
    for (int e = tile_count[t]; e < tile_count[t + 1]; ++e) {
      if (e == tile_count[t] || e_atom[e] != e_atom[e - 1]) {
        slot_atom.push_back(e_atom[e]);
        slot_ent.push_back(e);
      }
    }
  }
  tile_slot[ntile] = (int)slot_atom.size();
  slot_ent.push_back((int)nent);
  const int nslot = (int)slot_atom.size();
  std::vector<int> atom_slot(natom + 1, 0), atom_slot_list(nslot);
  for (int s = 0; s < nslot; ++s) atom_slot[slot_atom[s] + 1]++;
  for (int a = 0; a < natom; ++a) atom_slot[a + 1] += atom_slot[a];
  {
    std::vector<int> fill(atom_slot.begin(), atom_slot.end() - 1);
    for (int s = 0; s < nslot; ++s) atom_slot_list[fill[slot_atom[s]]++] = s;
  }
  std::vector<double> wg((size_t)std::max(natom, 1) * std::max(npmax, 1), 0.0);
  {
    long woff = 0;
    const double fac = ctx->vol / (double)ctx->ntotf;
    for (int a = 0; a < natom; ++a) {
      for (int q = 0; q < atom_nproj[a]; ++q) wg[(size_t)a * npmax + q] = weight[woff + q] * fac;
      woff += atom_nproj[a];
    }
  }
  int rc;
  auto up_int = [&](DevBuf& b, const std::vector<int>& v) -> int {
    int r = b.alloc(std::max<size_t>(v.size(), 1) * 4);
    if (r) return r;
    if (!v.empty()) PWB_CUDA(cudaMemcpy(b.p, v.data(), v.size() * 4, cudaMemcpyHostToDevice));
    return PW_OK;
  };
  if ((rc = up_int(nl.ent_xy, e_xy)) || (rc = up_int(nl.tile_slot, tile_slot)) ||
      (rc = up_int(nl.slot_atom, slot_atom)) || (rc = up_int(nl.slot_ent, slot_ent)) ||
      (rc = up_int(nl.atom_slot, atom_slot)) || (rc = up_int(nl.atom_slot_list, atom_slot_list)))
    return rc;
  if ((rc = upload_real(ctx, nl.ent_beta, e_beta.data(), e_beta.size()))) return rc;
  if ((rc = upload_real(ctx, nl.wgt, wg.data(), wg.size()))) return rc;
  nl.natom = natom;
  nl.npmax = npmax;
  nl.nent = (int)nent;
  nl.nslot = nslot;
  nl.ntile = ntile;
  nl.nchunk = nchunk;
  ctx->have_nl = true;
  const int cap = std::max(ctx->pair_cap, 1);
  ctx->pair_cap = 0;
  return ensure_scratch(ctx, cap);
}

int pw_hpsi(pw_ctx* ctx, const void* psi, int ld, void* hpsi, int ldh, int nband, int accumulate, void* stream) {
  PWB_CHECK(ctx && (nband == 0 || (psi && hpsi)), PW_EINVAL, "null argument");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot && ldh >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CHECK(ctx->have_vtot, PW_ENOTREADY, "local potential not set (pw_set_vtot)");
  PWB_CHECK(!ctx->gs || nband == 0 ||
                (ld % 2 == 0 && ldh % 2 == 0 && (uintptr_t)psi % (2 * ctx->esz) == 0 &&
                 (uintptr_t)hpsi % (2 * ctx->esz) == 0),
            PW_EINVAL, "G-space bands are complex: even leading dimensions and complex-aligned pointers");
  PWB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (ctx->wfn_filter && !accumulate) {
    int rc = prepare_wfn_filter(ctx);
    if (rc) return rc;
  }
  const int cap = ctx->pair_cap;
  for (int b0 = 0; b0 < nband; b0 += 2 * cap) {
    const int npair = std::min(cap, (nband - b0 + 1) / 2);
    int rc = run_hpsi(ctx, psi, ld, hpsi, ldh, nband, b0, npair, accumulate, st);
    if (rc) return rc;
  }
  if (ctx->check_errors) return gemm_error_check();
  return PW_OK;
}

int pw_set_fft_variant(pw_ctx* ctx, int variant) {
  PWB_CHECK(ctx && variant >= 0 && variant <= 2, PW_EINVAL, "FFT variant must be 0, 1 or 2");
  ctx->fft_variant = variant;
  return PW_OK;
}

int pw_set_nl_overlap(pw_ctx* ctx, int on) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  ctx->nl_overlap = on ? 1 : 0;
  if (ctx->twin) ctx->twin->nl_overlap = ctx->nl_overlap;
  return PW_OK;
}

int pw_set_wait_limit(pw_ctx* ctx, double seconds) {
  PWB_CHECK(ctx && seconds > 0 && seconds < 3600, PW_EINVAL, "wait limit must be in (0, 3600) s");
  PWB_CUDA(cudaSetDevice(ctx->device));
  return set_wait_limit_ns((unsigned long long)(seconds * 1e9));
}

int pw_wait_probe(pw_ctx* ctx, double seconds) {
  PWB_CHECK(ctx && seconds > 0 && seconds <= 10, PW_EINVAL, "probe limit must be in (0, 10] s");
  PWB_CUDA(cudaSetDevice(ctx->device));
  return wait_probe((unsigned long long)(seconds * 1e9), nullptr);
}

int pw_set_wfn_filter(pw_ctx* ctx, int enable, double ecut) {
  PWB_CHECK(ctx, PW_EINVAL, "null argument");
  if (!enable) {
    ctx->wfn_filter = false;
    return PW_OK;
  }
  PWB_CHECK(ecut > 0, PW_EINVAL, "the wavefunction filter needs a positive cut-off");
  PWB_CHECK(!ctx->gs, PW_EUNSUPPORTED,
            "sphere-cut contexts hold only the coefficients inside their Ecut sphere; the wavefunction filter "
            "belongs to real-space contexts");
  PWB_CUDA(cudaSetDevice(ctx->device));
  if (!ctx->wmask.p || ctx->wfn_ecut != ecut) {
    // the mask on the full coarse spectrum from the same |G|^2/2 as the kinetic
    // table, in double: zero where gkk > ecut (hamiltonian.cpp:3107-3111)
    std::vector<double> m(ctx->ntot);
    const int n0 = ctx->n[0], n1 = ctx->n[1], n2 = ctx->n[2];
    for (int k = 0; k < n2; ++k)
      for (int j = 0; j < n1; ++j)
        for (int i = 0; i < n0; ++i) {
          const double m0 = i <= n0 / 2 ? i : i - n0, m1 = j <= n1 / 2 ? j : j - n1, m2 = k <= n2 / 2 ? k : k - n2;
          const double g0 = 2 * M_PI / ctx->L[0] * m0, g1 = 2 * M_PI / ctx->L[1] * m1,
                       g2 = 2 * M_PI / ctx->L[2] * m2;
          m[i + (long)n0 * (j + (long)n1 * k)] = (g0 * g0 + g1 * g1 + g2 * g2) / 2 > ecut ? 0.0 : 1.0;
        }
    int rc = upload_real(ctx, ctx->wmask, m.data(), m.size());
    if (rc) return rc;
  }
  ctx->wfn_ecut = ecut;
  ctx->wfn_filter = true;
  return prepare_wfn_filter(ctx);
}

int pw_wfn_filter(pw_ctx* ctx, void* X, int ld, int nband, void* stream) {
  PWB_CHECK(ctx && (nband == 0 || X), PW_EINVAL, "null argument");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CHECK(ctx->wfn_filter, PW_ENOTREADY, "wavefunction filter not set (pw_set_wfn_filter)");
  PWB_CUDA(cudaSetDevice(ctx->device));
  return wfn_filter_pass(ctx, X, ld, nband, (cudaStream_t)stream);
}

int pw_teter_precond(pw_ctx* ctx, const void* r, int ld, void* w, int ldw, int nband, int accumulate, void* stream) {
  PWB_CHECK(ctx && (nband == 0 || (r && w)), PW_EINVAL, "null argument");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot && ldw >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int cap = ctx->pair_cap;
  for (int b0 = 0; b0 < nband; b0 += 2 * cap) {
    const int npair = std::min(cap, (nband - b0 + 1) / 2);
    int rc = run_teter(ctx, r, ld, w, ldw, nband, b0, npair, accumulate, st);
    if (rc) return rc;
  }
  return PW_OK;
}

int pw_set_host_chunk(pw_ctx* ctx, int nband) {
  PWB_CHECK(ctx && nband >= 0, PW_EINVAL, "bad arguments");
  ctx->host_chunk = nband == 0 ? 32 : std::max(2, nband + (nband & 1));
  return PW_OK;
}

static bool host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Host-buffer H*psi.  With page-locked host buffers the bands move in chunks:
// every chunk's host->device copy is queued on one stream, its H*psi on a
// second (after that copy) and its device->host copy on a third (after that
// H*psi), so the link carries chunk i+1 in and chunk i-1 out while chunk i
// computes (chunk: pw_set_host_chunk, 32 bands by default; the first and the
// last chunk are half as long, to shorten the fill and drain).  Pageable
// buffers, and blocks of at most 1.5 chunks, take one synchronous copy each way.
int pw_hpsi_host(pw_ctx* ctx, const void* psi, int ld, void* hpsi, int ldh, int nband, int accumulate) {
  PWB_CHECK(ctx && (nband == 0 || (psi && hpsi)), PW_EINVAL, "null argument");
  if (nband == 0) return PW_OK;
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot && ldh >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CUDA(cudaSetDevice(ctx->device));
  const size_t esz = ctx->esz, row = (size_t)ctx->ntot * esz;
  const size_t bytes = row * nband;
  int rc;
  if ((rc = ctx->s_host_in.alloc(bytes)) || (rc = ctx->s_host_out.alloc(bytes))) return rc;
  char* din = (char*)ctx->s_host_in.p;
  char* dout = (char*)ctx->s_host_out.p;
  const int chunk = ctx->host_chunk;
  if (nband <= chunk + chunk / 2 || !host_pinned(psi) || !host_pinned(hpsi)) {
    PWB_CUDA(cudaMemcpy2D(din, row, psi, (size_t)ld * esz, row, nband, cudaMemcpyHostToDevice));
    if (accumulate)
      PWB_CUDA(cudaMemcpy2D(dout, row, hpsi, (size_t)ldh * esz, row, nband, cudaMemcpyHostToDevice));
    rc = pw_hpsi(ctx, din, (int)ctx->ntot, dout, (int)ctx->ntot, nband, accumulate, nullptr);
    if (rc) return rc;
    PWB_CUDA(cudaMemcpy2D(hpsi, (size_t)ldh * esz, dout, row, row, nband, cudaMemcpyDeviceToHost));
    return PW_OK;
  }
  for (cudaStream_t& st : ctx->io_st)
    if (!st) PWB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaStream_t sh = ctx->io_st[0], sc = ctx->io_st[1], sd = ctx->io_st[2];
  // chunk sizes: half a chunk first and last (the pipeline's fill and drain)
  std::vector<int> start;
  {
    const int h = std::max(2, (chunk / 2) & ~1);
    int b = 0;
    start.push_back(0);
    b += h;
    while (nband - b > chunk + h) {
      start.push_back(b);
      b += chunk;
    }
    const int r = nband - b;   // at most chunk + h: one chunk, or an even one and a short last one
    start.push_back(b);
    if (r > chunk && ((r - h) & ~1) > 0) start.push_back(b + ((r - h) & ~1));
    start.push_back(nband);
  }
  const int nch = (int)start.size() - 1;
  std::vector<cudaEvent_t> ev((size_t)2 * nch + 1, nullptr);
  for (auto& e : ev) PWB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  auto done = [&]() {
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  };
  // after the work already queued on the legacy default stream
  cudaEvent_t e0 = ev[2 * nch];
  cudaEventRecord(e0, 0);
  cudaStreamWaitEvent(sh, e0, 0);
  cudaStreamWaitEvent(sc, e0, 0);
  cudaStreamWaitEvent(sd, e0, 0);
  for (int i = 0; i < nch; ++i) {
    const int b0 = start[i], nb = start[i + 1] - b0;
    const char* hin = (const char*)psi + (size_t)b0 * ld * esz;
    cudaError_t e1 = cudaMemcpy2DAsync(din + b0 * row, row, hin, (size_t)ld * esz, row, nb, cudaMemcpyHostToDevice, sh);
    if (e1 == cudaSuccess && accumulate)
      e1 = cudaMemcpy2DAsync(dout + b0 * row, row, (const char*)hpsi + (size_t)b0 * ldh * esz, (size_t)ldh * esz,
                             row, nb, cudaMemcpyHostToDevice, sh);
    if (e1 == cudaSuccess) e1 = cudaEventRecord(ev[2 * i], sh);
    if (e1 != cudaSuccess) {
      cudaStreamSynchronize(sh);
      done();
      PWB_CUDA(e1);
    }
  }
  for (int i = 0; i < nch && rc == PW_OK; ++i) {
    const int b0 = start[i], nb = start[i + 1] - b0;
    cudaStreamWaitEvent(sc, ev[2 * i], 0);
    rc = pw_hpsi(ctx, din + b0 * row, (int)ctx->ntot, dout + b0 * row, (int)ctx->ntot, nb, accumulate, sc);
    if (rc) break;
    cudaEventRecord(ev[2 * i + 1], sc);
    cudaStreamWaitEvent(sd, ev[2 * i + 1], 0);
    cudaMemcpy2DAsync((char*)hpsi + (size_t)b0 * ldh * esz, (size_t)ldh * esz, dout + b0 * row, row, row, nb,
                      cudaMemcpyDeviceToHost, sd);
  }
  const cudaError_t s1 = cudaStreamSynchronize(sh), s2 = cudaStreamSynchronize(sc), s3 = cudaStreamSynchronize(sd);
  done();
  if (rc) return rc;
  PWB_CUDA(s1);
  PWB_CUDA(s2);
  PWB_CUDA(s3);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

}  // extern "C"
