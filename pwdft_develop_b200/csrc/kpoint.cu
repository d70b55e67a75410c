// k-point (complex band) Hamiltonian: KohnSham::MultSpinor for complex
// wavefunctions, Spinor::AddMultSpinorFine complex version
// (src/SCF/spinor_complex.cpp:292-542, real-space branch).  The tables follow
// KohnSham::CalculateEkin, complex version (src/SCF/hamiltonian_complex.cpp:
// 234-277: ekin = 1/2 |k+G|^2, Teter of |k+G|^2 on the full coarse grid) and
// the projector Bloch phase e^{i k.(r - R_a)} of PeriodTable::CalculateNonlocalPP
// (src/SCF/periodtable.cpp:1104-1121).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.hpp"

namespace pwb {

// bytes of one k-point's split-BF16 projector operands (A1 and A2, hi and lo)
size_t kq_bf_bytes(const pw_ctx* c) {
  const size_t np = c->nproj, nt = c->ntot;
  return 2 * (2 * np * 2 * nt + 2 * nt * (size_t)c->nkp2) * sizeof(__nv_bfloat16);
}

static __device__ __forceinline__ void split2(float v, __nv_bfloat16* h, __nv_bfloat16* l) {
  const __nv_bfloat16 a = __float2bfloat16_rn(v);
  *h = a;
  *l = __float2bfloat16_rn(v - __bfloat162float(a));
}

// Q (complex, [np][nt]) -> the real GEMM operands of V_nl = Q diag(d) Q^H:
//   A1[l][2g], A1[l][2g+1]           = Re q, Im q       (row l:      Re(Q^H psi)_l)
//   A1[np+l][2g], A1[np+l][2g+1]     = -Im q, Re q      (row np + l: Im(Q^H psi)_l)
//   A2[2g][l] = Re q, A2[2g][np+l] = -Im q, A2[2g+1][l] = Im q, A2[2g+1][np+l] = Re q
// so that [Re; Im] of Q W = A2 [Re W; Im W] on interleaved (re, im) rows.
__global__ void k_kq_split(const float2* __restrict__ Q, int np, long nt, int nkp2, __nv_bfloat16* a1h,
                           __nv_bfloat16* a1l, __nv_bfloat16* a2h, __nv_bfloat16* a2l) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)np * nt) return;
  const int l = (int)(i / nt);
  const long g = i - (long)l * nt;
  const float2 q = Q[i];
  const long r0 = (long)l * 2 * nt + 2 * g, r1 = (long)(np + l) * 2 * nt + 2 * g;
  split2(q.x, a1h + r0, a1l + r0);
  split2(q.y, a1h + r0 + 1, a1l + r0 + 1);
  split2(-q.y, a1h + r1, a1l + r1);
  split2(q.x, a1h + r1 + 1, a1l + r1 + 1);
  const long s0 = 2 * g * (long)nkp2, s1 = s0 + nkp2;
  split2(q.x, a2h + s0 + l, a2l + s0 + l);
  split2(-q.y, a2h + s0 + np + l, a2l + s0 + np + l);
  split2(q.y, a2h + s1 + l, a2l + s1 + l);
  split2(q.x, a2h + s1 + np + l, a2l + s1 + np + l);
}

// the split operands of one k-point's projectors (FP32 contexts) at dst
int build_kq_bf(pw_ctx* c, const void* Qk, void* dst) {
  const long nt = c->ntot;
  const int np = c->nproj;
  __nv_bfloat16* a1h = (__nv_bfloat16*)dst;
  __nv_bfloat16* a1l = a1h + (size_t)2 * np * 2 * nt;
  __nv_bfloat16* a2h = a1l + (size_t)2 * np * 2 * nt;
  __nv_bfloat16* a2l = a2h + (size_t)2 * nt * c->nkp2;
  PWB_CUDA(cudaMemset(a2h, 0, (size_t)2 * (2 * nt * c->nkp2) * sizeof(__nv_bfloat16)));
  const long n = (long)np * nt;
  k_kq_split<<<(unsigned)((n + 255) / 256), 256>>>((const float2*)Qk, np, nt, c->nkp2, a1h, a1l, a2h, a2l);
  PWB_CUDA(cudaGetLastError());
  c->launches += 1;
  return PW_OK;
}

static bool kq_tensor_cores(const pw_ctx* c) { return c->prec == PW_F32 && c->nproj > 0; }

int run_hpsi_k(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int band0, int nb, int acc, cudaStream_t st);
int run_hpsi_kbatch(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int f0, int nf, int acc, cudaStream_t st,
                    int fpk, const void* ekin_all, const void* qk_all);
int run_build_q_k(pw_ctx* c, const int* d_idx, const double* d_beta, const double* d_disp, const long* d_pio,
                  const long* d_pbo, const int* d_pnp, int nproj, const double* kv, void* out, cudaStream_t st);
int ensure_scratch(pw_ctx* c, int npair);
int upload_real(pw_ctx* c, DevBuf& dst, const double* src, size_t n);

template <typename X> static int upload(DevBuf& b, const std::vector<X>& h) {
  int rc = b.alloc(std::max<size_t>(h.size(), 1) * sizeof(X));
  if (rc) return rc;
  if (!h.empty()) PWB_CUDA(cudaMemcpy(b.p, h.data(), h.size() * sizeof(X), cudaMemcpyHostToDevice));
  return PW_OK;
}

}  // namespace pwb

using namespace pwb;

extern "C" {

int pw_set_kpoint(pw_ctx* ctx, const double k[3]) {
  PWB_CHECK(ctx && k, PW_EINVAL, "null argument");
  PWB_CHECK(!ctx->gs, PW_EUNSUPPORTED, "k-points are built for real-space contexts only");
  PWB_CUDA(cudaSetDevice(ctx->device));
  const int n0 = ctx->n[0], n1 = ctx->n[1], n2 = ctx->n[2];
  const long nt = ctx->ntot;
  std::vector<double> ek(nt), te(nt);
  for (int z = 0; z < n2; ++z)
    for (int y = 0; y < n1; ++y)
      for (int x = 0; x < n0; ++x) {
        const double m0 = x <= n0 / 2 ? x : x - n0, m1 = y <= n1 / 2 ? y : y - n1, m2 = z <= n2 / 2 ? z : z - n2;
        const double g0 = k[0] + 2 * M_PI / ctx->L[0] * m0, g1 = k[1] + 2 * M_PI / ctx->L[1] * m1,
                     g2 = k[2] + 2 * M_PI / ctx->L[2] * m2;
        const long i = x + (long)n0 * (y + (long)n1 * z);
        ek[i] = 0.5 * (g0 * g0 + g1 * g1 + g2 * g2);
        const double a = 2.0 * ek[i];
        const double b = 27.0 + a * (18.0 + a * (12.0 + a * 8.0));
        te[i] = b / (b + 16.0 * a * a * a * a);
      }
  int rc;
  if ((rc = upload_real(ctx, ctx->ekin_k, ek.data(), nt)) || (rc = upload_real(ctx, ctx->teter_k, te.data(), nt)))
    return rc;
  const int np = (int)ctx->h_pnp.size();
  ctx->qk.release();
  if (np > 0) {
    size_t tot = 0;
    for (const auto& a : ctx->h_nl) tot += a.val.size();
    PWB_CHECK(tot == (size_t)np && !ctx->h_nl.empty(), PW_ENOTREADY,
              "k-point projectors need the sets of pw_set_atoms (grid-point displacements)");
    std::vector<double> disp;
    disp.reserve(3 * ctx->h_nl_idx.size());
    for (const auto& a : ctx->h_nl) disp.insert(disp.end(), a.disp.begin(), a.disp.end());
    PWB_CHECK(disp.size() == 3 * ctx->h_nl_idx.size(), PW_EINVAL, "projector sets changed since pw_set_atoms");
    DevBuf d_idx, d_beta, d_disp, d_pio, d_pbo, d_pnp;
    if ((rc = upload(d_idx, ctx->h_nl_idx)) || (rc = upload(d_beta, ctx->h_nl_beta)) || (rc = upload(d_disp, disp)) ||
        (rc = upload(d_pio, ctx->h_pio)) || (rc = upload(d_pbo, ctx->h_pbo)) || (rc = upload(d_pnp, ctx->h_pnp)))
      return rc;
    if ((rc = ctx->qk.alloc((size_t)np * nt * 2 * ctx->esz))) return rc;
    if ((rc = ensure_scratch(ctx, std::max(ctx->pair_cap, 1)))) return rc;
    if ((rc = run_build_q_k(ctx, (const int*)d_idx.p, (const double*)d_beta.p, (const double*)d_disp.p,
                            (const long*)d_pio.p, (const long*)d_pbo.p, (const int*)d_pnp.p, np, k, ctx->qk.p,
                            nullptr)))
      return rc;
    std::vector<double> qd(np);
    for (int l = 0; l < np; ++l) qd[l] = ctx->h_pgamma[l] * ctx->vol / (double)nt;
    if ((rc = upload_real(ctx, ctx->qdk, qd.data(), np))) return rc;
    ctx->launches += 5 * ((np + std::max(ctx->pair_cap, 1) - 1) / std::max(ctx->pair_cap, 1));
    if (kq_tensor_cores(ctx)) {
      ctx->nkp2 = (2 * np + 7) / 8 * 8;
      std::vector<float> d2(2 * np);
      for (int l = 0; l < np; ++l) d2[l] = d2[np + l] = (float)qd[l];
      if ((rc = ctx->qdk2.alloc(d2.size() * 4))) return rc;
      PWB_CUDA(cudaMemcpy(ctx->qdk2.p, d2.data(), d2.size() * 4, cudaMemcpyHostToDevice));
      if ((rc = ctx->qk_bf.alloc(kq_bf_bytes(ctx)))) return rc;
      if ((rc = build_kq_bf(ctx, ctx->qk.p, ctx->qk_bf.p))) return rc;
    }
  }
  PWB_CUDA(cudaDeviceSynchronize());
  for (int d = 0; d < 3; ++d) ctx->kvec[d] = k[d];
  ctx->have_k = true;
  return PW_OK;
}

int pw_hpsi_k(pw_ctx* ctx, const void* psi, int ld, void* hpsi, int ldh, int nband, int accumulate, void* stream) {
  PWB_CHECK(ctx && (nband == 0 || (psi && hpsi)), PW_EINVAL, "null argument");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot && ldh >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CHECK(ctx->have_vtot, PW_ENOTREADY, "local potential not set (pw_set_vtot)");
  PWB_CHECK(ctx->have_k, PW_ENOTREADY, "Bloch vector not set (pw_set_kpoint)");
  PWB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int cap = std::max(ctx->pair_cap, 1);
  for (int b0 = 0; b0 < nband; b0 += cap) {
    const int nb = std::min(cap, nband - b0);
    int rc = run_hpsi_k(ctx, psi, ld, hpsi, ldh, b0, nb, accumulate, st);
    if (rc) return rc;
  }
  return PW_OK;
}

int pw_set_kpoints(pw_ctx* ctx, int nk, const double* kpts) {
  PWB_CHECK(ctx && nk > 0 && kpts, PW_EINVAL, "bad arguments");
  PWB_CHECK(!ctx->gs, PW_EUNSUPPORTED, "k-points are built for real-space contexts only");
  PWB_CUDA(cudaSetDevice(ctx->device));
  const long nt = ctx->ntot;
  const size_t esz = ctx->esz;
  const int np = (int)ctx->h_pnp.size();
  int rc;
  if ((rc = ctx->ekin_kb.alloc((size_t)nk * nt * esz))) return rc;
  if (np > 0 && (rc = ctx->qkb.alloc((size_t)nk * np * nt * 2 * esz))) return rc;
  const bool tc = kq_tensor_cores(ctx) && np > 0;
  for (int k = 0; k < nk; ++k) {
    if ((rc = pw_set_kpoint(ctx, kpts + 3 * k))) return rc;
    PWB_CUDA(cudaMemcpy((char*)ctx->ekin_kb.p + (size_t)k * nt * esz, ctx->ekin_k.p, nt * esz, cudaMemcpyDeviceToDevice));
    if (np > 0)
      PWB_CUDA(cudaMemcpy((char*)ctx->qkb.p + (size_t)k * np * nt * 2 * esz, ctx->qk.p, (size_t)np * nt * 2 * esz,
                          cudaMemcpyDeviceToDevice));
    if (tc) {
      const size_t per = kq_bf_bytes(ctx);
      if (k == 0 && (rc = ctx->qkb_bf.alloc((size_t)nk * per))) return rc;
      PWB_CUDA(cudaMemcpy((char*)ctx->qkb_bf.p + (size_t)k * per, ctx->qk_bf.p, per, cudaMemcpyDeviceToDevice));
    }
  }
  ctx->kb_k.assign(kpts, kpts + 3 * nk);
  ctx->nkb = nk;
  return PW_OK;
}

int pw_hpsi_kbatch(pw_ctx* ctx, const void* psi, int ld, void* hpsi, int ldh, int nband, int accumulate, void* stream) {
  PWB_CHECK(ctx && (nband == 0 || (psi && hpsi)), PW_EINVAL, "null argument");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot && ldh >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CHECK(ctx->have_vtot, PW_ENOTREADY, "local potential not set (pw_set_vtot)");
  PWB_CHECK(ctx->nkb > 0, PW_ENOTREADY, "k-point batch not set (pw_set_kpoints)");
  PWB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int cap = std::max(ctx->pair_cap, 1);
  const int nf = ctx->nkb * nband;
  for (int f0 = 0; f0 < nf; f0 += cap) {
    const int n = std::min(cap, nf - f0);
    int rc = run_hpsi_kbatch(ctx, psi, ld, hpsi, ldh, f0, n, accumulate, st, nband, ctx->ekin_kb.p,
                             ctx->nproj > 0 ? ctx->qkb.p : nullptr);
    if (rc) return rc;
  }
  return PW_OK;
}

int pw_get_kpoint_tables(const pw_ctx* ctx, double* ekin_host, double* teter_host) {
  PWB_CHECK(ctx && ctx->have_k, PW_ENOTREADY, "Bloch vector not set (pw_set_kpoint)");
  const long nt = ctx->ntot;
  for (int which = 0; which < 2; ++which) {
    double* dst = which == 0 ? ekin_host : teter_host;
    if (!dst) continue;
    const pwb::DevBuf& b = which == 0 ? ctx->ekin_k : ctx->teter_k;
    if (ctx->prec == PW_F64) {
      PWB_CUDA(cudaMemcpy(dst, b.p, nt * 8, cudaMemcpyDeviceToHost));
    } else {
      std::vector<float> h(nt);
      PWB_CUDA(cudaMemcpy(h.data(), b.p, nt * 4, cudaMemcpyDeviceToHost));
      for (long i = 0; i < nt; ++i) dst[i] = h[i];
    }
  }
  return PW_OK;
}

}  // extern "C"
