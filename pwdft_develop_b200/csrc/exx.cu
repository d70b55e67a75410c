// Hybrid exact exchange on the coarse grid (Gamma point, real bands):
//
//  * Coulomb kernel      KohnSham::InitializeEXX   src/SCF/hamiltonian.cpp:3454-3551
//                        (divergence type 0 / 1, optional erfc screening mu)
//  * exchange orbitals   KohnSham::SetPhiEXX       hamiltonian.cpp:3554-3641
//                        (phi = sqrt(N_c / vol) psi, every state incl. empty ones)
//  * V_x psi             Spinor::AddMultSpinorEXX  src/SCF/spinor.cpp:682-781
//                        (pair-field kernels in hpsi.cu)
//  * ACE                 KohnSham::CalculateVexxACE hamiltonian.cpp:3686-3818:
//                        W = V_x psi, M = -psi^T W, M = L L^T, xi = W L^-T;
//                        applied in MultSpinor as a3 -= xi (xi^T psi) (:3135-3218)
//  * exchange energy     KohnSham::CalculateEXXEnergy hamiltonian.cpp:3936-4192
//                        E_x = numSpin / 2 * sum_j f_j psi_j^T (V_x psi_j)
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "blockops.hpp"
#include "common.hpp"
#include "gemm.hpp"

namespace pwb {

int run_exx(pw_ctx* c, const void* psi, int ld, int nb, void* out, int ldo, int acc, cudaStream_t st);
int run_ace(pw_ctx* c, const void* psi, int ld, int nb, void* out, int ldo, cudaStream_t st);
int gram(pw_ctx* c, const void* X, int ldx, int nx, const void* Y, int ldy, int ny, double* G, int ldg,
         cudaStream_t st, int nrow = -1);
int upload_real(pw_ctx* c, DevBuf& dst, const double* src, size_t n);

template <typename T>
__global__ void k_exx_scale_copy(long n, const T* __restrict__ x, long ldx, int nb, T s, T* __restrict__ y) {
  const long tot = n * nb;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {
    const long b = i / n, r = i - b * n;
    y[i] = s * x[b * ldx + r];
  }
}

template <typename T>
__global__ void k_exx_band_dots(const T* __restrict__ x, int ldx, const T* __restrict__ y, long n,
                                double* __restrict__ out) {
  __shared__ double sh[32];
  const int b = blockIdx.x;
  double s = 0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) s += (double)x[(long)b * ldx + i] * (double)y[(long)b * n + i];
  for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    out[b] = t;
  }
}

static int check_ready(const pw_ctx* ctx) {
  PWB_CHECK(ctx->exx_kern.p, PW_ENOTREADY, "exchange kernel not set (pw_exx_setup)");
  return PW_OK;
}

}  // namespace pwb

using namespace pwb;

extern "C" {

int pw_exx_setup(pw_ctx* ctx, double exx_fraction, double screen_mu, int divergence_type, double ecut_wavefunction) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  PWB_CHECK(divergence_type == 0 || divergence_type == 1, PW_EUNSUPPORTED,
            "EXX divergence types 0 and 1 are built (EXX_Divergence_Type)");
  PWB_CHECK(screen_mu >= 0.0 && ecut_wavefunction > 0.0, PW_EINVAL, "bad exchange parameters");
  PWB_CUDA(cudaSetDevice(ctx->device));
  if (ctx->gs) {
    int rc = gs_exx_setup(ctx, exx_fraction, screen_mu, divergence_type, ecut_wavefunction);
    if (rc) return rc;
    if (ctx->exx_nphi > 0 && !ctx->exx_occ.empty()) {
      std::vector<double> w(ctx->exx_nphi);
      for (int j = 0; j < ctx->exx_nphi; ++j) w[j] = -exx_fraction * ctx->exx_occ[j];
      if ((rc = upload_real(ctx, ctx->exx_w, w.data(), w.size()))) return rc;
    }
    return PW_OK;
  }
  const int n0 = ctx->n[0], n1 = ctx->n[1], n2 = ctx->n[2];
  const long nt = ctx->ntot;
  const double eps_div = 1e-8;
  const double alpha = 10.0 / (ecut_wavefunction * 2.0);
  const double mu = screen_mu;
  std::vector<double> g2(nt);
  for (int z = 0; z < n2; ++z)
    for (int y = 0; y < n1; ++y)
      for (int x = 0; x < n0; ++x) {
        const double m0 = x <= n0 / 2 ? x : x - n0, m1 = y <= n1 / 2 ? y : y - n1, m2 = z <= n2 / 2 ? z : z - n2;
        const double a = 2 * M_PI / ctx->L[0] * m0, b = 2 * M_PI / ctx->L[1] * m1, c = 2 * M_PI / ctx->L[2] * m2;
        g2[x + (long)n0 * (y + (long)n1 * z)] = a * a + b * b + c * c;
      }
  double div = 0.0;
  if (divergence_type == 1) {
    // auxiliary-function treatment of the G = 0 singularity (hamiltonian.cpp:3479-3517)
    for (long i = 0; i < nt; ++i) {
      const double q = g2[i];
      if (q > eps_div) {
        if (mu > 0.0) div += std::exp(-alpha * q) / q * (1.0 - std::exp(-q / (4.0 * mu * mu)));
        else div += std::exp(-alpha * q) / q;
      }
    }
    if (mu > 0.0) div += 1.0 / (4.0 * mu * mu);
    else div -= alpha;
    div *= 4.0 * M_PI;
    const double aa = mu > 0.0 ? 1.0 / std::sqrt(alpha * M_PI) - 1.0 / std::sqrt(M_PI * (alpha + 1.0 / (4.0 * mu * mu)))
                               : 1.0 / std::sqrt(alpha * M_PI);
    div -= ctx->vol * aa;
  }
  std::vector<double> k(nt);
  for (long i = 0; i < nt; ++i) {
    const double q = g2[i];
    if (q > eps_div) {
      k[i] = mu > 0.0 ? 4.0 * M_PI / q * (1.0 - std::exp(-q / (4.0 * mu * mu))) : 4.0 * M_PI / q;
    } else {
      k[i] = -div;
      if (mu > 0.0) k[i] += M_PI / (mu * mu);
    }
  }
  int rc = upload_real(ctx, ctx->exx_kern, k.data(), nt);
  if (rc) return rc;
  ctx->exx_frac = exx_fraction;
  ctx->exx_mu = mu;
  ctx->exx_div = div;
  if (ctx->exx_nphi > 0 && !ctx->exx_occ.empty()) {
    std::vector<double> w(ctx->exx_nphi);
    for (int j = 0; j < ctx->exx_nphi; ++j) w[j] = -exx_fraction * ctx->exx_occ[j];
    if ((rc = upload_real(ctx, ctx->exx_w, w.data(), w.size()))) return rc;
  }
  return PW_OK;
}

int pw_exx_get(const pw_ctx* ctx, double* exx_div, double* kern_host) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  int rc = check_ready(ctx);
  if (rc) return rc;
  if (exx_div) *exx_div = ctx->exx_div;
  if (kern_host) {
    const long nt = ctx->gs ? ctx->ntotf : ctx->ntot;   // G-space: the full N^3 grid
    if (ctx->prec == PW_F64) {
      PWB_CUDA(cudaMemcpy(kern_host, ctx->exx_kern.p, nt * 8, cudaMemcpyDeviceToHost));
    } else {
      std::vector<float> h(nt);
      PWB_CUDA(cudaMemcpy(h.data(), ctx->exx_kern.p, nt * 4, cudaMemcpyDeviceToHost));
      for (long i = 0; i < nt; ++i) kern_host[i] = h[i];
    }
  }
  return PW_OK;
}

int pw_exx_set_phi(pw_ctx* ctx, const void* psi, int ld, int nphi, const double* occ) {
  PWB_CHECK(ctx && nphi >= 0 && (nphi == 0 || (psi && occ)), PW_EINVAL, "bad arguments");
  PWB_CHECK(nphi == 0 || ld >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CUDA(cudaSetDevice(ctx->device));
  const long nt = ctx->ntot;
  int rc;
  ctx->exx_nphi = 0;
  ctx->gsx_phi_ready = false;
  ctx->exx_occ.assign(occ, occ + nphi);
  if (nphi == 0) return PW_OK;
  if ((rc = ctx->exx_phi.alloc((size_t)nphi * nt * ctx->esz))) return rc;
  // SetPhiEXX (hamiltonian.cpp:3568-3580, 3598-3612): sqrt(N_c / vol) for
  // real-space bands, sqrt(1 / (vol N)) for sphere coefficients
  const double fac = ctx->gs ? std::sqrt(1.0 / (ctx->vol * (double)ctx->ntotf)) : std::sqrt((double)nt / ctx->vol);
  const int nblk = (int)std::min<long>(4096, ((long)nphi * nt + 255) / 256);
  if (ctx->prec == PW_F64)
    k_exx_scale_copy<double><<<nblk, 256>>>(nt, (const double*)psi, ld, nphi, fac, (double*)ctx->exx_phi.p);
  else
    k_exx_scale_copy<float><<<nblk, 256>>>(nt, (const float*)psi, ld, nphi, (float)fac, (float*)ctx->exx_phi.p);
  ctx->launches += 1;
  PWB_CUDA(cudaGetLastError());
  std::vector<double> w(nphi);
  for (int j = 0; j < nphi; ++j) w[j] = -ctx->exx_frac * occ[j];
  if ((rc = upload_real(ctx, ctx->exx_w, w.data(), nphi))) return rc;
  PWB_CUDA(cudaDeviceSynchronize());
  ctx->exx_nphi = nphi;
  return PW_OK;
}

int pw_exx_set_scratch(pw_ctx* ctx, size_t bytes) {
  PWB_CHECK(ctx && bytes > 0, PW_EINVAL, "bad arguments");
  ctx->exx_scratch_bytes = bytes;
  ctx->s_exx.release();
  return PW_OK;
}

int pw_exx_set_mode(pw_ctx* ctx, int mode) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  PWB_CHECK(mode == PW_EXX_OFF || mode == PW_EXX_FULL || mode == PW_EXX_ACE, PW_EINVAL, "unknown exchange mode");
  if (mode != PW_EXX_OFF) {
    int rc = check_ready(ctx);
    if (rc) return rc;
  }
  ctx->exx_mode = mode;
  return PW_OK;
}

int pw_exx_apply(pw_ctx* ctx, const void* psi, int ld, void* out, int ldo, int nband, int accumulate, void* stream) {
  PWB_CHECK(ctx && (nband == 0 || (psi && out)), PW_EINVAL, "null argument");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot && ldo >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  int rc = check_ready(ctx);
  if (rc) return rc;
  PWB_CUDA(cudaSetDevice(ctx->device));
  if (nband == 0) return PW_OK;
  return run_exx(ctx, psi, ld, nband, out, ldo, accumulate ? 1 : 0, (cudaStream_t)stream);
}

int pw_ace_build(pw_ctx* ctx, const void* psi, int ld, int nband) {
  PWB_CHECK(ctx && psi && nband > 0, PW_EINVAL, "bad arguments");
  PWB_CHECK(ld >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  int rc = check_ready(ctx);
  if (rc) return rc;
  PWB_CUDA(cudaSetDevice(ctx->device));
  const long nt = ctx->ntot;
  const size_t esz = ctx->esz;
  DevBuf W, M, Ui, X;
  if ((rc = W.alloc((size_t)nband * nt * esz)) || (rc = M.alloc((size_t)nband * nband * 8)) ||
      (rc = Ui.alloc((size_t)nband * nband * 8)))
    return rc;
  // W = V_x psi
  if ((rc = run_exx(ctx, psi, ld, nband, W.p, (int)nt, 0, nullptr))) return rc;
  // M = -psi^T W, symmetrised
  if ((rc = gram(ctx, psi, ld, nband, W.p, (int)nt, nband, (double*)M.p, nband, nullptr))) return rc;
  std::vector<double> h((size_t)nband * nband);
  PWB_CUDA(cudaMemcpy(h.data(), M.p, h.size() * 8, cudaMemcpyDeviceToHost));
  for (int j = 0; j < nband; ++j)
    for (int i = 0; i <= j; ++i) {
      const double v = -0.5 * (h[(size_t)j * nband + i] + h[(size_t)i * nband + j]);
      h[(size_t)j * nband + i] = v;
      h[(size_t)i * nband + j] = v;
    }
  PWB_CUDA(cudaMemcpy(M.p, h.data(), h.size() * 8, cudaMemcpyHostToDevice));
  // M = U^T U (U = L^T); xi = W L^-T = W U^-1
  Dense dn;
  if ((rc = dn.init((cublasHandle_t)ctx->blas))) return rc;
  if ((rc = dn.potrf_upper(nband, (double*)M.p, nband, nullptr))) {
    set_error("ACE: -psi^T V_x psi is not positive definite");
    dn.release();
    return PW_ENUMERIC;
  }
  if ((rc = dense_trtri_upper(nband, (const double*)M.p, nband, (double*)Ui.p, nband, nullptr))) return rc;
  dn.release();
  if ((rc = ctx->ace_xi.alloc((size_t)nband * nt * esz))) return rc;
  RotBlock rb{W.p, nt, nband, (const double*)Ui.p, nband};
  if ((rc = rotate(ctx, (int)nt, nband, &rb, 1, ctx->ace_xi.p, nt, 0.0, nullptr, true))) return rc;
  std::vector<double> m1(nband, -1.0);
  if ((rc = upload_real(ctx, ctx->ace_qd, m1.data(), nband))) return rc;
  const int npad = (nband + 7) / 8 * 8;
  if (ctx->prec == PW_F32) {
    // rows of xi padded to a multiple of 8 (16-byte TMA strides; the tensor
    // maps cover K = nt, so the pad is never read), as the projector matrix
    const long ntp = (nt + 7) / 8 * 8;
    if ((rc = ctx->ace_bf.alloc((size_t)2 * nband * ntp * 2)) || (rc = ctx->ace_t_bf.alloc((size_t)2 * nt * npad * 2)))
      return rc;
    PWB_CUDA(cudaMemset(ctx->ace_t_bf.p, 0, (size_t)2 * nt * npad * 2));
    char* b = (char*)ctx->ace_bf.p;
    char* bt = (char*)ctx->ace_t_bf.p;
    if ((rc = split_bf16((const float*)ctx->ace_xi.p, nt, (int)nt, nband, b, b + (size_t)nband * ntp * 2, ntp, 1.0f,
                         nullptr)))
      return rc;
    if ((rc = split_bf16_t((const float*)ctx->ace_xi.p, nt, (int)nt, nband, bt, bt + (size_t)nt * npad * 2, npad,
                           nullptr)))
      return rc;
  }
  PWB_CUDA(cudaDeviceSynchronize());
  ctx->ace_n = nband;
  ctx->ace_npad = npad;
  ++ctx->ace_version;
  ctx->exx_mode = PW_EXX_ACE;
  return PW_OK;
}

int pw_ace_apply(pw_ctx* ctx, const void* psi, int ld, void* out, int ldo, int nband, void* stream) {
  PWB_CHECK(ctx && (nband == 0 || (psi && out)), PW_EINVAL, "null argument");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot && ldo >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CHECK(ctx->ace_n > 0, PW_ENOTREADY, "ACE operator not built (pw_ace_build)");
  PWB_CUDA(cudaSetDevice(ctx->device));
  if (nband == 0) return PW_OK;
  const int cap = std::max(1, 2 * ctx->pair_cap);
  for (int b0 = 0; b0 < nband; b0 += cap) {
    const int nb = std::min(cap, nband - b0);
    const size_t e = ctx->esz;
    int rc = run_ace(ctx, (const char*)psi + (size_t)b0 * ld * e, ld, nb, (char*)out + (size_t)b0 * ldo * e, ldo,
                     (cudaStream_t)stream);
    if (rc) return rc;
  }
  return PW_OK;
}

int pw_exx_energy(pw_ctx* ctx, const void* psi, int ld, int nband, const double* occ, int num_spin, int use_ace,
                  double* e) {
  PWB_CHECK(ctx && e && (nband == 0 || (psi && occ)), PW_EINVAL, "null argument");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CHECK(num_spin == 1 || num_spin == 2, PW_EINVAL, "num_spin must be 1 or 2");
  int rc = check_ready(ctx);
  if (rc) return rc;
  PWB_CUDA(cudaSetDevice(ctx->device));
  *e = 0.0;
  if (nband == 0) return PW_OK;
  const long nt = ctx->ntot;
  DevBuf W, d;
  if ((rc = W.alloc((size_t)nband * nt * ctx->esz)) || (rc = d.alloc((size_t)nband * 8))) return rc;
  if (use_ace) {
    PWB_CHECK(ctx->ace_n > 0, PW_ENOTREADY, "ACE operator not built (pw_ace_build)");
    // V_x psi ~ -xi (xi^T psi)
    PWB_CUDA(cudaMemset(W.p, 0, (size_t)nband * nt * ctx->esz));
    if ((rc = pw_ace_apply(ctx, psi, ld, W.p, (int)nt, nband, nullptr))) return rc;
  } else {
    if ((rc = run_exx(ctx, psi, ld, nband, W.p, (int)nt, 0, nullptr))) return rc;
  }
  if (ctx->prec == PW_F64)
    k_exx_band_dots<double><<<nband, 256>>>((const double*)psi, ld, (const double*)W.p, nt, (double*)d.p);
  else
    k_exx_band_dots<float><<<nband, 256>>>((const float*)psi, ld, (const float*)W.p, nt, (double*)d.p);
  ctx->launches += 1;
  PWB_CUDA(cudaGetLastError());
  std::vector<double> h(nband);
  PWB_CUDA(cudaMemcpy(h.data(), d.p, nband * 8, cudaMemcpyDeviceToHost));
  double s = 0.0;
  for (int j = 0; j < nband; ++j) s += occ[j] * h[j];
  *e = s * num_spin / 2.0;
  return PW_OK;
}

}  // extern "C"
