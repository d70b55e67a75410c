// Atomic forces, KohnSham::CalculateForce (src/SCF/hamiltonian.cpp:2670-3056),
// pseudocharge formulation, FP64 context.
//
//  * local (:2716-2800): F_a,d = w sum_{i in supp rho_ps,a} rho_ps,a(r_i) dV_H/dx_d(r_i),
//    dV_H/dx_d = IFFT(i G_d 2 pi / gkk FFT(rho - rho_ps)), gkk = |G|^2 / 2 (0 at G = 0),
//    w = vol / N_fine.  Three gradient components through the FP64 fine-grid
//    axis FFTs, then one CTA per atom gathers its pseudocharge support.
//  * nonlocal (:2907-3006, "Method 4"): the reference interpolates every band
//    and its three derivatives to the fine grid and integrates them against
//    the projectors.  Here the same quantity is formed on the coarse grid: with
//    q_l = T beta_l (the transpose of the coarse->fine interpolation applied to
//    the fine-grid projector) and tq_l,d = T (d_d beta_l) (the spectral
//    derivative taken inside the fine->coarse pipeline), the reference's
//    -2 f gamma res(VAL) res(D) numSpin equals
//        + 2 numSpin f gamma (vol / N_c) (q_l . psi)(tq_l,d . psi)
//    so the force is three coarse projector builds and four GEMMs with the
//    bands, and no per-band fine-grid FFT.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.hpp"
#include "fft3d.cuh"

namespace pwb {

int run_build_q(pw_ctx* c, const int* d_idx, const double* d_beta, const long* d_pio, const long* d_pbo,
                const int* d_pnp, int nproj, cudaStream_t st, int deriv, void* out);
int ensure_scratch(pw_ctx* c, int npair);
int run_density(pw_ctx* c, const void* psi, int ld, int nband, int band0, int npair, const double* w, double* rho,
                cudaStream_t st);

constexpr int FRC_THREADS = 256;

// block sum of three doubles; the result is valid in thread 0
__device__ __forceinline__ void block_sum3(double v[3], double* sh) {
  for (int d = 0; d < 3; ++d)
    for (int o = 16; o; o >>= 1) v[d] += __shfl_down_sync(0xffffffffu, v[d], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0)
    for (int d = 0; d < 3; ++d) sh[warp * 3 + d] = v[d];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) {
      double s = 0;
      for (int w = 0; w < nw; ++w) s += sh[w * 3 + d];
      v[d] = s;
    }
}

// F[a][d] = w sum_i val_i dv_d[idx_i] over the atom's pseudocharge support
__global__ void __launch_bounds__(FRC_THREADS)
k_force_local(const long* __restrict__ off, const int* __restrict__ idx, const double* __restrict__ val,
              const double* __restrict__ dv, long nf, double w, double* __restrict__ F) {
  __shared__ double sh[3 * FRC_THREADS / 32];
  const int a = blockIdx.x;
  double s[3] = {0, 0, 0};
  for (long i = off[a] + threadIdx.x; i < off[a + 1]; i += blockDim.x) {
    const long g = idx[i];
    const double v = val[i];
    s[0] += v * dv[g];
    s[1] += v * dv[nf + g];
    s[2] += v * dv[2 * nf + g];
  }
  block_sum3(s, sh);
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) F[a * 3 + d] = s[d] * w;
}

// F[a][d] += sum_{l in a} sum_b c_b g_l W[l][b] Wd[d][l][b]; W column-major np x nb
__global__ void __launch_bounds__(FRC_THREADS)
k_force_nl(const int* __restrict__ aoff, const double* __restrict__ W, const double* __restrict__ Wd, int np, int nb,
           const double* __restrict__ gl, const double* __restrict__ cb, double* __restrict__ F) {
  __shared__ double sh[3 * FRC_THREADS / 32];
  const int a = blockIdx.x;
  const int l0 = aoff[a], nl = aoff[a + 1] - l0;
  double s[3] = {0, 0, 0};
  for (int i = threadIdx.x; i < nl * nb; i += blockDim.x) {
    const int b = i / nl, l = l0 + (i - b * nl);
    const long e = (long)b * np + l;
    const double t = cb[b] * gl[l] * W[e];
    s[0] += t * Wd[e];
    s[1] += t * Wd[(long)np * nb + e];
    s[2] += t * Wd[2L * np * nb + e];
  }
  block_sum3(s, sh);
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) F[a * 3 + d] = s[d];
}

// d/dx_d of V_H[rho - rho_ps] on the fine grid for d = 0, 1, 2 into dv[d][nf]
template <int N>
static int grad_hartree_n(double2* work, const double* rho, const double* rps, const double* kern3, double* dv,
                          long nf, const double2* tw, cudaStream_t st) {
  const int nrowtiles = (N * N + AX_TILE - 1) / AX_TILE;
  const int nxt = (N + AX_TILE - 1) / AX_TILE;
  for (int d = 0; d < 3; ++d) {
    k_fft_axis<N, -1, 0, 1><<<nrowtiles, AX_THREADS, 0, st>>>(work, N, N, N, rho, rps, nullptr, nullptr, 1.0, tw);
    k_fft_axis<N, -1, 1, 0><<<dim3(nxt, N), AX_THREADS, 0, st>>>(work, N, N, N, nullptr, nullptr, nullptr, nullptr,
                                                                  1.0, tw);
    k_fft_axis<N, -1, 2, 4><<<dim3(nxt, N), AX_THREADS, 0, st>>>(work, N, N, N, nullptr, nullptr, kern3 + d * nf,
                                                                  nullptr, 1.0, tw);
    k_fft_axis<N, +1, 1, 0><<<dim3(nxt, N), AX_THREADS, 0, st>>>(work, N, N, N, nullptr, nullptr, nullptr, nullptr,
                                                                  1.0, tw);
    k_fft_axis<N, +1, 0, 3><<<nrowtiles, AX_THREADS, 0, st>>>(work, N, N, N, nullptr, nullptr, nullptr, dv + d * nf,
                                                               1.0, tw);
  }
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

static int grad_hartree(pw_ctx* c, double2* work, const double* rho, const double* rps, const double* kern3,
                        double* dv, const double2* tw, cudaStream_t st) {
  PWB_CHECK(c->nf[0] == c->nf[1] && c->nf[1] == c->nf[2], PW_EUNSUPPORTED, "forces need a cubic fine grid");
  const long nf = c->ntotf;
  switch (c->nf[0]) {
    case 24: return grad_hartree_n<24>(work, rho, rps, kern3, dv, nf, tw, st);
    case 32: return grad_hartree_n<32>(work, rho, rps, kern3, dv, nf, tw, st);
    case 48: return grad_hartree_n<48>(work, rho, rps, kern3, dv, nf, tw, st);
    case 96: return grad_hartree_n<96>(work, rho, rps, kern3, dv, nf, tw, st);
    case 144: return grad_hartree_n<144>(work, rho, rps, kern3, dv, nf, tw, st);
    default: set_error("fine grid size not built for the FP64 3-D FFT"); return PW_EUNSUPPORTED;
  }
}

template <typename X> static int upload(DevBuf& b, const std::vector<X>& h) {
  int rc = b.alloc(std::max<size_t>(h.size(), 1) * sizeof(X));
  if (rc) return rc;
  if (!h.empty()) PWB_CUDA(cudaMemcpy(b.p, h.data(), h.size() * sizeof(X), cudaMemcpyHostToDevice));
  return PW_OK;
}

static int local_part(pw_ctx* ctx, const double* rho, double* F_dev) {
  const long nf = ctx->ntotf;
  const int natom = (int)ctx->atom_z.size();
  const int N0 = ctx->nf[0], N1 = ctx->nf[1], N2 = ctx->nf[2];
  // i G_d 2 pi / gkk / N_fine, the whole spectrum (no energy cut-off)
  std::vector<double> k(3 * nf);
  for (int z = 0; z < N2; ++z)
    for (int y = 0; y < N1; ++y)
      for (int x = 0; x < N0; ++x) {
        const double m0 = x <= N0 / 2 ? x : x - N0, m1 = y <= N1 / 2 ? y : y - N1, m2 = z <= N2 / 2 ? z : z - N2;
        const double g[3] = {2 * M_PI / ctx->L[0] * m0, 2 * M_PI / ctx->L[1] * m1, 2 * M_PI / ctx->L[2] * m2};
        const double gkk = (g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) / 2;
        const double f = gkk == 0.0 ? 0.0 : 2.0 * M_PI / gkk / (double)nf;
        const size_t e = x + (size_t)N0 * (y + (size_t)N1 * z);
        for (int d = 0; d < 3; ++d) k[d * nf + e] = f * g[d];
      }
  std::vector<double> t(2 * N0);
  for (int m = 0; m < N0; ++m) {
    t[2 * m] = std::cos(2 * M_PI * m / N0);
    t[2 * m + 1] = -std::sin(2 * M_PI * m / N0);
  }
  DevBuf kern, work, tw, dv, rps, off, idx, val;
  int rc;
  if ((rc = upload(kern, k)) || (rc = upload(tw, t)) || (rc = upload(rps, ctx->h_rhops)) ||
      (rc = upload(off, ctx->h_ps_off)) || (rc = upload(idx, ctx->h_ps_idx)) || (rc = upload(val, ctx->h_ps_val)) ||
      (rc = work.alloc(nf * 16)) || (rc = dv.alloc(3 * nf * 8)))
    return rc;
  if ((rc = grad_hartree(ctx, (double2*)work.p, rho, (const double*)rps.p, (const double*)kern.p, (double*)dv.p,
                         (const double2*)tw.p, nullptr)))
    return rc;
  ctx->launches += 15;
  if (natom > 0) {
    k_force_local<<<natom, FRC_THREADS>>>((const long*)off.p, (const int*)idx.p, (const double*)val.p,
                                          (const double*)dv.p, nf, ctx->vol / (double)nf, F_dev);
    ctx->launches += 1;
  }
  PWB_CUDA(cudaGetLastError());
  PWB_CUDA(cudaDeviceSynchronize());
  return PW_OK;
}

// sum_{l in a} sum_b cb_b gamma_l (vol/N_c) (q_l . psi_b)(p_l,d . psi_b) into F_dev[a][d], where
// p_l,d = T(d_d beta_l) from the spectral derivative inside the fine->coarse
// pipeline (columns == false) or T applied to the projector's analytic
// derivative column DX/DY/DZ (columns == true, sets built by pw_set_atoms)
static int nl_contract(pw_ctx* ctx, const double* psi, int ld, int nb, const std::vector<double>& cb, bool columns,
                       double* F_dev) {
  const int np = (int)ctx->h_pnp.size();
  const int natom = (int)ctx->atom_z.size();
  const long nt = ctx->ntot;
  if (np == 0 || nb == 0 || natom == 0) {
    if (natom > 0) PWB_CUDA(cudaMemset(F_dev, 0, (size_t)natom * 3 * 8));
    return PW_OK;
  }
  // projectors of one atom are contiguous in the flattened order
  std::vector<int> aoff(natom + 1, 0);
  for (int l = 0; l < np; ++l) aoff[ctx->h_patom[l] + 1]++;
  for (int a = 0; a < natom; ++a) aoff[a + 1] += aoff[a];
  std::vector<double> gl(np);
  for (int l = 0; l < np; ++l) gl[l] = ctx->h_pgamma[l] * ctx->vol / (double)nt;
  std::vector<double> dcol[3];
  if (columns) {
    size_t tot = 0;
    for (const auto& a : ctx->h_nl) tot += a.val.size();
    PWB_CHECK(ctx->h_nl.size() == (size_t)natom && tot == (size_t)np, PW_ENOTREADY,
              "analytic projector derivatives need the sets of pw_set_atoms");
    for (int d = 0; d < 3; ++d) {
      dcol[d].reserve(ctx->h_nl_beta.size());
      for (const auto& a : ctx->h_nl)
        for (const auto& v : a.val)
          for (int g = 0; g < a.npts; ++g) dcol[d].push_back(v[4 * g + 1 + d]);
      PWB_CHECK(dcol[d].size() == ctx->h_nl_beta.size(), PW_EINVAL, "projector sets changed since pw_set_atoms");
    }
  }
  DevBuf d_idx, d_beta, d_pio, d_pbo, d_pnp, d_aoff, d_gl, d_cb, Qd, W, Wd, Qv, d_col;
  int rc;
  if ((rc = upload(d_idx, ctx->h_nl_idx)) || (rc = upload(d_beta, ctx->h_nl_beta)) || (rc = upload(d_pio, ctx->h_pio)) ||
      (rc = upload(d_pbo, ctx->h_pbo)) || (rc = upload(d_pnp, ctx->h_pnp)) || (rc = upload(d_aoff, aoff)) ||
      (rc = upload(d_gl, gl)) || (rc = upload(d_cb, cb)) || (rc = Qd.alloc((size_t)np * nt * 8)) ||
      (rc = W.alloc((size_t)np * nb * 8)) || (rc = Wd.alloc((size_t)3 * np * nb * 8)))
    return rc;
  if ((rc = ensure_scratch(ctx, std::max(ctx->pair_cap, 1)))) return rc;
  const double* Q = (const double*)ctx->q.p;
  if (ctx->nl_mode != PW_NL_DENSE || !ctx->have_nl) {
    // real-space projector mode keeps no coarse projector matrix: build one here
    if ((rc = Qv.alloc((size_t)np * nt * 8))) return rc;
    if ((rc = run_build_q(ctx, (const int*)d_idx.p, (const double*)d_beta.p, (const long*)d_pio.p,
                          (const long*)d_pbo.p, (const int*)d_pnp.p, np, nullptr, 0, Qv.p)))
      return rc;
    Q = (const double*)Qv.p;
  }
  cublasHandle_t h = (cublasHandle_t)ctx->blas;
  if (cublasSetStream(h, nullptr) != CUBLAS_STATUS_SUCCESS) { set_error("cublasSetStream failed"); return PW_ECUDA; }
  const double one = 1, zero = 0;
  if (cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, np, nb, (int)nt, &one, Q, (int)nt, psi, ld, &zero, (double*)W.p, np) !=
      CUBLAS_STATUS_SUCCESS) {
    set_error("projector GEMM failed");
    return PW_ECUDA;
  }
  ctx->lib_launches += 1;
  for (int d = 0; d < 3; ++d) {
    if (columns) {
      if ((rc = upload(d_col, dcol[d]))) return rc;
      rc = run_build_q(ctx, (const int*)d_idx.p, (const double*)d_col.p, (const long*)d_pio.p, (const long*)d_pbo.p,
                       (const int*)d_pnp.p, np, nullptr, 0, Qd.p);
    } else {
      rc = run_build_q(ctx, (const int*)d_idx.p, (const double*)d_beta.p, (const long*)d_pio.p, (const long*)d_pbo.p,
                       (const int*)d_pnp.p, np, nullptr, d + 1, Qd.p);
    }
    if (rc) return rc;
    if (cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, np, nb, (int)nt, &one, (const double*)Qd.p, (int)nt, psi, ld, &zero,
                    (double*)Wd.p + (size_t)d * np * nb, np) != CUBLAS_STATUS_SUCCESS) {
      set_error("derivative projector GEMM failed");
      return PW_ECUDA;
    }
    ctx->lib_launches += 1;
  }
  k_force_nl<<<natom, FRC_THREADS>>>((const int*)d_aoff.p, (const double*)W.p, (const double*)Wd.p, np, nb,
                                     (const double*)d_gl.p, (const double*)d_cb.p, F_dev);
  ctx->launches += 1;
  PWB_CUDA(cudaGetLastError());
  PWB_CUDA(cudaDeviceSynchronize());
  return PW_OK;
}

// sum_i w_b psi_b(i) y_b(i) per band, FP64 accumulation; one CTA per band
template <typename T>
__global__ void __launch_bounds__(FRC_THREADS)
k_band_dots(const T* __restrict__ x, int ldx, const T* __restrict__ y, int ldy, long n, double* __restrict__ out) {
  __shared__ double sh[3 * FRC_THREADS / 32];
  const int b = blockIdx.x;
  double s[3] = {0, 0, 0};
  for (long i = threadIdx.x; i < n; i += blockDim.x) s[0] += (double)x[(long)b * ldx + i] * (double)y[(long)b * ldy + i];
  block_sum3(s, sh);
  if (threadIdx.x == 0) out[b] = s[0];
}

}  // namespace pwb

using namespace pwb;

extern "C" {

int pw_forces(pw_ctx* ctx, const double* rho_dev, const void* psi_dev, int ldpsi, int nband, const double* occ,
              int num_spin, double* force, double* force_local, double* force_nonlocal) {
  PWB_CHECK(ctx && force, PW_EINVAL, "null argument");
  PWB_CHECK(!ctx->gs, PW_EUNSUPPORTED, "forces are built for real-space contexts only");
  PWB_CHECK(ctx->prec == PW_F64, PW_EINVAL, "forces take an FP64 context");
  PWB_CHECK(!ctx->atom_z.empty() && ctx->h_ps_off.size() == ctx->atom_z.size() + 1, PW_ENOTREADY,
            "atoms not set (pw_set_atoms)");
  PWB_CHECK(nband >= 0 && (nband == 0 || (psi_dev && occ && ldpsi >= ctx->ntot)), PW_EINVAL, "bad band arguments");
  PWB_CHECK(num_spin == 1 || num_spin == 2, PW_EINVAL, "num_spin must be 1 or 2");
  PWB_CHECK(rho_dev, PW_EINVAL, "null density");
  PWB_CUDA(cudaSetDevice(ctx->device));
  const int natom = (int)ctx->atom_z.size();
  for (int a : ctx->h_patom) PWB_CHECK(a < natom, PW_EINVAL, "projector sets do not match the atoms");
  DevBuf F;
  int rc;
  if ((rc = F.alloc((size_t)2 * natom * 3 * 8))) return rc;
  double* Floc = (double*)F.p;
  double* Fnl = Floc + natom * 3;
  PWB_CUDA(cudaMemset(F.p, 0, (size_t)2 * natom * 3 * 8));
  if ((rc = local_part(ctx, rho_dev, Floc))) return rc;
  std::vector<double> cb(nband);
  for (int b = 0; b < nband; ++b) cb[b] = 2.0 * num_spin * occ[b];
  if ((rc = nl_contract(ctx, (const double*)psi_dev, ldpsi, nband, cb, false, Fnl))) return rc;
  std::vector<double> h(2 * natom * 3);
  PWB_CUDA(cudaMemcpy(h.data(), F.p, h.size() * 8, cudaMemcpyDeviceToHost));
  for (int i = 0; i < natom * 3; ++i) force[i] = h[i] + h[natom * 3 + i];
  if (force_local) std::copy(h.begin(), h.begin() + natom * 3, force_local);
  if (force_nonlocal) std::copy(h.begin() + natom * 3, h.end(), force_nonlocal);
  return PW_OK;
}

int pw_band_energy(pw_ctx* ctx, const void* psi, int ld, int nband, const double* w, double* e) {
  PWB_CHECK(ctx && e && (nband == 0 || (psi && w)), PW_EINVAL, "null argument");
  PWB_CHECK(!ctx->gs, PW_EUNSUPPORTED, "the band-energy adjoint is built for real-space contexts only");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CUDA(cudaSetDevice(ctx->device));
  *e = 0.0;
  if (nband == 0) return PW_OK;
  const long nt = ctx->ntot;
  DevBuf hp, dd;
  int rc;
  if ((rc = hp.alloc((size_t)nband * nt * ctx->esz)) || (rc = dd.alloc((size_t)nband * 8))) return rc;
  if ((rc = pw_hpsi(ctx, psi, ld, hp.p, (int)nt, nband, 0, nullptr))) return rc;
  if (ctx->prec == PW_F64)
    k_band_dots<double><<<nband, FRC_THREADS>>>((const double*)psi, ld, (const double*)hp.p, (int)nt, nt, (double*)dd.p);
  else
    k_band_dots<float><<<nband, FRC_THREADS>>>((const float*)psi, ld, (const float*)hp.p, (int)nt, nt, (double*)dd.p);
  ctx->launches += 1;
  PWB_CUDA(cudaGetLastError());
  std::vector<double> h(nband);
  PWB_CUDA(cudaMemcpy(h.data(), dd.p, nband * 8, cudaMemcpyDeviceToHost));
  double s = 0;
  for (int b = 0; b < nband; ++b) s += w[b] * h[b];
  *e = s;
  return PW_OK;
}

int pw_band_energy_backward(pw_ctx* ctx, const void* psi, int ld, int nband, const double* w, double* dE_dV_dev,
                            double* dE_dR) {
  PWB_CHECK(ctx && (nband == 0 || (psi && w)), PW_EINVAL, "null argument");
  PWB_CHECK(!ctx->gs, PW_EUNSUPPORTED, "the band-energy adjoint is built for real-space contexts only");
  PWB_CHECK(nband >= 0 && ld >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CHECK(!dE_dR || ctx->prec == PW_F64, PW_EINVAL, "d/dR takes an FP64 context");
  PWB_CHECK(!dE_dR || !ctx->atom_z.empty(), PW_ENOTREADY, "atoms not set (pw_set_atoms)");
  PWB_CUDA(cudaSetDevice(ctx->device));
  int rc;
  if (dE_dV_dev) {
    // E = sum_b w_b <psi_b, T(V M psi_b)> = sum_r V(r) sum_b w_b (N_c/N_f) (M psi_b)(r)^2,
    // M the value-preserving coarse->fine interpolation, recomputed per batch
    PWB_CUDA(cudaMemset(dE_dV_dev, 0, ctx->ntotf * 8));
    if (nband > 0) {
      DevBuf wv;
      if ((rc = wv.alloc((size_t)(nband + 2) * 8))) return rc;
      std::vector<double> h(nband + 2, 0.0);
      for (int b = 0; b < nband; ++b) h[b] = w[b] * (double)ctx->ntot / (double)ctx->ntotf;
      PWB_CUDA(cudaMemcpy(wv.p, h.data(), h.size() * 8, cudaMemcpyHostToDevice));
      const int cap = ctx->pair_cap;
      for (int b0 = 0; b0 < nband; b0 += 2 * cap) {
        const int npair = std::min(cap, (nband - b0 + 1) / 2);
        if ((rc = run_density(ctx, psi, ld, nband, b0, npair, (const double*)wv.p, dE_dV_dev, nullptr))) return rc;
      }
      PWB_CUDA(cudaDeviceSynchronize());
    }
  }
  if (dE_dR) {
    const int natom = (int)ctx->atom_z.size();
    DevBuf F;
    if ((rc = F.alloc((size_t)natom * 3 * 8))) return rc;
    PWB_CUDA(cudaMemset(F.p, 0, (size_t)natom * 3 * 8));
    // E_nl = sum_b w_b sum_l D_l (q_l . psi_b)^2 with q_l = T beta_l(. - R_a):
    // dE/dR_a,d = -2 sum_b w_b sum_{l in a} D_l (q_l . psi_b)(T(d_d beta_l) . psi_b)
    std::vector<double> cb(nband);
    for (int b = 0; b < nband; ++b) cb[b] = -2.0 * w[b];
    if ((rc = nl_contract(ctx, (const double*)psi, ld, nband, cb, true, (double*)F.p))) return rc;
    PWB_CUDA(cudaMemcpy(dE_dR, F.p, (size_t)natom * 3 * 8, cudaMemcpyDeviceToHost));
  }
  return PW_OK;
}

int pw_scf_state(const pw_ctx* ctx, int* nband, double* occ, double* psi_dev, int ldpsi, double* rho_dev) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  PWB_CHECK(ctx->scf_nband > 0, PW_ENOTREADY, "no FP64 SCF state (run pw_scf_run to the FP64 stage first)");
  const int nb = ctx->scf_nband;
  if (nband) *nband = nb;
  if (occ) std::copy(ctx->scf_occ.begin(), ctx->scf_occ.end(), occ);
  if (psi_dev) {
    PWB_CHECK(ldpsi >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
    PWB_CUDA(cudaMemcpy2D(psi_dev, (size_t)ldpsi * 8, ctx->scf_psi.p, (size_t)ctx->ntot * 8, (size_t)ctx->ntot * 8, nb,
                          cudaMemcpyDeviceToDevice));
  }
  if (rho_dev) PWB_CUDA(cudaMemcpy(rho_dev, ctx->scf_rho.p, ctx->ntotf * 8, cudaMemcpyDeviceToDevice));
  return PW_OK;
}

int pw_scf_forces(pw_ctx* ctx, double* force, double* force_local, double* force_nonlocal) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  PWB_CHECK(!ctx->gs, PW_EUNSUPPORTED, "forces are built for real-space contexts only");
  PWB_CHECK(ctx->scf_nband > 0, PW_ENOTREADY, "no FP64 SCF state (run pw_scf_run to the FP64 stage first)");
  return pw_forces(ctx, (const double*)ctx->scf_rho.p, ctx->scf_psi.p, (int)ctx->ntot, ctx->scf_nband,
                   ctx->scf_occ.data(), 2, force, force_local, force_nonlocal);
}

}  // extern "C"
