// Exact exchange in the sphere-cut (G-space) mode, FP64 or FP32: the complex
// overload of Spinor::AddMultSpinorEXX (src/SCF/spinor.cpp:783-945) with the
// kernel of KohnSham::InitializeEXX for a sphere cut (src/SCF/hamiltonian.cpp:
// 3454-3551) on the Fock set of Fourier::InitializeSphere
// (src/SCF/fourier.cpp:642-666).
//
// Bands and exchange orbitals are sphere coefficients (the real view of
// pw_ctx_create_gspace); phi = sqrt(1 / (vol N)) psi (SetPhiEXX,
// hamiltonian.cpp:3568-3580).  Per call:
//   psi(r), phi(r)   unnormalised inverse transforms on the full N^3 G-space
//                    grid (c_0 at G = 0, c_s / sqrt(2) at +-G_s), two bands per
//                    complex field;
//   V_x psi_k (r)    = sum_j -alpha f_j phi_j(r) (1/N) IFFT(v FFT(psi_k phi_j))(r),
//                    v(G) = 4 pi / |G|^2 (times 1 - exp(-|G|^2 / 4 mu^2)) on the
//                    Fock set 1/2 |G|^2 < 4 Ecut, -exxDiv (+ pi / mu^2) at G = 0,
//                    zero outside; two orbitals per complex pair field (v is real
//                    and even), a batch of pair fields per launch of the axis FFTs;
//   out_s           (+)= f_s FFT(V_x psi_k)(G_s), f_0 = 1, f_s = sqrt(2), two
//                    bands per complex field, unpacked at G_s and -G_s.
#include <cmath>
#include <vector>

#include "common.hpp"
#include "fft3d.cuh"

namespace pwb {

int upload_real(pw_ctx* c, DevBuf& dst, const double* src, size_t n);   // ctx.cu

template <typename T> using VT = typename C2<T>::t;

namespace {

// sphere -> full spectrum of band pairs: Z(G_s) = a + i b, Z(-G_s) = conj(a) + i conj(b)
template <typename T>
__global__ void k_gsx_scatter(const T* __restrict__ psi, int ld, int nb, int b0, int npair,
                              const int2* __restrict__ gidx, int ns, T scale, long n3, VT<T>* __restrict__ Z) {
  using V = VT<T>;
  const long tot = (long)npair * ns;
  const T r2 = (T)0.70710678118654752440;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int p = (int)(t / ns), s = (int)(t - (long)p * ns);
    const int ba = b0 + 2 * p, bb = ba + 1;
    const T f = scale * (s == 0 ? (T)1 : r2);
    V a = mkc<V>(f * psi[(long)ba * ld + 2 * s], f * psi[(long)ba * ld + 2 * s + 1]);
    V b = mkc<V>(0, 0);
    if (bb < nb) b = mkc<V>(f * psi[(long)bb * ld + 2 * s], f * psi[(long)bb * ld + 2 * s + 1]);
    if (s == 0) { a.y = 0; b.y = 0; }
    V* zp = Z + (long)p * n3;
    const int2 g = gidx[s];
    zp[g.x] = mkc<V>(a.x - b.y, a.y + b.x);
    zp[g.y] = mkc<V>(a.x + b.y, b.x - a.y);
  }
}

// real and imaginary parts of pair fields -> bands b0 + 2p, b0 + 2p + 1
template <typename T>
__global__ void k_gsx_unpack(const VT<T>* __restrict__ Z, int npair, long n3, int b0, int nb, T* __restrict__ R) {
  const long tot = (long)npair * n3;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int p = (int)(t / n3);
    const long r = t - (long)p * n3;
    const VT<T> v = Z[t];
    const int ba = b0 + 2 * p;
    R[(long)ba * n3 + r] = v.x;
    if (ba + 1 < nb) R[(long)(ba + 1) * n3 + r] = v.y;
  }
}

// pair fields of bands k0 .. k0 + kb - 1: F[kk * njp + jp] = psi_k (phi_2jp + i phi_2jp+1) / N
template <typename T>
__global__ void k_gsx_product(const T* __restrict__ psi_r, const T* __restrict__ phi_r, int k0, int kb,
                              int njp, int nphi, long n3, T inv_n, VT<T>* __restrict__ F) {
  const long tot = (long)kb * njp * n3;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const long f = t / n3, r = t - f * n3;
    const int kk = (int)(f / njp), jp = (int)(f - (long)kk * njp);
    const int ja = 2 * jp, jb = ja + 1;
    const T p = psi_r[(long)(k0 + kk) * n3 + r] * inv_n;
    F[t] = mkc<VT<T>>(p * phi_r[(long)ja * n3 + r], jb < nphi ? p * phi_r[(long)jb * n3 + r] : (T)0);
  }
}

// acc_k(r) += sum_jp w_ja phi_ja(r) Re F + w_jb phi_jb(r) Im F
template <typename T>
__global__ void k_gsx_accumulate(const VT<T>* __restrict__ F, const T* __restrict__ phi_r,
                                 const T* __restrict__ w, int k0, int kb, int njp, int nphi, long n3,
                                 T* __restrict__ acc) {
  const long tot = (long)kb * n3;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int kk = (int)(t / n3);
    const long r = t - (long)kk * n3;
    T s = 0;
    for (int jp = 0; jp < njp; ++jp) {
      const VT<T> v = F[((long)kk * njp + jp) * n3 + r];
      const int ja = 2 * jp, jb = ja + 1;
      s += w[ja] * phi_r[(long)ja * n3 + r] * v.x;
      if (jb < nphi) s += w[jb] * phi_r[(long)jb * n3 + r] * v.y;
    }
    acc[(long)(k0 + kk) * n3 + r] += s;
  }
}

// bands b0 + 2p, b0 + 2p + 1 of acc -> complex pair fields
template <typename T>
__global__ void k_gsx_pack(const T* __restrict__ acc, int b0, int nb, int npair, long n3, VT<T>* __restrict__ Z) {
  const long tot = (long)npair * n3;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int p = (int)(t / n3);
    const long r = t - (long)p * n3;
    const int ba = b0 + 2 * p;
    Z[t] = mkc<VT<T>>(acc[(long)ba * n3 + r], ba + 1 < nb ? acc[(long)(ba + 1) * n3 + r] : (T)0);
  }
}

// spectrum of a band pair -> sphere: a = (Y(G) + conj Y(-G)) / 2, b = (Y(G) - conj Y(-G)) / 2i
template <typename T>
__global__ void k_gsx_gather(const VT<T>* __restrict__ Z, int npair, long n3, const int2* __restrict__ gidx, int ns,
                             int b0, int nb, T* __restrict__ out, int ldo, int accumulate) {
  using V = VT<T>;
  const long tot = (long)npair * ns;
  const T sq2 = (T)1.41421356237309504880;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int p = (int)(t / ns), s = (int)(t - (long)p * ns);
    const V* zp = Z + (long)p * n3;
    const int2 g = gidx[s];
    const V y = zp[g.x], ym = zp[g.y];
    const T f = s == 0 ? (T)1 : sq2;
    V a = mkc<V>((T)0.5 * f * (y.x + ym.x), (T)0.5 * f * (y.y - ym.y));
    V b = mkc<V>((T)0.5 * f * (y.y + ym.y), (T)0.5 * f * (ym.x - y.x));
    if (s == 0) { a.y = 0; b.y = 0; }
    const int ba = b0 + 2 * p, bb = ba + 1;
    T* oa = out + (long)ba * ldo + 2 * s;
    if (accumulate) { oa[0] += a.x; oa[1] += a.y; } else { oa[0] = a.x; oa[1] = a.y; }
    if (bb < nb) {
      T* ob = out + (long)bb * ldo + 2 * s;
      if (accumulate) { ob[0] += b.x; ob[1] += b.y; } else { ob[0] = b.x; ob[1] = b.y; }
    }
  }
}

inline int gs_blocks(long n) { return (int)std::min<long>((n + 255) / 256, 148L * 16); }

// F complex N^3 fields back to back: mode 0 forward, 1 inverse, 2 convolution with kern
template <typename T, int N>
int fft3_fields(VT<T>* d, int F, int mode, const T* kern, const VT<T>* tw, cudaStream_t st) {
  const int nxt = (N + AX_TILE - 1) / AX_TILE;
  const int rows = (int)(((long)N * N * F + AX_TILE - 1) / AX_TILE);
  const T one = 1;
  if (mode == 1) {
    k_fft_axis<N, +1, 2, 0, T><<<dim3(nxt, N, F), AX_THREADS, 0, st>>>(d, N, N, N, nullptr, nullptr, nullptr, nullptr, one, tw);
    k_fft_axis<N, +1, 1, 0, T><<<dim3(nxt, N * F), AX_THREADS, 0, st>>>(d, N, N, N * F, nullptr, nullptr, nullptr, nullptr, one, tw);
    k_fft_axis<N, +1, 0, 0, T><<<rows, AX_THREADS, 0, st>>>(d, N, N, N * F, nullptr, nullptr, nullptr, nullptr, one, tw);
  } else {
    k_fft_axis<N, -1, 0, 0, T><<<rows, AX_THREADS, 0, st>>>(d, N, N, N * F, nullptr, nullptr, nullptr, nullptr, one, tw);
    k_fft_axis<N, -1, 1, 0, T><<<dim3(nxt, N * F), AX_THREADS, 0, st>>>(d, N, N, N * F, nullptr, nullptr, nullptr, nullptr, one, tw);
    if (mode == 0) {
      k_fft_axis<N, -1, 2, 0, T><<<dim3(nxt, N, F), AX_THREADS, 0, st>>>(d, N, N, N, nullptr, nullptr, nullptr, nullptr, one, tw);
    } else {
      k_fft_axis<N, -1, 2, 2, T><<<dim3(nxt, N, F), AX_THREADS, 0, st>>>(d, N, N, N, nullptr, nullptr, kern, nullptr, one, tw);
      k_fft_axis<N, +1, 1, 0, T><<<dim3(nxt, N * F), AX_THREADS, 0, st>>>(d, N, N, N * F, nullptr, nullptr, nullptr, nullptr, one, tw);
      k_fft_axis<N, +1, 0, 0, T><<<rows, AX_THREADS, 0, st>>>(d, N, N, N * F, nullptr, nullptr, nullptr, nullptr, one, tw);
    }
  }
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

template <typename T>
int fft3_fields_n(int N, VT<T>* d, int F, int mode, const T* kern, const VT<T>* tw, cudaStream_t st) {
  switch (N) {
    case 24: return fft3_fields<T, 24>(d, F, mode, kern, tw, st);
    case 32: return fft3_fields<T, 32>(d, F, mode, kern, tw, st);
    case 48: return fft3_fields<T, 48>(d, F, mode, kern, tw, st);
    case 96: return fft3_fields<T, 96>(d, F, mode, kern, tw, st);
    case 144: return fft3_fields<T, 144>(d, F, mode, kern, tw, st);
    default: set_error("G-space exact exchange: grid size not built (24, 32, 48, 96, 144)"); return PW_EUNSUPPORTED;
  }
}

// sphere bands (real view, ld) -> real fields [nb][N^3] through pair fields of at most cap pairs
template <typename T>
int gs_to_real(pw_ctx* c, const T* psi, int ld, int nb, T scale, T* R, VT<T>* Z, int cap, cudaStream_t st) {
  const int N = c->nf[0];
  const long n3 = (long)N * N * N;
  for (int b0 = 0; b0 < nb; b0 += 2 * cap) {
    const int np = std::min(cap, (nb - b0 + 1) / 2);
    PWB_CUDA(cudaMemsetAsync(Z, 0, (size_t)np * n3 * sizeof(VT<T>), st));
    k_gsx_scatter<T><<<gs_blocks((long)np * c->gs_ns), 256, 0, st>>>(psi, ld, nb, b0, np,
                                                                     (const int2*)c->gs_full_idx.p, (int)c->gs_ns,
                                                                     scale, n3, Z);
    int rc = fft3_fields_n<T>(N, Z, np, 1, nullptr, (const VT<T>*)c->gs_exx_tw.p, st);
    if (rc) return rc;
    k_gsx_unpack<T><<<gs_blocks((long)np * n3), 256, 0, st>>>(Z, np, n3, b0, nb, R);
    c->launches += 5;
  }
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

// out (+)= V_x psi for nb sphere bands
template <typename T>
int gs_exx_apply_t(pw_ctx* c, const T* psi, int ld, int nb, T* out, int ldo, int accumulate, cudaStream_t st) {
  using V = VT<T>;
  const int N = c->nf[0];
  const long n3 = (long)N * N * N;
  const int nphi = c->exx_nphi;
  if (nphi == 0) {
    if (!accumulate) PWB_CUDA(cudaMemset2DAsync(out, (size_t)ldo * sizeof(T), 0, (size_t)c->ntot * sizeof(T), nb, st));
    return PW_OK;
  }
  const int njp = (nphi + 1) / 2;
  // fields per batch from the scratch budget (at least one band's pair fields)
  // (gridDim.y of the axis-1 pass is N * fields: at most 65535)
  const long fmax = 65535 / N;
  PWB_CHECK(njp <= fmax, PW_EUNSUPPORTED, "G-space exact exchange: too many exchange orbitals for one band batch");
  const long fcap = std::min<long>(fmax, std::max<long>(njp, (long)(c->exx_scratch_bytes / (size_t)(n3 * sizeof(V)))));
  const int kb = (int)std::max<long>(1, std::min<long>(nb, fcap / njp));
  const int pcap = (int)std::max<long>(1, std::min<long>((std::max(nb, nphi) + 1) / 2, fcap));
  // workspace kept in the context (reused while large enough); phi(r) is
  // transformed once per pw_exx_set_phi
  DevBuf &psir = c->gsx_psir, &phir = c->gsx_phir, &acc = c->gsx_acc, &F = c->gsx_fields;
  int rc;
  const size_t phib = (size_t)nphi * n3 * sizeof(T);
  if (phir.bytes < phib) c->gsx_phi_ready = false;
  if ((rc = psir.alloc((size_t)nb * n3 * sizeof(T))) || (rc = phir.alloc(phib)) ||
      (rc = acc.alloc((size_t)nb * n3 * sizeof(T))) ||
      (rc = F.alloc((size_t)std::max<long>((long)kb * njp, pcap) * n3 * sizeof(V))))
    return rc;
  V* Z = (V*)F.p;
  const V* tw = (const V*)c->gs_exx_tw.p;
  if (!c->gsx_phi_ready) {
    if ((rc = gs_to_real<T>(c, (const T*)c->exx_phi.p, (int)c->ntot, nphi, (T)1, (T*)phir.p, Z, pcap, st))) return rc;
    c->gsx_phi_ready = true;
  }
  if ((rc = gs_to_real<T>(c, psi, ld, nb, (T)1, (T*)psir.p, Z, pcap, st))) return rc;
  PWB_CUDA(cudaMemsetAsync(acc.p, 0, (size_t)nb * n3 * sizeof(T), st));
  for (int k0 = 0; k0 < nb; k0 += kb) {
    const int kn = std::min(kb, nb - k0);
    const int nf = kn * njp;
    k_gsx_product<T><<<gs_blocks((long)nf * n3), 256, 0, st>>>((const T*)psir.p, (const T*)phir.p, k0, kn, njp, nphi,
                                                               n3, (T)(1.0 / (double)n3), Z);
    if ((rc = fft3_fields_n<T>(N, Z, nf, 2, (const T*)c->exx_kern.p, tw, st))) return rc;
    k_gsx_accumulate<T><<<gs_blocks((long)kn * n3), 256, 0, st>>>(Z, (const T*)phir.p, (const T*)c->exx_w.p, k0, kn,
                                                                  njp, nphi, n3, (T*)acc.p);
    c->launches += 7;
  }
  for (int b0 = 0; b0 < nb; b0 += 2 * pcap) {
    const int np = std::min(pcap, (nb - b0 + 1) / 2);
    k_gsx_pack<T><<<gs_blocks((long)np * n3), 256, 0, st>>>((const T*)acc.p, b0, nb, np, n3, Z);
    if ((rc = fft3_fields_n<T>(N, Z, np, 0, nullptr, tw, st))) return rc;
    k_gsx_gather<T><<<gs_blocks((long)np * c->gs_ns), 256, 0, st>>>(Z, np, n3, (const int2*)c->gs_full_idx.p,
                                                                    (int)c->gs_ns, b0, nb, out, ldo, accumulate);
    c->launches += 5;
  }
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

}  // namespace

// exchange kernel and its auxiliary (Fock set, full-grid sphere indices, twiddles) of a G-space context
int gs_exx_setup(pw_ctx* c, double frac, double mu, int divergence_type, double ecut) {
  const int N = c->nf[0];
  PWB_CHECK(c->nf[1] == N && c->nf[2] == N, PW_EUNSUPPORTED, "G-space exact exchange needs a cubic grid");
  const long n3 = (long)N * N * N;
  const double eps_div = 1e-8, alpha = 10.0 / (ecut * 2.0);
  std::vector<double> g2(n3);
  for (int z = 0; z < N; ++z)
    for (int y = 0; y < N; ++y)
      for (int x = 0; x < N; ++x) {
        const double m0 = x <= N / 2 ? x : x - N, m1 = y <= N / 2 ? y : y - N, m2 = z <= N / 2 ? z : z - N;
        const double a = 2 * M_PI / c->L[0] * m0, b = 2 * M_PI / c->L[1] * m1, d = 2 * M_PI / c->L[2] * m2;
        g2[x + (long)N * (y + (long)N * z)] = a * a + b * b + d * d;
      }
  // exxDiv over the grid points with eps < |G|^2 < 4 Ecut (hamiltonian.cpp:3479-3517, sphere-cut test)
  double div = 0.0;
  if (divergence_type == 1) {
    for (long i = 0; i < n3; ++i) {
      const double q = g2[i];
      if (q > eps_div && q < ecut * 4.0)
        div += mu > 0.0 ? std::exp(-alpha * q) / q * (1.0 - std::exp(-q / (4.0 * mu * mu))) : std::exp(-alpha * q) / q;
    }
    if (mu > 0.0) div += 1.0 / (4.0 * mu * mu);
    else div -= alpha;
    div *= 4.0 * M_PI;
    const double aa = mu > 0.0 ? 1.0 / std::sqrt(alpha * M_PI) - 1.0 / std::sqrt(M_PI * (alpha + 1.0 / (4.0 * mu * mu)))
                               : 1.0 / std::sqrt(alpha * M_PI);
    div -= c->vol * aa;
  }
  // kernel on the Fock set 1/2 |G|^2 < 4 Ecut, full grid
  std::vector<double> k(n3, 0.0);
  for (long i = 0; i < n3; ++i) {
    const double q = g2[i];
    if (0.5 * q >= 4.0 * ecut) continue;
    if (q > eps_div) k[i] = mu > 0.0 ? 4.0 * M_PI / q * (1.0 - std::exp(-q / (4.0 * mu * mu))) : 4.0 * M_PI / q;
    else k[i] = -div + (mu > 0.0 ? M_PI / (mu * mu) : 0.0);
  }
  int rc = upload_real(c, c->exx_kern, k.data(), n3);
  if (rc) return rc;
  // full-grid indices of G_s and -G_s
  const long ns = c->gs_ns;
  std::vector<int> gi(2 * ns);
  auto wrap = [N](int m) { return m < 0 ? m + N : m; };
  for (long s = 0; s < ns; ++s) {
    const int* m = &c->h_gs_m[3 * s];
    gi[2 * s] = wrap(m[0]) + N * (wrap(m[1]) + N * wrap(m[2]));
    gi[2 * s + 1] = wrap(-m[0]) + N * (wrap(-m[1]) + N * wrap(-m[2]));
  }
  if ((rc = c->gs_full_idx.alloc(gi.size() * 4))) return rc;
  PWB_CUDA(cudaMemcpy(c->gs_full_idx.p, gi.data(), gi.size() * 4, cudaMemcpyHostToDevice));
  std::vector<double> tw(2 * N);
  for (int m = 0; m < N; ++m) {
    tw[2 * m] = std::cos(2 * M_PI * m / N);
    tw[2 * m + 1] = -std::sin(2 * M_PI * m / N);
  }
  if ((rc = upload_real(c, c->gs_exx_tw, tw.data(), 2 * (size_t)N))) return rc;   // complex, context precision
  c->exx_frac = frac;
  c->exx_mu = mu;
  c->exx_div = div;
  return PW_OK;
}

// out (+)= V_x psi for nb sphere bands, in the context's precision
int gs_exx_apply(pw_ctx* c, const void* psi, int ld, int nb, void* out, int ldo, int accumulate, cudaStream_t st) {
  PWB_CHECK(c->gs_full_idx.p && c->exx_kern.p, PW_ENOTREADY, "exchange kernel not set (pw_exx_setup)");
  if (nb <= 0) return PW_OK;
  if (c->prec == PW_F64)
    return gs_exx_apply_t<double>(c, (const double*)psi, ld, nb, (double*)out, ldo, accumulate, st);
  return gs_exx_apply_t<float>(c, (const float*)psi, ld, nb, (float*)out, ldo, accumulate, st);
}

}  // namespace pwb
